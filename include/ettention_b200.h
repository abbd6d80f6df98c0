/*
 * ettention_b200 -- C ABI of the B200 (sm_100a) block-iterative reconstruction
 * path (SART / SIRT / general block size) of Ettention's libReconstruction.
 *
 * Plain pointers, sizes and status codes only: no C++ or CUDA types cross this
 * boundary, so the reference's C++ host code (or any FFI) can bind it.  All
 * device memory is owned by the library behind opaque handles; host buffers
 * are only read or written inside explicit upload / download calls.  Calls on
 * one context are stream-ordered on that context's CUDA stream and are not
 * thread-safe (one host thread per context, as the reference's single in-order
 * OpenCL queue, LR = ettention/libReconstruction/src):
 *   LR/gpu/opencl/CLKernel.cpp:177-179.
 *
 * Errors: every call returns ETCU_OK or an error code and never throws; the
 * message of the last failure on a context is read with etcu_last_error().
 * The validation messages repeat the reference's exception texts.
 *
 * Each entry point names the reference interface it replaces.
 */
#ifndef ETTENTION_B200_H
#define ETTENTION_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ETCU_ABI_VERSION 2

#if defined(__GNUC__)
#define ETCU_API __attribute__((visibility("default")))
#else
#define ETCU_API
#endif

typedef enum {
    ETCU_OK = 0,
    ETCU_ERR_INVALID_ARGUMENT = 1, /* reference: ettention::Exception from validation */
    ETCU_ERR_CUDA = 2,             /* reference: GPUException from CL_ASSERT */
    ETCU_ERR_OUT_OF_MEMORY = 3,
    ETCU_ERR_STATE = 4,            /* call order violated (e.g. outputs not set) */
    ETCU_ERR_UNSUPPORTED = 5,
    ETCU_ERR_NO_DEVICE = 6
} etcu_status;

/* Voxel storage of the volume the projectors read.
 * FLOAT32: one FP32 volume (reference default, optimization.internalVoxelRepresentationType=float).
 * HALF16:  one IEEE-half volume re-rounded after every view's update
 *          (reference "half", LR/model/volume/HalfFloatVolume.cpp:38-89).
 * F16_MASTER / BF16_MASTER: FP32 master volume updated by back projection plus
 *          a 16-bit shadow copy that forward projection reads; the shadow is
 *          re-quantised once per block. */
typedef enum {
    ETCU_VOXEL_FLOAT32 = 0,
    ETCU_VOXEL_HALF16 = 1,
    ETCU_VOXEL_F16_MASTER = 2,
    ETCU_VOXEL_BF16_MASTER = 3
} etcu_voxel_type;

/* Bilinear sampling of residual / ray-length images in back projection.
 * Q8:         software bilinear with weights rounded (half up) to 1/256 and FP32
 *             arithmetic: the GPU image path of the reference
 *             (LR/algorithm/projections/back/BackProjectionKernel.cpp:146-163,
 *             CL_FILTER_LINEAR), which its golden volumes pin.  Default.
 * EXACT:      FP32 weights, the reference's buffer path
 *             (ettention/libReconstruction/ocl_src/ImageHandler.hl:20-40).
 * HW_TEXTURE: this GPU's texture unit; its FP32 filtering deviates from the
 *             reference's by ~1e-3 relative, so it is opt-in. */
typedef enum { ETCU_SAMPLING_Q8 = 0, ETCU_SAMPLING_EXACT = 1, ETCU_SAMPLING_HW_TEXTURE = 2 } etcu_sampling;

/* Projection iteration order, optimization.projectionIteration
 * (LR/model/projectionset/factory/ProjectionIteratorFactory.cpp:11-22). */
typedef enum {
    ETCU_ORDER_IDENTITY = 0,
    ETCU_ORDER_RANDOM = 1,
    ETCU_ORDER_MAXANGLE = 2,
    ETCU_ORDER_BUCKETS = 3
} etcu_order;

/* Scanner geometry of one view: LR/model/geometry/ScannerGeometry.cpp:39-46
 * (source base, detector base, horizontal / vertical pitch, resolution) and
 * the Parallel / Perspective subclass. */
typedef struct {
    float source[3];
    float detector[3];
    float hpitch[3];
    float vpitch[3];
    uint32_t width, height;
    int32_t perspective;
} etcu_view;

/* Volume geometry: LR/setup/parameterset/VolumeParameterSet.cpp:7-71 and the
 * z-slab sub-volume split of LR/model/volume/VolumeProperties.cpp:74-98. */
typedef struct {
    uint32_t resolution[3];  /* x, y, z */
    float bbox_min[3];       /* world bounding box (origin -+ dimension/2) */
    float bbox_max[3];
    uint32_t subvolume_count; /* 0 or 1: one slab */
} etcu_volume_desc;

typedef struct etcu_context etcu_context;
typedef struct etcu_volume etcu_volume;
typedef struct etcu_recon etcu_recon;

/* ---------------------------------------------------------------- context */
/* Replaces the OpenCL context / queue of LR/gpu/opencl/CLAbstractionLayer.cpp:41-107. */
ETCU_API int etcu_abi_version(void);
ETCU_API etcu_status etcu_context_create(int device, etcu_context** out);
ETCU_API etcu_status etcu_context_destroy(etcu_context* ctx);
/* Message of the last failed call on ctx (or of the last failed context creation when ctx is NULL). */
ETCU_API const char* etcu_last_error(const etcu_context* ctx);
ETCU_API etcu_status etcu_synchronize(etcu_context* ctx);
/* Make the context issue its work on an existing CUDA stream (cudaStream_t passed as void*; NULL = own stream). */
ETCU_API etcu_status etcu_set_stream(etcu_context* ctx, void* cuda_stream);
/* The CUDA stream (cudaStream_t as void*) the context issues its work on, for
 * callers that record CUDA events around library calls. */
ETCU_API void* etcu_context_stream(const etcu_context* ctx);
/* Sum of device bytes the context currently holds. */
ETCU_API size_t etcu_device_bytes(const etcu_context* ctx);
/* Launch-shape autotuner (no counterpart in the reference): with mode 1, reconstructions,
 * batches and the warm-start network created on this context take their launch shapes
 * (resident blocks per multiprocessor, threads per block, pipeline stages) from a cache
 * file ($ETCU_TUNE_CACHE, else ~/.cache/ettention_b200/launch_shapes.txt) and time the
 * candidates with CUDA events on the real problem when the cache has no entry; results
 * do not depend on the choice.  Mode 0 (default; ETCU_AUTOTUNE=1 in the environment of
 * etcu_context_create sets 1) keeps the built-in shapes. */
ETCU_API etcu_status etcu_context_set_autotune(etcu_context* ctx, int mode);
/* The tuner's choices on this context so far, one "key choice [cached | candidate=ms ...]"
 * line each; *needed receives the length including the terminating zero. */
ETCU_API etcu_status etcu_context_tune_report(const etcu_context* ctx, char* out, size_t capacity, size_t* needed);

/* ---------------------------------------------------------------- geometry */
/* SingleAxisTiltRotator::createRotatedScannerGeometry
 * (LR/model/geometry/SingleAxisTiltRotator.cpp:42-78): rotate the base geometry
 * by -tilt about +y (about the x-pre-tilted y axis when xaxis_tilt_deg != 0). */
ETCU_API etcu_status etcu_view_rotate(const etcu_view* base, float tilt_deg, float xaxis_tilt_deg, etcu_view* out);
/* ParallelScannerGeometry::getProjectionMatrix (LR/model/geometry/ParallelScannerGeometry.cpp:49-62)
 * and PerspectiveScannerGeometry::getProjectionMatrix (.../PerspectiveScannerGeometry.cpp:47-50),
 * 16 floats, column-major (Matrix4x4 layout). */
ETCU_API etcu_status etcu_view_projection_matrix(const etcu_view* view, float out16[16]);
/* ParallelBeamsBackProjectionKernel::generateSamplingPatternForPerVoxelSampling
 * (LR/algorithm/projections/back/parallel/ParallelBeamsBackProjectionKernel.cpp:55-98):
 * samples x {offset x, y, z, chord}; samples must be a perfect square. */
ETCU_API etcu_status etcu_view_sample_pattern(const etcu_view* view, const float voxel_size[3], uint32_t samples,
                                     float* out4);
/* ParallelScannerGeometry::getTraversalLengthThroughBoundingBox (ParallelScannerGeometry.cpp:64-69). */
ETCU_API etcu_status etcu_view_traversal_length(const etcu_view* view, const float bbox_min[3], const float bbox_max[3],
                                       float* out);

/* ---------------------------------------------------------------- volume */
/* GPUMappedVolume over Float/HalfFloatVolume (LR/model/volume/GPUMappedVolume.cpp:9-41),
 * device-resident for its whole life.  init_value fills every voxel. */
ETCU_API etcu_status etcu_volume_create(etcu_context* ctx, const etcu_volume_desc* desc, etcu_voxel_type type,
                               float init_value, etcu_volume** out);
ETCU_API etcu_status etcu_volume_destroy(etcu_volume* vol);
/* Host float32 volume (x fastest, z slowest) <-> device; converts to / from the storage type. */
ETCU_API etcu_status etcu_volume_upload(etcu_volume* vol, const float* host);
ETCU_API etcu_status etcu_volume_download(etcu_volume* vol, float* host);
/* Stream-ordered device-to-device copies of the FP32 volume (FLOAT32 and *_MASTER types;
 * an upload refreshes the 16-bit shadow): the device-memory counterpart of the
 * reference's `volume.initFile` (BlockIterativeConfiguration.cpp:36-41), used to start a
 * reconstruction from a warm start without a host round trip. */
ETCU_API etcu_status etcu_volume_upload_device(etcu_volume* vol, const float* d_src);
ETCU_API etcu_status etcu_volume_download_device(etcu_volume* vol, float* d_dst);
/* Prior-knowledge mask (UCHAR_8 volume, value/255 weights; LR/algorithm/projections/
 * forward/ForwardProjectionKernel.cpp:21 USE_PRIOR_KNOWLEDGE_MASK).  NULL removes it. */
ETCU_API etcu_status etcu_volume_set_mask(etcu_volume* vol, const uint8_t* host_mask);
/* Device address of the volume (FP32 master, or the half volume) for zero-copy consumers. */
ETCU_API void* etcu_volume_device_ptr(etcu_volume* vol);

/* ---------------------------------------------------------------- operators */
/* ForwardProjectionOperator::SetOutput + Execute(subVolume)
 * (LR/algorithm/projections/forward/ForwardProjectionOperator.cpp:31-55 over
 * ParallelBeamsForwardProjection.cl / PerspectiveBeamsForwardProjection.cl):
 * ADDS the sub-volume's line integrals of volume and mask into the device
 * images d_virtual and d_traversal (width x height floats each, row-major). */
ETCU_API etcu_status etcu_forward_project(etcu_volume* vol, const etcu_view* view, uint32_t subvolume, uint32_t samples,
                                 float* d_virtual, float* d_traversal);
/* BackProjectionOperator::setInput(residual, traversal, blockSize) + execute(subVolume)
 * (LR/algorithm/projections/back/BackProjectionOperator.cpp:43-98): voxel-driven
 * update of sub-volume `subvolume` with lambda / block_size (BackProjectionKernel.cpp:94).
 * samples: parallel = per-voxel detector-plane samples (perfect square);
 *          perspective = samples per dimension (0: derived from resolutions).
 * subvolume == ETCU_ALL_SUBVOLUMES runs every slab. */
#define ETCU_ALL_SUBVOLUMES 0xffffffffu
ETCU_API etcu_status etcu_back_project(etcu_volume* vol, const etcu_view* view, uint32_t subvolume, uint32_t samples,
                              float lambda, uint32_t block_size, const float* d_residual,
                              const float* d_traversal, etcu_sampling sampling);
/* Perspective back-projection intensity clamps (PerspectiveBeamsBackProjectionKernel.cpp:175-188). */
ETCU_API etcu_status etcu_volume_set_intensity_clamp(etcu_volume* vol, int use_min, float vmin, int use_max, float vmax);
/* CompareKernel: residual = real - virtual (ocl_src/Compare.cl:1-9), device images of n floats. */
ETCU_API etcu_status etcu_compare(etcu_context* ctx, const float* d_real, const float* d_virtual, float* d_residual,
                         size_t n);
/* VirtualProjectionKernel (ocl_src/VirtualProjection.cl:3-10): long-object compensation in place. */
ETCU_API etcu_status etcu_long_object_compensation(etcu_context* ctx, float* d_virtual, float* d_traversal,
                                          float constant_length, size_t n);
/* ComputeRayLengthKernel (ocl_src/ComputeRayLength.cl:21-34): parallel-ray chord through the complete volume. */
ETCU_API etcu_status etcu_compute_ray_length(etcu_volume* vol, const etcu_view* view, float* d_out);

/* ---------------------------------------------------------------- reconstruction */
/* BlockIterativeReconstructionOperator (LR/algorithm/reconstruction/blockiterative/
 * BlockIterativeReconstructionOperator.cpp:56-185) with AlgorithmParameterSet /
 * OptimizationParameterSet semantics (LR/setup/parameterset/AlgorithmParameterSet.cpp:8-53).
 * block_size: 1 = SART, ETCU_BLOCK_ALL = SIRT, else algorithm.blockSize. */
#define ETCU_BLOCK_ALL 0xffffffffu
/* Storage of the measured projections on the device (HalfFloatSupport.hl:6-14 applies the
 * reference's half storage to volumes; the same 16-bit storage is offered for the tilt
 * series): FP32 as given, or rounded to nearest FP16 / BF16 once when the reconstruction
 * is created and widened exactly where the residual is formed. */
typedef enum { ETCU_PROJ_F32 = 0, ETCU_PROJ_F16 = 1, ETCU_PROJ_BF16 = 2 } etcu_projection_storage;
typedef struct {
    float lambda;                 /* algorithm.lambda */
    uint32_t block_size;          /* algorithm.blockSize (1 SART, ETCU_BLOCK_ALL SIRT) */
    uint32_t fp_samples;          /* forwardProjection.samples (0 -> 1) */
    uint32_t bp_samples;          /* backProjection.samples */
    int32_t use_long_object_compensation; /* algorithm.useLongObjectCompensation */
    etcu_order order;             /* optimization.projectionIteration */
    etcu_sampling sampling;       /* residual sampling of the back projector */
    const uint32_t* skip;         /* input.skipProjections (may be NULL) */
    uint32_t skip_count;
    int32_t use_graph;            /* capture each iteration in a CUDA graph */
    etcu_projection_storage projection_storage; /* element type the measured projections are kept in */
} etcu_recon_params;

/* Uploads the tilt series (n_views x height x width floats, host memory) once
 * and prepares per-view geometry, textures and the per-iteration graph. */
ETCU_API etcu_status etcu_recon_create(etcu_volume* vol, const etcu_view* views, uint32_t n_views,
                              const float* host_projections, const etcu_recon_params* params, etcu_recon** out);
/* Same, with the tilt series already in device memory (n_views x height x width floats). */
ETCU_API etcu_status etcu_recon_create_device(etcu_volume* vol, const etcu_view* views, uint32_t n_views,
                                     const float* d_projections, const etcu_recon_params* params,
                                     etcu_recon** out);
ETCU_API etcu_status etcu_recon_destroy(etcu_recon* rec);
/* runNiterations (BlockIterativeReconstructionOperator.cpp:66-80). */
ETCU_API etcu_status etcu_recon_run(etcu_recon* rec, uint32_t iterations);
/* Sum over the last iteration's views of ||b - Ax||^2 as each view saw it before its
 * update (FP64 accumulation). */
ETCU_API etcu_status etcu_recon_last_residual_sq(etcu_recon* rec, double* out);
/* ||b - Ax||^2 over all views for the current volume (forward projection only, FP64). */
ETCU_API etcu_status etcu_recon_data_residual_sq(etcu_recon* rec, double* out);
/* Permutation of view indices the reconstruction iterates in. */
ETCU_API etcu_status etcu_recon_view_order(const etcu_recon* rec, uint32_t* out, uint32_t capacity, uint32_t* count);
/* Runs one real iteration launch by launch, with CUDA events around every forward
 * and back projection; returns their summed device times (ms) and launch counts.
 * (Per-kernel timing of the hot path; the reference's PerformanceReport of
 * LR/gpu/opencl/CLAbstractionLayer.cpp:295-324.) */
ETCU_API etcu_status etcu_recon_profile_iteration(etcu_recon* rec, float* fp_ms, float* bp_ms, uint32_t* fp_launches,
                                                  uint32_t* bp_launches);
/* One iteration as etcu_recon_run issues it, each step timed with CUDA events on the
 * context's stream: kinds[i] = 0 forward projection, 1 back projection, 2 fused SART
 * step (back projection of one view and forward projection of the next in one pass);
 * launches[i] = kernel launches of the step.  *count = the number of steps; with NULL
 * arrays only the count is returned. */
ETCU_API etcu_status etcu_recon_profile_steps(etcu_recon* rec, float* ms, uint32_t* kinds, uint32_t* launches,
                                              uint32_t capacity, uint32_t* count);
/* Kernel launches one iteration issues (graph nodes when captured). */
ETCU_API uint32_t etcu_recon_launches_per_iteration(const etcu_recon* rec);

/* One volume over several GPUs by z-slabs (one process per GPU; the reference's
 * sub-volume split, LR/model/volume/VolumeProperties.cpp:74-98, with one slab per rank):
 * `rec` reconstructs this rank's slab (a volume of the slab's resolution and bounding
 * box).  Per block b of etcu_recon_block_count():
 *   etcu_recon_slab_forward(rec, b, d_partial)   this slab's line integrals and lengths of
 *       the block's views, added into zeroed d_partial: count x 2 x height x width floats
 *       ((virtual, traversal) per view; the forward projections' += of
 *       ParallelBeamsForwardProjection.cl:56-57 across slabs)
 *   all-reduce (sum) of d_partial over the ranks, on the context's stream
 *   etcu_recon_slab_backward(rec, b, d_complete) residual b - Ax (long-object compensation
 *       over the complete volume, etcu_recon_set_complete_bbox) and the back projection of
 *       the block on this slab with lambda / block size.
 * Stream-ordered, no host synchronisation; the residual sum of the sweep is
 * etcu_recon_last_residual_sq (reset by block 0's forward call). */
ETCU_API etcu_status etcu_recon_block_count(const etcu_recon* rec, uint32_t* blocks, uint32_t* block_size);
ETCU_API etcu_status etcu_recon_set_complete_bbox(etcu_recon* rec, const float bbox_min[3], const float bbox_max[3]);
ETCU_API etcu_status etcu_recon_slab_forward(etcu_recon* rec, uint32_t block, float* d_partial);
ETCU_API etcu_status etcu_recon_slab_backward(etcu_recon* rec, uint32_t block, const float* d_complete);
/* etcu_recon_slab_backward(block) then etcu_recon_slab_forward(block + 1, d_next) in one
 * call (block + 1 < blocks; d_next a second count x 2 x height x width buffer).  For SART
 * on the fused path this is one fused step: the back projection of view p and the forward
 * projection of view p + 1 in one pass over the slab. */
ETCU_API etcu_status etcu_recon_slab_step(etcu_recon* rec, uint32_t block, const float* d_complete, float* d_next);

/* One-call host-buffer reconstruction: upload projections and initial volume,
 * run `iterations`, download the result (the path a frontend's "ettention --config" run takes). */
ETCU_API etcu_status etcu_reconstruct(etcu_context* ctx, const etcu_volume_desc* desc, etcu_voxel_type type,
                             const etcu_view* views, uint32_t n_views, const float* host_projections,
                             const etcu_recon_params* params, uint32_t iterations, float* host_volume_inout);

/* ---------------------------------------------------------------- files */
/* Host-side formats of the reference's front door; context-free (errors via
 * etcu_last_error(NULL)).  MRC stacks: LR/io/datasource/MRCStack.cpp:136-250 (modes
 * 0 = uint8, 1 = int16, 2 = float32, 6 = uint16; the extended header is skipped). */
typedef struct {
    uint32_t nx, ny, nz;     /* columns, rows, sections (projections of a stack) */
    int32_t mode;
    float dmin, dmax, dmean; /* as stored in the header */
    uint32_t extended_bytes;
} etcu_mrc_info;
ETCU_API etcu_status etcu_mrc_read_info(const char* path, etcu_mrc_info* out);
/* Every section as float32 (nx * ny * nz values, x fastest).  logarithmize != 0 applies
 * MRCStack's transform log(M / (raw - m)) over the stack's data range: M = max - min + 1,
 * m = min - 1 for modes 1 and 2; M = max + 1, m = -1 for modes 0 and 6
 * (MRCStack.cpp:161-172, 226-236; input.logarithmize). */
ETCU_API etcu_status etcu_mrc_read_stack(const char* path, int logarithmize, float* out, size_t capacity);
/* Tilt-angle file (ImageStackDatasource.cpp:49-79): every whitespace-separated float;
 * *count = the number in the file, at most capacity of them stored in out. */
ETCU_API etcu_status etcu_read_tilt_angles(const char* path, float* out, uint32_t capacity, uint32_t* count);
/* Coordinate order of a written volume (output.options.orientation,
 * LR/setup/parameterset/IOEnumerations.cpp:79-126): XZY (the reference's default)
 * stores y as the file's sections and z as its rows. */
typedef enum { ETCU_AXES_XYZ = 0, ETCU_AXES_XZY = 1 } etcu_orientation;
/* VolumeFileFormatWriter / MRCWriter with output.options.voxelType float32: mode-2 MRC
 * with min / max / mean in the header (VolumeStatistics::compute); volume is x fastest,
 * then y, then z. */
ETCU_API etcu_status etcu_mrc_write_volume(const char* path, const float* volume, const uint32_t resolution[3],
                                           etcu_orientation orientation);
/* output.options.voxelType (LR/setup/parameterset/IOEnumerations.h:8-13, the MRC mode). */
typedef enum {
    ETCU_OUT_UNSIGNED_8 = 0,
    ETCU_OUT_SIGNED_16 = 1,
    ETCU_OUT_FLOAT_32 = 2,
    ETCU_OUT_UNSIGNED_16 = 6
} etcu_output_voxel_type;
/* VolumeFileFormatWriter::write with output.options.voxelType and output.options.invert
 * (LR/io/serializer/VolumeFileFormatWriter.cpp:11-140, LinearRangeTransformation.cpp):
 * integer types map [min, max] of the volume linearly onto the type's range (reversed
 * with invert) and are C-cast; float32 is written as is (with invert the header's
 * min / max / mean are mapped onto [max, min], the data are not). */
ETCU_API etcu_status etcu_mrc_write_volume_typed(const char* path, const float* volume, const uint32_t resolution[3],
                                                 etcu_orientation orientation, etcu_output_voxel_type voxel_type,
                                                 int invert);

/* TIFF images (LR/io/deserializer/ImageDeserializer.cpp:10-62, replacing FreeImage):
 * grey, one sample per pixel, 8 / 16-bit unsigned or 32-bit float samples, converted
 * to float as the reference does (8-bit / 255, 16-bit / 65535, float as is); strips
 * or tiles; no compression, LZW, Deflate or PackBits; predictors 1, 2 and 3.  Image
 * row y is the y-th row of the file.  Multi-page files are image stacks. */
typedef struct {
    uint32_t width, height;
    uint32_t pages;            /* pages in the file */
    uint32_t bits_per_sample;  /* of the page asked for */
    uint32_t sample_format;    /* 1 unsigned, 2 signed, 3 float */
    uint32_t compression;      /* 1 none, 5 LZW, 8 / 32946 Deflate, 32773 PackBits */
} etcu_image_info;
ETCU_API etcu_status etcu_tiff_read_info(const char* path, uint32_t page, etcu_image_info* out);
/* One page as width * height floats (x fastest). */
ETCU_API etcu_status etcu_tiff_read(const char* path, uint32_t page, float* out, size_t capacity);
/* ImageSerializer::writeImage(..., TIFF_GRAY_32): one page of 32-bit float grey. */
ETCU_API etcu_status etcu_tiff_write(const char* path, const float* image, uint32_t width, uint32_t height);

/* A directory of projection images described by its metadata.xml
 * (LR/io/datasource/ImageStackDirectoryDatasource.cpp): <geometry> holds the base
 * parallel geometry (sourcePosition, detectorPosition, horizontalPitch,
 * verticalPitch); every <projection> an <image filename=.../>, a <tiltAngle
 * value=.../> and optionally <logscale/> (pixels are then exp()'d); a
 * <projectionstack> names a multi-page image whose pages share one tilt angle.
 * Projections are numbered by tilt angle in order of first appearance, repeated
 * angles after one another (:200-240); the detector size is the first image's. */
typedef struct etcu_image_stack etcu_image_stack;
typedef struct {
    uint32_t count;   /* projections */
    uint32_t width, height;
    etcu_view base;   /* untilted geometry; rotate with etcu_view_rotate */
} etcu_image_stack_info;
ETCU_API etcu_status etcu_image_stack_open(const char* directory, etcu_image_stack** out);
ETCU_API void etcu_image_stack_destroy(etcu_image_stack* stack);
ETCU_API etcu_status etcu_image_stack_info_get(const etcu_image_stack* stack, etcu_image_stack_info* out);
/* Tilt angle of every projection (degrees), count of them. */
ETCU_API etcu_status etcu_image_stack_tilt_angles(const etcu_image_stack* stack, float* out, uint32_t capacity);
/* Projections first .. first + count - 1 as count * height * width floats. */
ETCU_API etcu_status etcu_image_stack_load(const etcu_image_stack* stack, uint32_t first, uint32_t count, float* out,
                                           size_t capacity);
/* ImageStackDirectoryDatasource::writeMetaDataFile (:121-175): the base geometry,
 * volume dimensions and one <projection> per (file name, tilt angle). */
ETCU_API etcu_status etcu_image_stack_write_metadata(const char* path, const float* tilt_angles,
                                                     const char* const* filenames, uint32_t count,
                                                     const etcu_view* base, const uint32_t volume_resolution[3]);

/* XML parameter files (LR/setup/parametersource/XMLParameterSource.cpp): every element
 * with a value attribute becomes "path.to.element<TAB>value<NEWLINE>" (the first
 * element of a path wins, as a property-tree lookup does).  *needed = bytes of the
 * text including its terminating NUL; out (capacity bytes) receives it when it fits.
 * Relative paths in values are relative to the file's directory
 * (XMLParameterSource.cpp:24-35); resolving them is the caller's. */
ETCU_API etcu_status etcu_xml_config_read(const char* path, char* out, size_t capacity, size_t* needed);

/* ---------------------------------------------------------------- weighted back projection */
/* WBP plugin (plugins/WBPPlugin/src/reconstruction/WBP.cpp:22-86): each projection is
 * filtered with the RamLak kernel of 128 taps (ocl_src/GenerateRamLakKernel.cl) as
 * ConvolutionFourierSpaceImplementation does it (power-of-two grid, mirrored padding,
 * origin-moved kernel, circular convolution, centred crop; for an even grid height the
 * filtered row y is taken from padded row y + 1), its ray lengths through the complete
 * volume are computed (ComputeRayLength.cl), and every view is back projected into vol
 * with lambda / n_views, in view order.  vol is not cleared first.  Parallel views only.
 * host_projections: n_views x height x width floats. */
ETCU_API etcu_status etcu_wbp(etcu_volume* vol, const etcu_view* views, uint32_t n_views,
                              const float* host_projections, float lambda, uint32_t bp_samples,
                              etcu_sampling sampling);
/* The RamLak filtering of one device image (height x width floats) with filter_width taps. */
ETCU_API etcu_status etcu_wbp_filter(etcu_context* ctx, const float* d_in, float* d_out, uint32_t width,
                                     uint32_t height, uint32_t filter_width);

/* ---------------------------------------------------------------- blob basis functions */
/* Kaiser-Bessel blobs (model/blobs/BlobParameters.cpp; createDefault = 2.0, 2, 3.6) as the
 * basis of perspective projection (ocl_src/BlobRaytracer.hl,
 * PerspectiveBeams{Forward,Back}ProjectionWithBlobs.cl) and their voxelisation
 * (algorithm/blobs/BlobVoxelizerOperator.cpp).  The kernels take the projection matrix and
 * its inverse as the reference forms them: Matrix4x4 arithmetic in float with a cofactor
 * inverse. */
typedef struct {
    float support_radius;  /* a, in voxels */
    uint32_t degree;       /* m */
    float density_falloff; /* alpha */
} etcu_blob_params;
/* BlobRayIntegrationSampler: the blob's line integral at count distances 0 .. a. */
ETCU_API etcu_status etcu_blob_ray_integration_samples(const etcu_blob_params* params, uint32_t count, float* out);
/* BlobVoxelizationKernelValues: the blob integrated over each voxel of the
 * (2 ceil(a) + 1)^3 neighbourhood, [dz][dy][dx]; *size_per_dim = 2 ceil(a) + 1 (out may be
 * NULL to ask for it). */
ETCU_API etcu_status etcu_blob_voxelization_kernel(const etcu_blob_params* params, float* out, uint32_t capacity,
                                                  uint32_t* size_per_dim);
/* PerspectiveBeamsForwardProjectionWithBlobsKernel: ADDS the blob line integrals of the
 * coefficients in vol (FP32) and their weights into device images (height x width floats);
 * table of sample_count entries (the reference's callers use 128). */
ETCU_API etcu_status etcu_forward_project_blobs(etcu_volume* vol, const etcu_view* view, uint32_t subvolume,
                                               const etcu_blob_params* params, uint32_t sample_count,
                                               float* d_projection, float* d_traversal);
/* PerspectiveBeamsBackProjectionWithBlobsKernel: each blob takes lambda / block_size times the
 * weighted mean of residual / ray length over the pixels whose rays pass within its radius
 * (pixels with a nonzero residual and a ray length above 1). */
ETCU_API etcu_status etcu_back_project_blobs(etcu_volume* vol, const etcu_view* view, uint32_t subvolume,
                                            const etcu_blob_params* params, float lambda, uint32_t block_size,
                                            const float* d_residual, const float* d_raylength);
/* Block-iterative reconstruction with blob basis functions (algorithm.basisFunctions =
 * blobs; BlockIterativeReconstructionOperator.cpp:84-160 with the blob kernels that
 * DefaultForwardProjectionCreator.cpp:53-60 and DefaultBackProjectionCreator.cpp:51-59
 * pick for perspective beams, tables of 256 samples).  Same parameters as etcu_recon_create
 * (lambda, block_size, order, skip; long-object compensation is rejected as for every
 * perspective series); the coefficients live in vol (FP32).  Voxelise them with
 * etcu_blob_voxelize after etcu_blob_recon_run when output.options.enableVoxelization is set. */
typedef struct etcu_blob_recon etcu_blob_recon;
ETCU_API etcu_status etcu_blob_recon_create(etcu_volume* vol, const etcu_view* views, uint32_t n_views,
                                           const float* host_projections, const etcu_recon_params* params,
                                           const etcu_blob_params* blob, etcu_blob_recon** out);
ETCU_API etcu_status etcu_blob_recon_create_device(etcu_volume* vol, const etcu_view* views, uint32_t n_views,
                                                  const float* d_projections, const etcu_recon_params* params,
                                                  const etcu_blob_params* blob, etcu_blob_recon** out);
ETCU_API etcu_status etcu_blob_recon_run(etcu_blob_recon* rec, uint32_t iterations);
/* sum of the squared residuals of the last iteration (each view against the volume of its block) */
ETCU_API etcu_status etcu_blob_recon_last_residual_sq(const etcu_blob_recon* rec, double* out);
ETCU_API etcu_status etcu_blob_recon_view_order(const etcu_blob_recon* rec, uint32_t* out, uint32_t capacity,
                                               uint32_t* count);
ETCU_API uint32_t etcu_blob_recon_launches_per_iteration(const etcu_blob_recon* rec);
/* Runs one iteration as etcu_blob_recon_run does with CUDA events around every launch:
 * ms_by_kind[3] / n_by_kind[3] = total device milliseconds and launches of the forward
 * projections, the residual launches and the back projections. */
ETCU_API etcu_status etcu_blob_recon_profile_iteration(etcu_blob_recon* rec, float* ms_by_kind, uint32_t* n_by_kind);
ETCU_API etcu_status etcu_blob_recon_destroy(etcu_blob_recon* rec);
/* BlobVoxelizerOperator::voxelize: voxels = the blob coefficients convolved with the
 * voxelisation kernel (zero outside the volume); both FP32, same resolution. */
ETCU_API etcu_status etcu_blob_voxelize(etcu_volume* blobs, etcu_volume* voxels, const etcu_blob_params* params);

/* ---------------------------------------------------------------- batched series */
/* Many independent tilt series of uneven sizes reconstructed together.  When every
 * series can run the fused SART step (Q8 sampling, one sample each way, even rows of at
 * most 1024 voxels), each iteration of all series is one persistent launch; otherwise
 * every SART step runs one forward-projection launch and one back-projection launch
 * over all series (series without a view at that step sit it out), and each iteration
 * is one CUDA graph.  etcu_batch_run reports ETCU_ERR_CUDA if a step of the persistent
 * launch waited longer than its limit (1 s) for neighbouring rows.  Per series the result is the block-iterative reconstruction of
 * etcu_recon_* with block size 1 (BlockIterativeReconstructionOperator.cpp:92-142).
 * No counterpart in the reference, which reconstructs one series per run.
 * Supported: SART (block_size 1), one back-projection sample, parallel views whose
 * detector row depends on y only (single-axis tilt about y), FP32 volumes with one
 * sub-volume and no mask, ETCU_SAMPLING_Q8 or _EXACT; anything else returns
 * ETCU_ERR_UNSUPPORTED.  All volumes belong to ctx. */
typedef struct {
    etcu_volume* volume;
    const etcu_view* views;
    uint32_t n_views;
    const float* host_projections; /* n_views x height x width floats */
} etcu_batch_series;
typedef struct etcu_batch etcu_batch;

ETCU_API etcu_status etcu_batch_create(etcu_context* ctx, const etcu_batch_series* series, uint32_t n_series,
                                       const etcu_recon_params* params, etcu_batch** out);
ETCU_API etcu_status etcu_batch_destroy(etcu_batch* batch);
ETCU_API etcu_status etcu_batch_run(etcu_batch* batch, uint32_t iterations);
/* Per series (n_series doubles): sum over the last iteration's views of ||b - Ax||^2
 * as each view saw it before its update (FP64). */
ETCU_API etcu_status etcu_batch_last_residual_sq(etcu_batch* batch, double* out);
/* Kernel launches one iteration issues. */
ETCU_API uint32_t etcu_batch_launches_per_iteration(const etcu_batch* batch);

/* One SART update of one view (forward projection, residual b - Ax, back projection
 * with block size 1) that allocates no device memory, for callers that cannot
 * allocate: hosts whose device memory is reserved up front by their own pool
 * allocator, or processing loops in which allocation after start-up is not
 * allowed.  The caller passes the FP32 volume (device pointer, layout as
 * etcu_volume, one sub-volume), the measured projection of this view (device
 * pointer, height x width floats) and the stream to run on (NULL: the legacy
 * default stream).  The (residual, ray length) image lives in a static device
 * array of ETCU_NOALLOC_SCRATCH_TEXELS float2 (8 MiB) that every GPU loading
 * the library holds until the process exits.  The image carries a two-texel zero
 * border, so a detector fits when (width + 4) x (height + 4) <=
 * ETCU_NOALLOC_SCRATCH_TEXELS and width x height <= ETCU_NOALLOC_MAX_PIXELS: every
 * detector of up to 1024 x 1024 pixels fits, and so does, e.g., 2048 x 508; larger
 * ones (also 4096 x 256, which needs 4100 x 260 texels) are rejected.  The first
 * call on a device (and the first after that device's context was replaced, e.g.
 * by cudaDeviceReset) looks up that array's device address, so make the first
 * call before any stream capture.  All calls share the array and keep
 * the last call's contents: calls that overlap on the GPU (other streams or
 * threads on the same device) race and must be serialised by the caller.
 * residual_sq (optional, host) receives sum (b - Ax)^2 over the view, which
 * synchronises the stream.  Sampling is ETCU_SAMPLING_Q8.
 * No counterpart in the reference. */
#define ETCU_NOALLOC_MAX_PIXELS (1024u * 1024u)
#define ETCU_NOALLOC_SCRATCH_TEXELS (ETCU_NOALLOC_MAX_PIXELS + 8208u)
ETCU_API etcu_status etcu_sart_view_update_noalloc(const etcu_volume_desc* desc, float* d_volume,
                                                   const float* d_projection, const etcu_view* view,
                                                   uint32_t fp_samples, uint32_t bp_samples, float lambda,
                                                   void* cuda_stream, double* residual_sq);

/* ---------------------------------------------------------------- learned warm start
 * A 3-level 3-D convolutional encoder-decoder (3x3x3 convolutions, 16 / 32 / 64
 * channels, BF16 weights and activations, FP32 accumulation on the tensor cores) that
 * maps a few-iteration SART volume to a warm start from which plain SART continues,
 * trained on pairs the method itself generates.  The reference has no learned part; its
 * result enters the reference's loop where `volume.initFile` does
 * (LR/algorithm/reconstruction/blockiterative/BlockIterativeConfiguration.cpp:36-41).
 * Volumes are FP32 [batch][z][y][x] device arrays with x, y, z multiples of 4; every
 * call is ordered on the context's stream.  Parameters are one FP32 vector: per layer
 * W[27][cout][cin] (tap dz*9 + dy*3 + dx reads voxel (x+dx-1, y+dy-1, z+dz-1)), then
 * b[cout]; `scale` divides the input volume (and multiplies the residual output). */
typedef struct etcu_warmstart etcu_warmstart;
/* Number of FP32 parameters of the network. */
ETCU_API uint32_t etcu_warmstart_param_count(void);
/* Layer l (0..10): out[0..5] = real input channels of source 0, channels of source 1
 * (the skip connection, or 0), output channels, resolution level (1..3), offset of W and
 * offset of b in the parameter vector. */
ETCU_API etcu_status etcu_warmstart_layer_info(uint32_t layer, uint32_t out[6]);
ETCU_API etcu_status etcu_warmstart_create(etcu_context* ctx, const uint32_t resolution[3], uint32_t max_batch,
                                           etcu_warmstart** out);
ETCU_API etcu_status etcu_warmstart_destroy(etcu_warmstart* ws);
/* Replaces the parameters (host FP32, etcu_warmstart_param_count() values) and the input
 * scale; resets the optimiser state. */
ETCU_API etcu_status etcu_warmstart_set_params(etcu_warmstart* ws, const float* host_params, float scale);
ETCU_API etcu_status etcu_warmstart_get_params(etcu_warmstart* ws, float* host_params, float* scale);
/* d_out = d_in + scale * net(d_in / scale) for `batch` volumes (device pointers). */
ETCU_API etcu_status etcu_warmstart_infer(etcu_warmstart* ws, const float* d_in, float* d_out, uint32_t batch);
/* One Adam step (lr; beta 0.9 / 0.999, eps 1e-8) on the mean squared error between the
 * network's output and d_target, in units of the scale.  loss (optional, host) receives
 * the loss before the step and synchronises the stream. */
ETCU_API etcu_status etcu_warmstart_train_step(etcu_warmstart* ws, const float* d_in, const float* d_target,
                                               uint32_t batch, float lr, double* loss);
/* The loss and its gradient with respect to every parameter (host FP32 vector), without
 * an update; synchronises the stream. */
ETCU_API etcu_status etcu_warmstart_gradients(etcu_warmstart* ws, const float* d_in, const float* d_target,
                                              uint32_t batch, float* host_grads, double* loss);
/* Synchronises and reports a convolution that gave up waiting for its operands. */
ETCU_API etcu_status etcu_warmstart_check(etcu_warmstart* ws);

/* Projection orderings on their own (LR/model/projectionset/ProjectionSet*.cpp), for callers
 * that keep their own driver loop. */
ETCU_API etcu_status etcu_projection_order(etcu_order order, uint32_t n, const uint32_t* skip, uint32_t skip_count,
                                  uint32_t* out, uint32_t* count);

#ifdef __cplusplus
}
#endif
#endif /* ETTENTION_B200_H */
