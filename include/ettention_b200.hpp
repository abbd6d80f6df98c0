/*
 * C++ operator surface of the B200 block-iterative reconstruction path, over the
 * C ABI of ettention_b200.h (header-only; link libettention_b200.so).
 *
 * It keeps the class and method names of the reference's libReconstruction
 * operators (paths relative to ettention/libReconstruction/src):
 *   Framework                              LR/framework/Framework.cpp (owns the GPU context)
 *   ScannerGeometry                        LR/model/geometry/ScannerGeometry.cpp:39-46,
 *                                          ParallelScannerGeometry.cpp:44-69,
 *                                          SingleAxisTiltRotator.cpp:42-78, MRCStack.cpp:250-261
 *   GPUMappedVolume                        LR/model/volume/GPUMappedVolume.cpp:9-41,
 *                                          VolumeProperties.cpp:21-98 (z-slab sub-volumes)
 *   ForwardProjectionOperator              LR/algorithm/projections/forward/ForwardProjectionOperator.cpp:11-55
 *   BackProjectionOperator                 LR/algorithm/projections/back/BackProjectionOperator.cpp:13-98
 *   AlgebraicParameterSet::fromConfig      LR/setup/parameterset/AlgorithmParameterSet.cpp:8-53,
 *                                          OptimizationParameterSet, VolumeParameterSet, HardwareParameterSet
 *   BlockIterativeReconstructionOperator   LR/algorithm/reconstruction/blockiterative/
 *                                          BlockIterativeReconstructionOperator.cpp:56-185
 *   MRCStack, writeMrcVolume               LR/io/datasource/MRCStack.cpp, LR/io/serializer/MRCWriter.cpp
 *   ImageStackDirectoryDatasource,         LR/io/datasource/ImageStackDirectoryDatasource.cpp,
 *   readTiff, writeTiff                    LR/io/deserializer/ImageDeserializer.cpp, ImageSerializer.cpp
 *   XMLParameterSource                     LR/setup/parametersource/XMLParameterSource.cpp
 *   WBP                                    plugins/WBPPlugin/src/reconstruction/WBP.cpp
 *   BlobParameters, BlobVoxelizerOperator  LR/model/blobs/BlobParameters.cpp, LR/algorithm/blobs
 *                                          (algorithm.basisFunctions = blobs, perspective beams)
 *   BatchReconstructionOperator            many series per launch (no counterpart in the reference)
 * Errors: every non-OK status of the ABI is rethrown as ettention::b200::Exception
 * (validation) or GPUException (device errors), with the library's message, as
 * the reference throws ettention::Exception / GPUException.
 *
 * Device images (SetOutput / setInput) are device pointers of width * height
 * floats; the operators are stream-ordered on the Framework's stream and
 * synchronise after each call, as the reference waits after every launch.
 */
#pragma once

#include <array>
#include <cstdint>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "ettention_b200.h"

namespace ettention {
namespace b200 {

class Exception : public std::runtime_error {
public:
    Exception(etcu_status status, const std::string& what) : std::runtime_error(what), status_(status) {}
    etcu_status status() const { return status_; }

private:
    etcu_status status_;
};

class GPUException : public Exception {
public:
    using Exception::Exception;
};

inline void check(etcu_status status, const etcu_context* ctx) {
    if (status == ETCU_OK) return;
    const char* msg = etcu_last_error(ctx);
    std::string text = msg && *msg ? msg : "ettention_b200 status " + std::to_string((int)status);
    if (status == ETCU_ERR_CUDA || status == ETCU_ERR_NO_DEVICE || status == ETCU_ERR_OUT_OF_MEMORY)
        throw GPUException(status, text);
    throw Exception(status, text);
}

// The reference's Framework owns the OpenCL abstraction layer; here it owns the
// CUDA context and stream of one device.
class Framework {
public:
    explicit Framework(int device = 0) { check(etcu_context_create(device, &ctx_), nullptr); }
    ~Framework() { etcu_context_destroy(ctx_); }
    Framework(const Framework&) = delete;
    Framework& operator=(const Framework&) = delete;
    etcu_context* handle() const { return ctx_; }
    void synchronize() { check(etcu_synchronize(ctx_), ctx_); }
    // Work is ordered on this CUDA stream (nullptr: the context's own stream).
    void setStream(void* cuda_stream) { check(etcu_set_stream(ctx_, cuda_stream), ctx_); }

private:
    etcu_context* ctx_ = nullptr;
};

class ScannerGeometry {
public:
    ScannerGeometry() = default;
    explicit ScannerGeometry(const etcu_view& v) : view_(v) {}

    // MRCStack.cpp:250-261: parallel base geometry of an nx x ny tilt series.
    static ScannerGeometry mrcBase(uint32_t nx, uint32_t ny) {
        etcu_view v{};
        const float fx = (float)nx, fy = (float)ny;
        const float src[3] = {-0.5f * fx, -0.5f * fy, fx}, det[3] = {-0.5f * fx, -0.5f * fy, -fx};
        for (int i = 0; i < 3; ++i) {
            v.source[i] = src[i];
            v.detector[i] = det[i];
            v.hpitch[i] = i == 0 ? 1.f : 0.f;
            v.vpitch[i] = i == 1 ? 1.f : 0.f;
        }
        v.width = nx;
        v.height = ny;
        v.perspective = 0;
        return ScannerGeometry(v);
    }

    // SingleAxisTiltRotator::createRotatedScannerGeometry.
    ScannerGeometry rotated(float tilt_deg, float xaxis_tilt_deg = 0.f) const {
        etcu_view out{};
        check(etcu_view_rotate(&view_, tilt_deg, xaxis_tilt_deg, &out), nullptr);
        return ScannerGeometry(out);
    }

    std::array<float, 16> getProjectionMatrix() const {
        std::array<float, 16> m{};
        check(etcu_view_projection_matrix(&view_, m.data()), nullptr);
        return m;
    }

    float getTraversalLengthThroughBoundingBox(const float bbox_min[3], const float bbox_max[3]) const {
        float r = 0.f;
        check(etcu_view_traversal_length(&view_, bbox_min, bbox_max, &r), nullptr);
        return r;
    }

    const etcu_view& view() const { return view_; }
    uint32_t width() const { return view_.width; }
    uint32_t height() const { return view_.height; }

private:
    etcu_view view_{};
};

class GPUMappedVolume {
public:
    // resolution (x, y, z); bounding box centred on origin with extent dimension
    // (VolumeParameterSet.cpp:68-71); subVolumeCount z slabs.
    GPUMappedVolume(Framework& fw, const std::array<uint32_t, 3>& resolution, const std::array<float, 3>& bbox_min,
                    const std::array<float, 3>& bbox_max, etcu_voxel_type type = ETCU_VOXEL_FLOAT32,
                    uint32_t subvolume_count = 1, float init_value = 0.f)
        : fw_(&fw), res_(resolution) {
        desc_ = etcu_volume_desc{};
        for (int i = 0; i < 3; ++i) {
            desc_.resolution[i] = resolution[i];
            desc_.bbox_min[i] = bbox_min[i];
            desc_.bbox_max[i] = bbox_max[i];
        }
        desc_.subvolume_count = subvolume_count;
        check(etcu_volume_create(fw.handle(), &desc_, type, init_value, &vol_), fw.handle());
    }

    // Centred volume with unit voxels.
    GPUMappedVolume(Framework& fw, const std::array<uint32_t, 3>& resolution, etcu_voxel_type type = ETCU_VOXEL_FLOAT32,
                    uint32_t subvolume_count = 1)
        : GPUMappedVolume(fw, resolution,
                          {-0.5f * resolution[0], -0.5f * resolution[1], -0.5f * resolution[2]},
                          {0.5f * resolution[0], 0.5f * resolution[1], 0.5f * resolution[2]}, type,
                          subvolume_count) {}

    ~GPUMappedVolume() { etcu_volume_destroy(vol_); }
    GPUMappedVolume(const GPUMappedVolume&) = delete;
    GPUMappedVolume& operator=(const GPUMappedVolume&) = delete;

    size_t voxelCount() const { return (size_t)res_[0] * res_[1] * res_[2]; }
    const std::array<uint32_t, 3>& resolution() const { return res_; }
    const etcu_volume_desc& description() const { return desc_; }
    uint32_t getSubVolumeCount() const { return desc_.subvolume_count ? desc_.subvolume_count : 1; }
    etcu_volume* handle() const { return vol_; }
    Framework& framework() const { return *fw_; }

    // Host float32 volume, x fastest.
    void upload(const float* host) { check(etcu_volume_upload(vol_, host), fw_->handle()); }
    void download(float* host) const { check(etcu_volume_download(vol_, host), fw_->handle()); }
    std::vector<float> download() const {
        std::vector<float> out(voxelCount());
        download(out.data());
        return out;
    }
    // Prior-knowledge mask (value / 255); nullptr removes it.
    void setMask(const uint8_t* host_mask) { check(etcu_volume_set_mask(vol_, host_mask), fw_->handle()); }

private:
    Framework* fw_;
    std::array<uint32_t, 3> res_;
    etcu_volume_desc desc_{};
    etcu_volume* vol_ = nullptr;
};

// LR/model/blobs/BlobParameters.cpp: Kaiser-Bessel blob (support radius in voxels, degree,
// density fall-off); BlobParameterSet.cpp:7-29 reads blobs.supportRadius / degree /
// densityFalloff.
struct BlobParameters {
    float supportRadius = 2.0f;
    uint32_t degree = 2;
    float densityFalloff = 3.6f;

    static BlobParameters createDefault() { return BlobParameters(); }
    static BlobParameters createWithParameters(float a, uint32_t m, float alpha) { return {a, m, alpha}; }
    etcu_blob_params c() const { return etcu_blob_params{supportRadius, degree, densityFalloff}; }
    // BlobRayIntegrationSampler: the blob's line integral at count distances 0 .. a.
    std::vector<float> rayIntegrationSamples(uint32_t count) const {
        std::vector<float> out(count);
        const etcu_blob_params b = c();
        check(etcu_blob_ray_integration_samples(&b, count, out.data()), nullptr);
        return out;
    }
};

class ForwardProjectionOperator {
public:
    ForwardProjectionOperator(GPUMappedVolume& vol, uint32_t samples = 1) : vol_(&vol), samples_(samples) {}
    // algorithm.basisFunctions = blobs: the perspective blob kernel with a table of
    // blob_samples entries (DefaultForwardProjectionCreator.cpp:53-60 uses 256).
    ForwardProjectionOperator(GPUMappedVolume& vol, const BlobParameters& blob, uint32_t blob_samples = 256)
        : vol_(&vol), samples_(1), blobs_(true), blob_(blob), blobSamples_(blob_samples) {}
    void setScannerGeometry(const ScannerGeometry& g) { geo_ = g; }
    void SetOutput(float* d_virtual, float* d_traversal) {
        virt_ = d_virtual;
        trav_ = d_traversal;
    }
    // Adds the sub-volume's line integrals into the outputs (the caller clears them).
    void Execute(uint32_t subvolume) {
        etcu_context* ctx = vol_->framework().handle();
        if (blobs_) {
            const etcu_blob_params b = blob_.c();
            check(etcu_forward_project_blobs(vol_->handle(), &geo_.view(), subvolume, &b, blobSamples_, virt_, trav_),
                  ctx);
        } else {
            check(etcu_forward_project(vol_->handle(), &geo_.view(), subvolume, samples_, virt_, trav_), ctx);
        }
        vol_->framework().synchronize();
    }

private:
    GPUMappedVolume* vol_;
    uint32_t samples_;
    bool blobs_ = false;
    BlobParameters blob_;
    uint32_t blobSamples_ = 256;
    ScannerGeometry geo_;
    float* virt_ = nullptr;
    float* trav_ = nullptr;
};

class BackProjectionOperator {
public:
    static constexpr uint32_t ALL_SUB_VOLUMES = ETCU_ALL_SUBVOLUMES;

    BackProjectionOperator(GPUMappedVolume& vol, float lambda, uint32_t samples = 1,
                           etcu_sampling sampling = ETCU_SAMPLING_Q8)
        : vol_(&vol), lambda_(lambda), samples_(samples), sampling_(sampling) {}
    // algorithm.basisFunctions = blobs (DefaultBackProjectionCreator.cpp:51-59).
    BackProjectionOperator(GPUMappedVolume& vol, float lambda, const BlobParameters& blob)
        : vol_(&vol), lambda_(lambda), samples_(1), sampling_(ETCU_SAMPLING_Q8), blobs_(true), blob_(blob) {}
    void setScannerGeometry(const ScannerGeometry& g) { geo_ = g; }
    void setInput(const float* d_residual, const float* d_traversal, uint32_t block_size) {
        res_ = d_residual;
        trav_ = d_traversal;
        block_ = block_size;
    }
    // Updates with lambda / blockSize (BackProjectionKernel.cpp:94).
    void execute(uint32_t subvolume = ALL_SUB_VOLUMES) {
        etcu_context* ctx = vol_->framework().handle();
        if (blobs_) {
            const etcu_blob_params b = blob_.c();
            check(etcu_back_project_blobs(vol_->handle(), &geo_.view(), subvolume, &b, lambda_, block_, res_, trav_),
                  ctx);
        } else {
            check(etcu_back_project(vol_->handle(), &geo_.view(), subvolume, samples_, lambda_, block_, res_, trav_,
                                    sampling_),
                  ctx);
        }
        vol_->framework().synchronize();
    }

private:
    GPUMappedVolume* vol_;
    float lambda_;
    uint32_t samples_;
    etcu_sampling sampling_;
    bool blobs_ = false;
    BlobParameters blob_;
    ScannerGeometry geo_;
    const float* res_ = nullptr;
    const float* trav_ = nullptr;
    uint32_t block_ = 1;
};

// LR/algorithm/blobs/BlobVoxelizerOperator.cpp: the blob coefficients convolved with the
// voxelisation kernel into a second volume of the same resolution and box.
class BlobVoxelizerOperator {
public:
    BlobVoxelizerOperator(GPUMappedVolume& blobs, const BlobParameters& p)
        : blobs_(&blobs),
          p_(p),
          voxels_(blobs.framework(), blobs.resolution(),
                  {blobs.description().bbox_min[0], blobs.description().bbox_min[1], blobs.description().bbox_min[2]},
                  {blobs.description().bbox_max[0], blobs.description().bbox_max[1], blobs.description().bbox_max[2]}) {}
    void voxelize() {
        const etcu_blob_params b = p_.c();
        check(etcu_blob_voxelize(blobs_->handle(), voxels_.handle(), &b), blobs_->framework().handle());
    }
    GPUMappedVolume& getVoxelVolume() { return voxels_; }

private:
    GPUMappedVolume* blobs_;
    BlobParameters p_;
    GPUMappedVolume voxels_;
};

// The reference's configuration keys of the block-iterative reconstruction.
struct AlgebraicParameterSet {
    std::string algorithm = "sart";
    uint32_t blockSize = 1;
    uint32_t iterations = 1;
    float lambda = 0.3f;
    bool useLongObjectCompensation = false;
    uint32_t fpSamples = 1, bpSamples = 1;
    etcu_voxel_type voxelType = ETCU_VOXEL_FLOAT32;
    etcu_order order = ETCU_ORDER_RANDOM;  // optimization.projectionIteration default
    etcu_sampling sampling = ETCU_SAMPLING_Q8;
    etcu_projection_storage projectionStorage = ETCU_PROJ_F32;  // device storage of the tilt series
    std::string basisFunctions = "voxels";  // algorithm.basisFunctions
    BlobParameters blob;                    // blobs.*
    bool enableVoxelization = false;        // output.options.enableVoxelization
    uint32_t subVolumeCount = 1;
    std::array<uint32_t, 3> resolution{{0, 0, 0}};
    std::array<float, 3> dimension{{0.f, 0.f, 0.f}};
    std::array<float, 3> origin{{0.f, 0.f, 0.f}};
    bool hasDimension = false;
    float initValue = 0.f;
    std::vector<uint32_t> skip;
    float xAxisTilt = 0.f;

    static std::vector<float> vec(const std::string& s) {
        std::string t = s;
        for (char& c : t)
            if (c == ',') c = ' ';
        std::istringstream in(t);
        std::vector<float> out;
        float f;
        while (in >> f) out.push_back(f);
        return out;
    }

    // AlgorithmParameterSet.cpp:10-23 and the optimization / volume / hardware /
    // input parameter sets; the messages are the reference's.
    static AlgebraicParameterSet fromConfig(const std::map<std::string, std::string>& cfg) {
        auto get = [&](const std::string& k, const std::string& dflt) {
            auto it = cfg.find(k);
            return it == cfg.end() ? dflt : it->second;
        };
        AlgebraicParameterSet p;
        auto alg = cfg.find("algorithm");
        if (alg == cfg.end()) throw Exception(ETCU_ERR_INVALID_ARGUMENT, "missing parameter algorithm");
        p.algorithm = alg->second;
        if (p.algorithm == "sart") p.blockSize = 1;
        else if (p.algorithm == "sirt") p.blockSize = ETCU_BLOCK_ALL;
        else p.blockSize = (uint32_t)std::stoul(get("algorithm.blockSize", std::to_string(ETCU_BLOCK_ALL)));
        p.iterations = (uint32_t)std::stoul(get("algorithm.numberOfIterations", "1"));
        p.lambda = std::stof(get("algorithm.lambda", "0.3"));
        const std::string loc = get("algorithm.useLongObjectCompensation", "false");
        p.useLongObjectCompensation = loc == "true" || loc == "1" || loc == "yes";
        const std::string basis = get("algorithm.basisFunctions", "voxels");
        if (basis != "voxels" && basis != "blobs")
            throw Exception(ETCU_ERR_INVALID_ARGUMENT,
                            "Illegal value for parameter \"algorithm.basisFunctions\": " + basis + "!");
        p.basisFunctions = basis;
        p.blob.supportRadius = std::stof(get("blobs.supportRadius", "2.0"));
        p.blob.degree = (uint32_t)std::stoul(get("blobs.degree", "2"));
        p.blob.densityFalloff = std::stof(get("blobs.densityFalloff", "3.6"));
        const std::string vox = get("output.options.enableVoxelization", "false");
        p.enableVoxelization = vox == "true" || vox == "1" || vox == "yes";
        p.fpSamples = (uint32_t)std::stoul(get("forwardProjection.samples", "1"));
        p.bpSamples = (uint32_t)std::stoul(get("backProjection.samples", "1"));
        const std::string vt = get("optimization.internalVoxelRepresentationType", "float");
        if (vt == "float" || vt == "float32") p.voxelType = ETCU_VOXEL_FLOAT32;
        else if (vt == "half") p.voxelType = ETCU_VOXEL_HALF16;
        else if (vt == "half_master") p.voxelType = ETCU_VOXEL_F16_MASTER;
        else if (vt == "bf16_master") p.voxelType = ETCU_VOXEL_BF16_MASTER;
        else throw Exception(ETCU_ERR_INVALID_ARGUMENT, "UChar is not supported as a valid internal voxel storage data type.");
        const std::string ord = get("optimization.projectionIteration", "random");
        if (ord == "identity") p.order = ETCU_ORDER_IDENTITY;
        else if (ord == "random") p.order = ETCU_ORDER_RANDOM;
        else if (ord == "maxangle") p.order = ETCU_ORDER_MAXANGLE;
        else if (ord == "buckets") p.order = ETCU_ORDER_BUCKETS;
        else throw Exception(ETCU_ERR_INVALID_ARGUMENT, "Illegal ProjectionSetType!");
        p.subVolumeCount = (uint32_t)std::stoul(get("hardware.subVolumeCount", "1"));
        if (cfg.count("volume.dimension")) {
            const auto d = vec(cfg.at("volume.dimension"));
            for (int i = 0; i < 3 && i < (int)d.size(); ++i) {
                p.dimension[i] = d[i];
                p.resolution[i] = (uint32_t)d[i];
            }
            p.hasDimension = true;
        }
        if (cfg.count("volume.resolution")) {
            const auto r = vec(cfg.at("volume.resolution"));
            for (int i = 0; i < 3 && i < (int)r.size(); ++i) p.resolution[i] = (uint32_t)r[i];
        }
        if (cfg.count("volume.origin")) {
            const auto o = vec(cfg.at("volume.origin"));
            for (int i = 0; i < 3 && i < (int)o.size(); ++i) p.origin[i] = o[i];
        }
        p.initValue = std::stof(get("volume.initValue", "0"));
        if (cfg.count("input.skipProjections"))
            for (float f : vec(cfg.at("input.skipProjections"))) p.skip.push_back((uint32_t)f);
        p.xAxisTilt = std::stof(get("input.xAxisTilt", "0"));
        if (p.blockSize == 0) throw Exception(ETCU_ERR_INVALID_ARGUMENT, "Illegal ProjectionBlockSize!");
        return p;
    }

    etcu_recon_params reconParams(bool use_graph = true) const {
        etcu_recon_params r{};
        r.lambda = lambda;
        r.block_size = blockSize;
        r.fp_samples = fpSamples;
        r.bp_samples = bpSamples;
        r.use_long_object_compensation = useLongObjectCompensation ? 1 : 0;
        r.order = order;
        r.sampling = sampling;
        r.skip = skip.empty() ? nullptr : skip.data();
        r.skip_count = (uint32_t)skip.size();
        r.use_graph = use_graph ? 1 : 0;
        r.projection_storage = projectionStorage;
        return r;
    }
};

class BlockIterativeReconstructionOperator {
public:
    // The tilt series (views.size() x height x width floats, host) is uploaded once.
    BlockIterativeReconstructionOperator(GPUMappedVolume& vol, const std::vector<ScannerGeometry>& views,
                                         const float* host_projections, const AlgebraicParameterSet& p,
                                         bool use_graph = true)
        : vol_(&vol), params_(p) {
        std::vector<etcu_view> v;
        v.reserve(views.size());
        for (const auto& g : views) v.push_back(g.view());
        const etcu_recon_params rp = p.reconParams(use_graph);
        if (p.basisFunctions == "blobs") {  // the blob kernels of the projection factories
            const etcu_blob_params b = p.blob.c();
            check(etcu_blob_recon_create(vol.handle(), v.data(), (uint32_t)v.size(), host_projections, &rp, &b,
                                         &blobRec_),
                  vol.framework().handle());
            if (p.enableVoxelization) voxelizer_.reset(new BlobVoxelizerOperator(vol, p.blob));
            return;
        }
        check(etcu_recon_create(vol.handle(), v.data(), (uint32_t)v.size(), host_projections, &rp, &rec_),
              vol.framework().handle());
    }
    ~BlockIterativeReconstructionOperator() {
        etcu_recon_destroy(rec_);
        etcu_blob_recon_destroy(blobRec_);
    }
    BlockIterativeReconstructionOperator(const BlockIterativeReconstructionOperator&) = delete;
    BlockIterativeReconstructionOperator& operator=(const BlockIterativeReconstructionOperator&) = delete;

    void run() { runNiterations(params_.iterations); }
    void runSingleIteration() { runNiterations(1); }
    void runNiterations(uint32_t n) {
        if (blobRec_) {
            check(etcu_blob_recon_run(blobRec_, n), vol_->framework().handle());
            if (voxelizer_) voxelizer_->voxelize();  // BlockIterativeReconstructionOperator.cpp:75-78
        } else {
            check(etcu_recon_run(rec_, n), vol_->framework().handle());
        }
        vol_->framework().synchronize();
    }
    // the voxelised volume when blobs are voxelised (:82-90), else the volume
    void getReconstructedVolume(float* host) const {
        (voxelizer_ ? voxelizer_->getVoxelVolume() : *vol_).download(host);
    }
    std::vector<float> getReconstructedVolume() const {
        return (voxelizer_ ? voxelizer_->getVoxelVolume() : *vol_).download();
    }
    double lastResidualSq() const {
        double r = 0.0;
        if (blobRec_)
            check(etcu_blob_recon_last_residual_sq(blobRec_, &r), vol_->framework().handle());
        else
            check(etcu_recon_last_residual_sq(rec_, &r), vol_->framework().handle());
        return r;
    }
    double dataResidualSq() const {
        double r = 0.0;
        check(etcu_recon_data_residual_sq(rec_, &r), vol_->framework().handle());
        return r;
    }
    std::vector<uint32_t> viewOrder() const {
        std::vector<uint32_t> out(1u << 16);
        uint32_t n = 0;
        if (blobRec_)
            check(etcu_blob_recon_view_order(blobRec_, out.data(), (uint32_t)out.size(), &n),
                  vol_->framework().handle());
        else
            check(etcu_recon_view_order(rec_, out.data(), (uint32_t)out.size(), &n), vol_->framework().handle());
        out.resize(n);
        return out;
    }

private:
    GPUMappedVolume* vol_;
    AlgebraicParameterSet params_;
    etcu_recon* rec_ = nullptr;
    etcu_blob_recon* blobRec_ = nullptr;
    std::unique_ptr<BlobVoxelizerOperator> voxelizer_;
};

// LR/io/datasource/MRCStack.cpp: a tilt series in an MRC file (modes 0/1/2/6) with an
// optional tilt-angle file (ImageStackDatasource::readTiltAngles); projections as
// float32, log-transformed when logarithmize (input.logarithmize).
class MRCStack {
public:
    explicit MRCStack(const std::string& path, const std::string& tilt_path = std::string(), bool logarithmize = false)
        : path_(path), log_(logarithmize) {
        check(etcu_mrc_read_info(path.c_str(), &info_), nullptr);
        if (tilt_path.empty()) {
            angles_.assign(info_.nz, 0.f);  // MRCStack::setEmptyTiltAngles
        } else {
            uint32_t n = 0;
            check(etcu_read_tilt_angles(tilt_path.c_str(), nullptr, 0, &n), nullptr);
            angles_.resize(n);
            check(etcu_read_tilt_angles(tilt_path.c_str(), angles_.data(), n, &n), nullptr);
            if (n != info_.nz)
                throw Exception(ETCU_ERR_INVALID_ARGUMENT,
                                "Number of projections DIFFERS from number of Tilt Angles given in " + tilt_path);
        }
    }
    uint32_t getNumberOfProjections() const { return info_.nz; }
    std::array<uint32_t, 2> getResolution() const { return {{info_.nx, info_.ny}}; }
    const etcu_mrc_info& info() const { return info_; }
    const std::vector<float>& tiltAngles() const { return angles_; }
    // All projections, nz x ny x nx floats.
    std::vector<float> loadProjections() const {
        std::vector<float> out((size_t)info_.nx * info_.ny * info_.nz);
        check(etcu_mrc_read_stack(path_.c_str(), log_ ? 1 : 0, out.data(), out.size()), nullptr);
        return out;
    }
    ScannerGeometry createScannerGeometry(uint32_t index, float xaxis_tilt_deg = 0.f) const {
        return ScannerGeometry::mrcBase(info_.nx, info_.ny).rotated(angles_.at(index), xaxis_tilt_deg);
    }

private:
    std::string path_;
    bool log_;
    etcu_mrc_info info_{};
    std::vector<float> angles_;
};

// VolumeFileFormatWriter + MRCWriter (x fastest, then y, then z); XZY is the reference's
// default output.options.orientation, float32 its default output.options.voxelType.
inline void writeMrcVolume(const std::string& path, const float* volume, const std::array<uint32_t, 3>& resolution,
                           etcu_orientation orientation = ETCU_AXES_XZY,
                           etcu_output_voxel_type voxelType = ETCU_OUT_FLOAT_32, bool invert = false) {
    check(etcu_mrc_write_volume_typed(path.c_str(), volume, resolution.data(), orientation, voxelType, invert ? 1 : 0),
          nullptr);
}

// ImageDeserializer::readImage / readImageFromStack: one page as height x width floats.
inline std::vector<float> readTiff(const std::string& path, uint32_t page, uint32_t* width, uint32_t* height) {
    etcu_image_info info{};
    check(etcu_tiff_read_info(path.c_str(), page, &info), nullptr);
    std::vector<float> out((size_t)info.width * info.height);
    check(etcu_tiff_read(path.c_str(), page, out.data(), out.size()), nullptr);
    if (width) *width = info.width;
    if (height) *height = info.height;
    return out;
}

// ImageSerializer::writeImage(..., TIFF_GRAY_32).
inline void writeTiff(const std::string& path, const float* image, uint32_t width, uint32_t height) {
    check(etcu_tiff_write(path.c_str(), image, width, height), nullptr);
}

// ImageStackDirectoryDatasource: a directory of images described by metadata.xml.
class ImageStackDirectoryDatasource {
public:
    explicit ImageStackDirectoryDatasource(const std::string& directory) {
        check(etcu_image_stack_open(directory.c_str(), &stack_), nullptr);
        check(etcu_image_stack_info_get(stack_, &info_), nullptr);
        angles_.resize(info_.count);
        check(etcu_image_stack_tilt_angles(stack_, angles_.data(), info_.count), nullptr);
    }
    ~ImageStackDirectoryDatasource() { etcu_image_stack_destroy(stack_); }
    ImageStackDirectoryDatasource(const ImageStackDirectoryDatasource&) = delete;
    ImageStackDirectoryDatasource& operator=(const ImageStackDirectoryDatasource&) = delete;

    uint32_t getNumberOfProjections() const { return info_.count; }
    std::array<uint32_t, 2> getResolution() const { return {{info_.width, info_.height}}; }
    const std::vector<float>& tiltAngles() const { return angles_; }
    ScannerGeometry baseGeometry() const { return ScannerGeometry(info_.base); }
    ScannerGeometry createScannerGeometry(uint32_t index, float xaxis_tilt_deg = 0.f) const {
        return baseGeometry().rotated(angles_.at(index), xaxis_tilt_deg);
    }
    // Projections first .. first + count - 1, count x height x width floats.
    std::vector<float> loadProjections(uint32_t first = 0, uint32_t count = UINT32_MAX) const {
        if (count == UINT32_MAX) count = info_.count - first;
        std::vector<float> out((size_t)info_.width * info_.height * count);
        check(etcu_image_stack_load(stack_, first, count, out.data(), out.size()), nullptr);
        return out;
    }
    // ImageStackDirectoryDatasource::writeMetaDataFile.
    static void writeMetaDataFile(const std::string& path, const std::vector<float>& tilt_angles,
                                  const std::vector<std::string>& filenames, const ScannerGeometry& base,
                                  const std::array<uint32_t, 3>& volume_resolution) {
        if (tilt_angles.size() != filenames.size())
            throw Exception(ETCU_ERR_INVALID_ARGUMENT, "Filename count does not match tilt angle count!");
        std::vector<const char*> names;
        for (const auto& f : filenames) names.push_back(f.c_str());
        check(etcu_image_stack_write_metadata(path.c_str(), tilt_angles.data(), names.data(),
                                              (uint32_t)names.size(), &base.view(), volume_resolution.data()),
              nullptr);
    }

private:
    etcu_image_stack* stack_ = nullptr;
    etcu_image_stack_info info_{};
    std::vector<float> angles_;
};

// XMLParameterSource: the value attribute of every element by its dotted path, the
// input of AlgebraicParameterSet::fromConfig.  getPathParameter resolves a value
// relative to the file's directory, '\' read as '/'.
class XMLParameterSource {
public:
    explicit XMLParameterSource(const std::string& filename) : filename_(filename) {
        size_t n = 0;
        check(etcu_xml_config_read(filename.c_str(), nullptr, 0, &n), nullptr);
        std::string text(n, '\0');
        check(etcu_xml_config_read(filename.c_str(), &text[0], n, &n), nullptr);
        std::istringstream in(text.c_str());
        std::string line;
        while (std::getline(in, line)) {
            const size_t tab = line.find('\t');
            if (tab != std::string::npos) values_.emplace(line.substr(0, tab), line.substr(tab + 1));
        }
    }
    bool parameterExists(const std::string& name) const { return values_.count(name) != 0; }
    const std::string& getStringParameter(const std::string& name) const {
        auto it = values_.find(name);
        if (it == values_.end())
            throw Exception(ETCU_ERR_INVALID_ARGUMENT, "xml config file entry does not exist: " + name);
        return it->second;
    }
    std::string getPathParameter(const std::string& name) const {
        std::string v = getStringParameter(name);
        for (char& c : v)
            if (c == '\\') c = '/';
        if (!v.empty() && v[0] == '/') return v;
        const size_t slash = filename_.rfind('/');
        return slash == std::string::npos ? v : filename_.substr(0, slash + 1) + v;
    }
    const std::map<std::string, std::string>& values() const { return values_; }

private:
    std::string filename_;
    std::map<std::string, std::string> values_;
};

// WBP plugin (plugins/WBPPlugin/src/reconstruction/WBP.cpp): RamLak-filtered projections
// back projected with their ray lengths and lambda / N into the volume.
class WBP {
public:
    WBP(GPUMappedVolume& volume, const std::vector<ScannerGeometry>& views, const float* host_projections,
        const AlgebraicParameterSet& p)
        : vol_(&volume), host_(host_projections), p_(p) {
        for (const auto& g : views) views_.push_back(g.view());
    }
    void run() {
        check(etcu_wbp(vol_->handle(), views_.data(), (uint32_t)views_.size(), host_, p_.lambda, p_.bpSamples,
                       p_.sampling),
              vol_->framework().handle());
    }
    std::vector<float> getReconstructedVolume() const { return vol_->download(); }

private:
    GPUMappedVolume* vol_;
    std::vector<etcu_view> views_;
    const float* host_;
    AlgebraicParameterSet p_;
};

// Many independent tilt series reconstructed together with SART (etcu_batch_*): one
// forward and one back-projection launch per step over all series.
class BatchReconstructionOperator {
public:
    struct Series {
        GPUMappedVolume* volume;
        std::vector<ScannerGeometry> views;
        const float* host_projections;  // views.size() x height x width floats
    };
    BatchReconstructionOperator(Framework& fw, const std::vector<Series>& series, const AlgebraicParameterSet& p,
                                bool use_graph = true)
        : fw_(&fw) {
        std::vector<std::vector<etcu_view>> views(series.size());
        std::vector<etcu_batch_series> arr(series.size());
        for (size_t i = 0; i < series.size(); ++i) {
            for (const auto& g : series[i].views) views[i].push_back(g.view());
            arr[i].volume = series[i].volume->handle();
            arr[i].views = views[i].data();
            arr[i].n_views = (uint32_t)views[i].size();
            arr[i].host_projections = series[i].host_projections;
        }
        const etcu_recon_params rp = p.reconParams(use_graph);
        check(etcu_batch_create(fw.handle(), arr.data(), (uint32_t)arr.size(), &rp, &batch_), fw.handle());
        n_ = series.size();
    }
    ~BatchReconstructionOperator() { etcu_batch_destroy(batch_); }
    BatchReconstructionOperator(const BatchReconstructionOperator&) = delete;
    BatchReconstructionOperator& operator=(const BatchReconstructionOperator&) = delete;
    void runNiterations(uint32_t n) {
        check(etcu_batch_run(batch_, n), fw_->handle());
        fw_->synchronize();
    }
    std::vector<double> lastResidualSq() const {
        std::vector<double> r(n_);
        check(etcu_batch_last_residual_sq(batch_, r.data()), fw_->handle());
        return r;
    }
    uint32_t launchesPerIteration() const { return etcu_batch_launches_per_iteration(batch_); }

private:
    Framework* fw_;
    etcu_batch* batch_ = nullptr;
    size_t n_ = 0;
};

}  // namespace b200
}  // namespace ettention
