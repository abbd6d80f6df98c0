// C ABI of the B200 block-iterative reconstruction path: contexts, device
// volumes, the projector operators and the block-iterative driver.
//
// Reference host code replaced here (LR = ettention/libReconstruction/src):
//   LR/gpu/opencl/CLAbstractionLayer.cpp, LR/gpu/GPUMapped.cpp   -> context, device buffers
//   LR/algorithm/projections/forward/ForwardProjectionKernel.cpp   -> etcu_forward_project
//   LR/algorithm/projections/back/BackProjectionKernel.cpp         -> etcu_back_project
//   LR/algorithm/reconstruction/blockiterative/*.cpp               -> etcu_recon_*
#include <cuda_runtime.h>
#include <sys/stat.h>

#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "ettention_b200.h"
#include "geometry.hpp"
#include "kernels.cuh"
#include "blobs.cuh"
#include "tune.hpp"

etcu_status check_fused_waits(etcu_recon* r);

using namespace etcu;

struct etcu_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    std::string err;
    size_t bytes = 0;
    size_t tex_align = 512, tex_pitch_align = 32;
    // scratch of the single-view back projector: interleaved (residual, length) image
    float2* pair = nullptr;  // texel (0, 0) of the padded image
    float2* pair_base = nullptr;
    void* pair_raw = nullptr;
    size_t pair_pitch = 0;  // float2 units
    uint32_t pair_w = 0, pair_h = 0;
    cudaTextureObject_t pair_tex = 0;
    bool bp_column = true;  // column-pipelined single-view back projection (ETCU_BP_COLUMN=0 disables)
    bool fused_step = true; // fused SART step BP(p) + FP(p + 1) (ETCU_FUSED=0 disables)
    bool fused_persist = true; // all fused steps of an iteration in one launch (ETCU_PERSIST=0 disables)
    int fuse_withhold_row = -1; // tests of the bounded waits (ETCU_TEST_WITHHOLD_ROW)
    int autotune = 0;           // 1: launch shapes from the tuner's cache, timed on a miss (ETCU_AUTOTUNE)
    std::string tune_log;       // the choices made on this context, one line each
    // device memory of the context's objects: a stream-ordered pool that keeps freed memory
    // for the next allocation (volumes and reconstructions created and destroyed call after
    // call then cost no driver allocation or release); trimmed when the context is destroyed
    cudaMemPool_t pool = nullptr;
};

struct etcu_volume {
    etcu_context* ctx = nullptr;
    etcu_volume_desc desc{};
    etcu_voxel_type type = ETCU_VOXEL_FLOAT32;
    float* master = nullptr;  // FP32 volume / FP32 master
    void* low = nullptr;      // half volume (HALF16) or 16-bit shadow (*_MASTER)
    uint8_t* mask = nullptr;
    std::vector<SlabConst> slabs;
    int use_min = 0, use_max = 0;
    float vmin = 0.f, vmax = 0.f;
};

struct etcu_recon {
    etcu_volume* vol = nullptr;
    etcu_context* ctx = nullptr;
    etcu_recon_params params{};
    uint32_t n_input = 0, W = 0, H = 0;
    std::vector<etcu_view> hviews;  // the input views (the slab decomposition recomputes their LOC length)
    std::vector<uint32_t> order;
    uint32_t block = 1, nblocks = 0;
    float* d_proj = nullptr;  // measured projections, element type proj_kind (load_real)
    bool own_proj = false;
    int proj_kind = 0;         // etcu_projection_storage
    ViewConst* d_views = nullptr;
    uint32_t* d_order = nullptr;
    float4* d_samples = nullptr;
    uint32_t nsamples = 1;
    float2* rl = nullptr;       // texel (0, 0) of slot 0 (images are padded by kPad zero texels)
    float2* rl_base = nullptr;  // first byte of slot 0
    void* rl_raw = nullptr;
    size_t rl_pitch = 0, rl_slot = 0;  // float2 units
    uint32_t slots = 0;
    std::vector<cudaTextureObject_t> texs;
    cudaTextureObject_t* d_texs = nullptr;
    double* d_resid = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t launches = 0;
    bool persp = false;
    std::vector<int> fp_paths;      // per slab
    std::vector<uint8_t> row_const; // per view id
    std::vector<ViewConst> hvc;     // host copy of the view constants, [slab][view id]
    std::vector<float4> hsamples;   // host copy of the sample patterns, [view id][sample]
    // fused SART step (sart_fused_kernel): per view id its tap window, per (view id,
    // volume row) the detector rows of its rays
    bool fused = false;
    std::vector<int> fuse_x0lo, fuse_ntaps;
    int2* d_jrange = nullptr;
    size_t fuse_smem = 0;
    // every fused step of an iteration in one launch (sart_fused_persistent_kernel)
    bool fuse_persist = false;
    int fuse_window = 0, fuse_grid = 0;
    int fuse_per_sm = 0, fuse_sms = 0;  // resident blocks per SM of the persistent launch, SMs
    int2* d_tapwin = nullptr;     // per view id
    uint32_t* d_fuse_ctl = nullptr;  // unit counter + steps finished per row, then the error word
};

namespace {

thread_local std::string g_create_error;

etcu_status fail(etcu_context* ctx, etcu_status st, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (ctx) ctx->err = buf;
    else g_create_error = buf;
    return st;
}

#define CK(ctx, call)                                                                                   \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess)                                                                          \
            return fail(ctx, e_ == cudaErrorMemoryAllocation ? ETCU_ERR_OUT_OF_MEMORY : ETCU_ERR_CUDA, \
                        "%s failed: %s", #call, cudaGetErrorString(e_));                                \
    } while (0)

#define CKL(ctx) CK(ctx, cudaGetLastError())

etcu_status dalloc(etcu_context* ctx, void** p, size_t bytes) {
    *p = nullptr;
    if (bytes == 0) return ETCU_OK;
    cudaError_t e = ctx && ctx->pool ? cudaMallocFromPoolAsync(p, bytes, ctx->pool, ctx->stream) : cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, ETCU_ERR_OUT_OF_MEMORY, "device allocation of %zu bytes failed: %s", bytes,
                    cudaGetErrorString(e));
    }
    ctx->bytes += bytes;
    return ETCU_OK;
}

// Texture-bound images must start on cudaDeviceProp::textureAlignment; the raw
// allocation is over-sized by that much and the aligned base returned.
etcu_status dalloc_aligned(etcu_context* ctx, void** raw, void** aligned, size_t bytes, size_t align) {
    etcu_status s = dalloc(ctx, raw, bytes + align);
    if (s != ETCU_OK) return s;
    uintptr_t a = ((uintptr_t)*raw + align - 1) / align * align;
    *aligned = (void*)a;
    return ETCU_OK;
}

void dfree(etcu_context* ctx, void* p, size_t bytes) {
    if (p) {
        if (ctx->pool) cudaFreeAsync(p, ctx->stream);
        else cudaFree(p);
        ctx->bytes -= std::min(ctx->bytes, bytes);
    }
}

size_t voxel_count(const etcu_volume_desc& d) {
    return (size_t)d.resolution[0] * d.resolution[1] * d.resolution[2];
}

float4 f4(const float* p) { return make_float4(p[0], p[1], p[2], 0.f); }

// VolumeProperties::init / setSubVolumeCount (LR/model/volume/VolumeProperties.cpp:21-98).
bool make_slabs(const etcu_volume_desc& d, std::vector<SlabConst>& out, std::string& err) {
    uint32_t cnt = d.subvolume_count == 0 ? 1 : d.subvolume_count;
    if (d.resolution[2] < cnt) {
        char b[256];
        snprintf(b, sizeof b, "Volume of size %u in z direction cannot be split into %u subvolumes!", d.resolution[2],
                 cnt);
        err = b;
        return false;
    }
    float vs[3], ivs[3];
    for (int i = 0; i < 3; ++i) {
        vs[i] = (d.bbox_max[i] - d.bbox_min[i]) / (float)d.resolution[i];
        ivs[i] = 1.0f / vs[i];
    }
    uint32_t base = d.resolution[2] / cnt, rem = d.resolution[2] - cnt * base;
    float next_min[3] = {d.bbox_min[0], d.bbox_min[1], d.bbox_min[2]};
    uint32_t z0 = 0;
    out.clear();
    for (uint32_t i = 0; i < cnt; ++i) {
        SlabConst s{};
        s.rx = (int)d.resolution[0];
        s.ry = (int)d.resolution[1];
        s.rz = (int)(i < rem ? base + 1 : base);
        s.z0 = (int)z0;
        float smax[3] = {next_min[0] + (float)s.rx * vs[0], next_min[1] + (float)s.ry * vs[1],
                         next_min[2] + (float)s.rz * vs[2]};
        s.bmin = f4(next_min);
        s.bmax = f4(smax);
        s.cmin = f4(d.bbox_min);
        s.cmax = f4(d.bbox_max);
        s.vs = f4(vs);
        s.ivs = f4(ivs);
        next_min[2] = smax[2];
        z0 += (uint32_t)s.rz;
        out.push_back(s);
    }
    return true;
}

// Host packing of the per-view kernel constants (LR/model/geometry/ScannerGeometry.cpp:95-103).
ViewConst make_view_const(const etcu_view& v, const SlabConst& slab, float loc_length) {
    ViewConst c{};
    Vec3 r = ray_direction(v);
    c.ray = make_float4(r.x, r.y, r.z, 0.f);
    float inv[3] = {1.0f / r.x, 1.0f / r.y, 1.0f / r.z};
    if (r.x == 0.f) inv[0] = -FLT_MAX;
    if (r.y == 0.f) inv[1] = -FLT_MAX;
    if (r.z == 0.f) inv[2] = -FLT_MAX;
    c.inv = make_float4(inv[0], inv[1], inv[2], 0.f);
    c.source = f4(v.source);
    c.detector = f4(v.detector);
    c.hpitch = f4(v.hpitch);
    c.vpitch = f4(v.vpitch);
    projection_matrix(v, c.mat);
    c.loc_length = loc_length;
    c.perspective = v.perspective ? 1 : 0;
    // The xz walk is exact when y never steps (ray.y == 0) and every step
    // difference vs * inv * sign(ray) is finite (DDARaytracer.hl:79).
    auto sdf = [](float vs, float iv, float rr) {
        float sg = rr > 0.f ? 1.f : (rr < 0.f ? -1.f : rr);
        volatile float a = vs * iv;
        return a * sg;
    };
    float sdx = sdf(slab.vs.x, inv[0], r.x), sdy = sdf(slab.vs.y, inv[1], r.y), sdz = sdf(slab.vs.z, inv[2], r.z);
    // The xz walk decodes (iz, ix) from its 32-bit offset iz * rx * ry + ix: a step off
    // the x range must not alias a voxel of another z row (ry >= 2), and one below
    // z = 0 must wrap past the last row ((rz + 1) * rx * ry <= 2^32).
    const bool decodable = slab.ry >= 2 && (unsigned long long)slab.rx * (unsigned long long)slab.ry *
                                                   (unsigned long long)(slab.rz + 1) <= (1ull << 32);
    c.fast2d = (!v.perspective && r.y == 0.f && decodable && std::isfinite(sdx) && std::isfinite(sdy) &&
                std::isfinite(sdz)) ? 1 : 0;
    return c;
}

// Affine projection whose detector row depends only on y (parallel views tilted about y).
bool row_constant(const ViewConst& c) {
    return c.mat[1] == 0.f && c.mat[9] == 0.f && c.mat[3] == 0.f && c.mat[7] == 0.f && c.mat[11] == 0.f &&
           c.mat[15] == 1.f;
}

etcu_status check_view(etcu_context* ctx, const etcu_view* v) {
    if (!v) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "view is NULL");
    if (v->width == 0 || v->height == 0)
        return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "projection resolution must be non-zero");
    float m[16];
    if (!projection_matrix(*v, m)) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "matrix not invertible");
    return ETCU_OK;
}

size_t slab_offset_elems(const etcu_volume* vol, const SlabConst& s) {
    return (size_t)s.z0 * (size_t)s.rx * (size_t)s.ry;
}

// ------------------------------------------------------------- launches
template <typename VoxT, bool kMask, int kPath>
void launch_fp_t(const FpArgs& a, uint32_t nviews, cudaStream_t st) {
    dim3 block(128);
    dim3 grid;
    if (kPath == kFpPathPerspective) grid = dim3((a.W + 15) / 16, (a.H + 7) / 8, nviews);
    else grid = dim3((a.W + 127) / 128, a.H, nviews);
    forward_project_kernel<VoxT, kMask, kPath><<<grid, block, 0, st>>>(a);
}

template <typename VoxT, bool kMask>
void launch_fp_m(const FpArgs& a, int path, uint32_t nviews, cudaStream_t st) {
    switch (path) {
    case kFpPathXz: launch_fp_t<VoxT, kMask, kFpPathXz>(a, nviews, st); break;
    case kFpPathXzNoCap: launch_fp_t<VoxT, kMask, kFpPathXzNoCap>(a, nviews, st); break;
    case kFpPathPerspective: launch_fp_t<VoxT, kMask, kFpPathPerspective>(a, nviews, st); break;
    default: launch_fp_t<VoxT, kMask, kFpPathGeneral>(a, nviews, st); break;
    }
}

template <typename VoxT>
void launch_fp_v(const FpArgs& a, bool mask, int path, uint32_t nviews, cudaStream_t st) {
    if (mask) launch_fp_m<VoxT, true>(a, path, nviews, st);
    else launch_fp_m<VoxT, false>(a, path, nviews, st);
}

// Walk specialisation shared by every view of a launch.
int fp_path(bool persp, bool all_fast2d, const SlabConst& slab) {
    if (persp) return kFpPathPerspective;
    if (!all_fast2d) return kFpPathGeneral;
    return (slab.rx + slab.rz - 1 <= kMaxDdaIterations) ? kFpPathXzNoCap : kFpPathXz;
}

void launch_fp(const etcu_volume* vol, const FpArgs& a, int path, uint32_t nviews, cudaStream_t st) {
    bool mask = a.mask != nullptr;
    switch (vol->type) {
    case ETCU_VOXEL_FLOAT32: launch_fp_v<float>(a, mask, path, nviews, st); break;
    case ETCU_VOXEL_HALF16:
    case ETCU_VOXEL_F16_MASTER: launch_fp_v<__half>(a, mask, path, nviews, st); break;
    case ETCU_VOXEL_BF16_MASTER: launch_fp_v<__nv_bfloat16>(a, mask, path, nviews, st); break;
    }
}

constexpr size_t kBpSmemBudget = 160 * 1024;

template <bool kPersp, bool kMask, int kStore, int kSampling>
void launch_bp_t(const BpArgs& a, int device, cudaStream_t st) {
    // Opt in to the large dynamic shared-memory carve-out once per device and instantiation.
    // Host threads driving different devices may get here together: the set of opted-in
    // devices is one atomic word (setting the attribute twice is harmless).
    static std::atomic<unsigned long long> opted{0};
    // the perspective kernel with the intensity clamps compiled in only when a clamp is set
    auto persp = (a.use_min || a.use_max) ? bp_perspective_kernel<kMask, kStore, kSampling, true>
                                          : bp_perspective_kernel<kMask, kStore, kSampling, false>;
    auto kern = kPersp ? persp : bp_parallel_kernel<kMask, kStore, kSampling>;
    if (device < 64 && !(opted.load(std::memory_order_acquire) & (1ull << device))) {
        if (kPersp) {
            cudaFuncSetAttribute(bp_perspective_kernel<kMask, kStore, kSampling, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBpSmemBudget);
            cudaFuncSetAttribute(bp_perspective_kernel<kMask, kStore, kSampling, false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBpSmemBudget);
        } else {
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBpSmemBudget);
        }
        opted.fetch_or(1ull << device, std::memory_order_acq_rel);
    }
    // perspective: the per-(view, z voxel) table of the one-sample path in the sample slots
    const size_t smem = bp_smem_bytes(a.nviews, kPersp ? kBpZPersp : a.nsamples);
    const int zc = kPersp ? kBpZPersp : kBpZ;
    const int zchunks = (a.slab.rz + zc - 1) / zc;
    dim3 block(32, 8, 1);
    // parallel: each block walks up to 4 z-chunks (grid-stride) to amortise its staging;
    // perspective: z chunks fastest, so the blocks in flight share their texels in L2
    const dim3 grid = kPersp ? dim3(zchunks, (a.slab.rx + 31) / 32, (a.slab.ry + 7) / 8)
                             : dim3((a.slab.rx + 31) / 32, (a.slab.ry + 7) / 8, (zchunks + 3) / 4);
    kern<<<grid, block, smem, st>>>(a);
}

template <bool kPersp, bool kMask, int kStore>
void launch_bp_s(const BpArgs& a, etcu_sampling sm, int dev, cudaStream_t st) {
    if (sm == ETCU_SAMPLING_EXACT) launch_bp_t<kPersp, kMask, kStore, kSampleExact>(a, dev, st);
    else if (sm == ETCU_SAMPLING_HW_TEXTURE) launch_bp_t<kPersp, kMask, kStore, kSampleTexture>(a, dev, st);
    else launch_bp_t<kPersp, kMask, kStore, kSampleQ8>(a, dev, st);
}

template <bool kPersp, bool kMask>
void launch_bp_m(const BpArgs& a, etcu_voxel_type t, etcu_sampling sm, int dev, cudaStream_t st) {
    switch (t) {
    case ETCU_VOXEL_FLOAT32: launch_bp_s<kPersp, kMask, 0>(a, sm, dev, st); break;
    case ETCU_VOXEL_HALF16: launch_bp_s<kPersp, kMask, 1>(a, sm, dev, st); break;
    case ETCU_VOXEL_F16_MASTER: launch_bp_s<kPersp, kMask, 2>(a, sm, dev, st); break;
    case ETCU_VOXEL_BF16_MASTER: launch_bp_s<kPersp, kMask, 3>(a, sm, dev, st); break;
    }
}

template <bool kMask, int kStore>
void launch_bp_sart(const BpArgs& a, etcu_sampling sm, cudaStream_t st) {
    const int bx = (a.slab.rx + 31) / 32, by = (a.slab.ry + 7) / 8;
    // enough blocks for a few waves; each thread then walks its column's z range
    const int want = 148 * 16;
    int zs = std::max(1, std::min((a.slab.rz + 15) / 16, (want + bx * by - 1) / (bx * by)));
    dim3 block(32, 8, 1), grid(bx, by, zs);
    if (sm == ETCU_SAMPLING_EXACT) bp_sart_row_kernel<kMask, kStore, kSampleExact><<<grid, block, 0, st>>>(a);
    else bp_sart_row_kernel<kMask, kStore, kSampleQ8><<<grid, block, 0, st>>>(a);
}

template <bool kMask>
void launch_bp_sart_m(const BpArgs& a, etcu_voxel_type t, etcu_sampling sm, cudaStream_t st) {
    switch (t) {
    case ETCU_VOXEL_FLOAT32: launch_bp_sart<kMask, 0>(a, sm, st); break;
    case ETCU_VOXEL_HALF16: launch_bp_sart<kMask, 1>(a, sm, st); break;
    case ETCU_VOXEL_F16_MASTER: launch_bp_sart<kMask, 2>(a, sm, st); break;
    case ETCU_VOXEL_BF16_MASTER: launch_bp_sart<kMask, 3>(a, sm, st); break;
    }
}

struct BpColPlan {
    int groups = 0;  // 4-voxel x groups per thread (1 or 2)
    int shadow = 0;  // the master's 16-bit shadow written beside it (1: FP16, 2: BF16)
    int x0lo = 0, ntaps = 0;
    int zper = 0, zchunks = 0, grid = 0;
    size_t smem = 0;
};

template <int kGroups>
void bp_col_limits(int dev, size_t smem, int& per_sm) {
    static std::mutex mu;
    static std::vector<char> opted;
    {
        std::lock_guard<std::mutex> lock(mu);
        if ((int)opted.size() <= dev) opted.resize(dev + 1, 0);
        if (!opted[dev]) {
            cudaDeviceProp prop;
            if (cudaGetDeviceProperties(&prop, dev) == cudaSuccess) {
                cudaFuncSetAttribute(bp_sart_column_kernel<kGroups, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)prop.sharedMemPerBlockOptin);
                cudaFuncSetAttribute(bp_sart_column_kernel<kGroups, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)prop.sharedMemPerBlockOptin);
                cudaFuncSetAttribute(bp_sart_column_kernel<kGroups, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)prop.sharedMemPerBlockOptin);
            }
            cudaGetLastError();
            opted[dev] = 1;
        }
    }
    per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bp_sart_column_kernel<kGroups, 0>, kBpColThreads,
                                                      smem) != cudaSuccess) {
        cudaGetLastError();
        per_sm = 0;
    }
}

int device_sms(int dev) {
    static std::mutex mu;
    static std::vector<int> sms;
    std::lock_guard<std::mutex> lock(mu);
    if ((int)sms.size() <= dev) sms.resize(dev + 1, 0);
    if (sms[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) cudaGetLastError();
        sms[dev] = n;
    }
    return sms[dev];
}

// Whether the column-pipelined back projector applies to this view and
// sub-volume, and its tap window, item and grid sizes.  It needs an FP32 volume (or FP32 master)
// without mask and x rows of a multiple of 4 and at most 2048 voxels.  The tap window spans the
// columns floor(u - 0.5) of every voxel centre with two columns of margin on each
// side (the kernel's float coordinate is within a few ulps of the double
// evaluated here at the sub-volume's corners; u is affine in the voxel indices).
// FP32 volumes and FP32 masters with a 16-bit shadow (written beside the master).
bool plan_bp_col(const etcu_volume* vol, const SlabConst& g, const ViewConst& vc, const float4& smp, BpColPlan& p) {
    etcu_context* ctx = vol->ctx;
    if (!ctx->bp_column || vol->type == ETCU_VOXEL_HALF16 || vol->mask) return false;
    p.shadow = vol->type == ETCU_VOXEL_F16_MASTER ? 1 : (vol->type == ETCU_VOXEL_BF16_MASTER ? 2 : 0);
    if (g.rx <= 0 || g.ry <= 0 || g.rz <= 0 || g.rx % 4 != 0 || g.rx > 8 * kBpColThreads) return false;
    double umin = 1e300, umax = -1e300;
    for (int c = 0; c < 8; ++c) {
        const double x = (c & 1) ? g.rx - 1 : 0, y = (c & 2) ? g.ry - 1 : 0, z = (c & 4) ? g.rz - 1 : 0;
        const double px = (double)g.bmin.x + (x + 0.5) * g.vs.x + smp.x;
        const double py = (double)g.bmin.y + (y + 0.5) * g.vs.y + smp.y;
        const double pz = (double)g.bmin.z + (z + 0.5) * g.vs.z + smp.z;
        const double u = (double)vc.mat[0] * px + (double)vc.mat[4] * py + (double)vc.mat[8] * pz + vc.mat[12];
        umin = std::min(umin, u);
        umax = std::max(umax, u);
    }
    if (!(umin > -16000.0 && umax < 16000.0)) return false;  // |256 u| < 2^22 for the tap split
    p.x0lo = (int)std::floor(umin - 0.5) - 2;
    p.ntaps = (int)std::floor(umax - 0.5) + 2 - p.x0lo + 1;
    p.groups = g.rx <= 4 * kBpColThreads ? 1 : 2;
    p.smem = bp_col_smem_bytes(g.rz, p.ntaps, p.groups);
    if (p.smem > 112 * 1024) return false;
    const int dev = ctx->device;
    int per_sm = 0;
    if (p.groups == 1) bp_col_limits<1>(dev, p.smem, per_sm);
    else bp_col_limits<2>(dev, p.smem, per_sm);
    const int sms = device_sms(dev);
    if (per_sm < 1 || sms < 1) return false;
    const long long cap = (long long)sms * per_sm;
    // z chunking: balance items over the resident blocks, counting about eight
    // z rows of staging and pipeline start per item
    long long best = -1;
    for (int zc = 1; zc <= g.rz; ++zc) {
        const int zper = (g.rz + zc - 1) / zc;
        const int zcn = (g.rz + zper - 1) / zper;
        const long long items = (long long)g.ry * zcn;
        if (items > (1ll << 30)) break;
        const long long grid = std::min(items, cap);
        const long long cost = (items + grid - 1) / grid * (zper + 8);
        if (best < 0 || cost < best) {
            best = cost;
            p.zper = zper;
            p.zchunks = zcn;
            p.grid = (int)grid;
        }
        if (items >= 64 * cap) break;
    }
    return best > 0;
}

void launch_bp_col(const BpArgs& a0, const BpColPlan& p, cudaStream_t st) {
    BpColArgs a{};
    a.vol = (float*)a0.vol;
    a.slab = a0.slab;
    a.views = a0.views;
    a.order = a0.order;
    a.first = a0.first;
    a.inline_view = a0.inline_view;
    a.samples = a0.samples;
    a.inline_sample = a0.inline_samples[0];
    a.rl = a0.rl;
    a.rl_pitch = a0.rl_pitch;
    a.W = a0.W;
    a.H = a0.H;
    a.lambda = a0.lambda;
    a.x0lo = p.x0lo;
    a.ntaps = p.ntaps;
    a.zper = p.zper;
    a.zchunks = p.zchunks;
    a.shadow = a0.shadow;
    const dim3 grid(p.grid), block(kBpColThreads);
    const int sh = p.shadow;
    if (p.groups == 1) {
        if (sh == 1) bp_sart_column_kernel<1, 1><<<grid, block, p.smem, st>>>(a);
        else if (sh == 2) bp_sart_column_kernel<1, 2><<<grid, block, p.smem, st>>>(a);
        else bp_sart_column_kernel<1, 0><<<grid, block, p.smem, st>>>(a);
    } else {
        if (sh == 1) bp_sart_column_kernel<2, 1><<<grid, block, p.smem, st>>>(a);
        else if (sh == 2) bp_sart_column_kernel<2, 2><<<grid, block, p.smem, st>>>(a);
        else bp_sart_column_kernel<2, 0><<<grid, block, p.smem, st>>>(a);
    }
}

// Back projection of a.nviews views; when their staged constants exceed the
// shared-memory budget the views are split over consecutive launches, which
// applies them in the same order.  `hvc` / `hsmp` are host copies of the single
// view's constants and sample (they select the column-pipelined kernel).  Returns the
// number of launches.
uint32_t launch_bp(const etcu_volume* vol, const BpArgs& a0, bool persp, etcu_sampling sm, cudaStream_t st,
                   bool row_const = false, const ViewConst* hvc = nullptr, const float4* hsmp = nullptr) {
    const int dev = vol->ctx->device;
    if (!persp && row_const && a0.nviews == 1 && a0.nsamples == 1 && sm != ETCU_SAMPLING_HW_TEXTURE) {
        BpColPlan plan;
        if (sm == ETCU_SAMPLING_Q8 && hvc && hsmp && plan_bp_col(vol, a0.slab, *hvc, *hsmp, plan)) {
            launch_bp_col(a0, plan, st);
            return 1;
        }
        if (a0.mask) launch_bp_sart_m<true>(a0, vol->type, sm, st);
        else launch_bp_sart_m<false>(a0, vol->type, sm, st);
        return 1;
    }
    const size_t per_view = bp_smem_bytes(1, persp ? kBpZPersp : a0.nsamples);
    const int max_views = (int)std::max<size_t>(1, (kBpSmemBudget - 16) / per_view);
    uint32_t launches = 0;
    for (int c0 = 0; c0 < a0.nviews; c0 += max_views) {
        BpArgs a = a0;
        a.first = a0.first + (uint32_t)c0;
        a.nviews = std::min(max_views, a0.nviews - c0);
        a.rl = a0.rl + (size_t)c0 * a0.rl_slot;
        if (a0.texs) a.texs = a0.texs + c0;
        const bool mask = a.mask != nullptr;
        if (persp) {
            if (mask) launch_bp_m<true, true>(a, vol->type, sm, dev, st);
            else launch_bp_m<true, false>(a, vol->type, sm, dev, st);
        } else {
            if (mask) launch_bp_m<false, true>(a, vol->type, sm, dev, st);
            else launch_bp_m<false, false>(a, vol->type, sm, dev, st);
        }
        ++launches;
    }
    return launches;
}

void fill_bp_volume_ptrs(const etcu_volume* vol, const SlabConst& s, BpArgs& a) {
    size_t off = slab_offset_elems(vol, s);
    if (vol->type == ETCU_VOXEL_HALF16) {
        a.vol = (__half*)vol->low + off;
        a.shadow = nullptr;
    } else {
        a.vol = vol->master + off;
        a.shadow = vol->type == ETCU_VOXEL_FLOAT32 ? nullptr : (void*)((uint16_t*)vol->low + off);
    }
    a.mask = vol->mask ? vol->mask + off : nullptr;
}

void fill_fp_volume_ptrs(const etcu_volume* vol, const SlabConst& s, FpArgs& a) {
    size_t off = slab_offset_elems(vol, s);
    if (vol->type == ETCU_VOXEL_FLOAT32) a.vol = vol->master + off;
    else a.vol = (const uint16_t*)vol->low + off;
    a.mask = vol->mask ? vol->mask + off : nullptr;
}

etcu_status make_pair_texture(etcu_context* ctx, float2* base, size_t pitch_elems, uint32_t W, uint32_t H,
                              cudaTextureObject_t* out) {
    cudaResourceDesc rd{};
    rd.resType = cudaResourceTypePitch2D;
    rd.res.pitch2D.devPtr = base;
    rd.res.pitch2D.desc = cudaCreateChannelDesc<float2>();
    rd.res.pitch2D.width = W;
    rd.res.pitch2D.height = H;
    rd.res.pitch2D.pitchInBytes = pitch_elems * sizeof(float2);
    cudaTextureDesc td{};
    td.addressMode[0] = cudaAddressModeBorder;
    td.addressMode[1] = cudaAddressModeBorder;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    CK(ctx, cudaCreateTextureObject(out, &rd, &td, nullptr));
    return ETCU_OK;
}

size_t round_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Padded (residual, length) image of the single-view back projector: kPad zero
// texels around the W x H image, texel (0, 0) at `pair`.
etcu_status ensure_pair_scratch(etcu_context* ctx, uint32_t W, uint32_t H) {
    if (ctx->pair && ctx->pair_w == W && ctx->pair_h == H) return ETCU_OK;
    if (ctx->pair_tex) cudaDestroyTextureObject(ctx->pair_tex);
    ctx->pair_tex = 0;
    dfree(ctx, ctx->pair_raw, ctx->pair_pitch * sizeof(float2) * (ctx->pair_h + 2 * kPad) + ctx->tex_align);
    ctx->pair = nullptr;
    ctx->pair_raw = nullptr;
    const size_t pw = (size_t)W + 2 * kPad, ph = (size_t)H + 2 * kPad;
    size_t pitch_bytes = round_up(pw * sizeof(float2), ctx->tex_pitch_align);
    etcu_status s = dalloc_aligned(ctx, &ctx->pair_raw, (void**)&ctx->pair_base, pitch_bytes * ph, ctx->tex_align);
    if (s != ETCU_OK) return s;
    CK(ctx, cudaMemsetAsync(ctx->pair_base, 0, pitch_bytes * ph, ctx->stream));
    ctx->pair_pitch = pitch_bytes / sizeof(float2);
    ctx->pair = ctx->pair_base + kPad * ctx->pair_pitch + kPad;
    ctx->pair_w = W;
    ctx->pair_h = H;
    return make_pair_texture(ctx, ctx->pair_base, ctx->pair_pitch, (uint32_t)pw, (uint32_t)ph, &ctx->pair_tex);
}

etcu_status upload_host_float(etcu_context* ctx, float* dst, const float* host, size_t n) {
    CK(ctx, cudaMemcpyAsync(dst, host, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    return ETCU_OK;
}

void launch_1d_dims(size_t n, dim3& g, dim3& b) {
    b = dim3(256);
    g = dim3((unsigned)((n + 255) / 256));
}

etcu_status refresh_low_from_master(etcu_volume* vol) {
    etcu_context* ctx = vol->ctx;
    size_t n = voxel_count(vol->desc);
    dim3 g, b;
    launch_1d_dims(n, g, b);
    if (vol->type == ETCU_VOXEL_F16_MASTER)
        convert_from_float_kernel<__half><<<g, b, 0, ctx->stream>>>(vol->master, (__half*)vol->low, n);
    else if (vol->type == ETCU_VOXEL_BF16_MASTER)
        convert_from_float_kernel<__nv_bfloat16><<<g, b, 0, ctx->stream>>>(vol->master, (__nv_bfloat16*)vol->low, n);
    CKL(ctx);
    return ETCU_OK;
}

}  // namespace

// =============================================================== context
extern "C" int etcu_abi_version(void) { return ETCU_ABI_VERSION; }

extern "C" etcu_status etcu_context_create(int device, etcu_context** out) {
    if (!out) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(nullptr, ETCU_ERR_NO_DEVICE, "no CUDA device available (%s)", cudaGetErrorString(e));
    }
    if (device < 0 || device >= n) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "device %d out of range", device);
    std::unique_ptr<etcu_context> c(new etcu_context());
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess) return fail(nullptr, ETCU_ERR_CUDA, "cudaSetDevice failed");
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess)
        return fail(nullptr, ETCU_ERR_CUDA, "cudaGetDeviceProperties failed");
    if (prop.major < 10) return fail(nullptr, ETCU_ERR_UNSUPPORTED, "device %s (sm_%d%d) is not sm_100", prop.name,
                                     prop.major, prop.minor);
    c->tex_align = prop.textureAlignment;
    c->tex_pitch_align = prop.texturePitchAlignment;
    // A blocking stream: work on the legacy default stream (which other CUDA
    // users in the process write device images on) is ordered before and after it.
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamDefault) != cudaSuccess)
        return fail(nullptr, ETCU_ERR_CUDA, "cudaStreamCreate failed");
    c->stream = c->own_stream;
    {
        cudaMemPoolProps pp{};
        pp.allocType = cudaMemAllocationTypePinned;
        pp.handleTypes = cudaMemHandleTypeNone;
        pp.location.type = cudaMemLocationTypeDevice;
        pp.location.id = device;
        if (cudaMemPoolCreate(&c->pool, &pp) == cudaSuccess) {
            uint64_t keep = ~0ull;  // never release freed memory while the context lives
            cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep);
        } else {
            cudaGetLastError();
            c->pool = nullptr;  // plain cudaMalloc / cudaFree
        }
    }
    if (const char* env = getenv("ETCU_BP_COLUMN")) c->bp_column = atoi(env) != 0;
    if (const char* env = getenv("ETCU_FUSED")) c->fused_step = atoi(env) != 0;
    if (const char* env = getenv("ETCU_PERSIST")) c->fused_persist = atoi(env) != 0;
    if (const char* env = getenv("ETCU_TEST_WITHHOLD_ROW")) c->fuse_withhold_row = atoi(env);
    if (const char* env = getenv("ETCU_AUTOTUNE")) c->autotune = atoi(env) != 0;
    *out = c.release();
    return ETCU_OK;
}

extern "C" etcu_status etcu_context_destroy(etcu_context* ctx) {
    if (!ctx) return ETCU_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->pair_tex) cudaDestroyTextureObject(ctx->pair_tex);
    if (ctx->pair_raw) dfree(ctx, ctx->pair_raw, 0);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->pool) {
        cudaMemPoolTrimTo(ctx->pool, 0);
        cudaMemPoolDestroy(ctx->pool);  // released once every allocation from it is freed
    }
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return ETCU_OK;
}

void etcu_set_context_free_error(const char* message) { g_create_error = message ? message : ""; }

// Accessors for the library's other translation units (not exported).
int etcu_context_device_index(const etcu_context* ctx) { return ctx ? ctx->device : 0; }
int etcu_context_autotune(const etcu_context* ctx) { return ctx ? ctx->autotune : 0; }
void etcu_context_tune_note(etcu_context* ctx, const std::string& line) {
    if (ctx) ctx->tune_log += line + "\n";
}
void etcu_context_set_error(etcu_context* ctx, const char* message) {
    if (ctx) ctx->err = message ? message : "";
    else g_create_error = message ? message : "";
}

extern "C" const char* etcu_last_error(const etcu_context* ctx) {
    return ctx ? ctx->err.c_str() : g_create_error.c_str();
}

extern "C" etcu_status etcu_synchronize(etcu_context* ctx) {
    if (!ctx) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "ctx is NULL");
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    CKL(ctx);
    return ETCU_OK;
}

extern "C" etcu_status etcu_set_stream(etcu_context* ctx, void* stream) {
    if (!ctx) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "ctx is NULL");
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return ETCU_OK;
}

extern "C" size_t etcu_device_bytes(const etcu_context* ctx) { return ctx ? ctx->bytes : 0; }

extern "C" void* etcu_context_stream(const etcu_context* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

// =============================================================== launch-shape autotuner
namespace etcu_tune {
namespace {
std::mutex g_mu;
std::map<std::string, int> g_table;
bool g_loaded = false;

std::string cache_path() {
    if (const char* p = getenv("ETCU_TUNE_CACHE")) return p;
    const char* home = getenv("HOME");
    return std::string(home ? home : "/tmp") + "/.cache/ettention_b200/launch_shapes.txt";
}

void load_locked() {
    if (g_loaded) return;
    g_loaded = true;
    std::ifstream f(cache_path());
    std::string key;
    int value;
    while (f >> key >> value) g_table[key] = value;
}
}  // namespace

int lookup(const std::string& key) {
    std::lock_guard<std::mutex> lock(g_mu);
    load_locked();
    auto it = g_table.find(key);
    return it == g_table.end() ? -1 : it->second;
}

void store(const std::string& key, int value) {
    std::lock_guard<std::mutex> lock(g_mu);
    load_locked();
    g_table[key] = value;
    const std::string path = cache_path();
    const size_t slash = path.find_last_of('/');
    if (slash != std::string::npos) {  // create the directory chain
        for (size_t i = 1; i <= slash; ++i)
            if (path[i] == '/' || i == slash) {
                const std::string d = path.substr(0, i == slash ? slash : i);
                if (!d.empty()) mkdir(d.c_str(), 0755);
            }
    }
    std::ofstream f(path, std::ios::app);
    if (f) f << key << ' ' << value << '\n';
}

std::string device_tag(int device) {
    static std::mutex mu;
    static std::map<int, std::string> tags;  // device properties are slow to query: once per device
    std::lock_guard<std::mutex> lock(mu);
    auto it = tags.find(device);
    if (it != tags.end()) return it->second;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        cudaGetLastError();
        return "unknown";
    }
    std::string name(prop.name);
    for (char& c : name)
        if (c == ' ' || c == '|') c = '_';
    return tags[device] = name + "|sm" + std::to_string(prop.major) + std::to_string(prop.minor) + "|" +
                          std::to_string(prop.multiProcessorCount);
}

int search(cudaStream_t st, const std::vector<int>& candidates, const std::function<bool(int)>& run, int reps,
           std::string* log) {
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    int best = -1;
    float best_ms = 0.f;
    for (int c : candidates) {
        if (!run(c) || cudaStreamSynchronize(st) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        float ms = 1e30f;
        bool ok = true;
        for (int i = 0; i < reps && ok; ++i) {
            cudaEventRecord(e0, st);
            ok = run(c);
            cudaEventRecord(e1, st);
            if (cudaEventSynchronize(e1) != cudaSuccess) ok = false;
            float t = 0.f;
            if (ok && cudaEventElapsedTime(&t, e0, e1) == cudaSuccess) ms = std::min(ms, t);
        }
        cudaGetLastError();
        if (!ok) continue;
        if (log) *log += " " + std::to_string(c) + "=" + std::to_string(ms) + "ms";
        if (best < 0 || ms < best_ms) {
            best = c;
            best_ms = ms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}
}  // namespace etcu_tune

extern "C" etcu_status etcu_context_set_autotune(etcu_context* ctx, int mode) {
    if (!ctx) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "ctx is NULL");
    ctx->autotune = mode != 0;
    return ETCU_OK;
}

extern "C" etcu_status etcu_context_tune_report(const etcu_context* ctx, char* out, size_t capacity, size_t* needed) {
    if (!ctx) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "ctx is NULL");
    if (needed) *needed = ctx->tune_log.size() + 1;
    if (out && capacity) {
        const size_t n = std::min(capacity - 1, ctx->tune_log.size());
        memcpy(out, ctx->tune_log.data(), n);
        out[n] = 0;
    }
    return ETCU_OK;
}

// =============================================================== geometry
extern "C" etcu_status etcu_view_rotate(const etcu_view* base, float tilt, float xtilt, etcu_view* out) {
    if (!base || !out) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL view");
    *out = rotate_view(*base, tilt, xtilt);
    return ETCU_OK;
}

extern "C" etcu_status etcu_view_projection_matrix(const etcu_view* view, float out16[16]) {
    if (!view || !out16) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!projection_matrix(*view, out16)) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "matrix not invertible");
    return ETCU_OK;
}

extern "C" etcu_status etcu_view_sample_pattern(const etcu_view* view, const float vs[3], uint32_t samples,
                                                float* out4) {
    if (!view || !vs || !out4) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    std::string err;
    if (!sample_pattern(*view, vs, samples, out4, &err)) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "%s", err.c_str());
    return ETCU_OK;
}

extern "C" etcu_status etcu_view_traversal_length(const etcu_view* view, const float bmin[3], const float bmax[3],
                                                  float* out) {
    if (!view || !bmin || !bmax || !out) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    if (view->perspective)
        return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT,
                    "Calculation of traversal length is only supported for parallel scanner geometry!");
    *out = traversal_length(*view, bmin, bmax);
    return ETCU_OK;
}

extern "C" etcu_status etcu_projection_order(etcu_order order, uint32_t n, const uint32_t* skip, uint32_t nskip,
                                             uint32_t* out, uint32_t* count) {
    if (!out || !count) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    if ((int)order < 0 || (int)order > 3) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "Illegal ProjectionSetType!");
    std::vector<uint32_t> o = projection_order(order, n, skip, skip ? nskip : 0);
    for (size_t i = 0; i < o.size(); ++i) out[i] = o[i];
    *count = (uint32_t)o.size();
    return ETCU_OK;
}

// =============================================================== volume
extern "C" etcu_status etcu_volume_create(etcu_context* ctx, const etcu_volume_desc* desc, etcu_voxel_type type,
                                          float init_value, etcu_volume** out) {
    if (!ctx || !desc || !out) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    if (desc->resolution[0] == 0 || desc->resolution[1] == 0 || desc->resolution[2] == 0)
        return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "volume resolution must be non-zero");
    if ((int)type < 0 || (int)type > 3)
        return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "UChar is not supported as a valid internal voxel storage data type.");
    for (int i = 0; i < 3; ++i)
        if (!(desc->bbox_max[i] > desc->bbox_min[i]))
            return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "volume bounding box is empty along axis %d", i);
    std::unique_ptr<etcu_volume> v(new etcu_volume());
    v->ctx = ctx;
    v->desc = *desc;
    v->type = type;
    std::string err;
    if (!make_slabs(*desc, v->slabs, err)) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "%s", err.c_str());
    CK(ctx, cudaSetDevice(ctx->device));
    size_t n = voxel_count(*desc);
    etcu_status s;
    if (type != ETCU_VOXEL_HALF16) {
        if ((s = dalloc(ctx, (void**)&v->master, n * sizeof(float))) != ETCU_OK) return s;
    }
    if (type != ETCU_VOXEL_FLOAT32) {
        if ((s = dalloc(ctx, &v->low, n * 2)) != ETCU_OK) {
            dfree(ctx, v->master, n * sizeof(float));
            return s;
        }
    }
    dim3 g, b;
    launch_1d_dims(n, g, b);
    if (v->master) {
        fill_kernel<<<g, b, 0, ctx->stream>>>(v->master, init_value, n);
        CKL(ctx);
        if (type != ETCU_VOXEL_FLOAT32 && (s = refresh_low_from_master(v.get())) != ETCU_OK) return s;
    } else {
        float* tmp = nullptr;
        if ((s = dalloc(ctx, (void**)&tmp, n * sizeof(float))) != ETCU_OK) return s;
        fill_kernel<<<g, b, 0, ctx->stream>>>(tmp, init_value, n);
        convert_from_float_kernel<__half><<<g, b, 0, ctx->stream>>>(tmp, (__half*)v->low, n);
        cudaStreamSynchronize(ctx->stream);
        dfree(ctx, tmp, n * sizeof(float));
        CKL(ctx);
    }
    *out = v.release();
    return ETCU_OK;
}

extern "C" etcu_status etcu_volume_destroy(etcu_volume* vol) {
    if (!vol) return ETCU_OK;
    etcu_context* ctx = vol->ctx;
    cudaStreamSynchronize(ctx->stream);
    size_t n = voxel_count(vol->desc);
    dfree(ctx, vol->master, n * sizeof(float));
    dfree(ctx, vol->low, n * 2);
    dfree(ctx, vol->mask, n);
    delete vol;
    return ETCU_OK;
}

extern "C" etcu_status etcu_volume_upload(etcu_volume* vol, const float* host) {
    if (!vol || !host) return fail(vol ? vol->ctx : nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    etcu_context* ctx = vol->ctx;
    size_t n = voxel_count(vol->desc);
    etcu_status s;
    if (vol->master) {
        if ((s = upload_host_float(ctx, vol->master, host, n)) != ETCU_OK) return s;
        if (vol->type != ETCU_VOXEL_FLOAT32) return refresh_low_from_master(vol);
        return ETCU_OK;
    }
    float* tmp = nullptr;
    if ((s = dalloc(ctx, (void**)&tmp, n * sizeof(float))) != ETCU_OK) return s;
    s = upload_host_float(ctx, tmp, host, n);
    if (s == ETCU_OK) {
        dim3 g, b;
        launch_1d_dims(n, g, b);
        convert_from_float_kernel<__half><<<g, b, 0, ctx->stream>>>(tmp, (__half*)vol->low, n);
        cudaStreamSynchronize(ctx->stream);
    }
    dfree(ctx, tmp, n * sizeof(float));
    CKL(ctx);
    return s;
}

extern "C" etcu_status etcu_volume_upload_device(etcu_volume* vol, const float* d_src) {
    if (!vol || !d_src) return fail(vol ? vol->ctx : nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    etcu_context* ctx = vol->ctx;
    if (!vol->master) return fail(ctx, ETCU_ERR_UNSUPPORTED, "device-to-device upload needs an FP32 (master) volume");
    CK(ctx, cudaMemcpyAsync(vol->master, d_src, voxel_count(vol->desc) * sizeof(float), cudaMemcpyDeviceToDevice,
                            ctx->stream));
    if (vol->type != ETCU_VOXEL_FLOAT32) return refresh_low_from_master(vol);
    return ETCU_OK;
}

extern "C" etcu_status etcu_volume_download_device(etcu_volume* vol, float* d_dst) {
    if (!vol || !d_dst) return fail(vol ? vol->ctx : nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    etcu_context* ctx = vol->ctx;
    if (!vol->master) return fail(ctx, ETCU_ERR_UNSUPPORTED, "device-to-device download needs an FP32 (master) volume");
    CK(ctx, cudaMemcpyAsync(d_dst, vol->master, voxel_count(vol->desc) * sizeof(float), cudaMemcpyDeviceToDevice,
                            ctx->stream));
    return ETCU_OK;
}

extern "C" etcu_status etcu_volume_download(etcu_volume* vol, float* host) {
    if (!vol || !host) return fail(vol ? vol->ctx : nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    etcu_context* ctx = vol->ctx;
    size_t n = voxel_count(vol->desc);
    if (vol->master) {
        CK(ctx, cudaMemcpyAsync(host, vol->master, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
        CK(ctx, cudaStreamSynchronize(ctx->stream));
        return ETCU_OK;
    }
    float* tmp = nullptr;
    etcu_status s;
    if ((s = dalloc(ctx, (void**)&tmp, n * sizeof(float))) != ETCU_OK) return s;
    dim3 g, b;
    launch_1d_dims(n, g, b);
    convert_to_float_kernel<__half><<<g, b, 0, ctx->stream>>>((const __half*)vol->low, tmp, n);
    cudaError_t e = cudaMemcpyAsync(host, tmp, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    dfree(ctx, tmp, n * sizeof(float));
    CK(ctx, e);
    CKL(ctx);
    return ETCU_OK;
}

extern "C" etcu_status etcu_volume_set_mask(etcu_volume* vol, const uint8_t* host_mask) {
    if (!vol) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL volume");
    etcu_context* ctx = vol->ctx;
    size_t n = voxel_count(vol->desc);
    if (!host_mask) {
        cudaStreamSynchronize(ctx->stream);
        dfree(ctx, vol->mask, n);
        vol->mask = nullptr;
        return ETCU_OK;
    }
    etcu_status s;
    if (!vol->mask && (s = dalloc(ctx, (void**)&vol->mask, n)) != ETCU_OK) return s;
    CK(ctx, cudaMemcpyAsync(vol->mask, host_mask, n, cudaMemcpyHostToDevice, ctx->stream));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    return ETCU_OK;
}

extern "C" void* etcu_volume_device_ptr(etcu_volume* vol) {
    if (!vol) return nullptr;
    return vol->master ? (void*)vol->master : vol->low;
}

extern "C" etcu_status etcu_volume_set_intensity_clamp(etcu_volume* vol, int use_min, float vmin, int use_max,
                                                       float vmax) {
    if (!vol) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL volume");
    vol->use_min = use_min;
    vol->vmin = vmin;
    vol->use_max = use_max;
    vol->vmax = vmax;
    return ETCU_OK;
}

// =============================================================== operators
extern "C" etcu_status etcu_forward_project(etcu_volume* vol, const etcu_view* view, uint32_t subvolume,
                                            uint32_t samples, float* d_virtual, float* d_traversal) {
    if (!vol) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL volume");
    etcu_context* ctx = vol->ctx;
    etcu_status s;
    if ((s = check_view(ctx, view)) != ETCU_OK) return s;
    if (!d_virtual ^ !d_traversal)
        return fail(ctx, ETCU_ERR_INVALID_ARGUMENT,
                    "Virtual projection and traversal length must either be set both or none of them!");
    if (!d_virtual)
        return fail(ctx, ETCU_ERR_STATE,
                    "ForwardProjectionKernel cannot be run without setting output images! Be sure to call setOutput() "
                    "before with non-null parameters.");
    if (subvolume >= vol->slabs.size())
        return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "Tried to get resolution of subvolume %u while there are only %zu!",
                    subvolume, vol->slabs.size());
    const SlabConst& slab = vol->slabs[subvolume];
    FpArgs a{};
    fill_fp_volume_ptrs(vol, slab, a);
    a.slab = slab;
    a.views = nullptr;
    a.inline_view = make_view_const(*view, slab, 0.f);
    a.order = nullptr;
    a.first = 0;
    a.W = (int)view->width;
    a.H = (int)view->height;
    a.samples = samples == 0 ? 1 : (int)samples;  // ForwardProjectionKernel.cpp:65-68
    a.mode = kFpSeparateAccumulate;
    a.out_v = d_virtual;
    a.out_l = d_traversal;
    launch_fp(vol, a, fp_path(view->perspective != 0, a.inline_view.fast2d != 0, slab), 1, ctx->stream);
    CKL(ctx);
    return ETCU_OK;
}

namespace {
etcu_status bp_one_slab(etcu_volume* vol, const etcu_view* view, const SlabConst& slab, uint32_t samples,
                        float lambda_eff, const float4* pattern, etcu_sampling sampling) {
    etcu_context* ctx = vol->ctx;
    BpArgs a{};
    fill_bp_volume_ptrs(vol, slab, a);
    a.slab = slab;
    a.views = nullptr;
    a.inline_view = make_view_const(*view, slab, 0.f);
    a.order = nullptr;
    a.first = 0;
    a.nviews = 1;
    a.texs = nullptr;
    a.inline_tex = ctx->pair_tex;
    a.rl = ctx->pair;
    a.rl_pitch = ctx->pair_pitch;
    a.rl_slot = 0;
    a.W = (int)view->width;
    a.H = (int)view->height;
    a.lambda = lambda_eff;
    a.samples = nullptr;
    if (!view->perspective) {
        a.nsamples = (int)samples;
        for (uint32_t k = 0; k < samples; ++k) a.inline_samples[k] = pattern[k];
    } else {
        a.nsamples = 0;
        uint32_t res[3] = {(uint32_t)slab.rx, (uint32_t)slab.ry, (uint32_t)slab.rz};
        a.persp_n = (int)perspective_sampling_factor(view->width, view->height, res, samples);
    }
    a.use_min = vol->use_min;
    a.use_max = vol->use_max;
    a.vmin = vol->vmin;
    a.vmax = vol->vmax;
    launch_bp(vol, a, view->perspective != 0, sampling, ctx->stream, row_constant(a.inline_view), &a.inline_view,
              &a.inline_samples[0]);
    CKL(ctx);
    return ETCU_OK;
}
}  // namespace

extern "C" etcu_status etcu_back_project(etcu_volume* vol, const etcu_view* view, uint32_t subvolume,
                                         uint32_t samples, float lambda, uint32_t block_size, const float* d_residual,
                                         const float* d_traversal, etcu_sampling sampling) {
    if (!vol) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL volume");
    etcu_context* ctx = vol->ctx;
    etcu_status s;
    if ((s = check_view(ctx, view)) != ETCU_OK) return s;
    if (!d_residual ^ !d_traversal)
        return fail(ctx, ETCU_ERR_INVALID_ARGUMENT,
                    "Either residual and traversalLength images must be provided both or none of them!");
    if (!d_residual)
        return fail(ctx, ETCU_ERR_STATE,
                    "Residual and traversalLength images must both be provided via SetInput() before kernel launch!");
    if (block_size == 0) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "Illegal ProjectionBlockSize!");
    if (subvolume != ETCU_ALL_SUBVOLUMES && subvolume >= vol->slabs.size())
        return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "Tried to get resolution of subvolume %u while there are only %zu!",
                    subvolume, vol->slabs.size());
    std::vector<float> pattern;
    if (!view->perspective) {
        float vs[3] = {vol->slabs[0].vs.x, vol->slabs[0].vs.y, vol->slabs[0].vs.z};
        pattern.resize(4 * (size_t)std::max(samples, 1u));
        std::string err;
        if (!sample_pattern(*view, vs, samples, pattern.data(), &err))
            return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "%s", err.c_str());
        if (samples > (uint32_t)kMaxInlineSamples)
            return fail(ctx, ETCU_ERR_UNSUPPORTED, "at most %d back-projection samples per voxel", kMaxInlineSamples);
    }
    if ((s = ensure_pair_scratch(ctx, view->width, view->height)) != ETCU_OK) return s;
    dim3 b(128), g((view->width + 127) / 128, view->height);
    pack_pair_kernel<<<g, b, 0, ctx->stream>>>(d_residual, d_traversal, ctx->pair, ctx->pair_pitch, (int)view->width,
                                               (int)view->height);
    CKL(ctx);
    const float lam = lambda / (float)block_size;  // BackProjectionKernel.cpp:94
    const float4* pat = (const float4*)pattern.data();
    if (subvolume == ETCU_ALL_SUBVOLUMES) {  // BackProjectionOperator.cpp:43-57
        for (const SlabConst& sl : vol->slabs)
            if ((s = bp_one_slab(vol, view, sl, samples, lam, pat, sampling)) != ETCU_OK) return s;
    } else if ((s = bp_one_slab(vol, view, vol->slabs[subvolume], samples, lam, pat, sampling)) != ETCU_OK) {
        return s;
    }
    if (vol->type == ETCU_VOXEL_F16_MASTER || vol->type == ETCU_VOXEL_BF16_MASTER) {
        // the kernel already wrote the shadow of every updated voxel
    }
    return ETCU_OK;
}

extern "C" etcu_status etcu_compare(etcu_context* ctx, const float* d_real, const float* d_virtual,
                                    float* d_residual, size_t n) {
    if (!ctx || !d_real || !d_virtual || !d_residual) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n == 0) return ETCU_OK;
    dim3 g, b;
    launch_1d_dims(n, g, b);
    compare_kernel<<<g, b, 0, ctx->stream>>>(d_real, d_virtual, d_residual, n);
    CKL(ctx);
    return ETCU_OK;
}

extern "C" etcu_status etcu_long_object_compensation(etcu_context* ctx, float* d_virtual, float* d_traversal,
                                                     float constant_length, size_t n) {
    if (!ctx || !d_virtual || !d_traversal) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n == 0) return ETCU_OK;
    dim3 g, b;
    launch_1d_dims(n, g, b);
    loc_kernel<<<g, b, 0, ctx->stream>>>(d_virtual, d_traversal, constant_length, n);
    CKL(ctx);
    return ETCU_OK;
}

extern "C" etcu_status etcu_compute_ray_length(etcu_volume* vol, const etcu_view* view, float* d_out) {
    if (!vol || !d_out) return fail(vol ? vol->ctx : nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    etcu_context* ctx = vol->ctx;
    etcu_status s;
    if ((s = check_view(ctx, view)) != ETCU_OK) return s;
    ViewConst vc = make_view_const(*view, vol->slabs[0], 0.f);
    dim3 b(128), g((view->width + 127) / 128, view->height);
    ray_length_kernel<<<g, b, 0, ctx->stream>>>(vc, vol->slabs[0], (int)view->width, (int)view->height, d_out);
    CKL(ctx);
    return ETCU_OK;
}

// =============================================================== reconstruction
namespace {

size_t proj_elem_bytes(int kind) { return kind == ETCU_PROJ_F32 ? sizeof(float) : 2; }

// The tilt series (n floats, from the host or the device) in the given storage: FP32
// copied as is (or, from the device, used in place when `in_place`), FP16 / BF16 rounded
// to nearest on the device.  *out receives the buffer (allocated with alloc), *owned
// whether it must be freed.
template <typename Alloc>
etcu_status stage_projections(etcu_context* ctx, const float* host, const float* dev, size_t n, int kind,
                              bool in_place, Alloc alloc, float** out, bool* owned) {
    *owned = false;
    if (kind != ETCU_PROJ_F32 && kind != ETCU_PROJ_F16 && kind != ETCU_PROJ_BF16)
        return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "unknown projection storage %d", kind);
    if (kind == ETCU_PROJ_F32 && dev && in_place) {
        *out = const_cast<float*>(dev);
        return ETCU_OK;
    }
    etcu_status s;
    void* buf = nullptr;
    if ((s = alloc(&buf, n * proj_elem_bytes(kind))) != ETCU_OK) return s;
    *owned = true;
    *out = (float*)buf;
    if (kind == ETCU_PROJ_F32) {
        CK(ctx, cudaMemcpyAsync(buf, host ? (const void*)host : (const void*)dev, n * sizeof(float),
                                host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, ctx->stream));
        return ETCU_OK;
    }
    const float* src = dev;
    float* tmp = nullptr;
    if (host) {
        if ((s = dalloc(ctx, (void**)&tmp, n * sizeof(float))) != ETCU_OK) return s;
        CK(ctx, cudaMemcpyAsync(tmp, host, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
        src = tmp;
    }
    dim3 g, b;
    launch_1d_dims(n, g, b);
    if (kind == ETCU_PROJ_F16)
        convert_from_float_kernel<__half><<<g, b, 0, ctx->stream>>>(src, (__half*)buf, n);
    else
        convert_from_float_kernel<__nv_bfloat16><<<g, b, 0, ctx->stream>>>(src, (__nv_bfloat16*)buf, n);
    CKL(ctx);
    if (tmp) {
        CK(ctx, cudaStreamSynchronize(ctx->stream));
        dfree(ctx, tmp, n * sizeof(float));
    }
    return ETCU_OK;
}

void recon_free(etcu_recon* r) {
    etcu_context* ctx = r->ctx;
    cudaStreamSynchronize(ctx->stream);
    if (r->exec) cudaGraphExecDestroy(r->exec);
    if (r->graph) cudaGraphDestroy(r->graph);
    for (auto t : r->texs) cudaDestroyTextureObject(t);
    size_t N = r->n_input;
    if (r->own_proj) dfree(ctx, r->d_proj, N * (size_t)r->W * r->H * proj_elem_bytes(r->proj_kind));
    dfree(ctx, r->d_views, N * sizeof(ViewConst) * r->vol->slabs.size());
    dfree(ctx, r->d_order, r->order.size() * sizeof(uint32_t));
    dfree(ctx, r->d_samples, N * r->nsamples * sizeof(float4));
    dfree(ctx, r->rl_raw, r->rl_slot * r->slots * sizeof(float2) + ctx->tex_align);
    dfree(ctx, r->d_texs, r->slots * sizeof(cudaTextureObject_t));
    dfree(ctx, r->d_resid, sizeof(double));
    const size_t ry = r->vol->slabs.empty() ? 0 : r->vol->slabs[0].ry;
    dfree(ctx, r->d_jrange, (size_t)r->n_input * ry * sizeof(int2));
    dfree(ctx, r->d_tapwin, (size_t)r->n_input * sizeof(int2));
    dfree(ctx, r->d_fuse_ctl, (ry + 2) * sizeof(uint32_t));
}

// Forward projection of `count` views starting at order position `first`
// into slots 0..count-1: every slab in turn, the first overwriting and the
// last writing (residual, length) plus the FP64 sum of residual^2.
uint32_t issue_forward(etcu_recon* r, uint32_t first, uint32_t count, cudaStream_t st) {
    etcu_volume* vol = r->vol;
    const uint32_t S = (uint32_t)vol->slabs.size();
    for (uint32_t s = 0; s < S; ++s) {
        const SlabConst& slab = vol->slabs[s];
        FpArgs a{};
        fill_fp_volume_ptrs(vol, slab, a);
        a.slab = slab;
        a.views = r->d_views + (size_t)s * r->n_input;
        a.order = r->d_order;
        a.first = first;
        a.W = (int)r->W;
        a.H = (int)r->H;
        a.samples = r->params.fp_samples == 0 ? 1 : (int)r->params.fp_samples;
        a.mode = (s == S - 1) ? kFpPairResidual : kFpPairAccumulate;
        a.overwrite = (s == 0) ? 1 : 0;
        a.loc = r->params.use_long_object_compensation ? 1 : 0;
        a.rl = r->rl;
        a.rl_pitch = r->rl_pitch;
        a.rl_slot = r->rl_slot;
        a.real = r->d_proj;
        a.real_kind = r->proj_kind;
        a.resid_sq = r->d_resid;
        launch_fp(vol, a, r->fp_paths[s], count, st);
    }
    return S;
}

// Back projection of the block's views, slabs in reverse order
// (BlockIterativeReconstructionOperator.cpp:130-142), lambda / blockSize.
uint32_t issue_backward(etcu_recon* r, uint32_t first, uint32_t count, cudaStream_t st,
                        const float2* rl = nullptr) {
    etcu_volume* vol = r->vol;
    const uint32_t S = (uint32_t)vol->slabs.size();
    uint32_t n = 0;
    for (int s = (int)S - 1; s >= 0; --s) {
        const SlabConst& slab = vol->slabs[s];
        BpArgs a{};
        fill_bp_volume_ptrs(vol, slab, a);
        a.slab = slab;
        a.views = r->d_views + (size_t)s * r->n_input;
        a.order = r->d_order;
        a.first = first;
        a.nviews = (int)count;
        a.texs = r->d_texs;
        a.rl = rl ? rl : r->rl;
        a.rl_pitch = r->rl_pitch;
        a.rl_slot = r->rl_slot;
        a.W = (int)r->W;
        a.H = (int)r->H;
        a.lambda = r->params.lambda / (float)count;  // BackProjectionKernel.cpp:94
        a.samples = r->d_samples;
        a.nsamples = (int)r->nsamples;
        uint32_t res[3] = {(uint32_t)slab.rx, (uint32_t)slab.ry, (uint32_t)slab.rz};
        a.persp_n = (int)perspective_sampling_factor(r->W, r->H, res, r->params.bp_samples);
        a.use_min = vol->use_min;
        a.use_max = vol->use_max;
        a.vmin = vol->vmin;
        a.vmax = vol->vmax;
        const uint32_t vid = r->order[first];
        n += launch_bp(vol, a, r->persp, r->params.sampling, st, count == 1 && r->row_const[vid],
                       &r->hvc[(size_t)s * r->n_input + vid],
                       r->hsamples.empty() ? nullptr : &r->hsamples[(size_t)vid * r->nsamples]);
    }
    return n;
}

// SART with the fused step: FP of the first view into slot 0, then for every order
// position p the fused BP(p) + FP(p + 1) (slots alternate), then the BP of the last
// view.  Same operations in the same order as the unfused sequence.
void launch_fused_step(etcu_recon* r, uint32_t p, cudaStream_t st, const float2* rl_in = nullptr,
                       float* part = nullptr) {
    etcu_volume* vol = r->vol;
    const SlabConst& g = vol->slabs[0];
    const uint32_t vb = r->order[p];
    FuseArgs a{};
    a.vol = vol->master;
    a.slab = g;
    a.views = r->d_views;
    a.order = r->d_order;
    a.p = p;
    a.samples = r->d_samples;
    a.rl_in = rl_in ? rl_in : r->rl + (size_t)(p & 1) * r->rl_slot;
    a.rl_out = r->rl + (size_t)((p + 1) & 1) * r->rl_slot;
    a.rl_pitch = r->rl_pitch;
    a.W = (int)r->W;
    a.H = (int)r->H;
    a.lambda = r->params.lambda;  // block size 1
    a.x0lo = r->fuse_x0lo[vb];
    a.ntaps = r->fuse_ntaps[vb];
    a.jrange = r->d_jrange;
    a.real = r->d_proj;
    a.real_kind = r->proj_kind;
    a.resid_sq = part ? nullptr : r->d_resid;
    a.loc = r->params.use_long_object_compensation ? 1 : 0;
    a.part = part;
    const size_t smem = fuse_smem_bytes(g.rx, g.rz, a.ntaps);
    switch (vol->type) {
    case ETCU_VOXEL_F16_MASTER: sart_fused_kernel<1><<<g.ry, kFuseThreads, smem, st>>>(a); break;
    case ETCU_VOXEL_BF16_MASTER: sart_fused_kernel<2><<<g.ry, kFuseThreads, smem, st>>>(a); break;
    default: sart_fused_kernel<0><<<g.ry, kFuseThreads, smem, st>>>(a); break;
    }
}

// All M - 1 fused steps in one launch; the row counters are cleared first.
void launch_fused_persistent(etcu_recon* r, cudaStream_t st) {
    etcu_volume* vol = r->vol;
    const SlabConst& g = vol->slabs[0];
    const uint32_t M = (uint32_t)r->order.size();
    cudaMemsetAsync(r->d_fuse_ctl, 0, ((size_t)g.ry + 1) * sizeof(uint32_t), st);
    FuseArgs a{};
    a.vol = vol->master;
    a.slab = g;
    a.views = r->d_views;
    a.order = r->d_order;
    a.samples = r->d_samples;
    a.rl_pitch = r->rl_pitch;
    a.W = (int)r->W;
    a.H = (int)r->H;
    a.lambda = r->params.lambda;
    a.jrange = r->d_jrange;
    a.real = r->d_proj;
    a.real_kind = r->proj_kind;
    a.resid_sq = r->d_resid;
    a.loc = r->params.use_long_object_compensation ? 1 : 0;
    FusePersist q{};
    q.tapwin = r->d_tapwin;
    q.rl0 = r->rl;
    q.rl_slot = r->rl_slot;
    q.steps = M - 1;
    q.ctl = r->d_fuse_ctl;
    q.error = r->d_fuse_ctl + g.ry + 1;
    q.window = r->fuse_window;
    q.withhold_row = r->ctx->fuse_withhold_row;
    switch (vol->type) {
    case ETCU_VOXEL_F16_MASTER:
        sart_fused_persistent_kernel<1><<<r->fuse_grid, kFuseThreads, r->fuse_smem, st>>>(a, q);
        break;
    case ETCU_VOXEL_BF16_MASTER:
        sart_fused_persistent_kernel<2><<<r->fuse_grid, kFuseThreads, r->fuse_smem, st>>>(a, q);
        break;
    default: sart_fused_persistent_kernel<0><<<r->fuse_grid, kFuseThreads, r->fuse_smem, st>>>(a, q); break;
    }
}

uint32_t issue_fused_iteration(etcu_recon* r, cudaStream_t st) {
    const uint32_t M = (uint32_t)r->order.size();
    uint32_t n = issue_forward(r, 0, 1, st);
    if (r->fuse_persist) {
        launch_fused_persistent(r, st);
        ++n;
    } else {
        for (uint32_t p = 0; p + 1 < M; ++p) {
            launch_fused_step(r, p, st);
            ++n;
        }
    }
    // the last view's back projection reads the slot its FP wrote
    const uint32_t last = M - 1;
    n += issue_backward(r, last, 1, st, r->rl + (size_t)(last & 1) * r->rl_slot);
    return n;
}

void fuse_limits(int dev, size_t smem, int& per_sm, int& persist_per_sm, int& sms) {
    static std::mutex mu;
    static std::vector<char> opted;
    // two attributes, not cudaGetDeviceProperties (milliseconds per call, once per reconstruction)
    int optin = 0, nsm = 0;
    const bool have_prop = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess &&
                           cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess;
    if (!have_prop) cudaGetLastError();
    {
        std::lock_guard<std::mutex> lock(mu);
        if ((int)opted.size() <= dev) opted.resize(dev + 1, 0);
        if (!opted[dev]) {
            if (have_prop) {
                const int full = optin, persist = full - 16;
                cudaFuncSetAttribute(sart_fused_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, full);
                cudaFuncSetAttribute(sart_fused_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, full);
                cudaFuncSetAttribute(sart_fused_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, full);
                cudaFuncSetAttribute(sart_fused_persistent_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     persist);
                cudaFuncSetAttribute(sart_fused_persistent_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     persist);
                cudaFuncSetAttribute(sart_fused_persistent_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     persist);
            }
            cudaGetLastError();
            opted[dev] = 1;
        }
    }
    sms = have_prop ? nsm : 0;
    per_sm = persist_per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sart_fused_kernel<0>, kFuseThreads, smem) !=
        cudaSuccess) {
        cudaGetLastError();
        per_sm = 0;
    }
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&persist_per_sm, sart_fused_persistent_kernel<0>, kFuseThreads,
                                                      smem) != cudaSuccess) {
        cudaGetLastError();
        persist_per_sm = 0;
    }
}

constexpr int kFuseMaxWindow = 16;

// Dependency window of the persistent fused steps: the largest distance between a volume
// row and a row that owns (under any view) one of the two detector rows the row's back
// projection samples (under any view).  Covers both the residual a step reads (written
// by the owners in the step before) and the residual slot it overwrites (read by the
// samplers two steps before).  window = -1 when it exceeds kFuseMaxWindow.
etcu_status fuse_window_of(etcu_context* ctx, const ViewConst* d_views, const float4* d_samples, const SlabConst& g,
                           uint32_t N, uint32_t height, const std::vector<int2>& jrange, int& window) {
    const int H = (int)height;
    const size_t T = (size_t)N * g.ry;
    int* d_y0 = nullptr;
    etcu_status s;
    if ((s = dalloc(ctx, (void**)&d_y0, T * sizeof(int))) != ETCU_OK) return s;
    std::vector<int> y0(T);
    fuse_bp_rows_kernel<<<dim3((g.ry + 127) / 128, N), 128, 0, ctx->stream>>>(d_views, d_samples, g, H, d_y0);
    cudaMemcpyAsync(y0.data(), d_y0, T * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    const cudaError_t e = cudaStreamSynchronize(ctx->stream);
    dfree(ctx, d_y0, T * sizeof(int));
    CK(ctx, e);
    std::vector<int> omin(H, INT32_MAX), omax(H, -1);
    for (uint32_t v = 0; v < N; ++v)
        for (int y = 0; y < g.ry; ++y) {
            const int2 jr = jrange[(size_t)v * g.ry + y];
            for (int j = jr.x; j < jr.y; ++j) {
                omin[j] = std::min(omin[j], y);
                omax[j] = std::max(omax[j], y);
            }
        }
    window = 0;
    for (uint32_t v = 0; v < N; ++v)
        for (int y = 0; y < g.ry; ++y)
            for (int j = y0[(size_t)v * g.ry + y]; j <= y0[(size_t)v * g.ry + y] + 1; ++j) {
                if (j < 0 || j >= H || omax[j] < 0) continue;  // padding, or a row no ray writes
                window = std::max(window, std::max(std::abs(omin[j] - y), std::abs(omax[j] - y)));
                if (window > kFuseMaxWindow) {
                    window = -1;
                    return ETCU_OK;
                }
            }
    return ETCU_OK;
}

etcu_status fuse_window(etcu_recon* r, const std::vector<int2>& jrange, int& window) {
    return fuse_window_of(r->ctx, r->d_views, r->d_samples, r->vol->slabs[0], r->n_input, r->H, jrange, window);
}

// The (view, volume row) -> detector rows table of the fused steps (fuse_rows_kernel
// evaluates dda_setup's row assignment on the device); ok = false when some volume row
// has more than kFuseRays * kFuseThreads rays.
etcu_status fuse_row_table(etcu_context* ctx, const ViewConst* d_views, const SlabConst& g, uint32_t N, uint32_t W,
                           uint32_t H, std::vector<int2>& table, bool& ok) {
    ok = false;
    const size_t T = (size_t)N * (size_t)g.ry;
    int *jb = nullptr, *je = nullptr;
    etcu_status s;
    if ((s = dalloc(ctx, (void**)&jb, T * sizeof(int))) != ETCU_OK) return s;
    if ((s = dalloc(ctx, (void**)&je, T * sizeof(int))) != ETCU_OK) {
        dfree(ctx, jb, T * sizeof(int));
        return s;
    }
    std::vector<int> hb(T), he(T);
    cudaMemsetAsync(jb, 0x7f, T * sizeof(int), ctx->stream);
    cudaMemsetAsync(je, 0, T * sizeof(int), ctx->stream);
    fuse_rows_kernel<<<dim3((H + 127) / 128, N), 128, 0, ctx->stream>>>(d_views, g, (int)H, jb, je);
    cudaMemcpyAsync(hb.data(), jb, T * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    cudaMemcpyAsync(he.data(), je, T * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    const cudaError_t e = cudaStreamSynchronize(ctx->stream);
    dfree(ctx, jb, T * sizeof(int));
    dfree(ctx, je, T * sizeof(int));
    CK(ctx, e);
    table.assign(T, make_int2(0, 0));
    for (size_t i = 0; i < T; ++i) {
        const int b = hb[i], n = he[i] > b ? he[i] - b : 0;
        if ((long long)n * W > (long long)kFuseRays * kFuseThreads) return ETCU_OK;
        table[i] = make_int2(n ? b : 0, n ? he[i] : 0);
    }
    ok = true;
    return ETCU_OK;
}

// Whether every SART step of this reconstruction can run fused (sart_fused_kernel):
// SART on one sub-volume (FP32, or an FP32 master with a 16-bit shadow) without mask,
// one sample each way, 1/256 sampling,
// parallel views tilted about y (ray.y == 0, hpitch.y == 0, detector row constant
// in y), x rows of an even number of at most 2 * kFuseThreads voxels, walks that
// cannot reach the step cap, at most kFuseRays * kFuseThreads rays per volume row,
// and a tap window per view (plan_bp_col).  Builds the per-view tap windows and the
// (view, volume row) -> detector rows table.
etcu_status plan_fused(etcu_recon* r, const std::vector<ViewConst>& vc, bool& ok) {
    ok = false;
    etcu_volume* vol = r->vol;
    etcu_context* ctx = r->ctx;
    const uint32_t N = r->n_input;
    if (!ctx->fused_step || r->persp || vol->slabs.size() != 1 || r->block != 1 || r->order.size() < 2) return ETCU_OK;
    // FP32 volumes, and FP32 masters with a 16-bit shadow (the fused walk reads the chunk
    // rounded as the shadow holds it; the shadow is written by the last back projection)
    if (vol->type == ETCU_VOXEL_HALF16 || vol->mask || r->params.sampling != ETCU_SAMPLING_Q8) return ETCU_OK;
    if (r->params.fp_samples > 1 || r->params.bp_samples != 1 || r->hsamples.size() < N) return ETCU_OK;
    const SlabConst& g = vol->slabs[0];
    if (g.rx % 2 != 0 || g.rx > 2 * kFuseThreads || g.rx + g.rz - 1 > kMaxDdaIterations) return ETCU_OK;
    std::vector<int> x0lo(N), ntaps(N);
    size_t smem = 0;
    for (uint32_t v = 0; v < N; ++v) {
        const ViewConst& c = vc[v];
        if (!c.fast2d || !row_constant(c) || c.hpitch.y != 0.f) return ETCU_OK;
        BpColPlan plan;
        if (!plan_bp_col(vol, g, c, r->hsamples[v], plan)) return ETCU_OK;
        x0lo[v] = plan.x0lo;
        ntaps[v] = plan.ntaps;
        smem = std::max(smem, fuse_smem_bytes(g.rx, g.rz, plan.ntaps));
    }
    int per_sm = 0, persist_per_sm = 0, sms = 0;
    fuse_limits(ctx->device, smem, per_sm, persist_per_sm, sms);
    if (per_sm < 1) return ETCU_OK;
    // detector rows of every (view, volume row)
    const size_t T = (size_t)N * (size_t)g.ry;
    std::vector<int2> table;
    bool rows_ok = false;
    etcu_status s;
    if ((s = fuse_row_table(ctx, r->d_views, g, N, r->W, r->H, table, rows_ok)) != ETCU_OK) return s;
    if (!rows_ok) return ETCU_OK;
    if ((s = dalloc(ctx, (void**)&r->d_jrange, T * sizeof(int2))) != ETCU_OK) return s;
    CK(ctx, cudaMemcpyAsync(r->d_jrange, table.data(), T * sizeof(int2), cudaMemcpyHostToDevice, ctx->stream));
    r->fuse_smem = smem;
    ok = true;
    if (ctx->fused_persist && persist_per_sm >= 1 && sms > 0) {
        int window = 0;
        if ((s = fuse_window(r, table, window)) != ETCU_OK) return s;
        if (window >= 0 && window <= kFuseMaxWindow) {
            std::vector<int2> tw(N);
            for (uint32_t v = 0; v < N; ++v) tw[v] = make_int2(x0lo[v], ntaps[v]);
            if ((s = dalloc(ctx, (void**)&r->d_tapwin, N * sizeof(int2))) != ETCU_OK) return s;
            CK(ctx, cudaMemcpyAsync(r->d_tapwin, tw.data(), N * sizeof(int2), cudaMemcpyHostToDevice, ctx->stream));
            if ((s = dalloc(ctx, (void**)&r->d_fuse_ctl, ((size_t)g.ry + 2) * sizeof(uint32_t))) != ETCU_OK) return s;
            CK(ctx, cudaMemsetAsync(r->d_fuse_ctl, 0, ((size_t)g.ry + 2) * sizeof(uint32_t), ctx->stream));
            r->fuse_window = window;
            r->fuse_grid = (int)std::min<long long>((long long)persist_per_sm * sms,
                                                    (long long)(r->order.size() - 1) * g.ry);
            r->fuse_per_sm = persist_per_sm;
            r->fuse_sms = sms;
            r->fuse_persist = true;
        }
    }
    r->fuse_x0lo = std::move(x0lo);
    r->fuse_ntaps = std::move(ntaps);
    return ETCU_OK;
}

etcu_status issue_iteration(etcu_recon* r, cudaStream_t st, uint32_t* launches);

// Autotuner: resident blocks per SM of the persistent fused launch (1 .. the occupancy
// limit), timed on whole iterations of this reconstruction; the volume (master and
// shadow) is saved before and restored after the timing runs.
etcu_status tune_fused_grid(etcu_recon* r) {
    etcu_context* ctx = r->ctx;
    etcu_volume* vol = r->vol;
    const SlabConst& g = vol->slabs[0];
    const long long units = (long long)(r->order.size() - 1) * g.ry;
    char key[512];
    snprintf(key, sizeof(key), "sart_fused_persistent|%dx%dx%d|views%zu|det%ux%u|type%d|%s", g.rx, g.ry, g.rz,
             r->order.size(), r->W, r->H, (int)vol->type, etcu_tune::device_tag(ctx->device).c_str());
    int choice = etcu_tune::lookup(key);
    std::string log;
    if (choice < 1 || choice > r->fuse_per_sm) {
        const size_t n = voxel_count(vol->desc);
        const size_t lowb = vol->low ? n * 2 : 0;
        void* save = nullptr;
        etcu_status s = dalloc(ctx, &save, n * 4 + lowb);
        if (s != ETCU_OK) return s;
        CK(ctx, cudaMemcpyAsync(save, vol->master, n * 4, cudaMemcpyDeviceToDevice, ctx->stream));
        if (lowb) CK(ctx, cudaMemcpyAsync((char*)save + n * 4, vol->low, lowb, cudaMemcpyDeviceToDevice, ctx->stream));
        std::vector<int> cands;
        for (int b = 1; b <= r->fuse_per_sm; ++b) cands.push_back(b);
        choice = etcu_tune::search(ctx->stream, cands, [&](int b) {
            r->fuse_grid = (int)std::min<long long>((long long)b * r->fuse_sms, units);
            return issue_iteration(r, ctx->stream, nullptr) == ETCU_OK;
        }, 2, &log);
        CK(ctx, cudaMemcpyAsync(vol->master, save, n * 4, cudaMemcpyDeviceToDevice, ctx->stream));
        if (lowb) CK(ctx, cudaMemcpyAsync(vol->low, (char*)save + n * 4, lowb, cudaMemcpyDeviceToDevice, ctx->stream));
        CK(ctx, cudaStreamSynchronize(ctx->stream));
        dfree(ctx, save, n * 4 + lowb);
        if (choice < 1) choice = r->fuse_per_sm;
        etcu_tune::store(key, choice);
    } else {
        log = " cached";
    }
    r->fuse_grid = (int)std::min<long long>((long long)choice * r->fuse_sms, units);
    ctx->tune_log += std::string(key) + " " + std::to_string(choice) + log + "\n";
    CK(ctx, cudaMemsetAsync(r->d_resid, 0, sizeof(double), ctx->stream));
    return check_fused_waits(r);
}

// One iteration (BlockIterativeReconstructionOperator.cpp:92-103).
etcu_status issue_iteration(etcu_recon* r, cudaStream_t st, uint32_t* launches) {
    etcu_context* ctx = r->ctx;
    const uint32_t M = (uint32_t)r->order.size();
    uint32_t n = 0;
    CK(ctx, cudaMemsetAsync(r->d_resid, 0, sizeof(double), st));
    if (r->fused) {
        n = issue_fused_iteration(r, st);
        CKL(ctx);
        if (launches) *launches = n;
        return ETCU_OK;
    }
    for (uint32_t b = 0; b < r->nblocks; ++b) {
        const uint32_t first = b * r->block;
        const uint32_t bs = (b < r->nblocks - 1) ? r->block : M - first;  // BlockIterativeProjectionAccess.cpp:55-70
        n += issue_forward(r, first, bs, st);
        n += issue_backward(r, first, bs, st);
    }
    CKL(ctx);
    if (launches) *launches = n;
    return ETCU_OK;
}

etcu_status recon_build(etcu_volume* vol, const etcu_view* views, uint32_t n_views, const float* host_proj,
                        const float* dev_proj, const etcu_recon_params* params, etcu_recon** out) {
    etcu_context* ctx = vol ? vol->ctx : nullptr;
    if (!vol || !views || !params || !out || (!host_proj && !dev_proj))
        return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    if (n_views == 0) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "No projections given!");
    if (params->block_size == 0) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "Illegal ProjectionBlockSize!");
    if ((int)params->order < 0 || (int)params->order > 3)
        return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "Illegal ProjectionSetType!");
    const uint32_t W = views[0].width, H = views[0].height;
    const bool persp = views[0].perspective != 0;
    for (uint32_t i = 0; i < n_views; ++i) {
        etcu_status s = check_view(ctx, &views[i]);
        if (s != ETCU_OK) return s;
        if (views[i].width != W || views[i].height != H)
            return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "all projections must share one resolution");
        if ((views[i].perspective != 0) != persp)
            return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "all projections must share one beam geometry");
    }
    if (persp && params->use_long_object_compensation)
        return fail(ctx, ETCU_ERR_INVALID_ARGUMENT,
                    "Calculation of traversal length is only supported for parallel scanner geometry!");
    std::unique_ptr<etcu_recon, void (*)(etcu_recon*)> r(new etcu_recon(), [](etcu_recon* p) {
        recon_free(p);
        delete p;
    });
    r->vol = vol;
    r->ctx = ctx;
    r->params = *params;
    r->n_input = n_views;
    r->W = W;
    r->H = H;
    r->persp = persp;
    r->order = projection_order(params->order, n_views, params->skip, params->skip ? params->skip_count : 0);
    const uint32_t M = (uint32_t)r->order.size();
    if (M == 0) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "After applying SkipProjectionList no projections are left!");
    r->block = params->block_size == ETCU_BLOCK_ALL ? M : std::min(params->block_size, M);
    r->nblocks = (M + r->block - 1) / r->block;  // BlockIterativeProjectionAccess.cpp:46
    r->slots = r->block;
    etcu_status s;
    const size_t P = (size_t)W * H;
    // tilt series, device-resident for the whole reconstruction (FP32 device input is used in place)
    r->proj_kind = params->projection_storage;
    if ((s = stage_projections(ctx, host_proj, dev_proj, P * n_views, r->proj_kind, true,
                               [&](void** p, size_t bytes) { return dalloc(ctx, p, bytes); }, &r->d_proj,
                               &r->own_proj)) != ETCU_OK)
        return s;
    // view constants per slab (fast-path flags depend on the voxel size)
    const size_t S = vol->slabs.size();
    std::vector<ViewConst> vc(S * n_views);
    for (size_t sl = 0; sl < S; ++sl)
        for (uint32_t i = 0; i < n_views; ++i) {
            float loc = 0.f;
            if (params->use_long_object_compensation)
                loc = traversal_length(views[i], vol->desc.bbox_min, vol->desc.bbox_max);
            vc[sl * n_views + i] = make_view_const(views[i], vol->slabs[sl], loc);
        }
    r->hvc = vc;
    r->hviews.assign(views, views + n_views);
    r->row_const.resize(n_views);
    for (uint32_t i = 0; i < n_views; ++i) r->row_const[i] = row_constant(vc[i]) ? 1 : 0;
    r->fp_paths.resize(S);
    for (size_t sl = 0; sl < S; ++sl) {
        bool all = true;
        for (uint32_t i = 0; i < n_views; ++i) all &= vc[sl * n_views + i].fast2d != 0;
        r->fp_paths[sl] = fp_path(persp, all, vol->slabs[sl]);
    }
    if ((s = dalloc(ctx, (void**)&r->d_views, vc.size() * sizeof(ViewConst))) != ETCU_OK) return s;
    CK(ctx, cudaMemcpyAsync(r->d_views, vc.data(), vc.size() * sizeof(ViewConst), cudaMemcpyHostToDevice, ctx->stream));
    if ((s = dalloc(ctx, (void**)&r->d_order, M * sizeof(uint32_t))) != ETCU_OK) return s;
    CK(ctx, cudaMemcpyAsync(r->d_order, r->order.data(), M * sizeof(uint32_t), cudaMemcpyHostToDevice, ctx->stream));
    // back-projection sample patterns
    if (!persp) {
        r->nsamples = params->bp_samples;
        std::vector<float> pat(4 * (size_t)std::max(1u, params->bp_samples) * n_views);
        float vs[3] = {vol->slabs[0].vs.x, vol->slabs[0].vs.y, vol->slabs[0].vs.z};
        for (uint32_t i = 0; i < n_views; ++i) {
            std::string err;
            if (!sample_pattern(views[i], vs, params->bp_samples, pat.data() + 4 * (size_t)params->bp_samples * i, &err))
                return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "%s", err.c_str());
        }
        if (params->bp_samples > 0) {
            r->hsamples.resize(pat.size() / 4);
            std::memcpy(r->hsamples.data(), pat.data(), pat.size() * sizeof(float));
        }
        if ((s = dalloc(ctx, (void**)&r->d_samples, pat.size() * sizeof(float))) != ETCU_OK) return s;
        CK(ctx, cudaMemcpyAsync(r->d_samples, pat.data(), pat.size() * sizeof(float), cudaMemcpyHostToDevice,
                                ctx->stream));
    } else {
        r->nsamples = 0;
    }
    {
        bool fused = false;
        if ((s = plan_fused(r.get(), vc, fused)) != ETCU_OK) return s;
        r->fused = fused;
        if (fused) r->slots = std::max<uint32_t>(r->slots, 2);  // the fused steps alternate two images
    }
    // per-slot interleaved (residual, length) images, padded by kPad zero texels, and
    // their textures (texture-unit sampling mode)
    const size_t pw = (size_t)W + 2 * kPad, ph = (size_t)H + 2 * kPad;
    size_t pitch_bytes = round_up(pw * sizeof(float2), ctx->tex_pitch_align);
    size_t slot_bytes = round_up(pitch_bytes * ph, std::max<size_t>(ctx->tex_align, 256));
    r->rl_pitch = pitch_bytes / sizeof(float2);
    r->rl_slot = slot_bytes / sizeof(float2);
    // the data-residual pass (etcu_recon_data_residual_sq) projects as many views per
    // launch as there are slots: add slots up to all views while they fit in 64 MiB
    r->slots = std::max<uint32_t>(
        r->slots, std::min<uint32_t>(M, (uint32_t)std::max<size_t>(1, ((size_t)64 << 20) / slot_bytes)));
    if ((s = dalloc_aligned(ctx, &r->rl_raw, (void**)&r->rl_base, slot_bytes * r->slots, ctx->tex_align)) != ETCU_OK)
        return s;
    CK(ctx, cudaMemsetAsync(r->rl_base, 0, slot_bytes * r->slots, ctx->stream));
    r->rl = r->rl_base + kPad * r->rl_pitch + kPad;
    r->texs.resize(r->slots);
    for (uint32_t p = 0; p < r->slots; ++p)
        if ((s = make_pair_texture(ctx, r->rl_base + p * r->rl_slot, r->rl_pitch, (uint32_t)pw, (uint32_t)ph,
                                   &r->texs[p])) != ETCU_OK)
            return s;
    if ((s = dalloc(ctx, (void**)&r->d_texs, r->slots * sizeof(cudaTextureObject_t))) != ETCU_OK) return s;
    CK(ctx, cudaMemcpyAsync(r->d_texs, r->texs.data(), r->slots * sizeof(cudaTextureObject_t), cudaMemcpyHostToDevice,
                            ctx->stream));
    if ((s = dalloc(ctx, (void**)&r->d_resid, sizeof(double))) != ETCU_OK) return s;
    CK(ctx, cudaMemsetAsync(r->d_resid, 0, sizeof(double), ctx->stream));
    if (r->fuse_persist && ctx->autotune && (s = tune_fused_grid(r.get())) != ETCU_OK) return s;
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    if (params->use_graph) {
        // The launch sequence of one iteration never changes: capture it once.
        cudaStream_t cs = ctx->stream;
        CK(ctx, cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        uint32_t n = 0;
        etcu_status is = issue_iteration(r.get(), cs, &n);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(cs, &g);
        if (is != ETCU_OK) {
            if (g) cudaGraphDestroy(g);
            return is;
        }
        CK(ctx, e);
        r->graph = g;
        CK(ctx, cudaGraphInstantiate(&r->exec, g, 0));
        r->launches = n;
    } else {
        r->launches = r->fused ? (r->fuse_persist ? 3 : M + 1) : (uint32_t)(2 * S * r->nblocks);
    }
    *out = r.release();
    return ETCU_OK;
}

}  // namespace

extern "C" etcu_status etcu_recon_create(etcu_volume* vol, const etcu_view* views, uint32_t n_views,
                                         const float* host_projections, const etcu_recon_params* params,
                                         etcu_recon** out) {
    return recon_build(vol, views, n_views, host_projections, nullptr, params, out);
}

extern "C" etcu_status etcu_recon_create_device(etcu_volume* vol, const etcu_view* views, uint32_t n_views,
                                                const float* d_projections, const etcu_recon_params* params,
                                                etcu_recon** out) {
    if (!d_projections) return fail(vol ? vol->ctx : nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL projections");
    return recon_build(vol, views, n_views, nullptr, d_projections, params, out);
}

extern "C" etcu_status etcu_recon_destroy(etcu_recon* rec) {
    if (!rec) return ETCU_OK;
    recon_free(rec);
    delete rec;
    return ETCU_OK;
}

// The persistent fused steps' error word (a wait that gave up), read after the stream's
// work; cleared for the next run.
etcu_status check_fused_waits(etcu_recon* r) {
    if (!r->fuse_persist) return ETCU_OK;
    etcu_context* ctx = r->ctx;
    uint32_t* err = r->d_fuse_ctl + r->vol->slabs[0].ry + 1;
    uint32_t h = 0;
    CK(ctx, cudaMemcpyAsync(&h, err, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    if (h) {
        CK(ctx, cudaMemsetAsync(err, 0, sizeof(uint32_t), ctx->stream));
        return fail(ctx, ETCU_ERR_CUDA, "a fused SART step waited longer than its limit for its neighbour rows");
    }
    return ETCU_OK;
}

extern "C" etcu_status etcu_recon_run(etcu_recon* r, uint32_t iterations) {
    if (!r) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL reconstruction");
    etcu_context* ctx = r->ctx;
    for (uint32_t it = 0; it < iterations; ++it) {
        if (r->exec) {
            CK(ctx, cudaGraphLaunch(r->exec, ctx->stream));
        } else {
            etcu_status s = issue_iteration(r, ctx->stream, nullptr);
            if (s != ETCU_OK) return s;
        }
    }
    CKL(ctx);
    return check_fused_waits(r);
}

// =============================================================== z-slab decomposition over ranks
// Residual of one block from the all-reduced (virtual, traversal) images: the epilogue of
// the final sub-volume's forward projection (fp_store, kFpPairResidual: long-object
// compensation over the complete volume, r = b - Ax) written as (r, L) pairs into the
// block's slot images, and sum r^2 (FP64, one atomic per warp).
__global__ void slab_residual_kernel(const float* __restrict__ complete, float2* rl, size_t rl_pitch, size_t rl_slot,
                                     const float* __restrict__ real, int real_kind, const ViewConst* __restrict__ views,
                                     const uint32_t* __restrict__ order, uint32_t first, int W, int H, int loc,
                                     double* resid_sq) {
    const int p = blockIdx.z, gy = blockIdx.y, gx = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t vid = order[first + p];
    double r2 = 0.0;
    if (gx < W) {
        const size_t P = (size_t)W * H, i = (size_t)gy * W + gx;
        float vv = complete[(size_t)p * 2 * P + i], ll = complete[((size_t)p * 2 + 1) * P + i];
        if (loc) {  // VirtualProjection.cl:8-9
            const float c = views[vid].loc_length;
            vv = ll > kEps ? fdiv(fmul(vv, c), ll) : 0.f;
            ll = c;
        }
        const float r = fsub(load_real(real, real_kind, (size_t)vid * P + i), vv);  // Compare.cl:8
        rl[(size_t)p * rl_slot + (size_t)gy * rl_pitch + gx] = make_float2(r, ll);
        r2 = (double)r * (double)r;
    }
    for (int o = 16; o > 0; o >>= 1) r2 += __shfl_down_sync(0xffffffffu, r2, o);
    if ((threadIdx.x & 31) == 0 && r2 != 0.0) atomicAdd(resid_sq, r2);
}

extern "C" etcu_status etcu_recon_block_count(const etcu_recon* r, uint32_t* blocks, uint32_t* block_size) {
    if (!r || !blocks) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    *blocks = r->nblocks;
    if (block_size) *block_size = r->block;
    return ETCU_OK;
}

extern "C" etcu_status etcu_recon_set_complete_bbox(etcu_recon* r, const float bbox_min[3], const float bbox_max[3]) {
    if (!r || !bbox_min || !bbox_max) return fail(r ? r->ctx : nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    etcu_context* ctx = r->ctx;
    if (!r->params.use_long_object_compensation) return ETCU_OK;
    const uint32_t S = (uint32_t)r->vol->slabs.size();
    for (uint32_t sl = 0; sl < S; ++sl)
        for (uint32_t i = 0; i < r->n_input; ++i)
            r->hvc[(size_t)sl * r->n_input + i].loc_length = traversal_length(r->hviews[i], bbox_min, bbox_max);
    CK(ctx, cudaMemcpyAsync(r->d_views, r->hvc.data(), r->hvc.size() * sizeof(ViewConst), cudaMemcpyHostToDevice,
                            ctx->stream));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    return ETCU_OK;
}

extern "C" etcu_status etcu_recon_slab_forward(etcu_recon* r, uint32_t block, float* d_partial) {
    if (!r || !d_partial) return fail(r ? r->ctx : nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    etcu_context* ctx = r->ctx;
    if (block >= r->nblocks) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "block %u of %u", block, r->nblocks);
    const uint32_t M = (uint32_t)r->order.size(), first = block * r->block;
    const uint32_t count = std::min(r->block, M - first);
    const size_t P = (size_t)r->W * r->H;
    cudaStream_t st = ctx->stream;
    if (block == 0) CK(ctx, cudaMemsetAsync(r->d_resid, 0, sizeof(double), st));
    CK(ctx, cudaMemsetAsync(d_partial, 0, (size_t)count * 2 * P * sizeof(float), st));
    etcu_volume* vol = r->vol;
    for (uint32_t k = 0; k < count; ++k)
        for (uint32_t sl = 0; sl < (uint32_t)vol->slabs.size(); ++sl) {
            const SlabConst& slab = vol->slabs[sl];
            FpArgs a{};
            fill_fp_volume_ptrs(vol, slab, a);
            a.slab = slab;
            a.views = r->d_views + (size_t)sl * r->n_input;
            a.order = r->d_order;
            a.first = first + k;
            a.W = (int)r->W;
            a.H = (int)r->H;
            a.samples = r->params.fp_samples == 0 ? 1 : (int)r->params.fp_samples;
            a.mode = kFpSeparateAccumulate;  // partial line integrals of this rank's slab, added (+=)
            a.out_v = d_partial + (size_t)k * 2 * P;
            a.out_l = d_partial + ((size_t)k * 2 + 1) * P;
            launch_fp(vol, a, r->fp_paths[sl], 1, st);
        }
    CKL(ctx);
    return ETCU_OK;
}

extern "C" etcu_status etcu_recon_slab_backward(etcu_recon* r, uint32_t block, const float* d_complete) {
    if (!r || !d_complete) return fail(r ? r->ctx : nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    etcu_context* ctx = r->ctx;
    if (block >= r->nblocks) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "block %u of %u", block, r->nblocks);
    const uint32_t M = (uint32_t)r->order.size(), first = block * r->block;
    const uint32_t count = std::min(r->block, M - first);
    cudaStream_t st = ctx->stream;
    const dim3 grid((r->W + 127) / 128, r->H, count);
    slab_residual_kernel<<<grid, 128, 0, st>>>(d_complete, r->rl, r->rl_pitch, r->rl_slot, r->d_proj, r->proj_kind,
                                               r->d_views,
                                               r->d_order, first, (int)r->W, (int)r->H,
                                               r->params.use_long_object_compensation ? 1 : 0, r->d_resid);
    issue_backward(r, first, count, st);
    CKL(ctx);
    return ETCU_OK;
}

// Residual of block `block` from the complete images, then its back projection and the
// forward projection of block + 1 into d_next: for SART on the fused path one fused step
// (sart_fused_kernel writing the slab's partial images of view p + 1), otherwise the
// two calls above.
extern "C" etcu_status etcu_recon_slab_step(etcu_recon* r, uint32_t block, const float* d_complete, float* d_next) {
    if (!r || !d_complete || !d_next) return fail(r ? r->ctx : nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    etcu_context* ctx = r->ctx;
    if (block + 1 >= r->nblocks)
        return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "block %u has no next block (%u blocks)", block, r->nblocks);
    if (d_next == d_complete) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "the next block needs its own buffer");
    if (!r->fused) {
        etcu_status s = etcu_recon_slab_backward(r, block, d_complete);
        return s != ETCU_OK ? s : etcu_recon_slab_forward(r, block + 1, d_next);
    }
    cudaStream_t st = ctx->stream;
    const size_t P = (size_t)r->W * r->H;
    const dim3 grid((r->W + 127) / 128, r->H, 1);
    slab_residual_kernel<<<grid, 128, 0, st>>>(d_complete, r->rl, r->rl_pitch, r->rl_slot, r->d_proj, r->proj_kind,
                                               r->d_views, r->d_order, block, (int)r->W, (int)r->H,
                                               r->params.use_long_object_compensation ? 1 : 0, r->d_resid);
    CK(ctx, cudaMemsetAsync(d_next, 0, 2 * P * sizeof(float), st));
    launch_fused_step(r, block, st, r->rl, d_next);
    CKL(ctx);
    return ETCU_OK;
}

extern "C" etcu_status etcu_recon_last_residual_sq(etcu_recon* r, double* out) {
    if (!r || !out) return fail(r ? r->ctx : nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    etcu_context* ctx = r->ctx;
    CK(ctx, cudaMemcpyAsync(out, r->d_resid, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    return ETCU_OK;
}

extern "C" etcu_status etcu_recon_data_residual_sq(etcu_recon* r, double* out) {
    if (!r || !out) return fail(r ? r->ctx : nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    etcu_context* ctx = r->ctx;
    const uint32_t M = (uint32_t)r->order.size();
    CK(ctx, cudaMemsetAsync(r->d_resid, 0, sizeof(double), ctx->stream));
    for (uint32_t first = 0; first < M; first += r->slots)
        issue_forward(r, first, std::min(r->slots, M - first), ctx->stream);
    CKL(ctx);
    CK(ctx, cudaMemcpyAsync(out, r->d_resid, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    return ETCU_OK;
}

extern "C" etcu_status etcu_recon_view_order(const etcu_recon* r, uint32_t* out, uint32_t capacity, uint32_t* count) {
    if (!r || !count) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    *count = (uint32_t)r->order.size();
    if (out)
        for (uint32_t i = 0; i < std::min(capacity, *count); ++i) out[i] = r->order[i];
    return ETCU_OK;
}

extern "C" uint32_t etcu_recon_launches_per_iteration(const etcu_recon* r) { return r ? r->launches : 0; }

extern "C" etcu_status etcu_recon_profile_iteration(etcu_recon* r, float* fp_ms, float* bp_ms, uint32_t* fp_n,
                                                    uint32_t* bp_n) {
    if (!r || !fp_ms || !bp_ms || !fp_n || !bp_n) return fail(r ? r->ctx : nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    etcu_context* ctx = r->ctx;
    cudaStream_t st = ctx->stream;
    const uint32_t M = (uint32_t)r->order.size();
    std::vector<cudaEvent_t> ev(4 * r->nblocks);
    for (auto& e : ev) CK(ctx, cudaEventCreate(&e));
    CK(ctx, cudaMemsetAsync(r->d_resid, 0, sizeof(double), st));
    uint32_t nf = 0, nb = 0;
    for (uint32_t b = 0; b < r->nblocks; ++b) {
        const uint32_t first = b * r->block;
        const uint32_t bs = (b < r->nblocks - 1) ? r->block : M - first;
        cudaEventRecord(ev[4 * b + 0], st);
        nf += issue_forward(r, first, bs, st);
        cudaEventRecord(ev[4 * b + 1], st);
        cudaEventRecord(ev[4 * b + 2], st);
        nb += issue_backward(r, first, bs, st);
        cudaEventRecord(ev[4 * b + 3], st);
    }
    CKL(ctx);
    CK(ctx, cudaStreamSynchronize(st));
    float tf = 0.f, tb = 0.f;
    for (uint32_t b = 0; b < r->nblocks; ++b) {
        float a = 0.f, c = 0.f;
        cudaEventElapsedTime(&a, ev[4 * b + 0], ev[4 * b + 1]);
        cudaEventElapsedTime(&c, ev[4 * b + 2], ev[4 * b + 3]);
        tf += a;
        tb += c;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    *fp_ms = tf;
    *bp_ms = tb;
    *fp_n = nf;
    *bp_n = nb;
    return ETCU_OK;
}

// Runs one iteration as issue_iteration does, timing every step: kind 0 forward
// projection, 1 back projection, 2 fused step; launches per step.
extern "C" etcu_status etcu_recon_profile_steps(etcu_recon* r, float* ms, uint32_t* kinds, uint32_t* launches,
                                                uint32_t capacity, uint32_t* count) {
    if (!r || !count) return fail(r ? r->ctx : nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    etcu_context* ctx = r->ctx;
    cudaStream_t st = ctx->stream;
    const uint32_t M = (uint32_t)r->order.size();
    const uint32_t steps = r->fused ? (r->fuse_persist ? 3 : M + 1) : 2 * r->nblocks;
    *count = steps;
    if (!ms || !kinds || !launches) return ETCU_OK;
    if (capacity < steps) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "capacity %u < %u steps", capacity, steps);
    std::vector<cudaEvent_t> ev(steps + 1);
    for (auto& e : ev) CK(ctx, cudaEventCreate(&e));
    CK(ctx, cudaMemsetAsync(r->d_resid, 0, sizeof(double), st));
    uint32_t k = 0;
    auto mark = [&](uint32_t kind, uint32_t n) {
        kinds[k] = kind;
        launches[k] = n;
        cudaEventRecord(ev[++k], st);
    };
    cudaEventRecord(ev[0], st);
    if (r->fused) {
        mark(0, issue_forward(r, 0, 1, st));
        if (r->fuse_persist) {
            launch_fused_persistent(r, st);
            mark(2, 1);
        } else {
            for (uint32_t p = 0; p + 1 < M; ++p) {
                launch_fused_step(r, p, st);
                mark(2, 1);
            }
        }
        const uint32_t last = M - 1;
        mark(1, issue_backward(r, last, 1, st, r->rl + (size_t)(last & 1) * r->rl_slot));
    } else {
        for (uint32_t b = 0; b < r->nblocks; ++b) {
            const uint32_t first = b * r->block;
            const uint32_t bs = (b < r->nblocks - 1) ? r->block : M - first;
            mark(0, issue_forward(r, first, bs, st));
            mark(1, issue_backward(r, first, bs, st));
        }
    }
    CKL(ctx);
    CK(ctx, cudaStreamSynchronize(st));
    for (uint32_t i = 0; i < steps; ++i) cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]);
    for (auto& e : ev) cudaEventDestroy(e);
    return check_fused_waits(r);
}

// ================================================================ weighted back projection
namespace {

// GenerateRamLakKernel.cl: taps at positions gid - fres / 2 in float arithmetic; the
// nonzero ones (position 0 and the odd positions) with their positions.
void ramlak_taps(uint32_t fres, std::vector<float>& taps, std::vector<int>& pos) {
    const float pi_f = 3.14159274101257324f;  // M_PI_F
    const float pi2 = pi_f * pi_f;
    taps.clear();
    pos.clear();
    for (uint32_t gid = 0; gid < fres; ++gid) {
        const int p = (int)gid - (int)(fres / 2);
        float v;
        if (p == 0) v = 1.0f / 4.0f;
        else if (p % 2 == 0) v = 0.0f;
        else v = -1.0f / ((float)(p * p) * pi2);
        if (v != 0.0f) {
            taps.push_back(v);
            pos.push_back(p);
        }
    }
}

uint32_t next_pow2(uint32_t v) {  // NumericalAlgorithms::nearestPowerOfTwo
    v--;
    v |= v >> 1;
    v |= v >> 2;
    v |= v >> 4;
    v |= v >> 8;
    v |= v >> 16;
    return v + 1;
}

// PaddingForFFT.cl mirrors at most (nu - n) / 2 pixels into the image on each side; for a
// narrower image the reference reads outside its buffer.
bool wbp_padding_fits(uint32_t n, uint32_t nu) {
    const long long b = ((long long)nu - n) / 2, e = ((long long)nu + n) / 2;
    return b <= (long long)n - 1 && (long long)n + e - 1 - ((long long)nu - 1) >= 0;
}

struct WbpFilter {
    float* taps = nullptr;
    int* pos = nullptr;
    int ntaps = 0;
    etcu_context* ctx = nullptr;
    ~WbpFilter() {
        if (ctx) {
            dfree(ctx, taps, ntaps * sizeof(float));
            dfree(ctx, pos, ntaps * sizeof(int));
        }
    }
    etcu_status init(etcu_context* c, uint32_t fres) {
        ctx = c;
        // rows of up to 16384 padded pixels: 64 KB of shared memory
        CK(ctx, cudaFuncSetAttribute(wbp_filter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 16384 * 4));
        std::vector<float> t;
        std::vector<int> p;
        ramlak_taps(fres, t, p);
        ntaps = (int)t.size();
        etcu_status s;
        if ((s = dalloc(ctx, (void**)&taps, t.size() * sizeof(float))) != ETCU_OK) return s;
        if ((s = dalloc(ctx, (void**)&pos, p.size() * sizeof(int))) != ETCU_OK) return s;
        CK(ctx, cudaMemcpyAsync(taps, t.data(), t.size() * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
        CK(ctx, cudaMemcpyAsync(pos, p.data(), p.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
        return ETCU_OK;
    }
    void launch(WbpArgs a, uint32_t fres, cudaStream_t st) const {
        a.Wu = (int)next_pow2(std::max<uint32_t>((uint32_t)a.W, fres));
        a.Hu = (int)next_pow2((uint32_t)a.H);
        a.ntaps = ntaps;
        a.taps = taps;
        a.tap_pos = pos;
        wbp_filter_kernel<<<a.H, 256, (size_t)a.Wu * sizeof(float), st>>>(a);
    }
};

}  // namespace

extern "C" etcu_status etcu_wbp_filter(etcu_context* ctx, const float* d_in, float* d_out, uint32_t width,
                                       uint32_t height, uint32_t filter_width) {
    if (!ctx || !d_in || !d_out) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    if (width == 0 || height == 0 || filter_width == 0)
        return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "empty image or filter");
    if (next_pow2(std::max(width, filter_width)) > 16384)
        return fail(ctx, ETCU_ERR_UNSUPPORTED, "images up to 16384 pixels wide are filtered");
    if (!wbp_padding_fits(width, next_pow2(std::max(width, filter_width))) ||
        !wbp_padding_fits(height, next_pow2(height)))
        return fail(ctx, ETCU_ERR_UNSUPPORTED, "a %u x %u image is too small for the mirrored padding to %u x %u",
                    width, height, next_pow2(std::max(width, filter_width)), next_pow2(height));
    WbpFilter f;
    etcu_status s;
    if ((s = f.init(ctx, filter_width)) != ETCU_OK) return s;
    WbpArgs a{};
    a.proj = d_in;
    a.out_f = d_out;
    a.W = (int)width;
    a.H = (int)height;
    f.launch(a, filter_width, ctx->stream);
    CKL(ctx);
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    return ETCU_OK;
}

// WBP::WBP + WBP::runNiterations (WBPPlugin/src/reconstruction/WBP.cpp:22-86): every
// projection filtered, its ray lengths through the complete volume computed, and all
// views back projected with lambda / n_views (the operator's block size is the number
// of projections), in view order.
extern "C" etcu_status etcu_wbp(etcu_volume* vol, const etcu_view* views, uint32_t n_views,
                                const float* host_projections, float lambda, uint32_t bp_samples,
                                etcu_sampling sampling) {
    etcu_context* ctx = vol ? vol->ctx : nullptr;
    if (!vol || !views || !host_projections || n_views == 0)
        return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "NULL argument or no projections");
    for (uint32_t i = 0; i < n_views; ++i)
        if (views[i].perspective)
            return fail(ctx, ETCU_ERR_UNSUPPORTED, "WBP uses a parallel scanner geometry");
    const uint32_t fres = 128;  // WBP.cpp:40 filterSize
    if (next_pow2(std::max(views[0].width, fres)) > 16384)
        return fail(ctx, ETCU_ERR_UNSUPPORTED, "images up to 16384 pixels wide are filtered");
    if (!wbp_padding_fits(views[0].width, next_pow2(std::max(views[0].width, fres))) ||
        !wbp_padding_fits(views[0].height, next_pow2(views[0].height)))
        return fail(ctx, ETCU_ERR_UNSUPPORTED, "a %u x %u projection is too small for the mirrored padding",
                    views[0].width, views[0].height);
    etcu_recon_params p{};
    p.lambda = lambda;
    p.block_size = ETCU_BLOCK_ALL;
    p.fp_samples = 1;
    p.bp_samples = bp_samples;
    p.order = ETCU_ORDER_IDENTITY;
    p.sampling = sampling;
    p.use_graph = 0;
    etcu_recon* r = nullptr;
    etcu_status s = recon_build(vol, views, n_views, host_projections, nullptr, &p, &r);
    if (s != ETCU_OK) return s;
    WbpFilter f;
    if ((s = f.init(ctx, fres)) != ETCU_OK) {
        etcu_recon_destroy(r);
        return s;
    }
    const SlabConst& full = vol->slabs[0];
    for (uint32_t v = 0; v < n_views; ++v) {
        WbpArgs a{};
        a.proj = r->d_proj + (size_t)v * r->W * r->H;
        a.out = r->rl + (size_t)v * r->rl_slot;
        a.pitch = r->rl_pitch;
        a.W = (int)r->W;
        a.H = (int)r->H;
        a.vc = r->hvc[v];
        a.g = full;  // cmin / cmax: the complete box
        f.launch(a, fres, ctx->stream);
    }
    issue_backward(r, 0, n_views, ctx->stream);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    etcu_recon_destroy(r);
    if (e != cudaSuccess) return fail(ctx, ETCU_ERR_CUDA, "weighted back projection: %s", cudaGetErrorString(e));
    return ETCU_OK;
}

// ================================================================ blob basis functions
namespace {

// model/blobs/BlobParameters.cpp: Kaiser-Bessel blob of support radius a, degree m and
// density fall-off alpha (float members, evaluated in double).
struct BlobP {
    double a, alpha;
    unsigned m;
};

double uint_pow(double base, unsigned e) {  // NumericalAlgorithms::uintPow
    if (e == 0) return 1.0;
    if (e == 1) return base;
    const double f = uint_pow(base, e / 2);
    return f * f * (e % 2 == 0 ? 1.0 : base);
}

unsigned long long factorial(unsigned n) { return n < 2 ? 1ull : (unsigned long long)n * factorial(n - 1); }

// evaluateModifiedBessel: I_m(x) by 40 terms of its series (m = the degree).
double kb_bessel(const BlobP& p, double x) {
    double sum = 0.0, summand = uint_pow(0.5 * x, p.m) / (double)factorial(p.m);
    for (unsigned k = 0; k < 40; ++k) {
        sum += summand;
        summand *= 0.25 * x * x / (double)((k + 1) * (k + p.m + 1));
    }
    return sum;
}

double kb_evaluate(const BlobP& p, double x) {  // BlobParameters::evaluate (Lewitt 1992)
    if (0 <= x && x <= p.a) {
        const double root = std::sqrt(1.0 - (x * x) / (p.a * p.a));
        return 1.0 / kb_bessel(p, p.alpha) * uint_pow(root, p.m) * kb_bessel(p, p.alpha * root);
    }
    return 0.0;
}

etcu_status blob_params(etcu_context* ctx, const etcu_blob_params* in, BlobP& out) {
    if (!in) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "NULL blob parameters");
    if (!(in->support_radius > 0.f) || in->degree > 20)
        return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "invalid blob parameters");
    out.a = (double)in->support_radius;
    out.alpha = (double)in->density_falloff;
    out.m = in->degree;
    return ETCU_OK;
}

// BlobRayIntegrationSampler::generateSamples: the line integral through the blob at
// distance w = i a / (count - 1), 1000 steps.
void blob_table(const BlobP& p, unsigned count, std::vector<float>& out) {
    out.resize(count);
    for (unsigned i = 0; i < count; ++i) {
        const double w = (double)i * p.a / (double)(count - 1);
        const double d = std::sqrt(p.a * p.a - w * w), delta = d / 1000.0;
        double sum = 0.0;
        for (unsigned k = 1; k <= 1000; ++k) sum += kb_evaluate(p, std::sqrt(w * w + (double)(k * k) * delta * delta));
        out[i] = (float)(delta * (2.0 * sum + kb_evaluate(p, w)));
    }
}

// BlobVoxelizationKernelValues::generateValues: the blob integrated over every voxel of
// the (2 ceil(a) + 1)^3 neighbourhood with 20^3 samples, [dz][dy][dx].
void blob_voxel_kernel(const BlobP& p, std::vector<float>& out, int& ks) {
    const int r = (int)std::ceil((float)p.a);
    ks = 2 * r + 1;
    out.clear();
    for (int dz = -r; dz <= r; ++dz)
        for (int dy = -r; dy <= r; ++dy)
            for (int dx = -r; dx <= r; ++dx) {
                double val = 0.0;
                for (int sz = 0; sz < 20; ++sz)
                    for (int sy = 0; sy < 20; ++sy)
                        for (int sx = 0; sx < 20; ++sx) {
                            const double px = (double)dx - 0.5 + ((double)sx + 0.5) / 20.0;
                            const double py = (double)dy - 0.5 + ((double)sy + 0.5) / 20.0;
                            const double pz = (double)dz - 0.5 + ((double)sz + 0.5) / 20.0;
                            val += kb_evaluate(p, std::sqrt(px * px + py * py + pz * pz));
                        }
                out.push_back((float)(val / 8000.0));
            }
}

// framework/math/Matrix4x4.cpp in float, step by step: the blob kernels take the
// projection matrix and its inverse as the reference forms them (cofactor inverse in
// float), which for perspective views differs visibly from an exact inverse.
struct FMat {
    float v[16] = {};  // value 4 * column + row
    float at(int c, int r) const { return v[4 * c + r]; }
    float minor(int dc, int dr) const {
        int c[3], r[3];
        for (int i = 0; i < 3; ++i) {
            c[i] = i < dc ? i : i + 1;
            r[i] = i < dr ? i : i + 1;
        }
        const float t1 = at(c[1], r[1]) * at(c[2], r[2]) - at(c[1], r[2]) * at(c[2], r[1]);
        const float t2 = at(c[1], r[0]) * at(c[2], r[2]) - at(c[1], r[2]) * at(c[2], r[0]);
        const float t3 = at(c[1], r[0]) * at(c[2], r[1]) - at(c[1], r[1]) * at(c[2], r[0]);
        return at(c[0], r[0]) * t1 - at(c[0], r[1]) * t2 + at(c[0], r[2]) * t3;
    }
    bool inverse(FMat& out) const {
        const float det = at(0, 0) * minor(0, 0) - at(0, 1) * minor(0, 1) + at(0, 2) * minor(0, 2) -
                          at(0, 3) * minor(0, 3);
        if (std::fabs(det) == 0.0f) return false;
        const float o = 1.0f / det;
        for (int c = 0; c < 4; ++c)
            for (int r = 0; r < 4; ++r) {
                float x = minor(c, r) * o;
                if ((r + c) % 2 == 1) x *= -1.0f;
                out.v[4 * r + c] = x;
            }
        return true;
    }
};

FMat fmat_cols(const float c0[4], const float c1[4], const float c2[4], const float c3[4]) {
    FMat m;
    const float* cs[4] = {c0, c1, c2, c3};
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r) m.v[4 * c + r] = cs[c][r];
    return m;
}

FMat fmat_mul(const FMat& a, const FMat& b) {  // Matrix4x4.cpp multiply
    FMat m;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            float v = 0.0f;
            for (int k = 0; k < 4; ++k) v += a.at(k, j) * b.at(i, k);
            m.v[4 * i + j] = v;
        }
    return m;
}

// Matrix4x4::getPerspectiveProjection (Matrix4x4.cpp:376-399) in float, and its inverse.
bool float_perspective(const etcu_view& g, FMat& w2p, FMat& p2w) {
    float dc[3];
    for (int i = 0; i < 3; ++i)
        dc[i] = g.detector[i] + 0.5f * ((float)g.width * g.hpitch[i] + (float)g.height * g.vpitch[i]);
    const float c0[4] = {g.hpitch[0], g.hpitch[1], g.hpitch[2], 0.f};
    const float c1[4] = {g.vpitch[0], g.vpitch[1], g.vpitch[2], 0.f};
    const float c2[4] = {dc[0] - g.source[0], dc[1] - g.source[1], dc[2] - g.source[2], 0.f};
    const float c3[4] = {g.source[0], g.source[1], g.source[2], 1.f};
    FMat view;
    if (!fmat_cols(c0, c1, c2, c3).inverse(view)) return false;
    const float zn = 1e-2f;
    const float p0[4] = {1, 0, 0, 0}, p1[4] = {0, 1, 0, 0}, p2[4] = {0, 0, 1.0f / (1.0f - zn), 1.0f},
                p3[4] = {0, 0, -zn / (1.0f - zn), 0};
    const float t3[4] = {0.5f * (float)g.width, 0.5f * (float)g.height, 0.f, 1.f};
    const float e2[4] = {0, 0, 1, 0};
    w2p = fmat_mul(fmat_mul(fmat_cols(p0, p1, e2, t3), fmat_cols(p0, p1, p2, p3)), view);
    return w2p.inverse(p2w);
}

// The projection factories have blob kernels for perspective beams only
// (DefaultForwardProjectionCreator.cpp:30-62, DefaultBackProjectionCreator.cpp:28-63).
etcu_status blob_view(etcu_context* ctx, const etcu_view* view, FMat& w2p, FMat& p2w, const char* kind) {
    etcu_status s = check_view(ctx, view);
    if (s != ETCU_OK) return s;
    if (!view->perspective) return fail(ctx, ETCU_ERR_UNSUPPORTED, "No fitting %s projection kernel found!", kind);
    if (!float_perspective(*view, w2p, p2w)) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "matrix not invertible");
    return ETCU_OK;
}

struct DevBuf {  // a device buffer owned for one call
    etcu_context* ctx;
    void* p = nullptr;
    size_t n = 0;
    explicit DevBuf(etcu_context* c) : ctx(c) {}
    ~DevBuf() { dfree(ctx, p, n); }
    etcu_status alloc_copy(const void* host, size_t bytes) {
        n = bytes;
        etcu_status s = dalloc(ctx, &p, bytes);
        if (s != ETCU_OK) return s;
        CK(ctx, cudaMemcpyAsync(p, host, bytes, cudaMemcpyHostToDevice, ctx->stream));
        return ETCU_OK;
    }
};

constexpr int kBlobFpTable = 256;  // DefaultForwardProjectionCreator.cpp:56
constexpr int kBlobBpTable = 256;  // PerspectiveBeamsBackProjectionWithBlobsKernel.cpp:29

// one slab's forward projection of one view (BlobTraverseRay: blobRadius *= voxelSize.x)
void launch_blob_fp(const etcu_volume* vol, const SlabConst& g, const etcu_view& view, const FMat& p2w,
                    float support_radius, const float* table, int ntable, float* proj, float* len,
                    cudaStream_t st) {
    BlobFpArgs a{};
    a.vol = vol->master + slab_offset_elems(vol, g);
    a.rx = g.rx;
    a.ry = g.ry;
    a.rz = g.rz;
    a.bmin = g.bmin;
    a.vs = g.vs;
    std::memcpy(a.p2w.v, p2w.v, sizeof(a.p2w.v));
    a.source = make_float4(view.source[0], view.source[1], view.source[2], 0.f);
    a.R = support_radius * g.vs.x;
    a.grid = (int)ceilf(1.415f * a.R / g.vs.x);
    a.table = table;
    a.ntable = ntable;
    a.W = (int)view.width;
    a.H = (int)view.height;
    a.proj = proj;
    a.len = len;
    blob_fp_kernel<<<dim3((a.W + 31) / 32, a.H), dim3(32, kBlobFpParts), (size_t)ntable * sizeof(float), st>>>(a);
}

// one slab's back projection of one view with lambda already divided by the block size
// (BackProjectionKernel.cpp:94)
void launch_blob_bp(etcu_volume* vol, const SlabConst& g, const etcu_view& view, const FMat& w2p, const FMat& p2w,
                    float support_radius, const float* table, int ntable, const float* residual,
                    const float* raylength, float lambda, cudaStream_t st) {
    BlobBpArgs a{};
    const size_t off = slab_offset_elems(vol, g);
    a.vol = vol->master + off;
    a.rx = g.rx;
    a.ry = g.ry;
    a.rz = g.rz;
    a.bmin = g.bmin;
    a.vs = g.vs;
    std::memcpy(a.w2p.v, w2p.v, sizeof(a.w2p.v));
    std::memcpy(a.p2w.v, p2w.v, sizeof(a.p2w.v));
    a.source = make_float4(view.source[0], view.source[1], view.source[2], 0.f);
    a.detector = make_float4(view.detector[0], view.detector[1], view.detector[2], 0.f);
    a.hpitch = make_float4(view.hpitch[0], view.hpitch[1], view.hpitch[2], 0.f);
    a.vpitch = make_float4(view.vpitch[0], view.vpitch[1], view.vpitch[2], 0.f);
    a.R = support_radius * g.vs.x;
    a.table = table;
    a.ntable = ntable;
    a.residual = residual;
    a.raylength = raylength;
    a.W = (int)view.width;
    a.H = (int)view.height;
    a.lambda = lambda;
    a.mask = vol->mask ? vol->mask + off : nullptr;
    blob_bp_kernel<<<dim3((g.rx + 127) / 128, g.ry, g.rz), 128, 0, st>>>(a);
}

etcu_status blob_volume_ok(etcu_context* ctx, const etcu_volume* vol) {
    if (vol->type != ETCU_VOXEL_FLOAT32) return fail(ctx, ETCU_ERR_UNSUPPORTED, "blob coefficients are FP32 volumes");
    for (const SlabConst& g : vol->slabs)
        if (g.ry > 65535 || g.rz > 65535)
            return fail(ctx, ETCU_ERR_UNSUPPORTED, "sub-volume of %d x %d x %d exceeds the launch grid", g.rx, g.ry,
                        g.rz);
    return ETCU_OK;
}

}  // namespace

extern "C" etcu_status etcu_blob_ray_integration_samples(const etcu_blob_params* params, uint32_t count, float* out) {
    BlobP p;
    etcu_status s = blob_params(nullptr, params, p);
    if (s != ETCU_OK) return s;
    if (count < 2 || !out) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "at least two samples and an output");
    std::vector<float> t;
    blob_table(p, count, t);
    std::memcpy(out, t.data(), count * sizeof(float));
    return ETCU_OK;
}

extern "C" etcu_status etcu_blob_voxelization_kernel(const etcu_blob_params* params, float* out, uint32_t capacity,
                                                     uint32_t* size_per_dim) {
    BlobP p;
    etcu_status s = blob_params(nullptr, params, p);
    if (s != ETCU_OK) return s;
    if (!size_per_dim) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    const int ks = 2 * (int)std::ceil((float)p.a) + 1;
    *size_per_dim = (uint32_t)ks;
    if (!out) return ETCU_OK;
    if (capacity < (uint32_t)(ks * ks * ks))
        return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "output holds %u of %d values", capacity, ks * ks * ks);
    std::vector<float> k;
    int n;
    blob_voxel_kernel(p, k, n);
    std::memcpy(out, k.data(), k.size() * sizeof(float));
    return ETCU_OK;
}

extern "C" etcu_status etcu_forward_project_blobs(etcu_volume* vol, const etcu_view* view, uint32_t subvolume,
                                                  const etcu_blob_params* params, uint32_t sample_count,
                                                  float* d_projection, float* d_traversal) {
    etcu_context* ctx = vol ? vol->ctx : nullptr;
    if (!vol || !d_projection || !d_traversal) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    if (subvolume != ETCU_ALL_SUBVOLUMES && subvolume >= vol->slabs.size())
        return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "subvolume %u out of range", subvolume);
    if (sample_count < 2 || sample_count > 8192) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "2 to 8192 table samples");
    BlobP p;
    FMat w2p, p2w;
    etcu_status s;
    if ((s = blob_volume_ok(ctx, vol)) != ETCU_OK || (s = blob_params(ctx, params, p)) != ETCU_OK ||
        (s = blob_view(ctx, view, w2p, p2w, "forward")) != ETCU_OK)
        return s;
    std::vector<float> table;
    blob_table(p, sample_count, table);
    DevBuf dt(ctx);
    if ((s = dt.alloc_copy(table.data(), table.size() * sizeof(float))) != ETCU_OK) return s;
    for (size_t i = 0; i < vol->slabs.size(); ++i)
        if (subvolume == ETCU_ALL_SUBVOLUMES || i == subvolume)
            launch_blob_fp(vol, vol->slabs[i], *view, p2w, params->support_radius, (const float*)dt.p,
                           (int)sample_count, d_projection, d_traversal, ctx->stream);
    CKL(ctx);
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    return ETCU_OK;
}

extern "C" etcu_status etcu_back_project_blobs(etcu_volume* vol, const etcu_view* view, uint32_t subvolume,
                                               const etcu_blob_params* params, float lambda, uint32_t block_size,
                                               const float* d_residual, const float* d_raylength) {
    etcu_context* ctx = vol ? vol->ctx : nullptr;
    if (!vol || !d_residual || !d_raylength) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    if (block_size == 0) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "Illegal ProjectionBlockSize!");
    if (subvolume != ETCU_ALL_SUBVOLUMES && subvolume >= vol->slabs.size())
        return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "subvolume %u out of range", subvolume);
    BlobP p;
    FMat w2p, p2w;
    etcu_status s;
    if ((s = blob_volume_ok(ctx, vol)) != ETCU_OK || (s = blob_params(ctx, params, p)) != ETCU_OK ||
        (s = blob_view(ctx, view, w2p, p2w, "back")) != ETCU_OK)
        return s;
    std::vector<float> table;
    blob_table(p, kBlobBpTable, table);
    DevBuf dt(ctx);
    if ((s = dt.alloc_copy(table.data(), table.size() * sizeof(float))) != ETCU_OK) return s;
    for (size_t i = 0; i < vol->slabs.size(); ++i)
        if (subvolume == ETCU_ALL_SUBVOLUMES || i == subvolume)
            launch_blob_bp(vol, vol->slabs[i], *view, w2p, p2w, params->support_radius, (const float*)dt.p,
                           kBlobBpTable, d_residual, d_raylength, lambda / (float)block_size, ctx->stream);
    CKL(ctx);
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    return ETCU_OK;
}

// ---------------------------------------------------------------- blob block iterations
// BlockIterativeReconstructionOperator.cpp:84-160 with algorithm.basisFunctions = blobs:
// tables and matrices formed once, the tilt series device-resident, per block the forward
// projection of every view into cleared images, the residual, then the back projection
// of every view with lambda / block size; iterations stream-ordered, one sync per run.
struct etcu_blob_recon {
    etcu_volume* vol = nullptr;
    etcu_context* ctx = nullptr;
    float lambda = 1.f, support_radius = 2.f;
    uint32_t W = 0, H = 0, n_input = 0, block = 1;
    std::vector<uint32_t> order;
    std::vector<etcu_view> views;
    std::vector<FMat> w2p, p2w;
    float* d_proj = nullptr;
    bool own_proj = false;
    float* d_img = nullptr;  // virtual, traversal, residual: 3 x block x W x H
    float* d_tables = nullptr;  // forward table, back table
    double* d_rsq = nullptr;
    double last_rsq = 0.0;
    uint32_t launches = 0;
};

namespace {
void blob_recon_free(etcu_blob_recon* r) {
    etcu_context* ctx = r->ctx;
    const size_t P = (size_t)r->W * r->H;
    if (r->own_proj) dfree(ctx, r->d_proj, P * r->n_input * sizeof(float));
    dfree(ctx, r->d_img, 3 * P * r->block * sizeof(float));
    dfree(ctx, r->d_tables, (kBlobFpTable + kBlobBpTable) * sizeof(float));
    dfree(ctx, r->d_rsq, sizeof(double));
}

etcu_status blob_recon_build(etcu_volume* vol, const etcu_view* views, uint32_t n_views, const float* host_proj,
                             const float* dev_proj, const etcu_recon_params* params, const etcu_blob_params* blob,
                             etcu_blob_recon** out) {
    etcu_context* ctx = vol ? vol->ctx : nullptr;
    if (!vol || !views || !params || !out || (!host_proj && !dev_proj))
        return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n_views == 0) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "no projections");
    if (params->block_size == 0) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "Illegal ProjectionBlockSize!");
    if (params->use_long_object_compensation)
        return fail(ctx, ETCU_ERR_INVALID_ARGUMENT,
                    "Calculation of traversal length is only supported for parallel scanner geometry!");
    if (params->projection_storage != ETCU_PROJ_F32)
        return fail(ctx, ETCU_ERR_UNSUPPORTED, "blob reconstructions keep the projections in FP32");
    BlobP p;
    etcu_status s;
    if ((s = blob_volume_ok(ctx, vol)) != ETCU_OK || (s = blob_params(ctx, blob, p)) != ETCU_OK) return s;
    std::unique_ptr<etcu_blob_recon, void (*)(etcu_blob_recon*)> r(new etcu_blob_recon(), [](etcu_blob_recon* q) {
        blob_recon_free(q);
        delete q;
    });
    r->vol = vol;
    r->ctx = ctx;
    r->lambda = params->lambda;
    r->support_radius = blob->support_radius;
    r->n_input = n_views;
    r->W = views[0].width;
    r->H = views[0].height;
    r->views.assign(views, views + n_views);
    r->w2p.resize(n_views);
    r->p2w.resize(n_views);
    for (uint32_t i = 0; i < n_views; ++i) {
        if (views[i].width != r->W || views[i].height != r->H)
            return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "all projections must share one resolution");
        if ((s = blob_view(ctx, &views[i], r->w2p[i], r->p2w[i], "forward")) != ETCU_OK) return s;
    }
    r->order = projection_order(params->order, n_views, params->skip, params->skip ? params->skip_count : 0);
    const uint32_t M = (uint32_t)r->order.size();
    if (M == 0) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "After applying SkipProjectionList no projections are left!");
    r->block = params->block_size == ETCU_BLOCK_ALL ? M : std::min(params->block_size, M);
    const size_t P = (size_t)r->W * r->H;
    if (dev_proj) {
        r->d_proj = const_cast<float*>(dev_proj);
    } else {
        if ((s = dalloc(ctx, (void**)&r->d_proj, P * n_views * sizeof(float))) != ETCU_OK) return s;
        r->own_proj = true;
        CK(ctx, cudaMemcpyAsync(r->d_proj, host_proj, P * n_views * sizeof(float), cudaMemcpyHostToDevice,
                                ctx->stream));
    }
    if ((s = dalloc(ctx, (void**)&r->d_img, 3 * P * r->block * sizeof(float))) != ETCU_OK) return s;
    std::vector<float> tables, t;
    blob_table(p, kBlobFpTable, tables);
    blob_table(p, kBlobBpTable, t);
    tables.insert(tables.end(), t.begin(), t.end());
    if ((s = dalloc(ctx, (void**)&r->d_tables, tables.size() * sizeof(float))) != ETCU_OK) return s;
    CK(ctx, cudaMemcpyAsync(r->d_tables, tables.data(), tables.size() * sizeof(float), cudaMemcpyHostToDevice,
                            ctx->stream));
    if ((s = dalloc(ctx, (void**)&r->d_rsq, sizeof(double))) != ETCU_OK) return s;
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    *out = r.release();
    return ETCU_OK;
}

// ev (optional): one event pair per launch of kind 0 forward, 1 residual, 2 back, recorded
// around it on the stream; kinds gets the kind of every launch.
uint32_t issue_blob_iteration(etcu_blob_recon* r, std::vector<std::pair<cudaEvent_t, cudaEvent_t>>* ev = nullptr,
                              std::vector<int>* kinds = nullptr) {
    etcu_volume* vol = r->vol;
    cudaStream_t st = r->ctx->stream;
    const size_t P = (size_t)r->W * r->H;
    const uint32_t M = (uint32_t)r->order.size();
    const float* fpt = r->d_tables;
    const float* bpt = r->d_tables + kBlobFpTable;
    uint32_t launches = 0;
    cudaMemsetAsync(r->d_rsq, 0, sizeof(double), st);
    for (uint32_t b0 = 0; b0 < M; b0 += r->block) {
        const uint32_t n = std::min(r->block, M - b0);
        float* virt = r->d_img;
        float* trav = r->d_img + (size_t)r->block * P;
        float* res = r->d_img + 2 * (size_t)r->block * P;
        // BlockIterativeState::setCurrentBlockIndex clears the block's images
        cudaMemsetAsync(virt, 0, n * P * sizeof(float), st);
        cudaMemsetAsync(trav, 0, n * P * sizeof(float), st);
        for (size_t sl = 0; sl < vol->slabs.size(); ++sl)
            for (uint32_t j = 0; j < n; ++j) {
                const uint32_t v = r->order[b0 + j];
                if (ev) cudaEventRecord((*ev)[launches].first, st);
                launch_blob_fp(vol, vol->slabs[sl], r->views[v], r->p2w[v], r->support_radius, fpt, kBlobFpTable,
                               virt + j * P, trav + j * P, st);
                if (ev) {
                    cudaEventRecord((*ev)[launches].second, st);
                    kinds->push_back(0);
                }
                ++launches;
            }
        for (uint32_t j = 0; j < n; ++j) {
            const uint32_t v = r->order[b0 + j];
            const int blocks = (int)std::min<size_t>((P + 255) / 256, 148 * 8);
            if (ev) cudaEventRecord((*ev)[launches].first, st);
            blob_residual_kernel<<<blocks, 256, 0, st>>>(r->d_proj + (size_t)v * P, virt + j * P, res + j * P, P,
                                                         r->d_rsq);
            if (ev) {
                cudaEventRecord((*ev)[launches].second, st);
                kinds->push_back(1);
            }
            ++launches;
        }
        for (size_t k = vol->slabs.size(); k-- > 0;)  // doBackProjectionForBlock: sub-volumes last to first
            for (uint32_t j = 0; j < n; ++j) {
                const uint32_t v = r->order[b0 + j];
                if (ev) cudaEventRecord((*ev)[launches].first, st);
                launch_blob_bp(vol, vol->slabs[k], r->views[v], r->w2p[v], r->p2w[v], r->support_radius, bpt,
                               kBlobBpTable, res + j * P, trav + j * P, r->lambda / (float)n, st);
                if (ev) {
                    cudaEventRecord((*ev)[launches].second, st);
                    kinds->push_back(2);
                }
                ++launches;
            }
    }
    return launches;
}
}  // namespace

extern "C" etcu_status etcu_blob_recon_create(etcu_volume* vol, const etcu_view* views, uint32_t n_views,
                                              const float* host_projections, const etcu_recon_params* params,
                                              const etcu_blob_params* blob, etcu_blob_recon** out) {
    return blob_recon_build(vol, views, n_views, host_projections, nullptr, params, blob, out);
}

extern "C" etcu_status etcu_blob_recon_create_device(etcu_volume* vol, const etcu_view* views, uint32_t n_views,
                                                     const float* d_projections, const etcu_recon_params* params,
                                                     const etcu_blob_params* blob, etcu_blob_recon** out) {
    return blob_recon_build(vol, views, n_views, nullptr, d_projections, params, blob, out);
}

extern "C" etcu_status etcu_blob_recon_run(etcu_blob_recon* r, uint32_t iterations) {
    if (!r) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL reconstruction");
    etcu_context* ctx = r->ctx;
    for (uint32_t it = 0; it < iterations; ++it) r->launches = issue_blob_iteration(r);
    CKL(ctx);
    if (iterations) {
        CK(ctx, cudaMemcpyAsync(&r->last_rsq, r->d_rsq, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    }
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    return ETCU_OK;
}

extern "C" etcu_status etcu_blob_recon_profile_iteration(etcu_blob_recon* r, float* ms_by_kind, uint32_t* n_by_kind) {
    if (!r || !ms_by_kind || !n_by_kind) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    etcu_context* ctx = r->ctx;
    // per view: a forward and a back projection per sub-volume and one residual launch
    const uint32_t n = (uint32_t)r->order.size() * (2 * (uint32_t)r->vol->slabs.size() + 1);
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev(n);
    for (auto& e : ev) {
        CK(ctx, cudaEventCreate(&e.first));
        CK(ctx, cudaEventCreate(&e.second));
    }
    std::vector<int> kinds;
    r->launches = issue_blob_iteration(r, &ev, &kinds);
    CKL(ctx);
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    for (int k = 0; k < 3; ++k) {
        ms_by_kind[k] = 0.f;
        n_by_kind[k] = 0;
    }
    for (size_t i = 0; i < kinds.size(); ++i) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev[i].first, ev[i].second);
        ms_by_kind[kinds[i]] += ms;
        ++n_by_kind[kinds[i]];
    }
    for (auto& e : ev) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    CK(ctx, cudaMemcpy(&r->last_rsq, r->d_rsq, sizeof(double), cudaMemcpyDeviceToHost));
    return ETCU_OK;
}

extern "C" etcu_status etcu_blob_recon_last_residual_sq(const etcu_blob_recon* r, double* out) {
    if (!r || !out) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = r->last_rsq;
    return ETCU_OK;
}

extern "C" etcu_status etcu_blob_recon_view_order(const etcu_blob_recon* r, uint32_t* out, uint32_t capacity,
                                                  uint32_t* count) {
    if (!r || !count) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    *count = (uint32_t)r->order.size();
    if (out) std::memcpy(out, r->order.data(), std::min<size_t>(capacity, r->order.size()) * sizeof(uint32_t));
    return ETCU_OK;
}

extern "C" uint32_t etcu_blob_recon_launches_per_iteration(const etcu_blob_recon* r) { return r ? r->launches : 0; }

extern "C" etcu_status etcu_blob_recon_destroy(etcu_blob_recon* r) {
    if (!r) return ETCU_OK;
    blob_recon_free(r);
    delete r;
    return ETCU_OK;
}

extern "C" etcu_status etcu_blob_voxelize(etcu_volume* blobs, etcu_volume* voxels, const etcu_blob_params* params) {
    etcu_context* ctx = blobs ? blobs->ctx : nullptr;
    if (!blobs || !voxels) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "NULL volume");
    if (blobs->type != ETCU_VOXEL_FLOAT32 || voxels->type != ETCU_VOXEL_FLOAT32)
        return fail(ctx, ETCU_ERR_UNSUPPORTED, "blob voxelisation takes FP32 volumes");
    for (int i = 0; i < 3; ++i)
        if (blobs->desc.resolution[i] != voxels->desc.resolution[i])
            return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "Input and output volume resolutions for VolumeConvolutionKernel differ!");
    BlobP p;
    etcu_status s = blob_params(ctx, params, p);
    if (s != ETCU_OK) return s;
    std::vector<float> k;
    int ks;
    blob_voxel_kernel(p, k, ks);
    DevBuf dk(ctx);
    if ((s = dk.alloc_copy(k.data(), k.size() * sizeof(float))) != ETCU_OK) return s;
    const int X = (int)blobs->desc.resolution[0], Y = (int)blobs->desc.resolution[1], Z = (int)blobs->desc.resolution[2];
    blob_voxelize_kernel<<<dim3((X + 127) / 128, Y, Z), 128, 0, ctx->stream>>>(blobs->master, voxels->master, X, Y, Z,
                                                                               (const float*)dk.p, ks);
    CKL(ctx);
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    return ETCU_OK;
}

// ================================================================ batched series
struct etcu_batch {
    etcu_context* ctx = nullptr;
    uint32_t n = 0;
    std::vector<etcu_volume*> vols;
    std::vector<int> steps;                // views per series
    std::vector<std::pair<void*, size_t>> allocs;  // device allocations (pointer, bytes)
    FpArgs* d_fp = nullptr;                // per-series forward-projection arguments
    BpArgs* d_bp = nullptr;                // per-series back-projection arguments
    int* d_steps = nullptr;
    double* d_resid = nullptr;             // per series
    int fp_path = kFpPathGeneral;
    int max_steps = 0, max_w = 0, max_h = 0, max_rx = 0, max_ry = 0;
    etcu_sampling sampling = ETCU_SAMPLING_Q8;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t launches = 0;
    // the whole iteration of every series in one launch (sart_fused_batch_kernel)
    bool persist = false;
    FuseSeries* d_series = nullptr;
    FuseSegment* d_segs = nullptr;
    uint32_t nsegs = 0, total_units = 0, ctl_words = 0;
    uint32_t* d_ctl = nullptr;  // [0] unit counter, then every series' row counters, then the error word
    int grid = 0, threads = 0;
    size_t smem = 0;
    int shadow = 0;  // 1 / 2: every series is an FP32 master with an FP16 / BF16 shadow
    int per_sm128 = 0, per_sm512 = 0, sms = 0;  // occupancy of the persistent variants (autotuner)
    std::string shape_key;                       // the series' shapes, for the autotuner's cache
};

namespace {

void batch_free(etcu_batch* b) {
    etcu_context* ctx = b->ctx;
    cudaStreamSynchronize(ctx->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (auto& a : b->allocs) dfree(ctx, a.first, a.second);
    b->allocs.clear();
}

etcu_status batch_alloc(etcu_batch* b, void** p, size_t bytes) {
    etcu_status s = dalloc(b->ctx, p, bytes);
    if (s == ETCU_OK && *p) b->allocs.emplace_back(*p, bytes);
    return s;
}

template <int kPath>
void launch_fp_batch_t(const etcu_batch* b, int step, cudaStream_t st) {
    dim3 grid((b->max_w + 127) / 128, b->max_h, b->n);
    forward_project_batch_kernel<float, false, kPath><<<grid, 128, 0, st>>>(b->d_fp, b->d_steps, step);
}

// One SART step of every series: forward projection of the view at order position
// `step` with the residual epilogue, then its back projection.
void issue_batch_step(const etcu_batch* b, int step, cudaStream_t st) {
    switch (b->fp_path) {
    case kFpPathXzNoCap: launch_fp_batch_t<kFpPathXzNoCap>(b, step, st); break;
    case kFpPathXz: launch_fp_batch_t<kFpPathXz>(b, step, st); break;
    default: launch_fp_batch_t<kFpPathGeneral>(b, step, st); break;
    }
    dim3 grid((b->max_rx + 31) / 32, (b->max_ry + 7) / 8, b->n), block(32, 8, 1);
    if (b->sampling == ETCU_SAMPLING_EXACT)
        bp_sart_row_batch_kernel<kSampleExact><<<grid, block, 0, st>>>(b->d_bp, b->d_steps, step);
    else
        bp_sart_row_batch_kernel<kSampleQ8><<<grid, block, 0, st>>>(b->d_bp, b->d_steps, step);
}

etcu_status issue_batch_iteration(etcu_batch* b, cudaStream_t st) {
    etcu_context* ctx = b->ctx;
    CK(ctx, cudaMemsetAsync(b->d_resid, 0, sizeof(double) * b->n, st));
    if (b->persist) {
        CK(ctx, cudaMemsetAsync(b->d_ctl, 0, (size_t)(b->ctl_words - 1) * sizeof(uint32_t), st));
        uint32_t* err = b->d_ctl + b->ctl_words - 1;
        const int withhold = ctx->fuse_withhold_row;
        const bool narrow = b->threads == 128;
#define ETCU_BATCH_LAUNCH(T, SH)                                                                                   \
    sart_fused_batch_kernel<T, SH><<<b->grid, T, b->smem, st>>>(b->d_series, b->d_segs, b->nsegs, b->total_units, \
                                                                 b->d_ctl, err, withhold)
        if (b->shadow == 1) {
            if (narrow) ETCU_BATCH_LAUNCH(128, 1);
            else ETCU_BATCH_LAUNCH(kFuseThreads, 1);
        } else if (b->shadow == 2) {
            if (narrow) ETCU_BATCH_LAUNCH(128, 2);
            else ETCU_BATCH_LAUNCH(kFuseThreads, 2);
        } else {
            if (narrow) ETCU_BATCH_LAUNCH(128, 0);
            else ETCU_BATCH_LAUNCH(kFuseThreads, 0);
        }
#undef ETCU_BATCH_LAUNCH
        CKL(ctx);
        return ETCU_OK;
    }
    for (int k = 0; k < b->max_steps; ++k) issue_batch_step(b, k, st);
    CKL(ctx);
    return ETCU_OK;
}

// One series as the persistent batch plan needs it (host view constants, samples and
// the device copies made for the per-step path).
struct BatchSeriesRec {
    etcu_volume* vol;
    SlabConst slab;
    std::vector<ViewConst> vc;
    std::vector<float4> hs;
    const ViewConst* d_views;
    const uint32_t* d_order;
    const float4* d_samples;
    const float* d_proj;
    uint32_t W, H, M;
};

// Whether every series can run the fused SART steps (the conditions of plan_fused, series
// by series); if so, builds the persistent batch: per series its tap windows, row table,
// dependency window, two residual slots and row counters; the (step, series) segments in
// step-major order.  Otherwise the batch keeps its per-step launches.
etcu_status plan_batch_persistent(etcu_batch* b, const std::vector<BatchSeriesRec>& recs,
                                  const etcu_recon_params* params) {
    etcu_context* ctx = b->ctx;
    if (!ctx->fused_step || !ctx->fused_persist || params->sampling != ETCU_SAMPLING_Q8 || params->fp_samples > 1 ||
        params->bp_samples != 1)
        return ETCU_OK;
    const uint32_t n = (uint32_t)recs.size();
    std::vector<FuseSeries> fs(n);
    std::vector<std::vector<int2>> tables(n), tapwins(n);
    std::vector<int> windows(n);
    size_t smem = 0;
    bool narrow = true;  // every row fits a block of 128 threads (256 voxels, 256 rays)
    etcu_status s;
    for (uint32_t i = 0; i < n; ++i) {
        const BatchSeriesRec& rc = recs[i];
        const SlabConst& g = rc.slab;
        if (g.rx % 2 != 0 || g.rx > 2 * kFuseThreads || g.rx + g.rz - 1 > kMaxDdaIterations || g.ry > 65535 ||
            rc.M > 65534)
            return ETCU_OK;
        const uint32_t N = (uint32_t)rc.vc.size();
        tapwins[i].resize(N);
        for (uint32_t v = 0; v < N; ++v) {
            const ViewConst& c = rc.vc[v];
            if (!c.fast2d || !row_constant(c) || c.hpitch.y != 0.f) return ETCU_OK;
            BpColPlan plan;
            if (!plan_bp_col(rc.vol, g, c, rc.hs[v], plan)) return ETCU_OK;
            tapwins[i][v] = make_int2(plan.x0lo, plan.ntaps);
            smem = std::max(smem, fuse_smem_bytes(g.rx, g.rz, plan.ntaps));
        }
        bool ok = false;
        if ((s = fuse_row_table(ctx, rc.d_views, g, N, rc.W, rc.H, tables[i], ok)) != ETCU_OK) return s;
        if (!ok) return ETCU_OK;
        narrow &= g.rx <= 2 * 128;
        for (const int2& jr : tables[i]) narrow &= (long long)(jr.y - jr.x) * rc.W <= (long long)kFuseRays * 128;
        if ((s = fuse_window_of(ctx, rc.d_views, rc.d_samples, g, N, rc.H, tables[i], windows[i])) != ETCU_OK) return s;
        if (windows[i] < 0 || windows[i] > kFuseMaxWindow) return ETCU_OK;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, ctx->device) != cudaSuccess) {
        cudaGetLastError();
        return ETCU_OK;
    }
    const int threads = narrow ? 128 : kFuseThreads;
    const void* variants[3] = {
        narrow ? (const void*)sart_fused_batch_kernel<128, 0> : (const void*)sart_fused_batch_kernel<kFuseThreads, 0>,
        narrow ? (const void*)sart_fused_batch_kernel<128, 1> : (const void*)sart_fused_batch_kernel<kFuseThreads, 1>,
        narrow ? (const void*)sart_fused_batch_kernel<128, 2> : (const void*)sart_fused_batch_kernel<kFuseThreads, 2>};
    const void* kern = variants[b->shadow];
    // resident blocks per SM of the 512-thread variant and (narrow batches) the 128-thread one
    auto occupancy = [&](const void* k, int t) {
        cudaFuncAttributes fa;
        if (cudaFuncGetAttributes(&fa, k) != cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(prop.sharedMemPerBlockOptin - fa.sharedSizeBytes));
        cudaGetLastError();
        int per = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, t, smem) != cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
        return per;
    };
    const void* wide_variants[3] = {(const void*)sart_fused_batch_kernel<kFuseThreads, 0>,
                                    (const void*)sart_fused_batch_kernel<kFuseThreads, 1>,
                                    (const void*)sart_fused_batch_kernel<kFuseThreads, 2>};
    const int per_sm = occupancy(kern, threads);
    if (per_sm < 1) return ETCU_OK;
    b->per_sm512 = narrow ? occupancy(wide_variants[b->shadow], kFuseThreads) : per_sm;
    b->per_sm128 = narrow ? per_sm : 0;
    b->sms = prop.multiProcessorCount;
    // segments: unit steps 0 .. M of every series, step-major
    uint32_t max_m = 0;
    for (const auto& rc : recs) max_m = std::max(max_m, rc.M);
    std::vector<FuseSegment> segs;
    unsigned long long start = 0;
    for (uint32_t st = 0; st <= max_m; ++st)
        for (uint32_t i = 0; i < n; ++i)
            if (st <= recs[i].M) {
                segs.push_back(FuseSegment{(uint32_t)start, i, st});
                start += (unsigned long long)recs[i].slab.ry;
            }
    if (start >= 0xffffffffull) return ETCU_OK;
    // device data
    uint32_t words = 1;
    std::vector<uint32_t> done_off(n);
    for (uint32_t i = 0; i < n; ++i) {
        done_off[i] = words;
        words += (uint32_t)recs[i].slab.ry;
    }
    words += 1;  // the error word
    if ((s = batch_alloc(b, (void**)&b->d_ctl, (size_t)words * sizeof(uint32_t))) != ETCU_OK) return s;
    CK(ctx, cudaMemsetAsync(b->d_ctl, 0, (size_t)words * sizeof(uint32_t), ctx->stream));
    for (uint32_t i = 0; i < n; ++i) {
        const BatchSeriesRec& rc = recs[i];
        const SlabConst& g = rc.slab;
        const uint32_t N = (uint32_t)rc.vc.size();
        int2 *d_jr, *d_tw;
        if ((s = batch_alloc(b, (void**)&d_jr, tables[i].size() * sizeof(int2))) != ETCU_OK) return s;
        if ((s = batch_alloc(b, (void**)&d_tw, N * sizeof(int2))) != ETCU_OK) return s;
        CK(ctx, cudaMemcpyAsync(d_jr, tables[i].data(), tables[i].size() * sizeof(int2), cudaMemcpyHostToDevice,
                                ctx->stream));
        CK(ctx, cudaMemcpyAsync(d_tw, tapwins[i].data(), N * sizeof(int2), cudaMemcpyHostToDevice, ctx->stream));
        const size_t pw = (size_t)rc.W + 2 * kPad, ph = (size_t)rc.H + 2 * kPad, slot = pw * ph;
        float2* rl_base;
        if ((s = batch_alloc(b, (void**)&rl_base, 2 * slot * sizeof(float2))) != ETCU_OK) return s;
        CK(ctx, cudaMemsetAsync(rl_base, 0, 2 * slot * sizeof(float2), ctx->stream));
        FuseSeries& f = fs[i];
        f = FuseSeries{};
        f.a.vol = rc.vol->master + slab_offset_elems(rc.vol, g);
        f.a.slab = g;
        f.a.views = rc.d_views;
        f.a.order = rc.d_order;
        f.a.samples = rc.d_samples;
        f.a.rl_pitch = pw;
        f.a.W = (int)rc.W;
        f.a.H = (int)rc.H;
        f.a.lambda = params->lambda;  // block size 1
        f.a.jrange = d_jr;
        f.a.real = rc.d_proj;
        f.a.real_kind = params->projection_storage;
        f.a.resid_sq = b->d_resid + i;
        f.a.loc = params->use_long_object_compensation ? 1 : 0;
        f.tapwin = d_tw;
        f.rl0 = rl_base + kPad * pw + kPad;
        f.rl_slot = slot;
        f.done = b->d_ctl + done_off[i];
        f.views = rc.M;
        f.window = windows[i];
    }
    if ((s = batch_alloc(b, (void**)&b->d_series, n * sizeof(FuseSeries))) != ETCU_OK) return s;
    if ((s = batch_alloc(b, (void**)&b->d_segs, segs.size() * sizeof(FuseSegment))) != ETCU_OK) return s;
    CK(ctx, cudaMemcpyAsync(b->d_series, fs.data(), n * sizeof(FuseSeries), cudaMemcpyHostToDevice, ctx->stream));
    CK(ctx, cudaMemcpyAsync(b->d_segs, segs.data(), segs.size() * sizeof(FuseSegment), cudaMemcpyHostToDevice,
                            ctx->stream));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    b->nsegs = (uint32_t)segs.size();
    b->total_units = (uint32_t)start;
    b->ctl_words = words;
    b->smem = smem;
    b->grid = (int)std::min<long long>((long long)per_sm * prop.multiProcessorCount, (long long)start);
    b->threads = threads;
    b->persist = true;
    return ETCU_OK;
}

// The persistent batch's error word (a wait that gave up), read after the stream's work.
etcu_status check_batch_waits(etcu_batch* b) {
    if (!b->persist) return ETCU_OK;
    etcu_context* ctx = b->ctx;
    uint32_t* err = b->d_ctl + b->ctl_words - 1;
    uint32_t h = 0;
    CK(ctx, cudaMemcpyAsync(&h, err, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    if (h) {
        CK(ctx, cudaMemsetAsync(err, 0, sizeof(uint32_t), ctx->stream));
        return fail(ctx, ETCU_ERR_CUDA, "a fused SART step waited longer than its limit for its neighbour rows");
    }
    return ETCU_OK;
}

etcu_status issue_batch_iteration(etcu_batch* b, cudaStream_t st);

// Autotuner: threads per block (128 for batches whose rows fit, 512) and resident blocks
// per SM of the persistent batched iteration, timed on whole iterations; every series'
// volume (master and shadow) is saved before and restored after the timing runs.
etcu_status tune_batch(etcu_batch* b) {
    etcu_context* ctx = b->ctx;
    uint64_t h = 1469598103934665603ull;  // FNV-1a of the series' shapes
    for (etcu_volume* v : b->vols)
        for (int i = 0; i < 3; ++i) h = (h ^ v->desc.resolution[i]) * 1099511628211ull;
    for (int m : b->steps) h = (h ^ (uint64_t)m) * 1099511628211ull;
    char key[512];
    snprintf(key, sizeof(key), "sart_fused_batch|n%u|%016llx%s|type%d|%s", b->n, (unsigned long long)h,
             b->shape_key.c_str(), b->shadow, etcu_tune::device_tag(ctx->device).c_str());
    auto apply = [&](int c) {
        b->threads = c / 100;
        b->grid = (int)std::min<long long>((long long)(c % 100) * b->sms, (long long)b->total_units);
    };
    std::vector<int> cands;
    for (int bps = 1; bps <= std::min(b->per_sm512, 99); ++bps) cands.push_back(kFuseThreads * 100 + bps);
    for (int bps = 1; bps <= std::min(b->per_sm128, 99); ++bps) cands.push_back(128 * 100 + bps);
    int choice = etcu_tune::lookup(key);
    std::string log;
    if (std::find(cands.begin(), cands.end(), choice) == cands.end()) {
        std::vector<std::pair<void*, size_t>> saved;
        etcu_status s = ETCU_OK;
        for (etcu_volume* v : b->vols) {
            const size_t n = voxel_count(v->desc), bytes = n * 4 + (v->low ? n * 2 : 0);
            void* p = nullptr;
            if ((s = dalloc(ctx, &p, bytes)) != ETCU_OK) break;
            saved.emplace_back(p, bytes);
            CK(ctx, cudaMemcpyAsync(p, v->master, n * 4, cudaMemcpyDeviceToDevice, ctx->stream));
            if (v->low) CK(ctx, cudaMemcpyAsync((char*)p + n * 4, v->low, n * 2, cudaMemcpyDeviceToDevice, ctx->stream));
        }
        const int def_threads = b->threads, def_grid = b->grid;
        if (s == ETCU_OK)
            choice = etcu_tune::search(ctx->stream, cands, [&](int c) {
                apply(c);
                return issue_batch_iteration(b, ctx->stream) == ETCU_OK;
            }, 2, &log);
        for (size_t i = 0; i < saved.size(); ++i) {
            etcu_volume* v = b->vols[i];
            const size_t n = voxel_count(v->desc);
            cudaMemcpyAsync(v->master, saved[i].first, n * 4, cudaMemcpyDeviceToDevice, ctx->stream);
            if (v->low) cudaMemcpyAsync(v->low, (char*)saved[i].first + n * 4, n * 2, cudaMemcpyDeviceToDevice, ctx->stream);
        }
        CK(ctx, cudaStreamSynchronize(ctx->stream));
        for (auto& p : saved) dfree(ctx, p.first, p.second);
        if (s != ETCU_OK) return s;
        if (choice < 0) choice = def_threads * 100 + std::max(1, def_grid / std::max(1, b->sms));
        etcu_tune::store(key, choice);
    } else {
        log = " cached";
    }
    apply(choice);
    ctx->tune_log += std::string(key) + " " + std::to_string(choice) + log + "\n";
    CK(ctx, cudaMemsetAsync(b->d_resid, 0, sizeof(double) * b->n, ctx->stream));
    return check_batch_waits(b);
}

etcu_status batch_build(etcu_context* ctx, const etcu_batch_series* series, uint32_t n,
                        const etcu_recon_params* params, etcu_batch* b) {
    if (params->block_size != 1)
        return fail(ctx, ETCU_ERR_UNSUPPORTED, "batched series run SART (block size 1)");
    if (params->bp_samples > 1)
        return fail(ctx, ETCU_ERR_UNSUPPORTED, "batched series use one back-projection sample");
    if (params->sampling != ETCU_SAMPLING_Q8 && params->sampling != ETCU_SAMPLING_EXACT)
        return fail(ctx, ETCU_ERR_UNSUPPORTED, "batched series sample with ETCU_SAMPLING_Q8 or _EXACT");
    if ((int)params->order < 0 || (int)params->order > 3)
        return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "Illegal ProjectionSetType!");
    b->sampling = params->sampling;
    std::vector<FpArgs> fp(n);
    std::vector<BpArgs> bp(n);
    std::vector<BatchSeriesRec> recs;
    recs.reserve(n);
    bool all_fast2d = true, all_nocap = true;
    etcu_status s;
    for (uint32_t i = 0; i < n; ++i) {
        const etcu_batch_series& sr = series[i];
        etcu_volume* vol = sr.volume;
        if (!vol || !sr.views || !sr.host_projections || sr.n_views == 0)
            return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "series %u: NULL volume, views or projections", i);
        if (vol->ctx != ctx) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "series %u: volume of another context", i);
        if (vol->type == ETCU_VOXEL_HALF16 || vol->mask || vol->slabs.size() != 1)
            return fail(ctx, ETCU_ERR_UNSUPPORTED,
                        "series %u: batched series need an FP32 volume (or FP32 master), one sub-volume, no mask", i);
        const int shadow = vol->type == ETCU_VOXEL_F16_MASTER ? 1 : (vol->type == ETCU_VOXEL_BF16_MASTER ? 2 : 0);
        if (i > 0 && shadow != b->shadow)
            return fail(ctx, ETCU_ERR_UNSUPPORTED, "series %u: every series of a batch has the same voxel type", i);
        b->shadow = shadow;
        const SlabConst& slab = vol->slabs[0];
        const uint32_t W = sr.views[0].width, H = sr.views[0].height;
        for (uint32_t v = 0; v < sr.n_views; ++v) {
            if ((s = check_view(ctx, &sr.views[v])) != ETCU_OK) return s;
            if (sr.views[v].perspective || sr.views[v].width != W || sr.views[v].height != H)
                return fail(ctx, ETCU_ERR_UNSUPPORTED, "series %u: batched series need parallel views of one size", i);
        }
        const std::vector<uint32_t> order =
            projection_order(params->order, sr.n_views, params->skip, params->skip ? params->skip_count : 0);
        if (order.empty()) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "series %u: no projections left", i);
        std::vector<ViewConst> vc(sr.n_views);
        std::vector<float> pat(4 * (size_t)sr.n_views);
        float vs[3] = {slab.vs.x, slab.vs.y, slab.vs.z};
        for (uint32_t v = 0; v < sr.n_views; ++v) {
            float loc = 0.f;
            if (params->use_long_object_compensation)
                loc = traversal_length(sr.views[v], vol->desc.bbox_min, vol->desc.bbox_max);
            vc[v] = make_view_const(sr.views[v], slab, loc);
            if (!row_constant(vc[v]))
                return fail(ctx, ETCU_ERR_UNSUPPORTED, "series %u: batched series need views tilted about y", i);
            all_fast2d &= vc[v].fast2d != 0;
            std::string err;
            if (!sample_pattern(sr.views[v], vs, 1, pat.data() + 4 * (size_t)v, &err))
                return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "%s", err.c_str());
        }
        all_nocap &= slab.rx + slab.rz - 1 <= kMaxDdaIterations;
        // device copies: projections, view table, order, samples, padded (residual, length) image
        float* d_proj;
        ViewConst* d_views;
        uint32_t* d_order;
        float4* d_samples;
        const size_t P = (size_t)W * H;
        bool proj_owned;
        if ((s = stage_projections(ctx, sr.host_projections, nullptr, P * sr.n_views, params->projection_storage, false,
                                   [&](void** p, size_t bytes) { return batch_alloc(b, p, bytes); }, &d_proj,
                                   &proj_owned)) != ETCU_OK)
            return s;
        if ((s = batch_alloc(b, (void**)&d_views, vc.size() * sizeof(ViewConst))) != ETCU_OK) return s;
        if ((s = batch_alloc(b, (void**)&d_order, order.size() * sizeof(uint32_t))) != ETCU_OK) return s;
        if ((s = batch_alloc(b, (void**)&d_samples, pat.size() * sizeof(float))) != ETCU_OK) return s;
        CK(ctx, cudaMemcpyAsync(d_views, vc.data(), vc.size() * sizeof(ViewConst), cudaMemcpyHostToDevice, ctx->stream));
        CK(ctx, cudaMemcpyAsync(d_order, order.data(), order.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                ctx->stream));
        CK(ctx, cudaMemcpyAsync(d_samples, pat.data(), pat.size() * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
        const size_t pw = (size_t)W + 2 * kPad, ph = (size_t)H + 2 * kPad;
        const size_t pitch = pw, slot = pw * ph;
        float2* rl_base;
        if ((s = batch_alloc(b, (void**)&rl_base, slot * sizeof(float2))) != ETCU_OK) return s;
        CK(ctx, cudaMemsetAsync(rl_base, 0, slot * sizeof(float2), ctx->stream));
        float2* rl = rl_base + kPad * pitch + kPad;
        FpArgs& f = fp[i];
        f = FpArgs{};
        fill_fp_volume_ptrs(vol, slab, f);
        f.slab = slab;
        f.views = d_views;
        f.order = d_order;
        f.first = 0;
        f.W = (int)W;
        f.H = (int)H;
        f.samples = params->fp_samples == 0 ? 1 : (int)params->fp_samples;
        f.mode = kFpPairResidual;
        f.overwrite = 1;
        f.loc = params->use_long_object_compensation ? 1 : 0;
        f.rl = rl;
        f.rl_pitch = pitch;
        f.rl_slot = slot;
        f.real = d_proj;
        f.real_kind = params->projection_storage;
        f.resid_sq = nullptr;  // set below (per-series element of d_resid)
        BpArgs& g = bp[i];
        g = BpArgs{};
        fill_bp_volume_ptrs(vol, slab, g);
        g.slab = slab;
        g.views = d_views;
        g.order = d_order;
        g.first = 0;
        g.nviews = 1;
        g.rl = rl;
        g.rl_pitch = pitch;
        g.rl_slot = slot;
        g.W = (int)W;
        g.H = (int)H;
        g.lambda = params->lambda;  // block size 1 (BackProjectionKernel.cpp:94)
        g.samples = d_samples;
        g.nsamples = 1;
        {
            BatchSeriesRec rc{vol, slab, vc, std::vector<float4>(sr.n_views), d_views, d_order,
                              reinterpret_cast<const float4*>(d_samples), d_proj, W, H, (uint32_t)order.size()};
            for (uint32_t v = 0; v < sr.n_views; ++v)
                rc.hs[v] = make_float4(pat[4 * v], pat[4 * v + 1], pat[4 * v + 2], pat[4 * v + 3]);
            recs.push_back(std::move(rc));
        }
        b->vols.push_back(vol);
        b->steps.push_back((int)order.size());
        b->max_steps = std::max(b->max_steps, (int)order.size());
        b->max_w = std::max(b->max_w, (int)W);
        b->max_h = std::max(b->max_h, (int)H);
        b->max_rx = std::max(b->max_rx, slab.rx);
        b->max_ry = std::max(b->max_ry, slab.ry);
    }
    b->fp_path = !all_fast2d ? kFpPathGeneral : (all_nocap ? kFpPathXzNoCap : kFpPathXz);
    if ((s = batch_alloc(b, (void**)&b->d_resid, sizeof(double) * n)) != ETCU_OK) return s;
    for (uint32_t i = 0; i < n; ++i) fp[i].resid_sq = b->d_resid + i;
    if ((s = batch_alloc(b, (void**)&b->d_fp, sizeof(FpArgs) * n)) != ETCU_OK) return s;
    if ((s = batch_alloc(b, (void**)&b->d_bp, sizeof(BpArgs) * n)) != ETCU_OK) return s;
    if ((s = batch_alloc(b, (void**)&b->d_steps, sizeof(int) * n)) != ETCU_OK) return s;
    CK(ctx, cudaMemcpyAsync(b->d_fp, fp.data(), sizeof(FpArgs) * n, cudaMemcpyHostToDevice, ctx->stream));
    CK(ctx, cudaMemcpyAsync(b->d_bp, bp.data(), sizeof(BpArgs) * n, cudaMemcpyHostToDevice, ctx->stream));
    CK(ctx, cudaMemcpyAsync(b->d_steps, b->steps.data(), sizeof(int) * n, cudaMemcpyHostToDevice, ctx->stream));
    CK(ctx, cudaMemsetAsync(b->d_resid, 0, sizeof(double) * n, ctx->stream));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    if ((s = plan_batch_persistent(b, recs, params)) != ETCU_OK) return s;
    if (b->shadow && !b->persist)
        return fail(ctx, ETCU_ERR_UNSUPPORTED,
                    "batched series with a 16-bit shadow run the persistent fused iteration only (SART, one sample, "
                    "1/256 sampling, rows of an even number of voxels)");
    if (b->persist && ctx->autotune && (s = tune_batch(b)) != ETCU_OK) return s;
    b->launches = b->persist ? 1u : 2u * (uint32_t)b->max_steps;
    if (params->use_graph) {
        cudaStream_t cs = ctx->stream;
        CK(ctx, cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        etcu_status is = issue_batch_iteration(b, cs);
        cudaGraph_t gr = nullptr;
        cudaError_t e = cudaStreamEndCapture(cs, &gr);
        if (is != ETCU_OK) {
            if (gr) cudaGraphDestroy(gr);
            return is;
        }
        CK(ctx, e);
        b->graph = gr;
        CK(ctx, cudaGraphInstantiate(&b->exec, gr, 0));
    }
    return ETCU_OK;
}

}  // namespace

extern "C" etcu_status etcu_batch_create(etcu_context* ctx, const etcu_batch_series* series, uint32_t n_series,
                                         const etcu_recon_params* params, etcu_batch** out) {
    if (!ctx || !series || !params || !out) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    if (n_series == 0) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "no series");
    if (n_series > 65535) return fail(ctx, ETCU_ERR_UNSUPPORTED, "at most 65535 series per batch");
    std::unique_ptr<etcu_batch, void (*)(etcu_batch*)> b(new etcu_batch(), [](etcu_batch* p) {
        batch_free(p);
        delete p;
    });
    b->ctx = ctx;
    b->n = n_series;
    etcu_status s = batch_build(ctx, series, n_series, params, b.get());
    if (s != ETCU_OK) return s;
    *out = b.release();
    return ETCU_OK;
}

extern "C" etcu_status etcu_batch_destroy(etcu_batch* b) {
    if (!b) return ETCU_OK;
    batch_free(b);
    delete b;
    return ETCU_OK;
}

extern "C" etcu_status etcu_batch_run(etcu_batch* b, uint32_t iterations) {
    if (!b) return fail(nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL batch");
    etcu_context* ctx = b->ctx;
    for (uint32_t it = 0; it < iterations; ++it) {
        if (b->exec) {
            CK(ctx, cudaGraphLaunch(b->exec, ctx->stream));
        } else {
            etcu_status s = issue_batch_iteration(b, ctx->stream);
            if (s != ETCU_OK) return s;
        }
    }
    CKL(ctx);
    etcu_status s = check_batch_waits(b);
    // the fused iteration updates the FP32 masters only: bring the shadows up to date
    if (s == ETCU_OK && b->shadow && iterations > 0)
        for (etcu_volume* v : b->vols)
            if ((s = refresh_low_from_master(v)) != ETCU_OK) return s;
    return s;
}

extern "C" etcu_status etcu_batch_last_residual_sq(etcu_batch* b, double* out) {
    if (!b || !out) return fail(b ? b->ctx : nullptr, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    etcu_context* ctx = b->ctx;
    CK(ctx, cudaMemcpyAsync(out, b->d_resid, sizeof(double) * b->n, cudaMemcpyDeviceToHost, ctx->stream));
    CK(ctx, cudaStreamSynchronize(ctx->stream));
    return ETCU_OK;
}

extern "C" uint32_t etcu_batch_launches_per_iteration(const etcu_batch* b) { return b ? b->launches : 0; }

extern "C" etcu_status etcu_reconstruct(etcu_context* ctx, const etcu_volume_desc* desc, etcu_voxel_type type,
                                        const etcu_view* views, uint32_t n_views, const float* host_projections,
                                        const etcu_recon_params* params, uint32_t iterations,
                                        float* host_volume_inout) {
    if (!ctx || !host_volume_inout) return fail(ctx, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    etcu_volume* vol = nullptr;
    etcu_status s = etcu_volume_create(ctx, desc, type, 0.f, &vol);
    if (s != ETCU_OK) return s;
    etcu_recon* rec = nullptr;
    if ((s = etcu_volume_upload(vol, host_volume_inout)) == ETCU_OK &&
        (s = etcu_recon_create(vol, views, n_views, host_projections, params, &rec)) == ETCU_OK &&
        (s = etcu_recon_run(rec, iterations)) == ETCU_OK) {
        s = etcu_volume_download(vol, host_volume_inout);
    }
    etcu_recon_destroy(rec);
    etcu_volume_destroy(vol);
    return s;
}

// =============================================================== allocation-free view update
// Scratch of etcu_sart_view_update_noalloc: one interleaved (residual, length)
// image and the FP64 residual accumulator, in static device memory.
// (width + 2 kPad) x (height + 2 kPad) texels covers every detector of at most
// 1024 x 1024 pixels (1028 x 1028 = 1024^2 + 8208).
constexpr size_t kNoAllocScratchTexels = ETCU_NOALLOC_SCRATCH_TEXELS;
static_assert(kNoAllocScratchTexels >= (1024 + 2 * kPad) * (1024 + 2 * kPad), "scratch covers 1024^2 detectors");
static __device__ __align__(256) float2 g_noalloc_pairs[kNoAllocScratchTexels];
static __device__ __align__(256) double g_noalloc_resid[1];

namespace {
struct NoAllocScratch {
    float2* pairs = nullptr;
    double* resid = nullptr;
    void* context = nullptr;  // the driver context the addresses belong to
    bool ready = false;
};
NoAllocScratch g_noalloc[64];
std::mutex g_noalloc_mutex;
thread_local std::string g_noalloc_error;

etcu_status noalloc_fail(etcu_status st, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_noalloc_error = buf;
    g_create_error = buf;  // readable through etcu_last_error(NULL)
    return st;
}

// The calling thread's current driver context (cuCtxGetCurrent through the runtime's
// driver entry point, so the library needs no link against the driver library), or
// NULL when none is current or the entry point is unavailable.
void* current_driver_context() {
    using CtxGetCurrent = int (*)(void**);
    static CtxGetCurrent fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return (CtxGetCurrent)p;
    }();
    void* ctx = nullptr;
    if (!fn || fn(&ctx) != 0) return nullptr;
    return ctx;
}

// Device addresses of the static scratch for the current device: looked up once per
// device and looked up again when the device's context changed since (the addresses of
// a destroyed context are not valid in its successor).
etcu_status noalloc_scratch(int dev, NoAllocScratch& out) {
    if (dev < 0 || dev >= 64) return noalloc_fail(ETCU_ERR_UNSUPPORTED, "device %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    NoAllocScratch& s = g_noalloc[dev];
    void* ctx = current_driver_context();
    if (s.ready && (ctx == nullptr || ctx != s.context)) s.ready = false;
    if (!s.ready) {
        cudaError_t e = cudaGetSymbolAddress((void**)&s.pairs, g_noalloc_pairs);
        if (e != cudaSuccess)
            return noalloc_fail(ETCU_ERR_CUDA, "cudaGetSymbolAddress(scratch image) failed: %s", cudaGetErrorString(e));
        e = cudaGetSymbolAddress((void**)&s.resid, g_noalloc_resid);
        if (e != cudaSuccess)
            return noalloc_fail(ETCU_ERR_CUDA, "cudaGetSymbolAddress(residual) failed: %s", cudaGetErrorString(e));
        // the lookup made the device's primary context current if none was
        s.context = current_driver_context();
        s.ready = s.context != nullptr;
    }
    out = s;
    return ETCU_OK;
}
}  // namespace

extern "C" etcu_status etcu_sart_view_update_noalloc(const etcu_volume_desc* desc, float* d_volume,
                                                     const float* d_projection, const etcu_view* view,
                                                     uint32_t fp_samples, uint32_t bp_samples, float lambda,
                                                     void* cuda_stream, double* residual_sq) {
    if (!desc || !d_volume || !d_projection || !view)
        return noalloc_fail(ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    if (desc->subvolume_count > 1)
        return noalloc_fail(ETCU_ERR_UNSUPPORTED, "the allocation-free update takes a single sub-volume");
    if (view->width == 0 || view->height == 0)
        return noalloc_fail(ETCU_ERR_INVALID_ARGUMENT, "projection resolution must be non-zero");
    if ((uint64_t)view->width * view->height > ETCU_NOALLOC_MAX_PIXELS ||
        ((uint64_t)view->width + 2 * kPad) * ((uint64_t)view->height + 2 * kPad) > kNoAllocScratchTexels)
        return noalloc_fail(ETCU_ERR_INVALID_ARGUMENT,
                            "detector of %u x %u pixels exceeds the scratch of the allocation-free update "
                            "(at most %u pixels, and (width + 4) x (height + 4) <= %u texels)",
                            view->width, view->height, (unsigned)ETCU_NOALLOC_MAX_PIXELS,
                            (unsigned)ETCU_NOALLOC_SCRATCH_TEXELS);
    float mat[16];
    if (!projection_matrix(*view, mat)) return noalloc_fail(ETCU_ERR_INVALID_ARGUMENT, "matrix not invertible");
    if (desc->resolution[0] == 0 || desc->resolution[1] == 0 || desc->resolution[2] == 0)
        return noalloc_fail(ETCU_ERR_INVALID_ARGUMENT, "volume resolution must be non-zero");
    // the single sub-volume of VolumeProperties::setSubVolumeCount(1)
    SlabConst slab{};
    {
        float vs[3], ivs[3];
        for (int i = 0; i < 3; ++i) {
            vs[i] = (desc->bbox_max[i] - desc->bbox_min[i]) / (float)desc->resolution[i];
            ivs[i] = 1.0f / vs[i];
        }
        float smax[3] = {desc->bbox_min[0] + (float)desc->resolution[0] * vs[0],
                         desc->bbox_min[1] + (float)desc->resolution[1] * vs[1],
                         desc->bbox_min[2] + (float)desc->resolution[2] * vs[2]};
        slab.rx = (int)desc->resolution[0];
        slab.ry = (int)desc->resolution[1];
        slab.rz = (int)desc->resolution[2];
        slab.z0 = 0;
        slab.bmin = f4(desc->bbox_min);
        slab.bmax = f4(smax);
        slab.cmin = f4(desc->bbox_min);
        slab.cmax = f4(desc->bbox_max);
        slab.vs = f4(vs);
        slab.ivs = f4(ivs);
    }
    std::string err;
    float4 pattern[kMaxInlineSamples];
    if (!view->perspective) {
        if (bp_samples > (uint32_t)kMaxInlineSamples)
            return noalloc_fail(ETCU_ERR_UNSUPPORTED, "at most %d back-projection samples per voxel", kMaxInlineSamples);
        float vs[3] = {slab.vs.x, slab.vs.y, slab.vs.z};
        if (!sample_pattern(*view, vs, bp_samples, (float*)pattern, &err))
            return noalloc_fail(ETCU_ERR_INVALID_ARGUMENT, "%s", err.c_str());
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return noalloc_fail(ETCU_ERR_NO_DEVICE, "cudaGetDevice failed: %s", cudaGetErrorString(e));
    NoAllocScratch sc;
    etcu_status st = noalloc_scratch(dev, sc);
    if (st != ETCU_OK) return st;
    cudaStream_t stream = (cudaStream_t)cuda_stream;
    const int W = (int)view->width, H = (int)view->height;
    // the padded image of this call (its zero border included) starts from zero
    const size_t pitch = (size_t)W + 2 * kPad, rows = (size_t)H + 2 * kPad;
    float2* origin = sc.pairs + kPad * pitch + kPad;
    e = cudaMemsetAsync(sc.pairs, 0, pitch * rows * sizeof(float2), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(sc.resid, 0, sizeof(double), stream);
    if (e != cudaSuccess) return noalloc_fail(ETCU_ERR_CUDA, "cudaMemsetAsync failed: %s", cudaGetErrorString(e));
    // forward projection; the single slab overwrites every pixel of the scratch image
    FpArgs fa{};
    fa.vol = d_volume;
    fa.mask = nullptr;
    fa.slab = slab;
    fa.views = nullptr;
    fa.inline_view = make_view_const(*view, slab, 0.f);
    fa.order = nullptr;
    fa.first = 0;
    fa.W = W;
    fa.H = H;
    fa.samples = fp_samples == 0 ? 1 : (int)fp_samples;
    fa.mode = kFpPairResidual;
    fa.overwrite = 1;
    fa.loc = 0;
    fa.rl = origin;
    fa.rl_pitch = pitch;
    fa.rl_slot = pitch * rows;
    fa.real = d_projection;
    fa.resid_sq = sc.resid;
    launch_fp_m<float, false>(fa, fp_path(view->perspective != 0, fa.inline_view.fast2d != 0, slab), 1, stream);
    // back projection of the view with lambda / 1
    BpArgs ba{};
    ba.vol = d_volume;
    ba.shadow = nullptr;
    ba.mask = nullptr;
    ba.slab = slab;
    ba.views = nullptr;
    ba.inline_view = fa.inline_view;
    ba.order = nullptr;
    ba.first = 0;
    ba.nviews = 1;
    ba.rl = origin;
    ba.rl_pitch = pitch;
    ba.rl_slot = pitch * rows;
    ba.texs = nullptr;
    ba.inline_tex = 0;
    ba.W = W;
    ba.H = H;
    ba.lambda = lambda;
    ba.samples = nullptr;
    if (!view->perspective) {
        ba.nsamples = (int)bp_samples;
        for (uint32_t k = 0; k < bp_samples; ++k) ba.inline_samples[k] = pattern[k];
    } else {
        uint32_t res[3] = {(uint32_t)slab.rx, (uint32_t)slab.ry, (uint32_t)slab.rz};
        ba.persp_n = (int)perspective_sampling_factor(view->width, view->height, res, bp_samples);
    }
    if (view->perspective) launch_bp_t<true, false, 0, kSampleQ8>(ba, dev, stream);
    else if (bp_samples == 1 && row_constant(ba.inline_view)) launch_bp_sart<false, 0>(ba, ETCU_SAMPLING_Q8, stream);
    else launch_bp_t<false, false, 0, kSampleQ8>(ba, dev, stream);
    e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_fail(ETCU_ERR_CUDA, "launch failed: %s", cudaGetErrorString(e));
    if (residual_sq) {
        e = cudaMemcpyAsync(residual_sq, sc.resid, sizeof(double), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return noalloc_fail(ETCU_ERR_CUDA, "residual read-back failed: %s", cudaGetErrorString(e));
    }
    return ETCU_OK;
}
