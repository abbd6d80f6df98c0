// Host side of the learned warm start (C ABI etcu_warmstart_*): the 3-level 3-D conv
// encoder-decoder of learned.cuh, its buffers, tensor maps, forward pass, backward pass
// and Adam step.  Everything is stream-ordered on the owning context's stream.
//
// Network (3x3x3 convolutions, "same" size, ReLU after every convolution but the head):
//   level 1 (X, Y, Z):      e1a = conv(x, 1 -> 16)       e1b = conv(e1a, 16 -> 16)
//   level 2 (X/2 ...):      p1 = avgpool2(e1b)           e2a = conv(p1, 16 -> 32)   e2b = conv(e2a, 32 -> 32)
//   level 3 (X/4 ...):      p2 = avgpool2(e2b)           e3a = conv(p2, 32 -> 64)   e3b = conv(e3a, 64 -> 64)
//   level 2:                d2a = conv([up2(e3b), e2b], 96 -> 32)                   d2b = conv(d2a, 32 -> 32)
//   level 1:                d1a = conv([up2(d2b), e1b], 48 -> 16)                   d1b = conv(d1a, 16 -> 16)
//   head:                   out = v + scale * conv(d1b, 16 -> 1)      (x = v / scale, residual in volume units)
// Parameters (FP32 master, in this order per layer): W[27][cout][cin] with tap
// t = dz * 9 + dy * 3 + dx reading voxel (x + dx - 1, y + dy - 1, z + dz - 1), then b[cout].
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "ettention_b200.h"
#include "learned.cuh"
#include "tune.hpp"

int etcu_context_device_index(const etcu_context* ctx);
void etcu_context_set_error(etcu_context* ctx, const char* message);
int etcu_context_autotune(const etcu_context* ctx);
void etcu_context_tune_note(etcu_context* ctx, const std::string& line);

namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against the
// driver library, so the library still loads on machines without a GPU).
EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return (EncodeTiledFn)p;
    }();
    return fn;
}

struct Grid {
    int X, Y, Z;
    size_t plane() const { return (size_t)X * Y * Z; }
};

// NC8 bf16 tensor of C channels for `batch` items on a grid.
struct Tensor {
    __nv_bfloat16* p = nullptr;
    int C = 0;
    Grid g{};
};

struct LayerDef {
    int cin0, cin1;  // tensor channels of source 0 / 1 (cin1 = 0: one source)
    int cin_used0;   // real input channels of source 0 (1 for the first layer, whose tensor has 16)
    int cout;        // real output channels
    int npad;        // N of the forward MMA (>= cout, multiple of 16)
    int level;       // 1, 2 or 3
};

constexpr int kLayers = 11;
constexpr LayerDef kDefs[kLayers] = {
    {16, 0, 1, 16, 16, 1},  {16, 0, 16, 16, 16, 1}, {16, 0, 16, 32, 32, 2}, {32, 0, 32, 32, 32, 2},
    {32, 0, 32, 64, 64, 3}, {64, 0, 64, 64, 64, 3}, {64, 32, 64, 32, 32, 2}, {32, 0, 32, 32, 32, 2},
    {32, 16, 32, 16, 16, 1}, {16, 0, 16, 16, 16, 1}, {16, 0, 16, 1, 16, 1},
};

int cin_total(const LayerDef& d) { return d.cin_used0 + d.cin1; }
// The input gradient of a layer runs as one convolution of cin_total outputs, or, when
// that exceeds 64 (the 96-input decoder layer), as two: source 0's and source 1's.
int dx_split(const LayerDef& d) { return cin_total(d) > 64 ? d.cin0 : cin_total(d); }
size_t layer_params(const LayerDef& d) { return (size_t)27 * d.cout * cin_total(d) + d.cout; }
// Forward layers of 16 or 32 (padded) outputs that have a z-streamed form: all of those
// but the first, whose one input channel runs on the CUDA cores (the head's one output is
// padded to 16).
bool zfold_layer(int l) { return l > 0 && (kDefs[l].npad == 16 || kDefs[l].npad == 32); }

size_t total_params() {
    size_t n = 0;
    for (const auto& d : kDefs) n += layer_params(d);
    return n;
}

}  // namespace

struct etcu_warmstart {
    etcu_context* ctx = nullptr;
    cudaStream_t stream = nullptr;
    int device = 0, sms = 148;
    Grid g1{}, g2{}, g3{};
    int max_batch = 1;
    float scale = 1.f;
    size_t nparams = 0;
    size_t woff[kLayers] = {}, boff[kLayers] = {};
    std::vector<void*> allocs;
    // parameters
    float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
    __nv_bfloat16* wf[kLayers] = {};  // forward kernel layout
    __nv_bfloat16* wb[kLayers] = {};  // input-gradient kernel layout (input channels [0, dx_split))
    __nv_bfloat16* wb2[kLayers] = {}; // the rest of them, when the input gradient is split
    int adam_t = 0;
    // activations (level 1 / 2 / 3)
    Tensor x16, e1a, e1b, up1, d1a, d1b, dy16, gA1, gB1, gUp1, gSkip1;
    Tensor p1, e2a, e2b, up2, d2a, d2b, gA2, gB2, gUp2, gSkip2, dP1;
    Tensor p2, e3a, e3b, gA3, gB3, dP2;
    float* out = nullptr;      // fp32 network output of the last forward pass (training)
    float* partial = nullptr;  // weight-gradient partial sums
    size_t partial_floats = 0;
    unsigned* d_err = nullptr;
    double* d_loss = nullptr;
    std::string err;
    int loader = -1;  // convolution operand loads: -1 default (tensor copies), 0 tensor copies, 1 cp.async (ETCU_CONV_LOADER)
    // forward convolutions of 16 outputs as the z-streamed kernel with dz folded into N
    // (ws::conv_zfold_kernel; ETCU_CONV_ZFOLD=0 keeps them on conv_tc_kernel)
    int zfold = 1;
    __nv_bfloat16* wz[kLayers] = {};  // its weight layout
};

namespace {

etcu_status wfail(etcu_warmstart* w, etcu_status st, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    etcu_context_set_error(w ? w->ctx : nullptr, buf);
    return st;
}

#define WCK(w, call)                                                                                       \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess)                                                                             \
            return wfail(w, e_ == cudaErrorMemoryAllocation ? ETCU_ERR_OUT_OF_MEMORY : ETCU_ERR_CUDA,      \
                         "%s failed: %s", #call, cudaGetErrorString(e_));                                  \
    } while (0)

etcu_status walloc(etcu_warmstart* w, void** p, size_t bytes) {
    *p = nullptr;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return wfail(w, ETCU_ERR_OUT_OF_MEMORY, "device allocation of %zu bytes failed: %s", bytes,
                     cudaGetErrorString(e));
    }
    w->allocs.push_back(*p);
    return ETCU_OK;
}

etcu_status tensor(etcu_warmstart* w, Tensor& t, int C, const Grid& g, bool zero) {
    t.C = C;
    t.g = g;
    const size_t bytes = (size_t)w->max_batch * C * g.plane() * 2;
    etcu_status s = walloc(w, (void**)&t.p, bytes);
    if (s != ETCU_OK) return s;
    if (zero) WCK(w, cudaMemset(t.p, 0, bytes));
    return ETCU_OK;
}

// Tensor map of an NC8 tensor with box {8, bx, by, bz, bc}.
etcu_status make_map(etcu_warmstart* w, CUtensorMap* m, const Tensor& t, int batch, uint32_t bx, uint32_t by,
                     uint32_t bz, uint32_t bc) {
    EncodeTiledFn enc = encode_tiled();
    if (!enc) return wfail(w, ETCU_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled is not available");
    const cuuint64_t dims[5] = {8, (cuuint64_t)t.g.X, (cuuint64_t)t.g.Y, (cuuint64_t)t.g.Z,
                                (cuuint64_t)batch * (t.C / 8)};
    const cuuint64_t strides[4] = {16, (cuuint64_t)16 * t.g.X, (cuuint64_t)16 * t.g.X * t.g.Y,
                                   (cuuint64_t)16 * t.g.X * t.g.Y * t.g.Z};
    const cuuint32_t box[5] = {8, bx, by, bz, bc};
    const cuuint32_t es[5] = {1, 1, 1, 1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, (void*)t.p, dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return wfail(w, ETCU_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return ETCU_OK;
}

constexpr size_t kSmemBudget = 200 * 1024;      // weight-gradient kernel
constexpr size_t kConvSmemMax = 232448 - 1024 - 512;  // persistent convolution: stages + resident weights
constexpr size_t kResidentMax = 64 * 1024;       // weights kept in shared memory for the whole launch

template <int N, int TY>
etcu_status launch_conv_n(etcu_warmstart* w, const CUtensorMap& m0, const CUtensorMap& m1, ws::ConvArgs a,
                          int batch) {
    using SH = ws::ConvShape<N, TY>;
    const size_t wbytes = (size_t)a.nsteps * SH::kW;
    a.resident = wbytes <= kResidentMax ? 1 : 0;
    const size_t wres = a.resident ? (wbytes + 1023) & ~(size_t)1023 : 0;
    const size_t stage = (SH::kHalo + (a.resident ? 0 : SH::kW) + 1023) & ~(size_t)1023;
    const int smax = (int)std::min<size_t>(4, (kConvSmemMax - wres) / stage);
    if (smax < 1) return wfail(w, ETCU_ERR_UNSUPPORTED, "convolution stage of %zu bytes does not fit", stage);
    a.batch = batch;
    static std::atomic<unsigned long long> opted{0};
    if (w->device < 64 && !(opted.load() & (1ull << w->device))) {
        WCK(w, cudaFuncSetAttribute(ws::conv_tc_kernel<N, TY, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    232448));
        WCK(w, cudaFuncSetAttribute(ws::conv_tc_kernel<N, TY, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    232448));
        opted.fetch_or(1ull << w->device);
    }
    const int ntx = (a.X + ws::kTileX - 1) / ws::kTileX;
    const int nty = (a.Y + TY - 1) / TY;
    const long ntiles = (long)ntx * nty * a.Z * batch;
    const unsigned grid = (unsigned)std::min<long>(ntiles, w->sms);
    cudaError_t last = cudaSuccess;
    // choice = loader * 10 + stages (loader 0: one tensor copy per halo, 1: cp.async warps)
    auto launch = [&](int choice) {
        const int S = choice % 10, load = choice / 10;
        a.stages = S;
        // at least 120 KB, so that one CTA (and its tensor memory) owns each SM
        const size_t smem = std::max<size_t>(wres + (size_t)S * stage + (2 * S + 5) * 8 + 16 + 1024, 120 * 1024);
        if (load) ws::conv_tc_kernel<N, TY, 1><<<grid, ws::conv_threads<1>(), smem, w->stream>>>(m0, m1, a);
        else ws::conv_tc_kernel<N, TY, 0><<<grid, ws::conv_threads<0>(), smem, w->stream>>>(m0, m1, a);
        last = cudaGetLastError();
        return last == cudaSuccess;
    };
    int choice = (w->loader == 1 ? 10 : 0) + smax;
    if (w->loader < 0 && etcu_context_autotune(w->ctx)) {
        // autotuner: loader and ring stages of this convolution (the launch is idempotent)
        char key[256];
        snprintf(key, sizeof(key), "warmstart_conv|n%d|rows%d|%dx%dx%d|b%d|steps%d|res%d|%s", N, TY, a.X, a.Y, a.Z,
                 batch, a.nsteps, a.resident, etcu_tune::device_tag(w->device).c_str());
        int c = etcu_tune::lookup(key);
        if (c < 1 || c % 10 < 1 || c % 10 > smax || c / 10 > 1) {
            std::vector<int> cands;
            for (int load = 0; load <= 1; ++load)
                for (int k = 1; k <= smax; ++k) cands.push_back(load * 10 + k);
            std::string log;
            c = etcu_tune::search(w->stream, cands, launch, 3, &log);
            if (c < 1) c = choice;
            etcu_tune::store(key, c);
            etcu_context_tune_note(w->ctx, std::string(key) + " " + std::to_string(c) + log);
        }
        choice = c;
    }
    if (!launch(choice))
        return wfail(w, ETCU_ERR_CUDA, "convolution launch failed: %s", cudaGetErrorString(last));
    return ETCU_OK;
}

// The z-streamed convolution: 16 outputs with TY = 2 rows per tile, 32 outputs with TY = 1
// (four slices of 96 tensor-memory columns either way); work units of one (x tile, y tile)
// column over kZseg output slices.
constexpr int kZseg = 32;
constexpr int zfold_rows(int nout) { return nout == 16 ? 2 : 1; }

template <int NOUT>
etcu_status launch_zfold(etcu_warmstart* w, const CUtensorMap& m0, const CUtensorMap& m1, ws::ZfoldArgs a,
                         int batch) {
    constexpr int kZfoldRows = zfold_rows(NOUT);
    using SH = ws::ZfoldShape<NOUT, kZfoldRows>;
    const size_t wbytes = (size_t)a.nsteps * SH::kW;
    a.resident = wbytes <= kResidentMax ? 1 : 0;
    const size_t wres = a.resident ? (wbytes + 1023) & ~(size_t)1023 : 0;
    const size_t stage = (SH::kHalo + (a.resident ? 0 : SH::kW) + 1023) & ~(size_t)1023;
    const int S = (int)std::min<size_t>(4, (kConvSmemMax - wres) / stage);
    if (S < 2) return wfail(w, ETCU_ERR_UNSUPPORTED, "z-streamed convolution stage of %zu bytes does not fit", stage);
    a.batch = batch;
    a.stages = S;
    a.zseg = kZseg;
    static std::atomic<unsigned long long> opted{0};
    if (w->device < 64 && !(opted.load() & (1ull << w->device))) {
        WCK(w, cudaFuncSetAttribute(ws::conv_zfold_kernel<NOUT, kZfoldRows>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, 232448));
        opted.fetch_or(1ull << w->device);
    }
    const long units = (long)((a.X + ws::kTileX - 1) / ws::kTileX) * ((a.Y + kZfoldRows - 1) / kZfoldRows) *
                       ((a.Z + kZseg - 1) / kZseg) * batch;
    const unsigned grid = (unsigned)std::min<long>(units, w->sms);
    // at least 120 KB, so that one CTA (and its 512 tensor-memory columns) owns each SM
    const size_t smem = std::max<size_t>(wres + (size_t)S * stage + (2 * S + 9) * 8 + 16 + 1024, 120 * 1024);
    ws::conv_zfold_kernel<NOUT, kZfoldRows><<<grid, ws::kZfoldThreads, smem, w->stream>>>(m0, m1, a);
    WCK(w, cudaGetLastError());
    return ETCU_OK;
}

// Rows per tile of the persistent convolution by output width N (two accumulators of
// TY * N tensor-memory columns; halo ring and weights within shared memory).
int conv_rows(int n) { return n >= 64 ? 2 : 4; }

// Convolution of one or two sources into `n` channels (forward: weights wf, bias and
// ReLU; input gradient: weights wb, masks).
struct ConvCall {
    const Tensor* src0;
    const Tensor* src1;
    int nsteps0, nsteps1;
    const __nv_bfloat16* w;
    const float* bias;
    bool relu;
    int n;
    ws::ConvDst dst0{}, dst1{};
    int n0 = 0;
    bool head = false;
    const float* head_in = nullptr;
    float* head_out = nullptr;
    float head_scale = 1.f;
};

etcu_status conv(etcu_warmstart* w, const ConvCall& c, int batch) {
    const int TY = conv_rows(c.n);
    CUtensorMap m0, m1;
    etcu_status s = make_map(w, &m0, *c.src0, batch, ws::kHaloX, TY + 2, 3, 2);
    if (s != ETCU_OK) return s;
    s = make_map(w, &m1, c.src1 ? *c.src1 : *c.src0, batch, ws::kHaloX, TY + 2, 3, 2);
    if (s != ETCU_OK) return s;
    ws::ConvArgs a{};
    const Grid& g = c.src0->g;
    a.X = g.X;
    a.Y = g.Y;
    a.Z = g.Z;
    a.nsteps = c.nsteps0 + c.nsteps1;
    a.nkp0 = c.nsteps0;
    a.c8_0 = c.src0->C / 8;
    a.c8_1 = c.src1 ? c.src1->C / 8 : 0;
    a.p0 = c.src0->p;
    a.p1 = c.src1 ? c.src1->p : c.src0->p;
    a.w = c.w;
    a.bias = c.bias;
    a.relu = c.relu ? 1 : 0;
    a.head = c.head ? 1 : 0;
    a.dst0 = c.dst0;
    a.dst1 = c.dst1;
    a.n0 = c.n0 > 0 ? c.n0 : c.n;
    a.head_in = c.head_in;
    a.head_out = c.head_out;
    a.head_scale = c.head_scale;
    a.err = w->d_err;
    switch (c.n) {
    case 16: return launch_conv_n<16, 4>(w, m0, m1, a, batch);
    case 32: return launch_conv_n<32, 4>(w, m0, m1, a, batch);
    case 48: return launch_conv_n<48, 4>(w, m0, m1, a, batch);
    case 64: return launch_conv_n<64, 2>(w, m0, m1, a, batch);
    default: return wfail(w, ETCU_ERR_UNSUPPORTED, "no convolution kernel for %d output channels", c.n);
    }
}

ws::ConvDst dst(const Tensor& t, const Tensor* mask = nullptr) {
    ws::ConvDst d;
    d.ptr = t.p;
    d.mask = mask ? mask->p : nullptr;
    d.channels = t.C;
    return d;
}

template <int CIN>
etcu_status launch_wgrad_n(etcu_warmstart* w, const Tensor& in, const Tensor& dpre, int cout, int batch,
                           int* ranges_out) {
    const int mode = CIN == 16 ? 0 : (CIN == 32 ? 1 : 2);
    const int ny = mode == 2 ? 1 : 3, nz = mode == 0 ? 3 : 1;
    const int ngroups = mode == 0 ? 1 : (mode == 1 ? 3 : 9);
    CUtensorMap mi, md;
    etcu_status s = make_map(w, &mi, in, batch, ws::kHaloX, ny, nz, CIN / 8);
    if (s != ETCU_OK) return s;
    s = make_map(w, &md, dpre, batch, ws::kTileX, 1, 1, dpre.C / 8);
    if (s != ETCU_OK) return s;
    const Grid& g = in.g;
    const int ntiles = ((g.X + ws::kTileX - 1) / ws::kTileX) * g.Y * g.Z * batch;
    int ranges = std::max(1, std::min(ntiles, (w->sms + ngroups - 1) / ngroups));
    const uint32_t bbytes = (uint32_t)ws::kHaloX * ny * nz * 16u * (CIN / 8);
    const uint32_t stage = (16u * ws::kTileX * 16u + bbytes + 1023u) & ~1023u;
    int S = (int)std::max<size_t>(1, std::min<size_t>(4, kSmemBudget / stage));
    const size_t smem = (size_t)S * stage + (2 * S + 1) * 8 + 16 + 1024;
    const size_t need = (size_t)ranges * 27 * cout * CIN;
    if (need > w->partial_floats) return wfail(w, ETCU_ERR_STATE, "weight-gradient scratch too small");
    static std::atomic<unsigned long long> opted{0};
    if (w->device < 64 && !(opted.load() & (1ull << w->device))) {
        WCK(w, cudaFuncSetAttribute(ws::wgrad_tc_kernel<CIN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    227 * 1024));
        opted.fetch_or(1ull << w->device);
    }
    ws::WgradArgs a{};
    a.X = g.X;
    a.Y = g.Y;
    a.Z = g.Z;
    a.batch = batch;
    a.in_c8 = in.C / 8;
    a.out_c8 = dpre.C / 8;
    a.cout = cout;
    a.group_mode = mode;
    a.ranges = ranges;
    a.partial = w->partial;
    a.stages = S;
    a.err = w->d_err;
    ws::wgrad_tc_kernel<CIN><<<(unsigned)(ngroups * ranges), 128, smem, w->stream>>>(mi, md, a);
    WCK(w, cudaGetLastError());
    *ranges_out = ranges;
    return ETCU_OK;
}

// dW of one source of layer l (input channels [ci_off, ci_off + cin_used)).
etcu_status wgrad(etcu_warmstart* w, int l, const Tensor& in, int cin_used, int ci_off, const Tensor& dpre,
                  int batch) {
    const LayerDef& d = kDefs[l];
    int ranges = 0;
    etcu_status s;
    switch (in.C) {
    case 16: s = launch_wgrad_n<16>(w, in, dpre, d.cout, batch, &ranges); break;
    case 32: s = launch_wgrad_n<32>(w, in, dpre, d.cout, batch, &ranges); break;
    case 64: s = launch_wgrad_n<64>(w, in, dpre, d.cout, batch, &ranges); break;
    default: return wfail(w, ETCU_ERR_UNSUPPORTED, "no weight-gradient kernel for %d input channels", in.C);
    }
    if (s != ETCU_OK) return s;
    const int n = 27 * d.cout * cin_used;
    ws::wgrad_reduce_kernel<<<(n + 255) / 256, 256, 0, w->stream>>>(w->partial, ranges, d.cout, in.C, cin_used,
                                                                      w->grads + w->woff[l], cin_total(d), ci_off);
    WCK(w, cudaGetLastError());
    return ETCU_OK;
}

etcu_status bias_grad(etcu_warmstart* w, int l, const Tensor& dpre, int batch) {
    const int c8 = dpre.C / 8;
    dim3 grid((unsigned)std::max<size_t>(1, std::min<size_t>(256, (batch * dpre.g.plane() + 255) / 256)),
              (unsigned)c8);
    ws::channel_sum_kernel<<<grid, 256, 0, w->stream>>>(dpre.p, c8, batch, dpre.g.plane(), kDefs[l].cout,
                                                        w->grads + w->boff[l]);
    WCK(w, cudaGetLastError());
    return ETCU_OK;
}

unsigned blocks(size_t n, unsigned t = 256) { return (unsigned)((n + t - 1) / t); }

etcu_status relayout(etcu_warmstart* w) {
    for (int l = 0; l < kLayers; ++l) {
        const LayerDef& d = kDefs[l];
        const int nsteps_f = (d.cin0 + d.cin1) / 16;
        const int nf = nsteps_f * 27 * 2 * d.npad * 8;
        ws::relayout_forward_kernel<<<blocks(nf), 256, 0, w->stream>>>(w->params + w->woff[l], d.cout, cin_total(d),
                                                                       d.npad, nsteps_f, w->wf[l]);
        if (w->wz[l]) {
            const int nz = nsteps_f * 9 * 2 * 3 * d.npad * 8;
            ws::relayout_zfold_kernel<<<blocks(nz), 256, 0, w->stream>>>(w->params + w->woff[l], d.cout, cin_total(d),
                                                                         d.npad, nsteps_f, w->wz[l]);
        }
        if (l > 0) {
            const int nsteps_b = (d.cout + 15) / 16;
            const int n0 = dx_split(d), n1 = cin_total(d) - n0;
            const int nb0 = nsteps_b * 27 * 2 * n0 * 8;
            ws::relayout_backward_kernel<<<blocks(nb0), 256, 0, w->stream>>>(w->params + w->woff[l], d.cout,
                                                                             cin_total(d), 0, n0, nsteps_b, w->wb[l]);
            if (n1 > 0) {
                const int nb1 = nsteps_b * 27 * 2 * n1 * 8;
                ws::relayout_backward_kernel<<<blocks(nb1), 256, 0, w->stream>>>(
                    w->params + w->woff[l], d.cout, cin_total(d), n0, n1, nsteps_b, w->wb2[l]);
            }
        }
    }
    WCK(w, cudaGetLastError());
    return ETCU_OK;
}

#define WTRY(expr)                        \
    do {                                  \
        etcu_status s_ = (expr);          \
        if (s_ != ETCU_OK) return s_;     \
    } while (0)

// training: also store the BF16 input tensor the first layer's weight gradient reads.
etcu_status forward(etcu_warmstart* w, const float* d_in, float* d_out, int B, bool training = false) {
    const size_t p1n = w->g1.plane();
    if (training) {
        ws::prep_input_kernel<<<blocks((size_t)B * p1n), 256, 0, w->stream>>>(d_in, 1.f / w->scale, p1n, B,
                                                                              w->x16.p);
        WCK(w, cudaGetLastError());
    }
    auto fwd = [&](int l, const Tensor& s0, const Tensor* s1, const Tensor& out) {
        const LayerDef& d = kDefs[l];
        ConvCall c{};
        c.src0 = &s0;
        c.src1 = s1;
        c.nsteps0 = d.cin0 / 16;
        c.nsteps1 = d.cin1 / 16;
        c.w = w->wf[l];
        c.bias = w->params + w->boff[l];
        c.relu = true;
        c.n = d.npad;
        c.dst0 = dst(out);
        if (w->zfold && w->wz[l]) {  // 16 or 32 outputs: the z-streamed kernel
            const int rows = zfold_rows(d.npad);
            CUtensorMap m0, m1;
            WTRY(make_map(w, &m0, s0, B, ws::kHaloX, rows + 2, 1, 2));
            WTRY(make_map(w, &m1, s1 ? *s1 : s0, B, ws::kHaloX, rows + 2, 1, 2));
            ws::ZfoldArgs z{};
            z.X = s0.g.X;
            z.Y = s0.g.Y;
            z.Z = s0.g.Z;
            z.nsteps = c.nsteps0 + c.nsteps1;
            z.nkp0 = c.nsteps0;
            z.c8_0 = s0.C / 8;
            z.c8_1 = s1 ? s1->C / 8 : 0;
            z.w = w->wz[l];
            z.bias = c.bias;
            z.relu = 1;
            z.dst = c.dst0;
            z.err = w->d_err;
            return d.npad == 16 ? launch_zfold<16>(w, m0, m1, z, B) : launch_zfold<32>(w, m0, m1, z, B);
        }
        return conv(w, c, B);
    };
    // first layer (one input channel) on the CUDA cores
    const dim3 end_grid((w->g1.X + ws::kEndTx - 1) / ws::kEndTx, (w->g1.Y + ws::kEndTy - 1) / ws::kEndTy,
                        w->g1.Z * B);
    ws::conv_in_kernel<<<end_grid, 256, 0, w->stream>>>(d_in, 1.f / w->scale, w->g1.X, w->g1.Y, w->g1.Z, B,
                                                        w->params + w->woff[0], w->params + w->boff[0], w->e1a.p);
    WCK(w, cudaGetLastError());
    WTRY(fwd(1, w->e1a, nullptr, w->e1b));
    ws::pool_kernel<<<blocks((size_t)B * 2 * w->g2.plane()), 256, 0, w->stream>>>(w->e1b.p, w->g1.X, w->g1.Y,
                                                                                   w->g1.Z, B * 2, w->p1.p);
    WTRY(fwd(2, w->p1, nullptr, w->e2a));
    WTRY(fwd(3, w->e2a, nullptr, w->e2b));
    ws::pool_kernel<<<blocks((size_t)B * 4 * w->g3.plane()), 256, 0, w->stream>>>(w->e2b.p, w->g2.X, w->g2.Y,
                                                                                   w->g2.Z, B * 4, w->p2.p);
    WTRY(fwd(4, w->p2, nullptr, w->e3a));
    WTRY(fwd(5, w->e3a, nullptr, w->e3b));
    ws::upsample_kernel<<<blocks((size_t)B * w->g2.plane()), 256, 0, w->stream>>>(w->e3b.p, w->g2.X, w->g2.Y,
                                                                                       w->g2.Z, B * 8, w->up2.p);
    WTRY(fwd(6, w->up2, &w->e2b, w->d2a));
    WTRY(fwd(7, w->d2a, nullptr, w->d2b));
    ws::upsample_kernel<<<blocks((size_t)B * w->g1.plane() / 2), 256, 0, w->stream>>>(w->d2b.p, w->g1.X, w->g1.Y,
                                                                                       w->g1.Z, B * 4, w->up1.p);
    WTRY(fwd(8, w->up1, &w->e1b, w->d1a));
    WTRY(fwd(9, w->d1a, nullptr, w->d1b));
    // head (one output channel): out = v + scale * (conv(d1b) + b), as the z-streamed
    // tensor-core convolution (channel 0 of 16), or on the CUDA cores
    if (w->zfold && w->wz[10]) {
        CUtensorMap m0;
        WTRY(make_map(w, &m0, w->d1b, B, ws::kHaloX, zfold_rows(16) + 2, 1, 2));
        ws::ZfoldArgs z{};
        z.X = w->g1.X;
        z.Y = w->g1.Y;
        z.Z = w->g1.Z;
        z.nsteps = 1;
        z.nkp0 = 1;
        z.c8_0 = w->d1b.C / 8;
        z.w = w->wz[10];
        z.bias = w->params + w->boff[10];
        z.head = 1;
        z.head_in = d_in;
        z.head_out = d_out;
        z.head_scale = w->scale;
        z.err = w->d_err;
        return launch_zfold<16>(w, m0, m0, z, B);
    }
    ws::conv_head_kernel<<<end_grid, 256, 0, w->stream>>>(w->d1b.p, w->g1.X, w->g1.Y, w->g1.Z, B,
                                                          w->params + w->woff[10], w->params + w->boff[10], d_in,
                                                          w->scale, d_out);
    WCK(w, cudaGetLastError());
    return ETCU_OK;
}

etcu_status backward(etcu_warmstart* w, const float* d_in, const float* d_target, int B) {
    const size_t p1n = w->g1.plane();
    WCK(w, cudaMemsetAsync(w->grads, 0, w->nparams * sizeof(float), w->stream));
    WCK(w, cudaMemsetAsync(w->d_loss, 0, sizeof(double), w->stream));
    const float grad_scale = 2.f / (float)((double)B * p1n);
    ws::loss_grad_kernel<<<blocks((size_t)B * p1n), 256, 0, w->stream>>>(w->out, d_target, 1.f / w->scale,
                                                                          grad_scale, p1n, B, w->dy16.p, w->d_loss);
    WCK(w, cudaGetLastError());
    // input gradient of layer l from dPre_l into `out` (two outputs for the two-source layers)
    auto dx = [&](int l, const Tensor& dpre, const Tensor& out0, const Tensor* mask0, const Tensor* out1) {
        const LayerDef& d = kDefs[l];
        ConvCall c{};
        c.src0 = &dpre;
        c.src1 = nullptr;
        c.nsteps0 = (d.cout + 15) / 16;
        c.nsteps1 = 0;
        c.w = w->wb[l];
        c.bias = nullptr;
        c.relu = false;
        c.n = dx_split(d);
        c.dst0 = dst(out0, mask0);
        if (out1 && dx_split(d) == cin_total(d)) {  // both sources' gradients from one launch
            c.dst1 = dst(*out1);
            c.n0 = d.cin0;
            c.n = cin_total(d);
        }
        etcu_status st = conv(w, c, B);
        if (st != ETCU_OK || !out1 || dx_split(d) == cin_total(d)) return st;
        ConvCall c2 = c;  // source 1's input gradient
        c2.w = w->wb2[l];
        c2.n = cin_total(d) - dx_split(d);
        c2.dst0 = dst(*out1);
        return conv(w, c2, B);
    };
    // head (layer 10): dPre(d1b) = conv^T(dy) * [d1b > 0]
    WTRY(wgrad(w, 10, w->d1b, 16, 0, w->dy16, B));
    WTRY(bias_grad(w, 10, w->dy16, B));
    WTRY(dx(10, w->dy16, w->gA1, &w->d1b, nullptr));
    // layer 9: d1b = relu(conv(d1a))
    WTRY(wgrad(w, 9, w->d1a, 16, 0, w->gA1, B));
    WTRY(bias_grad(w, 9, w->gA1, B));
    WTRY(dx(9, w->gA1, w->gB1, &w->d1a, nullptr));
    // layer 8: d1a = relu(conv([up1, e1b]))
    WTRY(wgrad(w, 8, w->up1, 32, 0, w->gB1, B));
    WTRY(wgrad(w, 8, w->e1b, 16, 32, w->gB1, B));
    WTRY(bias_grad(w, 8, w->gB1, B));
    WTRY(dx(8, w->gB1, w->gUp1, nullptr, &w->gSkip1));
    // through the upsampling into d2b
    ws::upsample_backward_kernel<<<blocks((size_t)B * 4 * w->g2.plane()), 256, 0, w->stream>>>(
        w->gUp1.p, w->d2b.p, w->g2.X, w->g2.Y, w->g2.Z, B * 4, w->gA2.p);
    WCK(w, cudaGetLastError());
    // layer 7: d2b = relu(conv(d2a))
    WTRY(wgrad(w, 7, w->d2a, 32, 0, w->gA2, B));
    WTRY(bias_grad(w, 7, w->gA2, B));
    WTRY(dx(7, w->gA2, w->gB2, &w->d2a, nullptr));
    // layer 6: d2a = relu(conv([up2, e2b]))
    WTRY(wgrad(w, 6, w->up2, 64, 0, w->gB2, B));
    WTRY(wgrad(w, 6, w->e2b, 32, 64, w->gB2, B));
    WTRY(bias_grad(w, 6, w->gB2, B));
    WTRY(dx(6, w->gB2, w->gUp2, nullptr, &w->gSkip2));
    ws::upsample_backward_kernel<<<blocks((size_t)B * 8 * w->g3.plane()), 256, 0, w->stream>>>(
        w->gUp2.p, w->e3b.p, w->g3.X, w->g3.Y, w->g3.Z, B * 8, w->gA3.p);
    WCK(w, cudaGetLastError());
    // layer 5: e3b = relu(conv(e3a))
    WTRY(wgrad(w, 5, w->e3a, 64, 0, w->gA3, B));
    WTRY(bias_grad(w, 5, w->gA3, B));
    WTRY(dx(5, w->gA3, w->gB3, &w->e3a, nullptr));
    // layer 4: e3a = relu(conv(p2)); p2 = pool(e2b)
    WTRY(wgrad(w, 4, w->p2, 32, 0, w->gB3, B));
    WTRY(bias_grad(w, 4, w->gB3, B));
    WTRY(dx(4, w->gB3, w->dP2, nullptr, nullptr));
    ws::pool_backward_kernel<<<blocks((size_t)B * 4 * w->g2.plane()), 256, 0, w->stream>>>(
        w->dP2.p, w->gSkip2.p, w->e2b.p, w->g2.X, w->g2.Y, w->g2.Z, B * 4, w->gA2.p);
    WCK(w, cudaGetLastError());
    // layer 3: e2b = relu(conv(e2a))
    WTRY(wgrad(w, 3, w->e2a, 32, 0, w->gA2, B));
    WTRY(bias_grad(w, 3, w->gA2, B));
    WTRY(dx(3, w->gA2, w->gB2, &w->e2a, nullptr));
    // layer 2: e2a = relu(conv(p1)); p1 = pool(e1b)
    WTRY(wgrad(w, 2, w->p1, 16, 0, w->gB2, B));
    WTRY(bias_grad(w, 2, w->gB2, B));
    WTRY(dx(2, w->gB2, w->dP1, nullptr, nullptr));
    ws::pool_backward_kernel<<<blocks((size_t)B * 2 * w->g1.plane()), 256, 0, w->stream>>>(
        w->dP1.p, w->gSkip1.p, w->e1b.p, w->g1.X, w->g1.Y, w->g1.Z, B * 2, w->gA1.p);
    WCK(w, cudaGetLastError());
    // layer 1: e1b = relu(conv(e1a))
    WTRY(wgrad(w, 1, w->e1a, 16, 0, w->gA1, B));
    WTRY(bias_grad(w, 1, w->gA1, B));
    WTRY(dx(1, w->gA1, w->gB1, &w->e1a, nullptr));
    // layer 0: e1a = relu(conv(x))
    WTRY(wgrad(w, 0, w->x16, 1, 0, w->gB1, B));
    WTRY(bias_grad(w, 0, w->gB1, B));
    (void)d_in;
    return ETCU_OK;
}

etcu_status check_err(etcu_warmstart* w) {
    unsigned e = 0;
    WCK(w, cudaMemcpyAsync(&e, w->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, w->stream));
    WCK(w, cudaStreamSynchronize(w->stream));
    if (e) {
        cudaMemsetAsync(w->d_err, 0, sizeof(unsigned), w->stream);
        cudaStreamSynchronize(w->stream);
        return wfail(w, ETCU_ERR_CUDA, "a warm-start convolution gave up waiting for its operands (error word %u)",
                     e);
    }
    return ETCU_OK;
}

etcu_status check_batch(etcu_warmstart* w, uint32_t batch) {
    if (batch == 0 || (int)batch > w->max_batch)
        return wfail(w, ETCU_ERR_INVALID_ARGUMENT, "batch %u outside 1..%d", batch, w->max_batch);
    return ETCU_OK;
}

}  // namespace

extern "C" uint32_t etcu_warmstart_param_count(void) { return (uint32_t)total_params(); }

extern "C" etcu_status etcu_warmstart_layer_info(uint32_t layer, uint32_t out[6]) {
    if (layer >= (uint32_t)kLayers || !out) {
        etcu_context_set_error(nullptr, "layer index out of range");
        return ETCU_ERR_INVALID_ARGUMENT;
    }
    const LayerDef& d = kDefs[layer];
    size_t off = 0;
    for (uint32_t l = 0; l < layer; ++l) off += layer_params(kDefs[l]);
    out[0] = (uint32_t)d.cin_used0;
    out[1] = (uint32_t)d.cin1;
    out[2] = (uint32_t)d.cout;
    out[3] = (uint32_t)d.level;
    out[4] = (uint32_t)off;                                      // W offset in the parameter vector
    out[5] = (uint32_t)(off + (size_t)27 * d.cout * cin_total(d));  // b offset
    return ETCU_OK;
}

extern "C" etcu_status etcu_warmstart_create(etcu_context* ctx, const uint32_t resolution[3], uint32_t max_batch,
                                             etcu_warmstart** out) {
    if (!ctx || !resolution || !out) {
        etcu_context_set_error(ctx, "NULL argument");
        return ETCU_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    for (int i = 0; i < 3; ++i)
        if (resolution[i] < 4 || resolution[i] % 4 != 0 || resolution[i] > 4096) {
            etcu_context_set_error(ctx, "warm-start volumes need x, y, z multiples of 4 (4 .. 4096)");
            return ETCU_ERR_INVALID_ARGUMENT;
        }
    if (max_batch == 0 || max_batch > 64) {
        etcu_context_set_error(ctx, "max_batch must be 1 .. 64");
        return ETCU_ERR_INVALID_ARGUMENT;
    }
    std::unique_ptr<etcu_warmstart> w(new etcu_warmstart());
    w->ctx = ctx;
    w->stream = (cudaStream_t)etcu_context_stream(ctx);
    w->device = etcu_context_device_index(ctx);
    WCK(w.get(), cudaSetDevice(w->device));
    WCK(w.get(), cudaDeviceGetAttribute(&w->sms, cudaDevAttrMultiProcessorCount, w->device));
    w->max_batch = (int)max_batch;
    if (const char* env = getenv("ETCU_CONV_LOADER")) w->loader = atoi(env) ? 1 : 0;
    if (const char* env = getenv("ETCU_CONV_ZFOLD")) w->zfold = atoi(env) ? 1 : 0;
    w->g1 = Grid{(int)resolution[0], (int)resolution[1], (int)resolution[2]};
    w->g2 = Grid{w->g1.X / 2, w->g1.Y / 2, w->g1.Z / 2};
    w->g3 = Grid{w->g2.X / 2, w->g2.Y / 2, w->g2.Z / 2};
    w->nparams = total_params();
    size_t off = 0;
    for (int l = 0; l < kLayers; ++l) {
        w->woff[l] = off;
        w->boff[l] = off + (size_t)27 * kDefs[l].cout * cin_total(kDefs[l]);
        off += layer_params(kDefs[l]);
    }
    etcu_warmstart* p = w.get();
    WTRY(walloc(p, (void**)&p->params, p->nparams * 4));
    WTRY(walloc(p, (void**)&p->grads, p->nparams * 4));
    WTRY(walloc(p, (void**)&p->adam_m, p->nparams * 4));
    WTRY(walloc(p, (void**)&p->adam_v, p->nparams * 4));
    WCK(p, cudaMemset(p->params, 0, p->nparams * 4));
    WCK(p, cudaMemset(p->adam_m, 0, p->nparams * 4));
    WCK(p, cudaMemset(p->adam_v, 0, p->nparams * 4));
    size_t max_partial = 0;
    for (int l = 0; l < kLayers; ++l) {
        const LayerDef& d = kDefs[l];
        WTRY(walloc(p, (void**)&p->wf[l], (size_t)(d.cin0 + d.cin1) / 16 * 27 * 2 * d.npad * 8 * 2));
        if (zfold_layer(l))
            WTRY(walloc(p, (void**)&p->wz[l], (size_t)(d.cin0 + d.cin1) / 16 * 9 * 2 * 3 * d.npad * 8 * 2));
        if (l > 0) {
            const size_t per = (size_t)((d.cout + 15) / 16) * 27 * 2 * 8 * 2;
            WTRY(walloc(p, (void**)&p->wb[l], per * dx_split(d)));
            if (cin_total(d) > dx_split(d)) WTRY(walloc(p, (void**)&p->wb2[l], per * (cin_total(d) - dx_split(d))));
        }
        for (int cin : {d.cin0, d.cin1}) {
            if (cin == 0) continue;
            const int ngroups = cin == 16 ? 1 : (cin == 32 ? 3 : 9);
            const size_t r = (size_t)(p->sms + ngroups - 1) / ngroups;
            max_partial = std::max(max_partial, r * 27 * d.cout * cin);
        }
    }
    p->partial_floats = max_partial;
    WTRY(walloc(p, (void**)&p->partial, max_partial * 4));
    WTRY(walloc(p, (void**)&p->d_err, 64));
    WTRY(walloc(p, (void**)&p->d_loss, 64));
    WCK(p, cudaMemset(p->d_err, 0, 64));
    WTRY(walloc(p, (void**)&p->out, (size_t)p->max_batch * p->g1.plane() * 4));
    const Grid &g1 = p->g1, &g2 = p->g2, &g3 = p->g3;
    WTRY(tensor(p, p->x16, 16, g1, true));
    WTRY(tensor(p, p->e1a, 16, g1, false));
    WTRY(tensor(p, p->e1b, 16, g1, false));
    WTRY(tensor(p, p->up1, 32, g1, false));
    WTRY(tensor(p, p->d1a, 16, g1, false));
    WTRY(tensor(p, p->d1b, 16, g1, false));
    WTRY(tensor(p, p->dy16, 16, g1, true));
    WTRY(tensor(p, p->gA1, 16, g1, false));
    WTRY(tensor(p, p->gB1, 16, g1, false));
    WTRY(tensor(p, p->gUp1, 32, g1, false));
    WTRY(tensor(p, p->gSkip1, 16, g1, false));
    WTRY(tensor(p, p->p1, 16, g2, false));
    WTRY(tensor(p, p->e2a, 32, g2, false));
    WTRY(tensor(p, p->e2b, 32, g2, false));
    WTRY(tensor(p, p->up2, 64, g2, false));
    WTRY(tensor(p, p->d2a, 32, g2, false));
    WTRY(tensor(p, p->d2b, 32, g2, false));
    WTRY(tensor(p, p->gA2, 32, g2, false));
    WTRY(tensor(p, p->gB2, 32, g2, false));
    WTRY(tensor(p, p->gUp2, 64, g2, false));
    WTRY(tensor(p, p->gSkip2, 32, g2, false));
    WTRY(tensor(p, p->dP1, 16, g2, false));
    WTRY(tensor(p, p->p2, 32, g3, false));
    WTRY(tensor(p, p->e3a, 64, g3, false));
    WTRY(tensor(p, p->e3b, 64, g3, false));
    WTRY(tensor(p, p->gA3, 64, g3, false));
    WTRY(tensor(p, p->gB3, 64, g3, false));
    WTRY(tensor(p, p->dP2, 32, g3, false));
    WTRY(relayout(p));
    WCK(p, cudaStreamSynchronize(p->stream));
    *out = w.release();
    return ETCU_OK;
}

extern "C" etcu_status etcu_warmstart_destroy(etcu_warmstart* w) {
    if (!w) return ETCU_OK;
    cudaStreamSynchronize(w->stream);
    for (void* p : w->allocs) cudaFree(p);
    delete w;
    return ETCU_OK;
}

extern "C" etcu_status etcu_warmstart_set_params(etcu_warmstart* w, const float* host_params, float scale) {
    if (!w || !host_params) return wfail(w, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!(scale > 0.f)) return wfail(w, ETCU_ERR_INVALID_ARGUMENT, "scale must be positive");
    w->scale = scale;
    WCK(w, cudaMemcpyAsync(w->params, host_params, w->nparams * 4, cudaMemcpyHostToDevice, w->stream));
    WCK(w, cudaMemsetAsync(w->adam_m, 0, w->nparams * 4, w->stream));
    WCK(w, cudaMemsetAsync(w->adam_v, 0, w->nparams * 4, w->stream));
    w->adam_t = 0;
    WTRY(relayout(w));
    WCK(w, cudaStreamSynchronize(w->stream));
    return ETCU_OK;
}

extern "C" etcu_status etcu_warmstart_get_params(etcu_warmstart* w, float* host_params, float* scale) {
    if (!w || !host_params) return wfail(w, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    WCK(w, cudaMemcpyAsync(host_params, w->params, w->nparams * 4, cudaMemcpyDeviceToHost, w->stream));
    WCK(w, cudaStreamSynchronize(w->stream));
    if (scale) *scale = w->scale;
    return ETCU_OK;
}

extern "C" etcu_status etcu_warmstart_infer(etcu_warmstart* w, const float* d_in, float* d_out, uint32_t batch) {
    if (!w || !d_in || !d_out) return wfail(w, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    WTRY(check_batch(w, batch));
    return forward(w, d_in, d_out, (int)batch);
}

extern "C" etcu_status etcu_warmstart_gradients(etcu_warmstart* w, const float* d_in, const float* d_target,
                                                uint32_t batch, float* host_grads, double* loss) {
    if (!w || !d_in || !d_target) return wfail(w, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    WTRY(check_batch(w, batch));
    WTRY(forward(w, d_in, w->out, (int)batch, true));
    WTRY(backward(w, d_in, d_target, (int)batch));
    if (host_grads)
        WCK(w, cudaMemcpyAsync(host_grads, w->grads, w->nparams * 4, cudaMemcpyDeviceToHost, w->stream));
    double l = 0.0;
    WCK(w, cudaMemcpyAsync(&l, w->d_loss, sizeof(double), cudaMemcpyDeviceToHost, w->stream));
    WTRY(check_err(w));
    if (loss) *loss = l / ((double)batch * w->g1.plane());
    return ETCU_OK;
}

extern "C" etcu_status etcu_warmstart_train_step(etcu_warmstart* w, const float* d_in, const float* d_target,
                                                 uint32_t batch, float lr, double* loss) {
    if (!w || !d_in || !d_target) return wfail(w, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    WTRY(check_batch(w, batch));
    WTRY(forward(w, d_in, w->out, (int)batch, true));
    WTRY(backward(w, d_in, d_target, (int)batch));
    w->adam_t += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f / (1.f - std::pow(b1, (float)w->adam_t));
    const float c2 = 1.f / (1.f - std::pow(b2, (float)w->adam_t));
    ws::adam_kernel<<<blocks(w->nparams), 256, 0, w->stream>>>(w->params, w->grads, w->adam_m, w->adam_v,
                                                               (int)w->nparams, lr, b1, b2, 1e-8f, c1, c2);
    WCK(w, cudaGetLastError());
    WTRY(relayout(w));
    if (loss) {
        double l = 0.0;
        WCK(w, cudaMemcpyAsync(&l, w->d_loss, sizeof(double), cudaMemcpyDeviceToHost, w->stream));
        WTRY(check_err(w));
        *loss = l / ((double)batch * w->g1.plane());
    }
    return ETCU_OK;
}

extern "C" etcu_status etcu_warmstart_check(etcu_warmstart* w) {
    if (!w) return wfail(w, ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    return check_err(w);
}
