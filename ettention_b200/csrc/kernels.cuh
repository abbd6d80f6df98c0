// Device kernels of the B200 block-iterative reconstruction path (sm_100a).
//
// Reference semantics (paths relative to ettention/libReconstruction):
//   forward projection  ocl_src/ParallelBeamsForwardProjection.cl:12-57,
//                       ocl_src/PerspectiveBeamsForwardProjection.cl:13-52,
//                       ocl_src/DDARaytracer.hl:20-110, ocl_src/RayUtils.hl:7-35
//   back projection     ocl_src/ParallelBeamsBackProjection.cl:9-52,
//                       ocl_src/PerspectiveBeamsBackProjection.cl:10-71
//   residual / LOC      ocl_src/Compare.cl:1-9, ocl_src/VirtualProjection.cl:3-10
//   ray length          ocl_src/ComputeRayLength.cl:21-34
//
// Layout in HBM: volume x-fastest [z][y][x] (ocl_src/Math.hl:8-11), projection
// images row-major [v][u]; the per-block residual / ray-length pairs are one
// interleaved float2 image per block slot with a texture-aligned row pitch, so a
// single bilinear texture fetch returns both values.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cfloat>
#include <type_traits>
#include <stdint.h>

namespace etcu {

constexpr float kEps = 1e-4f;           // ocl_src/Math.hl:4
constexpr int kMaxDdaIterations = 2048; // DDARaytracer.hl:85-107: counter < 4096, bumped twice per step
constexpr int kMaxInlineSamples = 64;
// Zero border (texels) around every (residual, length) image: bilinear taps of
// any coordinate, clamped into [-kPad, W] x [-kPad, H], stay inside the
// allocation and read zeros outside the image, as the reference's
// clamp-to-border sampler does.
constexpr int kPad = 2;

struct ViewConst {
    float4 ray;       // normalised ray direction (parallel) / central direction (perspective)
    float4 inv;       // invertVectorSafely(ray)
    float4 source;
    float4 detector;
    float4 hpitch;
    float4 vpitch;
    float mat[16];    // column-major projection matrix
    float loc_length; // long-object constant length
    int perspective;
    int fast2d;       // parallel view with ray.y == 0, finite step differences, a decodable sub-volume
    int pad;
};

struct SlabConst {
    int rx, ry, rz;   // sub-volume resolution
    int z0;           // first z plane of the sub-volume in the full volume
    float4 bmin, bmax;  // sub-volume bounding box
    float4 cmin, cmax;  // complete bounding box
    float4 vs, ivs;     // voxel size and its reciprocal
};

// ---------------------------------------------------------------- helpers
// Setup arithmetic uses explicit round-to-nearest intrinsics so that no
// multiply-add is contracted; the result then matches the operation order of
// the OpenCL source step by step.
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float clsign(float x) { return x > 0.f ? 1.f : (x < 0.f ? -1.f : x); }
__device__ __forceinline__ float clclamp(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }

template <typename T> __device__ __forceinline__ float load_voxel(const T* p);
template <> __device__ __forceinline__ float load_voxel<float>(const float* p) { return __ldg(p); }
template <> __device__ __forceinline__ float load_voxel<__half>(const __half* p) { return __half2float(__ldg(p)); }
template <> __device__ __forceinline__ float load_voxel<__nv_bfloat16>(const __nv_bfloat16* p) {
    return __bfloat162float(__ldg(p));
}

template <typename T> __device__ __forceinline__ T store_cast(float v);
template <> __device__ __forceinline__ float store_cast<float>(float v) { return v; }
template <> __device__ __forceinline__ __half store_cast<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 store_cast<__nv_bfloat16>(float v) {
    return __float2bfloat16_rn(v);
}

__device__ __forceinline__ float mask_weight(const uint8_t* m) { return fdiv((float)__ldg(m), 255.0f); }

// RayUtils.hl:7-16
__device__ __forceinline__ void slab_test(float3 bmin, float3 bmax, float3 s, float3 inv, float& tin, float& tout) {
    float t0x = fmul(fsub(bmin.x, s.x), inv.x), t1x = fmul(fsub(bmax.x, s.x), inv.x);
    float t0y = fmul(fsub(bmin.y, s.y), inv.y), t1y = fmul(fsub(bmax.y, s.y), inv.y);
    float t0z = fmul(fsub(bmin.z, s.z), inv.z), t1z = fmul(fsub(bmax.z, s.z), inv.z);
    tin = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fminf(t0z, t1z));
    tout = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fmaxf(t0z, t1z));
}

__device__ __forceinline__ float3 inv_safe(float3 r) {
    float3 o = make_float3(fdiv(1.f, r.x), fdiv(1.f, r.y), fdiv(1.f, r.z));
    if (r.x == 0.f) o.x = -FLT_MAX;
    if (r.y == 0.f) o.y = -FLT_MAX;
    if (r.z == 0.f) o.z = -FLT_MAX;
    return o;
}

struct DdaStart {
    int ix, iy, iz;
    float3 res;  // remaining distance to the next border per axis
    float3 sd;   // step difference per axis
    int sx, sy, sz;
};

// DDARaytracer.hl:64-83: entry point, initial voxel, step differences and
// initial remaining distances.  Returns false when the ray misses the box.
__device__ __forceinline__ bool dda_setup(float3 src, float3 ray, float3 inv, const SlabConst& g, DdaStart& st) {
    float3 bmin = make_float3(g.bmin.x, g.bmin.y, g.bmin.z), bmax = make_float3(g.bmax.x, g.bmax.y, g.bmax.z);
    float tin, tout;
    slab_test(bmin, bmax, src, inv, tin, tout);
    if (!(fsub(tout, tin) > kEps)) return false;
    float px = clclamp(fadd(src.x, fmul(tin, ray.x)), bmin.x, bmax.x);
    float py = clclamp(fadd(src.y, fmul(tin, ray.y)), bmin.y, bmax.y);
    float pz = clclamp(fadd(src.z, fmul(tin, ray.z)), bmin.z, bmax.z);
    int ix = (int)fmul(fsub(px, bmin.x), g.ivs.x);
    int iy = (int)fmul(fsub(py, bmin.y), g.ivs.y);
    int iz = (int)fmul(fsub(pz, bmin.z), g.ivs.z);
    st.ix = min(max(ix, 0), g.rx - 1);
    st.iy = min(max(iy, 0), g.ry - 1);
    st.iz = min(max(iz, 0), g.rz - 1);
    float sgx = clsign(ray.x), sgy = clsign(ray.y), sgz = clsign(ray.z);
    st.sd = make_float3(fmul(fmul(g.vs.x, inv.x), sgx), fmul(fmul(g.vs.y, inv.y), sgy),
                        fmul(fmul(g.vs.z, inv.z), sgz));
    st.sx = (int)sgx; st.sy = (int)sgy; st.sz = (int)sgz;
    float rx = fmul(floorf(fmul(px, g.ivs.x)), g.vs.x);
    float ry = fmul(floorf(fmul(py, g.ivs.y)), g.vs.y);
    float rz = fmul(floorf(fmul(pz, g.ivs.z)), g.vs.z);
    rx = (ray.x > 0.f) ? fmul(fsub(fadd(rx, g.vs.x), px), inv.x) : fmul(fsub(rx, px), inv.x);
    ry = (ray.y > 0.f) ? fmul(fsub(fadd(ry, g.vs.y), py), inv.y) : fmul(fsub(ry, py), inv.y);
    rz = (ray.z > 0.f) ? fmul(fsub(fadd(rz, g.vs.z), pz), inv.z) : fmul(fsub(rz, pz), inv.z);
    if (ray.x == 0.f) rx = FLT_MAX;
    if (ray.y == 0.f) ry = FLT_MAX;
    if (ray.z == 0.f) rz = FLT_MAX;
    if (rx == 0.f) rx = st.sd.x;
    if (ry == 0.f) ry = st.sd.y;
    if (rz == 0.f) rz = st.sd.z;
    st.res = make_float3(rx, ry, rz);
    return true;
}

// General 3-D Amanatides-Woo walk (DDARaytracer.hl:84-108).  kLiteral keeps the
// reference's arithmetic step update step*sd + (1-step)*(res-dt) so that
// non-finite step differences propagate as in the reference; otherwise the
// update is an exact select.
template <typename VoxT, bool kMask, bool kLiteral>
__device__ __forceinline__ void dda_walk3(const DdaStart& st, const SlabConst& g, const VoxT* __restrict__ vol,
                                         const uint8_t* __restrict__ mask, float& acc, float& accl) {
    int ix = st.ix, iy = st.iy, iz = st.iz;
    float rx = st.res.x, ry = st.res.y, rz = st.res.z;
    const size_t plane = (size_t)g.rx * (size_t)g.ry;
    for (int it = 0; it < kMaxDdaIterations; ++it) {
        if ((unsigned)ix >= (unsigned)g.rx || (unsigned)iy >= (unsigned)g.ry || (unsigned)iz >= (unsigned)g.rz) break;
        float dt = fminf(fminf(rx, ry), rz);
        size_t idx = (size_t)iz * plane + (size_t)iy * (size_t)g.rx + (size_t)ix;
        acc = fmaf(dt, load_voxel(vol + idx), acc);
        if (kMask) accl = fmaf(dt, mask_weight(mask + idx), accl);
        else accl += dt;
        bool bx = rx <= ry && rx <= rz;
        bool by = ry < rx && ry <= rz;
        bool bz = rz < rx && rz < ry;
        if (kLiteral) {
            float fx = bx ? 1.f : 0.f, fy = by ? 1.f : 0.f, fz = bz ? 1.f : 0.f;
            rx = fadd(fmul(fx, st.sd.x), fmul(fsub(1.f, fx), fsub(rx, dt)));
            ry = fadd(fmul(fy, st.sd.y), fmul(fsub(1.f, fy), fsub(ry, dt)));
            rz = fadd(fmul(fz, st.sd.z), fmul(fsub(1.f, fz), fsub(rz, dt)));
        } else {
            rx = bx ? st.sd.x : fsub(rx, dt);
            ry = by ? st.sd.y : fsub(ry, dt);
            rz = bz ? st.sd.z : fsub(rz, dt);
        }
        ix += bx ? st.sx : 0;
        iy += by ? st.sy : 0;
        iz += bz ? st.sz : 0;
    }
}

// Parallel-beam walk for views tilted about y: ray.y == 0, so the y
// component stays FLT_MAX and never wins; the walk stays in one xz plane of
// the volume.  Valid (and bit-identical to dda_walk3) when the x and z step
// differences are finite.
//
// The loop is restructured for memory-level parallelism without changing
// the arithmetic: instead of re-testing the voxel index against the slab
// bounds every step, the walk decodes the current voxel from its offset,
// takes the number of steps each axis may still make before it leaves the
// slab (the same exit condition) and runs the smaller count unchecked,
// kUnroll steps at a time, issuing the kUnroll voxel loads before the kUnroll
// accumulations (which stay in walk order).  The decode needs ry >= 2 and
// (rz + 1) * rx * ry <= 2^32 (ViewConst::fast2d).
template <typename VoxT, bool kMask, bool kCapped = true, int kUnroll = 16>
__device__ __forceinline__ void dda_walk_xz(const DdaStart& st, const SlabConst& g, const VoxT* __restrict__ vol,
                                           const uint8_t* __restrict__ mask, float& acc, float& accl) {
    const unsigned plane = (unsigned)g.rx * (unsigned)g.ry;
    const VoxT* row = vol + (size_t)st.iy * (size_t)g.rx;
    const uint8_t* mrow = kMask ? mask + (size_t)st.iy * (size_t)g.rx : nullptr;
    const float sdx = st.sd.x, sdz = st.sd.z;
    const unsigned dx = (unsigned)st.sx, dz = (unsigned)st.sz * plane;  // two's-complement deltas
    int left = kMaxDdaIterations;
    unsigned off = (unsigned)st.iz * plane + (unsigned)st.ix;  // iz * plane + ix (row carries iy)
    float rx = st.res.x, rz = st.res.z;
    // One DDA step (DDARaytracer.hl:89-105): returns the segment length and the voxel it crossed.
    auto step = [&](float& dt, unsigned& at) {
        dt = fminf(rx, rz);
        const bool bx = rx <= rz;
        at = off;
        rx = bx ? sdx : fsub(rx, dt);
        rz = bx ? fsub(rz, dt) : sdz;
        off += bx ? dx : dz;
    };
    for (;;) {
        // Steps each axis may still take before it leaves the slab, from the current
        // voxel; neither axis (nor the loop cap) can run out within the next
        // min(nx, nz[, left]) steps, so they run without exit tests.
        const unsigned iz = off / plane, ix = off - iz * plane;
        const int nx = st.sx > 0 ? g.rx - (int)ix : (st.sx < 0 ? (int)ix + 1 : 0x7fffffff);
        const int nz = st.sz > 0 ? g.rz - (int)iz : (st.sz < 0 ? (int)iz + 1 : 0x7fffffff);
        if (nx <= 0 || nz <= 0 || ix >= (unsigned)g.rx || iz >= (unsigned)g.rz) break;
        int m = min(nx, nz);
        if (kCapped) m = min(m, left);
        if (m <= 0) break;
        if (kCapped) left -= m;
        for (; m >= kUnroll; m -= kUnroll) {
            float dts[kUnroll], vals[kUnroll], mws[kUnroll];
#pragma unroll
            for (int j = 0; j < kUnroll; ++j) {
                unsigned at;
                step(dts[j], at);
                vals[j] = load_voxel(row + at);
                if (kMask) mws[j] = mask_weight(mrow + at);
            }
#pragma unroll
            for (int j = 0; j < kUnroll; ++j) {
                acc = fmaf(dts[j], vals[j], acc);
                if (kMask) accl = fmaf(dts[j], mws[j], accl);
                else accl += dts[j];
            }
        }
        for (; m > 0; --m) {
            float dt;
            unsigned at;
            step(dt, at);
            acc = fmaf(dt, load_voxel(row + at), acc);
            if (kMask) accl = fmaf(dt, mask_weight(mrow + at), accl);
            else accl += dt;
        }
    }
}

// General 3-D walk with finite step differences, restructured like
// dda_walk_xz (per-axis step budgets, kUnroll loads in flight, accumulation
// in walk order).  Idx is the offset type (32-bit when the sub-volume has
// fewer than 2^32 voxels).
template <typename VoxT, bool kMask, typename Idx, int kUnroll = 4>
__device__ __forceinline__ void dda_walk3_fast(const DdaStart& st, const SlabConst& g, const VoxT* __restrict__ vol,
                                              const uint8_t* __restrict__ mask, float& acc, float& accl) {
    const Idx rowlen = (Idx)g.rx, plane = (Idx)g.rx * (Idx)g.ry;
    const Idx dx = (Idx)st.sx, dy = (Idx)st.sy * rowlen, dz = (Idx)st.sz * plane;
    int nx = st.sx > 0 ? g.rx - st.ix : (st.sx < 0 ? st.ix + 1 : 0x7fffffff);
    int ny = st.sy > 0 ? g.ry - st.iy : (st.sy < 0 ? st.iy + 1 : 0x7fffffff);
    int nz = st.sz > 0 ? g.rz - st.iz : (st.sz < 0 ? st.iz + 1 : 0x7fffffff);
    int left = kMaxDdaIterations;
    Idx off = (Idx)st.iz * plane + (Idx)st.iy * rowlen + (Idx)st.ix;
    float rx = st.res.x, ry = st.res.y, rz = st.res.z;
    const float sdx = st.sd.x, sdy = st.sd.y, sdz = st.sd.z;
    for (;;) {
        float dts[kUnroll], vals[kUnroll], mws[kUnroll];
        const int budget = min(min(nx, ny), min(nz, left));
        if (budget > kUnroll) {
            // Each step spends one step of one axis, so no axis can run out within
            // budget - 1 steps: walk a multiple of kUnroll of them without step budgets,
            // then recover the indices from the offset and renew the budgets.
            const int run = (budget - 1) / kUnroll * kUnroll;
            for (int s = 0; s < run; s += kUnroll) {
#pragma unroll
                for (int j = 0; j < kUnroll; ++j) {
                    const float dt = fminf(fminf(rx, ry), rz);
                    // rx <= ry && rx <= rz, and ry < rx && ry <= rz, from the minimum
                    const bool bx = rx == dt;
                    const bool by = !bx && ry == dt;
                    const bool bz = !bx && !by;
                    dts[j] = dt;
                    vals[j] = load_voxel(vol + off);
                    mws[j] = 0.f;
                    if (kMask) mws[j] = mask_weight(mask + off);
                    rx = bx ? sdx : fsub(rx, dt);
                    ry = by ? sdy : fsub(ry, dt);
                    rz = bz ? sdz : fsub(rz, dt);
                    off += bx ? dx : (by ? dy : dz);
                }
#pragma unroll
                for (int j = 0; j < kUnroll; ++j) {
                    acc = fmaf(dts[j], vals[j], acc);
                    if (kMask) accl = fmaf(dts[j], mws[j], accl);
                    else accl += dts[j];
                }
            }
            left -= run;
            const Idx iz = off / plane, rem = off - iz * plane, iy = rem / rowlen;
            const int ix = (int)(rem - iy * rowlen);
            nx = st.sx > 0 ? g.rx - ix : (st.sx < 0 ? ix + 1 : 0x7fffffff);
            ny = st.sy > 0 ? g.ry - (int)iy : (st.sy < 0 ? (int)iy + 1 : 0x7fffffff);
            nz = st.sz > 0 ? g.rz - (int)iz : (st.sz < 0 ? (int)iz + 1 : 0x7fffffff);
            continue;
        }
        {
#pragma unroll
            for (int j = 0; j < kUnroll; ++j) {
                const bool live = (nx > 0) & (ny > 0) & (nz > 0) & (left > 0);
                const float dt = fminf(fminf(rx, ry), rz);
                const bool bx = rx == dt;
                const bool by = !bx && ry == dt;
                const bool bz = !bx && !by;  // rz < rx && rz < ry for finite values
                dts[j] = live ? dt : 0.f;
                vals[j] = 0.f;
                mws[j] = 0.f;
                if (live) {
                    vals[j] = load_voxel(vol + off);
                    if (kMask) mws[j] = mask_weight(mask + off);
                }
                rx = bx ? sdx : fsub(rx, dt);
                ry = by ? sdy : fsub(ry, dt);
                rz = bz ? sdz : fsub(rz, dt);
                off += bx ? dx : (by ? dy : dz);
                nx -= bx ? 1 : 0;
                ny -= by ? 1 : 0;
                nz -= bz ? 1 : 0;
                left -= 1;
            }
        }
#pragma unroll
        for (int j = 0; j < kUnroll; ++j) {
            acc = fmaf(dts[j], vals[j], acc);
            if (kMask) accl = fmaf(dts[j], mws[j], accl);
            else accl += dts[j];
        }
        if (!((nx > 0) & (ny > 0) & (nz > 0) & (left > 0))) break;
    }
}

template <typename VoxT, bool kMask>
__device__ __forceinline__ void trace_ray(float3 src, float3 ray, float3 inv, bool fast2d, const SlabConst& g,
                                          const VoxT* vol, const uint8_t* mask, float& v, float& l) {
    v = 0.f;
    l = 0.f;
    DdaStart st;
    if (!dda_setup(src, ray, inv, g, st)) return;
    const bool small = (unsigned long long)g.rx * (unsigned long long)g.ry * (unsigned long long)g.rz < (1ull << 32);
    if (fast2d) {
        dda_walk_xz<VoxT, kMask>(st, g, vol, mask, v, l);
    } else if (isfinite(st.sd.x) && isfinite(st.sd.y) && isfinite(st.sd.z)) {
        if (small) dda_walk3_fast<VoxT, kMask, unsigned>(st, g, vol, mask, v, l);
        else dda_walk3_fast<VoxT, kMask, unsigned long long>(st, g, vol, mask, v, l);
    } else {
        dda_walk3<VoxT, kMask, true>(st, g, vol, mask, v, l);
    }
}

// Measured projection i stored as FP32 (kind 0), FP16 (1) or BF16 (2), widened exactly to float.
__device__ __forceinline__ float load_real(const float* base, int kind, size_t i) {
    if (kind == 1) return __half2float(reinterpret_cast<const __half*>(base)[i]);
    if (kind == 2) return __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(base)[i]);
    return base[i];
}

// ---------------------------------------------------------------- forward projection
enum FpMode : int {
    kFpSeparateAccumulate = 0,  // d_virtual += ..., d_traversal += ...   (ForwardProjectionKernel semantics)
    kFpPairAccumulate = 1,      // rl = (first ? 0 : rl) + (proj, len)    (non-final slab of a block)
    kFpPairResidual = 2         // rl = (b - ((first ? 0 : rl.x) + proj) [LOC], len)  (final slab)
};

struct FpArgs {
    const void* vol;            // sub-volume base (element type VoxT)
    const uint8_t* mask;        // sub-volume mask base or nullptr
    SlabConst slab;
    const ViewConst* views;     // device view table (nullptr: use inline_view)
    ViewConst inline_view;
    const uint32_t* order;      // iteration order (view ids), may be nullptr
    uint32_t first;             // order position of grid.z == 0
    int W, H, samples;
    int mode, overwrite, loc;
    float* out_v;               // mode 0
    float* out_l;
    float2* rl;                 // modes 1/2: slot p at rl + p * rl_slot, row pitch rl_pitch (float2 units)
    size_t rl_pitch, rl_slot;
    const float* real;          // mode 2: measured projections, view id * W * H (element type real_kind)
    int real_kind;              // 0 FP32, 1 FP16, 2 BF16 (load_real)
    double* resid_sq;           // mode 2: optional sum of residual^2 (FP64)
};

// kPath: kFpPathGeneral parallel rays (walk chosen per ray), kFpPathXz / kFpPathXzNoCap
// parallel views tilted about y (xz walk; the loop cap is dropped when the sub-volume
// cannot reach it, rx + rz - 1 <= 2048 steps), kFpPathPerspective.
enum FpPath : int { kFpPathGeneral = 0, kFpPathXz = 1, kFpPathXzNoCap = 2, kFpPathPerspective = 3 };

// Projection epilogue of one detector pixel (ForwardProjectionKernel /
// VirtualProjection.cl:8-9 / Compare.cl:8): normalise by the sub-ray count and
// write by mode.  Returns residual^2 (mode 2) or 0.
__device__ __forceinline__ double fp_store(const FpArgs& a, const ViewConst& vc, uint32_t vid, int p, int gx, int gy,
                                           float accv, float accl, float total) {
    float pv = fdiv(accv, total), pl = fdiv(accl, total);
    const size_t i = (size_t)gy * (size_t)a.W + (size_t)gx;
    if (a.mode == kFpSeparateAccumulate) {
        a.out_v[i] = fadd(a.out_v[i], pv);
        a.out_l[i] = fadd(a.out_l[i], pl);
        return 0.0;
    }
    float2* slot = a.rl + (size_t)p * a.rl_slot + (size_t)gy * a.rl_pitch + (size_t)gx;
    float2 prev = a.overwrite ? make_float2(0.f, 0.f) : *slot;
    float vv = fadd(prev.x, pv), ll = fadd(prev.y, pl);
    if (a.mode == kFpPairAccumulate) {
        *slot = make_float2(vv, ll);
        return 0.0;
    }
    if (a.loc) {  // VirtualProjection.cl:8-9
        vv = ll > kEps ? fdiv(fmul(vv, vc.loc_length), ll) : 0.f;
        ll = vc.loc_length;
    }
    float r = fsub(load_real(a.real, a.real_kind, (size_t)vid * (size_t)a.W * (size_t)a.H + i), vv);  // Compare.cl:8
    *slot = make_float2(r, ll);
    return (double)r * (double)r;
}

// FP64 warp reduction of the squared residuals, one atomic per warp (no block
// barrier, so warps whose rays finish early do not wait for the others).
__device__ __forceinline__ void fp_reduce_resid(const FpArgs& a, double r2) {
    if (a.mode == kFpPairResidual && a.resid_sq) {
        for (int o = 16; o > 0; o >>= 1) r2 += __shfl_down_sync(0xffffffffu, r2, o);
        if ((threadIdx.x & 31) == 0 && r2 != 0.0) atomicAdd(a.resid_sq, r2);
    }
}

// One detector pixel (gx, gy) of view slot p (order position first + p).
template <typename VoxT, bool kMask, int kPath>
__device__ __forceinline__ void fp_pixel(const FpArgs& a, uint32_t first, int p) {
    constexpr bool kPerspective = kPath == kFpPathPerspective;
    int gx, gy;
    if (kPerspective) {
        gx = blockIdx.x * 16 + (threadIdx.x & 15);
        gy = blockIdx.y * 8 + (threadIdx.x >> 4);
    } else {
        gx = blockIdx.x * blockDim.x + threadIdx.x;
        gy = blockIdx.y;
    }
    const uint32_t vid = a.order ? a.order[first + p] : (first + p);
    const ViewConst& vc = a.views ? a.views[vid] : a.inline_view;
    const bool active = gx < a.W && gy < a.H;
    const VoxT* vol = (const VoxT*)a.vol;
    const int S = a.samples;
    float accv = 0.f, accl = 0.f, total;
    if (active) {
        if (!kPerspective) {
            // ParallelBeamsForwardProjection.cl:12-24 sub-ray origins, :37-57 accumulation
            const float3 ray = make_float3(vc.ray.x, vc.ray.y, vc.ray.z);
            const float3 inv = make_float3(vc.inv.x, vc.inv.y, vc.inv.z);
            const float sdist = fdiv(1.f, (float)S), off = fdiv(sdist, 2.f);
            total = (float)(S * S);
            for (int sx = 0; sx < S; ++sx) {
                for (int sy = 0; sy < S; ++sy) {
                    float fx = fadd(fadd((float)gx, off), fmul(sdist, (float)sx));
                    float fy = fadd(fadd((float)gy, off), fmul(sdist, (float)sy));
                    float3 s = make_float3(fadd(fadd(vc.source.x, fmul(vc.hpitch.x, fx)), fmul(vc.vpitch.x, fy)),
                                           fadd(fadd(vc.source.y, fmul(vc.hpitch.y, fx)), fmul(vc.vpitch.y, fy)),
                                           fadd(fadd(vc.source.z, fmul(vc.hpitch.z, fx)), fmul(vc.vpitch.z, fy)));
                    float v = 0.f, l = 0.f;
                    if (kPath == kFpPathGeneral) {
                        trace_ray<VoxT, kMask>(s, ray, inv, vc.fast2d != 0, a.slab, vol, a.mask, v, l);
                    } else {
                        DdaStart st;
                        if (dda_setup(s, ray, inv, a.slab, st))
                            dda_walk_xz<VoxT, kMask, kPath == kFpPathXz>(st, a.slab, vol, a.mask, v, l);
                    }
                    accv += v;
                    accl += l;
                }
            }
        } else {
            // PerspectiveBeamsForwardProjection.cl:13-52
            const unsigned tot = (unsigned)(S * S);
            total = (float)tot;
            const float3 src = make_float3(vc.source.x, vc.source.y, vc.source.z);
            for (unsigned k = 0; k < tot; ++k) {
                float bx = fadd(fadd(vc.detector.x, fmul((float)gx, vc.hpitch.x)), fmul((float)gy, vc.vpitch.x));
                float by = fadd(fadd(vc.detector.y, fmul((float)gx, vc.hpitch.y)), fmul((float)gy, vc.vpitch.y));
                float bz = fadd(fadd(vc.detector.z, fmul((float)gx, vc.hpitch.z)), fmul((float)gy, vc.vpitch.z));
                unsigned dh = k % (unsigned)S, dv = k / (unsigned)S;
                float fh = fdiv(fadd((float)dh, 0.5f), (float)S), fv = fdiv(fadd((float)dv, 0.5f), (float)S);
                float px = fadd(fadd(bx, fmul(fh, vc.hpitch.x)), fmul(fv, vc.vpitch.x));
                float py = fadd(fadd(by, fmul(fh, vc.hpitch.y)), fmul(fv, vc.vpitch.y));
                float pz = fadd(fadd(bz, fmul(fh, vc.hpitch.z)), fmul(fv, vc.vpitch.z));
                float dx = fsub(px, src.x), dy = fsub(py, src.y), dz = fsub(pz, src.z);
                float n = __fsqrt_rn(fadd(fadd(fmul(dx, dx), fmul(dy, dy)), fmul(dz, dz)));
                float3 d = make_float3(fdiv(dx, n), fdiv(dy, n), fdiv(dz, n));
                float v, l;
                trace_ray<VoxT, kMask>(src, d, inv_safe(d), false, a.slab, vol, a.mask, v, l);
                accv += v;
                accl += l;
            }
        }
    }
    double r2 = 0.0;
    if (active) r2 = fp_store(a, vc, vid, p, gx, gy, accv, accl, total);
    fp_reduce_resid(a, r2);
}

// Minimum resident blocks: 7 for the xz walks, 8 for perspective rays (their gathers are
// latency-bound: 8 x 4 warps per SM cut the C3 forward projection by 19 % against 4),
// 4 otherwise.
template <typename VoxT, bool kMask, int kPath>
__global__ void __launch_bounds__(128, (kPath == kFpPathXz || kPath == kFpPathXzNoCap) ? 7
                                           : (kPath == kFpPathPerspective ? 8 : 4))
    forward_project_kernel(const __grid_constant__ FpArgs a) {
    fp_pixel<VoxT, kMask, kPath>(a, a.first, blockIdx.z);
}

// Batched tilt series: series s = blockIdx.z reads its arguments from table[s]
// and projects the view at order position `step` when it has one (steps[s] views);
// the grid covers the largest detector of the batch.
template <typename VoxT, bool kMask, int kPath>
__global__ void __launch_bounds__(128, (kPath == kFpPathXz || kPath == kFpPathXzNoCap) ? 7 : 4)
    forward_project_batch_kernel(const FpArgs* __restrict__ table, const int* __restrict__ steps, int step) {
    const int s = blockIdx.z;
    if (step >= steps[s]) return;
    const FpArgs& a = table[s];
    if ((int)(blockIdx.x * blockDim.x) >= a.W || (int)blockIdx.y >= a.H) return;
    fp_pixel<VoxT, kMask, kPath>(a, (uint32_t)step, 0);
}

// ---------------------------------------------------------------- back projection
// Residual / ray-length sampling of the back projector.
//   kSampleQ8:      bilinear with weights rounded (half up) to 1/256 and FP32 arithmetic --
//                   the GPU image path of the reference (BackProjectionKernel.cpp:146-163,
//                   CL_FILTER_LINEAR), which its golden volumes pin
//   kSampleExact:   FP32 weights, the reference's buffer path (ImageHandler.hl:20-40)
//   kSampleTexture: this GPU's texture unit (fast, but its FP32 filtering deviates from the
//                   reference's by ~1e-3 relative, so it is opt-in)
enum Sampling : int { kSampleQ8 = 0, kSampleExact = 1, kSampleTexture = 2 };

struct BpArgs {
    void* vol;                     // FP32 master / FP32 volume / half volume (sub-volume base)
    void* shadow;                  // 16-bit shadow written after the block (or nullptr)
    const uint8_t* mask;
    SlabConst slab;
    const ViewConst* views;        // view table by view id (nullptr: inline_view)
    ViewConst inline_view;
    const uint32_t* order;
    uint32_t first;
    int nviews;                    // views of the block, applied in order
    const float2* rl;              // slot p: interleaved (residual, length) at rl + p * rl_slot
    size_t rl_pitch, rl_slot;      // float2 units
    const cudaTextureObject_t* texs;  // per slot (kSampleTexture)
    cudaTextureObject_t inline_tex;
    int W, H;
    float lambda;                  // lambda / blockSize (BackProjectionKernel.cpp:94)
    const float4* samples;         // parallel: per view id, nsamples (x, y, z, chord); nullptr -> inline
    float4 inline_samples[kMaxInlineSamples];
    int nsamples;
    int persp_n;                   // perspective samples per dimension
    int use_min, use_max;
    float vmin, vmax;
};

// Per-view constants staged in shared memory by every back-projection block.
struct BpView {
    float mu[4], mv[4], mw[4];     // matrix rows: (m0, m4, m8, m12), (m1, m5, m9, m13), (m3, m7, m11, m15)
    float src[3];
    int affine;                    // mw == (0, 0, 0, 1): the divide by w is the identity
    int inside;                    // perspective back projection: every voxel centre of the block's
                                   // brick projects well inside the padded image (no clamps needed)
    cudaTextureObject_t tex;
};

__host__ __device__ constexpr size_t bp_smem_bytes(int nviews, int nsamples) {
    return ((size_t)nviews * sizeof(BpView) + 15) / 16 * 16 + (size_t)nviews * (size_t)nsamples * sizeof(float4);
}

__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// a / b to within one ulp: reciprocal estimate, one Newton correction of the quotient.
__device__ __forceinline__ float div_fast(float a, float b) {
    const float r = rcp_approx(b);
    const float q = a * r;
    const float e = fmaf(-b, q, a);
    return fmaf(e, r, q);
}

// Bilinear taps of the four texels around (x0, y0) from a padded image.
__device__ __forceinline__ void taps(const float2* __restrict__ row0, size_t pitch, int x0, float2& t00, float2& t10,
                                     float2& t01, float2& t11) {
    const float2* r1 = row0 + pitch;
    t00 = __ldg(row0 + x0);
    t10 = __ldg(row0 + x0 + 1);
    t01 = __ldg(r1 + x0);
    t11 = __ldg(r1 + x0 + 1);
}

// 1/256 weight of the texture filter: the fraction rounded half up to 8 bits.
__device__ __forceinline__ float q8_weight(float a) { return fmul(floorf(fadd(fmul(a, 256.f), 0.5f)), 1.f / 256.f); }

template <int kSampling>
__device__ __forceinline__ float2 blend(float a, float b, float2 t00, float2 t10, float2 t01, float2 t11) {
    if (kSampling == kSampleQ8) {
        const float w00 = fmul(fsub(1.f, a), fsub(1.f, b)), w10 = fmul(a, fsub(1.f, b));
        const float w01 = fmul(fsub(1.f, a), b), w11 = fmul(a, b);
        return make_float2(
            fadd(fadd(fadd(fmul(w00, t00.x), fmul(w10, t10.x)), fmul(w01, t01.x)), fmul(w11, t11.x)),
            fadd(fadd(fadd(fmul(w00, t00.y), fmul(w10, t10.y)), fmul(w01, t01.y)), fmul(w11, t11.y)));
    }
    // ImageHandler.hl:20-40: mix along x inside each row, then along y (zero rows mix to zero)
    const float2 p0 = make_float2(fadd(t00.x, fmul(fsub(t10.x, t00.x), a)), fadd(t00.y, fmul(fsub(t10.y, t00.y), a)));
    const float2 p1 = make_float2(fadd(t01.x, fmul(fsub(t11.x, t01.x), a)), fadd(t01.y, fmul(fsub(t11.y, t01.y), a)));
    return make_float2(fadd(p0.x, fmul(fsub(p1.x, p0.x), b)), fadd(p0.y, fmul(fsub(p1.y, p0.y), b)));
}

// Texel-space fraction and clamped base index of one coordinate.
template <int kSampling>
__device__ __forceinline__ void split_coord(float c, int n, int& i0, float& frac) {
    const float cs = fsub(c, 0.5f);
    const float cb = floorf(cs);
    frac = fminf(fsub(cs, cb), 0x1.fffffep-1f);  // OpenCL fract() clamp
    if (kSampling == kSampleQ8) frac = q8_weight(frac);
    i0 = min(max((int)cb, -kPad), n);
}

// img points at texel (0, 0) of a padded image with row pitch `pitch` (float2 units).
template <int kSampling>
__device__ __forceinline__ float2 sample_pair(const float2* __restrict__ img, size_t pitch, int W, int H,
                                              cudaTextureObject_t tex, float u, float v) {
    if (kSampling == kSampleTexture) return tex2D<float2>(tex, u + (float)kPad, v + (float)kPad);
    int x0, y0;
    float a, b;
    split_coord<kSampling>(u, W, x0, a);
    split_coord<kSampling>(v, H, y0, b);
    float2 t00, t10, t01, t11;
    taps(img + (ptrdiff_t)y0 * (ptrdiff_t)pitch, pitch, x0, t00, t10, t01, t11);
    return blend<kSampling>(a, b, t00, t10, t01, t11);
}

// Stages the block's view constants (and parallel sample patterns) in shared memory.
__device__ __forceinline__ void bp_stage(const BpArgs& a, BpView* sv, float4* ss, bool parallel) {
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y;
    for (int p = tid; p < a.nviews; p += nt) {
        const uint32_t vid = a.order ? a.order[a.first + p] : (a.first + p);
        const ViewConst& vc = a.views ? a.views[vid] : a.inline_view;
        BpView v;
        v.mu[0] = vc.mat[0]; v.mu[1] = vc.mat[4]; v.mu[2] = vc.mat[8]; v.mu[3] = vc.mat[12];
        v.mv[0] = vc.mat[1]; v.mv[1] = vc.mat[5]; v.mv[2] = vc.mat[9]; v.mv[3] = vc.mat[13];
        v.mw[0] = vc.mat[3]; v.mw[1] = vc.mat[7]; v.mw[2] = vc.mat[11]; v.mw[3] = vc.mat[15];
        v.src[0] = vc.source.x; v.src[1] = vc.source.y; v.src[2] = vc.source.z;
        v.affine = (v.mw[0] == 0.f && v.mw[1] == 0.f && v.mw[2] == 0.f && v.mw[3] == 1.f) ? 1 : 0;
        v.inside = 0;
        v.tex = a.texs ? a.texs[p] : a.inline_tex;
        sv[p] = v;
    }
    if (parallel) {
        const int ns = a.nsamples;
        for (int i = tid; i < a.nviews * ns; i += nt) {
            const int p = i / ns, k = i - p * ns;
            const uint32_t vid = a.order ? a.order[a.first + p] : (a.first + p);
            ss[i] = a.samples ? a.samples[(size_t)vid * ns + k] : a.inline_samples[k];
        }
    }
    __syncthreads();
}

template <int kStore>
__device__ __forceinline__ float bp_load(const BpArgs& a, size_t idx) {
    if (kStore == 1) return __half2float(((const __half*)a.vol)[idx]);
    return ((const float*)a.vol)[idx];
}

template <int kStore>
__device__ __forceinline__ void bp_store(const BpArgs& a, size_t idx, float val) {
    if (kStore == 1) ((__half*)a.vol)[idx] = __float2half_rn(val);
    else ((float*)a.vol)[idx] = val;
    if (kStore == 2) ((__half*)a.shadow)[idx] = __float2half_rn(val);
    if (kStore == 3) ((__nv_bfloat16*)a.shadow)[idx] = __float2bfloat16_rn(val);
}

constexpr int kBpZ = 8;  // voxels per thread along z (parallel)
// perspective: 16 z voxels per thread, so a column's per-view terms (matrix rows, source
// offsets, chord bounds) are formed once per 16 voxels; 64 registers at 4 blocks per SM
constexpr int kBpZPersp = 16;

// Row-constant view, one sample, 1/256 weights: the per-voxel sequence reduced to the
// column coordinate.  q = floor((u - 0.5) * 256 + 0.5) is the 1/256-rounded texel
// coordinate (u * 256 - 127.5 is exact for |u| < 2^15); x0 = floor(q / 256) and
// a = q / 256 - x0 give the same taps and weights as split_coord (a weight that rounds
// up to 1 becomes weight 0 on the next texel, which blends to the same value).
template <bool kMask>
__device__ __forceinline__ void bp_rowconst_q8_single(const BpArgs& a, const BpView& V, float4 s,
                                                      const float2* __restrict__ img, float cx, float cy,
                                                      const float* cz, int nzc, const float* mwt, float* val) {
    const float px = fadd(cx, s.x), py = fadd(cy, s.y);
    const float au = fadd(fmul(V.mu[0], px), fmul(V.mu[1], py));
    const float av = fadd(fmul(V.mv[0], px), fmul(V.mv[1], py));
    int y0;
    float b;
    split_coord<kSampleQ8>(fadd(av, V.mv[3]), a.H, y0, b);
    const float2* row0 = img + (ptrdiff_t)y0 * (ptrdiff_t)a.rl_pitch;
    const float2* row1 = row0 + a.rl_pitch;
    const float mu2 = V.mu[2], mu3 = V.mu[3], lam = a.lambda, d = s.w;
    const int W = a.W;
#pragma unroll
    for (int j = 0; j < kBpZ; ++j) {
        if (j < nzc) {
            const float pz = fadd(cz[j], s.z);
            const float u = fadd(fadd(au, fmul(mu2, pz)), mu3);
            const float qf = floorf(fmaf(u, 256.f, -127.5f));
            const float x0f = floorf(qf * (1.f / 256.f));
            const float ax = fmaf(qf, 1.f / 256.f, -x0f);
            const int x0 = min(max((int)x0f, -kPad), W);
            const float2 t00 = __ldg(row0 + x0), t10 = __ldg(row0 + x0 + 1);
            const float2 t01 = __ldg(row1 + x0), t11 = __ldg(row1 + x0 + 1);
            const float2 rl = blend<kSampleQ8>(ax, b, t00, t10, t01, t11);
            const float contrib = fmul(fmul(rl.x, lam), div_fast(d, rl.y));
            if (rl.y > kEps) val[j] = fadd(val[j], kMask ? fmul(mwt[j], contrib) : contrib);
        }
    }
}

// One view's update of kBpZ voxels of a column (ParallelBeamsBackProjection.cl:26-51).
// kRowConst: the detector row coordinate does not depend on x or z (affine matrix with
// m1 == m9 == 0, every view tilted about y), so the row taps are fixed per sample and
// only the column coordinate is evaluated per voxel -- in the same operations as the
// general form (the skipped terms are exact zeros).
template <bool kMask, int kSampling, bool kRowConst>
__device__ __forceinline__ void bp_parallel_view(const BpArgs& a, const BpView& V, const float4* __restrict__ smp,
                                                 const float2* __restrict__ img, float cx, float cy,
                                                 const float* cz, int nzc, const float* mwt, float* val) {
    const int ns = a.nsamples;
    if (kRowConst && kSampling == kSampleQ8 && ns == 1) {
        bp_rowconst_q8_single<kMask>(a, V, smp[0], img, cx, cy, cz, nzc, mwt, val);
        return;
    }
    if (ns == 1) {
        // one sample: used is 0 or 1, the average is the sample itself
        const float4 s = smp[0];
        const float px = fadd(cx, s.x), py = fadd(cy, s.y);
        const float au = fadd(fmul(V.mu[0], px), fmul(V.mu[1], py));
        const float av = fadd(fmul(V.mv[0], px), fmul(V.mv[1], py));
        const float aw = fadd(fmul(V.mw[0], px), fmul(V.mw[1], py));
        int y0 = 0;
        float b = 0.f;
        const float2* row0 = img;
        if (kRowConst) {
            split_coord<kSampling>(fadd(av, V.mv[3]), a.H, y0, b);
            row0 = img + (ptrdiff_t)y0 * (ptrdiff_t)a.rl_pitch;
        }
#pragma unroll
        for (int j = 0; j < kBpZ; ++j) {
            if (j < nzc) {
                const float pz = fadd(cz[j], s.z);
                float u = fadd(fadd(au, fmul(V.mu[2], pz)), V.mu[3]);
                float2 rl;
                if (kRowConst && kSampling != kSampleTexture) {
                    int x0;
                    float ax;
                    split_coord<kSampling>(u, a.W, x0, ax);
                    float2 t00, t10, t01, t11;
                    taps(row0, a.rl_pitch, x0, t00, t10, t01, t11);
                    rl = blend<kSampling>(ax, b, t00, t10, t01, t11);
                } else {
                    float v = fadd(fadd(av, fmul(V.mv[2], pz)), V.mv[3]);
                    if (!V.affine) {  // Matrix4x4.hl:54-58 divide by w
                        const float w = fadd(fadd(aw, fmul(V.mw[2], pz)), V.mw[3]);
                        u = fdiv(u, w);
                        v = fdiv(v, w);
                    }
                    rl = sample_pair<kSampling>(img, a.rl_pitch, a.W, a.H, V.tex, u, v);
                }
                const float contrib = fmul(fmul(rl.x, a.lambda), div_fast(s.w, rl.y));
                if (rl.y > kEps) val[j] = fadd(val[j], kMask ? fmul(mwt[j], contrib) : contrib);
            }
        }
        return;
    }
    float pv[kBpZ];
    unsigned used[kBpZ];
#pragma unroll
    for (int j = 0; j < kBpZ; ++j) {
        pv[j] = 0.f;
        used[j] = 0;
    }
    for (int k = 0; k < ns; ++k) {
        const float4 s = smp[k];
        const float px = fadd(cx, s.x), py = fadd(cy, s.y);
        const float au = fadd(fmul(V.mu[0], px), fmul(V.mu[1], py));
        const float av = fadd(fmul(V.mv[0], px), fmul(V.mv[1], py));
        const float aw = fadd(fmul(V.mw[0], px), fmul(V.mw[1], py));
        int y0 = 0;
        float b = 0.f;
        const float2* row0 = img;
        if (kRowConst) {
            split_coord<kSampling>(fadd(av, V.mv[3]), a.H, y0, b);
            row0 = img + (ptrdiff_t)y0 * (ptrdiff_t)a.rl_pitch;
        }
#pragma unroll
        for (int j = 0; j < kBpZ; ++j) {
            if (j < nzc) {
                const float pz = fadd(cz[j], s.z);
                float u = fadd(fadd(au, fmul(V.mu[2], pz)), V.mu[3]);
                float2 rl;
                if (kRowConst && kSampling != kSampleTexture) {
                    int x0;
                    float ax;
                    split_coord<kSampling>(u, a.W, x0, ax);
                    float2 t00, t10, t01, t11;
                    taps(row0, a.rl_pitch, x0, t00, t10, t01, t11);
                    rl = blend<kSampling>(ax, b, t00, t10, t01, t11);
                } else {
                    float v = fadd(fadd(av, fmul(V.mv[2], pz)), V.mv[3]);
                    if (!V.affine) {  // Matrix4x4.hl:54-58 divide by w
                        const float w = fadd(fadd(aw, fmul(V.mw[2], pz)), V.mw[3]);
                        u = fdiv(u, w);
                        v = fdiv(v, w);
                    }
                    rl = sample_pair<kSampling>(img, a.rl_pitch, a.W, a.H, V.tex, u, v);
                }
                const float contrib = fmul(fmul(rl.x, a.lambda), div_fast(s.w, rl.y));
                if (rl.y > kEps) {
                    pv[j] = fadd(pv[j], contrib);
                    used[j] += 1;
                }
            }
        }
    }
#pragma unroll
    for (int j = 0; j < kBpZ; ++j) {
        if (used[j] != 0) {
            const float num = kMask ? fmul(mwt[j], pv[j]) : pv[j];
            val[j] = fadd(val[j], used[j] == 1 ? num : div_fast(num, (float)used[j]));
        }
    }
}

// ParallelBeamsBackProjection.cl:9-52.  Each thread owns kBpZ voxels of one (x, y)
// column at a time and applies the block's views to them in order (no atomics); blocks
// walk z-chunks in a grid-stride loop so the view constants staged in shared memory
// serve many voxels.  Storage kStore: 0 FP32 volume, 1 half volume re-rounded after
// every view (reference half mode), 2 FP32 master + half shadow, 3 FP32 master + bf16 shadow.
template <bool kMask, int kStore, int kSampling>
__global__ void __launch_bounds__(256, 4) bp_parallel_kernel(const __grid_constant__ BpArgs a) {
    extern __shared__ __align__(16) unsigned char bp_smem[];
    BpView* sv = (BpView*)bp_smem;
    float4* ss = (float4*)(bp_smem + ((size_t)a.nviews * sizeof(BpView) + 15) / 16 * 16);
    bp_stage(a, sv, ss, true);
    const SlabConst& g = a.slab;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= g.rx || y >= g.ry) return;
    bool row_const = true;
    for (int p = 0; p < a.nviews; ++p)
        row_const &= sv[p].affine && sv[p].mv[0] == 0.f && sv[p].mv[2] == 0.f;
    const size_t plane = (size_t)g.rx * (size_t)g.ry;
    const float cx = fadd(g.bmin.x, fmul(fadd((float)x, 0.5f), g.vs.x));
    const float cy = fadd(g.bmin.y, fmul(fadd((float)y, 0.5f), g.vs.y));
    for (int z0 = blockIdx.z * kBpZ; z0 < g.rz; z0 += gridDim.z * kBpZ) {
        const int nzc = min(kBpZ, g.rz - z0);
        const size_t base = (size_t)z0 * plane + (size_t)y * (size_t)g.rx + (size_t)x;
        float val[kBpZ], mwt[kBpZ], cz[kBpZ];
#pragma unroll
        for (int j = 0; j < kBpZ; ++j) {
            val[j] = 0.f;
            mwt[j] = 1.f;
            cz[j] = fadd(g.bmin.z, fmul(fadd((float)(z0 + j), 0.5f), g.vs.z));  // VolumeGeometry.hl:17-20
            if (j < nzc) {
                val[j] = bp_load<kStore>(a, base + (size_t)j * plane);
                if (kMask) mwt[j] = mask_weight(a.mask + base + (size_t)j * plane);
            }
        }
        for (int p = 0; p < a.nviews; ++p) {
            const float2* img = a.rl + (size_t)p * a.rl_slot;
            const float4* smp = ss + p * a.nsamples;
            if (row_const) bp_parallel_view<kMask, kSampling, true>(a, sv[p], smp, img, cx, cy, cz, nzc, mwt, val);
            else bp_parallel_view<kMask, kSampling, false>(a, sv[p], smp, img, cx, cy, cz, nzc, mwt, val);
            if (kStore == 1) {
#pragma unroll
                for (int j = 0; j < kBpZ; ++j) val[j] = __half2float(__float2half_rn(val[j]));  // vstore_half per view
            }
        }
#pragma unroll
        for (int j = 0; j < kBpZ; ++j)
            if (j < nzc) bp_store<kStore>(a, base + (size_t)j * plane, val[j]);
    }
}

// ---- single-view, single-sample parallel back projection (SART's hot case) ----
// Paired FP32 helpers.  The compiler fuses a paired multiply into a following
// paired add (even with -fmad=false), so they are used only where no product
// feeds a sum; every product that feeds a sum is a scalar __fmul_rn.
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 splat(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// One voxel's sample from a detector row pair fixed by (row0, row0 + pitch, b):
// column split and blend exactly as sample_pair.
template <int kSampling>
__device__ __forceinline__ float2 row_sample(float u, const float2* __restrict__ row0, size_t pitch, float b, int W) {
    int x0;
    float ax;
    split_coord<kSampling>(u, W, x0, ax);
    float2 t00, t10, t01, t11;
    taps(row0, pitch, x0, t00, t10, t01, t11);
    return blend<kSampling>(ax, b, t00, t10, t01, t11);
}

// voxel + mask * r * lambda * (d / L) when L > eps (ParallelBeamsBackProjection.cl:40-50),
// the division refined from the reciprocal estimate.
__device__ __forceinline__ float sart_update(float v, float2 rl, float lam, float d, float mw, bool masked) {
    const float L = rl.y;
    const float rc = rcp_approx(L);
    float q = fmul(d, rc);
    const float e = fmaf(-L, q, d);
    q = fmaf(e, rc, q);
    float c = fmul(fmul(rl.x, lam), q);
    if (masked) c = fmul(mw, c);
    return L > kEps ? fadd(v, c) : v;
}

// ParallelBeamsBackProjection.cl:9-52 for one view with one sample per voxel and a
// detector row that depends only on y (every view tilted about y): each thread owns
// an (x, y) column over a z range, computes the view's row taps once and updates
// two voxels per iteration.  Same operations as bp_parallel_kernel.
template <bool kMask, int kStore, int kSampling>
__device__ __forceinline__ void bp_sart_row_column(const BpArgs& a, uint32_t first, int x, int y, int zb, int ze) {
    const SlabConst& g = a.slab;
    const uint32_t vid = a.order ? a.order[first] : first;
    const ViewConst& vc = a.views ? a.views[vid] : a.inline_view;
    const float4 s = a.samples ? a.samples[vid] : a.inline_samples[0];
    const float cx = fadd(g.bmin.x, fmul(fadd((float)x, 0.5f), g.vs.x));
    const float cy = fadd(g.bmin.y, fmul(fadd((float)y, 0.5f), g.vs.y));
    const float px = fadd(cx, s.x), py = fadd(cy, s.y);
    const float au = fadd(fmul(vc.mat[0], px), fmul(vc.mat[4], py));
    const float av = fadd(fmul(vc.mat[1], px), fmul(vc.mat[5], py));
    int y0;
    float b;
    split_coord<kSampling>(fadd(av, vc.mat[13]), a.H, y0, b);
    const float2* row0 = a.rl + (ptrdiff_t)y0 * (ptrdiff_t)a.rl_pitch;
    const float m8 = vc.mat[8], m12 = vc.mat[12], lam = a.lambda, d = s.w;
    const size_t plane = (size_t)g.rx * (size_t)g.ry;
    size_t idx = (size_t)zb * plane + (size_t)y * (size_t)g.rx + (size_t)x;
    for (int z = zb; z < ze; z += 2) {
        const bool two = z + 1 < ze;
        // VolumeGeometry.hl:17-20 voxel centres of z and z + 1
        const float pza = fadd(fadd(g.bmin.z, fmul(fadd((float)z, 0.5f), g.vs.z)), s.z);
        const float pzb = fadd(fadd(g.bmin.z, fmul(fadd((float)(z + 1), 0.5f), g.vs.z)), s.z);
        const float2 ra = row_sample<kSampling>(fadd(fadd(au, fmul(m8, pza)), m12), row0, a.rl_pitch, b, a.W);
        const float2 rb = row_sample<kSampling>(fadd(fadd(au, fmul(m8, pzb)), m12), row0, a.rl_pitch, b, a.W);
        float va = bp_load<kStore>(a, idx);
        float vb = two ? bp_load<kStore>(a, idx + plane) : 0.f;
        const float mwa = kMask ? mask_weight(a.mask + idx) : 1.f;
        const float mwb = kMask && two ? mask_weight(a.mask + idx + plane) : 1.f;
        va = sart_update(va, ra, lam, d, mwa, kMask);
        vb = sart_update(vb, rb, lam, d, mwb, kMask);
        bp_store<kStore>(a, idx, va);
        if (two) bp_store<kStore>(a, idx + plane, vb);
        idx += 2 * plane;
    }
}

template <bool kMask, int kStore, int kSampling>
__global__ void __launch_bounds__(256, 8) bp_sart_row_kernel(const __grid_constant__ BpArgs a) {
    const SlabConst& g = a.slab;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= g.rx || y >= g.ry) return;
    const int zper = (g.rz + gridDim.z - 1) / gridDim.z;
    const int zb = blockIdx.z * zper, ze = min(g.rz, zb + zper);
    if (zb >= ze) return;
    bp_sart_row_column<kMask, kStore, kSampling>(a, a.first, x, y, zb, ze);
}

// Batched tilt series (FP32 volumes, no mask): series s = blockIdx.z back projects the
// view at order position `step` when it has one; each thread owns a whole (x, y) column.
template <int kSampling>
__global__ void __launch_bounds__(256, 8)
    bp_sart_row_batch_kernel(const BpArgs* __restrict__ table, const int* __restrict__ steps, int step) {
    const int s = blockIdx.z;
    if (step >= steps[s]) return;
    const BpArgs& a = table[s];
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.slab.rx || y >= a.slab.ry) return;
    bp_sart_row_column<false, 0, kSampling>(a, (uint32_t)step, x, y, 0, a.slab.rz);
}

// ---- column-pipelined single-view back projection (SART's hot case, FP32 volume) ----
// A block owns items (y, z range) of the sub-volume; each thread owns groups of
// four consecutive x voxels of the item and walks them down z.  The volume rows
// come in through a per-thread ring of kBpColDepth 16-byte shared-memory slots
// filled by cp.async kBpColDepth - 1 rows ahead: a thread only ever reads the
// slots its own copies filled (cp.async.wait_group), so the walk needs no
// barrier and holds no prefetched values in registers; the four updated voxels
// leave as one 16-byte store.
// Sampling: the view's detector row coordinate is fixed for the item, so its row
// weight b is too, and the two detector rows are blended once per item,
// P[x] = (1 - b) * t0[x] + b * t1[x], into a staged window of tap pairs
// (P[x0], P[x0 + 1] - P[x0]) over the columns [x0lo, x0lo + ntaps) that the host
// bounds from the view and sub-volume corners.  Each voxel then takes one 16-byte
// shared load and one multiply-add per channel with the 1/256 weight a:
// P[x0] + a * (P[x0 + 1] - P[x0]).  This is the bilinear weighting of
// blend<kSampleQ8> (same coordinates, same 1/256 weights) evaluated in another
// order, and the update r * lambda * d / L takes the reciprocal estimate of L
// (within an ulp): each update is within a few ulps of the direct kernels'.  The
// window holds zeros outside the padded image, where the direct kernels clamp
// onto zero border texels, so no clamp is needed per voxel.  The 1/256 split of
// the column coordinate is integer work on the bits of fl_down(t + 1.5 * 2^23),
// which is 1.5 * 2^23 + floor(t) for |t| < 2^22.
struct BpColArgs {
    float* vol;                 // sub-volume base, x-fastest [z][y][x] (FP32, or the FP32 master)
    void* shadow;               // the 16-bit shadow of the master (kShadow 1: FP16, 2: BF16), same indexing
    SlabConst slab;
    const ViewConst* views;     // view table by view id (nullptr: inline_view)
    const uint32_t* order;
    uint32_t first;
    ViewConst inline_view;
    const float4* samples;      // one (x, y, z, chord) per view id; nullptr -> inline_sample
    float4 inline_sample;
    const float2* rl;           // texel (0, 0) of the padded (residual, length) image
    size_t rl_pitch;            // float2 units
    int W, H;
    float lambda;
    int x0lo, ntaps;            // staged tap pairs: columns x0lo .. x0lo + ntaps - 1
    int zper;                   // z rows per item
    int zchunks;                // items per y
};

constexpr int kBpColThreads = 256;
constexpr int kBpColDepth = 8;  // ring slots per thread: rows in flight + the one being updated

// Tap pair e sits at index e + e / 8 (one 16-byte pad per 8 entries): the lanes of a
// warp read entries about 4 cos(theta) apart (four x voxels per thread), which the
// pad spreads over distinct shared-memory banks.
__host__ __device__ constexpr int bp_col_tap_slots(int ntaps) { return ntaps + ntaps / 8 + 1; }

// row-blended tap pairs, per-z term, per-thread rings of kGroups 16-byte slots
__host__ __device__ constexpr size_t bp_col_smem_bytes(int rz, int ntaps, int groups) {
    return (size_t)bp_col_tap_slots(ntaps) * 16 + ((size_t)rz * 4 + 15) / 16 * 16 +
           (size_t)kBpColDepth * (size_t)groups * kBpColThreads * 16;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// The float 1 + k 2^-15 for k = bits & 255: one byte permute puts k in bits 8..15 under
// the exponent of 1 (bytes 3, 2, 0 from 0x3F800000).  The perspective back projector's
// weights; in the fused SART step the shift and mask-or of q8_tap_bits measured faster.
__device__ __forceinline__ float q8_k1(unsigned bits) { return __uint_as_float(__byte_perm(bits, 0x3F800000u, 0x7604)); }

// The 1/256 weights k / 256 from two q8_k1 values: 128 (1 + k 2^-15) - 128, exact.
__device__ __forceinline__ float2 q8_weight2(float2 k1) { return fma2(k1, splat(128.f), splat(-128.f)); }

// Column tap of one voxel from f = fl_down(t + 1.5 * 2^23) = 1.5 * 2^23 + floor(t),
// t = u * 256 - 127.5 (exact): tap-pair index x0 - x0lo and 1 + a, where
// a = (floor(t) mod 256) / 256 is the 1/256 weight (exact).
__device__ __forceinline__ void q8_tap_bits(float f, int x0lo, int& e, float& a1) {
    const int bits = __float_as_int(f);
    e = (bits >> 8) - ((0x4B400000 >> 8) + x0lo);
    a1 = __int_as_float(((bits << 15) & 0x007F8000) | 0x3F800000);
}

// kFull: every thread owns all kCols columns (rx == kCols * kBpColThreads).
// kGroups: 4-voxel x groups per thread (rx <= 4 * kGroups * kBpColThreads, rx % 4 == 0).
template <int kGroups, int kShadow = 0>
__global__ void __launch_bounds__(kBpColThreads, 4) bp_sart_column_kernel(const __grid_constant__ BpColArgs a) {
    extern __shared__ __align__(16) unsigned char bp_col_smem[];
    const SlabConst& g = a.slab;
    const int rx = g.rx, ry = g.ry, rz = g.rz, tid = threadIdx.x;
    const int ntaps = a.ntaps, x0lo = a.x0lo;
    float4* taps = (float4*)bp_col_smem;
    float* K = (float*)(taps + bp_col_tap_slots(ntaps));
    // slot (ring row r, group k) of this thread: ring[(r * kGroups + k) * kBpColThreads + tid]
    float4* ring = (float4*)(bp_col_smem + (size_t)bp_col_tap_slots(ntaps) * 16 + ((size_t)rz * 4 + 15) / 16 * 16);
    const float4* my = ring + tid;
    const uint32_t my_s = smem_addr(my);
    constexpr uint32_t kSlotBytes = kGroups * kBpColThreads * 16, kGroupBytes = kBpColThreads * 16;

    const uint32_t vid = a.order ? a.order[a.first] : a.first;
    const ViewConst& vc = a.views ? a.views[vid] : a.inline_view;
    const float4 s = a.samples ? a.samples[vid] : a.inline_sample;

    // ParallelBeamsBackProjection.cl coordinate terms, in the kernel's operation order
    for (int z = tid; z < rz; z += kBpColThreads)
        K[z] = fmul(vc.mat[8], fadd(fadd(g.bmin.z, fmul(fadd((float)z, 0.5f), g.vs.z)), s.z));
    float A[kGroups][4];
    bool on[kGroups];
#pragma unroll
    for (int k = 0; k < kGroups; ++k) {
        const int x4 = 4 * (tid + k * kBpColThreads);
        on[k] = x4 < rx;
#pragma unroll
        for (int j = 0; j < 4; ++j)
            A[k][j] = fmul(vc.mat[0], fadd(fadd(g.bmin.x, fmul(fadd((float)(x4 + j), 0.5f), g.vs.x)), s.x));
    }
    const float lamd = fmul(a.lambda, s.w);
    const float2 m12 = splat(vc.mat[12]);
    const float px0 = fadd(fadd(g.bmin.x, fmul(0.5f, g.vs.x)), s.x);
    const size_t plane = (size_t)rx * (size_t)ry;
    const float2 zero = make_float2(0.f, 0.f);
    const int items = ry * a.zchunks;

    // Fetch cursor: walks the rows of this block's items in the order they are
    // updated, one row (or, past the last row, nothing) per commit group, so the
    // j-th row updated is in the j-th group; kBpColDepth - 1 groups run ahead.
    int fit = blockIdx.x, fz = 0, fz1 = 0, ws = 0;
    const float* src = nullptr;
    auto start_item = [&](int i) {
        const int iy = i / a.zchunks;
        fz = (i - iy * a.zchunks) * a.zper;
        fz1 = min(rz, fz + a.zper);
        src = a.vol + ((size_t)fz * ry + iy) * rx + 4 * tid;
    };
    if (fit < items) start_item(fit);
    auto fetch = [&]() {
        if (fit < items) {
#pragma unroll
            for (int k = 0; k < kGroups; ++k)
                if (on[k]) cp_async16(my_s + (uint32_t)ws * kSlotBytes + k * kGroupBytes, src + 4 * k * kBpColThreads);
            ws = (ws + 1) & (kBpColDepth - 1);
            src += plane;
            if (++fz == fz1) {
                fit += gridDim.x;
                if (fit < items) start_item(fit);
            }
        }
        cp_async_commit();
    };
    for (int i = 0; i < kBpColDepth - 1; ++i) fetch();

    int rs = 0;  // read slot
    for (int it = blockIdx.x; it < items; it += gridDim.x) {
        const int y = it / a.zchunks;
        const int z0 = (it - y * a.zchunks) * a.zper, z1 = min(rz, z0 + a.zper);
        // the item's detector row (uniform over the block)
        const float py = fadd(fadd(g.bmin.y, fmul(fadd((float)y, 0.5f), g.vs.y)), s.y);
        const float av = fadd(fmul(vc.mat[1], px0), fmul(vc.mat[5], py));
        int y0;
        float b;
        split_coord<kSampleQ8>(fadd(av, vc.mat[13]), a.H, y0, b);
        const float omb = fsub(1.f, b);
        const float cy4 = fmul(vc.mat[4], py);
        const float2* r0 = a.rl + (ptrdiff_t)y0 * (ptrdiff_t)a.rl_pitch;
        const float2* r1 = r0 + a.rl_pitch;
        __syncthreads();  // the previous item's taps are no longer read (K is ready the first time)
        for (int e = tid; e < ntaps; e += kBpColThreads) {
            // columns outside the padded image read zero, as the clamped taps of the
            // direct kernels read the zero border; the residual taps carry lambda * d
            const int x0 = x0lo + e;
            const bool in0 = x0 >= -kPad && x0 < a.W + kPad, in1 = x0 + 1 >= -kPad && x0 + 1 < a.W + kPad;
            const float2 p0 = in0 ? __ldg(r0 + x0) : zero, q0 = in1 ? __ldg(r0 + x0 + 1) : zero;
            const float2 p1 = in0 ? __ldg(r1 + x0) : zero, q1 = in1 ? __ldg(r1 + x0 + 1) : zero;
            const float2 P0 = make_float2(fadd(fmul(omb, p0.x), fmul(b, p1.x)), fadd(fmul(omb, p0.y), fmul(b, p1.y)));
            const float2 P1 = make_float2(fadd(fmul(omb, q0.x), fmul(b, q1.x)), fadd(fmul(omb, q0.y), fmul(b, q1.y)));
            taps[e + (e >> 3)] = make_float4(fmul(P0.x, lamd), P0.y, fmul(fsub(P1.x, P0.x), lamd), fsub(P1.y, P0.y));
        }
        __syncthreads();
        float2 au[kGroups][2];
#pragma unroll
        for (int k = 0; k < kGroups; ++k) {
            au[k][0] = f2(fadd(A[k][0], cy4), fadd(A[k][1], cy4));
            au[k][1] = f2(fadd(A[k][2], cy4), fadd(A[k][3], cy4));
        }
        float* dst = a.vol + ((size_t)z0 * ry + y) * rx + 4 * tid;
        const int nrows = z1 - z0;
        for (int r = 0; r < nrows; ++r) {
            fetch();
            cp_async_wait<kBpColDepth - 1>();  // the row in read slot rs has landed
            const float2 kz = splat(K[z0 + r]);
#pragma unroll
            for (int k = 0; k < kGroups; ++k) {
                if (!on[k]) continue;
                const float4 v = my[(rs * kGroups + k) * kBpColThreads];
                const float vin[4] = {v.x, v.y, v.z, v.w};
                float vout[4];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    // u = (au + m8 * pz) + m12 and the column split, two voxels per instruction
                    const float2 u = add2(add2(au[k][h], kz), m12);
                    const float2 f = __fadd2_rd(fma2(u, splat(256.f), splat(-127.5f)), splat(12582912.0f));
                    int e0, e1;
                    float a0, a1;
                    q8_tap_bits(f.x, x0lo, e0, a0);
                    q8_tap_bits(f.y, x0lo, e1, a1);
                    const float2 ax = add2(f2(a0, a1), splat(-1.f));
#pragma unroll
                    for (int q = 0; q < 2; ++q) {
                        const int eq = q ? e1 : e0;
                        const float4 t = taps[eq + (eq >> 3)];
                        const float w = q ? ax.y : ax.x;
                        const float R = fmaf(w, t.z, t.x), L = fmaf(w, t.w, t.y);
                        // ParallelBeamsBackProjection.cl:40-50: v + r * lambda * d / L where L > eps
                        const float c = fmul(R, rcp_approx(L));
                        const float vi = vin[2 * h + q];
                        vout[2 * h + q] = L > kEps ? fadd(vi, c) : vi;
                    }
                }
                *reinterpret_cast<float4*>(dst + 4 * k * kBpColThreads) = make_float4(vout[0], vout[1], vout[2], vout[3]);
                if (kShadow) {  // the master's 16-bit shadow, as bp_store writes it
                    const size_t e = (size_t)(dst - a.vol) + 4 * k * kBpColThreads;
                    uint2 h;
                    if (kShadow == 1) {
                        const __half2 lo = __floats2half2_rn(vout[0], vout[1]), hi = __floats2half2_rn(vout[2], vout[3]);
                        h = make_uint2(*reinterpret_cast<const uint32_t*>(&lo), *reinterpret_cast<const uint32_t*>(&hi));
                    } else {
                        const __nv_bfloat162 lo = __floats2bfloat162_rn(vout[0], vout[1]),
                                             hi = __floats2bfloat162_rn(vout[2], vout[3]);
                        h = make_uint2(*reinterpret_cast<const uint32_t*>(&lo), *reinterpret_cast<const uint32_t*>(&hi));
                    }
                    *reinterpret_cast<uint2*>((uint16_t*)a.shadow + e) = h;
                }
            }
            rs = (rs + 1) & (kBpColDepth - 1);
            dst += plane;
        }
    }
    cp_async_wait<0>();
}

// ---- fused SART step: back projection of one view, forward projection of the next ----
// SART alternates BP(view p) and FP(view p + 1) (BlockIterativeReconstructionOperator.cpp:
// 92-142 with blockSize 1).  For parallel views tilted about y both touch one xz plane
// of the volume per volume row y: the BP of row y reads only the detector rows its
// voxels project to, and every ray of the next view stays in the volume row its
// detector row maps to.  One block owns a volume row and streams it once, z chunk by
// z chunk through shared memory: it applies the BP update of view p to the chunk
// (as bp_sart_column_kernel: same tap window, same arithmetic), writes the chunk
// back, and advances the rays of view p + 1 that lie in the row through the updated
// chunk.  Chunks are taken in the direction the rays travel in z, and each ray
// keeps its walk state (voxel, remaining distances, sums) between chunks, so its
// steps and its sums are those of dda_walk_xz in the same order.  After the last
// chunk the block writes the (residual, length) pairs of its rays, as fp_store does
// for one sample and one sub-volume.  The volume then crosses HBM once per view
// (read + write) instead of twice for the BP and once more for the FP.
constexpr int kFuseThreads = 512;
constexpr int kFuseZc = 8;    // z rows per chunk
constexpr int kFuseRays = 2;  // detector pixels per thread: at most 1024 rays per volume row

struct FuseArgs {
    float* vol;                 // FP32 volume, x-fastest [z][y][x], one sub-volume
    SlabConst slab;
    const ViewConst* views;     // by view id
    const uint32_t* order;
    uint32_t p;                 // order position of the back-projected view; p + 1 is projected
    const float4* samples;      // one (x, y, z, chord) per view id
    const float2* rl_in;        // texel (0, 0) of view p's padded (residual, length) image
    float2* rl_out;             // texel (0, 0) of view p + 1's image
    size_t rl_pitch;            // float2 units
    int W, H;
    float lambda;
    int x0lo, ntaps;            // view p's tap window (plan_bp_col)
    const int2* jrange;         // [view id * ry + y]: detector rows [x, y) whose rays lie in volume row y
    const float* real;          // measured projections, view id * W * H (element type real_kind)
    int real_kind;              // 0 FP32, 1 FP16, 2 BF16 (load_real)
    double* resid_sq;           // sum of residual^2 (FP64), or nullptr
    int loc;                    // long-object compensation
    float* part;                // non-null: view p + 1's (projection, ray length) of this sub-volume go to
                                // part[pixel] and part[W * H + pixel] (kFpSeparateAccumulate into
                                // zeros) instead of the residual (the z-slab block step)
};

__host__ __device__ constexpr size_t fuse_smem_bytes(int rx, int rz, int ntaps) {
    return (size_t)bp_col_tap_slots(ntaps) * 16 + ((size_t)rz * 4 + 15) / 16 * 16 + 2 * (size_t)kFuseZc * rx * 4;
}

// Global loads of data that other blocks of the same launch write (the persistent
// step's residual images): plain loads, not the read-only path.
template <bool kCoherent>
__device__ __forceinline__ float2 ld_rl(const float2* p) {
    if (kCoherent) return *p;
    return __ldg(p);
}

// Unit kinds of fused_row_step: the fused step (BP of p, FP of p + 1), the forward
// projection alone (the first view of an iteration, p + 1 = 0), the back projection alone
// (the last view).
constexpr int kUnitFused = 0, kUnitForward = 1, kUnitBack = 2;

// One fused step of volume row y: BP of the view at order position p, FP of the view at
// p + 1.  Each thread owns two consecutive x voxels of the row and two rays.  Requires
// rx % 2 == 0, rx <= 2 * kFuseThreads, rx + rz - 1 <= kMaxDdaIterations (the walk cap is
// never reached), at most kFuseRays * kFuseThreads rays per volume row (kThreads in place of
// kFuseThreads for a block of kThreads threads).  kCoherent: the
// residual images may have been written by other blocks of the same launch.  kKind
// kUnitForward skips the back projection (the volume is only read; p + 1 is the view),
// kUnitBack the forward projection; each half performs the same operations as in the
// fused step.
// Value of the 16-bit shadow a forward projection reads for an FP32 master voxel
// (kShadow 1: FP16, 2: BF16, 0: no shadow, the FP32 value itself).
template <int kShadow>
__device__ __forceinline__ float shadow_value(float v) {
    if (kShadow == 1) return __half2float(__float2half_rn(v));
    if (kShadow == 2) return __bfloat162float(__float2bfloat16_rn(v));
    return v;
}

// kShadow (1: FP16, 2: BF16 shadow of an FP32 master): the walk reads the chunk rounded as
// the shadow stores it, so the forward projection sees what the separate forward
// projector reads from the shadow; the master is updated in FP32 (the shadow itself is
// refreshed by the last back projection of the iteration).
template <bool kCoherent, int kKind = kUnitFused, int kThreads = kFuseThreads, int kShadow = 0>
__device__ __forceinline__ void fused_row_step(const FuseArgs& a, uint32_t p, int y, int x0lo, int ntaps,
                                               const float2* rl_in, float2* rl_out,
                                               unsigned char* fuse_smem) {
    constexpr bool kBP = kKind != kUnitForward, kFP = kKind != kUnitBack;
    const SlabConst& g = a.slab;
    const int rx = g.rx, ry = g.ry, rz = g.rz, tid = threadIdx.x;
    float4* taps = (float4*)fuse_smem;
    float* K = (float*)(taps + bp_col_tap_slots(ntaps));
    float* buf = (float*)(fuse_smem + (size_t)bp_col_tap_slots(ntaps) * 16 + ((size_t)rz * 4 + 15) / 16 * 16);
    const size_t chunk_elems = (size_t)kFuseZc * rx;

    // ---- back projection constants of view p (bp_sart_column_kernel, one item = row y)
    const uint32_t vb = kBP ? a.order[p] : a.order[p + 1];
    const ViewConst& vc = a.views[vb];
    const float4 s = a.samples[vb];
    if (kBP)
        for (int z = tid; z < rz; z += kThreads)
            K[z] = fmul(vc.mat[8], fadd(fadd(g.bmin.z, fmul(fadd((float)z, 0.5f), g.vs.z)), s.z));
    const int x2 = 2 * tid;
    const bool on = x2 < rx;
    float A[2];
#pragma unroll
    for (int j = 0; j < 2; ++j)
        A[j] = fmul(vc.mat[0], fadd(fadd(g.bmin.x, fmul(fadd((float)(x2 + j), 0.5f), g.vs.x)), s.x));
    const float lamd = fmul(a.lambda, s.w);
    const float2 m12 = splat(vc.mat[12]);
    const float px0 = fadd(fadd(g.bmin.x, fmul(0.5f, g.vs.x)), s.x);
    {
        const float py = fadd(fadd(g.bmin.y, fmul(fadd((float)y, 0.5f), g.vs.y)), s.y);
        const float av = fadd(fmul(vc.mat[1], px0), fmul(vc.mat[5], py));
        int y0;
        float b;
        split_coord<kSampleQ8>(fadd(av, vc.mat[13]), a.H, y0, b);
        const float omb = fsub(1.f, b);
        const float2* r0 = rl_in + (ptrdiff_t)y0 * (ptrdiff_t)a.rl_pitch;
        const float2* r1 = r0 + a.rl_pitch;
        const float2 zero = make_float2(0.f, 0.f);
        for (int e = tid; kBP && e < ntaps; e += kThreads) {
            const int x0 = x0lo + e;
            const bool in0 = x0 >= -kPad && x0 < a.W + kPad, in1 = x0 + 1 >= -kPad && x0 + 1 < a.W + kPad;
            const float2 p0 = in0 ? ld_rl<kCoherent>(r0 + x0) : zero, q0 = in1 ? ld_rl<kCoherent>(r0 + x0 + 1) : zero;
            const float2 p1 = in0 ? ld_rl<kCoherent>(r1 + x0) : zero, q1 = in1 ? ld_rl<kCoherent>(r1 + x0 + 1) : zero;
            const float2 P0 = make_float2(fadd(fmul(omb, p0.x), fmul(b, p1.x)), fadd(fmul(omb, p0.y), fmul(b, p1.y)));
            const float2 P1 = make_float2(fadd(fmul(omb, q0.x), fmul(b, q1.x)), fadd(fmul(omb, q0.y), fmul(b, q1.y)));
            taps[e + (e >> 3)] = make_float4(fmul(P0.x, lamd), P0.y, fmul(fsub(P1.x, P0.x), lamd), fsub(P1.y, P0.y));
        }
        const float cy4 = fmul(vc.mat[4], py);
        A[0] = fadd(A[0], cy4);
        A[1] = fadd(A[1], cy4);
    }
    const float2 au = f2(A[0], A[1]);

    // ---- rays of view p + 1 in volume row y (fp_pixel with one sample, dda_setup)
    const uint32_t vf = kFP ? a.order[p + 1] : vb;
    const ViewConst& fc = a.views[vf];
    const int2 jr = kFP ? a.jrange[(size_t)vf * ry + y] : make_int2(0, 0);
    const int nrays = jr.y > jr.x ? (jr.y - jr.x) * a.W : 0;
    const float3 ray = make_float3(fc.ray.x, fc.ray.y, fc.ray.z);
    const float3 inv = make_float3(fc.inv.x, fc.inv.y, fc.inv.z);
    int rix[kFuseRays], riz[kFuseRays];
    float rrx[kFuseRays], rrz[kFuseRays], acc[kFuseRays], accl[kFuseRays];
    bool walking[kFuseRays];
    // the step differences and directions are the view's (dda_setup; every ray of the
    // view has the same direction), so the chunk order is uniform over the block
    const float sgx = clsign(ray.x), sgz = clsign(ray.z);
    const float sdx = fmul(fmul(g.vs.x, inv.x), sgx), sdz = fmul(fmul(g.vs.z, inv.z), sgz);
    const int sx = (int)sgx, sz = (int)sgz;
    {
        const float sdist = fdiv(1.f, 1.f), off = fdiv(sdist, 2.f);
#pragma unroll
        for (int i = 0; i < kFuseRays; ++i) {
            const int k = tid + i * kThreads;
            acc[i] = 0.f;
            accl[i] = 0.f;
            walking[i] = false;
            rix[i] = riz[i] = 0;
            rrx[i] = rrz[i] = 0.f;
            if (k < nrays) {
                const int gy = jr.x + k / a.W, gx = k - (k / a.W) * a.W;
                const float fx = fadd(fadd((float)gx, off), fmul(sdist, 0.f));
                const float fy = fadd(fadd((float)gy, off), fmul(sdist, 0.f));
                const float3 src = make_float3(fadd(fadd(fc.source.x, fmul(fc.hpitch.x, fx)), fmul(fc.vpitch.x, fy)),
                                               fadd(fadd(fc.source.y, fmul(fc.hpitch.y, fx)), fmul(fc.vpitch.y, fy)),
                                               fadd(fadd(fc.source.z, fmul(fc.hpitch.z, fx)), fmul(fc.vpitch.z, fy)));
                DdaStart st;
                if (dda_setup(src, ray, inv, g, st)) {
                    walking[i] = true;
                    rix[i] = st.ix;
                    riz[i] = st.iz;
                    rrx[i] = st.res.x;
                    rrz[i] = -st.res.z;  // kept negated by the walk
                }
            }
        }
    }
    const bool up = sz >= 0;
    const int nchunks = (rz + kFuseZc - 1) / kFuseZc;
    const size_t plane = (size_t)rx * (size_t)ry;

    // chunk c (in walk order) -> its first z row
    auto chunk_z0 = [&](int c) { return (up ? c : nchunks - 1 - c) * kFuseZc; };
    auto fetch = [&](int c) {
        if (c < nchunks && on) {
            const int z0 = chunk_z0(c), z1 = min(rz, z0 + kFuseZc);
            float* dst = buf + (size_t)(c & 1) * chunk_elems + x2;
            const float* src = a.vol + ((size_t)z0 * ry + y) * rx + x2;
            if (z1 - z0 == kFuseZc) {  // a whole chunk: its rows unrolled
                const uint32_t d0 = smem_addr(dst);
#pragma unroll
                for (int k = 0; k < kFuseZc; ++k) cp_async8(d0 + 4u * (uint32_t)(k * rx), src + (size_t)k * plane);
            } else {
                for (int z = z0; z < z1; ++z, dst += rx, src += plane) cp_async8(smem_addr(dst), src);
            }
        }
        cp_async_commit();
    };
    // BP update of chunk c in place (this thread's two columns), written back to the volume
    auto update = [&](int c) {
        if (!kBP && kShadow && c < nchunks && on) {  // the walk reads the shadow's values
            const int z0 = chunk_z0(c), z1 = min(rz, z0 + kFuseZc);
            float* cb = buf + (size_t)(c & 1) * chunk_elems;
            for (int z = z0; z < z1; ++z) {
                float2* slot = reinterpret_cast<float2*>(cb + (size_t)(z - z0) * rx + x2);
                const float2 v = *slot;
                *slot = make_float2(shadow_value<kShadow>(v.x), shadow_value<kShadow>(v.y));
            }
        }
        if (!kBP || c >= nchunks || !on) return;
        const int z0 = chunk_z0(c), z1 = min(rz, z0 + kFuseZc);
        float* cb = buf + (size_t)(c & 1) * chunk_elems;
        float* dst = a.vol + ((size_t)z0 * ry + y) * rx + x2;
        auto voxel = [&](int z, float* d) {
            float2* slot = reinterpret_cast<float2*>(cb + (size_t)(z - z0) * rx + x2);
            const float2 v = *slot;
            const float vin[2] = {v.x, v.y};
            float vout[2];
            // u = (au + m8 * pz) + m12 and the column split, two voxels per instruction
            const float2 u = add2(add2(au, splat(K[z])), m12);
            const float2 f = __fadd2_rd(fma2(u, splat(256.f), splat(-127.5f)), splat(12582912.0f));
            int e0, e1;
            float a0, a1;
            q8_tap_bits(f.x, x0lo, e0, a0);
            q8_tap_bits(f.y, x0lo, e1, a1);
            const float2 ax = add2(f2(a0, a1), splat(-1.f));
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int eq = q ? e1 : e0;
                const float4 t = taps[eq + (eq >> 3)];
                const float w = q ? ax.y : ax.x;
                const float2 RL = fma2(splat(w), f2(t.z, t.w), f2(t.x, t.y));  // (R, L), one fma each
                // ParallelBeamsBackProjection.cl:40-50: v + r * lambda * d / L where L > eps
                const float cc = fmul(RL.x, rcp_approx(RL.y));
                vout[q] = RL.y > kEps ? fadd(vin[q], cc) : vin[q];
            }
            const float2 o = make_float2(vout[0], vout[1]);
            *reinterpret_cast<float2*>(d) = o;
            *slot = kShadow ? make_float2(shadow_value<kShadow>(o.x), shadow_value<kShadow>(o.y)) : o;
        };
        if (z1 - z0 == kFuseZc) {  // a whole chunk: its rows unrolled
#pragma unroll
            for (int k = 0; k < kFuseZc; ++k) voxel(z0 + k, dst + (size_t)k * plane);
        } else {
            for (int z = z0; z < z1; ++z, dst += plane) voxel(z, dst);
        }
    };
    // FP walk of the rays through the updated chunk c (dda_walk_xz's steps, chunk-local
    // byte offsets): x may take nxr more steps before the ray leaves the volume, z nzr
    // more before it leaves the chunk; blocks of 4 steps run unchecked while both
    // budgets allow.  The remaining z distance is kept negated (nz = -rz): s = rx + nz
    // is fsub(rx, rz), whose sign decides the axis (rx <= rz iff s <= 0) and which is
    // the new remaining distance of the axis that did not step (rx - rz, or
    // -(rz - rx)); dt = min(rx, -nz).  Same values as dda_walk_xz's updates.
    const float nsdz = -sdz;
    auto walk = [&](int c) {
        const int z0 = chunk_z0(c), z1 = min(rz, z0 + kFuseZc);
        const unsigned char* cb = (const unsigned char*)(buf + (size_t)(c & 1) * chunk_elems);
        const int dxo = 4 * sx, dzo = 4 * sz * rx;
#pragma unroll
        for (int i = 0; i < kFuseRays; ++i) {
            if (!walking[i] || riz[i] < z0 || riz[i] >= z1) continue;
            const int ix = rix[i], iz = riz[i];
            const int nxr = sx > 0 ? rx - ix : (sx < 0 ? ix + 1 : 0x3fffffff);
            const int nzr = sz > 0 ? z1 - iz : (sz < 0 ? iz - z0 + 1 : 0x3fffffff);
            float rxv = rrx[i], nzv = rrz[i], av = acc[i], al = accl[i];
            int off = 4 * ((iz - z0) * rx + ix), nxs = 0, n = 0;
            auto step = [&]() {
                const float sdiff = rxv + nzv;
                const bool bx = sdiff <= 0.f;
                const float dt = fminf(rxv, -nzv);
                av = fmaf(dt, *(const float*)(cb + off), av);
                al += dt;
                rxv = bx ? sdx : sdiff;
                nzv = bx ? sdiff : nsdz;
                off += bx ? dxo : dzo;
                nxs += bx ? 1 : 0;
            };
            while (min(nxr - nxs, nzr - (n - nxs)) >= 4) {
                step();
                step();
                step();
                step();
                n += 4;
            }
            while (nxs < nxr && n - nxs < nzr) {
                step();
                ++n;
            }
            rix[i] = ix + sx * nxs;
            riz[i] = iz + sz * (n - nxs);
            // x ran out: the ray left the volume; z ran out: it continues in the next chunk
            // unless it left the volume in z
            walking[i] = nxs < nxr && riz[i] >= 0 && riz[i] < rz;
            rrx[i] = rxv;
            rrz[i] = nzv;
            acc[i] = av;
            accl[i] = al;
        }
    };

    // Skewed pipeline, one barrier per chunk: while the rays walk chunk c, chunk c + 1
    // is in flight; it is then updated in place, and the barrier publishes it (and
    // frees chunk c's buffer for chunk c + 2).
    fetch(0);
    cp_async_wait<0>();
    __syncthreads();  // K and the taps are staged
    update(0);
    __syncthreads();  // chunk 0 is updated
    for (int c = 0; c < nchunks; ++c) {
        fetch(c + 1);
        walk(c);
        cp_async_wait<0>();  // this thread's rows of chunk c + 1 have landed
        update(c + 1);
        __syncthreads();
    }
    cp_async_wait<0>();

    // ---- epilogue of view p + 1 (fp_store, mode kFpPairResidual, one sample, one sub-volume)
    double r2 = 0.0;
#pragma unroll
    for (int i = 0; i < kFuseRays; ++i) {
        const int k = tid + i * kThreads;
        if (k < nrays) {
            const int gy = jr.x + k / a.W, gx = k - (k / a.W) * a.W;
            // fp_pixel sums its one sub-ray into zero, fp_store divides by the count
            const float pv = fdiv(fadd(0.f, acc[i]), 1.f), pl = fdiv(fadd(0.f, accl[i]), 1.f);
            float vv = fadd(0.f, pv), ll = fadd(0.f, pl);
            if (a.part) {
                const size_t pix = (size_t)gy * (size_t)a.W + (size_t)gx;
                a.part[pix] = vv;
                a.part[(size_t)a.W * (size_t)a.H + pix] = ll;
                continue;
            }
            if (a.loc) {
                vv = ll > kEps ? fdiv(fmul(vv, fc.loc_length), ll) : 0.f;
                ll = fc.loc_length;
            }
            const size_t pix = (size_t)gy * (size_t)a.W + (size_t)gx;
            const float r = fsub(load_real(a.real, a.real_kind, (size_t)vf * (size_t)a.W * (size_t)a.H + pix), vv);
            rl_out[(size_t)gy * a.rl_pitch + (size_t)gx] = make_float2(r, ll);
            r2 += (double)r * (double)r;
        }
    }
    if (a.resid_sq) {
        for (int o = 16; o > 0; o >>= 1) r2 += __shfl_down_sync(0xffffffffu, r2, o);
        if ((tid & 31) == 0 && r2 != 0.0) atomicAdd(a.resid_sq, r2);
    }
}

template <int kShadow>
__global__ void __launch_bounds__(kFuseThreads, 2) sart_fused_kernel(const __grid_constant__ FuseArgs a) {
    extern __shared__ __align__(16) unsigned char fuse_smem[];
    fused_row_step<false, kUnitFused, kFuseThreads, kShadow>(a, a.p, (int)blockIdx.x, a.x0lo, a.ntaps, a.rl_in,
                                                             a.rl_out, fuse_smem);
}

// All fused steps of one SART iteration in one launch.  With parallel views tilted about
// y, step p of volume row y reads and writes only row y of the volume, the detector rows
// of row y's rays (written) and the two detector rows its back projection samples (read);
// those belong to rows y - window .. y + window.  Blocks take (step, row) units from a
// counter in step-major order and start a unit once those rows have finished the step
// before, so rows run ahead of one another instead of every step waiting for the whole
// volume (and its last partial wave of blocks).  A unit only waits on units taken before
// it by running blocks, so the waits end; each is still bounded by kFuseWaitNs, after which
// the block sets the error word and leaves, and every block leaves once it is set.
struct FusePersist {
    const int2* tapwin;   // per view id: (x0lo, ntaps) of its back projection
    float2* rl0;          // texel (0, 0) of residual slot 0; slot 1 follows at rl_slot
    size_t rl_slot;       // float2 units
    uint32_t steps;       // fused steps per iteration (views - 1)
    uint32_t* ctl;        // [0] unit counter, [1 + y] steps row y has finished (zeroed per iteration)
    uint32_t* error;      // nonzero once a wait gave up (sticky)
    int window;
    int withhold_row;     // tests of the bounded waits: this row never reports step 0 (else -1)
};

constexpr unsigned long long kFuseWaitNs = 1000000000ull;

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_u32(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

template <int kShadow>
__global__ void __launch_bounds__(kFuseThreads, 2)
    sart_fused_persistent_kernel(const __grid_constant__ FuseArgs a, const __grid_constant__ FusePersist q) {
    extern __shared__ __align__(16) unsigned char fuse_smem[];
    __shared__ uint32_t unit_s;
    const uint32_t ry = (uint32_t)a.slab.ry;
    const uint32_t total = q.steps * ry;
    uint32_t* done = q.ctl + 1;
    for (;;) {
        if (threadIdx.x == 0) {
            uint32_t u = total;
            if (ld_acquire_u32(q.error) == 0) {
                u = atomicAdd(q.ctl, 1u);
                if (u < total) {
                    const uint32_t p = u / ry;
                    const int y = (int)(u - p * ry);
                    if (p > 0) {
                        const int lo = max(0, y - q.window), hi = min((int)ry - 1, y + q.window);
                        const unsigned long long t0 = global_ns();
                        for (int yy = lo; yy <= hi && u < total; ++yy)
                            while (ld_acquire_u32(done + yy) < p) {
                                if (global_ns() - t0 > kFuseWaitNs) {
                                    atomicExch(q.error, 1u);
                                    u = total;
                                    break;
                                }
                                if (ld_acquire_u32(q.error) != 0) {  // another block gave up
                                    u = total;
                                    break;
                                }
                                __nanosleep(128);
                            }
                    }
                } else {
                    u = total;
                }
            }
            unit_s = u;
        }
        __syncthreads();
        const uint32_t u = unit_s;
        if (u >= total) return;
        const uint32_t p = u / ry;
        const int y = (int)(u - p * ry);
        const int2 tw = q.tapwin[a.order[p]];
        fused_row_step<true, kUnitFused, kFuseThreads, kShadow>(a, p, y, tw.x, tw.y, q.rl0 + (size_t)(p & 1) * q.rl_slot,
                                                                q.rl0 + (size_t)((p + 1) & 1) * q.rl_slot, fuse_smem);
        __syncthreads();  // the unit's stores are issued and its shared memory is free
        if (threadIdx.x == 0 && !(p == 0 && y == q.withhold_row)) {
            __threadfence();
            st_release_u32(done + y, p + 1);
        }
    }
}

// Many independent series in one launch per SART iteration.  Per series and volume row
// the unit steps are 0 (forward projection of the first view), 1 .. M - 1 (the fused
// steps) and M (back projection of the last view); units are numbered step-major over
// all series (segments of (step, series) in that order), so a unit waits only on units
// of smaller numbers, as in sart_fused_persistent_kernel, with the same bounded waits.
struct FuseSeries {
    FuseArgs a;           // p, rl_in, rl_out, x0lo and ntaps unused
    const int2* tapwin;   // per view id: (x0lo, ntaps)
    float2* rl0;          // texel (0, 0) of residual slot 0; slot 1 follows at rl_slot
    size_t rl_slot;       // float2 units
    uint32_t* done;       // per volume row: unit steps finished (zeroed per iteration)
    uint32_t views;       // M
    int window;
};

struct FuseSegment {
    uint32_t start;       // first unit number
    uint32_t series;
    uint32_t step;        // unit step
};

// kThreads = 512 for rows of up to 1024 voxels, 128 for batches whose rows are at most 256
// voxels wide with at most 256 rays each (two voxels and two rays per thread either way).
// kShadow: every series holds an FP32 master with a 16-bit shadow of that kind
// (fused_row_step); the shadows are refreshed from the masters after the launch.
template <int kThreads, int kShadow = 0>
__global__ void __launch_bounds__(kThreads, 1024 / kThreads)
    sart_fused_batch_kernel(const FuseSeries* series, const FuseSegment* segs, uint32_t nsegs, uint32_t total,
                            uint32_t* counter, uint32_t* error, int withhold_row) {
    extern __shared__ __align__(16) unsigned char fuse_smem[];
    __shared__ __align__(16) FuseSeries cur;
    __shared__ uint32_t unit_s[3];
    for (;;) {
        if (threadIdx.x == 0) {
            uint32_t u = total, si = 0, st = 0, y = 0;
            if (ld_acquire_u32(error) == 0) {
                u = atomicAdd(counter, 1u);
                if (u < total) {
                    uint32_t lo = 0, hi = nsegs - 1;  // last segment with start <= u
                    while (lo < hi) {
                        const uint32_t mid = (lo + hi + 1) / 2;
                        if (segs[mid].start <= u) lo = mid;
                        else hi = mid - 1;
                    }
                    si = segs[lo].series;
                    st = segs[lo].step;
                    y = u - segs[lo].start;
                    if (st > 0) {
                        const FuseSeries& f = series[si];
                        const int ry = f.a.slab.ry, w = f.window;
                        const int yl = max(0, (int)y - w), yh = min(ry - 1, (int)y + w);
                        const unsigned long long t0 = global_ns();
                        for (int yy = yl; yy <= yh && u < total; ++yy)
                            while (ld_acquire_u32(f.done + yy) < st) {
                                if (global_ns() - t0 > kFuseWaitNs) {
                                    atomicExch(error, 1u);
                                    u = total;
                                    break;
                                }
                                if (ld_acquire_u32(error) != 0) {
                                    u = total;
                                    break;
                                }
                                __nanosleep(128);
                            }
                    }
                } else {
                    u = total;
                }
            }
            unit_s[0] = u;
            unit_s[1] = si;
            unit_s[2] = (st << 16) | y;
        }
        __syncthreads();
        const uint32_t u = unit_s[0];
        if (u >= total) return;
        const uint32_t si = unit_s[1], st = unit_s[2] >> 16;
        const int y = (int)(unit_s[2] & 0xffffu);
        // the unit's series arguments, staged in shared memory
        {
            const uint32_t* src = reinterpret_cast<const uint32_t*>(series + si);
            uint32_t* dst = reinterpret_cast<uint32_t*>(&cur);
            for (int i = threadIdx.x; i < (int)(sizeof(FuseSeries) / 4); i += blockDim.x) dst[i] = src[i];
        }
        __syncthreads();
        if (st == 0) {
            fused_row_step<true, kUnitForward, kThreads, kShadow>(cur.a, 0xffffffffu, y, 0, 0, cur.rl0, cur.rl0,
                                                                  fuse_smem);
        } else {
            const uint32_t p = st - 1;
            const int2 tw = cur.tapwin[cur.a.order[p]];
            const float2* rin = cur.rl0 + (size_t)(p & 1) * cur.rl_slot;
            float2* rout = cur.rl0 + (size_t)((p + 1) & 1) * cur.rl_slot;
            if (st < cur.views)
                fused_row_step<true, kUnitFused, kThreads, kShadow>(cur.a, p, y, tw.x, tw.y, rin, rout, fuse_smem);
            else
                fused_row_step<true, kUnitBack, kThreads, kShadow>(cur.a, p, y, tw.x, tw.y, rin, rout, fuse_smem);
        }
        __syncthreads();  // the unit's stores are issued; its shared memory is free
        // withhold_row (tests of the bounded waits): series 0 never reports that row's step 0
        if (threadIdx.x == 0 && !(si == 0 && st == 0 && y == withhold_row)) {
            __threadfence();
            st_release_u32(cur.done + y, st + 1);
        }
    }
}

// Detector row pair (y0, y0 + 1) the fused back projection of view v samples for volume
// row y (the same arithmetic as fused_row_step), for the dependency window.
__global__ void fuse_bp_rows_kernel(const ViewConst* views, const float4* samples, SlabConst g, int H, int* y0out) {
    const int y = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y;
    if (y >= g.ry) return;
    const ViewConst& vc = views[v];
    const float4 s = samples[v];
    const float px0 = fadd(fadd(g.bmin.x, fmul(0.5f, g.vs.x)), s.x);
    const float py = fadd(fadd(g.bmin.y, fmul(fadd((float)y, 0.5f), g.vs.y)), s.y);
    const float av = fadd(fmul(vc.mat[1], px0), fmul(vc.mat[5], py));
    int y0;
    float b;
    split_coord<kSampleQ8>(fadd(av, vc.mat[13]), H, y0, b);
    y0out[(size_t)v * g.ry + y] = y0;
}

// Detector rows per volume row for the fused step: the rays of detector row j of a
// parallel view with ray.y == 0 and hpitch.y == 0 stay in the volume row dda_setup
// assigns them (the clamp of the source's y); jb / je receive the first and one past
// the last detector row of every (view, volume row).
__global__ void fuse_rows_kernel(const ViewConst* views, SlabConst g, int H, int* jb, int* je) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y;
    if (j >= H) return;
    const ViewConst& vc = views[v];
    const float sdist = fdiv(1.f, 1.f), off = fdiv(sdist, 2.f);
    const float fx = fadd(fadd(0.f, off), fmul(sdist, 0.f));
    const float fy = fadd(fadd((float)j, off), fmul(sdist, 0.f));
    const float sy = fadd(fadd(vc.source.y, fmul(vc.hpitch.y, fx)), fmul(vc.vpitch.y, fy));
    const float py = clclamp(sy, g.bmin.y, g.bmax.y);
    const int iy = min(max((int)fmul(fsub(py, g.bmin.y), g.ivs.y), 0), g.ry - 1);
    atomicMin(jb + (size_t)v * g.ry + iy, j);
    atomicMax(je + (size_t)v * g.ry + iy, j + 1);
}

// PerspectiveBeamsBackProjection.cl:10-17 getRayLengthInVoxel
__device__ __forceinline__ float chord_in_voxel(float3 o, float3 dir, float3 c, float3 vs) {
    float3 bmin = make_float3(fsub(c.x, fmul(0.5f, vs.x)), fsub(c.y, fmul(0.5f, vs.y)), fsub(c.z, fmul(0.5f, vs.z)));
    float3 bmax = make_float3(fadd(c.x, fmul(0.5f, vs.x)), fadd(c.y, fmul(0.5f, vs.y)), fadd(c.z, fmul(0.5f, vs.z)));
    const float n = __fsqrt_rn(fadd(fadd(fmul(dir.x, dir.x), fmul(dir.y, dir.y)), fmul(dir.z, dir.z)));
    // 1 / normalize(dir) = |dir| / dir
    float3 inv = make_float3(div_fast(n, dir.x), div_fast(n, dir.y), div_fast(n, dir.z));
    float tin, tout;
    slab_test(bmin, bmax, o, inv, tin, tout);
    return fmaxf(0.f, fsub(tout, tin));
}

// Whether every voxel centre of the brick [x0, x1] x [y0, y1] x [z0, z1] projects with
// w > 0 and (u, v) at least 1/64 texel inside [ulo, uhi] x [vlo, vhi]: w is affine in the
// position, so its minimum over the brick is at a corner, and with w > 0 on the brick the
// projected brick is the convex hull of the projected corners.  The margin covers the
// rounding of the per-voxel evaluation.
__device__ __forceinline__ int brick_projects_inside(const BpView& V, const SlabConst& g, int x0, int x1, int y0,
                                                     int y1, int z0, int z1, float ulo, float uhi, float vlo,
                                                     float vhi) {
    float wmin = FLT_MAX, wmax = 0.f, umin = FLT_MAX, umax = -FLT_MAX, vmin = FLT_MAX, vmax = -FLT_MAX;
    for (int c = 0; c < 8; ++c) {
        const float px = g.bmin.x + ((float)((c & 1) ? x1 : x0) + 0.5f) * g.vs.x;
        const float py = g.bmin.y + ((float)((c & 2) ? y1 : y0) + 0.5f) * g.vs.y;
        const float pz = g.bmin.z + ((float)((c & 4) ? z1 : z0) + 0.5f) * g.vs.z;
        const float w = V.mw[0] * px + V.mw[1] * py + V.mw[2] * pz + V.mw[3];
        if (!(w > 0.f)) return 0;
        const float u = (V.mu[0] * px + V.mu[1] * py + V.mu[2] * pz + V.mu[3]) / w;
        const float v = (V.mv[0] * px + V.mv[1] * py + V.mv[2] * pz + V.mv[3]) / w;
        wmin = fminf(wmin, w);
        wmax = fmaxf(wmax, w);
        umin = fminf(umin, u);
        umax = fmaxf(umax, u);
        vmin = fminf(vmin, v);
        vmax = fmaxf(vmax, v);
    }
    const float m = 1.f / 64.f;
    return (wmin > 1e-5f * wmax && umin >= ulo + m && umax <= uhi - m && vmin >= vlo + m && vmax <= vhi - m) ? 1 : 0;
}

// PerspectiveBeamsBackProjection.cl:28-71: n^3 sub-voxel samples, each weighted by
// its own chord through the voxel; optional intensity clamps.
template <bool kMask, int kStore, int kSampling, bool kClamp>
__global__ void __launch_bounds__(256, 4) bp_perspective_kernel(const __grid_constant__ BpArgs a) {
    extern __shared__ __align__(16) unsigned char bp_smem[];
    BpView* sv = (BpView*)bp_smem;
    bp_stage(a, sv, nullptr, false);
    const SlabConst& g = a.slab;
    // grid (z chunks, x tiles, y tiles): consecutive blocks take the z chunks of one
    // column tile, whose texels they share
    const int x = blockIdx.y * blockDim.x + threadIdx.x;
    const int y = blockIdx.z * blockDim.y + threadIdx.y;
    const int z0 = blockIdx.x * kBpZPersp;
    // one sample per voxel, 1/256 weights, no mask: per (view, z voxel of the chunk) the
    // terms that depend on the view and z only, shared by the block's columns (a table after
    // the views in shared memory; the other variants form them per voxel, where the table's
    // registers would not fit the 64 of four blocks per SM)
    constexpr bool kZTable = kSampling == kSampleQ8 && !kMask;
    float4* zt = (float4*)(bp_smem + ((size_t)a.nviews * sizeof(BpView) + 15) / 16 * 16);
    if (a.persp_n == 1) {
        const int tid = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y;
        if (kSampling == kSampleQ8) {
            // per view, whether the block's voxels can skip the texel-coordinate clamps
            const int bx0 = blockIdx.y * blockDim.x, by0 = blockIdx.z * blockDim.y;
            const int bx1 = min(g.rx, bx0 + (int)blockDim.x) - 1, by1 = min(g.ry, by0 + (int)blockDim.y) - 1;
            const int bz1 = min(g.rz, z0 + kBpZPersp) - 1;
            for (int p = tid; p < a.nviews; p += nt)
                sv[p].inside = brick_projects_inside(sv[p], g, bx0, bx1, by0, by1, z0, bz1, -1.5f,
                                                     (float)a.W + 1.49609375f, -1.5f, (float)a.H + 1.49609375f);
        }
        // (m_w2 pz, dz^2, |dz| / vs_z, pz) with pz the voxel centre's z, dz = pz - source z:
        // the same operations as at the voxel (z voxels past the slab get unused entries)
        for (int i = tid; kZTable && i < a.nviews * kBpZPersp; i += nt) {
            const int p = i / kBpZPersp, j = i - p * kBpZPersp;
            const float cz = fadd(g.bmin.z, fmul(fadd((float)(z0 + j), 0.5f), g.vs.z));
            const float pzj = fadd(fsub(cz, fmul(0.5f, g.vs.z)), fmul(g.vs.z, 0.5f));
            const float dz = fsub(pzj, sv[p].src[2]);
            zt[i] = make_float4(fmul(sv[p].mw[2], pzj), fmul(dz, dz), fmul(fabsf(dz), g.ivs.z), pzj);
        }
        __syncthreads();
    }
    if (x >= g.rx || y >= g.ry) return;
    const int nzc = min(kBpZPersp, g.rz - z0);
    const size_t plane = (size_t)g.rx * (size_t)g.ry;
    const size_t base = (size_t)z0 * plane + (size_t)y * (size_t)g.rx + (size_t)x;
    const int n = a.persp_n;
    const unsigned count = (unsigned)(n * n * n);
    const float3 vs = make_float3(g.vs.x, g.vs.y, g.vs.z);
    const float cx = fadd(g.bmin.x, fmul(fadd((float)x, 0.5f), g.vs.x));
    const float cy = fadd(g.bmin.y, fmul(fadd((float)y, 0.5f), g.vs.y));
    if (n == 1) {
        // One sample per voxel, at its centre.  The views run outermost and the thread's
        // z voxels innermost, so every term that depends on the column and the view only
        // is formed once: the x / y parts of the three projection rows, (dx, dy), dx^2 + dy^2
        // and the x / y bounds of the chord.  The perspective divide takes one refined
        // reciprocal of w, and the chord of a ray through the voxel's centre is
        // vs_i * |d| / |d_i| minimised over the axes (the slab test of
        // getRayLengthInVoxel for that ray).  Same operations, in the same order per voxel,
        // as evaluating everything per voxel.
        const float px = fadd(fsub(cx, fmul(0.5f, g.vs.x)), fmul(g.vs.x, 0.5f));
        const float py = fadd(fsub(cy, fmul(0.5f, g.vs.y)), fmul(g.vs.y, 0.5f));
        // the voxel centres' z (pz): from the table, or in registers
        float val[kBpZPersp], mw[kBpZPersp], pz[kZTable ? 1 : kBpZPersp];
#pragma unroll
        for (int j = 0; j < kBpZPersp; ++j) {
            val[j] = 0.f;
            mw[j] = 1.f;
            if constexpr (!kZTable) pz[j] = 0.f;
            if (j < nzc) {
                const size_t idx = base + (size_t)j * plane;
                if constexpr (!kZTable) {
                    const float cz = fadd(g.bmin.z, fmul(fadd((float)(z0 + j), 0.5f), g.vs.z));
                    pz[j] = fadd(fsub(cz, fmul(0.5f, g.vs.z)), fmul(g.vs.z, 0.5f));
                }
                val[j] = bp_load<kStore>(a, idx);
                if (kMask) mw[j] = mask_weight(a.mask + idx);
            }
        }
        // full chunks (every z voxel of the thread inside the volume) skip the per-voxel test
        auto views = [&](auto full_tag) {
            constexpr bool kFull = decltype(full_tag)::value;
            for (int p = 0; p < a.nviews; ++p) {
                const BpView& V = sv[p];
                [[maybe_unused]] const float4* zv = zt + p * kBpZPersp;
                const float2* img = a.rl + (size_t)p * a.rl_slot;
                const float2 cuv = f2(fadd(fmul(V.mu[0], px), fmul(V.mu[1], py)), fadd(fmul(V.mv[0], px), fmul(V.mv[1], py)));
                const float2 m2 = f2(V.mu[2], V.mv[2]), m3 = f2(V.mu[3], V.mv[3]);
                const float cw = fadd(fmul(V.mw[0], px), fmul(V.mw[1], py));
                const float dx = fsub(px, V.src[0]), dy = fsub(py, V.src[1]);
                const float dxy = fadd(fmul(dx, dx), fmul(dy, dy));
                // chord of the ray through the centre: |d| / max_i(|d_i| / vs_i)
                const float mxy = fmaxf(fmul(fabsf(dx), g.ivs.x), fmul(fabsf(dy), g.ivs.y));
                // the coordinate clamps keep the taps inside the padded image (texels -2 .. W + 1);
                // out there every texel is a zero pad, as it is for the unclamped coordinate
                const float2 lo = splat(-1.5f), hi = f2((float)a.W + 1.49609375f, (float)a.H + 1.49609375f);
                const int pitch = (int)a.rl_pitch;
                const unsigned kq = 0x4B4000u * (unsigned)(pitch + 1);
                // kCoordClamp false when the whole brick projects inside (V.inside): the clamps
                // would change no coordinate
                auto zloop = [&](auto clamp_tag) {
                constexpr bool kCoordClamp = decltype(clamp_tag)::value;
#pragma unroll
                for (int j = 0; j < kBpZPersp; ++j) {
                    if (!kFull && j >= nzc) continue;
                    // (m_w2 pz, dz^2, |dz| / vs_z, pz) of this view and z voxel
                    float4 zq;
                    if constexpr (kZTable) {
                        zq = zv[j];
                    } else {
                        const float dz = fsub(pz[j], V.src[2]);
                        zq = make_float4(fmul(V.mw[2], pz[j]), fmul(dz, dz), fmul(fabsf(dz), g.ivs.z), pz[j]);
                    }
                    // u and v as paired operations (each lane the same operations as alone)
                    float2 uv = add2(add2(cuv, __fmul2_rn(m2, splat(zq.w))), m3);
                    const float w = fadd(fadd(cw, zq.x), V.mw[3]);
                    float rw = rcp_approx(w);
                    rw = fmaf(rw, fmaf(-w, rw, 1.f), rw);
                    uv = __fmul2_rn(uv, splat(rw));
                    float2 rl;
                    if (kSampling == kSampleQ8) {
                        // q = floor(256 c - 127.5) in the mantissa of 1.5 * 2^23 + q (exact for
                        // the clamped coordinates): texel floor(q / 256), weight (q & 255) / 256,
                        // the split of split_coord with its 1/256 weights (a weight that rounds
                        // up to 1 is weight 0 on the next texel, the same blend)
                        const float2 uc =
                            kCoordClamp ? f2(fminf(fmaxf(uv.x, lo.x), hi.x), fminf(fmaxf(uv.y, lo.y), hi.y)) : uv;
                        const float2 fq = __fadd2_rd(fma2(uc, splat(256.f), splat(-127.5f)), splat(12582912.0f));
                        const unsigned bu = __float_as_uint(fq.x), bv = __float_as_uint(fq.y);
                        const float2 wab = q8_weight2(f2(q8_k1(bu), q8_k1(bv)));
                        // texel index in 32 bits (a slot holds fewer than 2^31 texels):
                        // bu >> 8 = 0x4B4000 + floor(q / 256), so y0 * pitch + x0 is
                        // (bv >> 8) * pitch + (bu >> 8) - 0x4B4000 (pitch + 1), in wrapping
                        // unsigned arithmetic
                        const int t = (int)((bv >> 8) * (unsigned)pitch + (bu >> 8) - kq);
                        const float2 t00 = __ldg(img + t), t10 = __ldg(img + t + 1);
                        const float2 t01 = __ldg(img + (t + pitch)), t11 = __ldg(img + (t + pitch + 1));
                        // bilinear blend of (r, L) as two lerps along x and one along y, both
                        // channels per instruction
                        const float2 p0 = fma2(splat(wab.x), fma2(t00, splat(-1.f), t10), t00);
                        const float2 p1 = fma2(splat(wab.x), fma2(t01, splat(-1.f), t11), t01);
                        rl = fma2(splat(wab.y), fma2(p0, splat(-1.f), p1), p0);
                    } else {
                        rl = sample_pair<kSampling>(img, a.rl_pitch, a.W, a.H, V.tex, uv.x, uv.y);
                    }
                    // r * chord / L with chord = |d| / m: r * nd2 * rsqrt(nd2 * (m L)^2),
                    // one reciprocal square root for the chord and the division by L; formed
                    // for every sample and selected (0 where L < kEps, which the reference skips)
                    const float nd2 = fadd(dxy, zq.y);
                    const float mL = fmul(fmaxf(mxy, zq.z), rl.y);
                    const float q = fmul(rl.x, fmul(nd2, rsqrtf(fmul(nd2, fmul(mL, mL)))));
                    const float value = rl.y >= kEps ? q : 0.f;
                    float vj = fadd(val[j], fmul(fmul(a.lambda, value), mw[j]));
                    if (kClamp) {
                        if (a.use_min) vj = fmaxf(a.vmin, vj);
                        if (a.use_max) vj = fminf(a.vmax, vj);
                    }
                    if (kStore == 1) vj = __half2float(__float2half_rn(vj));
                    val[j] = vj;
                }
                };
                if (kSampling == kSampleQ8 && V.inside) zloop(std::false_type{});
                else zloop(std::true_type{});
            }
        };
        if (nzc == kBpZPersp) views(std::true_type{});
        else views(std::false_type{});
#pragma unroll
        for (int j = 0; j < kBpZPersp; ++j)
            if (j < nzc) bp_store<kStore>(a, base + (size_t)j * plane, val[j]);
        return;
    }
    for (int j = 0; j < nzc; ++j) {
        const size_t idx = base + (size_t)j * plane;
        const float cz = fadd(g.bmin.z, fmul(fadd((float)(z0 + j), 0.5f), g.vs.z));
        const float3 c = make_float3(cx, cy, cz);
        const float bxv = fsub(cx, fmul(0.5f, g.vs.x)), byv = fsub(cy, fmul(0.5f, g.vs.y)),
                    bzv = fsub(cz, fmul(0.5f, g.vs.z));
        float val = bp_load<kStore>(a, idx);
        const float mw = kMask ? mask_weight(a.mask + idx) : 1.f;
        for (int p = 0; p < a.nviews; ++p) {
            const BpView& V = sv[p];
            const float2* img = a.rl + (size_t)p * a.rl_slot;
            float value = 0.f;
            for (unsigned k = 0; k < count; ++k) {
                const unsigned dx = k % (unsigned)n, dy = (k / (unsigned)n) % (unsigned)n, dz = k / (unsigned)(n * n);
                const float px = fadd(bxv, fdiv(fmul(g.vs.x, fadd((float)dx, 0.5f)), (float)n));
                const float py = fadd(byv, fdiv(fmul(g.vs.y, fadd((float)dy, 0.5f)), (float)n));
                const float pz = fadd(bzv, fdiv(fmul(g.vs.z, fadd((float)dz, 0.5f)), (float)n));
                float u = fadd(fadd(fadd(fmul(V.mu[0], px), fmul(V.mu[1], py)), fmul(V.mu[2], pz)), V.mu[3]);
                float v = fadd(fadd(fadd(fmul(V.mv[0], px), fmul(V.mv[1], py)), fmul(V.mv[2], pz)), V.mv[3]);
                const float w = fadd(fadd(fadd(fmul(V.mw[0], px), fmul(V.mw[1], py)), fmul(V.mw[2], pz)), V.mw[3]);
                u = div_fast(u, w);
                v = div_fast(v, w);
                float2 rl;
                if (kSampling == kSampleQ8) {
                    // the bilinear blend of (r, L) as paired FMAs: both channels per
                    // instruction (weights as the 1/256 texture filter rounds them)
                    int x0, y0;
                    float wa, wb;
                    split_coord<kSampling>(u, a.W, x0, wa);
                    split_coord<kSampling>(v, a.H, y0, wb);
                    float2 t00, t10, t01, t11;
                    taps(img + (ptrdiff_t)y0 * (ptrdiff_t)a.rl_pitch, a.rl_pitch, x0, t00, t10, t01, t11);
                    const float ob = fsub(1.f, wb), oa = fsub(1.f, wa);
                    rl = __fmul2_rn(splat(fmul(oa, ob)), t00);
                    rl = fma2(splat(fmul(wa, ob)), t10, rl);
                    rl = fma2(splat(fmul(oa, wb)), t01, rl);
                    rl = fma2(splat(fmul(wa, wb)), t11, rl);
                } else {
                    rl = sample_pair<kSampling>(img, a.rl_pitch, a.W, a.H, V.tex, u, v);
                }
                if (rl.y >= kEps) {
                    const float3 dir = make_float3(fsub(px, V.src[0]), fsub(py, V.src[1]), fsub(pz, V.src[2]));
                    const float l = chord_in_voxel(make_float3(px, py, pz), dir, c, vs);
                    value = fadd(value, div_fast(fmul(rl.x, l), rl.y));
                }
            }
            val = fadd(val, div_fast(fmul(fmul(a.lambda, value), mw), (float)count));
            if (a.use_min) val = fmaxf(a.vmin, val);
            if (a.use_max) val = fminf(a.vmax, val);
            if (kStore == 1) val = __half2float(__float2half_rn(val));
        }
        bp_store<kStore>(a, idx, val);
    }
}

// ---------------------------------------------------------------- weighted back projection
// WBP (WBPPlugin/src/reconstruction/WBP.cpp:22-86) filters every projection with the
// RamLak kernel of GenerateRamLakKernel.cl (fres taps, value at position p = tap -
// fres / 2: 1/4 at 0, 0 at even p, -1 / (p^2 pi^2) at odd p) through
// ConvolutionFourierSpaceImplementation: the projection is padded to the power-of-two
// grid (Wu, Hu) (PaddingForFFT.cl computePaddedCopyForFourierSpace: centred, mirrored
// at the edges), the kernel is zero-padded centred and its origin moved to (0, 0)
// (MoveOriginToCenter.cl), the two are multiplied in Fourier space (a circular
// convolution) and the result is cropped centred (CroppingForFFT.cl).  The kernel row
// sits at row (Hu - 1) / 2 and is moved by Hu / 2, so for an even Hu the filtered row y
// comes from padded row y + 1 (mod Hu).  This kernel evaluates that circular
// convolution directly, one output row per block: the padded source row is staged in
// shared memory and every output pixel sums the nonzero taps.  It also writes the
// pixel's ray length through the complete volume (ComputeRayLength.cl) beside the
// filtered value, the (residual, length) pair the back projector reads.
struct WbpArgs {
    const float* proj;  // H x W projection
    float2* out;        // texel (0, 0) of the padded pair image, or nullptr:
    float* out_f;       //   the filtered image alone, H x W
    size_t pitch;       // float2 units
    int W, H, Wu, Hu;
    int ntaps;          // nonzero taps
    const float* taps;  // device: tap values
    const int* tap_pos; // device: tap positions p
    ViewConst vc;
    SlabConst g;        // complete bounding box in cmin / cmax
};

__device__ __forceinline__ int wbp_pad_index(int i, int n, int nu) {
    const int b = (nu - n) / 2, e = (nu + n) / 2;
    if (i >= b && i < e) return i - b;
    return i < e ? b - i : (n + e - 1) - i;
}

__global__ void __launch_bounds__(256) wbp_filter_kernel(const __grid_constant__ WbpArgs a) {
    extern __shared__ float wbp_row[];  // Wu floats: the padded source row
    const int y = blockIdx.x;
    const int yy = y + (a.Hu / 2 - a.H / 2);                          // row of the padded result
    const int ys = a.Hu > 1 ? a.Hu - 1 : 0;                           // the kernel row after the origin move
    const int sy = wbp_pad_index(((yy - ys) % a.Hu + a.Hu) % a.Hu, a.H, a.Hu);
    const float* src = a.proj + (size_t)sy * a.W;
    for (int x = threadIdx.x; x < a.Wu; x += blockDim.x) wbp_row[x] = src[wbp_pad_index(x, a.W, a.Wu)];
    __syncthreads();
    const int cx = a.Wu / 2 - a.W / 2;
    for (int x = threadIdx.x; x < a.W; x += blockDim.x) {
        const int xx = x + cx;
        float acc = 0.f;
        for (int k = 0; k < a.ntaps; ++k) {
            const int xs = ((xx - a.tap_pos[k]) % a.Wu + a.Wu) % a.Wu;
            acc = fmaf(a.taps[k], wbp_row[xs], acc);
        }
        if (!a.out) {
            a.out_f[(size_t)y * a.W + x] = acc;
            continue;
        }
        // ComputeRayLength.cl:21-33: chord of the pixel-centre ray through the complete box
        const ViewConst& vc = a.vc;
        const float fx = fadd((float)x, 0.5f), fy = fadd((float)y, 0.5f);
        const float3 s = make_float3(fadd(fadd(vc.source.x, fmul(vc.hpitch.x, fx)), fmul(vc.vpitch.x, fy)),
                                     fadd(fadd(vc.source.y, fmul(vc.hpitch.y, fx)), fmul(vc.vpitch.y, fy)),
                                     fadd(fadd(vc.source.z, fmul(vc.hpitch.z, fx)), fmul(vc.vpitch.z, fy)));
        float tin, tout;
        slab_test(make_float3(a.g.cmin.x, a.g.cmin.y, a.g.cmin.z), make_float3(a.g.cmax.x, a.g.cmax.y, a.g.cmax.z), s,
                  make_float3(vc.inv.x, vc.inv.y, vc.inv.z), tin, tout);
        a.out[(size_t)y * a.pitch + x] = make_float2(acc, fmaxf(fsub(tout, tin), 0.f));
    }
}

// ---------------------------------------------------------------- small kernels
__global__ void compare_kernel(const float* real, const float* virt, float* res, size_t n) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) res[i] = fsub(real[i], virt[i]);
}

__global__ void loc_kernel(float* proj, float* len, float c, size_t n) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        float l = len[i];
        proj[i] = l > kEps ? fdiv(fmul(proj[i], c), l) : 0.f;
        len[i] = c;
    }
}

__global__ void ray_length_kernel(ViewConst vc, SlabConst g, int W, int H, float* out) {
    int gx = blockIdx.x * blockDim.x + threadIdx.x, gy = blockIdx.y;
    if (gx >= W || gy >= H) return;
    float fx = fadd((float)gx, 0.5f), fy = fadd((float)gy, 0.5f);
    float3 s = make_float3(fadd(fadd(vc.source.x, fmul(vc.hpitch.x, fx)), fmul(vc.vpitch.x, fy)),
                           fadd(fadd(vc.source.y, fmul(vc.hpitch.y, fx)), fmul(vc.vpitch.y, fy)),
                           fadd(fadd(vc.source.z, fmul(vc.hpitch.z, fx)), fmul(vc.vpitch.z, fy)));
    float tin, tout;
    slab_test(make_float3(g.cmin.x, g.cmin.y, g.cmin.z), make_float3(g.cmax.x, g.cmax.y, g.cmax.z), s,
              make_float3(vc.inv.x, vc.inv.y, vc.inv.z), tin, tout);
    out[(size_t)gy * W + gx] = fmaxf(fsub(tout, tin), 0.f);
}

// Interleave separate residual / ray-length images into a pitched float2 image.
__global__ void pack_pair_kernel(const float* r, const float* l, float2* out, size_t pitch, int W, int H) {
    int gx = blockIdx.x * blockDim.x + threadIdx.x, gy = blockIdx.y;
    if (gx >= W || gy >= H) return;
    size_t i = (size_t)gy * W + gx;
    out[(size_t)gy * pitch + gx] = make_float2(r[i], l[i]);
}

template <typename T>
__global__ void convert_from_float_kernel(const float* in, T* out, size_t n) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = store_cast<T>(in[i]);
}

template <typename T>
__global__ void convert_to_float_kernel(const T* in, float* out, size_t n) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = load_voxel(in + i);
}

__global__ void fill_kernel(float* out, float v, size_t n) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = v;
}

}  // namespace etcu
