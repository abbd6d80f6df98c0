/*
 * TEST INFRASTRUCTURE ONLY -- never linked into, loaded by or called from the
 * product library (ettention_b200).  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU baseline / reference arm use it, and only as the checker.
 *
 * CPU oracle for Ettention's block-iterative reconstruction hot path
 * (c3di/ettention, libReconstruction).  The reference cannot be built here
 * (it needs Boost, OpenCL headers and an ICD, FreeImage, clAmdFft and GTest),
 * so this file restates the OpenCL kernels and the host-side driver loop in
 * plain C, in two precisions:
 *   *_f32  FP32 "reference order": the kernels' float operations in their order
 *   *_f64  FP64 "truth": the same algorithm in double precision
 * The restatement is pinned against the reference's own golden fixtures
 * (ettention/test/data/{forward_projection,back_projection,...}); the
 * fixtures are converted to NumPy archives under tests/golden by
 * tests/golden/make_golden.py.
 *
 * Build: oracle/build_oracle.sh -> oracle/liboracle.so (OpenMP).
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_EPS 1e-4            /* ocl_src/Math.hl:4 EPSILON */
#define ORC_MAX_LOOP 4096u      /* ocl_src/DDARaytracer.hl:86 maxLoopExecs */
#define ORC_FRACT_MAX 0x1.fffffep-1 /* OpenCL fract() upper clamp */

enum { ORC_WEIGHTS_EXACT = 0, ORC_WEIGHTS_Q8 = 1, ORC_WEIGHTS_Q8_TRUNC = 2 };

/* View geometry as the reference packs it (ocl_src/ProjectionGeometry.hl:4-15). */
typedef struct {
    double source[3], detector[3], hpitch[3], vpitch[3];
    double ray[3];          /* normalised direction used by the parallel kernels */
    int width, height;
    int perspective;
} orc_view;

/* Volume geometry of one sub-volume (ocl_src/VolumeGeometry.hl:4-15). */
typedef struct {
    int res[3];
    double bmin[3], bmax[3];
    double cmin[3], cmax[3];
    double voxel[3];
} orc_volgeom;

/* IEEE binary16 <-> binary32, round to nearest even (vload_half/vstore_half). */
static float orc_half_to_float(uint16_t h)
{
    uint32_t s = (uint32_t)(h >> 15) << 31, e = (h >> 10) & 0x1f, m = h & 0x3ff, bits;
    if (e == 0) {
        if (m == 0) bits = s;
        else {
            int sh = 0;
            while (!(m & 0x400)) { m <<= 1; ++sh; }
            m &= 0x3ff;
            bits = s | ((uint32_t)(127 - 15 - sh + 1) << 23) | (m << 13);
        }
    } else if (e == 31) bits = s | 0x7f800000u | (m << 13);
    else bits = s | ((e + 127 - 15) << 23) | (m << 13);
    float f;
    memcpy(&f, &bits, 4);
    return f;
}

static uint16_t orc_float_to_half(float f)
{
    uint32_t x;
    memcpy(&x, &f, 4);
    uint32_t s = (x >> 16) & 0x8000u;
    uint32_t ax = x & 0x7fffffffu;
    if (ax >= 0x7f800000u) return (uint16_t)(s | 0x7c00u | (ax > 0x7f800000u ? 0x200u : 0));
    if (ax >= 0x477ff000u) return (uint16_t)(s | 0x7c00u); /* overflow after rounding */
    if (ax < 0x38800000u) {                                 /* subnormal or zero */
        if (ax < 0x33000000u) return (uint16_t)s;
        uint32_t m = (ax & 0x7fffffu) | 0x800000u;
        int shift = 126 - (int)(ax >> 23);                  /* 14..24 */
        uint32_t r = m >> shift, rem = m & ((1u << shift) - 1), half = 1u << (shift - 1);
        if (rem > half || (rem == half && (r & 1))) ++r;
        return (uint16_t)(s | r);
    }
    uint32_t r = ((ax >> 13) - (112u << 10));
    uint32_t rem = ax & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (r & 1))) ++r;
    return (uint16_t)(s | r);
}

/* 1/256 fixed-point weight of GPU texture filtering: the fractional position is
 * rounded half up to 8 bits (measured on the texture unit; the reference's golden
 * back-projection volumes are reproduced to ~1e-7 with it). */
static int orc_q8_mode = ORC_WEIGHTS_Q8;
static double orc_q8(double a)
{
    if (orc_q8_mode == ORC_WEIGHTS_Q8_TRUNC) return floor(a * 256.0) / 256.0;
    return floor(a * 256.0 + 0.5) / 256.0;
}

/* ---- FP32 reference-order instantiation ---- */
#define REAL float
#define SUF _f32
#define FMIN fminf
#define FMAX fmaxf
#define FLOOR floorf
#define SQRT sqrtf
#define RMAXV FLT_MAX
#include "oracle_impl.h"
#undef REAL
#undef SUF
#undef FMIN
#undef FMAX
#undef FLOOR
#undef SQRT
#undef RMAXV

/* ---- FP64 truth instantiation ---- */
#define REAL double
#define SUF _f64
#define FMIN fmin
#define FMAX fmax
#define FLOOR floor
#define SQRT sqrt
#define RMAXV DBL_MAX
#include "oracle_impl.h"
#undef REAL
#undef SUF
#undef FMIN
#undef FMAX
#undef FLOOR
#undef SQRT
#undef RMAXV

/* ------------------------------------------------------------------------- */
/* Exported API (ctypes).  prec is 32 or 64.  Arrays are float32 in both modes
 * so that the FP64 mode's output can be compared with the FP32 paths; the FP64
 * mode accumulates every ray and voxel in double.                           */

int orc_abi_version(void) { return 3; }

void orc_set_q8_mode(int mode) { orc_q8_mode = mode; }

void orc_half_from_float(const float* in, uint16_t* out, long n)
{
    for (long i = 0; i < n; ++i) out[i] = orc_float_to_half(in[i]);
}

void orc_float_from_half(const uint16_t* in, float* out, long n)
{
    for (long i = 0; i < n; ++i) out[i] = orc_half_to_float(in[i]);
}

void orc_forward(int prec, const orc_view* view, const orc_volgeom* vg, const void* vol, int half,
                 const uint8_t* mask, int samples, float* proj, float* len)
{
    if (prec == 64) forward_f64(view, vg, vol, half, mask, samples, proj, len);
    else forward_f32(view, vg, vol, half, mask, samples, proj, len);
}

void orc_back_parallel(int prec, const orc_volgeom* vg, const double* mat16, const float* samples4, int nsamples,
                       const float* residual, const float* raylen, int W, int H, void* vol, int half,
                       const uint8_t* mask, float lambda, int weights)
{
    if (weights != ORC_WEIGHTS_EXACT) orc_q8_mode = weights;
    if (prec == 64) back_parallel_f64(vg, mat16, samples4, nsamples, residual, raylen, W, H, vol, half, mask, lambda, weights);
    else back_parallel_f32(vg, mat16, samples4, nsamples, residual, raylen, W, H, vol, half, mask, lambda, weights);
}

void orc_back_perspective(int prec, const orc_volgeom* vg, const double* mat16, const double* source3, int n,
                          const float* residual, const float* raylen, int W, int H, void* vol, int half,
                          const uint8_t* mask, float lambda, int weights, int use_min, float vmin, int use_max,
                          float vmax)
{
    if (weights != ORC_WEIGHTS_EXACT) orc_q8_mode = weights;
    if (prec == 64)
        back_perspective_f64(vg, mat16, source3, n, residual, raylen, W, H, vol, half, mask, lambda, weights,
                             use_min, vmin, use_max, vmax);
    else
        back_perspective_f32(vg, mat16, source3, n, residual, raylen, W, H, vol, half, mask, lambda, weights,
                             use_min, vmin, use_max, vmax);
}

void orc_ray_length(int prec, const orc_view* view, const orc_volgeom* vg, float* out)
{
    if (prec == 64) ray_length_f64(view, vg, out);
    else ray_length_f32(view, vg, out);
}

/* Compare.cl:1-9 residual = real - virtual */
void orc_compare(const float* real, const float* virt, float* residual, long n)
{
    for (long i = 0; i < n; ++i) residual[i] = real[i] - virt[i];
}

/* VirtualProjection.cl:3-10 long-object compensation */
void orc_long_object_compensation(float* proj, float* len, float constant_length, long n)
{
    for (long i = 0; i < n; ++i) {
        proj[i] = len[i] > 1e-4f ? proj[i] * constant_length / len[i] : 0.0f;
        len[i] = constant_length;
    }
}

/*
 * Host driver loop of BlockIterativeReconstructionOperator.cpp:92-142.  The
 * caller passes views and projections already in iteration order, every
 * sub-volume's geometry (slabs[S]) and, per view, the back-projection matrix
 * and (parallel beams) the sample pattern.  Per block: forward projection of
 * every slab into zeroed virtual / traversal buffers, residuals (with optional
 * long-object compensation, constant length per view), then back projection
 * of the slabs in reverse order with lambda / blockSize.
 * vol_slabs[s] points at sub-volume s (x-fastest, z-slab split).
 */
int orc_block_iterative(int prec, int nviews, const orc_view* views, const float* real_proj,
                        int nslabs, const orc_volgeom* slabs, void** vol_slabs, int half,
                        uint8_t** mask_slabs, int fp_samples, const double* mats, const float* bp_samples4,
                        int bp_nsamples, int persp_n, float lambda, int block_size, int iterations,
                        int use_loc, const float* loc_lengths, int weights, int use_min, float vmin,
                        int use_max, float vmax)
{
    if (nviews <= 0 || block_size <= 0) return -1;
    const int W = views[0].width, H = views[0].height;
    const size_t P = (size_t)W * H;
    int nblocks = (nviews + block_size - 1) / block_size;
    float* virt = (float*)malloc(sizeof(float) * P * (size_t)block_size);
    float* len = (float*)malloc(sizeof(float) * P * (size_t)block_size);
    float* res = (float*)malloc(sizeof(float) * P * (size_t)block_size);
    if (!virt || !len || !res) { free(virt); free(len); free(res); return -2; }
    for (int it = 0; it < iterations; ++it) {
        for (int b = 0; b < nblocks; ++b) {
            int first = b * block_size;
            int bs = (b < nblocks - 1) ? block_size : nviews - first;
            memset(virt, 0, sizeof(float) * P * (size_t)bs);
            memset(len, 0, sizeof(float) * P * (size_t)bs);
            for (int s = 0; s < nslabs; ++s)
                for (int p = 0; p < bs; ++p)
                    orc_forward(prec, &views[first + p], &slabs[s], vol_slabs[s], half,
                                mask_slabs ? mask_slabs[s] : NULL, fp_samples, virt + P * p, len + P * p);
            for (int p = 0; p < bs; ++p) {
                if (use_loc) orc_long_object_compensation(virt + P * p, len + P * p, loc_lengths[first + p], (long)P);
                orc_compare(real_proj + P * (size_t)(first + p), virt + P * p, res + P * p, (long)P);
            }
            float lam = lambda / (float)bs;
            for (int s = nslabs - 1; s >= 0; --s)
                for (int p = 0; p < bs; ++p) {
                    const orc_view* v = &views[first + p];
                    if (!v->perspective)
                        orc_back_parallel(prec, &slabs[s], mats + 16 * (size_t)(first + p),
                                          bp_samples4 + 4 * (size_t)bp_nsamples * (size_t)(first + p), bp_nsamples,
                                          res + P * p, len + P * p, W, H, vol_slabs[s], half,
                                          mask_slabs ? mask_slabs[s] : NULL, lam, weights);
                    else
                        orc_back_perspective(prec, &slabs[s], mats + 16 * (size_t)(first + p), v->source, persp_n,
                                             res + P * p, len + P * p, W, H, vol_slabs[s], half,
                                             mask_slabs ? mask_slabs[s] : NULL, lam, weights, use_min, vmin,
                                             use_max, vmax);
                }
        }
    }
    free(virt);
    free(len);
    free(res);
    return 0;
}
