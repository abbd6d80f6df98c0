// Blob basis functions: perspective forward and back projection of Kaiser-Bessel blob
// coefficients and their voxelisation (ettention/libReconstruction: ocl_src/BlobRaytracer.hl,
// ocl_src/PerspectiveBeamsForwardProjectionWithBlobs.cl,
// ocl_src/PerspectiveBeamsBackProjectionWithBlobs.cl, ocl_src/VolumeConvolution.cl,
// src/algorithm/blobs/*).  Included by etcu_api.cu after kernels.cuh.
#pragma once

namespace etcu {

// Column-major 4x4 matrix as the reference's Matrix4x4 (value index 4 * column + row).
struct Mat4f {
    float v[16];
};

// Matrix4x4.hl multiply: result component = sum over columns, left to right.
__device__ __forceinline__ float4 mat_mul(const Mat4f& m, float4 p) {
    const float* c = m.v;
    return make_float4(fadd(fadd(fadd(fmul(c[0], p.x), fmul(c[4], p.y)), fmul(c[8], p.z)), fmul(c[12], p.w)),
                       fadd(fadd(fadd(fmul(c[1], p.x), fmul(c[5], p.y)), fmul(c[9], p.z)), fmul(c[13], p.w)),
                       fadd(fadd(fadd(fmul(c[2], p.x), fmul(c[6], p.y)), fmul(c[10], p.z)), fmul(c[14], p.w)),
                       fadd(fadd(fadd(fmul(c[3], p.x), fmul(c[7], p.y)), fmul(c[11], p.z)), fmul(c[15], p.w)));
}

// BlobRaytracer.hl SampleBlob: linear interpolation of the ray-integration table; OpenCL's
// clamp(t, 0, 1) is min(max(t, 0), 1), so a NaN distance reads entry 0.
__device__ __forceinline__ float sample_blob(const float* table, int n, float t) {
    const float coord = fmul(fminf(fmaxf(t, 0.f), 1.f), (float)(n - 1));
    const int left = (int)floorf(coord);
    const float lv = table[left], rv = table[min(n - 1, left + 1)];
    return fadd(lv, fmul(fsub(rv, lv), fsub(coord, (float)left)));
}

struct BlobFpArgs {
    const float* vol;       // sub-volume base, x fastest
    int rx, ry, rz;
    float4 bmin, vs;        // sub-volume box corner and voxel size
    Mat4f p2w;              // projection -> world (the float inverse of the projection matrix)
    float4 source;
    float R;                // blob radius in world units (support radius * vs.x)
    int grid;               // neighbourhood radius in voxels
    const float* table;     // ray-integration table
    int ntable;
    int W, H;
    float* proj;            // H x W, added to
    float* len;
};

// PerspectiveBeamsForwardProjectionWithBlobs.cl execute + BlobTraverseRay: one ray per
// pixel through (x, y, 1) of the projection space, stepped slice by slice along its
// dominant axis; every voxel of the slice neighbourhood whose centre is closer than R to
// the ray adds table(dist / R) times its value (and the weight alone to the length).
// A block is 32 pixels x kBlobFpParts threads: part k of a pixel walks its k-th run of
// slices (its slice positions accumulated from the first slice exactly as one walker
// would), and part 0 adds the parts' sums in order.  The sums within a part follow the
// reference's order (slice, neighbour row, neighbour); the parts split the ray so that a
// 256^2 detector fills the GPU.
constexpr int kBlobFpParts = 8;

__global__ void __launch_bounds__(32 * kBlobFpParts) blob_fp_kernel(const __grid_constant__ BlobFpArgs a) {
    extern __shared__ float blob_table[];
    __shared__ float part_val[kBlobFpParts][32], part_len[kBlobFpParts][32];
    const int tid = threadIdx.y * 32 + threadIdx.x;
    for (int i = tid; i < a.ntable; i += 32 * kBlobFpParts) blob_table[i] = a.table[i];
    __syncthreads();
    const int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y, part = threadIdx.y;
    float val = 0.f, lval = 0.f;
    if (x < a.W && y < a.H) {
        // TransformCoordG(projection2world, (x, y, 1))
        const float4 wp = mat_mul(a.p2w, make_float4((float)x, (float)y, 1.f, 1.f));
        const float3 world = make_float3(fdiv(wp.x, wp.w), fdiv(wp.y, wp.w), fdiv(wp.z, wp.w));
        const float3 src = make_float3(a.source.x, a.source.y, a.source.z);
        float3 d = make_float3(fsub(world.x, src.x), fsub(world.y, src.y), fsub(world.z, src.z));
        const float nd = __fsqrt_rn(fadd(fadd(fmul(d.x, d.x), fmul(d.y, d.y)), fmul(d.z, d.z)));
        const float3 ray = make_float3(fdiv(d.x, nd), fdiv(d.y, nd), fdiv(d.z, nd));
        const float3 ar = make_float3(fabsf(ray.x), fabsf(ray.y), fabsf(ray.z));
        int axis;
        if (ar.x >= fmaxf(ar.y, ar.z)) axis = 0;
        else if (ar.y >= fmaxf(ar.x, ar.z)) axis = 1;
        else axis = 2;
        const float rc[3] = {ray.x, ray.y, ray.z}, sc[3] = {src.x, src.y, src.z};
        const float bm[3] = {a.bmin.x, a.bmin.y, a.bmin.z}, vsz[3] = {a.vs.x, a.vs.y, a.vs.z};
        const int res[3] = {a.rx, a.ry, a.rz};
        // pointOnRay = source + tMin[axis] * ray, tMin = (bBoxMin + vs / 2 - source) / ray
        const float tmin = fdiv(fsub(fadd(bm[axis], fmul(0.5f, vsz[axis])), sc[axis]), rc[axis]);
        float p[3] = {fadd(sc[0], fmul(tmin, rc[0])), fadd(sc[1], fmul(tmin, rc[1])), fadd(sc[2], fmul(tmin, rc[2]))};
        const float st[3] = {fmul(fdiv(rc[0], rc[axis]), vsz[0]), fmul(fdiv(rc[1], rc[axis]), vsz[1]),
                             fmul(fdiv(rc[2], rc[axis]), vsz[2])};
        const int ex = axis == 0 ? 1 : (axis == 1 ? 2 : 0);  // slice axes: x -> (y, z), y -> (z, x), z -> (x, y)
        const int ey = axis == 0 ? 2 : (axis == 1 ? 0 : 1);
        const float R2 = fmul(a.R, a.R);
        const size_t plane = (size_t)a.rx * (size_t)a.ry;
        const int nslices = res[axis];
        const int per = (nslices + kBlobFpParts - 1) / kBlobFpParts;
        const int s0 = min(nslices, part * per), s1 = min(nslices, s0 + per);
        for (int slice = 0; slice < s0; ++slice)
            for (int k = 0; k < 3; ++k) p[k] = fadd(p[k], st[k]);
        for (int slice = s0; slice < s1; ++slice) {
            int base[3];
            for (int k = 0; k < 3; ++k) base[k] = (int)floorf(fdiv(fsub(p[k], bm[k]), vsz[k]));
            for (int dy = -a.grid; dy <= a.grid; ++dy) {
                for (int dx = -a.grid; dx <= a.grid; ++dx) {
                    int gc[3] = {base[0], base[1], base[2]};
                    gc[ex] += dx;
                    gc[ey] += dy;
                    if (gc[0] < 0 || gc[1] < 0 || gc[2] < 0 || gc[0] >= res[0] || gc[1] >= res[1] || gc[2] >= res[2])
                        continue;
                    float cen[3];
                    for (int k = 0; k < 3; ++k)
                        cen[k] = fadd(fadd(bm[k], fmul(0.5f, vsz[k])), fmul((float)gc[k], vsz[k]));
                    const float t = -fadd(fadd(fmul(fsub(sc[0], cen[0]), rc[0]), fmul(fsub(sc[1], cen[1]), rc[1])),
                                          fmul(fsub(sc[2], cen[2]), rc[2]));
                    const float c0 = fsub(fadd(sc[0], fmul(t, rc[0])), cen[0]);
                    const float c1 = fsub(fadd(sc[1], fmul(t, rc[1])), cen[1]);
                    const float c2 = fsub(fadd(sc[2], fmul(t, rc[2])), cen[2]);
                    const float d2 = fadd(fadd(fmul(c0, c0), fmul(c1, c1)), fmul(c2, c2));
                    if (d2 < R2) {
                        const float w = sample_blob(blob_table, a.ntable, fdiv(__fsqrt_rn(d2), a.R));
                        val = fadd(val, fmul(w, a.vol[(size_t)gc[2] * plane + (size_t)gc[1] * a.rx + gc[0]]));
                        lval = fadd(lval, w);
                    }
                }
            }
            for (int k = 0; k < 3; ++k) p[k] = fadd(p[k], st[k]);
        }
    }
    part_val[part][threadIdx.x] = val;
    part_len[part][threadIdx.x] = lval;
    __syncthreads();
    if (part == 0 && x < a.W && y < a.H) {
        float v = part_val[0][threadIdx.x], l = part_len[0][threadIdx.x];
        for (int k = 1; k < kBlobFpParts; ++k) {
            v = fadd(v, part_val[k][threadIdx.x]);
            l = fadd(l, part_len[k][threadIdx.x]);
        }
        const size_t i = (size_t)y * a.W + x;
        a.proj[i] = fadd(a.proj[i], v);
        a.len[i] = fadd(a.len[i], l);
    }
}

struct BlobBpArgs {
    float* vol;             // sub-volume base
    int rx, ry, rz;
    float4 bmin, vs;
    Mat4f w2p, p2w;         // projection matrix and its float inverse
    float4 source, detector, hpitch, vpitch;
    float R;
    const float* table;
    int ntable;
    const float* residual;  // H x W
    const float* raylength;
    int W, H;
    float lambda;
    const uint8_t* mask;    // or nullptr
};

// PerspectiveBeamsBackProjectionWithBlobs.cl correct: one blob (voxel) per thread.
__global__ void __launch_bounds__(128) blob_bp_kernel(const __grid_constant__ BlobBpArgs a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, z = blockIdx.z;
    if (x >= a.rx) return;
    const float4 c = make_float4(fadd(a.bmin.x, fmul(fadd((float)x, 0.5f), a.vs.x)),
                                 fadd(a.bmin.y, fmul(fadd((float)y, 0.5f), a.vs.y)),
                                 fadd(a.bmin.z, fmul(fadd((float)z, 0.5f), a.vs.z)), 1.f);
    const float4 pc = mat_mul(a.w2p, c);
    if (!(pc.w > 0.f)) return;
    const float u = fdiv(pc.x, pc.w), v = fdiv(pc.y, pc.w);
    const float3 pv = make_float3(fsub(fadd(fadd(a.detector.x, fmul(u, a.hpitch.x)), fmul(v, a.vpitch.x)), a.source.x),
                                  fsub(fadd(fadd(a.detector.y, fmul(u, a.hpitch.y)), fmul(v, a.vpitch.y)), a.source.y),
                                  fsub(fadd(fadd(a.detector.z, fmul(u, a.hpitch.z)), fmul(v, a.vpitch.z)), a.source.z));
    const float3 q = make_float3(fsub(c.x, a.source.x), fsub(c.y, a.source.y), fsub(c.z, a.source.z));
    const float lp = __fsqrt_rn(fadd(fadd(fmul(pv.x, pv.x), fmul(pv.y, pv.y)), fmul(pv.z, pv.z)));
    const float lq = __fsqrt_rn(fadd(fadd(fmul(q.x, q.x), fmul(q.y, q.y)), fmul(q.z, q.z)));
    const float ldx = __fsqrt_rn(fadd(fadd(fmul(a.hpitch.x, a.hpitch.x), fmul(a.hpitch.y, a.hpitch.y)),
                                      fmul(a.hpitch.z, a.hpitch.z)));
    const float ldy = __fsqrt_rn(fadd(fadd(fmul(a.vpitch.x, a.vpitch.x), fmul(a.vpitch.y, a.vpitch.y)),
                                      fmul(a.vpitch.z, a.vpitch.z)));
    const float r = fdiv(fmul(a.R, lp), lq);
    const float alpha = asinf(fdiv(a.R, lq));
    const float bx = acosf(fdiv(fadd(fadd(fmul(a.hpitch.x, pv.x), fmul(a.hpitch.y, pv.y)), fmul(a.hpitch.z, pv.z)),
                                fmul(ldx, lp)));
    const float by = acosf(fdiv(fadd(fadd(fmul(a.vpitch.x, pv.x), fmul(a.vpitch.y, pv.y)), fmul(a.vpitch.z, pv.z)),
                                fmul(ldy, lp)));
    // convert_int_rtp: the window half-sizes rounded up
    const float wx = fdiv(fmaxf(fdiv(r, sinf(fsub(bx, alpha))), fdiv(r, sinf(fadd(bx, alpha)))), ldx);
    const float wy = fdiv(fmaxf(fdiv(r, sinf(fsub(by, alpha))), fdiv(r, sinf(fadd(by, alpha)))), ldy);
    // a window that is not finite or wider than any detector (a blob next to the source):
    // the blob is skipped
    if (!(wx < 4096.f) || !(wy < 4096.f)) return;
    const int sx = (int)ceilf(wx), sy = (int)ceilf(wy);
    // convert_int2_rtz(params + 0.5 * sign(params))
    const int bxp = (int)truncf(fadd(u, fmul(0.5f, clsign(u)))), byp = (int)truncf(fadd(v, fmul(0.5f, clsign(v))));
    const float R2 = fmul(a.R, a.R);
    float acc = 0.f, val = 0.f;
    for (int dy = -sy; dy <= sy; ++dy) {
        for (int dx = -sx; dx <= sx; ++dx) {
            const int px = bxp + dx, py = byp + dy;
            if (px < 0 || py < 0 || px >= a.W || py >= a.H) continue;
            const size_t pi = (size_t)py * a.W + px;
            const float len = a.raylength[pi], res = a.residual[pi];
            if (!(res != 0.f && len > 1.f)) continue;
            const float4 w = mat_mul(a.p2w, make_float4((float)px, (float)py, 1.f, 1.f));
            // divisions of the window loop to within one ulp (reciprocal and one correction):
            // the loop runs per (coefficient, pixel) and its IEEE divisions were most of it
            float3 dd = make_float3(fsub(div_fast(w.x, w.w), a.source.x), fsub(div_fast(w.y, w.w), a.source.y),
                                    fsub(div_fast(w.z, w.w), a.source.z));
            const float n = __fsqrt_rn(fadd(fadd(fmul(dd.x, dd.x), fmul(dd.y, dd.y)), fmul(dd.z, dd.z)));
            dd = make_float3(div_fast(dd.x, n), div_fast(dd.y, n), div_fast(dd.z, n));
            const float t0 = fadd(fadd(fmul(dd.x, q.x), fmul(dd.y, q.y)), fmul(dd.z, q.z));
            const float dist2 = fsub(fadd(fadd(fmul(q.x, q.x), fmul(q.y, q.y)), fmul(q.z, q.z)), fmul(t0, t0));
            if (R2 > dist2) {
                const float wt = sample_blob(a.table, a.ntable, __fsqrt_rn(div_fast(dist2, R2)));
                acc = fadd(acc, wt);
                val = fadd(val, div_fast(fmul(res, wt), len));
            }
        }
    }
    if (acc > 1e-2f) {  // WEAK_EPSILON
        const size_t id = ((size_t)z * a.ry + y) * a.rx + x;
        const float m = a.mask ? mask_weight(a.mask + id) : 1.f;
        a.vol[id] = fadd(a.vol[id], fdiv(fmul(fmul(a.lambda, val), m), acc));
    }
}

// VolumeConvolution.cl over the blob coefficients with a zero border of the kernel
// radius (VolumeConvolutionOperator.cpp:30-37): out = sum over the kernel (z, y, x order)
// of kernel * input.
__global__ void __launch_bounds__(128) blob_voxelize_kernel(const float* in, float* out, int X, int Y, int Z,
                                                            const float* kernel, int ks) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, z = blockIdx.z;
    if (x >= X) return;
    const int r = ks / 2;
    float value = 0.f;
    for (int kz = 0; kz < ks; ++kz)
        for (int ky = 0; ky < ks; ++ky)
            for (int kx = 0; kx < ks; ++kx) {
                const int sx = x + kx - r, sy = y + ky - r, sz = z + kz - r;
                const float iv = (sx < 0 || sy < 0 || sz < 0 || sx >= X || sy >= Y || sz >= Z)
                                     ? 0.f : in[((size_t)sz * Y + sy) * X + sx];
                value = fadd(value, fmul(kernel[(kz * ks + ky) * ks + kx], iv));
            }
    out[((size_t)z * Y + y) * X + x] = value;
}

// CompareKernel for the blob iterations: residual = real - virtual, and the sum of the
// squared residuals (double, one atomic per block) for the iteration's report.
__global__ void __launch_bounds__(256) blob_residual_kernel(const float* real, const float* virt, float* res,
                                                            size_t n, double* sum_sq) {
    __shared__ double part[8];
    double acc = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float r = fsub(real[i], virt[i]);
        res[i] = r;
        acc += (double)r * (double)r;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[w];
        atomicAdd(sum_sq, t);
    }
}

}  // namespace etcu
