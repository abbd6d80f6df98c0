/*
 * TEST INFRASTRUCTURE ONLY -- never linked into, loaded by or called from the
 * product library.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline use it, and only as the checker.
 *
 * Precision-generic body of the CPU oracle for Ettention's block-iterative hot
 * path.  ettention_oracle.c includes this file twice: once with REAL=float
 * (the "reference-order" FP32 mode that repeats the OpenCL kernels'
 * operations in their order) and once with REAL=double (the FP64 "truth"
 * mode).  Every function names the reference file:line it restates; paths are
 * relative to the reference project root (ettention/libReconstruction/...).
 */

#define FN(name) CAT(name, SUF)
#define CAT(a, b) CAT2(a, b)
#define CAT2(a, b) a##b

typedef struct { REAL x, y, z; } FN(vec);

static inline FN(vec) FN(mk)(REAL x, REAL y, REAL z) { FN(vec) v; v.x = x; v.y = y; v.z = z; return v; }
static inline FN(vec) FN(fromd)(const double* d) { return FN(mk)((REAL)d[0], (REAL)d[1], (REAL)d[2]); }
static inline REAL FN(fminr)(REAL a, REAL b) { return FMIN(a, b); }
static inline REAL FN(fmaxr)(REAL a, REAL b) { return FMAX(a, b); }
/* OpenCL clamp(x, lo, hi) = fmin(fmax(x, lo), hi) */
static inline REAL FN(clampr)(REAL x, REAL lo, REAL hi) { return FMIN(FMAX(x, lo), hi); }
/* OpenCL sign(): +-1 for non-zero, the zero itself for +-0 */
static inline REAL FN(signr)(REAL x) { return x > 0 ? (REAL)1 : (x < 0 ? (REAL)-1 : x); }

/* Per-launch volume constants: ocl_src/VolumeGeometry.hl:4-15 */
typedef struct {
    int res[3];               /* sub-volume resolution (x, y, z) */
    FN(vec) bmin, bmax;       /* sub-volume bounding box */
    FN(vec) cmin, cmax;       /* complete-volume bounding box */
    FN(vec) vs;               /* voxel size */
} FN(vgeo);

static void FN(load_vgeo)(const orc_volgeom* in, FN(vgeo)* g)
{
    for (int i = 0; i < 3; ++i) g->res[i] = in->res[i];
    g->bmin = FN(fromd)(in->bmin); g->bmax = FN(fromd)(in->bmax);
    g->cmin = FN(fromd)(in->cmin); g->cmax = FN(fromd)(in->cmax);
    g->vs = FN(fromd)(in->voxel);
}

/* RayUtils.hl:25-35 invertVectorSafely: zero components become -max */
static inline FN(vec) FN(inv_safe)(FN(vec) r)
{
    FN(vec) o = FN(mk)((REAL)1 / r.x, (REAL)1 / r.y, (REAL)1 / r.z);
    if (r.x == 0) o.x = -RMAXV;
    if (r.y == 0) o.y = -RMAXV;
    if (r.z == 0) o.z = -RMAXV;
    return o;
}

/* RayUtils.hl:7-16 slab test, returns (t_in, t_out) */
static inline void FN(slab)(FN(vec) bmin, FN(vec) bmax, FN(vec) src, FN(vec) inv, REAL* tin, REAL* tout)
{
    REAL t0x = (bmin.x - src.x) * inv.x, t1x = (bmax.x - src.x) * inv.x;
    REAL t0y = (bmin.y - src.y) * inv.y, t1y = (bmax.y - src.y) * inv.y;
    REAL t0z = (bmin.z - src.z) * inv.z, t1z = (bmax.z - src.z) * inv.z;
    REAL mnx = FMIN(t0x, t1x), mny = FMIN(t0y, t1y), mnz = FMIN(t0z, t1z);
    REAL mxx = FMAX(t0x, t1x), mxy = FMAX(t0y, t1y), mxz = FMAX(t0z, t1z);
    *tin = FMAX(FMAX(mnx, mny), mnz);
    *tout = FMIN(FMIN(mxx, mxy), mxz);
}

static inline REAL FN(read_voxel)(const void* vol, int half, size_t idx)
{
    if (half) return (REAL)orc_half_to_float(((const uint16_t*)vol)[idx]);
    return (REAL)((const float*)vol)[idx];
}

/*
 * DDARaytracer.hl:59-110 ddaTraverseRay with the forward projector's
 * FILTER_OPERATOR (ParallelBeamsForwardProjection.cl:5-8): accumulates
 * deltaT * volume(voxel) and deltaT * mask(voxel) (1 without a mask).
 * The step update is written in the kernel's arithmetic form
 * step*stepDifference + (1-step)*(res-deltaT), so non-finite step
 * differences propagate exactly as they do in the reference.
 */
static void FN(dda)(FN(vec) src, FN(vec) ray, const FN(vgeo)* g, const void* vol, int half,
                    const uint8_t* mask, REAL* out_v, REAL* out_l)
{
    FN(vec) inv = FN(inv_safe)(ray);
    REAL tin, tout;
    FN(slab)(g->bmin, g->bmax, src, inv, &tin, &tout);
    FN(vec) ivs = FN(mk)((REAL)1 / g->vs.x, (REAL)1 / g->vs.y, (REAL)1 / g->vs.z);
    REAL acc = 0, accl = 0;
    *out_v = 0; *out_l = 0;
    if (!(tout - tin > (REAL)ORC_EPS)) return;

    /* DDARaytracer.hl:52-57 calculateRayEntryPoint */
    FN(vec) pos = FN(mk)(src.x + tin * ray.x, src.y + tin * ray.y, src.z + tin * ray.z);
    pos.x = FN(clampr)(pos.x, g->bmin.x, g->bmax.x);
    pos.y = FN(clampr)(pos.y, g->bmin.y, g->bmax.y);
    pos.z = FN(clampr)(pos.z, g->bmin.z, g->bmax.z);

    /* DDARaytracer.hl:20-31 getInitialVoxelIndex (round toward zero, clamp) */
    int ix = (int)((pos.x - g->bmin.x) * ivs.x);
    int iy = (int)((pos.y - g->bmin.y) * ivs.y);
    int iz = (int)((pos.z - g->bmin.z) * ivs.z);
    ix = ix < 0 ? 0 : (ix > g->res[0] - 1 ? g->res[0] - 1 : ix);
    iy = iy < 0 ? 0 : (iy > g->res[1] - 1 ? g->res[1] - 1 : iy);
    iz = iz < 0 ? 0 : (iz > g->res[2] - 1 ? g->res[2] - 1 : iz);

    /* DDARaytracer.hl:78-80 */
    FN(vec) sg = FN(mk)(FN(signr)(ray.x), FN(signr)(ray.y), FN(signr)(ray.z));
    FN(vec) sd = FN(mk)(g->vs.x * inv.x * sg.x, g->vs.y * inv.y * sg.y, g->vs.z * inv.z * sg.z);
    int six = (int)sg.x, siy = (int)sg.y, siz = (int)sg.z;

    /* DDARaytracer.hl:33-50 getRemainingDifferenceToVoxelBorder (world-origin grid) */
    FN(vec) r;
    r.x = FLOOR(pos.x * ivs.x) * g->vs.x;
    r.y = FLOOR(pos.y * ivs.y) * g->vs.y;
    r.z = FLOOR(pos.z * ivs.z) * g->vs.z;
    r.x = (ray.x > 0) ? (r.x + g->vs.x - pos.x) * inv.x : (r.x - pos.x) * inv.x;
    r.y = (ray.y > 0) ? (r.y + g->vs.y - pos.y) * inv.y : (r.y - pos.y) * inv.y;
    r.z = (ray.z > 0) ? (r.z + g->vs.z - pos.z) * inv.z : (r.z - pos.z) * inv.z;
    if (ray.x == 0) r.x = RMAXV;
    if (ray.y == 0) r.y = RMAXV;
    if (ray.z == 0) r.z = RMAXV;
    if (r.x == 0) r.x = sd.x;
    if (r.y == 0) r.y = sd.y;
    if (r.z == 0) r.z = sd.z;

    const int rx = g->res[0], ry = g->res[1], rz = g->res[2];
    unsigned brk = 0;
    while (ix >= 0 && iy >= 0 && iz >= 0 && ix < rx && iy < ry && iz < rz && ++brk < ORC_MAX_LOOP) {
        REAL dt = FMIN(FMIN(r.x, r.y), r.z);
        size_t idx = ((size_t)iz * (size_t)ry + (size_t)iy) * (size_t)rx + (size_t)ix;
        acc += dt * FN(read_voxel)(vol, half, idx);
        accl += dt * (mask ? (REAL)((float)mask[idx] / 255.0f) : (REAL)1);
        int incx = (r.x <= r.y && r.x <= r.z);
        int incy = (r.y < r.x && r.y <= r.z);
        int incz = (r.z < r.x && r.z < r.y);
        REAL stx = (REAL)incx, sty = (REAL)incy, stz = (REAL)incz;
        r.x = stx * sd.x + ((REAL)1 - stx) * (r.x - dt);
        r.y = sty * sd.y + ((REAL)1 - sty) * (r.y - dt);
        r.z = stz * sd.z + ((REAL)1 - stz) * (r.z - dt);
        ix += incx * six; iy += incy * siy; iz += incz * siz;
        ++brk;
    }
    *out_v = acc;
    *out_l = accl;
}

/*
 * ParallelBeamsForwardProjection.cl:12-57 (parallel) and
 * PerspectiveBeamsForwardProjection.cl:13-52 (perspective): samples x samples
 * sub-rays per detector pixel, averaged and ADDED (+=) to the outputs.
 */
static void FN(forward)(const orc_view* view, const orc_volgeom* vgin, const void* vol, int half,
                        const uint8_t* mask, int samples, float* proj, float* len)
{
    FN(vgeo) g; FN(load_vgeo)(vgin, &g);
    if (samples == 0) samples = 1; /* ForwardProjectionKernel.cpp:65-68 */
    const int W = view->width, H = view->height;
    FN(vec) src = FN(fromd)(view->source), det = FN(fromd)(view->detector);
    FN(vec) hp = FN(fromd)(view->hpitch), vp = FN(fromd)(view->vpitch);
    FN(vec) ray = FN(fromd)(view->ray);
#pragma omp parallel for schedule(dynamic, 1)
    for (int gy = 0; gy < H; ++gy) {
        for (int gx = 0; gx < W; ++gx) {
            REAL acc = 0, accl = 0, v, l;
            if (!view->perspective) {
                REAL total = (REAL)(samples * samples);
                REAL sdist = (REAL)1 / (REAL)samples, off = sdist / (REAL)2;
                for (int sx = 0; sx < samples; ++sx) {
                    for (int sy = 0; sy < samples; ++sy) {
                        REAL fx = (REAL)gx + off + sdist * (REAL)sx;
                        REAL fy = (REAL)gy + off + sdist * (REAL)sy;
                        FN(vec) s = FN(mk)(src.x + hp.x * fx + vp.x * fy,
                                           src.y + hp.y * fx + vp.y * fy,
                                           src.z + hp.z * fx + vp.z * fy);
                        FN(dda)(s, ray, &g, vol, half, mask, &v, &l);
                        acc += v; accl += l;
                    }
                }
                size_t i = (size_t)gy * W + gx;
                proj[i] = (float)((REAL)proj[i] + acc / total);
                len[i] = (float)((REAL)len[i] + accl / total);
            } else {
                unsigned total = (unsigned)(samples * samples);
                for (unsigned k = 0; k < total; ++k) {
                    FN(vec) base = FN(mk)(det.x + (REAL)gx * hp.x + (REAL)gy * vp.x,
                                          det.y + (REAL)gx * hp.y + (REAL)gy * vp.y,
                                          det.z + (REAL)gx * hp.z + (REAL)gy * vp.z);
                    unsigned dh = k % (unsigned)samples, dv = k / (unsigned)samples;
                    REAL fh = ((REAL)dh + (REAL)0.5) / (REAL)samples;
                    REAL fv = ((REAL)dv + (REAL)0.5) / (REAL)samples;
                    FN(vec) p = FN(mk)(base.x + fh * hp.x + fv * vp.x,
                                       base.y + fh * hp.y + fv * vp.y,
                                       base.z + fh * hp.z + fv * vp.z);
                    FN(vec) d = FN(mk)(p.x - src.x, p.y - src.y, p.z - src.z);
                    REAL n = SQRT(d.x * d.x + d.y * d.y + d.z * d.z);
                    d = FN(mk)(d.x / n, d.y / n, d.z / n);
                    FN(dda)(src, d, &g, vol, half, mask, &v, &l);
                    acc += v; accl += l;
                }
                size_t i = (size_t)gy * W + gx;
                proj[i] = (float)((REAL)proj[i] + acc / (REAL)total);
                len[i] = (float)((REAL)len[i] + accl / (REAL)total);
            }
        }
    }
}

/*
 * Bilinear sample of a W x H image at unnormalised coordinates (u, v) with
 * texel centres at +0.5 and zero outside (CL_ADDRESS_CLAMP border).
 * weights == ORC_WEIGHTS_EXACT restates the buffer path
 * ocl_src/ImageHandler.hl:20-40 (mix along x, then along y);
 * weights == ORC_WEIGHTS_Q8 / _Q8_TRUNC model GPU texture filtering, whose fractional
 * weights carry 8 bits (1/256 steps), the image path of
 * BackProjectionKernel.cpp:146-163 with CLImageProperties' linear filter.
 */
static inline REAL FN(texel)(const float* img, int W, int H, int x, int y)
{
    return (x >= 0 && x < W && y >= 0 && y < H) ? (REAL)img[(size_t)y * W + x] : (REAL)0;
}

static inline REAL FN(bilinear)(const float* img, int W, int H, REAL u, REAL v, int weights)
{
    REAL xb = FLOOR(u - (REAL)0.5), yb = FLOOR(v - (REAL)0.5);
    REAL a = (u - (REAL)0.5) - xb, b = (v - (REAL)0.5) - yb;
    /* fract() is clamped just below 1 in OpenCL */
    if (a > (REAL)ORC_FRACT_MAX) a = (REAL)ORC_FRACT_MAX;
    if (b > (REAL)ORC_FRACT_MAX) b = (REAL)ORC_FRACT_MAX;
    int x0 = (int)xb, y0 = (int)yb;
    if (weights != ORC_WEIGHTS_EXACT) {
        a = (REAL)orc_q8((double)a);
        b = (REAL)orc_q8((double)b);
        REAL t00 = FN(texel)(img, W, H, x0, y0), t10 = FN(texel)(img, W, H, x0 + 1, y0);
        REAL t01 = FN(texel)(img, W, H, x0, y0 + 1), t11 = FN(texel)(img, W, H, x0 + 1, y0 + 1);
        return ((REAL)1 - a) * ((REAL)1 - b) * t00 + a * ((REAL)1 - b) * t10
             + ((REAL)1 - a) * b * t01 + a * b * t11;
    }
    REAL r0 = 0, r1 = 0;
    if (y0 >= 0 && y0 < H) {
        REAL p = FN(texel)(img, W, H, x0, y0), q = FN(texel)(img, W, H, x0 + 1, y0);
        r0 = p + (q - p) * a;
    }
    if (y0 + 1 >= 0 && y0 + 1 < H) {
        REAL p = FN(texel)(img, W, H, x0, y0 + 1), q = FN(texel)(img, W, H, x0 + 1, y0 + 1);
        r1 = p + (q - p) * a;
    }
    return r0 + (r1 - r0) * b;
}

/* Matrix4x4.hl:54-58 TransformCoordG, column-major m[4*col + row] */
static inline void FN(xform)(const REAL* m, FN(vec) p, REAL* u, REAL* v)
{
    REAL x = m[0] * p.x + m[4] * p.y + m[8] * p.z + m[12];
    REAL y = m[1] * p.x + m[5] * p.y + m[9] * p.z + m[13];
    REAL w = m[3] * p.x + m[7] * p.y + m[11] * p.z + m[15];
    *u = x / w;
    *v = y / w;
}

/*
 * ParallelBeamsBackProjection.cl:9-52 correct(): per voxel of the sub-volume,
 * the nSamples detector-plane offsets (samples4: x, y, z, chord) are projected
 * through the 4x4 matrix, ray length and residual are sampled bilinearly and
 * vol += mask * sum(r * lambda * d / L) / usedSamples over samples with L > eps.
 */
static void FN(back_parallel)(const orc_volgeom* vgin, const double* mat16, const float* samples4, int nsamples,
                              const float* residual, const float* raylen, int W, int H,
                              void* vol, int half, const uint8_t* mask, float lambda, int weights)
{
    FN(vgeo) g; FN(load_vgeo)(vgin, &g);
    REAL m[16];
    for (int i = 0; i < 16; ++i) m[i] = (REAL)mat16[i];
    const REAL lam = (REAL)lambda;
    const int X = g.res[0], Y = g.res[1], Z = g.res[2];
#pragma omp parallel for schedule(static)
    for (int z = 0; z < Z; ++z) {
        for (int y = 0; y < Y; ++y) {
            for (int x = 0; x < X; ++x) {
                FN(vec) c = FN(mk)(g.bmin.x + ((REAL)x + (REAL)0.5) * g.vs.x,
                                   g.bmin.y + ((REAL)y + (REAL)0.5) * g.vs.y,
                                   g.bmin.z + ((REAL)z + (REAL)0.5) * g.vs.z);
                REAL pv = 0; unsigned used = 0;
                for (int k = 0; k < nsamples; ++k) {
                    FN(vec) p = FN(mk)(c.x + (REAL)samples4[4 * k + 0], c.y + (REAL)samples4[4 * k + 1],
                                       c.z + (REAL)samples4[4 * k + 2]);
                    REAL d = (REAL)samples4[4 * k + 3];
                    REAL u, v;
                    FN(xform)(m, p, &u, &v);
                    REAL L = FN(bilinear)(raylen, W, H, u, v, weights);
                    REAL r = FN(bilinear)(residual, W, H, u, v, weights);
                    REAL w = d / L;
                    REAL contrib = r * lam * w;
                    if (L > (REAL)ORC_EPS) { pv += contrib; used += 1; }
                }
                size_t idx = ((size_t)z * Y + y) * X + x;
                REAL val = FN(read_voxel)(vol, half, idx);
                if (used != 0) {
                    REAL mv = mask ? (REAL)((float)mask[idx] / 255.0f) : (REAL)1;
                    val += mv * pv / (REAL)used;
                }
                if (half) ((uint16_t*)vol)[idx] = orc_float_to_half((float)val);
                else ((float*)vol)[idx] = (float)val;
            }
        }
    }
}

/* PerspectiveBeamsBackProjection.cl:10-17 getRayLengthInVoxel */
static inline REAL FN(chord_in_voxel)(FN(vec) o, FN(vec) dir, FN(vec) c, FN(vec) vs)
{
    FN(vec) bmin = FN(mk)(c.x - (REAL)0.5 * vs.x, c.y - (REAL)0.5 * vs.y, c.z - (REAL)0.5 * vs.z);
    FN(vec) bmax = FN(mk)(c.x + (REAL)0.5 * vs.x, c.y + (REAL)0.5 * vs.y, c.z + (REAL)0.5 * vs.z);
    REAL n = SQRT(dir.x * dir.x + dir.y * dir.y + dir.z * dir.z);
    FN(vec) inv = FN(mk)((REAL)1 / (dir.x / n), (REAL)1 / (dir.y / n), (REAL)1 / (dir.z / n));
    REAL tin, tout;
    FN(slab)(bmin, bmax, o, inv, &tin, &tout);
    return FMAX((REAL)0, tout - tin);
}

/*
 * PerspectiveBeamsBackProjection.cl:28-71 correct(): n^3 sub-voxel samples,
 * each weighted by its own chord through the voxel; optional intensity clamp
 * (VOLUME_MINIMUM/MAXIMUM_INTENSITY defines of
 * PerspectiveBeamsBackProjectionKernel.cpp:175-188).
 */
static void FN(back_perspective)(const orc_volgeom* vgin, const double* mat16, const double* source3, int n,
                                 const float* residual, const float* raylen, int W, int H,
                                 void* vol, int half, const uint8_t* mask, float lambda, int weights,
                                 int use_min, float vmin, int use_max, float vmax)
{
    FN(vgeo) g; FN(load_vgeo)(vgin, &g);
    REAL m[16];
    for (int i = 0; i < 16; ++i) m[i] = (REAL)mat16[i];
    FN(vec) src = FN(fromd)(source3);
    const int X = g.res[0], Y = g.res[1], Z = g.res[2];
    const unsigned count = (unsigned)(n * n * n);
#pragma omp parallel for schedule(static)
    for (int z = 0; z < Z; ++z) {
        for (int y = 0; y < Y; ++y) {
            for (int x = 0; x < X; ++x) {
                FN(vec) c = FN(mk)(g.bmin.x + ((REAL)x + (REAL)0.5) * g.vs.x,
                                   g.bmin.y + ((REAL)y + (REAL)0.5) * g.vs.y,
                                   g.bmin.z + ((REAL)z + (REAL)0.5) * g.vs.z);
                REAL value = 0;
                for (unsigned k = 0; k < count; ++k) {
                    unsigned dx = k % (unsigned)n, dy = (k / (unsigned)n) % (unsigned)n, dz = k / (unsigned)(n * n);
                    FN(vec) base = FN(mk)(c.x - (REAL)0.5 * g.vs.x, c.y - (REAL)0.5 * g.vs.y, c.z - (REAL)0.5 * g.vs.z);
                    FN(vec) p = FN(mk)(base.x + g.vs.x * ((REAL)dx + (REAL)0.5) / (REAL)n,
                                       base.y + g.vs.y * ((REAL)dy + (REAL)0.5) / (REAL)n,
                                       base.z + g.vs.z * ((REAL)dz + (REAL)0.5) / (REAL)n);
                    REAL u, v;
                    FN(xform)(m, p, &u, &v);
                    REAL L = FN(bilinear)(raylen, W, H, u, v, weights);
                    if (L >= (REAL)ORC_EPS) {
                        FN(vec) dir = FN(mk)(p.x - src.x, p.y - src.y, p.z - src.z);
                        REAL l = FN(chord_in_voxel)(p, dir, c, g.vs);
                        REAL r = FN(bilinear)(residual, W, H, u, v, weights);
                        value += r * l / L;
                    }
                }
                size_t idx = ((size_t)z * Y + y) * X + x;
                REAL val = FN(read_voxel)(vol, half, idx);
                REAL mv = mask ? (REAL)((float)mask[idx] / 255.0f) : (REAL)1;
                val += (REAL)lambda * value * mv / (REAL)count;
                if (use_min) val = FMAX((REAL)vmin, val);
                if (use_max) val = FMIN((REAL)vmax, val);
                if (half) ((uint16_t*)vol)[idx] = orc_float_to_half((float)val);
                else ((float*)vol)[idx] = (float)val;
            }
        }
    }
}

/* ComputeRayLength.cl:21-34: chord of each pixel-centre ray through the complete bbox */
static void FN(ray_length)(const orc_view* view, const orc_volgeom* vgin, float* out)
{
    FN(vgeo) g; FN(load_vgeo)(vgin, &g);
    FN(vec) src = FN(fromd)(view->source), hp = FN(fromd)(view->hpitch), vp = FN(fromd)(view->vpitch);
    FN(vec) ray = FN(fromd)(view->ray);
    FN(vec) inv = FN(inv_safe)(ray);
    for (int gy = 0; gy < view->height; ++gy) {
        for (int gx = 0; gx < view->width; ++gx) {
            REAL fx = (REAL)gx + (REAL)0.5, fy = (REAL)gy + (REAL)0.5;
            FN(vec) s = FN(mk)(src.x + hp.x * fx + vp.x * fy, src.y + hp.y * fx + vp.y * fy,
                               src.z + hp.z * fx + vp.z * fy);
            REAL tin, tout;
            FN(slab)(g.cmin, g.cmax, s, inv, &tin, &tout);
            out[(size_t)gy * view->width + gx] = (float)FMAX(tout - tin, (REAL)0);
        }
    }
}

#undef FN
#undef CAT
#undef CAT2
