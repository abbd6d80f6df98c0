// Host-side scanner geometry of the block-iterative path, restated for the
// CUDA backend.  Paths are relative to ettention/libReconstruction/src (LR).
// Values are computed the way the reference stores them (float), with matrix
// inverses taken in double and rounded to float.
#pragma once

#include <cmath>
#include <cstdint>
#include <limits>
#include <random>
#include <string>
#include <vector>

#include "ettention_b200.h"

namespace etcu {

struct Vec3 {
    float x, y, z;
};

inline Vec3 v3(const float* p) { return Vec3{p[0], p[1], p[2]}; }
inline Vec3 operator-(Vec3 a, Vec3 b) { return Vec3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Vec3 operator+(Vec3 a, Vec3 b) { return Vec3{a.x + b.x, a.y + b.y, a.z + b.z}; }
inline Vec3 operator*(float s, Vec3 a) { return Vec3{s * a.x, s * a.y, s * a.z}; }

// Vec3f doNormalize (framework/math/Vec3.h): v / |v| in float.
inline Vec3 normalize(Vec3 v) {
    float n = std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
    return Vec3{v.x / n, v.y / n, v.z / n};
}

// ScannerGeometry::getDetectorCenter (LR/model/geometry/ScannerGeometry.cpp:80-83).
inline Vec3 detector_center(const etcu_view& g) {
    Vec3 h = v3(g.hpitch), v = v3(g.vpitch);
    return v3(g.detector) + 0.5f * ((float)g.width * h + (float)g.height * v);
}

// ParallelScannerGeometry::getRayDirection (ParallelScannerGeometry.cpp:44-47),
// PerspectiveScannerGeometry::getRayDirection (PerspectiveScannerGeometry.cpp:37-40).
inline Vec3 ray_direction(const etcu_view& g) {
    if (g.perspective) return normalize(detector_center(g) - v3(g.source));
    return normalize(v3(g.detector) - v3(g.source));
}

// SingleAxisTiltRotator::doRotate (LR/model/geometry/SingleAxisTiltRotator.cpp:62-78).
inline Vec3 tilt_rotate(Vec3 c, float t, float xt) {
    if (xt == 0.0f) {
        return Vec3{c.x * std::cos(t) - c.z * std::sin(t), c.y, c.x * std::sin(t) + c.z * std::cos(t)};
    }
    Vec3 q{c.x, c.y * std::cos(xt) + c.z * std::sin(xt), -c.y * std::sin(xt) + c.z * std::cos(xt)};
    Vec3 a = normalize(Vec3{0.f, std::cos(xt), -std::sin(xt)});
    float ct = std::cos(t), st = std::sin(t), oc = 1.0f - ct;
    return Vec3{(ct + oc * a.x * a.x) * q.x + (oc * a.x * a.y - st * a.z) * q.y + (oc * a.x * a.z + st * a.y) * q.z,
                (oc * a.x * a.y + st * a.z) * q.x + (ct + oc * a.y * a.y) * q.y + (oc * a.y * a.z - st * a.x) * q.z,
                (oc * a.x * a.z - st * a.y) * q.x + (oc * a.y * a.z + st * a.x) * q.y + (ct + oc * a.z * a.z) * q.z};
}

// SingleAxisTiltRotator::createRotatedScannerGeometry (SingleAxisTiltRotator.cpp:42-60).
inline etcu_view rotate_view(const etcu_view& base, float tilt_deg, float xtilt_deg) {
    float t = -tilt_deg / 180.f * (float)M_PI;
    float xt = xtilt_deg / 180.f * (float)M_PI;
    etcu_view o = base;
    auto put = [&](float* dst, const float* src) {
        Vec3 r = tilt_rotate(v3(src), t, xt);
        dst[0] = r.x; dst[1] = r.y; dst[2] = r.z;
    };
    put(o.source, base.source);
    put(o.detector, base.detector);
    put(o.hpitch, base.hpitch);
    put(o.vpitch, base.vpitch);
    return o;
}

// 4x4 helpers, row-major double M[r][c]; output column-major float (Matrix4x4::values).
struct Mat4 {
    double m[4][4];
};

inline Mat4 from_columns(const double c[4][4]) {
    Mat4 r;
    for (int col = 0; col < 4; ++col)
        for (int row = 0; row < 4; ++row) r.m[row][col] = c[col][row];
    return r;
}

inline Mat4 mul(const Mat4& a, const Mat4& b) {
    Mat4 r;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            double s = 0;
            for (int k = 0; k < 4; ++k) s += a.m[i][k] * b.m[k][j];
            r.m[i][j] = s;
        }
    return r;
}

// Gauss-Jordan with partial pivoting; throws the reference's message when singular
// (framework/math/Matrix4x4.cpp:90-97).
inline bool invert(const Mat4& in, Mat4& out) {
    double a[4][8];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            a[i][j] = in.m[i][j];
            a[i][j + 4] = (i == j) ? 1.0 : 0.0;
        }
    for (int c = 0; c < 4; ++c) {
        int p = c;
        for (int r = c + 1; r < 4; ++r)
            if (std::fabs(a[r][c]) > std::fabs(a[p][c])) p = r;
        if (a[p][c] == 0.0) return false;
        if (p != c)
            for (int j = 0; j < 8; ++j) std::swap(a[p][j], a[c][j]);
        double d = a[c][c];
        for (int j = 0; j < 8; ++j) a[c][j] /= d;
        for (int r = 0; r < 4; ++r) {
            if (r == c || a[r][c] == 0.0) continue;
            double f = a[r][c];
            for (int j = 0; j < 8; ++j) a[r][j] -= f * a[c][j];
        }
    }
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) out.m[i][j] = a[i][j + 4];
    return true;
}

inline void to_column_major(const Mat4& m, float out[16]) {
    for (int col = 0; col < 4; ++col)
        for (int row = 0; row < 4; ++row) out[4 * col + row] = (float)m.m[row][col];
}

// ParallelScannerGeometry::getProjectionMatrix (ParallelScannerGeometry.cpp:49-62) and
// Matrix4x4::getPerspectiveProjection (framework/math/Matrix4x4.cpp:376-399).
inline bool projection_matrix(const etcu_view& g, float out[16]) {
    Mat4 base, inv;
    if (!g.perspective) {
        Vec3 r = ray_direction(g);
        double c[4][4] = {{g.hpitch[0], g.hpitch[1], g.hpitch[2], 0.0},
                          {g.vpitch[0], g.vpitch[1], g.vpitch[2], 0.0},
                          {r.x, r.y, r.z, 0.0},
                          {0.0, 0.0, 0.0, 1.0}};
        base = from_columns(c);
        if (!invert(base, inv)) return false;
        double tx = 0.5 * (double)(float)g.width + 0.5, ty = 0.5 * (double)(float)g.height + 0.5;
        double t[4][4] = {{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}, {tx, ty, 0, 1}};
        to_column_major(mul(from_columns(t), inv), out);
        return true;
    }
    Vec3 src = v3(g.source), dc = detector_center(g);
    Vec3 d = dc - src;
    double c[4][4] = {{g.hpitch[0], g.hpitch[1], g.hpitch[2], 0.0},
                      {g.vpitch[0], g.vpitch[1], g.vpitch[2], 0.0},
                      {d.x, d.y, d.z, 0.0},
                      {src.x, src.y, src.z, 1.0}};
    base = from_columns(c);
    if (!invert(base, inv)) return false;
    const double zn = 1e-2;
    double p[4][4] = {{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1.0 / (1.0 - zn), 1.0}, {0, 0, -zn / (1.0 - zn), 0}};
    double t[4][4] = {{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}, {0.5 * g.width, 0.5 * g.height, 0, 1}};
    to_column_major(mul(mul(from_columns(t), from_columns(p)), inv), out);
    return true;
}

// ParallelBeamsBackProjectionKernel::setSamples + generateSamplingPatternForPerVoxelSampling
// (LR/algorithm/projections/back/parallel/ParallelBeamsBackProjectionKernel.cpp:55-98).
inline bool sample_pattern(const etcu_view& g, const float vs[3], unsigned samples, float* out4, std::string* err) {
    if (samples == 0) {
        if (err) *err = "zero samples not supported for BackProjection";
        return false;
    }
    unsigned n = (unsigned)std::sqrt((float)samples);
    if (n * n != samples) {
        if (err) *err = "non-square root number of samples not supported for BackProjection";
        return false;
    }
    float mvs = std::fmax(std::fmax(vs[0], vs[1]), vs[2]);
    Vec3 h = mvs * normalize(v3(g.hpitch)), v = mvs * normalize(v3(g.vpitch));
    Vec3 r = normalize(ray_direction(g));
    float inv[3] = {r.x != 0.f ? 1.0f / r.x : std::numeric_limits<float>::max(),
                    r.y != 0.f ? 1.0f / r.y : std::numeric_limits<float>::max(),
                    r.z != 0.f ? 1.0f / r.z : std::numeric_limits<float>::max()};
    unsigned k = 0;
    for (unsigned yi = 0; yi < n; ++yi) {
        float yp = (((float)yi + 0.5f) / (float)n) - 0.5f;
        for (unsigned xi = 0; xi < n; ++xi) {
            float xp = (((float)xi + 0.5f) / (float)n) - 0.5f;
            Vec3 p = (xp * h) + (yp * v);
            float pp[3] = {p.x, p.y, p.z};
            float tmin = -std::numeric_limits<float>::infinity(), tmax = std::numeric_limits<float>::infinity();
            for (int a = 0; a < 3; ++a) {
                float t0 = (-0.5f * vs[a] - pp[a]) * inv[a];
                float t1 = (0.5f * vs[a] - pp[a]) * inv[a];
                float lo = std::min(t0, t1), hi = std::max(t0, t1);
                tmin = (a == 0) ? lo : std::fmax(tmin, lo);
                tmax = (a == 0) ? hi : std::fmin(tmax, hi);
            }
            out4[4 * k + 0] = p.x;
            out4[4 * k + 1] = p.y;
            out4[4 * k + 2] = p.z;
            out4[4 * k + 3] = tmax - tmin;
            ++k;
        }
    }
    return true;
}

// ParallelScannerGeometry::getTraversalLengthThroughBoundingBox (ParallelScannerGeometry.cpp:64-69).
inline float traversal_length(const etcu_view& g, const float bmin[3], const float bmax[3]) {
    Vec3 r = ray_direction(g);
    float zin = (bmin[2] - g.source[2]) / r.z;
    float zout = (bmax[2] - g.source[2]) / r.z;
    return std::max(zin, zout) - std::min(zin, zout);
}

// PerspectiveBeamsBackProjectionKernel::computeSamplingFactor
// (LR/algorithm/projections/back/perspective/PerspectiveBeamsBackProjectionKernel.cpp:72-81).
inline unsigned perspective_sampling_factor(unsigned w, unsigned h, const uint32_t res[3], unsigned spv) {
    if (spv != 0) return spv;
    unsigned mp = std::max(w, h), mv = std::max(std::max(res[0], res[1]), res[2]);
    return std::max(1u, mp / mv);
}

// Projection orderings (LR/model/projectionset/ProjectionSet.cpp:14-25 and the
// Identity / Random / MaxAngle / Buckets reorder() implementations).
inline uint32_t boost_uniform_int(std::mt19937& eng, uint32_t lo, uint32_t hi) {
    // boost::uniform_int<> on a 32-bit engine: bucketed rejection sampling.
    const uint32_t range = hi - lo;
    if (range == 0) return lo;
    const uint32_t brange = 0xffffffffu;
    uint32_t bucket = brange / (range + 1);
    if (brange % (range + 1) == range) ++bucket;
    for (;;) {
        uint32_t r = (uint32_t)eng() / bucket;
        if (r <= range) return r + lo;
    }
}

inline std::vector<uint32_t> projection_order(etcu_order order, uint32_t n, const uint32_t* skip, uint32_t nskip) {
    std::vector<uint32_t> idx;
    for (uint32_t i = 0; i < n; ++i) {
        bool skipped = false;
        for (uint32_t k = 0; k < nskip; ++k) skipped |= (skip[k] == i);
        if (!skipped) idx.push_back(i);
    }
    const size_t m = idx.size();
    std::vector<uint32_t> out(m);
    switch (order) {
    case ETCU_ORDER_IDENTITY:
        return idx;
    case ETCU_ORDER_MAXANGLE: {  // ProjectionSetMaxAngle.cpp:16-38
        size_t j = m / 2, k = 0;
        for (size_t i = 0; i < m; ++i) out[i] = (i % 2 == 0) ? idx[j++] : idx[k++];
        return out;
    }
    case ETCU_ORDER_BUCKETS: {  // ProjectionSetBuckets.cpp:16-42
        size_t cur[4];
        for (int i = 0; i < 4; ++i) cur[i] = (size_t)i * m / 4;
        for (size_t i = 0; i < m; ++i) out[i] = idx[cur[i % 4]++];
        return out;
    }
    case ETCU_ORDER_RANDOM: {  // ProjectionSetRandom.cpp:17-38: mt19937(default seed) + random_shuffle
        std::mt19937 eng;  // default seed 5489, same sequence as boost::mt19937
        for (size_t i = 0; i < m; ++i) out[i] = (uint32_t)i;  // the reference resets to 0..m-1
        for (size_t i = 1; i < m; ++i) {
            size_t j = boost_uniform_int(eng, 0, (uint32_t)i);
            if (i != j) std::swap(out[i], out[j]);
        }
        return out;
    }
    }
    return idx;
}

}  // namespace etcu
