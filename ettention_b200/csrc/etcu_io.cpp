// Host-side file formats of the reconstruction path (no device code): MRC tilt
// series in, MRC volumes out, tilt-angle files.
//
// Behaviour follows (paths relative to ettention/libReconstruction/src):
//   io/datasource/MRCStack.cpp:136-250      modes 0/1/2/6, data range, log transform,
//                                            1024-byte header + extended header
//   io/datasource/ImageStackDatasource.cpp:49-79  tilt angles, one float per token
//   io/serializer/VolumeFileFormatWriter.cpp, MRCWriter.cpp,
//   setup/parameterset/IOEnumerations.cpp:39-126  volume in XYZ / XZY order, voxel types
//   io/rangetransformation/LinearRangeTransformation.cpp, VolumeStatistics.cpp
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <string>
#include <vector>

#include "ettention_b200.h"

// Records the message of a failed context-free call for etcu_last_error(NULL)
// (defined with the context code in etcu_api.cu).
void etcu_set_context_free_error(const char* message);

namespace {

etcu_status io_fail(etcu_status st, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    etcu_set_context_free_error(buf);
    return st;
}

// The 1024-byte MRC header: the fields this path reads or writes, at their offsets.
struct MrcHeader {
    int32_t nx, ny, nz, mode;        // 0, 4, 8, 12
    int32_t nxstart, nystart, nzstart;
    int32_t mx, my, mz;              // 28
    float cella[3];                  // 40
    float cellb[3];                  // 52
    int32_t mapc, mapr, maps;        // 64
    float dmin, dmax, dmean;         // 76
    int16_t ispg, nsymbt;            // 88
    int32_t extra;                   // 92: bytes of extended header
    uint8_t rest[1024 - 96];
};
static_assert(sizeof(MrcHeader) == 1024, "MRC header is 1024 bytes");

size_t mode_bytes(int mode) {
    switch (mode) {
    case 0: return 1;
    case 1: return 2;
    case 2: return 4;
    case 6: return 2;
    default: return 0;
    }
}

float raw_value(const uint8_t* p, int mode) {
    switch (mode) {
    case 0: return (float)*p;
    case 1: { int16_t v; std::memcpy(&v, p, 2); return (float)v; }
    case 2: { float v; std::memcpy(&v, p, 4); return v; }
    default: { uint16_t v; std::memcpy(&v, p, 2); return (float)v; }
    }
}

bool read_header(const char* path, MrcHeader& h, std::ifstream& f) {
    f.open(path, std::ios::binary);
    if (!f.good()) return false;
    f.read((char*)&h, sizeof(h));
    return f.good();
}

}  // namespace

extern "C" etcu_status etcu_mrc_read_info(const char* path, etcu_mrc_info* out) {
    if (!path || !out) return io_fail(ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    MrcHeader h;
    std::ifstream f;
    if (!read_header(path, h, f)) return io_fail(ETCU_ERR_INVALID_ARGUMENT, "Could not open MRC stack %s", path);
    if (h.nx <= 0 || h.ny <= 0 || h.nz <= 0 || h.extra < 0)
        return io_fail(ETCU_ERR_INVALID_ARGUMENT, "%s: invalid MRC header", path);
    out->nx = (uint32_t)h.nx;
    out->ny = (uint32_t)h.ny;
    out->nz = (uint32_t)h.nz;
    out->mode = h.mode;
    out->dmin = h.dmin;
    out->dmax = h.dmax;
    out->dmean = h.dmean;
    out->extended_bytes = (uint32_t)h.extra;
    return ETCU_OK;
}

// MRCStack::init + readImageData for every section: the data range of the whole
// stack, then each value as float, or log(M / (raw - m)) with
// M = max - min + 1, m = min - 1 (modes 1, 2) and M = max + 1, m = -1 (modes 0, 6).
extern "C" etcu_status etcu_mrc_read_stack(const char* path, int logarithmize, float* out, size_t capacity) {
    if (!path || !out) return io_fail(ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    MrcHeader h;
    std::ifstream f;
    if (!read_header(path, h, f)) return io_fail(ETCU_ERR_INVALID_ARGUMENT, "Could not open MRC stack %s", path);
    const size_t bpv = mode_bytes(h.mode);
    if (bpv == 0)
        return io_fail(ETCU_ERR_UNSUPPORTED, "Format of the MRC stack is either unknown or not supported (mode %d)",
                       h.mode);
    if (h.nx <= 0 || h.ny <= 0 || h.nz <= 0 || h.extra < 0)
        return io_fail(ETCU_ERR_INVALID_ARGUMENT, "%s: invalid MRC header", path);
    const size_t n = (size_t)h.nx * (size_t)h.ny * (size_t)h.nz;
    if (capacity < n) return io_fail(ETCU_ERR_INVALID_ARGUMENT, "output holds %zu of %zu values", capacity, n);
    f.seekg((std::streamoff)sizeof(MrcHeader) + h.extra);
    std::vector<uint8_t> raw(n * bpv);
    f.read((char*)raw.data(), (std::streamsize)raw.size());
    if (!f.good()) return io_fail(ETCU_ERR_INVALID_ARGUMENT, "Error reading %zu voxel value(s) from %s!", n, path);
    float dmax = -std::numeric_limits<float>::infinity(), dmin = std::numeric_limits<float>::infinity();
    for (size_t i = 0; i < n; ++i) {
        const float v = raw_value(raw.data() + i * bpv, h.mode);
        dmax = std::max(v, dmax);
        dmin = std::min(v, dmin);
    }
    float M = dmax, m = -1.f;
    if (h.mode == 1 || h.mode == 2) {
        M = dmax - dmin + 1.f;
        m = dmin - 1.f;
    } else {
        M = dmax + 1.f;
    }
    for (size_t i = 0; i < n; ++i) {
        const float v = raw_value(raw.data() + i * bpv, h.mode);
        out[i] = logarithmize ? logf(M / (v - m)) : v;
    }
    return ETCU_OK;
}

// ImageStackDatasource::readTiltAngles: every whitespace-separated float of the file.
extern "C" etcu_status etcu_read_tilt_angles(const char* path, float* out, uint32_t capacity, uint32_t* count) {
    if (!path || !count) return io_fail(ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    FILE* fp = std::fopen(path, "rt");
    if (!fp) return io_fail(ETCU_ERR_INVALID_ARGUMENT, "Could not open file: %s", path);
    uint32_t k = 0;
    float a;
    while (std::fscanf(fp, "%f", &a) == 1) {
        if (out && k < capacity) out[k] = a;
        ++k;
    }
    std::fclose(fp);
    *count = k;
    return ETCU_OK;
}

namespace {

// VolumeStatistics::compute (algorithm/volumestatistics/VolumeStatistics.cpp:17-48): min
// from FLT_MAX, max from FLT_MIN (the smallest positive normal, as the reference starts
// it), NaN voxels skipped, the mean a float sum in voxel order times 1 / (float)count of
// all voxels.
struct VolumeStats {
    float min, max, mean;
};
VolumeStats volume_statistics(const float* v, size_t n) {
    float mn = std::numeric_limits<float>::max(), mx = std::numeric_limits<float>::min(), sum = 0.f;
    for (size_t i = 0; i < n; ++i) {
        const float x = v[i];
        if (!std::isnan(x)) {
            if (x < mn) mn = x;
            if (x > mx) mx = x;
            sum += x;
        }
    }
    const float scale = 1.f / (float)n;
    return {mn, mx, sum * scale};
}

// LinearRangeTransformation::transformRange (io/rangetransformation/
// LinearRangeTransformation.cpp:14-21), float by float.
struct LinearRange {
    float smin, smax, out_min, out_max;
    float operator()(float value) const {
        const float zero_to_max = value - smin;
        const float zero_to_one = zero_to_max / (smax - smin);
        const float zero_to_new_max = zero_to_one * (out_max - out_min);
        return zero_to_new_max + out_min;
    }
};

// VolumeFileFormatWriter::writeValue: a C cast of the transformed float.  A value the
// target type cannot hold (NaN when max == min) is written as 0.
template <typename T>
T cast_value(float v) {
    if (!(v > (float)std::numeric_limits<T>::min() - 1.f && v < (float)std::numeric_limits<T>::max() + 1.f)) return 0;
    return (T)v;
}

}  // namespace

// VolumeFileFormatWriter::write + MRCWriter::writeHeader: the volume (x fastest, then y,
// then z) written in the given coordinate order; header mode = the voxel type, the
// resolution in that order and the (transformed) min / max / mean.  createRangeTransformation
// (VolumeFileFormatWriter.cpp:107-140): unsigned8 / unsigned16 / signed16 map [min, max]
// linearly onto [0, 255] / [0, 65535] / [-32768, 32767] (inverted: the range reversed);
// float32 is written as is, and with invert only the header's statistics are mapped onto
// [max, min] (the reference writes float data slice by slice from the untransformed volume).
extern "C" etcu_status etcu_mrc_write_volume_typed(const char* path, const float* volume, const uint32_t resolution[3],
                                                   etcu_orientation orientation, etcu_output_voxel_type voxel_type,
                                                   int invert) {
    if (!path || !volume || !resolution) return io_fail(ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    const uint32_t X = resolution[0], Y = resolution[1], Z = resolution[2];
    if (X == 0 || Y == 0 || Z == 0) return io_fail(ETCU_ERR_INVALID_ARGUMENT, "empty volume");
    if (orientation != ETCU_AXES_XYZ && orientation != ETCU_AXES_XZY)
        return io_fail(ETCU_ERR_UNSUPPORTED, "orientation %d is not supported", (int)orientation);
    float out_lo = 0.f, out_hi = 0.f;
    switch (voxel_type) {
    case ETCU_OUT_UNSIGNED_8: out_lo = 0.f; out_hi = 255.f; break;
    case ETCU_OUT_SIGNED_16: out_lo = -32768.f; out_hi = 32767.f; break;
    case ETCU_OUT_UNSIGNED_16: out_lo = 0.f; out_hi = 65535.f; break;
    case ETCU_OUT_FLOAT_32: break;
    default: return io_fail(ETCU_ERR_INVALID_ARGUMENT, "ParseVoxelValueType: Unknown file mode ");
    }
    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    if (!f.good()) return io_fail(ETCU_ERR_INVALID_ARGUMENT, "Failed to open output file %s for writing!", path);
    const size_t n = (size_t)X * Y * Z;
    const VolumeStats st = volume_statistics(volume, n);
    const bool identity = voxel_type == ETCU_OUT_FLOAT_32 && !invert;
    LinearRange tr{st.min, st.max, invert ? out_hi : out_lo, invert ? out_lo : out_hi};
    if (voxel_type == ETCU_OUT_FLOAT_32) tr = LinearRange{st.min, st.max, st.max, st.min};  // inverted float32
    MrcHeader h;
    std::memset(&h, 0, sizeof(h));
    // file sections / rows / columns: XYZ -> z / y / x, XZY -> y / z / x
    const uint32_t fx = X, fy = orientation == ETCU_AXES_XZY ? Z : Y, fz = orientation == ETCU_AXES_XZY ? Y : Z;
    h.nx = h.mx = (int32_t)fx;
    h.ny = h.my = (int32_t)fy;
    h.nz = h.mz = (int32_t)fz;
    h.mode = (int32_t)voxel_type;
    h.cella[0] = (float)fx;
    h.cella[1] = (float)fy;
    h.cella[2] = (float)fz;
    h.mapc = 1;
    h.mapr = 2;
    h.maps = 3;
    h.dmin = identity ? st.min : tr(st.min);
    h.dmax = identity ? st.max : tr(st.max);
    h.dmean = identity ? st.mean : tr(st.mean);
    std::memcpy(h.rest + (208 - 96), "MAP ", 4);  // map identifier at byte 208
    f.write((const char*)&h, sizeof(h));
    // one file row (x) at a time: volume row (y, z)
    const size_t bpv = mode_bytes((int)voxel_type);
    std::vector<uint8_t> row((size_t)X * bpv);
    auto write_row = [&](const float* src) {
        if (voxel_type == ETCU_OUT_FLOAT_32) {
            f.write((const char*)src, (std::streamsize)(X * sizeof(float)));
            return;
        }
        for (uint32_t x = 0; x < X; ++x) {
            const float t = tr(src[x]);
            if (voxel_type == ETCU_OUT_UNSIGNED_8) {
                row[x] = cast_value<uint8_t>(t);
            } else if (voxel_type == ETCU_OUT_SIGNED_16) {
                const int16_t v = cast_value<int16_t>(t);
                std::memcpy(row.data() + 2 * x, &v, 2);
            } else {
                const uint16_t v = cast_value<uint16_t>(t);
                std::memcpy(row.data() + 2 * x, &v, 2);
            }
        }
        f.write((const char*)row.data(), (std::streamsize)row.size());
    };
    if (orientation == ETCU_AXES_XYZ) {
        for (size_t r = 0; r < (size_t)Y * Z; ++r) write_row(volume + r * X);
    } else {
        for (uint32_t y = 0; y < Y; ++y)
            for (uint32_t z = 0; z < Z; ++z) write_row(volume + ((size_t)z * Y + y) * X);
    }
    if (!f.good()) return io_fail(ETCU_ERR_INVALID_ARGUMENT, "Error encountered while writing to output file %s !", path);
    return ETCU_OK;
}

// VolumeFileFormatWriter::write + MRCWriter::writeHeader for float32 output.
extern "C" etcu_status etcu_mrc_write_volume(const char* path, const float* volume, const uint32_t resolution[3],
                                             etcu_orientation orientation) {
    return etcu_mrc_write_volume_typed(path, volume, resolution, orientation, ETCU_OUT_FLOAT_32, 0);
}
