// TIFF images in and out, host side (no device code).
//
// The reference reads projection images through FreeImage
// (ettention/libReconstruction/src/io/deserializer/ImageDeserializer.cpp:10-62):
// the page is converted to float (8-bit grey / 255, 16-bit grey / 65535, 32-bit
// float as is), and image row y is the y-th row of the file (FreeImage keeps rows
// bottom-up and the reference flips them back, :57-59).  Multi-page files are image
// stacks (:21-51).  Images are written as 32-bit float grey TIFFs
// (io/serializer/ImageSerializer.cpp:36-60, TIFF_GRAY_32), top row first.
//
// This file restates the TIFF 6.0 baseline from the published specification:
// little- and big-endian files, strips and tiles, compression none / LZW (with
// the specification's early code-width change) / Deflate (zlib) / PackBits,
// horizontal-difference predictor (2) and the floating-point predictor (3, bytes
// of a row stored as planes, most significant plane first).  Grey images with one
// sample per pixel only; other layouts are reported as unsupported.
#include <zlib.h>

#include <algorithm>
#include <cstring>
#include <set>

#include "io_util.hpp"

using etcu_io::fail;

namespace {

enum : uint16_t {
    kWidth = 256, kLength = 257, kBits = 258, kCompression = 259, kPhotometric = 262, kFillOrder = 266,
    kStripOffsets = 273, kSamples = 277, kRowsPerStrip = 278, kStripByteCounts = 279, kPlanar = 284,
    kPredictor = 317, kTileWidth = 322, kTileLength = 323, kTileOffsets = 324, kTileByteCounts = 325,
    kSampleFormat = 339,
};

struct Bytes {
    const uint8_t* p;
    size_t n;
    bool big;
    bool u16(size_t off, uint32_t& v) const {
        if (off + 2 > n) return false;
        v = big ? (uint32_t(p[off]) << 8 | p[off + 1]) : (uint32_t(p[off + 1]) << 8 | p[off]);
        return true;
    }
    bool u32(size_t off, uint32_t& v) const {
        if (off + 4 > n) return false;
        v = big ? (uint32_t(p[off]) << 24 | uint32_t(p[off + 1]) << 16 | uint32_t(p[off + 2]) << 8 | p[off + 3])
                : (uint32_t(p[off + 3]) << 24 | uint32_t(p[off + 2]) << 16 | uint32_t(p[off + 1]) << 8 | p[off]);
        return true;
    }
};

struct Page {
    uint32_t width = 0, height = 0, bits = 1, samples = 1, format = 1, compression = 1, predictor = 1;
    uint32_t photometric = 1, planar = 1, fill_order = 1, rows_per_strip = 0xFFFFFFFFu, tile_w = 0, tile_h = 0;
    bool tiled = false;
    std::vector<uint64_t> offsets, counts;
};

// Integer values of one IFD entry (BYTE, SHORT, LONG); false for other types.
bool entry_values(const Bytes& b, size_t entry, uint32_t type, uint32_t count, std::vector<uint64_t>& out) {
    size_t size;
    switch (type) {
    case 1: size = 1; break;
    case 3: size = 2; break;
    case 4: size = 4; break;
    default: return false;
    }
    if (count > (1u << 28)) return false;
    size_t at = entry + 8;
    if (size * count > 4) {
        uint32_t off;
        if (!b.u32(entry + 8, off)) return false;
        at = off;
    }
    if (at + size * count > b.n) return false;
    out.resize(count);
    for (uint32_t i = 0; i < count; ++i) {
        uint32_t v = 0;
        if (size == 1) v = b.p[at + i];
        else if (size == 2) b.u16(at + 2 * i, v);
        else b.u32(at + 4 * i, v);
        out[i] = v;
    }
    return true;
}

etcu_status parse_pages(const std::vector<uint8_t>& file, const char* path, std::vector<Page>& pages) {
    if (file.size() < 8) return fail(ETCU_ERR_INVALID_ARGUMENT, "unable to load image %s: not a TIFF file", path);
    Bytes b{file.data(), file.size(), false};
    if (file[0] == 'I' && file[1] == 'I') b.big = false;
    else if (file[0] == 'M' && file[1] == 'M') b.big = true;
    else return fail(ETCU_ERR_INVALID_ARGUMENT, "unable to load image %s: not a TIFF file", path);
    uint32_t magic, ifd;
    b.u16(2, magic);
    if (magic == 43) return fail(ETCU_ERR_UNSUPPORTED, "unable to load image %s: BigTIFF is not supported", path);
    if (magic != 42) return fail(ETCU_ERR_INVALID_ARGUMENT, "unable to load image %s: not a TIFF file", path);
    b.u32(4, ifd);
    std::set<uint32_t> seen;
    while (ifd != 0) {
        if (!seen.insert(ifd).second || seen.size() > (1u << 20))
            return fail(ETCU_ERR_INVALID_ARGUMENT, "unable to load image %s: directory chain loops", path);
        uint32_t nent;
        if (!b.u16(ifd, nent)) return fail(ETCU_ERR_INVALID_ARGUMENT, "unable to load image %s: truncated", path);
        Page pg;
        bool have_length = false, have_width = false;
        for (uint32_t e = 0; e < nent; ++e) {
            const size_t ent = size_t(ifd) + 2 + 12 * size_t(e);
            uint32_t tag, type, count;
            if (!b.u16(ent, tag) || !b.u16(ent + 2, type) || !b.u32(ent + 4, count))
                return fail(ETCU_ERR_INVALID_ARGUMENT, "unable to load image %s: truncated directory", path);
            std::vector<uint64_t> v;
            if (!entry_values(b, ent, type, count, v) || v.empty()) continue;
            switch (tag) {
            case kWidth: pg.width = uint32_t(v[0]); have_width = true; break;
            case kLength: pg.height = uint32_t(v[0]); have_length = true; break;
            case kBits:
                pg.bits = uint32_t(v[0]);
                for (uint64_t x : v)
                    if (x != v[0]) pg.bits = 0;  // mixed sample sizes: unsupported
                break;
            case kCompression: pg.compression = uint32_t(v[0]); break;
            case kPhotometric: pg.photometric = uint32_t(v[0]); break;
            case kFillOrder: pg.fill_order = uint32_t(v[0]); break;
            case kStripOffsets: pg.offsets = v; break;
            case kTileOffsets: pg.offsets = v; pg.tiled = true; break;
            case kSamples: pg.samples = uint32_t(v[0]); break;
            case kRowsPerStrip: pg.rows_per_strip = uint32_t(v[0]); break;
            case kStripByteCounts: case kTileByteCounts: pg.counts = v; break;
            case kPlanar: pg.planar = uint32_t(v[0]); break;
            case kPredictor: pg.predictor = uint32_t(v[0]); break;
            case kTileWidth: pg.tile_w = uint32_t(v[0]); break;
            case kTileLength: pg.tile_h = uint32_t(v[0]); break;
            case kSampleFormat: pg.format = uint32_t(v[0]); break;
            default: break;
            }
        }
        if (!have_width || !have_length || pg.width == 0 || pg.height == 0)
            return fail(ETCU_ERR_INVALID_ARGUMENT, "unable to load image %s: page %zu has no size", path, pages.size());
        pages.push_back(std::move(pg));
        if (!b.u32(size_t(ifd) + 2 + 12 * size_t(nent), ifd)) ifd = 0;
    }
    if (pages.empty()) return fail(ETCU_ERR_INVALID_ARGUMENT, "unable to load image %s: no pages", path);
    return ETCU_OK;
}

// LZW as in TIFF 6.0 section 13: codes most significant bit first, 256 = Clear,
// 257 = end of information, code width 9..12 bits, widened one code early (when
// the next free code reaches 2^width - 1).  Returns false on an invalid code.
bool lzw_decode(const uint8_t* in, size_t n, uint8_t* out, size_t cap, size_t& produced) {
    std::vector<uint16_t> prefix(4096), length(4096);
    std::vector<uint8_t> suffix(4096), first(4096);
    for (int i = 0; i < 256; ++i) {
        length[i] = 1;
        suffix[i] = first[i] = uint8_t(i);
    }
    size_t bit = 0, o = 0;
    const size_t nbits = n * 8;
    auto read = [&](int w) -> int {
        if (bit + size_t(w) > nbits) return 257;
        int v = 0;
        for (int k = 0; k < w; ++k, ++bit) v = (v << 1) | ((in[bit >> 3] >> (7 - (bit & 7))) & 1);
        return v;
    };
    auto emit = [&](int code) {  // the string of `code`, written back to front
        const size_t len = length[code];
        size_t at = o + len;
        for (int c = code; at > o; c = prefix[c]) {
            --at;
            if (at < cap) out[at] = suffix[c];
        }
        o += len;
    };
    int width = 9, next = 258, prev = -1;
    for (;;) {
        const int code = read(width);
        if (code == 257) break;
        if (code == 256) {
            width = 9;
            next = 258;
            prev = -1;
            continue;
        }
        if (prev < 0) {
            if (code > 255) return false;
            emit(code);
            prev = code;
        } else {
            uint8_t k;
            if (code < next) {
                emit(code);
                k = first[code];
            } else if (code == next) {
                emit(prev);
                if (o < cap) out[o] = first[prev];
                ++o;
                k = first[prev];
            } else {
                return false;
            }
            if (next < 4096) {
                prefix[next] = uint16_t(prev);
                suffix[next] = k;
                first[next] = first[prev];
                length[next] = uint16_t(length[prev] + 1);
                ++next;
            }
            prev = code;
        }
        if (next >= (1 << width) - 1 && width < 12) ++width;
        if (o >= cap) break;
    }
    produced = std::min(o, cap);
    return true;
}

bool inflate_decode(const uint8_t* in, size_t n, uint8_t* out, size_t cap, size_t& produced) {
    z_stream s;
    std::memset(&s, 0, sizeof(s));
    if (inflateInit(&s) != Z_OK) return false;
    s.next_in = const_cast<Bytef*>(in);
    s.avail_in = uInt(n);
    s.next_out = out;
    s.avail_out = uInt(cap);
    const int r = inflate(&s, Z_FINISH);
    produced = cap - s.avail_out;
    inflateEnd(&s);
    return r == Z_STREAM_END || ((r == Z_BUF_ERROR || r == Z_OK) && s.avail_out == 0);
}

bool packbits_decode(const uint8_t* in, size_t n, uint8_t* out, size_t cap, size_t& produced) {
    size_t i = 0, o = 0;
    while (i < n && o < cap) {
        const int h = int(int8_t(in[i++]));
        if (h >= 0) {
            for (int k = 0; k <= h && i < n && o < cap; ++k) out[o++] = in[i++];
        } else if (h != -128) {
            if (i >= n) break;
            const uint8_t v = in[i++];
            for (int k = 0; k <= -h && o < cap; ++k) out[o++] = v;
        }
    }
    produced = o;
    return true;
}

// One row of `w` samples of `bytes` bytes each: file byte order -> host order, the
// predictor undone, converted to float.
void row_to_float(uint8_t* row, uint32_t w, const Page& pg, bool big, float* dst) {
    const uint32_t bytes = pg.bits / 8;
    if (pg.predictor == 3) {  // byte planes, most significant first, then differenced bytes
        const size_t nb = size_t(w) * bytes;
        for (size_t i = 1; i < nb; ++i) row[i] = uint8_t(row[i] + row[i - 1]);
        std::vector<uint8_t> tmp(row, row + nb);
        for (uint32_t x = 0; x < w; ++x)
            for (uint32_t k = 0; k < bytes; ++k) row[size_t(x) * bytes + k] = tmp[size_t(bytes - 1 - k) * w + x];
        big = false;  // now host (little-endian) order
    }
    if (big && bytes > 1)
        for (uint32_t x = 0; x < w; ++x) std::reverse(row + size_t(x) * bytes, row + size_t(x + 1) * bytes);
    if (pg.predictor == 2) {
        if (bytes == 1) {
            for (uint32_t x = 1; x < w; ++x) row[x] = uint8_t(row[x] + row[x - 1]);
        } else if (bytes == 2) {
            uint16_t p, c;
            std::memcpy(&p, row, 2);
            for (uint32_t x = 1; x < w; ++x) {
                std::memcpy(&c, row + 2 * x, 2);
                p = uint16_t(p + c);
                std::memcpy(row + 2 * x, &p, 2);
            }
        } else {
            uint32_t p, c;
            std::memcpy(&p, row, 4);
            for (uint32_t x = 1; x < w; ++x) {
                std::memcpy(&c, row + 4 * x, 4);
                p += c;
                std::memcpy(row + 4 * x, &p, 4);
            }
        }
    }
    for (uint32_t x = 0; x < w; ++x) {
        if (bytes == 1) {
            dst[x] = float(row[x]) / 255.0f;
        } else if (bytes == 2) {
            uint16_t v;
            std::memcpy(&v, row + 2 * x, 2);
            dst[x] = float(v) / 65535.0f;
        } else {
            std::memcpy(dst + x, row + 4 * x, 4);
        }
    }
}

etcu_status check_supported(const Page& pg, const char* path) {
    if (pg.samples != 1 || pg.photometric != 1)  // BlackIsZero grey
        return fail(ETCU_ERR_UNSUPPORTED,
                    "unable to load image %s: only grey images with one sample per pixel are supported", path);
    const bool ok_type = (pg.format == 1 && (pg.bits == 8 || pg.bits == 16)) || (pg.format == 3 && pg.bits == 32);
    if (!ok_type)
        return fail(ETCU_ERR_UNSUPPORTED,
                    "unable to load image %s: %u-bit samples of format %u cannot be converted to float", path,
                    pg.bits, pg.format);
    if (pg.compression != 1 && pg.compression != 5 && pg.compression != 8 && pg.compression != 32946 &&
        pg.compression != 32773)
        return fail(ETCU_ERR_UNSUPPORTED, "unable to load image %s: compression %u is not supported", path,
                    pg.compression);
    if (pg.predictor != 1 && pg.predictor != 2 && pg.predictor != 3)
        return fail(ETCU_ERR_UNSUPPORTED, "unable to load image %s: predictor %u is not supported", path,
                    pg.predictor);
    if (pg.predictor == 3 && pg.format != 3)
        return fail(ETCU_ERR_UNSUPPORTED, "unable to load image %s: floating-point predictor on integers", path);
    if (pg.fill_order != 1)
        return fail(ETCU_ERR_UNSUPPORTED, "unable to load image %s: fill order %u is not supported", path,
                    pg.fill_order);
    if (pg.tiled && (pg.tile_w == 0 || pg.tile_h == 0))
        return fail(ETCU_ERR_INVALID_ARGUMENT, "unable to load image %s: tiles without a tile size", path);
    return ETCU_OK;
}

// One strip or tile: `rows` rows of `w` samples.
etcu_status decode_block(const std::vector<uint8_t>& file, const Page& pg, size_t idx, uint32_t w, uint32_t rows,
                         std::vector<uint8_t>& buf, const char* path) {
    const size_t want = size_t(w) * (pg.bits / 8) * rows;
    buf.assign(want, 0);
    if (idx >= pg.offsets.size() || idx >= pg.counts.size())
        return fail(ETCU_ERR_INVALID_ARGUMENT, "unable to load image %s: missing strip or tile %zu", path, idx);
    const uint64_t off = pg.offsets[idx], cnt = pg.counts[idx];
    if (off > file.size() || cnt > file.size() - off)
        return fail(ETCU_ERR_INVALID_ARGUMENT, "unable to load image %s: strip or tile %zu lies outside the file",
                    path, idx);
    const uint8_t* src = file.data() + off;
    size_t got = 0;
    bool ok = true;
    switch (pg.compression) {
    case 1:
        got = std::min<size_t>(cnt, want);
        std::memcpy(buf.data(), src, got);
        break;
    case 5: ok = lzw_decode(src, cnt, buf.data(), want, got); break;
    case 8: case 32946: ok = inflate_decode(src, cnt, buf.data(), want, got); break;
    default: ok = packbits_decode(src, cnt, buf.data(), want, got); break;
    }
    if (!ok) return fail(ETCU_ERR_INVALID_ARGUMENT, "unable to load image %s: corrupt data in block %zu", path, idx);
    if (got < want)
        return fail(ETCU_ERR_INVALID_ARGUMENT, "unable to load image %s: block %zu holds %zu of %zu bytes", path, idx,
                    got, want);
    return ETCU_OK;
}

}  // namespace

namespace etcu_io {

etcu_status tiff_page_count(const std::vector<uint8_t>& file, const char* path, uint32_t* count) {
    std::vector<Page> pages;
    const etcu_status st = parse_pages(file, path, pages);
    if (st != ETCU_OK) return st;
    *count = uint32_t(pages.size());
    return ETCU_OK;
}

etcu_status tiff_decode_page(const std::vector<uint8_t>& file, const char* path, uint32_t page, uint32_t* width,
                             uint32_t* height, std::vector<float>& pixels) {
    std::vector<Page> pages;
    etcu_status st = parse_pages(file, path, pages);
    if (st != ETCU_OK) return st;
    if (page >= pages.size())
        return fail(ETCU_ERR_INVALID_ARGUMENT, "index out of bound: image stack %s has %zu images, not %u", path,
                    pages.size(), page + 1);
    const Page& pg = pages[page];
    if ((st = check_supported(pg, path)) != ETCU_OK) return st;
    const bool big = file[0] == 'M';
    const uint32_t W = pg.width, H = pg.height;
    pixels.assign(size_t(W) * H, 0.f);
    std::vector<uint8_t> buf;
    const size_t row_bytes_max = size_t(std::max(W, pg.tile_w)) * (pg.bits / 8);
    std::vector<uint8_t> row(row_bytes_max);
    std::vector<float> frow(std::max(W, pg.tile_w));
    if (!pg.tiled) {
        const uint32_t rps = std::min(pg.rows_per_strip == 0 ? H : pg.rows_per_strip, H);
        const uint32_t strips = (H + rps - 1) / rps;
        const size_t rb = size_t(W) * (pg.bits / 8);
        for (uint32_t s = 0; s < strips; ++s) {
            const uint32_t rows = std::min(rps, H - s * rps);
            if ((st = decode_block(file, pg, s, W, rows, buf, path)) != ETCU_OK) return st;
            for (uint32_t r = 0; r < rows; ++r) {
                std::memcpy(row.data(), buf.data() + r * rb, rb);
                row_to_float(row.data(), W, pg, big, pixels.data() + (size_t(s) * rps + r) * W);
            }
        }
    } else {
        const uint32_t tw = pg.tile_w, th = pg.tile_h;
        const uint32_t across = (W + tw - 1) / tw, down = (H + th - 1) / th;
        const size_t rb = size_t(tw) * (pg.bits / 8);
        for (uint32_t ty = 0; ty < down; ++ty)
            for (uint32_t tx = 0; tx < across; ++tx) {
                if ((st = decode_block(file, pg, size_t(ty) * across + tx, tw, th, buf, path)) != ETCU_OK) return st;
                for (uint32_t r = 0; r < th && ty * th + r < H; ++r) {
                    std::memcpy(row.data(), buf.data() + r * rb, rb);
                    row_to_float(row.data(), tw, pg, big, frow.data());
                    const uint32_t x0 = tx * tw, nx = std::min(tw, W - x0);
                    std::memcpy(pixels.data() + size_t(ty * th + r) * W + x0, frow.data(), nx * sizeof(float));
                }
            }
    }
    *width = W;
    *height = H;
    return ETCU_OK;
}

}  // namespace etcu_io

extern "C" etcu_status etcu_tiff_read_info(const char* path, uint32_t page, etcu_image_info* out) {
    if (!path || !out) return fail(ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    std::vector<uint8_t> file;
    if (!etcu_io::read_file(path, file)) return fail(ETCU_ERR_INVALID_ARGUMENT, "unable to load image %s", path);
    std::vector<Page> pages;
    const etcu_status st = parse_pages(file, path, pages);
    if (st != ETCU_OK) return st;
    if (page >= pages.size())
        return fail(ETCU_ERR_INVALID_ARGUMENT, "index out of bound: image stack %s has %zu images, not %u", path,
                    pages.size(), page + 1);
    const Page& pg = pages[page];
    out->width = pg.width;
    out->height = pg.height;
    out->pages = uint32_t(pages.size());
    out->bits_per_sample = pg.bits;
    out->sample_format = pg.format;
    out->compression = pg.compression;
    return ETCU_OK;
}

extern "C" etcu_status etcu_tiff_read(const char* path, uint32_t page, float* out, size_t capacity) {
    if (!path || !out) return fail(ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    std::vector<uint8_t> file;
    if (!etcu_io::read_file(path, file)) return fail(ETCU_ERR_INVALID_ARGUMENT, "unable to load image %s", path);
    uint32_t w, h;
    std::vector<float> px;
    const etcu_status st = etcu_io::tiff_decode_page(file, path, page, &w, &h, px);
    if (st != ETCU_OK) return st;
    if (capacity < px.size())
        return fail(ETCU_ERR_INVALID_ARGUMENT, "output holds %zu of %zu pixels", capacity, px.size());
    std::memcpy(out, px.data(), px.size() * sizeof(float));
    return ETCU_OK;
}

// One page, 32-bit float grey, one uncompressed strip, little-endian.
extern "C" etcu_status etcu_tiff_write(const char* path, const float* image, uint32_t width, uint32_t height) {
    if (!path || !image) return fail(ETCU_ERR_INVALID_ARGUMENT, "NULL argument");
    if (width == 0 || height == 0) return fail(ETCU_ERR_INVALID_ARGUMENT, "Image to save to %s is invalid!", path);
    const uint64_t bytes = uint64_t(width) * height * 4;
    constexpr uint32_t kData = 160;  // header 8 + directory 2 + 11 * 12 + 4 = 146, rounded up
    if (bytes + kData > 0xFFFFFFFFull)
        return fail(ETCU_ERR_UNSUPPORTED, "image %u x %u is too large for a TIFF file", width, height);
    std::vector<uint8_t> head(kData, 0);
    auto put16 = [&](size_t at, uint32_t v) { head[at] = uint8_t(v); head[at + 1] = uint8_t(v >> 8); };
    auto put32 = [&](size_t at, uint32_t v) {
        for (int k = 0; k < 4; ++k) head[at + k] = uint8_t(v >> (8 * k));
    };
    head[0] = head[1] = 'I';
    put16(2, 42);
    put32(4, 8);
    const struct { uint16_t tag, type; uint32_t value; } entries[] = {
        {kWidth, 4, width}, {kLength, 4, height}, {kBits, 3, 32}, {kCompression, 3, 1}, {kPhotometric, 3, 1},
        {kStripOffsets, 4, kData}, {kSamples, 3, 1}, {kRowsPerStrip, 4, height},
        {kStripByteCounts, 4, uint32_t(bytes)}, {kPlanar, 3, 1}, {kSampleFormat, 3, 3},
    };
    put16(8, uint16_t(sizeof(entries) / sizeof(entries[0])));
    size_t at = 10;
    for (const auto& e : entries) {
        put16(at, e.tag);
        put16(at + 2, e.type);
        put32(at + 4, 1);
        if (e.type == 3) put16(at + 8, e.value);
        else put32(at + 8, e.value);
        at += 12;
    }
    put32(at, 0);  // no next page
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return fail(ETCU_ERR_INVALID_ARGUMENT, "Failed to open output file %s for writing!", path);
    bool ok = std::fwrite(head.data(), 1, head.size(), fp) == head.size();
    for (uint32_t y = 0; ok && y < height; ++y) {  // little-endian host: float rows as they are
        ok = std::fwrite(image + size_t(y) * width, sizeof(float), width, fp) == width;
    }
    ok = (std::fclose(fp) == 0) && ok;
    if (!ok) return fail(ETCU_ERR_INVALID_ARGUMENT, "Error encountered while writing to output file %s !", path);
    return ETCU_OK;
}
