// Shared helpers of the host-side file-format code (no device code).
#pragma once

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "ettention_b200.h"

// Records the message of a failed context-free call for etcu_last_error(NULL)
// (defined with the context code in etcu_api.cu).
void etcu_set_context_free_error(const char* message);

namespace etcu_io {

inline etcu_status fail(etcu_status st, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    etcu_set_context_free_error(buf);
    return st;
}

// Whole file into memory; false if it cannot be opened or read.
inline bool read_file(const char* path, std::vector<uint8_t>& out) {
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return false;
    out.clear();
    uint8_t buf[1 << 16];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof(buf), fp)) > 0) out.insert(out.end(), buf, buf + n);
    const bool ok = !std::ferror(fp);
    std::fclose(fp);
    return ok;
}

// TIFF pages of a file (etcu_tiff.cpp): count, and one page decoded to float32.
etcu_status tiff_page_count(const std::vector<uint8_t>& file, const char* path, uint32_t* pages);
etcu_status tiff_decode_page(const std::vector<uint8_t>& file, const char* path, uint32_t page,
                             uint32_t* width, uint32_t* height, std::vector<float>& pixels);

}  // namespace etcu_io
