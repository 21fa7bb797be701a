// film_io.cu — writes a rendered film (width x height RGBA floats, top row first) to
// disk: OpenEXR (the reference's output, OpenexrDisplay, frontend/openexrDisplay.cpp:
// 132-244, half RGBA) as an uncompressed scanline file, or PFM (RGB float). Host code.
#include "aur_capi_internal.h"
#include <cuda_fp16.h>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace aur {
namespace {

struct Out {
    std::vector<unsigned char> b;
    void bytes(const void* p, size_t n) { const unsigned char* c = (const unsigned char*)p; b.insert(b.end(), c, c + n); }
    void u8(uint8_t v) { b.push_back(v); }
    void i32(int32_t v) { for (int k = 0; k < 4; ++k) b.push_back((unsigned char)((uint32_t)v >> (8 * k))); }
    void u64(uint64_t v) { for (int k = 0; k < 8; ++k) b.push_back((unsigned char)(v >> (8 * k))); }
    void f32(float f) { uint32_t u; memcpy(&u, &f, 4); i32((int32_t)u); }
    void str(const char* s) { bytes(s, strlen(s) + 1); }
    void attr(const char* name, const char* type, int32_t size) { str(name); str(type); i32(size); }
};

bool write_file(const char* path, const void* data, size_t n) {
    FILE* f = fopen(path, "wb");
    if (!f) return false;
    const size_t w = fwrite(data, 1, n, f);
    const bool ok = fclose(f) == 0 && w == n;
    return ok;
}

// OpenEXR 2 single-part scanline file, NO_COMPRESSION (one scanline per block),
// channels A, B, G, R (the format stores channels in name order), little endian.
std::vector<unsigned char> exr(const float* film, int w, int h, bool half) {
    Out o;
    o.i32(20000630);                 // magic
    o.i32(2);                        // version 2, single-part scanline
    const int ptype = half ? 1 : 2;  // HALF = 1, FLOAT = 2
    const char* names[4] = {"A", "B", "G", "R"};
    o.attr("channels", "chlist", 4 * (2 + 4 + 1 + 3 + 4 + 4) + 1);
    for (const char* n : names) {
        o.str(n);
        o.i32(ptype);
        o.u8(0); o.u8(0); o.u8(0); o.u8(0);   // pLinear + reserved
        o.i32(1); o.i32(1);                   // x / y sampling
    }
    o.u8(0);
    o.attr("compression", "compression", 1); o.u8(0);
    o.attr("dataWindow", "box2i", 16); o.i32(0); o.i32(0); o.i32(w - 1); o.i32(h - 1);
    o.attr("displayWindow", "box2i", 16); o.i32(0); o.i32(0); o.i32(w - 1); o.i32(h - 1);
    o.attr("lineOrder", "lineOrder", 1); o.u8(0);
    o.attr("pixelAspectRatio", "float", 4); o.f32(1.f);
    o.attr("screenWindowCenter", "v2f", 8); o.f32(0.f); o.f32(0.f);
    o.attr("screenWindowWidth", "float", 4); o.f32(1.f);
    o.u8(0);                                 // end of header
    const size_t esz = half ? 2 : 4;
    const size_t line = 4 * esz * (size_t)w;
    const size_t table = o.b.size();
    const size_t first = table + 8 * (size_t)h;
    for (int y = 0; y < h; ++y) o.u64(first + (size_t)y * (8 + line));
    const int chan_of[4] = {3, 2, 1, 0};     // A, B, G, R from RGBA
    for (int y = 0; y < h; ++y) {
        o.i32(y);
        o.i32((int32_t)line);
        for (int c = 0; c < 4; ++c)
            for (int x = 0; x < w; ++x) {
                const float v = film[4 * ((size_t)y * w + x) + chan_of[c]];
                if (half) {
                    const __half hv = __float2half_rn(v);
                    o.bytes(&hv, 2);
                } else {
                    o.f32(v);
                }
            }
    }
    return std::move(o.b);
}

// PFM: "PF", width height, -1 (little endian), RGB rows bottom to top.
std::vector<unsigned char> pfm(const float* film, int w, int h) {
    Out o;
    const std::string head = "PF\n" + std::to_string(w) + " " + std::to_string(h) + "\n-1.0\n";
    o.bytes(head.data(), head.size());
    for (int y = h - 1; y >= 0; --y)
        for (int x = 0; x < w; ++x)
            for (int c = 0; c < 3; ++c) o.f32(film[4 * ((size_t)y * w + x) + c]);
    return std::move(o.b);
}

}  // namespace
}  // namespace aur

using namespace aur;

extern "C" aur_status aur_film_write(const char* path, const float* film_rgba, int32_t width, int32_t height,
                                     int32_t format) {
    if (!path || !film_rgba) return fail(AUR_ERR_INVALID_ARG, "aur_film_write: NULL argument");
    if (width <= 0 || height <= 0 || (long long)width * height > (1ll << 30))
        return fail(AUR_ERR_INVALID_ARG, "aur_film_write: bad size");
    if (format != AUR_FILM_PFM && format != AUR_FILM_EXR_HALF && format != AUR_FILM_EXR_FLOAT)
        return fail(AUR_ERR_INVALID_ARG, "aur_film_write: unknown format");
    const size_t n = 4 * (size_t)width * height;
    std::vector<float> host;
    const float* f = film_rgba;
    if (is_device_ptr(film_rgba)) {
        host.resize(n);
        const cudaError_t e = cudaMemcpy(host.data(), film_rgba, n * sizeof(float), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(e, "aur_film_write");
        f = host.data();
    }
    const std::vector<unsigned char> bytes =
        format == AUR_FILM_PFM ? pfm(f, width, height) : exr(f, width, height, format == AUR_FILM_EXR_HALF);
    if (!write_file(path, bytes.data(), bytes.size()))
        return fail(AUR_ERR_IO, std::string("aur_film_write: cannot write ") + path);
    return AUR_OK;
}
