// exr_read.cu — reads the RGB channels of OpenEXR images for textures and environment
// maps, as Texture2D's constructor does through Imf::RgbaInputFile
// (Aurora/src/frontend/texture2D.cpp:23-46): the data window, top row first. Host code.
//
// Supported: single-part scanline files (OpenEXR 2 header, version 2), channels of type
// HALF, FLOAT or UINT with sampling 1, compression NONE, RLE, ZIPS and ZIP (zlib), any
// line order. R, G and B are read (a missing one is 0; a file with only Y gives
// R = G = B = Y). Tiled, deep and multi-part files and the other compressions (PIZ,
// PXR24, B44, DWA) are reported as unsupported.
//
// Layout (the published OpenEXR file layout): magic 20000630, version word, attributes
// (name, type, size, value) up to an empty name, a table of chunk offsets, then chunks
// (int32 first scanline, int32 byte count, data). A chunk holds 1 (NONE, RLE, ZIPS) or
// 16 (ZIP) scanlines; within it each scanline stores its channels one after another in
// the channel list's (name) order. RLE and ZIP data, once decoded, are byte-interleaved
// (even bytes then odd bytes) and delta-coded (each byte + previous - 128); a chunk whose
// byte count equals the uncompressed size is stored raw.
#include "aur_capi_internal.h"
#include "aur_image_io.h"
#include <cuda_fp16.h>
#include <zlib.h>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace aur {
namespace {

enum : int { kNone = 0, kRle = 1, kZips = 2, kZip = 3 };

struct Channel { std::string name; int type; };   // type: 0 UINT, 1 HALF, 2 FLOAT

int type_bytes(int t) { return t == 1 ? 2 : 4; }

uint32_t rd32(const unsigned char* p) { return (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24; }
uint64_t rd64(const unsigned char* p) { return (uint64_t)rd32(p) | (uint64_t)rd32(p + 4) << 32; }

// Reverses the byte interleave and the delta coding of RLE / ZIP chunks.
void undo_predictor(std::vector<unsigned char>& t) {
    const size_t n = t.size();
    for (size_t i = 1; i < n; ++i) t[i] = (unsigned char)(t[i - 1] + t[i] - 128);
    std::vector<unsigned char> out(n);
    const size_t half = (n + 1) / 2;
    for (size_t i = 0; i < n; ++i) out[i] = (i & 1) ? t[half + i / 2] : t[i / 2];
    t.swap(out);
}

// Run-length decoding: a signed count byte c < 0 is followed by -c literal bytes, c >= 0 by
// one byte repeated c + 1 times.
bool rle_decode(const unsigned char* in, size_t n, std::vector<unsigned char>& out, size_t expect) {
    out.clear();
    size_t i = 0;
    while (i < n) {
        const int c = (int)(signed char)in[i++];
        if (c < 0) {
            const size_t k = (size_t)(-c);
            if (i + k > n || out.size() + k > expect) return false;
            out.insert(out.end(), in + i, in + i + k);
            i += k;
        } else {
            if (i >= n || out.size() + (size_t)c + 1 > expect) return false;
            out.insert(out.end(), (size_t)c + 1, in[i++]);
        }
    }
    return out.size() == expect;
}

}  // namespace

aur_status read_exr_rgb(const std::string& path, std::vector<float>* rgb, int* w_out, int* h_out, std::string* err) {
    auto bad = [&](aur_status s, const std::string& m) { *err = m + ": " + path; return s; };
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) return bad(AUR_ERR_IO, "cannot open EXR file");
    std::vector<unsigned char> b;
    {
        unsigned char buf[1 << 16];
        size_t k;
        while ((k = fread(buf, 1, sizeof(buf), f)) > 0) b.insert(b.end(), buf, buf + k);
        fclose(f);
    }
    const size_t n = b.size();
    if (n < 8 || rd32(b.data()) != 20000630u) return bad(AUR_ERR_PARSE, "not an OpenEXR file");
    const uint32_t ver = rd32(b.data() + 4);
    if ((ver & 0xff) != 2) return bad(AUR_ERR_UNSUPPORTED, "unsupported OpenEXR version");
    if (ver & 0x200) return bad(AUR_ERR_UNSUPPORTED, "tiled OpenEXR files are not read");
    if (ver & 0x1800) return bad(AUR_ERR_UNSUPPORTED, "deep or multi-part OpenEXR files are not read");
    size_t pos = 8;
    auto cstr = [&](std::string* s) {
        size_t e = pos;
        while (e < n && b[e] != 0) ++e;
        if (e >= n) return false;
        s->assign((const char*)b.data() + pos, e - pos);
        pos = e + 1;
        return true;
    };
    std::vector<Channel> chans;
    int comp = -1;
    int x0 = 0, y0 = 0, x1 = -1, y1 = -1;
    bool have_dw = false;
    while (true) {
        std::string name, type;
        if (!cstr(&name)) return bad(AUR_ERR_PARSE, "truncated EXR header");
        if (name.empty()) break;
        if (!cstr(&type) || pos + 4 > n) return bad(AUR_ERR_PARSE, "truncated EXR header");
        const uint32_t size = rd32(b.data() + pos);
        pos += 4;
        if (size > n - pos) return bad(AUR_ERR_PARSE, "truncated EXR attribute");
        const unsigned char* v = b.data() + pos;
        if (name == "channels" && type == "chlist") {
            size_t q = 0;
            while (q < size && v[q] != 0) {
                size_t e = q;
                while (e < size && v[e] != 0) ++e;
                if (e + 17 > size) return bad(AUR_ERR_PARSE, "bad EXR channel list");
                Channel c;
                c.name.assign((const char*)v + q, e - q);
                c.type = (int)rd32(v + e + 1);
                const int xs = (int)rd32(v + e + 9), ys = (int)rd32(v + e + 13);
                if (c.type < 0 || c.type > 2) return bad(AUR_ERR_PARSE, "bad EXR channel type");
                if (xs != 1 || ys != 1) return bad(AUR_ERR_UNSUPPORTED, "subsampled EXR channels are not read");
                chans.push_back(c);
                q = e + 17;
            }
        } else if (name == "compression" && size >= 1) {
            comp = v[0];
        } else if (name == "dataWindow" && size >= 16) {
            x0 = (int)rd32(v); y0 = (int)rd32(v + 4); x1 = (int)rd32(v + 8); y1 = (int)rd32(v + 12);
            have_dw = true;
        }
        pos += size;   // lineOrder is not needed: every chunk carries its first scanline
    }
    if (!have_dw || chans.empty() || comp < 0) return bad(AUR_ERR_PARSE, "EXR header lacks channels, compression or dataWindow");
    if (comp != kNone && comp != kRle && comp != kZips && comp != kZip)
        return bad(AUR_ERR_UNSUPPORTED, "EXR compression " + std::to_string(comp) +
                                            " is not read (NONE, RLE, ZIPS and ZIP are)");
    const long long W = (long long)x1 - x0 + 1, H = (long long)y1 - y0 + 1;
    if (W <= 0 || H <= 0 || W * H > (1ll << 28)) return bad(AUR_ERR_PARSE, "bad EXR data window");
    const int lines = comp == kZip ? 16 : 1;
    const long long nchunks = (H + lines - 1) / lines;
    if (pos + 8 * (size_t)nchunks > n) return bad(AUR_ERR_PARSE, "truncated EXR offset table");
    size_t line_bytes = 0;
    for (const Channel& c : chans) line_bytes += (size_t)W * type_bytes(c.type);
    int ci[3] = {-1, -1, -1}, cy = -1;
    for (size_t k = 0; k < chans.size(); ++k) {
        if (chans[k].name == "R") ci[0] = (int)k;
        else if (chans[k].name == "G") ci[1] = (int)k;
        else if (chans[k].name == "B") ci[2] = (int)k;
        else if (chans[k].name == "Y") cy = (int)k;
    }
    if (ci[0] < 0 && ci[1] < 0 && ci[2] < 0 && cy >= 0) ci[0] = ci[1] = ci[2] = cy;   // luminance only
    rgb->assign((size_t)W * H * 3, 0.f);
    std::vector<unsigned char> raw;
    for (long long c = 0; c < nchunks; ++c) {
        const uint64_t off = rd64(b.data() + pos + 8 * c);
        if (off > n || n - off < 8) return bad(AUR_ERR_PARSE, "bad EXR chunk offset");
        const int ys = (int)rd32(b.data() + off);
        const uint32_t size = rd32(b.data() + off + 4);
        if (size > n - off - 8) return bad(AUR_ERR_PARSE, "truncated EXR chunk");
        const long long row0 = (long long)ys - y0;
        if (row0 < 0 || row0 >= H || row0 % lines) return bad(AUR_ERR_PARSE, "bad EXR chunk scanline");
        const int nl = (int)std::min<long long>(lines, H - row0);
        const size_t expect = line_bytes * nl;
        const unsigned char* data = b.data() + off + 8;
        if (size == expect || comp == kNone) {
            if (size != expect) return bad(AUR_ERR_PARSE, "bad EXR chunk size");
            raw.assign(data, data + size);
        } else if (comp == kRle) {
            if (!rle_decode(data, size, raw, expect)) return bad(AUR_ERR_PARSE, "bad EXR RLE chunk");
            undo_predictor(raw);
        } else {
            raw.resize(expect);
            uLongf got = (uLongf)expect;
            if (uncompress(raw.data(), &got, data, size) != Z_OK || got != expect)
                return bad(AUR_ERR_PARSE, "bad EXR ZIP chunk");
            undo_predictor(raw);
        }
        size_t q = 0;
        for (int l = 0; l < nl; ++l) {
            float* row = rgb->data() + (size_t)(row0 + l) * W * 3;
            for (size_t k = 0; k < chans.size(); ++k) {
                const int t = chans[k].type, tb = type_bytes(t);
                for (int out = 0; out < 3; ++out) {
                    if (ci[out] != (int)k) continue;
                    for (long long x = 0; x < W; ++x) {
                        const unsigned char* p = raw.data() + q + (size_t)x * tb;
                        float val;
                        if (t == 1) {
                            const uint16_t bits = (uint16_t)(p[0] | p[1] << 8);
                            __half h;
                            memcpy(&h, &bits, 2);
                            val = __half2float(h);
                        } else if (t == 2) {
                            const uint32_t bits = rd32(p);
                            memcpy(&val, &bits, 4);
                        } else {
                            val = (float)rd32(p);
                        }
                        row[3 * x + out] = val;
                    }
                }
                q += (size_t)W * tb;
            }
        }
    }
    *w_out = (int)W;
    *h_out = (int)H;
    return AUR_OK;
}

}  // namespace aur
