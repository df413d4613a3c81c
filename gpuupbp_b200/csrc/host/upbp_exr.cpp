// OpenEXR writer: scanline image, no compression, three HALF channels named
// B, G, R (the channel set and pixel type tinyexr_wrapper::save_exr writes,
// gpuupbp/misc/tinyexr_wrapper.cpp:34-95).  Written from the OpenEXR file
// layout specification: magic + version, attribute header, per-scanline
// offset table, then one block per scanline (y, byte count, channel rows in
// alphabetical channel order).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "upbp_scene.h"

namespace {

// float -> IEEE 754 binary16, round to nearest even, with overflow to inf.
uint16_t to_half(float f)
{
    uint32_t x;
    std::memcpy(&x, &f, 4);
    const uint32_t sign = (x >> 16) & 0x8000u;
    const uint32_t ex = (x >> 23) & 0xffu;
    uint32_t mant = x & 0x7fffffu;
    if (ex == 0xffu) return (uint16_t)(sign | 0x7c00u | (mant ? 0x200u : 0u));  // inf / nan
    int e = (int)ex - 127 + 15;
    if (e >= 31) return (uint16_t)(sign | 0x7c00u);                           // overflow
    if (e <= 0) {                                                             // subnormal or zero
        if (e < -10) return (uint16_t)sign;
        mant |= 0x800000u;
        const int shift = 14 - e;
        uint32_t h = mant >> shift;
        const uint32_t rem = mant & ((1u << shift) - 1u);
        const uint32_t half = 1u << (shift - 1);
        if (rem > half || (rem == half && (h & 1u))) h++;
        return (uint16_t)(sign | h);
    }
    uint32_t h = ((uint32_t)e << 10) | (mant >> 13);
    const uint32_t rem = mant & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h++;  // may carry into the exponent: correct
    return (uint16_t)(sign | h);
}

void put_u32(std::vector<uint8_t>& b, uint32_t v)
{
    for (int i = 0; i < 4; i++) b.push_back((uint8_t)(v >> (8 * i)));
}
void put_i32(std::vector<uint8_t>& b, int32_t v) { put_u32(b, (uint32_t)v); }
void put_u64(std::vector<uint8_t>& b, uint64_t v)
{
    for (int i = 0; i < 8; i++) b.push_back((uint8_t)(v >> (8 * i)));
}
void put_f32(std::vector<uint8_t>& b, float f)
{
    uint32_t u;
    std::memcpy(&u, &f, 4);
    put_u32(b, u);
}
void put_str(std::vector<uint8_t>& b, const char* s)
{
    while (*s) b.push_back((uint8_t)*s++);
    b.push_back(0);
}
void attr(std::vector<uint8_t>& b, const char* name, const char* type, const std::vector<uint8_t>& val)
{
    put_str(b, name);
    put_str(b, type);
    put_u32(b, (uint32_t)val.size());
    b.insert(b.end(), val.begin(), val.end());
}

}  // namespace

extern "C" int upbp_write_exr(const char* path, const float* rgb, uint32_t w, uint32_t h)
{
    return upbp_host::abi_guard([&]() -> int {
        if (!path || !rgb || w == 0 || h == 0) return UPBP_ERR_ARGS;
        std::vector<uint8_t> out;
        put_u32(out, 20000630u);  // magic
        put_u32(out, 2u);         // version 2, scanline
        {
            std::vector<uint8_t> ch;
            for (const char* name : {"B", "G", "R"}) {
                put_str(ch, name);
                put_i32(ch, 1);  // HALF
                ch.push_back(0);  // pLinear
                ch.push_back(0);
                ch.push_back(0);
                ch.push_back(0);
                put_i32(ch, 1);  // x sampling
                put_i32(ch, 1);  // y sampling
            }
            ch.push_back(0);
            attr(out, "channels", "chlist", ch);
        }
        attr(out, "compression", "compression", std::vector<uint8_t>{0});
        std::vector<uint8_t> box;
        put_i32(box, 0);
        put_i32(box, 0);
        put_i32(box, (int32_t)w - 1);
        put_i32(box, (int32_t)h - 1);
        attr(out, "dataWindow", "box2i", box);
        attr(out, "displayWindow", "box2i", box);
        attr(out, "lineOrder", "lineOrder", std::vector<uint8_t>{0});
        std::vector<uint8_t> one;
        put_f32(one, 1.f);
        attr(out, "pixelAspectRatio", "float", one);
        std::vector<uint8_t> center;
        put_f32(center, 0.f);
        put_f32(center, 0.f);
        attr(out, "screenWindowCenter", "v2f", center);
        attr(out, "screenWindowWidth", "float", one);
        out.push_back(0);  // end of header
        const uint32_t row_bytes = w * 3u * 2u;
        const uint64_t table_pos = out.size();
        const uint64_t first_block = table_pos + 8ull * h;
        for (uint32_t y = 0; y < h; y++) put_u64(out, first_block + (uint64_t)y * (8ull + row_bytes));
        for (uint32_t y = 0; y < h; y++) {
            put_i32(out, (int32_t)y);
            put_u32(out, row_bytes);
            for (int c : {2, 1, 0}) {  // B, G, R
                for (uint32_t x = 0; x < w; x++) {
                    const uint16_t hv = to_half(rgb[3 * ((size_t)y * w + x) + c]);
                    out.push_back((uint8_t)(hv & 0xff));
                    out.push_back((uint8_t)(hv >> 8));
                }
            }
        }
        FILE* f = std::fopen(path, "wb");
        if (!f) {
            upbp_host::set_error(std::string("could not write ") + path);
            return UPBP_ERR_IO;
        }
        const size_t n = std::fwrite(out.data(), 1, out.size(), f);
        std::fclose(f);
        return n == out.size() ? UPBP_OK : UPBP_ERR_IO;
    });
}

// ---- BMP and Radiance HDR (host/framebuffer.cpp:129-233 of the reference)

// 24-bit BMP, rows bottom up, BGR bytes of pow(c, 1/gamma) * 255 clamped to
// [0, 255] and truncated; no row padding, as the reference writes it (its
// files are valid BMPs when the width is a multiple of 4).
extern "C" int upbp_write_bmp(const char* path, const float* rgb, uint32_t w, uint32_t h, float gamma)
{
    return upbp_host::abi_guard([&]() -> int {
        if (!path || !rgb || w == 0 || h == 0 || !(gamma > 0.f)) return UPBP_ERR_ARGS;
        FILE* f = std::fopen(path, "wb");
        if (!f) {
            upbp_host::set_error(std::string("could not open ") + path);
            return UPBP_ERR_IO;
        }
        auto u32 = [&](uint32_t v) { std::fwrite(&v, 4, 1, f); };
        auto i32 = [&](int32_t v) { std::fwrite(&v, 4, 1, f); };
        auto u16 = [&](uint16_t v) { std::fwrite(&v, 2, 1, f); };
        const uint32_t header = 52;  // the reference's header struct (52 bytes) after "BM"
        std::fwrite("BM", 1, 2, f);
        u32(header + 2 + w * h * 3);
        u32(0);
        u32(header + 2);
        u32(40);
        i32((int32_t)w);
        i32((int32_t)h);
        u16(1);
        u16(24);
        u32(0);
        u32(w * h * 3);
        u32(2953);
        u32(2953);
        u32(0);
        u32(0);
        const float inv = 1.f / gamma;
        std::vector<unsigned char> row((size_t)w * 3);
        for (uint32_t y = 0; y < h; y++) {
            const float* src = rgb + (size_t)(h - y - 1) * w * 3;
            for (uint32_t x = 0; x < w; x++)
                for (int c = 0; c < 3; c++) {
                    const float v = std::pow(src[3 * x + 2 - c], inv) * 255.f;
                    row[3 * x + c] = (unsigned char)std::min(255.f, std::max(0.f, v));
                }
            std::fwrite(row.data(), 1, row.size(), f);
        }
        const bool ok = std::fclose(f) == 0;
        return ok ? UPBP_OK : UPBP_ERR_IO;
    });
}

// Radiance RGBE: the "#?RADIANCE" header, -Y h +X w, then uncompressed
// 4-byte pixels (mantissas scaled by frexp of the largest component).
extern "C" int upbp_write_hdr(const char* path, const float* rgb, uint32_t w, uint32_t h)
{
    return upbp_host::abi_guard([&]() -> int {
        if (!path || !rgb || w == 0 || h == 0) return UPBP_ERR_ARGS;
        FILE* f = std::fopen(path, "wb");
        if (!f) {
            upbp_host::set_error(std::string("could not open ") + path);
            return UPBP_ERR_IO;
        }
        std::fprintf(f, "#?RADIANCE\n# SmallUPBP\nFORMAT=32-bit_rle_rgbe\n\n-Y %u +X %u\n", h, w);
        std::vector<unsigned char> px((size_t)w * h * 4, 0);
        for (size_t i = 0; i < (size_t)w * h; i++) {
            const float* c = rgb + 3 * i;
            float v = std::max(c[0], std::max(c[1], c[2]));
            if (v >= 1e-32f) {
                int e;
                v = float(std::frexp(v, &e) * 256.f / v);
                px[4 * i + 0] = (unsigned char)(c[0] * v);
                px[4 * i + 1] = (unsigned char)(c[1] * v);
                px[4 * i + 2] = (unsigned char)(c[2] * v);
                px[4 * i + 3] = (unsigned char)(e + 128);
            }
        }
        std::fwrite(px.data(), 1, px.size(), f);
        const bool ok = std::fclose(f) == 0;
        return ok ? UPBP_OK : UPBP_ERR_IO;
    });
}

// The reference's save(fb, name, gamma) (host/framebuffer.cpp:114-127): the
// writer chosen by the name's last three characters.
extern "C" int upbp_write_image(const char* path, const float* rgb, uint32_t w, uint32_t h, float gamma)
{
    if (!path) return UPBP_ERR_ARGS;
    const std::string p = path;
    const std::string ext = p.size() >= 3 ? p.substr(p.size() - 3) : "";
    if (ext == "bmp") return upbp_write_bmp(path, rgb, w, h, gamma);
    if (ext == "hdr") return upbp_write_hdr(path, rgb, w, h);
    if (ext == "exr") return upbp_write_exr(path, rgb, w, h);
    upbp_host::set_error("unknown image extension " + ext);
    return UPBP_ERR_ARGS;
}
