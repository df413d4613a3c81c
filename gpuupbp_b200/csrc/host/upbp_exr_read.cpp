// OpenEXR reader for environment maps: single-part scanline images with
// NONE, RLE, ZIPS or ZIP compression and HALF or FLOAT channels, returned as
// RGB floats by channel name the way tinyexr's LoadEXR hands them to the
// reference (gpuupbp/misc/tinyexr_wrapper.cpp:97-136): R, G, B (a single
// channel of another name fills all three), rows top to bottom over the data
// window.  Written from the OpenEXR file layout specification: magic and
// version, attribute header (chlist, compression, dataWindow), chunk offset
// table, then chunks of (y, byte count, data) holding each scanline's
// channels in channel-list order; RLE and ZIP data are byte-interleaved and
// delta-coded before compression.
#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <iterator>
#include <string>
#include <vector>

#include "upbp_scene.h"

namespace upbp_host {
namespace {

enum : int { kNone = 0, kRle = 1, kZips = 2, kZip = 3 };
enum : int { kUint = 0, kHalf = 1, kFloat = 2 };

struct Channel {
    std::string name;
    int type;
};

float half_to_float(uint16_t h)
{
    const uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
    const int ex = (h >> 10) & 0x1f;
    uint32_t mant = h & 0x3ffu;
    uint32_t bits;
    if (ex == 0x1f) {
        bits = sign | 0x7f800000u | (mant << 13);  // inf, nan
    } else if (ex != 0) {
        bits = sign | ((uint32_t)(ex - 15 + 127) << 23) | (mant << 13);
    } else if (mant == 0) {
        bits = sign;
    } else {  // subnormal half: normalise
        int e = -14;
        while (!(mant & 0x400u)) {
            mant <<= 1;
            e--;
        }
        bits = sign | ((uint32_t)(e + 127) << 23) | ((mant & 0x3ffu) << 13);
    }
    float f;
    std::memcpy(&f, &bits, 4);
    return f;
}

// Undoes the byte delta coding and the split into even and odd bytes that
// RLE and ZIP apply before compressing.
void undo_predictor_interleave(std::vector<uint8_t>& t)
{
    for (size_t i = 1; i < t.size(); i++) t[i] = (uint8_t)(t[i - 1] + t[i] - 128);
    std::vector<uint8_t> out(t.size());
    const size_t half = (t.size() + 1) / 2;
    for (size_t k = 0; k < t.size(); k++) out[k] = (k & 1) ? t[half + k / 2] : t[k / 2];
    t.swap(out);
}

bool rle_decode(const uint8_t* in, size_t n, std::vector<uint8_t>& out, size_t expect)
{
    out.clear();
    size_t i = 0;
    while (i < n) {
        const int c = (int8_t)in[i++];
        if (c < 0) {
            if (i + (size_t)(-c) > n) return false;
            out.insert(out.end(), in + i, in + i + (-c));
            i += (size_t)(-c);
        } else {
            if (i >= n) return false;
            out.insert(out.end(), (size_t)c + 1, in[i++]);
        }
        if (out.size() > expect) return false;
    }
    return out.size() == expect;
}

}  // namespace

bool read_exr_rgb(const std::string& path, int& width, int& height, std::vector<float>& rgb, std::string& err)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        err = "could not open " + path;
        return false;
    }
    const std::vector<uint8_t> buf((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    size_t pos = 0;
    auto need = [&](size_t n) { return pos + n <= buf.size(); };
    auto rd32 = [&]() {
        int32_t v;
        std::memcpy(&v, &buf[pos], 4);
        pos += 4;
        return v;
    };
    auto rdstr = [&](std::string& s) {
        s.clear();
        while (pos < buf.size() && buf[pos]) s.push_back((char)buf[pos++]);
        if (pos >= buf.size()) return false;
        pos++;
        return true;
    };
    if (!need(8) || rd32() != 20000630) {
        err = path + ": not an OpenEXR file";
        return false;
    }
    const int32_t version = rd32();
    if ((version & 0xff) != 2 || (version & 0x200) || (version & 0x1000)) {
        err = path + ": only single-part scanline OpenEXR images are supported";
        return false;
    }
    std::vector<Channel> chans;
    int compression = -1;
    int32_t dw[4] = {0, 0, -1, -1};
    for (;;) {
        std::string name, type;
        if (!rdstr(name)) break;
        if (name.empty()) break;
        if (!rdstr(type) || !need(4)) break;
        const int32_t size = rd32();
        if (size < 0 || !need((size_t)size)) break;
        const size_t end = pos + (size_t)size;
        if (name == "channels" && type == "chlist") {
            while (pos < end && buf[pos]) {
                Channel c;
                if (!rdstr(c.name) || pos + 16 > end) break;
                c.type = rd32();
                pos += 12;  // pLinear, reserved, x/y sampling
                chans.push_back(c);
            }
        } else if (name == "compression" && size == 1) {
            compression = buf[pos];
        } else if (name == "dataWindow" && size == 16) {
            for (int k = 0; k < 4; k++) dw[k] = rd32();
        }
        pos = end;
    }
    const int64_t w = (int64_t)dw[2] - dw[0] + 1, h = (int64_t)dw[3] - dw[1] + 1;
    if (chans.empty() || w <= 0 || h <= 0 || w * h > (int64_t)1 << 28) {
        err = path + ": missing or invalid channels or data window";
        return false;
    }
    if (compression != kNone && compression != kRle && compression != kZips && compression != kZip) {
        err = path + ": unsupported OpenEXR compression (NONE, RLE, ZIPS and ZIP are read)";
        return false;
    }
    int src[3] = {-1, -1, -1};
    for (size_t k = 0; k < chans.size(); k++) {
        if (chans[k].type != kHalf && chans[k].type != kFloat) continue;
        if (chans[k].name == "R") src[0] = (int)k;
        if (chans[k].name == "G") src[1] = (int)k;
        if (chans[k].name == "B") src[2] = (int)k;
    }
    if (src[0] < 0 || src[1] < 0 || src[2] < 0) {
        if (chans.size() == 1 && chans[0].type != kUint) {
            src[0] = src[1] = src[2] = 0;
        } else {
            err = path + ": needs HALF or FLOAT channels R, G and B";
            return false;
        }
    }
    size_t line_bytes = 0;
    std::vector<size_t> chan_off(chans.size());
    for (size_t k = 0; k < chans.size(); k++) {
        chan_off[k] = line_bytes;
        line_bytes += (size_t)w * (chans[k].type == kHalf ? 2 : 4);
    }
    const int lines_per_chunk = compression == kZip ? 16 : 1;
    const int64_t chunks = (h + lines_per_chunk - 1) / lines_per_chunk;
    if (!need((size_t)chunks * 8)) {
        err = path + ": truncated offset table";
        return false;
    }
    std::vector<uint64_t> offs((size_t)chunks);
    std::memcpy(offs.data(), &buf[pos], (size_t)chunks * 8);
    width = (int)w;
    height = (int)h;
    rgb.assign((size_t)w * (size_t)h * 3, 0.f);
    std::vector<uint8_t> raw;
    for (int64_t c = 0; c < chunks; c++) {
        pos = (size_t)offs[(size_t)c];
        if (!need(8)) {
            err = path + ": truncated chunk";
            return false;
        }
        const int64_t y0 = (int64_t)rd32() - dw[1];
        const int32_t n = rd32();
        if (n < 0 || !need((size_t)n) || y0 < 0 || y0 >= h) {
            err = path + ": invalid chunk";
            return false;
        }
        const int lines = (int)std::min<int64_t>(lines_per_chunk, h - y0);
        const size_t expect = line_bytes * (size_t)lines;
        const uint8_t* data = &buf[pos];
        if ((size_t)n == expect || compression == kNone) {  // stored as is
            if ((size_t)n != expect) {
                err = path + ": chunk size does not match the data window";
                return false;
            }
            raw.assign(data, data + n);
        } else if (compression == kRle) {
            if (!rle_decode(data, (size_t)n, raw, expect)) {
                err = path + ": corrupt RLE chunk";
                return false;
            }
            undo_predictor_interleave(raw);
        } else {
            raw.resize(expect);
            uLongf got = (uLongf)expect;
            if (uncompress(raw.data(), &got, data, (uLong)n) != Z_OK || got != expect) {
                err = path + ": corrupt ZIP chunk";
                return false;
            }
            undo_predictor_interleave(raw);
        }
        for (int l = 0; l < lines; l++) {
            const uint8_t* line = raw.data() + (size_t)l * line_bytes;
            float* out = rgb.data() + ((size_t)(y0 + l) * (size_t)w) * 3;
            for (int ch = 0; ch < 3; ch++) {
                const Channel& cc = chans[(size_t)src[ch]];
                const uint8_t* p = line + chan_off[(size_t)src[ch]];
                for (int64_t x = 0; x < w; x++) {
                    float v;
                    if (cc.type == kHalf) {
                        uint16_t hv;
                        std::memcpy(&hv, p + 2 * x, 2);
                        v = half_to_float(hv);
                    } else {
                        std::memcpy(&v, p + 4 * x, 4);
                    }
                    out[3 * x + ch] = v;
                }
            }
        }
    }
    return true;
}

}  // namespace upbp_host
