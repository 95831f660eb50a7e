// ffb_png.cpp -- the PNG the reference's CLI writes for a frame: RGBA8 with
// the render's numbers and its config in tEXt chunks
// (src/png_metadata.rs:144-183 for the keys and their formats,
// encode_png_with_metadata 229-262; wasm/python/src/render.rs:97-103).
// Host-side byte work on the boundary: the frame is already in host memory.

#include "ffb_png.hpp"

#include <zlib.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>

namespace ffb {

namespace {

void put32(std::vector<uint8_t>& v, uint32_t x) {
    v.push_back((uint8_t)(x >> 24)); v.push_back((uint8_t)(x >> 16)); v.push_back((uint8_t)(x >> 8)); v.push_back((uint8_t)x);
}

void chunk(std::vector<uint8_t>& png, const char type[4], const uint8_t* data, size_t n) {
    if (n > 0x7FFFFFFFu) throw std::runtime_error("PNG chunk too large");
    put32(png, (uint32_t)n);
    const size_t at = png.size();
    png.insert(png.end(), type, type + 4);
    if (n) png.insert(png.end(), data, data + n);
    uLong crc = crc32(0L, Z_NULL, 0);
    crc = crc32(crc, png.data() + at, (uInt)(4 + n));
    put32(png, (uint32_t)crc);
}

// UTF-8 to Latin-1 (tEXt's encoding); code points above 0xFF become '?'.
std::string latin1(const std::string& s) {
    std::string o;
    for (size_t i = 0; i < s.size();) {
        const unsigned char c = (unsigned char)s[i];
        if (c < 0x80) { o.push_back((char)c); ++i; continue; }
        int len = (c >> 5) == 6 ? 2 : (c >> 4) == 14 ? 3 : (c >> 3) == 30 ? 4 : 1;
        uint32_t cp = len == 2 ? (c & 0x1F) : len == 3 ? (c & 0x0F) : len == 4 ? (c & 0x07) : '?';
        for (int k = 1; k < len && i + k < s.size(); ++k) cp = (cp << 6) | ((unsigned char)s[i + k] & 0x3F);
        o.push_back(cp <= 0xFF ? (char)cp : '?');
        i += len;
    }
    return o;
}

}  // namespace

// SHA-256 (FIPS 180-4).
std::string sha256_hex(const std::string& msg) {
    static const uint32_t K[64] = {
        0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
        0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
        0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
        0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
        0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
        0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
        0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
        0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};
    uint32_t h[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a, 0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
    std::vector<uint8_t> m(msg.begin(), msg.end());
    const uint64_t bits = (uint64_t)msg.size() * 8;
    m.push_back(0x80);
    while (m.size() % 64 != 56) m.push_back(0);
    for (int i = 7; i >= 0; --i) m.push_back((uint8_t)(bits >> (8 * i)));
    auto rotr = [](uint32_t x, int n) { return (x >> n) | (x << (32 - n)); };
    for (size_t b = 0; b < m.size(); b += 64) {
        uint32_t w[64];
        for (int i = 0; i < 16; ++i)
            w[i] = (uint32_t)m[b + 4 * i] << 24 | (uint32_t)m[b + 4 * i + 1] << 16 | (uint32_t)m[b + 4 * i + 2] << 8 | m[b + 4 * i + 3];
        for (int i = 16; i < 64; ++i) {
            const uint32_t s0 = rotr(w[i - 15], 7) ^ rotr(w[i - 15], 18) ^ (w[i - 15] >> 3);
            const uint32_t s1 = rotr(w[i - 2], 17) ^ rotr(w[i - 2], 19) ^ (w[i - 2] >> 10);
            w[i] = w[i - 16] + s0 + w[i - 7] + s1;
        }
        uint32_t a = h[0], bb = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], hh = h[7];
        for (int i = 0; i < 64; ++i) {
            const uint32_t S1 = rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25);
            const uint32_t ch = (e & f) ^ (~e & g);
            const uint32_t t1 = hh + S1 + ch + K[i] + w[i];
            const uint32_t S0 = rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22);
            const uint32_t mj = (a & bb) ^ (a & c) ^ (bb & c);
            const uint32_t t2 = S0 + mj;
            hh = g; g = f; f = e; e = d + t1; d = c; c = bb; bb = a; a = t1 + t2;
        }
        h[0] += a; h[1] += bb; h[2] += c; h[3] += d; h[4] += e; h[5] += f; h[6] += g; h[7] += hh;
    }
    char out[65];
    for (int i = 0; i < 8; ++i) std::snprintf(out + 8 * i, 9, "%08x", h[i]);
    return std::string(out, 64);
}

// An f32 as Rust's Display writes it: the shortest decimal that reads back
// as the same f32, without an exponent.
std::string rust_f32(float v) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v > 0 ? "inf" : "-inf";
    char buf[64];
    for (int p = 1; p <= 9; ++p) {
        std::snprintf(buf, sizeof buf, "%.*g", p, (double)v);
        if (std::strtof(buf, nullptr) == v) break;
    }
    std::string s = buf;
    if (s.find('e') != std::string::npos || s.find('E') != std::string::npos) {
        // Spell the same digits out positionally.
        for (int d = 0; d <= 60; ++d) {
            std::snprintf(buf, sizeof buf, "%.*f", d, (double)v);
            if (std::strtof(buf, nullptr) == v) break;
        }
        s = buf;
    }
    return s;
}

std::vector<uint8_t> png_encode(const uint8_t* rgba, uint32_t w, uint32_t h,
                                const std::vector<std::pair<std::string, std::string>>& text) {
    if (w == 0 || h == 0) throw std::runtime_error("PNG of no pixels");
    std::vector<uint8_t> png = {0x89, 'P', 'N', 'G', 0x0D, 0x0A, 0x1A, 0x0A};
    uint8_t ihdr[13];
    for (int i = 0; i < 4; ++i) { ihdr[i] = (uint8_t)(w >> (24 - 8 * i)); ihdr[4 + i] = (uint8_t)(h >> (24 - 8 * i)); }
    ihdr[8] = 8;    // bit depth
    ihdr[9] = 6;    // colour type: RGBA
    ihdr[10] = 0; ihdr[11] = 0; ihdr[12] = 0;   // deflate, adaptive filtering, no interlace
    chunk(png, "IHDR", ihdr, 13);
    for (auto& kv : text) {
        const std::string k = latin1(kv.first), v = latin1(kv.second);
        if (k.empty() || k.size() > 79) throw std::runtime_error("bad PNG text keyword");
        std::vector<uint8_t> d(k.begin(), k.end());
        d.push_back(0);
        d.insert(d.end(), v.begin(), v.end());
        chunk(png, "tEXt", d.data(), d.size());
    }
    // Scanlines, each behind filter byte 1 (Sub: each byte minus the one
    // four to its left), which the long black runs of a flame compress well.
    const size_t row = (size_t)w * 4;
    std::vector<uint8_t> raw((row + 1) * h);
    for (uint32_t y = 0; y < h; ++y) {
        uint8_t* o = raw.data() + (row + 1) * y;
        const uint8_t* in = rgba + row * y;
        o[0] = 1;
        for (size_t i = 0; i < row; ++i) o[1 + i] = (uint8_t)(in[i] - (i >= 4 ? in[i - 4] : 0));
    }
    uLongf zn = compressBound((uLong)raw.size());
    std::vector<uint8_t> z(zn);
    if (compress2(z.data(), &zn, raw.data(), (uLong)raw.size(), 6) != Z_OK) throw std::runtime_error("deflate failed");
    const size_t step = 1u << 20;                  // IDAT chunks of at most 1 MiB
    for (size_t at = 0; at < zn; at += step) chunk(png, "IDAT", z.data() + at, std::min<size_t>(step, zn - at));
    chunk(png, "IEND", nullptr, 0);
    return png;
}

std::vector<std::pair<std::string, std::string>> png_metadata(const std::string& config_json, uint32_t w, uint32_t h,
                                                              uint64_t iterations, double ms, uint32_t ipt, const PngInfo& in) {
    char rt[64], sf[64];
    std::snprintf(rt, sizeof rt, "%.2fms", ms);
    std::snprintf(sf, sizeof sf, "%.2f", (double)in.speed_factor);
    return {
        {"Software", in.software},
        {"GitHash", ""},
        {"Branch", ""},
        {"BuildDate", in.build_date},
        {"Platform", "Linux"},
        {"RustcVersion", "n/a"},
        {"BuildProfile", "release"},
        {"Resolution", std::to_string(w) + "x" + std::to_string(h)},
        {"Iterations", std::to_string(iterations)},
        {"RenderTime", rt},
        {"IterationsPerThread", std::to_string(ipt)},
        {"SpeedFactor", sf},
        {"ConfigChecksum", "sha256:" + sha256_hex(config_json)},
        {"Config", config_json},
        {"BackgroundColor", rust_f32(in.background[0]) + "," + rust_f32(in.background[1]) + "," + rust_f32(in.background[2])},
        {"Exposure", rust_f32(in.exposure)},
        {"Gamma", rust_f32(in.gamma)},
        {"ToneCurve", in.tone_curve ? "true" : "false"},
        {"RenderMode", "2D"},
        {"Projection", "N/A"},
        {"ShaderVariations", std::to_string(in.variations)},
    };
}

}  // namespace ffb
