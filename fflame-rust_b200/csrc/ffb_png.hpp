// ffb_png.hpp -- PNG encoding with the reference's metadata (ffb_png.cpp).
#pragma once

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

namespace ffb {

// What the metadata says beyond the render's own numbers.
struct PngInfo {
    std::string software;        // this build's name and version
    std::string build_date;
    float speed_factor = 0.5f;   // the config's (DEFAULT_SPEED_FACTOR)
    float background[3] = {0, 0, 0};
    float exposure = 1.0f, gamma = 4.0f;
    bool tone_curve = false;     // more than the two end points
    size_t variations = 0;       // distinct variations the flame uses
};

// RGBA8 (w*h*4 bytes) as a PNG with the given tEXt chunks, in order.
std::vector<uint8_t> png_encode(const uint8_t* rgba, uint32_t w, uint32_t h,
                                const std::vector<std::pair<std::string, std::string>>& text);
// The tEXt chunks of png_metadata.rs:144-183, in its order and formats.
std::vector<std::pair<std::string, std::string>> png_metadata(const std::string& config_json, uint32_t w, uint32_t h,
                                                              uint64_t iterations, double ms, uint32_t ipt, const PngInfo& in);
std::string sha256_hex(const std::string& msg);
std::string rust_f32(float v);

}  // namespace ffb
