// Image files of the `image` shader node (image_io.cpp).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace vs {

// Decoded pixels: `channels` floats per pixel, row 0 the top of the image;
// 8- and 16-bit formats scaled to [0, 1], HDR as stored.
struct Image {
    uint32_t width = 0, height = 0;
    int channels = 0;
    std::vector<float> data;
};

// PNG, baseline JPEG, Radiance HDR or OpenEXR (scanline; NONE, RLE, ZIPS or
// ZIP compression), by file extension; throws std::runtime_error with the
// reason otherwise ("unsupported: ..." for a valid file using a feature that
// is not implemented).
Image load_image(const std::string &path);

// The sRGB transfer function's inverse (IEC 61966-2-1).
float srgb_to_linear(float c);

}  // namespace vs
