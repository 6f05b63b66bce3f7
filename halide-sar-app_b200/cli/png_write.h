// png_write.h -- 8-bit grayscale PNG writer (the CLI's image output,
// sarbp.cpp:324 Halide::Tools::convert_and_save_image of a uint8 {nu, nv}
// buffer: width nu, height nv, row y = buffer row y).
#pragma once

#include <cstdint>
#include <string>

namespace sarbp_cli {

// Throws std::runtime_error on I/O or compression failure.
void png_write_gray8(const std::string &path, const uint8_t *pixels, int width, int height);

}  // namespace sarbp_cli
