// png_write.cpp -- PNG (ISO/IEC 15948) grayscale writer on zlib.
//
// Layout: 8-byte signature, IHDR (width, height, bit depth 8, colour type 0,
// deflate, filter method 0, no interlace), one IDAT holding the zlib stream
// of the rows, each row led by filter type 0, then IEND.  Every chunk is
// length (big-endian) + type + data + CRC-32 of type and data.
#include "png_write.h"

#include <zlib.h>

#include <cstdio>
#include <memory>
#include <stdexcept>
#include <vector>

namespace sarbp_cli {

namespace {

void put_be32(std::vector<unsigned char> &v, uint32_t x) {
    v.push_back((unsigned char)(x >> 24));
    v.push_back((unsigned char)(x >> 16));
    v.push_back((unsigned char)(x >> 8));
    v.push_back((unsigned char)x);
}

void chunk(std::vector<unsigned char> &out, const char type[4], const unsigned char *data, size_t n) {
    put_be32(out, (uint32_t)n);
    const size_t start = out.size();
    out.insert(out.end(), type, type + 4);
    if (n) out.insert(out.end(), data, data + n);
    const uLong crc = crc32(0L, out.data() + start, (uInt)(n + 4));
    put_be32(out, (uint32_t)crc);
}

}  // namespace

void png_write_gray8(const std::string &path, const uint8_t *pixels, int width, int height) {
    if (width < 1 || height < 1) throw std::runtime_error("png: empty image");
    const size_t row = (size_t)width + 1;
    std::vector<unsigned char> raw(row * (size_t)height);
    for (int y = 0; y < height; ++y) {
        raw[row * y] = 0;  // filter type None
        std::copy(pixels + (size_t)y * width, pixels + (size_t)(y + 1) * width, raw.begin() + row * y + 1);
    }
    uLongf zlen = compressBound((uLong)raw.size());
    std::vector<unsigned char> z(zlen);
    if (compress2(z.data(), &zlen, raw.data(), (uLong)raw.size(), 6) != Z_OK)
        throw std::runtime_error("png: deflate failed");

    std::vector<unsigned char> out = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    std::vector<unsigned char> ihdr;
    put_be32(ihdr, (uint32_t)width);
    put_be32(ihdr, (uint32_t)height);
    ihdr.insert(ihdr.end(), {8, 0, 0, 0, 0});
    chunk(out, "IHDR", ihdr.data(), ihdr.size());
    chunk(out, "IDAT", z.data(), zlen);
    chunk(out, "IEND", nullptr, 0);

    std::unique_ptr<FILE, int (*)(FILE *)> f(std::fopen(path.c_str(), "wb"), &std::fclose);
    if (!f) throw std::runtime_error("png: cannot write " + path);
    if (std::fwrite(out.data(), 1, out.size(), f.get()) != out.size())
        throw std::runtime_error("png: short write to " + path);
}

}  // namespace sarbp_cli
