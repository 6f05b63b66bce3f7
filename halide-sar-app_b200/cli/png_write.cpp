// png_write.cpp -- PNG (ISO/IEC 15948) grayscale writer on zlib.
//
// Layout: 8-byte signature, IHDR (width, height, bit depth 8, colour type 0,
// deflate, filter method 0, no interlace), one IDAT holding the zlib stream
// of the rows, each row led by filter type 0, then IEND.  Every chunk is
// length (big-endian) + type + data + CRC-32 of type and data.
//
// The zlib stream is compressed on several threads: the filtered rows are
// cut into pieces, each deflated on its own as raw deflate data (it refers
// to no byte before it); every piece but the last ends with a sync flush
// (an empty stored block: byte-aligned and not final) and the last with the
// final block, so the pieces concatenate into one deflate stream.  The
// zlib header (32 KB window, default level) and the Adler-32 of all the
// rows, combined from the pieces' checksums, wrap it.
#include "png_write.h"

#include <zlib.h>

#include <algorithm>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <thread>
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

// Raw deflate of data[0, n) at `level`, ending with a sync flush or (last)
// the final block; false on a zlib error.
bool deflate_piece(const unsigned char *data, size_t n, int level, bool last, std::vector<unsigned char> &out) {
    z_stream s{};
    if (deflateInit2(&s, level, Z_DEFLATED, -15, 8, Z_DEFAULT_STRATEGY) != Z_OK) return false;
    out.resize(deflateBound(&s, (uLong)n) + 64);
    s.next_in = const_cast<Bytef *>(data);
    s.avail_in = (uInt)n;
    s.next_out = out.data();
    s.avail_out = (uInt)out.size();
    const int flush = last ? Z_FINISH : Z_SYNC_FLUSH;
    bool ok = true;
    for (;;) {
        const int r = deflate(&s, flush);
        if (r == Z_STREAM_ERROR) {
            ok = false;
            break;
        }
        if (last ? r == Z_STREAM_END : (s.avail_in == 0 && s.avail_out > 0)) break;
        if (s.avail_out == 0) {  // more output is pending: grow the buffer
            const size_t used = out.size();
            out.resize(used * 2);
            s.next_out = out.data() + used;
            s.avail_out = (uInt)(out.size() - used);
        } else if (r == Z_BUF_ERROR) {
            ok = false;
            break;
        }
    }
    out.resize(out.size() - s.avail_out);
    deflateEnd(&s);
    return ok;
}

// The zlib stream of raw at `level`, its pieces deflated in parallel.
std::vector<unsigned char> zlib_stream(const std::vector<unsigned char> &raw, int level) {
    const size_t n = raw.size();
    const size_t min_piece = 256u << 10, max_piece = 1u << 30;  // uInt counts per piece
    const size_t hw = std::max(1u, std::thread::hardware_concurrency());
    size_t parts = std::min<size_t>(std::min<size_t>(hw, 32), std::max<size_t>(1, n / min_piece));
    parts = std::max(parts, (n + max_piece - 1) / max_piece);
    std::vector<std::vector<unsigned char>> z(parts);
    std::vector<uLong> ad(parts);
    std::vector<char> ok(parts, 0);
    auto piece = [&](size_t i) {
        const size_t a = n * i / parts, b = n * (i + 1) / parts;
        ok[i] = deflate_piece(raw.data() + a, b - a, level, i + 1 == parts, z[i]);
        ad[i] = adler32(adler32(0L, Z_NULL, 0), raw.data() + a, (uInt)(b - a));
    };
    std::vector<std::thread> th;
    for (size_t i = 1; i < parts; ++i) th.emplace_back(piece, i);
    piece(0);
    for (auto &t : th) t.join();
    std::vector<unsigned char> out = {0x78, 0x9c};
    uLong adler = ad[0];
    for (size_t i = 0; i < parts; ++i) {
        if (!ok[i]) throw std::runtime_error("png: deflate failed");
        out.insert(out.end(), z[i].begin(), z[i].end());
        if (i) adler = adler32_combine(adler, ad[i], (z_off_t)(n * (i + 1) / parts - n * i / parts));
    }
    put_be32(out, (uint32_t)adler);
    return out;
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
    const std::vector<unsigned char> z = zlib_stream(raw, 6);

    std::vector<unsigned char> out = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    std::vector<unsigned char> ihdr;
    put_be32(ihdr, (uint32_t)width);
    put_be32(ihdr, (uint32_t)height);
    ihdr.insert(ihdr.end(), {8, 0, 0, 0, 0});
    chunk(out, "IHDR", ihdr.data(), ihdr.size());
    chunk(out, "IDAT", z.data(), z.size());
    chunk(out, "IEND", nullptr, 0);

    std::unique_ptr<FILE, int (*)(FILE *)> f(std::fopen(path.c_str(), "wb"), &std::fclose);
    if (!f) throw std::runtime_error("png: cannot write " + path);
    if (std::fwrite(out.data(), 1, out.size(), f.get()) != out.size())
        throw std::runtime_error("png: short write to " + path);
}

}  // namespace sarbp_cli
