// npy.cpp -- .npy reader/writer (see npy.h).
#include "npy.h"

#include <unistd.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <thread>
#include <vector>

namespace sarbp_cli {

namespace {

struct FileCloser {
    void operator()(FILE *f) const { if (f) std::fclose(f); }
};
using File = std::unique_ptr<FILE, FileCloser>;

[[noreturn]] void bad(const std::string &path, const std::string &what) {
    throw std::runtime_error("npy: " + path + ": " + what);
}

// n bytes of fd from offset off into dst; payloads of many megabytes (the
// phase history) in pieces on several threads; false on a short read
bool read_at(int fd, off_t off, unsigned char *dst, size_t n) {
    const size_t min_piece = 8u << 20;
    const size_t hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t parts = std::max<size_t>(1, std::min<size_t>(std::min<size_t>(hw, 8), n / min_piece));
    std::vector<char> ok(parts, 0);
    auto piece = [&](size_t i) {
        size_t a = n * i / parts;
        const size_t b = n * (i + 1) / parts;
        while (a < b) {
            const ssize_t r = pread(fd, dst + a, b - a, off + (off_t)a);
            if (r <= 0) return;
            a += (size_t)r;
        }
        ok[i] = 1;
    };
    std::vector<std::thread> th;
    for (size_t i = 1; i < parts; ++i) th.emplace_back(piece, i);
    piece(0);
    for (auto &t : th) t.join();
    return std::all_of(ok.begin(), ok.end(), [](char c) { return c != 0; });
}

// value text that follows 'key': in the header dict, trimmed at the next
// top-level comma or closing brace
std::string dict_value(const std::string &h, const std::string &key, const std::string &path) {
    const std::string k1 = "'" + key + "'", k2 = "\"" + key + "\"";
    size_t p = h.find(k1);
    size_t klen = k1.size();
    if (p == std::string::npos) {
        p = h.find(k2);
        klen = k2.size();
    }
    if (p == std::string::npos) bad(path, "header has no " + key);
    p = h.find(':', p + klen);
    if (p == std::string::npos) bad(path, "malformed header");
    ++p;
    while (p < h.size() && h[p] == ' ') ++p;
    int depth = 0;
    size_t q = p;
    for (; q < h.size(); ++q) {
        const char c = h[q];
        if (c == '(' || c == '[') ++depth;
        else if (c == ')' || c == ']') --depth;
        else if ((c == ',' || c == '}') && depth == 0) break;
    }
    std::string v = h.substr(p, q - p);
    while (!v.empty() && v.back() == ' ') v.pop_back();
    return v;
}

}  // namespace

NpyArray npy_load(const std::string &path) {
    File f(std::fopen(path.c_str(), "rb"));
    if (!f) bad(path, "cannot open");
    unsigned char pre[10];
    if (std::fread(pre, 1, 8, f.get()) != 8 || std::memcmp(pre, "\x93NUMPY", 6) != 0)
        bad(path, "not an npy file");
    const int major = pre[6];
    size_t hlen = 0;
    if (major == 1) {
        unsigned char b[2];
        if (std::fread(b, 1, 2, f.get()) != 2) bad(path, "truncated header");
        hlen = b[0] | (size_t)b[1] << 8;
    } else if (major == 2 || major == 3) {
        unsigned char b[4];
        if (std::fread(b, 1, 4, f.get()) != 4) bad(path, "truncated header");
        hlen = b[0] | (size_t)b[1] << 8 | (size_t)b[2] << 16 | (size_t)b[3] << 24;
    } else {
        bad(path, "unsupported format version " + std::to_string(major));
    }
    if (hlen > (1u << 20)) bad(path, "header too long");
    std::string h(hlen, '\0');
    if (std::fread(&h[0], 1, hlen, f.get()) != hlen) bad(path, "truncated header");

    NpyArray a;
    std::string descr = dict_value(h, "descr", path);
    if (descr.size() < 4 || (descr.front() != '\'' && descr.front() != '"')) bad(path, "bad descr");
    descr = descr.substr(1, descr.size() - 2);
    const char order = descr[0];
    if (order == '>') bad(path, "big-endian data is not supported");
    if (order != '<' && order != '|' && order != '=') bad(path, "bad descr " + descr);
    a.kind = descr[1];
    a.word_size = std::strtoul(descr.c_str() + 2, nullptr, 10);
    if (a.word_size == 0) bad(path, "bad descr " + descr);

    const std::string fo = dict_value(h, "fortran_order", path);
    a.fortran_order = (fo == "True");

    std::string shp = dict_value(h, "shape", path);
    if (shp.size() < 2 || shp.front() != '(' || shp.back() != ')') bad(path, "bad shape");
    shp = shp.substr(1, shp.size() - 2);
    size_t p = 0;
    while (p < shp.size()) {
        while (p < shp.size() && (shp[p] == ' ' || shp[p] == ',')) ++p;
        if (p >= shp.size()) break;
        char *end = nullptr;
        const unsigned long long v = std::strtoull(shp.c_str() + p, &end, 10);
        if (end == shp.c_str() + p) bad(path, "bad shape");
        a.shape.push_back((size_t)v);
        p = (size_t)(end - shp.c_str());
    }

    const size_t n = a.num_vals() * a.word_size;
    a.bytes.reset(new unsigned char[n ? n : 1]);
    const long pos = std::ftell(f.get());
    if (n && (pos < 0 || !read_at(fileno(f.get()), (off_t)pos, a.bytes.get(), n))) bad(path, "truncated data");
    return a;
}

void npy_save(const std::string &path, const std::string &descr, const std::vector<size_t> &shape,
              const void *data, size_t word_size) {
    std::string h = "{'descr': '" + descr + "', 'fortran_order': False, 'shape': (";
    size_t n = 1;
    for (size_t i = 0; i < shape.size(); ++i) {
        h += std::to_string(shape[i]);
        if (shape.size() == 1 || i + 1 < shape.size()) h += ",";
        if (i + 1 < shape.size()) h += " ";
        n *= shape[i];
    }
    h += "), }";
    // pad so that magic(6) + version(2) + len(2) + header is a multiple of 64
    const size_t total = 10 + h.size() + 1;
    h.append((64 - total % 64) % 64, ' ');
    h += '\n';
    File f(std::fopen(path.c_str(), "wb"));
    if (!f) throw std::runtime_error("npy: cannot write " + path);
    const unsigned char pre[10] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0,
                                   (unsigned char)(h.size() & 0xff), (unsigned char)(h.size() >> 8)};
    bool ok = std::fwrite(pre, 1, 10, f.get()) == 10 && std::fwrite(h.data(), 1, h.size(), f.get()) == h.size();
    if (ok && n) ok = std::fwrite(data, word_size, n, f.get()) == n;
    if (!ok) throw std::runtime_error("npy: short write to " + path);
}

}  // namespace sarbp_cli
