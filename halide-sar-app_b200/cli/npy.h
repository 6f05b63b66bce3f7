// npy.h -- reader and writer for NumPy .npy files (format versions 1-3).
//
// The platform loader (PlatformData.cpp:21-256) reads its inputs with cnpy,
// which exposes the element size ("word size"), the shape, the fortran_order
// flag and the raw little-endian payload.  NpyArray keeps the same four
// facts; the loader decides what a word size means, as the reference does.
#pragma once

#include <cstddef>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

namespace sarbp_cli {

struct NpyArray {
    char kind = '?';              // 'f', 'c', 'i', 'u', 'b'
    size_t word_size = 0;         // bytes per element
    bool fortran_order = false;
    std::vector<size_t> shape;
    // num_vals() * word_size bytes of payload (not zero-filled before the read)
    std::unique_ptr<unsigned char[]> bytes;

    size_t num_vals() const {
        size_t n = 1;
        for (size_t s : shape) n *= s;
        return n;
    }
    template <class T>
    const T *data() const { return reinterpret_cast<const T *>(bytes.get()); }
};

// Throws std::runtime_error with the file name on malformed input.
NpyArray npy_load(const std::string &path);

// Writes a C-order little-endian array; descr is e.g. "<f8", "<c16", "|u1".
void npy_save(const std::string &path, const std::string &descr, const std::vector<size_t> &shape,
              const void *data, size_t word_size);

}  // namespace sarbp_cli
