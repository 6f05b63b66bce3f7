// platform_data.cpp -- platform_load (PlatformData.cpp:21-256), see
// platform_data.h for the files and the error behaviour.
#include "platform_data.h"

#include <algorithm>
#include <cstdio>
#include <iostream>
#include <stdexcept>
#include <thread>
#include <vector>

#include "npy.h"

namespace sarbp_cli {

namespace {

// out[i] = (float)in[i]; large arrays (the phase history) on several
// threads, each converting one contiguous piece
void downcast(const double *in, float *out, size_t n) {
    const size_t min_piece = 1u << 20;
    const size_t hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t parts = std::max<size_t>(1, std::min<size_t>(std::min<size_t>(hw, 16), n / min_piece));
    auto piece = [&](size_t i) {
        const size_t a = n * i / parts, b = n * (i + 1) / parts;
        for (size_t k = a; k < b; ++k) out[k] = (float)in[k];
    };
    std::vector<std::thread> th;
    for (size_t i = 1; i < parts; ++i) th.emplace_back(piece, i);
    piece(0);
    for (auto &t : th) t.join();
}

bool file_exists(const std::string &path) {
    if (FILE *f = std::fopen(path.c_str(), "rb")) {
        std::fclose(f);
        return true;
    }
    return false;
}

class Loader {
public:
    explicit Loader(std::string dir) : dir_(std::move(dir)) {}

    bool has(const char *name) const { return file_exists(path(name)); }

    NpyArray load(const char *name) const { return npy_load(path(name)); }

    // first element of an f64 file (B, delta_r, delta_t, ...)
    double f64_scalar(const char *name) const {
        NpyArray a = load(name);
        if (a.word_size != sizeof(double) || a.num_vals() < 1) bad_word(name);
        return a.data<double>()[0];
    }

    // int32 or int64 scalar (nsamples, npulses)
    int int_scalar(const char *name) const {
        NpyArray a = load(name);
        if (a.num_vals() < 1) bad_word(name);
        if (a.word_size == sizeof(int)) return a.data<int>()[0];
        if (a.word_size == sizeof(long long)) return (int)a.data<long long>()[0];
        bad_word(name);
    }

    // f32 array, or f64 downcast with the reference's message; shape checked
    // against `dims` when given
    std::vector<float> f32_array(const char *name, const std::vector<size_t> &dims) const {
        NpyArray a = load(name);
        check_shape(a, name, dims);
        std::vector<float> out(a.num_vals());
        if (a.word_size == sizeof(float)) {
            const float *s = a.data<float>();
            std::copy(s, s + out.size(), out.begin());
        } else if (a.word_size == sizeof(double)) {
            std::cout << "PlatformData: downcasting " << name << " from double to float" << std::endl;
            downcast(a.data<double>(), out.data(), out.size());
        } else {
            bad_word(name);
        }
        return out;
    }

    // f32-only array (n_hat)
    std::vector<float> f32_only(const char *name, const std::vector<size_t> &dims) const {
        NpyArray a = load(name);
        check_shape(a, name, dims);
        if (a.word_size != sizeof(float)) bad_word(name);
        const float *s = a.data<float>();
        return std::vector<float>(s, s + a.num_vals());
    }

    // f64-only array (k_y, t)
    std::vector<double> f64_array(const char *name, const std::vector<size_t> &dims) const {
        NpyArray a = load(name);
        check_shape(a, name, dims);
        if (a.word_size != sizeof(double)) bad_word(name);
        const double *s = a.data<double>();
        return std::vector<double>(s, s + a.num_vals());
    }

    // complex64 phase history, or complex128 downcast
    std::vector<float> complex64_array(const char *name, const std::vector<size_t> &dims) const {
        NpyArray a = load(name);
        check_shape(a, name, dims);
        std::vector<float> out(a.num_vals() * 2);
        if (a.word_size == 2 * sizeof(float)) {
            const float *s = a.data<float>();
            std::copy(s, s + out.size(), out.begin());
        } else if (a.word_size == 2 * sizeof(double)) {
            std::cout << "PlatformData: downcasting " << name
                      << " from complex<double> to complex<float>" << std::endl;
            downcast(a.data<double>(), out.data(), out.size());
        } else {
            bad_word(name);
        }
        return out;
    }

private:
    std::string path(const char *name) const { return dir_ + "/" + name + ".npy"; }

    [[noreturn]] static void bad_word(const char *name) {
        throw std::runtime_error(std::string("Bad word size: ") + name);
    }
    static void check_shape(const NpyArray &a, const char *name, const std::vector<size_t> &dims) {
        if (a.shape != dims) throw std::runtime_error(std::string("Bad shape: ") + name);
    }

    std::string dir_;
};

}  // namespace

PlatformData platform_load(const std::string &platform_dir) {
    const Loader L(platform_dir);
    PlatformData pd;
    // scalars, in the reference's order (PlatformData.cpp:24-107)
    if (L.has("B")) pd.B = L.f64_scalar("B");
    if (L.has("B_IF")) {
        NpyArray a = L.load("B_IF");
        if (a.word_size == sizeof(float) && a.num_vals()) {
            pd.B_IF = a.data<float>()[0];
        } else if (a.word_size == sizeof(double) && a.num_vals()) {
            std::cout << "PlatformData: downcasting B_IF from double to float" << std::endl;
            pd.B_IF = (float)a.data<double>()[0];
        } else {
            throw std::runtime_error("Bad word size: B_IF");
        }
    }
    pd.delta_r = L.f64_scalar("delta_r");
    if (L.has("delta_t")) pd.delta_t = L.f64_scalar("delta_t");
    if (L.has("chirprate")) pd.chirprate = L.f64_scalar("chirprate");
    if (L.has("f_0")) pd.f_0 = L.f64_scalar("f_0");
    pd.nsamples = L.int_scalar("nsamples");
    pd.npulses = L.int_scalar("npulses");
    if (L.has("vp")) pd.vp = L.f64_scalar("vp");
    const size_t S = (size_t)pd.nsamples, P = (size_t)pd.npulses;
    // arrays (PlatformData.cpp:110-251)
    if (L.has("freq")) pd.freq = L.f32_array("freq", {S});
    pd.k_r = L.f32_array("k_r", {S});
    if (L.has("k_y")) pd.k_y = L.f64_array("k_y", {P});
    if (L.has("n_hat")) pd.n_hat = L.f32_only("n_hat", {3});
    pd.R_c = L.f32_array("R_c", {3});
    if (L.has("t")) pd.t = L.f64_array("t", {S});
    pd.pos = L.f32_array("pos", {P, 3});
    pd.phs = L.complex64_array("phs", {P, S});
    return pd;
}

}  // namespace sarbp_cli
