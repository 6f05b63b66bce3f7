// platform_data.h -- the CLI's platform input directory (PlatformData.h:9-62,
// PlatformData.cpp:21-256).
//
// Required files: delta_r.npy (f64), nsamples.npy / npulses.npy (int32 or
// int64), k_r.npy [S], R_c.npy [3], pos.npy [P, 3] (f32, or f64 downcast to
// f32), phs.npy [P, S] (complex64, or complex128 downcast).  Optional files
// are validated the same way when present: B, delta_t, chirprate, f_0, vp
// (f64), B_IF (f32/f64), freq [S] (f32/f64), k_y [P] (f64), n_hat [3] (f32),
// t [S] (f64).  Errors are std::runtime_error("Bad word size: <name>") or
// ("Bad shape: <name>"), downcasts print "PlatformData: downcasting ..." on
// stdout, as the reference loader does.
#pragma once

#include <optional>
#include <string>
#include <vector>

namespace sarbp_cli {

struct PlatformData {
    std::optional<double> B, delta_t, chirprate, f_0, vp;
    std::optional<float> B_IF;
    double delta_r = 0.0;
    int nsamples = 0;
    int npulses = 0;
    std::optional<std::vector<float>> freq;
    std::vector<float> k_r;                   // [S]
    std::optional<std::vector<double>> k_y;   // [P]
    std::optional<std::vector<float>> n_hat;  // [3]
    std::vector<float> R_c;                   // [3]
    std::optional<std::vector<double>> t;     // [S]
    std::vector<float> pos;                   // [P][3], xyz fastest
    std::vector<float> phs;                   // [P][S][2], interleaved complex64
};

PlatformData platform_load(const std::string &platform_dir);

}  // namespace sarbp_cli
