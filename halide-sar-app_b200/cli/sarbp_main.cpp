// sarbp -- command-line image formation, flag-for-flag with the reference
// CLI (sarbp.cpp:50-339) for its `-s cuda` schedule.
//
//   sarbp -p DIR -o FILE [-d dBmin] [-D dBmax] [-s cuda] [-t taylor]
//         [-u upsample] [-r res_factor] [-a aspect] [-n iters]
//
// Steps (sarbp.cpp:250-324): platform_load -> img_plane_create ->
// N_fft = 2^(floor(log2(S*upsample)) + 1) -> backprojection (num_iters
// times) -> dB -> u8 -> PNG.  Defaults and argument constraints are the
// reference's (sarbp.cpp:44-49, :141-175).  The schedule names of the
// reference's CPU, distributed and RITSAR variants are recognised and
// refused: this build provides the CUDA path only and has no CPU fallback.
#include <getopt.h>

#include <chrono>
#include <cmath>
#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>

#include "platform_data.h"
#include "png_write.h"
#include "sarbp_b200.h"

using namespace std::chrono;

namespace {

const char kSchedDefault[] = "cuda";
constexpr double kDbMinDefault = 0;
constexpr double kDbMaxDefault = 0;
constexpr int kUpsampleDefault = 6;
constexpr int kTaylorDefault = 20;
constexpr double kResFactorDefault = 1.0;  // ImgPlane.h RES_FACTOR
constexpr double kAspectDefault = 1.0;     // ImgPlane.h ASPECT
const float kNHat[3] = {0.0f, 0.0f, 1.0f};  // ImgPlane.h N_HAT

const char short_options[] = "p:o:d:D:s:t:u:r:a:n:h";
const struct option long_options[] = {
    {"platform-dir", required_argument, nullptr, 'p'},
    {"output", required_argument, nullptr, 'o'},
    {"db-min", required_argument, nullptr, 'd'},
    {"db-max", required_argument, nullptr, 'D'},
    {"schedule", required_argument, nullptr, 's'},
    {"taylor", required_argument, nullptr, 't'},
    {"upsample", required_argument, nullptr, 'u'},
    {"res-factor", required_argument, nullptr, 'r'},
    {"aspect", required_argument, nullptr, 'a'},
    {"num-iters", required_argument, nullptr, 'n'},
    {"help", no_argument, nullptr, 'h'},
    {nullptr, 0, nullptr, 0}};

void print_usage(const std::string &prog, std::ostream &os) {
    os << "Usage: " << prog << " -p DIR -o FILE [OPTION]...\n"
       << "Options:\n"
       << "  -p, --platform-dir=DIR  Platform input directory\n"
       << "  -o, --output=FILE       Output image file (PNG)\n"
       << "  -d, --db-min=REAL       Output image min dB\n"
       << "                          Default: " << kDbMinDefault << "\n"
       << "  -D, --db-max=REAL       Output image max dB\n"
       << "                          Default: " << kDbMaxDefault << "\n"
       << "  -s, --schedule=NAME     cuda (B200 kernels)\n"
       << "                          Default: " << kSchedDefault << "\n"
       << "  -t, --taylor=INT        Taylor count\n"
       << "                          Default: " << kTaylorDefault << "\n"
       << "  -u, --upsample=INT      Upsample factor\n"
       << "                          Default: " << kUpsampleDefault << "\n"
       << "  -r, --res-factor=REAL   Image res in units of theoretical resolution size\n"
       << "                          Default: " << kResFactorDefault << "\n"
       << "  -a, --aspect=REAL       Aspect ratio of range to cross range\n"
       << "                          Default: " << kAspectDefault << "\n"
       << "  -n, --num-iters=INT     Number of backprojection iterations\n"
       << "                          Default: 1\n"
       << "  -h, --help              Print this message and exit" << std::endl;
}

long long ms_since(steady_clock::time_point t0) {
    return duration_cast<milliseconds>(steady_clock::now() - t0).count();
}

bool known_other_schedule(const std::string &s) {
    for (const char *n : {"cpu", "cpu_distributed", "cuda_distributed", "ritsar", "ritsar-s",
                          "ritsar-p", "ritsar-vp", "auto-m16"})
        if (s == n) return true;
    return false;
}

int run(int argc, char **argv) {
    std::string platform_dir, output_png, bp_sched = kSchedDefault;
    int taylor = kTaylorDefault, upsample = kUpsampleDefault;
    double dB_min = kDbMinDefault, dB_max = kDbMaxDefault;
    double res_factor = kResFactorDefault, aspect = kAspectDefault;
    unsigned num_iters = 1;
    for (;;) {
        const int c = getopt_long(argc, argv, short_options, long_options, nullptr);
        if (c == -1) break;
        switch (c) {
            case 'p': platform_dir = optarg; break;
            case 'o': output_png = optarg; break;
            case 'd': dB_min = std::atof(optarg); break;
            case 'D': dB_max = std::atof(optarg); break;
            case 's': bp_sched = optarg; break;
            case 't': taylor = std::atoi(optarg); break;
            case 'u': upsample = std::atoi(optarg); break;
            case 'r': res_factor = std::atof(optarg); break;
            case 'a': aspect = std::atof(optarg); break;
            case 'n': num_iters = (unsigned)std::atoi(optarg); break;
            case 'h': print_usage(argv[0], std::cout); return 0;
            default: print_usage(argv[0], std::cerr); return EXIT_FAILURE;
        }
    }
    auto constraint = [&](bool ok, const char *what) {
        if (!ok) {
            std::cerr << what << std::endl;
            print_usage(argv[0], std::cerr);
        }
        return ok;
    };
    if (!constraint(!platform_dir.empty() && !output_png.empty(), "Missing required parameters") ||
        !constraint(dB_min < dB_max, "Constraint failed: dB_min < dB_max") ||
        !constraint(taylor >= 1, "Constraint failed: taylor >= 1") ||
        !constraint(upsample >= 1, "Constraint failed: upsample >= 1") ||
        !constraint(res_factor > 0, "Constraint failed: res-factor > 0") ||
        !constraint(aspect > 0, "Constraint failed: aspect > 0"))
        return EXIT_FAILURE;
    if (bp_sched == "cuda") {
        std::cout << "Using schedule with CUDA" << std::endl;
    } else if (known_other_schedule(bp_sched)) {
        std::cerr << "Schedule not provided by this build: " << bp_sched << " (use cuda)" << std::endl;
        return EXIT_FAILURE;
    } else {
        std::cerr << "Unknown schedule: " << bp_sched << std::endl;
        print_usage(argv[0], std::cerr);
        return EXIT_FAILURE;
    }

    auto t0 = steady_clock::now();
    sarbp_cli::PlatformData pd = sarbp_cli::platform_load(platform_dir);
    std::cout << "Loaded platform data in " << ms_since(t0) << " ms" << std::endl;
    std::cout << "Number of pulses: " << pd.npulses << std::endl;
    std::cout << "Pulse sample size: " << pd.nsamples << std::endl;

    const float *n_hat = pd.n_hat ? pd.n_hat->data() : kNHat;
    t0 = steady_clock::now();
    int nu = 0, nv = 0;
    int rv = sarbp_img_plane_dims(pd.nsamples, pd.npulses, upsample, &nu, &nv);
    if (rv) {
        std::cerr << sarbp_last_error() << std::endl;
        return rv;
    }
    std::vector<double> u(nu), v(nv), k_u(nu), k_v(nv);
    double d_u = 0, d_v = 0, u_hat[3], v_hat[3];
    rv = sarbp_img_plane(pd.nsamples, pd.npulses, pd.delta_r, pd.R_c.data(), n_hat, res_factor, aspect,
                         upsample, &d_u, &d_v, u.data(), v.data(), k_u.data(), k_v.data(), u_hat, v_hat,
                         nullptr);
    if (rv) {
        std::cerr << sarbp_last_error() << std::endl;
        return rv;
    }
    std::cout << "Computed image plane parameters in " << ms_since(t0) << " ms" << std::endl;
    std::cout << "X length: " << nu << std::endl;
    std::cout << "Y length: " << nv << std::endl;

    // FFT width (sarbp.cpp:258)
    const int N_fft = (int)std::pow(2, (int)std::log2(pd.nsamples * upsample) + 1);

    sarbp_ctx *ctx = nullptr;
    if ((rv = sarbp_ctx_create(0, &ctx)) != 0) {
        std::cerr << sarbp_last_error() << std::endl;
        return rv;
    }
    struct CtxGuard {
        sarbp_ctx *c;
        ~CtxGuard() { sarbp_ctx_destroy(c); }
    } guard{ctx};

    std::vector<double> img((size_t)nu * nv * 2);
    for (unsigned i = 1; i <= num_iters; ++i) {
        // the reference's progress lines verbatim (sarbp.cpp:275,279), so
        // that tools reading its output keep working
        std::cout << "(" << i << ") Halide backprojection start " << std::endl;
        t0 = steady_clock::now();
        rv = sarbp_backprojection_plane(ctx, pd.phs.data(), pd.nsamples, pd.npulses, pd.k_r.data(), taylor,
                                        N_fft, pd.delta_r, u.data(), nu, v.data(), nv, u_hat, v_hat,
                                        pd.pos.data(), img.data(), nullptr);
        std::cout << "(" << i << ") Halide backprojection returned " << rv << " in " << ms_since(t0) << " ms"
                  << std::endl;
        if (rv != 0) {
            std::cerr << sarbp_last_error() << std::endl;
            return rv;
        }
    }

    std::vector<double> dB((size_t)nu * nv);
    std::cout << "Halide dB conversion start" << std::endl;
    t0 = steady_clock::now();
    rv = sarbp_img_output_to_dB(ctx, img.data(), nu, nv, dB.data());
    std::cout << "Halide dB conversion returned " << rv << " in " << ms_since(t0) << " ms" << std::endl;
    if (rv != 0) {
        std::cerr << sarbp_last_error() << std::endl;
        return rv;
    }

    std::vector<uint8_t> u8((size_t)nu * nv);
    std::cout << "Halide PNG production start" << std::endl;
    t0 = steady_clock::now();
    rv = sarbp_img_output_u8(ctx, dB.data(), nu, nv, dB_min, dB_max, u8.data());
    std::cout << "Halide PNG production returned " << rv << " in " << ms_since(t0) << " ms" << std::endl;
    if (rv != 0) {
        std::cerr << sarbp_last_error() << std::endl;
        return rv;
    }
    t0 = steady_clock::now();
    sarbp_cli::png_write_gray8(output_png, u8.data(), nu, nv);
    std::cout << "Wrote " << output_png << " in " << ms_since(t0) << " ms" << std::endl;
    return 0;
}

}  // namespace

int main(int argc, char **argv) {
    try {
        return run(argc, argv);
    } catch (const std::exception &e) {
        // the reference lets loader exceptions terminate the process
        std::cerr << "sarbp: " << e.what() << std::endl;
        return EXIT_FAILURE;
    }
}
