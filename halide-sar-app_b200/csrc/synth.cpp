// synth.cpp -- seeded synthetic stepped-frequency phase histories.
//
// Stand-in for the reference's AFRL / Sandia inputs at the sizes the
// benchmark configurations name.  For pulse p at position pos_p and
// scatterer i at x_i with complex amplitude a_i:
//     D_i(p)    = |pos_p| - |pos_p - x_i|
//     S(f_k, p) = sum_i a_i exp(+j (4 pi f_k / c) D_i(p))
// which focuses under the reference's conventions (forward FFT, then
// exp(-j k_c dr) with dr = |pos| - |r - pos|).  The frequency ramp is
// advanced by a complex rotation and re-seeded exactly every 32 samples.
// Noise is complex Gaussian from a counter-based hash of (seed, index), so
// the output does not depend on the thread count.
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

#include "runner.h"
#include "sarbp_b200.h"

namespace {

constexpr double kC = 299792458.0;
constexpr double kPi = 3.14159265358979323846;

uint64_t mix64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
double unit(uint64_t h) { return ((h >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

template <class F>
void parallel_for(int n, int nthreads, F f) {
    if (nthreads <= 0) nthreads = (int)std::thread::hardware_concurrency();
    if (nthreads < 1) nthreads = 1;
    if (nthreads > n) nthreads = n;
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; ++t)
        th.emplace_back([=] {
            for (int i = t; i < n; i += nthreads) f(i);
        });
    for (auto &x : th) x.join();
}

}  // namespace

extern "C" int sarbp_synth_phase_history(int S, int P, double f0, double df, double R0,
                                         double dep_deg, double span_deg, const double *scat,
                                         int nscat, double snr_db, uint64_t seed, float *phs,
                                         double *pos, double *k_r, int nthreads) {
    if (S < 1 || P < 1 || !phs || !pos || !k_r || (nscat > 0 && !scat) || nscat < 0)
        return sarbp::fail(SARBP_ERR_INVALID, "synth: bad arguments");
    const double dep = dep_deg * kPi / 180.0, span = span_deg * kPi / 180.0;
    for (int k = 0; k < S; ++k) k_r[k] = 4.0 * kPi * (f0 + df * k) / kC;
    for (int p = 0; p < P; ++p) {
        const double phi = (P > 1 ? ((double)p / (P - 1) - 0.5) : 0.0) * span;
        pos[3 * p] = R0 * std::cos(dep) * std::cos(phi);
        pos[3 * p + 1] = R0 * std::cos(dep) * std::sin(phi);
        pos[3 * p + 2] = R0 * std::sin(dep);
    }
    const double dk = 4.0 * kPi * df / kC;
    std::vector<double> acc((size_t)P * S * 2, 0.0);
    std::vector<double> pw(P, 0.0);
    parallel_for(P, nthreads, [&](int p) {
        const double *pp = pos + 3 * p;
        const double np = std::sqrt(pp[0] * pp[0] + pp[1] * pp[1] + pp[2] * pp[2]);
        double *a = acc.data() + (size_t)p * S * 2;
        for (int i = 0; i < nscat; ++i) {
            const double *s = scat + 5 * i;
            const double ex = pp[0] - s[0], ey = pp[1] - s[1], ez = pp[2] - s[2];
            const double D = np - std::sqrt(ex * ex + ey * ey + ez * ez);
            const double rr = std::cos(dk * D), ri = std::sin(dk * D);
            double zr = 0, zi = 0;
            for (int k = 0; k < S; ++k) {
                if ((k & 31) == 0) {
                    const double ph = k_r[k] * D;
                    zr = std::cos(ph);
                    zi = std::sin(ph);
                } else {
                    const double tr = zr * rr - zi * ri;
                    zi = zr * ri + zi * rr;
                    zr = tr;
                }
                a[2 * k] += s[3] * zr - s[4] * zi;
                a[2 * k + 1] += s[3] * zi + s[4] * zr;
            }
        }
        double sp = 0;
        for (int k = 0; k < S; ++k) sp += a[2 * k] * a[2 * k] + a[2 * k + 1] * a[2 * k + 1];
        pw[p] = sp;
    });
    double total = 0;
    for (double v : pw) total += v;
    const double mean_pw = total / ((double)P * S);
    const double sigma = snr_db < 300 ? std::sqrt(mean_pw / std::pow(10.0, snr_db / 10.0) / 2.0) : 0.0;
    parallel_for(P, nthreads, [&](int p) {
        for (int k = 0; k < S; ++k) {
            const size_t idx = (size_t)p * S + k;
            double nr = 0, ni = 0;
            if (sigma > 0) {
                const double u1 = unit(mix64(seed ^ mix64(2 * idx)));
                const double u2 = unit(mix64(seed ^ mix64(2 * idx + 1)));
                const double rad = std::sqrt(-2.0 * std::log(u1));
                nr = sigma * rad * std::cos(2 * kPi * u2);
                ni = sigma * rad * std::sin(2 * kPi * u2);
            }
            phs[2 * idx] = (float)(acc[2 * idx] + nr);
            phs[2 * idx + 1] = (float)(acc[2 * idx + 1] + ni);
        }
    });
    return SARBP_OK;
}
