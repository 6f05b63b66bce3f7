// host_math.cpp -- Taylor window coefficients and the image plane, with the
// types the reference's Halide expressions give them.
#include "host_math.h"

#include <cmath>

#include "sarbp_b200.h"

namespace sarbp {

namespace {
constexpr double kPi = 3.14159265358979323846;

// Halide's Int32 division rounds toward negative infinity.
long long div_floor(long long a, long long b) {
    long long q = a / b;
    if ((a % b != 0) && ((a < 0) != (b < 0))) --q;
    return q;
}
}  // namespace

// signal.h:28-41.  pow(10, S_L/20) has an integer base, which Halide casts
// to f32 (pow and acosh then run in f32); pow(e, 2) with a constant integer
// exponent is a square in e's own type, so the F_m denominator term
// pow(m+1, 2) / pow(r+1, 2) is an Int32 division; the f32 sign
// pow(-1, m+2) multiplies the numerator once per r.  With
// SARBP_TAYLOR_FLOAT the denominator term is a floating-point quotient
// (the published RITSAR window, which the Halide expression restates);
// everything else is the same.  Writes min(count, cap) coefficients into
// out and returns count = n_bar - 1; allocates nothing.
int taylor_coefficients_into(double S_L, double *out, int cap, int mode) {
    const float p10 = std::pow(10.0f, (float)(S_L * (1.0 / 20)));
    const float acosh_f = std::log(p10 + std::sqrt(p10 * p10 - 1.0f));
    const double A = (1.0 / kPi) * (double)acosh_f;
    const double A2 = A * A;
    const int n_bar = (int)(2 * A2 + 0.5) + 1;
    const double nh = (double)n_bar - 0.5;
    const double sigma_p = (double)n_bar / std::sqrt(A2 + nh * nh);
    const double sp2 = sigma_p * sigma_p;
    const int nr = n_bar - 1;
    for (int m = 0; m < nr && m < cap; ++m) {
        const long long m1sq = (long long)(m + 1) * (m + 1);
        const float sgn = std::pow(-1.0f, (float)(m + 2));
        double num = 1.0, den = 1.0;
        for (int r = 0; r < nr; ++r) {
            const double rh = (double)r + 0.5;
            num = num * ((double)sgn * (1.0 - (double)m1sq / sp2 / (A2 + rh * rh)));
            if (r != m) {
                const long long r1sq = (long long)(r + 1) * (r + 1);
                const double q = mode == SARBP_TAYLOR_FLOAT ? (double)m1sq / (double)r1sq
                                                            : (double)div_floor(m1sq, r1sq);
                den = den * (1.0 - q);
            }
        }
        out[m] = num / den;
    }
    return nr > 0 ? nr : 0;
}

std::vector<double> taylor_coefficients(double S_L, int mode) {
    const int n = taylor_coefficients_into(S_L, nullptr, 0, mode);
    std::vector<double> F(n);
    taylor_coefficients_into(S_L, F.data(), n, mode);
    return F;
}

// signal.h:43-48: w(x) = 1 + sum_r F(r) cos(2 pi (r+1) xi), xi = linspace(-1/2, 1/2, num)
void taylor_window(int num, double S_L, double *out, int mode) {
    const std::vector<double> F = taylor_coefficients(S_L, mode);
    const double step = (0.5 - (-0.5)) / (double)(num - 1);
    double wmax = -INFINITY;
    for (int x = 0; x < num; ++x) {
        double xi = -0.5 + (double)x * step;
        xi = std::fmin(std::fmax(xi, -0.5), 0.5);
        double w = 1.0;
        for (size_t r = 0; r < F.size(); ++r) w = w + F[r] * std::cos((2 * kPi) * (double)(r + 1) * xi);
        out[x] = w;
        wmax = std::fmax(wmax, w);
    }
    for (int x = 0; x < num; ++x) out[x] = out[x] / wmax;
}

int ip_upsample(int n) {
    const double l = std::log2((double)n);
    const int r = (l - (int)l) > 0;
    return (int)std::pow(2, (int)(l + r));
}

ImgPlane img_plane_create(int nsamples, int npulses, double delta_r, const float *R_c,
                          const float *n_hat, double res_factor, double aspect, bool upsample) {
    ImgPlane ip;
    ip.nu = upsample ? ip_upsample(nsamples) : nsamples;
    ip.nv = upsample ? ip_upsample(npulses) : npulses;
    ip.d_u = delta_r * res_factor * nsamples / ip.nu;  // ip.h:11-13
    ip.d_v = aspect * ip.d_u;                          // ip.h:15-17
    // img_plane.cpp:12-14: arange(-n/2, 1) * d (Halide floor division)
    ip.u.resize(ip.nu);
    ip.v.resize(ip.nv);
    for (int i = 0; i < ip.nu; ++i) ip.u[i] = (double)(div_floor(-(long long)ip.nu, 2) + i) * ip.d_u;
    for (int i = 0; i < ip.nv; ++i) ip.v[i] = (double)(div_floor(-(long long)ip.nv, 2) + i) * ip.d_v;
    // img_plane.cpp:17-19: 2 pi * linspace(-1/(2d), 1/(2d), n)
    auto kvec = [](int n, double d, std::vector<double> &k) {
        k.resize(n);
        const double a = -1.0 / (2 * d), b = 1.0 / (2 * d);
        const double step = (b - a) / (double)(n - 1);
        for (int i = 0; i < n; ++i) k[i] = (2 * kPi) * std::fmin(std::fmax(a + (double)i * step, a), b);
    };
    kvec(ip.nu, ip.d_u, ip.k_u);
    kvec(ip.nv, ip.d_v, ip.k_v);
    // v_hat = cross(n_hat, R_c) / |.| in f32, then widened (img_plane.cpp:59-61)
    float c[3];
    for (int x = 0; x < 3; ++x)
        c[x] = n_hat[(x + 1) % 3] * R_c[(x + 2) % 3] - n_hat[(x + 2) % 3] * R_c[(x + 1) % 3];
    float s = 0.0f;
    for (int x = 0; x < 3; ++x) s = s + c[x] * c[x];
    const float nrm = std::sqrt(s);
    for (int x = 0; x < 3; ++x) ip.v_hat[x] = (double)(c[x] / nrm);
    // u_hat = cross(v_hat, n_hat) / |.| in f64 (img_plane.cpp:71-73)
    double cd[3];
    for (int x = 0; x < 3; ++x)
        cd[x] = ip.v_hat[(x + 1) % 3] * (double)n_hat[(x + 2) % 3] -
                ip.v_hat[(x + 2) % 3] * (double)n_hat[(x + 1) % 3];
    double sd = 0.0;
    for (int x = 0; x < 3; ++x) sd = sd + cd[x] * cd[x];
    const double nd = std::sqrt(sd);
    for (int x = 0; x < 3; ++x) ip.u_hat[x] = cd[x] / nd;
    return ip;
}

// img_plane.cpp:92-102: pixel i at u[i % nu], v[i / nu]; (0 + u_hat*u) + v_hat*v
void pixel_locs(const ImgPlane &ip, double *out) {
    const long long npix = (long long)ip.nu * ip.nv;
    for (int d = 0; d < 3; ++d) {
        double *o = out + (size_t)d * (size_t)npix;
        for (long long i = 0; i < npix; ++i) {
            const double a = ip.u_hat[d] * ip.u[i % ip.nu];
            const double b = ip.v_hat[d] * ip.v[i / ip.nu];
            o[i] = a + b;
        }
    }
}

}  // namespace sarbp
