/*
 * sarbp_oracle.c -- CPU oracle for the SAR backprojection hot path.
 *
 * TEST INFRASTRUCTURE ONLY (parity checker and timed CPU baseline); the
 * product library never links this file.  See sarbp_oracle.h for the parity
 * status.  Every function cites the reference file:line it restates
 * (paths relative to the ISI-apex/halide-sar-app project root).
 *
 * Built with -ffp-contract=off so that every f32/f64 operation rounds
 * separately, which pins the op order the reference source writes.
 */
#define _GNU_SOURCE
#include "sarbp_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

static void set_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
}

/* Halide integer division rounds toward negative infinity for a positive
 * divisor (Halide IROperator semantics); C truncates toward zero. */
static long long floordiv(long long a, long long b) {
    long long q = a / b;
    if ((a % b != 0) && ((a < 0) != (b < 0))) q -= 1;
    return q;
}
static long long floormod(long long a, long long b) {
    long long m = a % b;
    if (m < 0) m += (b < 0 ? -b : b);
    return m;
}

/* ip.h:5-9 */
int orc_ip_upsample(int n) {
    double l = log2((double)n);
    int r = (l - (int)l) > 0;
    return (int)pow(2, (int)(l + r));
}

/* util.h:83-87 -- clamp(start + x*step, start, stop), step=(stop-start)/(num-1) */
void orc_linspace_f32(float start, float stop, int num, float *out) {
    float step = (stop - start) / (float)(num - 1);
    for (int x = 0; x < num; x++) {
        float v = start + (float)x * step;
        if (v < start) v = start;
        if (v > stop) v = stop;
        out[x] = v;
    }
}
void orc_linspace_f64(double start, double stop, int num, double *out) {
    double step = (stop - start) / (double)(num - 1);
    for (int x = 0; x < num; x++) {
        double v = start + (double)x * step;
        if (v < start) v = start;
        if (v > stop) v = stop;
        out[x] = v;
    }
}

/* util.h:89-91 */
void orc_arange_f32(float start, float step, int n, float *out) {
    for (int x = 0; x < n; x++) out[x] = start + (float)x * step;
}

/* util.h:63-65 -- sqrt(sum(x*x)), sequential sum from 0 */
float orc_norm_f32(const float *in, int n) {
    float s = 0.0f;
    for (int i = 0; i < n; i++) s = s + in[i] * in[i];
    return sqrtf(s);
}

/* util.h:21-29 */
void orc_cross3_f32(const float *a, const float *b, float *out) {
    for (int x = 0; x < 3; x++)
        out[x] = a[(x + 1) % 3] * b[(x + 2) % 3] - a[(x + 2) % 3] * b[(x + 1) % 3];
}

/* util.h:67-71 on a float buffer: (x*x + y*y) + z*z, then sqrt (f32) */
float orc_norm3d_f32(const float *p) {
    float s = p[0] * p[0];
    s = s + p[1] * p[1];
    s = s + p[2] * p[2];
    return sqrtf(s);
}

/*
 * Taylor window, signal.h:23-49, evaluated with the types Halide gives the
 * expressions:
 *  - pow(10, S_L/20) has an integer base, so Halide casts it to f32 and
 *    evaluates pow and acosh in f32 (signal.h:28); A is then f64.
 *  - pow(e, 2) with a constant integer exponent is a plain square in the
 *    type of e, so pow(x+1, 2) / pow(r+1, 2) is an Int32 division
 *    (Halide rounds it toward -inf) in F_m_den (signal.h:40).
 *  - the sign pow(-1, x+2) is an f32 pow and multiplies F_m_num once per
 *    r, i.e. n_bar-1 times (signal.h:39).
 *  - xi = linspace(-0.5, 0.5, num) with no factor 2 inside the cosine
 *    (signal.h:27,45); the result is divided by its maximum (signal.h:48).
 */
void orc_taylor(int num, double S_L, double *out) { orc_taylor_mode(num, S_L, 0, out); }

/* The same window with the F_m denominator quotient (m+1)^2/(r+1)^2 taken
 * in f64 when float_den is non-zero (the float-division variant; the
 * published RITSAR taylor() that signal.h restates divides in floating
 * point). */
void orc_taylor_mode(int num, double S_L, int float_den, double *out) {
    float p10 = powf(10.0f, (float)(S_L * (1.0 / 20)));
    float ach = logf(p10 + sqrtf(p10 * p10 - 1.0f)); /* acosh_f32 */
    double A = (1.0 / (double)M_PI) * (double)ach;
    double A2 = A * A;
    int n_bar = (int)(2 * A2 + 0.5) + 1;
    double nbh = (double)n_bar - 0.5;
    double sigma_p = (double)n_bar / sqrt(A2 + nbh * nbh);
    double sp2 = sigma_p * sigma_p;
    int nr = n_bar - 1;
    double *F = (double *)calloc((size_t)(nr > 0 ? nr : 1), sizeof(double));
    for (int m = 0; m < nr; m++) {
        double fnum = 1.0, fden = 1.0;
        int m1sq = (m + 1) * (m + 1);
        float sgn = powf(-1.0f, (float)(m + 2));
        for (int r = 0; r < nr; r++) {
            double rh = (double)r + 0.5;
            fnum = fnum * ((double)sgn * (1.0 - (double)m1sq / sp2 / (A2 + rh * rh)));
            if (m != r) {
                int r1sq = (r + 1) * (r + 1);
                double q = float_den ? (double)m1sq / (double)r1sq : (double)floordiv(m1sq, r1sq);
                fden = fden * (1.0 - q);
            }
        }
        F[m] = fnum / fden;
    }
    double step = (0.5 - (-0.5)) / (double)(num - 1);
    double wmax = -INFINITY;
    for (int x = 0; x < num; x++) {
        double xi = -0.5 + (double)x * step;
        if (xi < -0.5) xi = -0.5;
        if (xi > 0.5) xi = 0.5;
        double w = 1.0;
        for (int r = 0; r < nr; r++)
            w = w + F[r] * cos((2 * (double)M_PI) * (double)(r + 1) * xi);
        out[x] = w;
        if (w > wmax) wmax = w;
    }
    for (int x = 0; x < num; x++) out[x] = out[x] / wmax;
    free(F);
}

/* img_plane.cpp:22-27 -- cross(a,b) / norm(cross(a,b)) */
static void ip_hat_f32(const float *a, const float *b, double *out) {
    float c[3];
    orc_cross3_f32(a, b, c);
    float n = orc_norm_f32(c, 3);
    for (int i = 0; i < 3; i++) out[i] = (double)(c[i] / n);
}
static void ip_hat_f64(const double *a, const double *b, double *out) {
    double c[3];
    for (int x = 0; x < 3; x++)
        c[x] = a[(x + 1) % 3] * b[(x + 2) % 3] - a[(x + 2) % 3] * b[(x + 1) % 3];
    double s = 0.0;
    for (int i = 0; i < 3; i++) s = s + c[i] * c[i];
    double n = sqrt(s);
    for (int i = 0; i < 3; i++) out[i] = c[i] / n;
}

/* img_plane.cpp:92-102 -- pixel i: u index i % nu, v index i / nu */
void orc_pixel_locs(const double *u, int nu, const double *v, int nv,
                    const double *u_hat, const double *v_hat, double *out) {
    long long npix = (long long)nu * nv;
    for (int d = 0; d < 3; d++) {
        double *o = out + (size_t)d * (size_t)npix;
        for (long long i = 0; i < npix; i++) {
            double s = 0.0;
            s = s + u_hat[d] * u[i % nu];
            s = s + v_hat[d] * v[i / nu];
            o[i] = s;
        }
    }
}

/* ImgPlane.cpp:16-63 with ip.h and img_plane.cpp:11-19 */
void orc_img_plane(int nsamples, int npulses, double delta_r, const float *R_c,
                   const float *n_hat, double res_factor, double aspect,
                   int upsample, int *nu_out, int *nv_out, double *d_u_out,
                   double *d_v_out, double *u, double *v, double *k_u,
                   double *k_v, double *u_hat, double *v_hat,
                   double *pixel_locs) {
    int nu, nv;
    if (upsample) {
        nu = orc_ip_upsample(nsamples);
        nv = orc_ip_upsample(npulses);
    } else {
        nu = nsamples;
        nv = npulses;
    }
    double d_u = delta_r * res_factor * nsamples / nu; /* ip.h:11-13 */
    double d_v = aspect * d_u;                          /* ip.h:15-17 */
    *nu_out = nu;
    *nv_out = nv;
    *d_u_out = d_u;
    *d_v_out = d_v;
    if (!u) return;
    /* arange(-n/2, 1, x) * d with Halide's floor division for -n/2 */
    for (int i = 0; i < nu; i++) u[i] = (double)(floordiv(-(long long)nu, 2) + i) * d_u;
    for (int i = 0; i < nv; i++) v[i] = (double)(floordiv(-(long long)nv, 2) + i) * d_v;
    /* 2*pi * linspace(-1/(2d), 1/(2d), n) */
    orc_linspace_f64(-1.0 / (2 * d_u), 1.0 / (2 * d_u), nu, k_u);
    for (int i = 0; i < nu; i++) k_u[i] = (2 * M_PI) * k_u[i];
    orc_linspace_f64(-1.0 / (2 * d_v), 1.0 / (2 * d_v), nv, k_v);
    for (int i = 0; i < nv; i++) k_v[i] = (2 * M_PI) * k_v[i];
    /* v_hat in f32 (img_plane.cpp:59-61), u_hat in f64 (img_plane.cpp:71-73) */
    ip_hat_f32(n_hat, R_c, v_hat);
    double n_hat64[3] = {(double)n_hat[0], (double)n_hat[1], (double)n_hat[2]};
    ip_hat_f64(v_hat, n_hat64, u_hat);
    if (pixel_locs) orc_pixel_locs(u, nu, v, nv, u_hat, v_hat, pixel_locs);
}

/* ---------------------------------------------------------------------- */
/* Forward unnormalised DFT, X[k] = sum_n x[n] exp(-2*pi*i*n*k/N)
 * (dft.cpp:26, FFTW_FORWARD).  Iterative radix-2 with directly evaluated
 * twiddles; plain O(N^2) sum when N is not a power of two. */
static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

void orc_fft_forward(double *x, int n) {
    if (n <= 1) return;
    if (!is_pow2(n)) {
        double *tmp = (double *)malloc(sizeof(double) * 2 * (size_t)n);
        for (int k = 0; k < n; k++) {
            double sr = 0, si = 0;
            for (int j = 0; j < n; j++) {
                long long e = ((long long)j * k) % n;
                double a = -2.0 * M_PI * (double)e / (double)n;
                double c = cos(a), s = sin(a);
                sr += x[2 * j] * c - x[2 * j + 1] * s;
                si += x[2 * j] * s + x[2 * j + 1] * c;
            }
            tmp[2 * k] = sr;
            tmp[2 * k + 1] = si;
        }
        memcpy(x, tmp, sizeof(double) * 2 * (size_t)n);
        free(tmp);
        return;
    }
    /* bit reversal */
    for (int i = 1, j = 0; i < n; i++) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double tr = x[2 * i], ti = x[2 * i + 1];
            x[2 * i] = x[2 * j];
            x[2 * i + 1] = x[2 * j + 1];
            x[2 * j] = tr;
            x[2 * j + 1] = ti;
        }
    }
    double *tw = (double *)malloc(sizeof(double) * (size_t)n); /* n/2 complex */
    for (int k = 0; k < n / 2; k++) {
        double a = -2.0 * M_PI * (double)k / (double)n;
        tw[2 * k] = cos(a);
        tw[2 * k + 1] = sin(a);
    }
    for (int len = 2; len <= n; len <<= 1) {
        int half = len >> 1, stride = n / len;
        for (int i = 0; i < n; i += len) {
            for (int k = 0; k < half; k++) {
                double wr = tw[2 * k * stride], wi = tw[2 * k * stride + 1];
                double *a = x + 2 * (i + k), *b = x + 2 * (i + k + half);
                double br = b[0] * wr - b[1] * wi;
                double bi = b[0] * wi + b[1] * wr;
                b[0] = a[0] - br;
                b[1] = a[1] - bi;
                a[0] = a[0] + br;
                a[1] = a[1] + bi;
            }
        }
    }
    free(tw);
}

/*
 * Range compression, backprojection.cpp:79-104:
 *   win(s,p)      = taylor_S(s) * taylor_P(p)                  (:80-82)
 *   filt(s)       = |k_r(s)| (f32)                               (:85)
 *   phs_filt(s,p) = (phs(s,p) * filt(s)) * win(s,p)             (:88-90)
 *   phs_pad       = pad to N_fft with leading (N_fft-S)/2 zeros  (:93-95, signal_complex.h:10-21)
 *   fftsh         = fftshift over BOTH axes by ceil(extent/2)     (:98, signal_complex.h:24-29)
 *   dft           = forward FFT of each pulse row                 (:101, dft.cpp:40-79)
 *   Q             = fftshift over both axes again                 (:104)
 * The pulse axis is shifted twice by ceil(P/2); for odd P that is a
 * rotation by one row, so Q row p is built from phase-history row
 * (p + 2*ceil(P/2)) mod P with that row's pulse window.
 */
int orc_range_compress(const float *phs, int S, int P, const double *k_r,
                       int taylor_s_l, int N, int mode, double *Q,
                       int nthreads) {
    if (S <= 0 || P <= 0 || N <= 0) return -1;
    double *wS = (double *)malloc(sizeof(double) * (size_t)S);
    double *wP = (double *)malloc(sizeof(double) * (size_t)P);
    int float_den = (mode & ORC_TAYLOR_FLOAT) != 0;
    mode &= ~ORC_TAYLOR_FLOAT;
    orc_taylor_mode(S, (double)taylor_s_l, float_den, wS);
    orc_taylor_mode(P, (double)taylor_s_l, float_den, wP);
    long long x_pad = floordiv((long long)N - S, 2);
    long long xm = N / 2 + N % 2;
    long long pm = P / 2 + P % 2;
    set_threads(nthreads);
#pragma omp parallel
    {
        double *row = (double *)malloc(sizeof(double) * 2 * (size_t)N);
#pragma omp for schedule(dynamic, 4)
        for (int p = 0; p < P; p++) {
            int src = (int)floormod((long long)p + 2 * pm, P);
            const float *ph = phs + (size_t)src * 2 * (size_t)S;
            for (int x = 0; x < N; x++) {
                long long xs = floormod((long long)x + xm, N); /* fftsh sample index */
                double re = 0.0, im = 0.0;
                if (!(xs < x_pad || xs >= S + x_pad)) {
                    long long s = xs - x_pad;
                    if (s < 0) s = 0;
                    if (s > S - 1) s = S - 1;
                    double w = wS[s] * wP[src];
                    if (mode == ORC_MODE_REF) {
                        float filt = fabsf((float)k_r[s]);
                        float fr = ph[2 * s] * filt;
                        float fi = ph[2 * s + 1] * filt;
                        re = (double)fr * w;
                        im = (double)fi * w;
                    } else {
                        double filt = fabs(k_r[s]);
                        re = ((double)ph[2 * s] * filt) * w;
                        im = ((double)ph[2 * s + 1] * filt) * w;
                    }
                }
                row[2 * x] = re;
                row[2 * x + 1] = im;
            }
            orc_fft_forward(row, N);
            double *q = Q + (size_t)p * 2 * (size_t)N;
            for (int x = 0; x < N; x++) {
                long long xs = floormod((long long)x + xm, N);
                q[2 * x] = row[2 * xs];
                q[2 * x + 1] = row[2 * xs + 1];
            }
        }
        free(row);
    }
    free(wS);
    free(wP);
    return 0;
}

/* backprojection.cpp:108 with util.h:67-71 */
void orc_norm_r0(const double *pos, int P, int mode, double *nr0) {
    for (int p = 0; p < P; p++) {
        if (mode == ORC_MODE_REF) {
            float f[3] = {(float)pos[3 * p], (float)pos[3 * p + 1], (float)pos[3 * p + 2]};
            nr0[p] = (double)orc_norm3d_f32(f);
        } else {
            const double *q = pos + 3 * p;
            double s = q[0] * q[0];
            s = s + q[1] * q[1];
            s = s + q[2] * q[2];
            nr0[p] = sqrt(s);
        }
    }
}

static inline double dr_at(const double *pp, double nr0, double rx, double ry,
                           double rz) {
    /* rr0 = r - pos (pos promoted to f64), norm3d in f64 (:111-117) */
    double dx = rx - pp[0], dy = ry - pp[1], dz = rz - pp[2];
    double s = dx * dx;
    s = s + dy * dy;
    s = s + dz * dz;
    return nr0 - sqrt(s);
}

/*
 * The interp of backprojection.cpp:52-65 on a linspace axis: t = (x - lsa)
 * / lsr, lower index floor(t), both indices clamped to [0, n-1] and the
 * offset to [0, 1], lerp of the complex samples q ([n][2]).
 */
static inline void interp_at(const double *q, long long n, double t, double *qr, double *qi) {
    if (!(t > -1e9)) t = -1e9; /* keep the int conversion defined */
    if (t > 1e9) t = 1e9;
    double fl = floor(t);
    long long l = (long long)fl;
    double fr = t - (double)l;
    long long cl = l < 0 ? 0 : (l > n - 1 ? n - 1 : l);
    long long cu = l + 1 < 0 ? 0 : (l + 1 > n - 1 ? n - 1 : l + 1);
    if (fr < 0.0) fr = 0.0;
    if (fr > 1.0) fr = 1.0;
    *qr = q[2 * cl] * (1.0 - fr) + q[2 * cu] * fr;
    *qi = q[2 * cl + 1] * (1.0 - fr) + q[2 * cu + 1] * fr;
}

void orc_interp_linspace(const double *xs, long long nx, double lsa, double lsb, int lsn,
                         const double *q, double *out) {
    double lsr = (lsb - lsa) / (double)(lsn - 1);
    for (long long i = 0; i < nx; i++)
        interp_at(q, lsn, (xs[i] - lsa) / lsr, &out[2 * i], &out[2 * i + 1]);
}

/*
 * backprojection.cpp:110-138 and the interp of :52-65:
 *   dr    = norm_r0(p) - |r(pix) - pos(p)|
 *   t     = (dr - lsa) / lsr, lsa = floor(-S*dr/2), lsb = floor(S*dr/2),
 *           lsr = (lsb - lsa) / (N_fft - 1)
 *   l     = floor(t); indices clamped to [0, N_fft-1], frac to [0, 1]
 *   Q_hat = lerp(Q[l], Q[l+1], frac) = Q[l]*(1-frac) + Q[l+1]*frac
 *   img   = sum_p Q_hat * exp(-j*k_c*dr),  k_c = k_r[S/2]
 *   out(x,y) = img[nu*(nv-y-1) + x] * exp(+j*k_c*dr(pix, P/2))
 */
int orc_backproject(const double *Q, int P, int N, int S, double delta_r,
                    const double *k_r, const double *pos, const double *r,
                    int nu, int nv, const long long *out_idx, long long n_out,
                    int mode, double *out, int nthreads) {
    if (P <= 0 || N <= 0 || nu <= 0 || nv <= 0) return -1;
    long long npix = (long long)nu * nv;
    if (!out_idx) n_out = npix;
    double *pos_e = (double *)malloc(sizeof(double) * 3 * (size_t)P);
    double *nr0 = (double *)malloc(sizeof(double) * (size_t)P);
    for (int i = 0; i < 3 * P; i++)
        pos_e[i] = (mode == ORC_MODE_REF) ? (double)(float)pos[i] : pos[i];
    orc_norm_r0(pos_e, P, mode, nr0);
    double k_c = (mode == ORC_MODE_REF) ? (double)(float)k_r[S / 2] : k_r[S / 2];
    double lsa = floor((double)(-S) * delta_r / 2);
    double lsb = floor((double)S * delta_r / 2);
    double lsr = (lsb - lsa) / (double)(N - 1);
    const double *rx = r, *ry = r + npix, *rz = r + 2 * npix;
    long long ngroups = (n_out + 3) / 4;
    set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
    for (long long g = 0; g < ngroups; g++) {
        long long pix[4];
        int nv4 = 0;
        double ar[4] = {0, 0, 0, 0}, ai[4] = {0, 0, 0, 0};
        for (int k = 0; k < 4; k++) {
            long long o = g * 4 + k;
            if (o >= n_out) break;
            long long oi = out_idx ? out_idx[o] : o;
            long long x = oi % nu, y = oi / nu;
            pix[k] = (long long)nu * (nv - y - 1) + x;
            nv4++;
        }
        for (int p = 0; p < P; p++) {
            const double *pp = pos_e + 3 * p;
            const double *q = Q + (size_t)p * 2 * (size_t)N;
            for (int k = 0; k < nv4; k++) {
                long long i = pix[k];
                double dr = dr_at(pp, nr0[p], rx[i], ry[i], rz[i]);
                double qr, qi;
                interp_at(q, N, (dr - lsa) / lsr, &qr, &qi);
                double ph = (-k_c) * dr;
                double s, c;
                sincos(ph, &s, &c);
                ar[k] = ar[k] + (qr * c - qi * s);
                ai[k] = ai[k] + (qr * s + qi * c);
            }
        }
        const double *pm = pos_e + 3 * (P / 2);
        for (int k = 0; k < nv4; k++) {
            long long i = pix[k];
            double dr = dr_at(pm, nr0[P / 2], rx[i], ry[i], rz[i]);
            double s, c;
            sincos(k_c * dr, &s, &c);
            long long o = g * 4 + k;
            out[2 * o] = ar[k] * c - ai[k] * s;
            out[2 * o + 1] = ar[k] * s + ai[k] * c;
        }
    }
    free(pos_e);
    free(nr0);
    return 0;
}

int orc_backprojection(const float *phs, int S, int P, const double *k_r,
                       int taylor_s_l, int N, double delta_r,
                       const double *pos, const double *r, int nu, int nv,
                       int mode, double *out_img, int nthreads) {
    double *Q = (double *)malloc(sizeof(double) * 2 * (size_t)P * (size_t)N);
    if (!Q) return -2;
    int rc = orc_range_compress(phs, S, P, k_r, taylor_s_l, N, mode, Q, nthreads);
    mode &= ~ORC_TAYLOR_FLOAT;
    if (rc == 0)
        rc = orc_backproject(Q, P, N, S, delta_r, k_r, pos, r, nu, nv, NULL, 0,
                             mode, out_img, nthreads);
    free(Q);
    return rc;
}

/* img_output.cpp:18-34: m = max|z|; dB = 10 * log(|z|/m) / log(10), where
 * log(Expr(10)) has an integer argument and is therefore an f32 log
 * (util.h:56-58). */
void orc_img_output_to_dB(const double *img, long long npix, double *dB) {
    double m = -INFINITY;
    for (long long i = 0; i < npix; i++) {
        double a = sqrt(img[2 * i] * img[2 * i] + img[2 * i + 1] * img[2 * i + 1]);
        if (a > m) m = a;
    }
    double ln10 = (double)logf(10.0f);
    for (long long i = 0; i < npix; i++) {
        double a = sqrt(img[2 * i] * img[2 * i] + img[2 * i + 1] * img[2 * i + 1]);
        dB[i] = 10.0 * (log(a / m) / ln10);
    }
}

/* img_output.cpp:41-52 with signal.h:55-57 and util.h:13-15:
 * u8(clamp((clamp(dB,min,max) - min)/(max - min) * 255, 0, 255)) */
void orc_img_output_u8(const double *dB, long long npix, double dB_min,
                       double dB_max, unsigned char *out) {
    for (long long i = 0; i < npix; i++) {
        double v = dB[i];
        if (v != v) v = dB_min; /* NaN (all-zero image): lowest level */
        v = v < dB_min ? dB_min : v; /* clamp = min(max(v, lo), hi) */
        v = v > dB_max ? dB_max : v;
        double n = (v - dB_min) / (dB_max - dB_min) * 255.0;
        n = n < 0.0 ? 0.0 : n;
        n = n > 255.0 ? 255.0 : n;
        out[i] = (unsigned char)n;
    }
}

/*
 * Seeded synthetic stepped-frequency phase history for the CPU reference
 * arm of the benchmark (it stands in for the reference's AFRL / Sandia
 * inputs at the configurations' sizes): for pulse p at pos_p (a circular
 * arc of P positions at slant range R0, depression dep_deg, azimuth span
 * span_deg) and scatterer i (x, y, z, Re a, Im a),
 *     S(f_k, p) = sum_i a_i exp(+j (4 pi f_k / c)(|pos_p| - |pos_p - x_i|))
 * plus complex Gaussian noise at snr_db (none at 300 dB and above) from a
 * counter-based hash of (seed, sample index).  The frequency ramp advances
 * by a complex rotation and is re-seeded every 32 samples.  The same
 * formulas, in the same order, as the product library's generator, so both
 * arms of the benchmark see the same data.
 */
static unsigned long long orc_mix64(unsigned long long z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
static double orc_unit(unsigned long long h) { return ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

int orc_synth_phase_history(int S, int P, double f0, double df, double R0, double dep_deg,
                            double span_deg, const double *scat, int nscat, double snr_db,
                            unsigned long long seed, float *phs, double *pos, double *k_r,
                            int nthreads) {
    const double c = 299792458.0, pi = 3.14159265358979323846;
    if (S < 1 || P < 1 || !phs || !pos || !k_r || nscat < 0 || (nscat > 0 && !scat)) return -1;
    const double dep = dep_deg * pi / 180.0, span = span_deg * pi / 180.0;
    for (int k = 0; k < S; k++) k_r[k] = 4.0 * pi * (f0 + df * k) / c;
    for (int p = 0; p < P; p++) {
        double phi = (P > 1 ? ((double)p / (P - 1) - 0.5) : 0.0) * span;
        pos[3 * p] = R0 * cos(dep) * cos(phi);
        pos[3 * p + 1] = R0 * cos(dep) * sin(phi);
        pos[3 * p + 2] = R0 * sin(dep);
    }
    const double dk = 4.0 * pi * df / c;
    double *acc = (double *)calloc((size_t)P * S * 2, sizeof(double));
    double *pw = (double *)calloc((size_t)P, sizeof(double));
    if (!acc || !pw) {
        free(acc);
        free(pw);
        return -2;
    }
    set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4)
    for (int p = 0; p < P; p++) {
        const double *pp = pos + 3 * p;
        const double np = sqrt(pp[0] * pp[0] + pp[1] * pp[1] + pp[2] * pp[2]);
        double *a = acc + (size_t)p * S * 2;
        for (int i = 0; i < nscat; i++) {
            const double *s = scat + 5 * i;
            const double ex = pp[0] - s[0], ey = pp[1] - s[1], ez = pp[2] - s[2];
            const double D = np - sqrt(ex * ex + ey * ey + ez * ez);
            const double rr = cos(dk * D), ri = sin(dk * D);
            double zr = 0, zi = 0;
            for (int k = 0; k < S; k++) {
                if ((k & 31) == 0) {
                    const double ph = k_r[k] * D;
                    zr = cos(ph);
                    zi = sin(ph);
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
        for (int k = 0; k < S; k++) sp += a[2 * k] * a[2 * k] + a[2 * k + 1] * a[2 * k + 1];
        pw[p] = sp;
    }
    double total = 0;
    for (int p = 0; p < P; p++) total += pw[p];
    const double mean_pw = total / ((double)P * S);
    const double sigma = snr_db < 300 ? sqrt(mean_pw / pow(10.0, snr_db / 10.0) / 2.0) : 0.0;
#pragma omp parallel for schedule(static)
    for (int p = 0; p < P; p++) {
        for (int k = 0; k < S; k++) {
            const size_t idx = (size_t)p * S + k;
            double nr = 0, ni = 0;
            if (sigma > 0) {
                const double u1 = orc_unit(orc_mix64(seed ^ orc_mix64(2 * idx)));
                const double u2 = orc_unit(orc_mix64(seed ^ orc_mix64(2 * idx + 1)));
                const double rad = sqrt(-2.0 * log(u1));
                nr = sigma * rad * cos(2 * pi * u2);
                ni = sigma * rad * sin(2 * pi * u2);
            }
            phs[2 * idx] = (float)(acc[2 * idx] + nr);
            phs[2 * idx + 1] = (float)(acc[2 * idx + 1] + ni);
        }
    }
    free(acc);
    free(pw);
    return 0;
}
