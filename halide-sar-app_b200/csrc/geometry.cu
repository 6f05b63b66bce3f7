// geometry.cu -- f64 geometry of the pixel tiles, ahead of the FP32 loop.
//
// tile_setup_kernel (one CTA per (job, tile), whatever the pulse parts of the
// backprojection's work items) forms the tile's geometry and
// then its pulse records:
//   rc    = centre of the bounding box of the tile's pixel positions
//   wide  = k_c * rho > kWideRad (rho below); then w0 = unit
//           vector from rc to the mid-aperture antenna
//   rho   = max |(f32)(r - rc)|, the same f32 offsets the backprojection
//           kernel forms, padded; K = ceil(1.004 X / lsr) + 2 for a bound X
//           <= rho on the pixels' range offsets (window_half_width)
//   fin   = exp(+j k_c dr(pixel, P/2)) per pixel (backprojection.cpp:135),
//           dr = |pos| - |r - pos| in f64, phase reduced in f64; wide tiles
//           multiply in exp(-j w0 . k_c (r - rc)), also in f64
// record of each pulse (make_record):
//   w = pos - rc, R = |w|, dr_c = |pos| - R, t_c = (dr_c - lsa) / lsr,
//   base = floor(t_c) - K, theta = k_c dr_c reduced to [-pi, pi),
//   c0 = t_c - floor(t_c) + K - 1/2 - theta / (k_c lsr), and the series
//   order the pulse needs for the tile radius (see backproject.cu).
#include <cfloat>

#include "internal.h"
#include "kernels.h"

namespace sarbp {

namespace {

constexpr int kThreadsGeom = 256;
constexpr double kInv2Pi = 0.15915494309189533577;
constexpr double kTwoPi = 6.28318530717958647693;
constexpr float kPhaseTol = 2e-5f;  // rad, truncation budget of the series

__device__ __forceinline__ void pixel_pos(const DevJob &jb, int ix, int iy, double &x, double &y,
                                          double &z) {
    if (jb.r) {
        const long long npix = (long long)jb.nu * jb.nv;
        const long long pix = (long long)iy * jb.nu + ix;
        x = jb.r[pix];
        y = jb.r[npix + pix];
        z = jb.r[2 * npix + pix];
    } else {
        // img_plane.cpp:92-102: (0 + u_hat*u) + v_hat*v
        const double uu = jb.u[ix], vv = jb.v[iy];
        x = __dadd_rn(__dmul_rn(jb.uh[0], uu), __dmul_rn(jb.vh[0], vv));
        y = __dadd_rn(__dmul_rn(jb.uh[1], uu), __dmul_rn(jb.vh[1], vv));
        z = __dadd_rn(__dmul_rn(jb.uh[2], uu), __dmul_rn(jb.vh[2], vv));
    }
}

// Per-job constants of the records: k_c, 1/(2 k_c), 1/(k_c lsr).
struct RecConst {
    double k_c, half_inv_kc, ilk;
};

// The record of pulse p for tile t (see the file comment); false when the
// pulse has non-finite geometry (its window then stays zero).
__device__ __forceinline__ bool make_record(const DevJob &jb, const TileInfo &t, const RecConst &cst, int p,
                                            PulseRec &rec) {
    const double k_c = cst.k_c;
    const double4 g = jb.pulse[p];
    const double wx = g.x - t.rc[0], wy = g.y - t.rc[1], wz = g.z - t.rc[2];
    const double R2 = wx * wx + wy * wy + wz * wz;
    const double iR = rsqrt(R2);  // 1/R and R from one reciprocal square root
    const double R = R2 * iR;
    const double drc = g.w - R;
    double tc = (drc - jb.lsa) * jb.inv_lsr;
    tc = fmin(fmax(tc, -1.0e8), 1.0e8);
    const double fl = floor(tc);
    if (isfinite(R) && R > 0.0 && isfinite(tc)) {
        double th = drc * (k_c * kInv2Pi);
        th = th - rint(th);
        const double theta = kTwoPi * th;  // in [-pi, pi]
        const float gm = (float)(t.rho * 0.5 * iR);                    // max |g| = rho / (2R)
        const float kcf = (float)k_c;
        // truncation of the series after 2, 3, 4 terms: C_n y^n |h| with
        // y <= gm and |h| <= k_c rho (rad)
        const float rk = t.rho * kcf;
        const float e2 = 2.0f * rk * gm * gm;
        const float e3 = 5.0f * rk * gm * gm * gm;
        const float e4 = 14.0f * rk * gm * gm * gm * gm;
        int order = (e4 > kPhaseTol || gm > 5e-3f) ? 3 : e3 > kPhaseTol ? 2 : e2 > kPhaseTol ? 1 : 0;
        const int base = (int)fl - t.K;
        const double e = iR * cst.half_inv_kc;
        const double c0 = (tc - fl) + ((double)t.K - 0.5) - theta * cst.ilk;
        if (t.wide) {
            rec.a = make_float4((float)(wx * iR - (double)t.w0[0]), (float)(wy * iR - (double)t.w0[1]),
                                (float)(wz * iR - (double)t.w0[2]), (float)e);
            rec.b = make_float4((float)c0, (float)theta, (float)(k_c * R), __int_as_float(8 * base + order));
        } else {
            // theta folded into the linear term: sigma = kappa (w_hat . d + theta)
            // + e theta^2 with kappa = 1 - 2 e theta, so that theta + s + e t =
            // sigma + e' (sigma^2 - |d|^2) + (e - e')(-|d|^2), e' = e / kappa^2;
            // the last term is below 4 pi gm^2 rad and is added from series
            // order 1 on, which tiles with gm > 4e-4 always use
            if (gm > 4e-4f) order = max(order, 1);
            const double x = 2.0 * e * theta, kap = 1.0 - x;
            // 1 / kappa^2 = 1 + 2x + 3x^2 + 4x^3 + ... (|x| <= pi / (k_c R)); the
            // series through x^3 is exact to f64 rounding for |x| < 1e-3
            const double ik2 = fabs(x) < 1e-3 ? fma(x, fma(x, fma(x, 4.0, 3.0), 2.0), 1.0) : 1.0 / (kap * kap);
            rec.a = make_float4((float)(kap * wx * iR), (float)(kap * wy * iR), (float)(kap * wz * iR),
                                (float)(e * ik2));
            rec.b = make_float4((float)c0, (float)(kap * theta + e * theta * theta), (float)(k_c * R),
                                __int_as_float(8 * base + order));
        }
        return true;
    }
    // no contribution: the staging leaves this pulse's window at zero
    rec.a = make_float4(0.f, 0.f, 0.f, 0.f);
    rec.b = make_float4((float)t.K - 0.5f, 0.f, 1.f, __int_as_float(kOrderInvalid));
    return false;
}



// Half-width K (bins) of the range window every pulse's bins of this tile
// fall in: K = ceil(1.004 X / lsr) + 2 for a bound X on |Delta| =
// |R - |pos - r|| over the tile's pixels r = rc + d and all pulses.  The
// triangle inequality gives X = rho.  Tighter, with s = w_hat . d and E the
// job's orthonormal image-plane frame (prep kernel):
//   |Delta| = |2 R s - |d|^2| / (R + |pos - r|) <= (2 R |s| + rho^2) / (2 R - rho),
//   |s| <= sum_i |d . E_i| |w_hat . E_i|,  |d . E_i| <= hq_i over the tile,
//   |w_hat . E_i| <= los_abs_i + 2 |rc| / pos_min,
// since w_hat = (pos - rc) / |pos - rc| differs from pos / |pos| by at most
// 2 |rc| / |pos|, with R >= pos_min - |rc|.  hq comes from f32 offsets and
// an f32 copy of E, so it is taken with margins well above their rounding.
// For an image plane seen from above at an angle this halves the window
// (more pulses per staged chunk), whatever the plane's orientation.
__device__ __forceinline__ int window_half_width(const DevJob &jb, float rho_f, const double (&rc)[3],
                                                 const float (&hq)[3]) {
    const double rho = (double)rho_f;
    double X = rho;
    const double pmin = jb.sc->pos_min;
    const double c = sqrt(rc[0] * rc[0] + rc[1] * rc[1] + rc[2] * rc[2]);
    if (pmin > 0.0 && isfinite(pmin) && 2.0 * c < pmin) {
        const double Rt = pmin - c, dl = 2.0 * c / pmin;
        if (Rt > 2.0 * rho) {
            double B = 0.0;
            for (int i = 0; i < 3; ++i)
                B += ((double)hq[i] * (1.0 + 1e-5) + 1e-6 * rho) * fmin(1.0, jb.sc->los_abs[i] + dl + 1e-9);
            B = B * (1.0 + 1e-6) + 1e-5 * rho;
            X = fmin(rho, (2.0 * Rt * B + rho * rho) / (2.0 * Rt - rho));
        }
    }
    return (int)ceil(X * jb.inv_lsr * 1.004) + 2;
}

__device__ __forceinline__ double warp_min_d(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_max_d(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// GP: pixels per thread (tile pixels / 256: 2, 4 or 8), kept in registers
// between the two passes.  Up to 4, registers are sized for four CTAs per
// SM (64, with a few spills): the kernel is latency-bound, and the extra CTA
// measured 0.150 ms against 0.157 ms at three (2048^2 x 1999, same output).
template <int GP>
__global__ void __launch_bounds__(kThreadsGeom, GP <= 4 ? 4 : 2)
    tile_setup_kernel(const DevJob *__restrict__ jobs, const WorkItem *__restrict__ items, int records) {
    constexpr int kWarps = kThreadsGeom / 32;
    __shared__ double sbox[kWarps][6];
    __shared__ float srho[kWarps];
    __shared__ int sflags[kWarps][2];
    __shared__ float shq[kWarps][3];
    __shared__ TileInfo s_tile;
    const WorkItem wi = items[blockIdx.x];
    const DevJob &jb = jobs[wi.job];
    const int TX = jb.tile_x, TY = jb.tile_y;
    const int lx = __ffs(TX) - 1;  // tile widths are powers of two
    const int tx0 = (wi.tile % jb.tiles_x) * TX, ty0 = (wi.tile / jb.tiles_x) * TY;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // this thread's pixels, kept in registers for both passes
    double px[GP], py[GP], pz[GP];
    unsigned live = 0u;  // bit k: pixel k is inside the image and finite
    double mn[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, mx[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    int bad = 0;
#pragma unroll
    for (int k = 0; k < GP; ++k) {
        px[k] = py[k] = pz[k] = 0.0;
        const int idx = threadIdx.x + k * kThreadsGeom;
        if (idx >= TX * TY) continue;
        const int ix = tx0 + (idx & (TX - 1)), iy = ty0 + (idx >> lx);
        if (ix >= jb.nu || iy >= jb.nv) continue;
        double x, y, z;
        pixel_pos(jb, ix, iy, x, y, z);
        if (!(isfinite(x) && isfinite(y) && isfinite(z))) {
            bad = 1;
            continue;
        }
        px[k] = x;
        py[k] = y;
        pz[k] = z;
        live |= 1u << k;
        mn[0] = fmin(mn[0], x); mx[0] = fmax(mx[0], x);
        mn[1] = fmin(mn[1], y); mx[1] = fmax(mx[1], y);
        mn[2] = fmin(mn[2], z); mx[2] = fmax(mx[2], z);
    }
    // bounding box: one pass through shared memory for all six extrema
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        mn[d] = warp_min_d(mn[d]);
        mx[d] = warp_max_d(mx[d]);
    }
    if (lane == 0)
        for (int d = 0; d < 3; ++d) {
            sbox[warp][d] = mn[d];
            sbox[warp][3 + d] = mx[d];
        }
    __syncthreads();
    double rc[3];
    for (int d = 0; d < 3; ++d) {
        double a = sbox[0][d], b = sbox[0][3 + d];
        for (int w = 1; w < kWarps; ++w) {
            a = fmin(a, sbox[w][d]);
            b = fmax(b, sbox[w][3 + d]);
        }
        rc[d] = a <= b ? 0.5 * (a + b) : 0.0;
    }
    // radius, extents in the job's image-plane frame and flags of the tile,
    // from the same f32 offsets the backprojection kernel forms
    float Ef[3][3];  // the job's image-plane frame (f32 copy)
    for (int i = 0; i < 3; ++i)
        for (int c = 0; c < 3; ++c) Ef[i][c] = (float)jb.sc->frame[i][c];
    float hq[3] = {0.f, 0.f, 0.f};  // max |(r - rc) . E_i| over the tile's pixels
    float rho = 0.0f;
    int planar = 1;
#pragma unroll
    for (int k = 0; k < GP; ++k) {
        if (!(live & (1u << k))) continue;
        const float ox = (float)(px[k] - rc[0]), oy = (float)(py[k] - rc[1]), oz = (float)(pz[k] - rc[2]);
        rho = fmaxf(rho, sqrtf(fmaf(ox, ox, fmaf(oy, oy, oz * oz))));
        planar &= (oz == 0.0f);
        for (int i = 0; i < 3; ++i) hq[i] = fmaxf(hq[i], fabsf(fmaf(ox, Ef[i][0], fmaf(oy, Ef[i][1], oz * Ef[i][2]))));
    }
    for (int o = 16; o > 0; o >>= 1) {
        rho = fmaxf(rho, __shfl_xor_sync(0xffffffffu, rho, o));
        planar &= __shfl_xor_sync(0xffffffffu, planar, o);
        bad |= __shfl_xor_sync(0xffffffffu, bad, o);
        for (int i = 0; i < 3; ++i) hq[i] = fmaxf(hq[i], __shfl_xor_sync(0xffffffffu, hq[i], o));
    }
    if (lane == 0) {
        srho[warp] = rho;
        sflags[warp][0] = planar;
        sflags[warp][1] = bad;
        for (int i = 0; i < 3; ++i) shq[warp][i] = hq[i];
    }
    __syncthreads();
    for (int w = 0; w < kWarps; ++w) {
        rho = fmaxf(rho, srho[w]);
        planar &= sflags[w][0];
        bad |= sflags[w][1];
        for (int i = 0; i < 3; ++i) hq[i] = fmaxf(hq[i], shq[w][i]);
    }
    const double k_c = jb.sc->k_c;
    const double4 pm = jb.pulse[jb.P / 2];
    // wide tile (k_c times the tile's radius above kWideRad): reference
    // direction w0 toward the mid-aperture antenna; the phase w0 . k_c (r - rc)
    // leaves the pulse loop and enters fin in f64
    float w0f[3] = {0.f, 0.f, 0.f};
    bool wide = false;
    {
        const double gx = pm.x - rc[0], gy = pm.y - rc[1], gz = pm.z - rc[2];
        const double g = sqrt(gx * gx + gy * gy + gz * gz);
        if (k_c * (double)rho > kWideRad && g > 0.0 && isfinite(g)) {
            wide = true;
            w0f[0] = (float)(gx / g);
            w0f[1] = (float)(gy / g);
            w0f[2] = (float)(gz / g);
        }
    }
#pragma unroll
    for (int k = 0; k < GP; ++k) {
        const int idx = threadIdx.x + k * kThreadsGeom;
        if (idx >= TX * TY) continue;
        const int ix = tx0 + (idx & (TX - 1)), iy = ty0 + (idx >> lx);
        if (ix >= jb.nu || iy >= jb.nv) continue;
        const double x = px[k], y = py[k], z = pz[k];
        float2 f = make_float2(0.f, 0.f);
        if (live & (1u << k)) {
            const double ex = x - pm.x, ey = y - pm.y, ez = z - pm.z;
            const double drm = pm.w - sqrt(ex * ex + ey * ey + ez * ez);
            double th = drm * (k_c * kInv2Pi);
            if (wide) {
                const double s0 = k_c * ((double)w0f[0] * (x - rc[0]) + (double)w0f[1] * (y - rc[1]) +
                                         (double)w0f[2] * (z - rc[2]));
                th -= s0 * kInv2Pi;
            }
            th = th - rint(th);
            float s, c;
            sincospif(2.0f * (float)th, &s, &c);
            f = make_float2(c, s);
        }
        jb.fin[(long long)iy * jb.nu + ix] = f;
    }
    if (threadIdx.x == 0) {
        TileInfo t;
        t.rc[0] = rc[0];
        t.rc[1] = rc[1];
        t.rc[2] = rc[2];
        t.rho = rho * (1.0f + 1e-5f) + 1e-6f;
        t.K = window_half_width(jb, t.rho, rc, hq);
        t.planar = planar;
        t.wide = wide ? 1 : 0;
        t.w0[0] = w0f[0];
        t.w0[1] = w0f[1];
        t.w0[2] = w0f[2];
        // Lane orientation: the window entries that neighbouring lanes read
        // are |w . step| / lsr bins apart for a one-pixel step; apart by one
        // or more, eight lanes span more than the eight 16-byte banks of a
        // shared-memory wavefront and collide.  Run the lanes along the axis
        // with the smaller step (square tiles only).
        t.transposed = 0;
        if (TX == TY && tx0 + 1 < jb.nu && ty0 + 1 < jb.nv) {
            double x0, y0, z0, x1, y1, z1, x2, y2, z2;
            pixel_pos(jb, tx0, ty0, x0, y0, z0);
            pixel_pos(jb, tx0 + 1, ty0, x1, y1, z1);
            pixel_pos(jb, tx0, ty0 + 1, x2, y2, z2);
            const double gx = pm.x - rc[0], gy = pm.y - rc[1], gz = pm.z - rc[2];
            const double g = sqrt(gx * gx + gy * gy + gz * gz);
            if (g > 0.0 && isfinite(g)) {
                const double sx = fabs(gx * (x1 - x0) + gy * (y1 - y0) + gz * (z1 - z0)) / (g * jb.lsr);
                const double sy = fabs(gx * (x2 - x0) + gy * (y2 - y0) + gz * (z2 - z0)) / (g * jb.lsr);
                if (sx >= 1.0 && sy < sx) t.transposed = 1;
            }
        }
        jb.tiles[wi.tile] = t;
        s_tile = t;
        if (bad) atomicOr(&jb.sc->status, kStatusNonFinite);
    }
    __syncthreads();
    if (!records) return;  // pulse-chunked jobs form their records per chunk
    // ---- this tile's pulse records ----
    const TileInfo t = s_tile;
    bool bad_pulse = false;
    PulseRec *recs = jb.recs + (size_t)wi.tile * jb.P;
    RecConst rk;
    rk.k_c = k_c;
    rk.half_inv_kc = 0.5 / k_c;
    rk.ilk = jb.inv_lsr / k_c;
    for (int p = threadIdx.x; p < jb.P; p += kThreadsGeom) {
        PulseRec rec;
        bad_pulse |= !make_record(jb, t, rk, p, rec);
        recs[p] = rec;
    }
    if (__any_sync(0xffffffffu, bad_pulse) && lane == 0) atomicOr(&jb.sc->status, kStatusNonFinite);
}

// Records only, for the pulses of one chunk of a pulse-chunked job: the
// tile table was formed ahead of the first chunk (tile_setup_kernel with
// records = 0), jb.P is the chunk's pulse count and jb.pulse its pulse table.
__global__ void __launch_bounds__(kThreadsGeom)
    tile_records_kernel(const DevJob *__restrict__ jobs, const WorkItem *__restrict__ items) {
    const WorkItem wi = items[blockIdx.x];
    const DevJob &jb = jobs[wi.job];
    const TileInfo t = jb.tiles[wi.tile];
    RecConst rk;
    rk.k_c = jb.sc->k_c;
    rk.half_inv_kc = 0.5 / rk.k_c;
    rk.ilk = jb.inv_lsr / rk.k_c;
    PulseRec *recs = jb.recs + (size_t)wi.tile * jb.P;
    bool bad_pulse = false;
    for (int p = threadIdx.x; p < jb.P; p += kThreadsGeom) {
        PulseRec rec;
        bad_pulse |= !make_record(jb, t, rk, p, rec);
        recs[p] = rec;
    }
    if (__any_sync(0xffffffffu, bad_pulse) && (threadIdx.x & 31) == 0) atomicOr(&jb.sc->status, kStatusNonFinite);
}

}  // namespace

cudaError_t launch_tile_setup(const DevJob *d_jobs, const WorkItem *d_items, int nitems, int tile_pixels,
                              cudaStream_t st, int records) {
    if (nitems <= 0) return cudaSuccess;
    if (tile_pixels < 1 || tile_pixels > 8 * kThreadsGeom) return cudaErrorInvalidValue;
    if (tile_pixels <= 2 * kThreadsGeom)
        tile_setup_kernel<2><<<nitems, kThreadsGeom, 0, st>>>(d_jobs, d_items, records);
    else if (tile_pixels <= 4 * kThreadsGeom)
        tile_setup_kernel<4><<<nitems, kThreadsGeom, 0, st>>>(d_jobs, d_items, records);
    else
        tile_setup_kernel<8><<<nitems, kThreadsGeom, 0, st>>>(d_jobs, d_items, records);
    return cudaGetLastError();
}

cudaError_t launch_tile_records(const DevJob *d_jobs, const WorkItem *d_items, int nitems, cudaStream_t st) {
    if (nitems <= 0) return cudaSuccess;
    tile_records_kernel<<<nitems, kThreadsGeom, 0, st>>>(d_jobs, d_items);
    return cudaGetLastError();
}


}  // namespace sarbp
