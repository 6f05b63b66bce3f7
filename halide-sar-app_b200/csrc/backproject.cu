// backproject.cu -- per-pixel pulse accumulation (backprojection.cpp:106-138).
//
// Split-precision tile kernel
// ---------------------------
// One CTA forms one pixel tile (TX x TY pixels, NT threads, PPT pixels per
// thread).  The tile centre r_c and radius rho are found once.  For every
// (tile, pulse) the large terms are evaluated once in f64:
//     w    = pos_p - r_c,  R = |w|,  dr_c = |pos_p| - R
//     t_c  = (dr_c - lsa) / lsr        (range-bin coordinate of the centre)
//     B    = exp(-j k_c dr_c)          (phase reduced in f64, then sincospi)
// and only the small offset of a pixel, delta = r - r_c (|delta| <= rho, a
// metre or two), goes through FP32 per pixel*pulse:
//     h     = w_hat . delta - |delta|^2 / (2R)
//     Delta = h (1 + g [+ 2 g^2]),  g = h / (2R)   = R - |w - delta|
//     dr    = dr_c + Delta
// (a series of R - sqrt(R^2 - 2Rh); a chunk whose pulses are too close for
// the series to meet the phase tolerance switches to the closed form
// 2Rh / (R + sqrt(R (R - 2h)))).  Delta is at most rho, so each pulse only
// touches a window of W = 2K+1 range bins around floor(t_c); the window is
// staged in shared memory per pulse chunk as
//     (m, d) = ((Q[k] + Q[k+1]) / 2, Q[k+1] - Q[k]) * B
// so the reference's clamped lerp Q[l](1-w) + Q[l+1]w becomes m + (w-1/2) d
// (one 16-byte shared load), and the carrier left per pixel is
// exp(-j k_c Delta), a few hundred radians at most, evaluated with the SFU.
// The bin index comes from the float itself (add 1.5*2^23 and read the low
// mantissa bits), which keeps the floor off the conversion pipe.
//
// Work list: items are (job, tile); with `persistent` the grid is the number
// of resident CTAs and each CTA pulls items (ordered longest first by the
// host) from an atomic counter, so uneven jobs of a batch share one launch.
//
// Naive kernel: the same quantity with plain FP32 range |pos| - |r - pos|
// and phase k_c * dr per pixel*pulse; kept as the precision-study baseline.
#include <cfloat>

#include "internal.h"
#include "kernels.h"

namespace sarbp {

namespace {

constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23
constexpr int kMagicBits = 0x4B400000;
constexpr int kNT = 256;               // threads per CTA
constexpr double kInv2Pi = 0.15915494309189533577;
constexpr float kPhaseTol = 2e-5f;     // rad, truncation budget of the series

struct __align__(16) PulseA {
    float wx, wy, wz, e;  // w_hat, 1/(2R)
};
struct __align__(16) PulseB {
    float c0;    // t_c - floor(t_c) + K - 1/2
    float R;     // |w|
    int off;     // offset of the pulse's window in the staging buffer
    int pad;
};

__device__ __forceinline__ double warp_min(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Inner loop over the nc pulses of a chunk for the thread's PPT pixels.
// MODE 0: Delta = h(1+g); 1: Delta = h(1+g+2g^2); 2: closed form.
template <int MODE, int PPT>
__device__ __forceinline__ void accumulate(int nc, const PulseA *__restrict__ pa,
                                           const PulseB *__restrict__ pb,
                                           const float4 *__restrict__ stage, float inv_lsr,
                                           float kc, float hi_clamp, const float (&dx)[PPT],
                                           const float (&dy)[PPT], const float (&dz)[PPT],
                                           const float (&nd2)[PPT], float (&ar)[PPT],
                                           float (&ai)[PPT]) {
#pragma unroll 2
    for (int i = 0; i < nc; ++i) {
        const PulseA a = pa[i];
        const PulseB b = pb[i];
        const float4 *__restrict__ st = stage + b.off;
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
            float h = fmaf(a.wx, dx[k], fmaf(a.wy, dy[k], fmaf(a.wz, dz[k], nd2[k] * a.e)));
            float D;
            if constexpr (MODE == 0) {
                const float g = h * a.e;
                D = fmaf(h, g, h);
            } else if constexpr (MODE == 1) {
                const float g = h * a.e;
                D = fmaf(h * g, fmaf(2.0f, g, 1.0f), h);
            } else {
                // 2Rh / (R + sqrt(R (R - 2h)))
                const float q = fmaxf(fmaf(-2.0f, h, b.R), 0.0f);
                const float s = sqrtf(b.R * q);
                D = (2.0f * b.R * h) / (b.R + s);
            }
            float tl = fmaf(D, inv_lsr, b.c0);
            if constexpr (MODE == 2) tl = fminf(fmaxf(tl, 0.0f), hi_clamp);
            const float f = tl + kMagic;
            const float wgt = tl - (f - kMagic);
            const int j = __float_as_int(f) - kMagicBits;
            const float4 md = st[j];
            const float vr = fmaf(wgt, md.z, md.x);
            const float vi = fmaf(wgt, md.w, md.y);
            float s, c;
            __sincosf(D * kc, &s, &c);
            ar[k] = fmaf(vr, c, fmaf(vi, s, ar[k]));
            ai[k] = fmaf(vi, c, fmaf(-vr, s, ai[k]));
        }
    }
}

template <int TX, int TY>
__global__ void __launch_bounds__(kNT) bp_tile_kernel(const DevJob *__restrict__ jobs,
                                                      const WorkItem *__restrict__ items, int nitems,
                                                      int *__restrict__ counter, int stage_cap,
                                                      int cmax, int persistent) {
    constexpr int PPT = TX * TY / kNT;
    constexpr int ROWS = kNT / TX;
    static_assert(PPT >= 1 && TX * TY == PPT * kNT, "tile must be a multiple of the CTA");
    extern __shared__ float4 smem[];
    float4 *stage = smem;
    PulseA *pa = reinterpret_cast<PulseA *>(stage + stage_cap);
    PulseB *pb = reinterpret_cast<PulseB *>(pa + cmax);
    float2 *pB = reinterpret_cast<float2 *>(pb + cmax);
    int *pbase = reinterpret_cast<int *>(pB + cmax);
    float2 *fin = reinterpret_cast<float2 *>(pbase + cmax);  // [TX*TY]
    __shared__ double sred[6][kNT / 32];
    __shared__ float sredf[kNT / 32];
    __shared__ int s_item;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int lx = tid % TX, ly = tid / TX;

    int item = blockIdx.x;
    for (;;) {
        if (persistent) {
            if (tid == 0) s_item = atomicAdd(counter, 1);
            __syncthreads();
            item = s_item;
            __syncthreads();
        }
        if (item >= nitems) break;
        const WorkItem wi = items[item];
        const DevJob &jb = jobs[wi.job];
        const int nu = jb.nu, nv = jb.nv, P = jb.P, N = jb.N;
        const long long npix = (long long)nu * nv;
        const int tx0 = (wi.tile % jb.tiles_x) * TX;
        const int ty0 = (wi.tile / jb.tiles_x) * TY;

        // ---- pixel positions (f64) and the tile's bounding box ----
        double prx[PPT], pry[PPT], prz[PPT];
        bool act[PPT];
        double mn[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, mx[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
        bool bad = false;
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
            const int ix = tx0 + lx, iy = ty0 + ly + k * ROWS;
            act[k] = ix < nu && iy < nv;
            prx[k] = pry[k] = prz[k] = 0.0;
            if (act[k]) {
                if (jb.r) {
                    const long long pix = (long long)iy * nu + ix;
                    prx[k] = jb.r[pix];
                    pry[k] = jb.r[npix + pix];
                    prz[k] = jb.r[2 * npix + pix];
                } else {
                    // img_plane.cpp:92-102: (0 + u_hat*u) + v_hat*v
                    const double uu = jb.u[ix], vv = jb.v[iy];
                    prx[k] = __dadd_rn(__dmul_rn(jb.uh[0], uu), __dmul_rn(jb.vh[0], vv));
                    pry[k] = __dadd_rn(__dmul_rn(jb.uh[1], uu), __dmul_rn(jb.vh[1], vv));
                    prz[k] = __dadd_rn(__dmul_rn(jb.uh[2], uu), __dmul_rn(jb.vh[2], vv));
                }
                if (!(isfinite(prx[k]) && isfinite(pry[k]) && isfinite(prz[k]))) {
                    bad = true;
                    act[k] = false;
                } else {
                    mn[0] = fmin(mn[0], prx[k]); mx[0] = fmax(mx[0], prx[k]);
                    mn[1] = fmin(mn[1], pry[k]); mx[1] = fmax(mx[1], pry[k]);
                    mn[2] = fmin(mn[2], prz[k]); mx[2] = fmax(mx[2], prz[k]);
                }
            }
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double a = warp_min(mn[d]), b = warp_max(mx[d]);
            if (lane == 0) { sred[d][warp] = a; sred[3 + d][warp] = b; }
        }
        __syncthreads();
        double rc[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double a = DBL_MAX, b = -DBL_MAX;
            for (int w = 0; w < kNT / 32; ++w) { a = fmin(a, sred[d][w]); b = fmax(b, sred[3 + d][w]); }
            rc[d] = a <= b ? 0.5 * (a + b) : 0.0;
        }
        // ---- offsets, radius, final phase exp(+j k_c dr(pixel, P/2)) ----
        float dx[PPT], dy[PPT], dz[PPT], nd2[PPT];
        float rho = 0.0f;
        const double4 pmid = jb.pulse[P / 2];
        const double k_c = jb.sc->k_c;
        const double kc2pi = k_c * kInv2Pi;
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
            dx[k] = dy[k] = dz[k] = nd2[k] = 0.0f;
            float2 f = make_float2(0.f, 0.f);
            if (act[k]) {
                dx[k] = (float)(prx[k] - rc[0]);
                dy[k] = (float)(pry[k] - rc[1]);
                dz[k] = (float)(prz[k] - rc[2]);
                const float d2 = fmaf(dx[k], dx[k], fmaf(dy[k], dy[k], dz[k] * dz[k]));
                nd2[k] = -d2;
                rho = fmaxf(rho, sqrtf(d2));
                const double ex = prx[k] - pmid.x, ey = pry[k] - pmid.y, ez = prz[k] - pmid.z;
                const double drm = pmid.w - sqrt(ex * ex + ey * ey + ez * ez);
                double th = drm * kc2pi;
                th = th - rint(th);
                float s, c;
                sincospif(2.0f * (float)th, &s, &c);
                f = make_float2(c, s);
            }
            fin[tid + k * kNT] = f;
        }
        {
            float m = rho;
            for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
            if (lane == 0) sredf[warp] = m;
        }
        if (__syncthreads_or(bad) && tid == 0) atomicOr(&jb.sc->status, kStatusNonFinite);
        float rho_t = 0.0f;
        for (int w = 0; w < kNT / 32; ++w) rho_t = fmaxf(rho_t, sredf[w]);
        rho_t = rho_t * (1.0f + 1e-5f) + 1e-6f;

        const float inv_lsr = (float)jb.inv_lsr;
        const float kc = (float)k_c;
        const int K = (int)ceilf(rho_t * inv_lsr * 1.004f) + 2;
        const int W = 2 * K + 1;
        int C = stage_cap / W;
        if (C > cmax) C = cmax;
        if (C > P) C = P;
        float ar[PPT], ai[PPT];
#pragma unroll
        for (int k = 0; k < PPT; ++k) ar[k] = ai[k] = 0.0f;

        if (C < 1) {
            if (tid == 0) atomicOr(&jb.sc->status, kStatusTileTooWide);
        } else {
            for (int p0 = 0; p0 < P; p0 += C) {
                const int nc = min(C, P - p0);
                // ---- per-pulse constants of this chunk (f64) ----
                bool need3 = false, need_exact = false;
                if (tid < nc) {
                    const int p = p0 + tid;
                    const double4 g = jb.pulse[p];
                    const double wx = g.x - rc[0], wy = g.y - rc[1], wz = g.z - rc[2];
                    const double R = sqrt(wx * wx + wy * wy + wz * wz);
                    const double drc = g.w - R;
                    double tc = (drc - jb.lsa) * jb.inv_lsr;
                    tc = fmin(fmax(tc, -1.0e8), 1.0e8);
                    const double fl = floor(tc);
                    PulseA A;
                    PulseB Bq;
                    float2 Bp;
                    int base;
                    if (isfinite(R) && R > 0.0 && isfinite(tc)) {
                        const double iR = 1.0 / R;
                        A.wx = (float)(wx * iR); A.wy = (float)(wy * iR); A.wz = (float)(wz * iR);
                        A.e = (float)(0.5 * iR);
                        Bq.c0 = (float)((tc - fl) + ((double)K - 0.5));
                        Bq.R = (float)R;
                        base = (int)fl - K;
                        double th = drc * kc2pi;
                        th = th - rint(th);
                        float s, c;
                        sincospif(2.0f * (float)th, &s, &c);
                        Bp = make_float2(c, -s);
                        const float gm = rho_t * A.e;  // max |g|
                        const float e2 = 2.0f * rho_t * gm * gm * kc;
                        const float e3 = 5.0f * rho_t * gm * gm * gm * kc;
                        need3 = e2 > kPhaseTol;
                        need_exact = e3 > kPhaseTol || gm > 1e-3f;
                    } else {
                        A.wx = A.wy = A.wz = A.e = 0.0f;
                        Bq.c0 = (float)K - 0.5f;
                        Bq.R = 1.0f;
                        base = 0;
                        Bp = make_float2(0.f, 0.f);
                        atomicOr(&jb.sc->status, kStatusNonFinite);
                    }
                    Bq.off = tid * W;
                    Bq.pad = 0;
                    pa[tid] = A;
                    pb[tid] = Bq;
                    pB[tid] = Bp;
                    pbase[tid] = base;
                }
                const int mode = __syncthreads_or(need_exact) ? 2 : (__syncthreads_or(need3) ? 1 : 0);
                // ---- stage the chunk's range windows: (m, d) * B ----
                for (int i = warp; i < nc; i += kNT / 32) {
                    const float2 *__restrict__ q = jb.Q + (size_t)(p0 + i) * N;
                    const int base = pbase[i];
                    const float2 B = pB[i];
                    float4 *dst = stage + i * W;
                    for (int j = lane; j < W; j += 32) {
                        const int g0 = min(max(base + j, 0), N - 1);
                        const int g1 = min(max(base + j + 1, 0), N - 1);
                        const float2 a = __ldg(&q[g0]);
                        const float2 b = __ldg(&q[g1]);
                        const float mr = 0.5f * (a.x + b.x), mi = 0.5f * (a.y + b.y);
                        const float dr = b.x - a.x, di = b.y - a.y;
                        dst[j] = make_float4(fmaf(mr, B.x, -mi * B.y), fmaf(mr, B.y, mi * B.x),
                                             fmaf(dr, B.x, -di * B.y), fmaf(dr, B.y, di * B.x));
                    }
                }
                __syncthreads();
                const float hi = (float)(W - 1) - 0.5f;
                if (mode == 0)
                    accumulate<0, PPT>(nc, pa, pb, stage, inv_lsr, kc, hi, dx, dy, dz, nd2, ar, ai);
                else if (mode == 1)
                    accumulate<1, PPT>(nc, pa, pb, stage, inv_lsr, kc, hi, dx, dy, dz, nd2, ar, ai);
                else
                    accumulate<2, PPT>(nc, pa, pb, stage, inv_lsr, kc, hi, dx, dy, dz, nd2, ar, ai);
                __syncthreads();
            }
        }
        // ---- epilogue: final phase, row flip (backprojection.cpp:130-138), max|z| ----
        double zmax = 0.0;
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
            const int ix = tx0 + lx, iy = ty0 + ly + k * ROWS;
            if (ix < nu && iy < nv) {
                const float2 f = fin[tid + k * kNT];
                const double zr = (double)fmaf(ar[k], f.x, -ai[k] * f.y);
                const double zi = (double)fmaf(ar[k], f.y, ai[k] * f.x);
                jb.out[(long long)(nv - 1 - iy) * nu + ix] = make_double2(zr, zi);
                zmax = fmax(zmax, sqrt(zr * zr + zi * zi));
            }
        }
        zmax = warp_max(zmax);
        if (lane == 0) sred[0][warp] = zmax;
        __syncthreads();
        if (tid == 0) {
            double m = 0.0;
            for (int w = 0; w < kNT / 32; ++w) m = fmax(m, sred[0][w]);
            atomicMax(&jb.sc->maxabs, (unsigned long long)__double_as_longlong(m));
        }
        __syncthreads();
        if (!persistent) break;
    }
}

// ---- naive FP32 kernel: one thread per pixel ----
__global__ void __launch_bounds__(256) bp_naive_kernel(const DevJob *__restrict__ jobs, int job) {
    const DevJob &jb = jobs[job];
    const long long npix = (long long)jb.nu * jb.nv;
    const long long pix = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= npix) return;
    const int ix = (int)(pix % jb.nu), iy = (int)(pix / jb.nu);
    float rx, ry, rz;
    if (jb.r) {
        rx = (float)jb.r[pix]; ry = (float)jb.r[npix + pix]; rz = (float)jb.r[2 * npix + pix];
    } else {
        rx = (float)(jb.uh[0] * jb.u[ix] + jb.vh[0] * jb.v[iy]);
        ry = (float)(jb.uh[1] * jb.u[ix] + jb.vh[1] * jb.v[iy]);
        rz = (float)(jb.uh[2] * jb.u[ix] + jb.vh[2] * jb.v[iy]);
    }
    const float lsa = (float)jb.lsa, inv_lsr = (float)jb.inv_lsr, kc = (float)jb.sc->k_c;
    const int N = jb.N;
    float ar = 0.f, ai = 0.f;
    for (int p = 0; p < jb.P; ++p) {
        const double4 g = jb.pulse[p];
        const float ex = rx - (float)g.x, ey = ry - (float)g.y, ez = rz - (float)g.z;
        const float dr = (float)g.w - sqrtf(ex * ex + ey * ey + ez * ez);
        const float t = (dr - lsa) * inv_lsr;
        const float fl = floorf(t);
        const int l = (int)fminf(fmaxf(fl, -2.0f), (float)N + 1.0f);
        const float w = fminf(fmaxf(t - fl, 0.f), 1.f);
        const int l0 = min(max(l, 0), N - 1), l1 = min(max(l + 1, 0), N - 1);
        const float2 *q = jb.Q + (size_t)p * N;
        const float2 a = __ldg(&q[l0]), b = __ldg(&q[l1]);
        const float vr = fmaf(w, b.x - a.x, a.x), vi = fmaf(w, b.y - a.y, a.y);
        float s, c;
        __sincosf(kc * dr, &s, &c);
        ar = fmaf(vr, c, fmaf(vi, s, ar));
        ai = fmaf(vi, c, fmaf(-vr, s, ai));
    }
    const double4 g = jb.pulse[jb.P / 2];
    const float ex = rx - (float)g.x, ey = ry - (float)g.y, ez = rz - (float)g.z;
    const float drm = (float)g.w - sqrtf(ex * ex + ey * ey + ez * ez);
    float s, c;
    __sincosf(kc * drm, &s, &c);
    const double zr = (double)(ar * c - ai * s), zi = (double)(ar * s + ai * c);
    jb.out[(long long)(jb.nv - 1 - iy) * jb.nu + ix] = make_double2(zr, zi);
    atomicMax(&jb.sc->maxabs, (unsigned long long)__double_as_longlong(sqrt(zr * zr + zi * zi)));
}

template <int TX, int TY>
cudaError_t set_attr(size_t smem) {
    return cudaFuncSetAttribute(bp_tile_kernel<TX, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem);
}

template <int TX, int TY>
int active_blocks(size_t smem) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, bp_tile_kernel<TX, TY>, kNT, smem) != cudaSuccess)
        return 0;
    return n;
}

}  // namespace

bool bp_tile_supported(int tx, int ty) {
    return (tx == 32 && (ty == 8 || ty == 16 || ty == 32 || ty == 64)) ||
           (tx == 64 && (ty == 16 || ty == 32)) || (tx == 16 && (ty == 16 || ty == 32 || ty == 64));
}

size_t bp_smem_bytes(const BpLaunch &L) {
    return (size_t)L.stage_cap * sizeof(float4) +
           (size_t)L.cmax * (sizeof(PulseA) + sizeof(PulseB) + sizeof(float2) + sizeof(int)) +
           (size_t)L.tile_x * L.tile_y * sizeof(float2);
}

#define SARBP_BP_TILES(X)                                                                      \
    X(32, 8) X(32, 16) X(32, 32) X(32, 64) X(64, 16) X(64, 32) X(16, 16) X(16, 32) X(16, 64)

cudaError_t init_backproject_attributes() {
    const size_t maxs = 200 * 1024;
    cudaError_t e = cudaSuccess;
#define X(a, b) \
    if (e == cudaSuccess) e = set_attr<a, b>(maxs);
    SARBP_BP_TILES(X)
#undef X
    return e;
}

int bp_max_active_blocks(const BpLaunch &L) {
    const size_t smem = bp_smem_bytes(L);
#define X(a, b) \
    if (L.tile_x == a && L.tile_y == b) return active_blocks<a, b>(smem);
    SARBP_BP_TILES(X)
#undef X
    return 0;
}

cudaError_t launch_backproject(const BpLaunch &L, const DevJob *d_jobs, const WorkItem *d_items,
                               int nitems, int *d_counter, cudaStream_t st) {
    const size_t smem = bp_smem_bytes(L);
    const int grid = L.persistent ? L.grid : nitems;
    if (grid <= 0) return cudaSuccess;
#define X(a, b)                                                                              \
    if (L.tile_x == a && L.tile_y == b) {                                                    \
        bp_tile_kernel<a, b><<<grid, kNT, smem, st>>>(d_jobs, d_items, nitems, d_counter,    \
                                                      L.stage_cap, L.cmax, L.persistent);    \
        return cudaGetLastError();                                                           \
    }
    SARBP_BP_TILES(X)
#undef X
    return cudaErrorInvalidValue;
}

cudaError_t launch_backproject_naive(const DevJob *d_jobs, int job, int nu, int nv, cudaStream_t st) {
    const long long npix = (long long)nu * nv;
    const int blocks = (int)((npix + 255) / 256);
    bp_naive_kernel<<<blocks, 256, 0, st>>>(d_jobs, job);
    return cudaGetLastError();
}

}  // namespace sarbp
