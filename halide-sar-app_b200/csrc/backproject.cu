// backproject.cu -- per-pixel pulse accumulation (backprojection.cpp:106-138).
//
// Split-precision tile kernel
// ---------------------------
// One CTA forms one pixel tile (TX x TY pixels).  All f64 geometry was done
// ahead of it (geometry.cu): the tile centre rc, radius rho, window
// half-width K, the final phase per pixel, and per (tile, pulse) a record
// with w_hat = (pos - rc)/R, e = 1/(2 k_c R), the base bin, and the phase
// theta = k_c dr_c reduced to [-pi, pi).  Only the small offset of a pixel,
// d = k_c (r - rc) (|r - rc| <= rho, a metre or two), goes through FP32 per
// pixel*pulse, in radians:
//     s     = w_hat . d,   t = s^2 - |d|^2
//     Delta = s + e t     (= k_c (R - |pos - r|) up to k_c rho^3/(2R^2))
//     phase = theta + Delta,  range bin = t_c + Delta / (k_c lsr)
// A chunk whose pulses are close enough for that truncation to exceed the
// phase budget adds terms of the series in h = s - e|d|^2 (three or four);
// in the near field the closed form 2R'h / (R' + sqrt(R'(R' - 2h))),
// R' = k_c R, is used.  Tiles wider than kWideRad radians take the linear
// phase toward a reference direction out of the loop (see accumulate).  |Delta| <= k_c rho, so each pulse only touches W = 2K+1 range
// bins; range compression stored every bin as the pair
//     (m, d) = ((Q[k] + Q[k+1]) / 2, Q[k+1] - Q[k])
// so the reference's clamped lerp Q[l](1-w) + Q[l+1]w is m + (w-1/2) d: one
// 16-byte shared load.  The bin index is read from the float itself (add
// 1.5*2^23; the low mantissa bits are the integer) and one shift-add turns
// it into the staging address.
//
// Warp roles: 8 consumer warps own the pixels (PPT per thread) and run only
// the accumulation loop.  One producer warp stages chunk c into half b = c&1
// of a double buffer: a bulk asynchronous copy of the chunk's pulse records,
// then one bulk copy per pulse of its W-entry window of (m, d) pairs (window
// parts outside the profile are filled with the clamped edge pair), both
// completing on mbarriers with bounded waits.  Hand-over uses named
// barriers: FULL[b] producer -> consumers, EMPTY[b] consumers -> producer;
// each instance gets one arrival set from each side, and the producer
// drains the last two EMPTY instances of every tile.
//
// Work list: items are (job, tile, pulse part); with `persistent` the grid
// is the number of resident CTAs and each CTA pulls items (ordered longest
// first by the host) from an atomic counter, so uneven jobs of a batch share
// one launch.  A job with too few tiles to fill the resident CTAs has each
// tile split into nsplit items over consecutive pulse ranges; each stores
// its sums into its own slice of the job's parts buffer (plain stores, no
// atomics), and the combine kernel adds the slices in a fixed order.
//
// Naive kernel: the same quantity with plain FP32 range |pos| - |r - pos|
// and phase k_c * dr per pixel*pulse; kept as the precision-study baseline.
#include <cfloat>
#include <cstdint>

#include "internal.h"
#include "kernels.h"

namespace sarbp {

namespace {

constexpr float kMagic = 12582912.0f;             // 1.5 * 2^23
constexpr uint32_t kMagicBits = 0x4B400000u;
constexpr uint32_t kMagicOff = kMagicBits << 4;   // (mod 2^32) byte offset of index 0
constexpr int kConsumers = 256;                   // consumer threads (8 warps)
constexpr int kConsumerWarps = kConsumers / 32;
constexpr int kThreads = kConsumers + 32;         // plus one producer warp
constexpr int kBarFull0 = 1;                      // named barriers 1, 2: chunk staged
constexpr int kBarEmpty0 = 3;                     // named barriers 3, 4: chunk consumed

__device__ __forceinline__ void bar_sync(int id) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(kThreads) : "memory");
}
__device__ __forceinline__ void bar_arrive(int id) {
    asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(kThreads) : "memory");
}
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ double warp_max(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Bounded wait on an mbarrier phase; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    for (int it = 0; it < (1 << 22); ++it) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}
__device__ __forceinline__ void mbar_expect(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_copy(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Inner loop over the nc pulses of a chunk for a consumer's PPT pixels.
// With h = s - e|d|^2 and y = e h, the exact range difference is the series
//     Delta = h (1 + y + 2y^2 + 5y^3 + 14y^4 + ...)   (Catalan numbers)
// MODE 0: Delta = s + e t, t = s^2 - |d|^2 (two terms); MODE 1 adds the
// third term 2e^2 s t (on wide tiles as (e + 2e^2 s) t); MODE 2 the
// fourth, e^2 (-|d|^2 (h + s) + h^3 (2 + 5y)) over the two-term form; MODE 3 uses the closed form 2R'h / (R' + r),
// r = sqrt(R'(R' - 2h)) (near field), as its nonlinear part
// N = (s Delta - |d|^2) / (R' + r), free of the cancellation in Delta - s.
// Narrow tiles: the records carry kappa w_hat, e' and sigma0 = kappa theta +
// e theta^2 (tile geometry kernel), so the phase theta + s + e t is
//     sigma = kappa w_hat . d + sigma0,   D = sigma + e' (sigma^2 - |d|^2)
// (three FMAs for a planar tile), plus from MODE 1 on the small terms
// (e - e')(-|d|^2) and the higher series terms, formed from
// s ~= sigma - sigma0 (relative error ~1e-6, on terms of < 1e-2 rad).
// PLANAR: every pixel of the tile has dz == 0.
// WIDE: the records hold w_hat - w0 and theta, so the product with d is the
// small sd = s - s0 (s0 = w0 . d per pixel); the phase is theta + sd + N with
// every term small, and only the range bin uses the full s0 + ...:
// exp(-j s0) is applied in f64 through the final phase.
// Paired form: the consumer's pixels go in pairs through the f32x2
// instructions of sm_100 (FFMA2/FADD2/FMUL2: two lanes of FP32 per
// instruction, the same rounding as two scalar operations), so every
// per-pixel FP32 step up to the range bin costs half an issue slot; the
// window loads, the interpolation and the sine/cosine stay per pixel.  Each
// record is staged as four float4 of broadcast pairs (see stage_chunk).
// The images are the same bit for bit as with scalar arithmetic.
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

// One pulse (record rec, window at byte offset poff) for a consumer's pixel
// pairs.  The sine and cosine are written straight into the pair registers
// that the accumulation's f32x2 FMAs read.  PRE: the series products (2 e^2
// in mode 1, e^2 in mode 2, e - e') come from the record's fourth float4
// (formed by the producer for the chunk's mode) instead of being formed per
// pulse here; the same f32 products either way.
// Kernels at 3 CTAs per SM take them from the record (0.9 % faster at
// 2048^2 x 1999 by register assignment), those at 2 form them (batches of
// uneven jobs, where the extra shared load cost as much as it saved).
template <int MODE, bool PLANAR, bool WIDE, int NP, bool PRE>
__device__ __forceinline__ void pulse_step(const float4 *__restrict__ rec, uint32_t poff, float2 ILK, float2 CL,
                                           const float2 (&dx)[NP], const float2 (&dy)[NP],
                                           const float2 (&dz)[NP], const float2 (&nd2)[NP],
                                           const float2 (&s0)[NP], float2 (&ar)[NP], float2 (&ai)[NP]) {
    const float2 M2 = f2(kMagic), NEG1 = f2(-1.0f);
    const float4 q0 = rec[0];  // ax ax ay ay   (narrow: kappa w_hat; wide: w_hat - w0)
    const float4 q1 = rec[1];  // az az e  e    (narrow: e')
    const float4 q2 = rec[2];  // c0 c0 b  b    (narrow: sigma0; wide: theta)
    const float2 AX = f2(q0.x, q0.y), AY = f2(q0.z, q0.w), AZ = f2(q1.x, q1.y);
    const float2 E = f2(q1.z, q1.w), C0 = f2(q2.x, q2.y), B = f2(q2.z, q2.w);
    float Rp = 0.0f;
    float2 EE = f2(0.0f), EE2 = f2(0.0f), DE = f2(0.0f);  // e^2, 2 e^2, e - e'
    if constexpr (PRE) {
        if constexpr (MODE >= 1) {
            // (2 e^2, 2 e^2, e - e', e - e') in mode 1, (e^2, e^2, ...) in
            // mode 2, (k_c R, 0, ...) in mode 3
            const float4 q3 = rec[3];
            DE = f2(q3.z, q3.w);
            if constexpr (MODE == 3) Rp = q3.x;
            else if constexpr (MODE == 1) EE2 = f2(q3.x, q3.y);
            else EE = f2(q3.x, q3.y);
        }
    } else {
        if constexpr (MODE == 3) Rp = rec[3].x;
        const float ee = q1.z * q1.z;
        EE = f2(ee);
        EE2 = __fadd2_rn(EE, EE);
        const float de = -4.0f * ee * q2.z;  // e - e' (narrow tiles)
        DE = f2(de);
    }
#pragma unroll
    for (int j = 0; j < NP; ++j) {
        float2 D, s;  // phase argument; s = w_hat . d (approximate for narrow tiles)
        if constexpr (!WIDE) {
            float2 sg = __ffma2_rn(AX, dx[j], B);
            sg = __ffma2_rn(AY, dy[j], sg);
            if constexpr (!PLANAR) sg = __ffma2_rn(AZ, dz[j], sg);
            D = __ffma2_rn(E, __ffma2_rn(sg, sg, nd2[j]), sg);
            s = __ffma2_rn(B, NEG1, sg);
            if constexpr (MODE >= 1) D = __ffma2_rn(DE, nd2[j], D);
        } else {
            float2 sd = __fmul2_rn(AX, dx[j]);
            sd = __ffma2_rn(AY, dy[j], sd);
            if constexpr (!PLANAR) sd = __ffma2_rn(AZ, dz[j], sd);
            s = __fadd2_rn(s0[j], sd);
            // mode 1 folds its third series term into the second:
            // e t + 2 e^2 s t = (e + 2 e^2 s) t
            const float2 Et = MODE == 1 ? __ffma2_rn(EE2, s, E) : E;
            D = __fadd2_rn(__ffma2_rn(Et, __ffma2_rn(s, s, nd2[j]), sd), B);
        }
        if constexpr (MODE == 1 && !WIDE) {
            D = __ffma2_rn(__fmul2_rn(EE2, s), __ffma2_rn(s, s, nd2[j]), D);
        } else if constexpr (MODE == 2) {
            const float2 h = __ffma2_rn(E, nd2[j], s);
            const float2 q = __ffma2_rn(__fmul2_rn(f2(5.0f), E), h, f2(2.0f));
            const float2 h3 = __fmul2_rn(__fmul2_rn(h, h), h);
            D = __ffma2_rn(EE, __ffma2_rn(h3, q, __fmul2_rn(nd2[j], __fadd2_rn(h, s))), D);
        } else if constexpr (MODE == 3) {
            float n[2];
#pragma unroll
            for (int l = 0; l < 2; ++l) {
                const float sl = l ? s.y : s.x, nl = l ? nd2[j].y : nd2[j].x, el = q1.z;
                const float h = fmaf(el, nl, sl);
                const float q = fmaxf(fmaf(-2.0f, h, Rp), 0.0f);
                const float den = Rp + sqrtf(Rp * q);
                const float Dn = __fdividef(2.0f * Rp * h, den);
                // exact nonlinear part less the two-term one
                n[l] = __fdividef(fmaf(sl, Dn, nl), den) - el * fmaf(sl, sl, nl);
            }
            D = __fadd2_rn(D, f2(n[0], n[1]));
        }
        const float2 Di = WIDE ? __fadd2_rn(s0[j], D) : D;  // range-bin argument
        float2 tl = __ffma2_rn(Di, ILK, C0);
        if constexpr (MODE >= 2) {
            tl.x = fminf(fmaxf(tl.x, CL.x), CL.y);
            tl.y = fminf(fmaxf(tl.y, CL.x), CL.y);
        }
        const float2 f = __fadd2_rn(tl, M2);
        const float2 w = __ffma2_rn(__fadd2_rn(f, f2(-kMagic)), NEG1, tl);  // tl - rint(tl)
        float4 m0, m1;
        const uint32_t o0 = (__float_as_uint(f.x) << 4) + poff;  // shared-window addresses
        const uint32_t o1 = (__float_as_uint(f.y) << 4) + poff;
        asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
                     : "=f"(m0.x), "=f"(m0.y), "=f"(m0.z), "=f"(m0.w)
                     : "r"(o0));
        asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
                     : "=f"(m1.x), "=f"(m1.y), "=f"(m1.z), "=f"(m1.w)
                     : "r"(o1));
        const float vr0 = fmaf(w.x, m0.z, m0.x), vi0 = fmaf(w.x, m0.w, m0.y);
        const float vr1 = fmaf(w.y, m1.z, m1.x), vi1 = fmaf(w.y, m1.w, m1.y);
        float2 SN, CS;
        __sincosf(D.x, &SN.x, &CS.x);
        __sincosf(D.y, &SN.y, &CS.y);
        const float2 VR = f2(vr0, vr1), VI = f2(vi0, vi1);
        ar[j] = __ffma2_rn(VR, CS, __ffma2_rn(VI, SN, ar[j]));
        ai[j] = __ffma2_rn(f2(-vr0, -vr1), SN, __ffma2_rn(VI, CS, ai[j]));  // negation folds into the FMA
    }
}

// Inner loop over the nc pulses of a chunk (records rec2, windows from byte
// offset poff, pstride bytes apart); CL clamps the bin argument (modes 2, 3).
template <int MODE, bool PLANAR, bool WIDE, int NP, bool PRE>
__device__ __forceinline__ void accumulate(int nc, const float4 *__restrict__ rec2, uint32_t poff,
                                           uint32_t pstride, float2 ILK, float2 CL,
                                           const float2 (&dx)[NP], const float2 (&dy)[NP],
                                           const float2 (&dz)[NP], const float2 (&nd2)[NP],
                                           const float2 (&s0)[NP], float2 (&ar)[NP], float2 (&ai)[NP]) {
#pragma unroll 6
    for (int i = 0; i < nc; ++i, poff += pstride)
        pulse_step<MODE, PLANAR, WIDE, NP, PRE>(rec2 + 4 * i, poff, ILK, CL, dx, dy, dz, nd2, s0, ar, ai);
}

template <bool WIDE, int NP, bool PRE>
__device__ __forceinline__ void accumulate_mode(int mode, bool planar, int nc, const float4 *rec2,
                                                uint32_t poff, uint32_t pstride, float2 ILK, float2 CL,
                                                const float2 (&dx)[NP], const float2 (&dy)[NP],
                                                const float2 (&dz)[NP], const float2 (&nd2)[NP],
                                                const float2 (&s0)[NP], float2 (&ar)[NP], float2 (&ai)[NP]) {
#define SARBP_ACC(M, PL) accumulate<M, PL, WIDE, NP, PRE>(nc, rec2, poff, pstride, ILK, CL, dx, dy, dz, nd2, s0, ar, ai)
    if (mode == 0) {
        if (planar) SARBP_ACC(0, true);
        else SARBP_ACC(0, false);
    } else if (mode == 1) {
        if (planar) SARBP_ACC(1, true);
        else SARBP_ACC(1, false);
    } else if (mode == 2) {
        if (planar) SARBP_ACC(2, true);
        else SARBP_ACC(2, false);
    } else {
        SARBP_ACC(3, false);
    }
#undef SARBP_ACC
}

// Shared memory of the tile kernel.
struct TileSmem {
    float4 *stage;       // [2][stage_cap] (m, d) windows
    PulseRec *raw;       // [cmax] records as copied (producer only)
    float4 *rec2;        // [2][4 cmax] records as broadcast pairs (see accumulate)
    uint64_t *mbar_rec;  // [2]
    uint64_t *mbar_win;  // [2]
    double *sred;        // [kConsumerWarps]
    int *s_item, *s_mode;
};

struct TileShape {
    int K, W, C, nchunks;
};

// Chunking of an item's np pulses: C pulses per chunk (the windows of a
// chunk fill at most one staging half), nchunks chunks.
__device__ __forceinline__ TileShape tile_shape(const TileInfo &t, int np, int stage_cap, int cmax) {
    TileShape s;
    s.K = t.K;
    s.W = 2 * t.K + 1;
    int C = stage_cap / s.W;
    if (C > cmax) C = cmax;
    if (C > np) C = np;
    s.C = C;
    s.nchunks = C >= 1 ? (np + C - 1) / C : 0;
    return s;
}

// Producer warp, one chunk into half b: records, then windows.
__device__ __forceinline__ bool stage_chunk(const DevJob &jb, int tile, int lane, int p0, int nc, int b,
                                            const TileShape &sh, int stage_cap, int cmax,
                                            const TileSmem &sm, uint32_t (&uses)[4]) {
    const int N = jb.N, W = sh.W;
    PulseRec *rec = sm.raw;
    float4 *win = sm.stage + b * stage_cap;
    // prior generic-proxy reads of these buffers come before the async writes
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (lane == 0) {
        mbar_expect(&sm.mbar_rec[b], (uint32_t)(nc * (int)sizeof(PulseRec)));
        bulk_copy(rec, jb.recs + (size_t)tile * jb.P + p0, (uint32_t)(nc * (int)sizeof(PulseRec)),
                  &sm.mbar_rec[b]);
    }
    bool ok = mbar_wait(&sm.mbar_rec[b], uses[b] & 1u);
    uses[b]++;
    // window copies: bins [base, base + W) of row p; the in-profile part
    // [max(base, 0), min(base + W, N)) comes from the pairs row
    uint32_t bytes = 0;
    int mode = 0;
    for (int i = lane; i < nc; i += 32) {
        const int bits = __float_as_int(rec[i].b.w);
        const int base = bits >> 3, order = bits & 7;
        if (order == kOrderInvalid) continue;  // invalid pulse: window stays zero
        mode = max(mode, order);
        const int lo = max(base, 0), hi = min(base + W, N);
        if (hi > lo) bytes += (uint32_t)(hi - lo) * 16u;
    }
    for (int o = 16; o > 0; o >>= 1) {
        bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
        mode = max(mode, __shfl_xor_sync(0xffffffffu, mode, o));
    }
    // records as the consumers read them: four float4 of broadcast pairs;
    // the fourth holds the per-pulse products of the series terms the
    // chunk's mode uses (2 e^2 in mode 1, e^2 in mode 2, and e - e' =
    // -4 e^2 sigma0), or k_c R for the closed form (mode 3)
    float4 *r2 = sm.rec2 + (size_t)b * 4 * cmax;
    for (int i = lane; i < nc; i += 32) {
        const float4 a = rec[i].a, q = rec[i].b;
        r2[4 * i] = make_float4(a.x, a.x, a.y, a.y);
        r2[4 * i + 1] = make_float4(a.z, a.z, a.w, a.w);
        r2[4 * i + 2] = make_float4(q.x, q.x, q.y, q.y);
        const float ee = a.w * a.w;
        const float de = -4.0f * ee * q.y;
        const float e2 = mode == 1 ? ee + ee : ee;
        r2[4 * i + 3] = mode == 3 ? make_float4(q.z, 0.0f, de, de) : make_float4(e2, e2, de, de);
    }
    if (lane == 0) {
        sm.s_mode[b] = mode;
        mbar_expect(&sm.mbar_win[b], bytes);  // the arrival of this phase
    }
    __syncwarp();
    for (int i = lane; i < nc; i += 32) {
        const int bits = __float_as_int(rec[i].b.w);
        const int base = bits >> 3, order = bits & 7;
        const float4 *row = jb.Qp + (size_t)(p0 + i) * (N + 1);
        float4 *dst = win + i * W;
        if (order == kOrderInvalid) {
            for (int j = 0; j < W; ++j) dst[j] = make_float4(0.f, 0.f, 0.f, 0.f);
            continue;
        }
        const int lo = max(base, 0), hi = min(base + W, N);
        if (hi > lo) bulk_copy(dst + (lo - base), row + lo, (uint32_t)(hi - lo) * 16u, &sm.mbar_win[b]);
        // bins < 0 read Q[0] twice, bins >= N-1 read Q[N-1] twice (clamp)
        for (int j = 0; j < W && base + j < 0; ++j) dst[j] = row[N];
        for (int j = max(N - base, 0); j < W; ++j) dst[j] = row[N - 1];
    }
    ok = mbar_wait(&sm.mbar_win[b], uses[2 + b] & 1u) && ok;
    uses[2 + b]++;
    return ok;
}

// Producer warp: the same barrier sequence as the consumers.
__device__ __forceinline__ void producer_loop(const DevJob *__restrict__ jobs,
                                              const WorkItem *__restrict__ items, int nitems,
                                              int stage_cap, int cmax, int persistent, const TileSmem &sm) {
    const int lane = threadIdx.x & 31;
    // completed phases of each mbarrier: records [0..1], windows [2..3]
    uint32_t uses[4] = {0u, 0u, 0u, 0u};
    int item = blockIdx.x;
    for (;;) {
        if (persistent) {
            __syncthreads();  // s_item written
            item = *sm.s_item;
        }
        if (item >= nitems) break;
        const WorkItem wi = items[item];
        const DevJob &jb = jobs[wi.job];
        int pb, pe;  // the item's pulses
        part_range(jb.P, jb.nsplit, wi.part, pb, pe);
        const TileShape sh = tile_shape(jb.tiles[wi.tile], pe - pb, stage_cap, cmax);
        bool ok = true;
        for (int c = 0; c < sh.nchunks; ++c) {
            const int b = c & 1;
            if (c >= 2) bar_sync(kBarEmpty0 + b);  // consumers are done with chunk c-2
            const int p0 = pb + c * sh.C;
            ok = stage_chunk(jb, wi.tile, lane, p0, min(sh.C, pe - p0), b, sh, stage_cap, cmax, sm, uses) &&
                 ok;
            bar_arrive(kBarFull0 + b);
        }
        for (int c = sh.nchunks > 2 ? sh.nchunks - 2 : 0; c < sh.nchunks; ++c) bar_sync(kBarEmpty0 + (c & 1));
        if (!ok && lane == 0) atomicOr(&jb.sc->status, kStatusTimeout);
        __syncthreads();  // epilogue partials
        if (!persistent) break;
    }
}

template <int TX, int TY, bool PRE>
__device__ __forceinline__ void consumer_loop(const DevJob *__restrict__ jobs,
                                              const WorkItem *__restrict__ items, int nitems,
                                              int *__restrict__ counter, int stage_cap, int cmax,
                                              int persistent, const TileSmem &sm) {
    constexpr int PPT = TX * TY / kConsumers;
    constexpr int ROWS = kConsumers / TX;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int lx = tid % TX, ly = tid / TX;
    // pixel k of this thread: lanes run along x, or along y on transposed
    // tiles (square tiles whose range bins step faster along x than along y,
    // so that neighbouring lanes read neighbouring or equal window entries)
    auto pixel_of = [&](bool tr, int tx0, int ty0, int k, int &ix, int &iy) {
        if (TX == TY && tr) {
            ix = tx0 + ly + k * ROWS;
            iy = ty0 + lx;
        } else {
            ix = tx0 + lx;
            iy = ty0 + ly + k * ROWS;
        }
    };
    const uint32_t stage_base = smem_u32(sm.stage) - kMagicOff;
    int item = blockIdx.x;
    for (;;) {
        if (persistent) {
            if (tid == 0) *sm.s_item = atomicAdd(counter, 1);
            __syncthreads();
            item = *sm.s_item;
        }
        if (item >= nitems) break;
        const WorkItem wi = items[item];
        const DevJob &jb = jobs[wi.job];
        const int nu = jb.nu, nv = jb.nv, P = jb.P;
        const int tx0 = (wi.tile % jb.tiles_x) * TX;
        const int ty0 = (wi.tile / jb.tiles_x) * TY;
        const TileInfo ti = jb.tiles[wi.tile];
        int pb, pe;  // the item's pulses
        part_range(P, jb.nsplit, wi.part, pb, pe);
        const TileShape sh = tile_shape(ti, pe - pb, stage_cap, cmax);
        const double k_c = jb.sc->k_c;
        const float kcf = (float)k_c;

        // ---- pixel offsets from the tile centre, in radians ----
        float dx[PPT], dy[PPT], dz[PPT], nd2[PPT], s0[PPT];
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
            int ix, iy;
            pixel_of(ti.transposed != 0, tx0, ty0, k, ix, iy);
            dx[k] = dy[k] = dz[k] = nd2[k] = s0[k] = 0.0f;
            if (ix < nu && iy < nv) {
                double x, y, z;
                if (jb.r) {
                    const long long npix = (long long)nu * nv;
                    const long long pix = (long long)iy * nu + ix;
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
                if (isfinite(x) && isfinite(y) && isfinite(z)) {
                    // the same f32 offsets the tile set-up measured rho on
                    dx[k] = kcf * (float)(x - ti.rc[0]);
                    dy[k] = kcf * (float)(y - ti.rc[1]);
                    dz[k] = kcf * (float)(z - ti.rc[2]);
                    nd2[k] = -fmaf(dx[k], dx[k], fmaf(dy[k], dy[k], dz[k] * dz[k]));
                    s0[k] = fmaf(ti.w0[2], dz[k], fmaf(ti.w0[1], dy[k], ti.w0[0] * dx[k]));
                }
            }
        }
        // pixel pairs (2j, 2j + 1) for the f32x2 arithmetic
        constexpr int NP = PPT / 2;
        float2 dxp[NP], dyp[NP], dzp[NP], nd2p[NP], s0p[NP], arp[NP], aip[NP];
#pragma unroll
        for (int j = 0; j < NP; ++j) {
            dxp[j] = make_float2(dx[2 * j], dx[2 * j + 1]);
            dyp[j] = make_float2(dy[2 * j], dy[2 * j + 1]);
            dzp[j] = make_float2(dz[2 * j], dz[2 * j + 1]);
            nd2p[j] = make_float2(nd2[2 * j], nd2[2 * j + 1]);
            s0p[j] = make_float2(s0[2 * j], s0[2 * j + 1]);
            arp[j] = aip[j] = make_float2(0.0f, 0.0f);
        }
        if (sh.C < 1) {
            if (tid == 0) atomicOr(&jb.sc->status, kStatusTileTooWide);
        } else {
            const float ilk = (float)(jb.inv_lsr / k_c);  // range bins per radian of Delta
            const float2 ILK = make_float2(ilk, ilk);
            const float2 CL = f2(0.0f, (float)(sh.W - 1) - 0.5f);  // bin-argument clamp (modes 2, 3)
            const uint32_t pstride = (uint32_t)sh.W * 16u;
            for (int c = 0; c < sh.nchunks; ++c) {
                const int b = c & 1;
                bar_sync(kBarFull0 + b);
                const int p0 = pb + c * sh.C;
                const uint32_t poff = stage_base + (uint32_t)(b * stage_cap) * 16u;
                const int nc = min(sh.C, pe - p0);
                const float4 *rec2 = sm.rec2 + (size_t)b * 4 * cmax;
                if (ti.wide)
                    accumulate_mode<true, NP, PRE>(sm.s_mode[b], ti.planar != 0, nc, rec2, poff, pstride, ILK, CL,
                                              dxp, dyp, dzp, nd2p, s0p, arp, aip);
                else
                    accumulate_mode<false, NP, PRE>(sm.s_mode[b], ti.planar != 0, nc, rec2, poff, pstride, ILK, CL,
                                               dxp, dyp, dzp, nd2p, s0p, arp, aip);
                bar_arrive(kBarEmpty0 + b);
            }
        }
        // ---- final phase, row flip (backprojection.cpp:130-138), max|z|;
        // a pulse part stores its sums into its slice, a pulse chunk adds
        // them to the partial image instead ----
        double zmax = 0.0;
        if (jb.nsplit > 1) {
            float2 *slice = jb.parts + (long long)wi.part * ((long long)nu * nv);
#pragma unroll
            for (int k = 0; k < PPT; ++k) {
                int ix, iy;
                pixel_of(ti.transposed != 0, tx0, ty0, k, ix, iy);
                if (ix < nu && iy < nv)
                    slice[(long long)iy * nu + ix] = make_float2((k & 1) ? arp[k >> 1].y : arp[k >> 1].x,
                                                                 (k & 1) ? aip[k >> 1].y : aip[k >> 1].x);
            }
        } else if (jb.acc) {
#pragma unroll
            for (int k = 0; k < PPT; ++k) {
                int ix, iy;
                pixel_of(ti.transposed != 0, tx0, ty0, k, ix, iy);
                if (ix < nu && iy < nv) {
                    float2 *a = jb.acc + (long long)iy * nu + ix;
                    const float2 s = *a;
                    *a = make_float2(s.x + ((k & 1) ? arp[k >> 1].y : arp[k >> 1].x),
                                     s.y + ((k & 1) ? aip[k >> 1].y : aip[k >> 1].x));
                }
            }
        } else
#pragma unroll
        for (int k = 0; k < PPT; ++k) {
            int ix, iy;
            pixel_of(ti.transposed != 0, tx0, ty0, k, ix, iy);
            if (ix < nu && iy < nv) {
                const float2 f = jb.fin[(long long)iy * nu + ix];
                const float ark = (k & 1) ? arp[k >> 1].y : arp[k >> 1].x;
                const float aik = (k & 1) ? aip[k >> 1].y : aip[k >> 1].x;
                const double zr = (double)fmaf(ark, f.x, -aik * f.y);
                const double zi = (double)fmaf(ark, f.y, aik * f.x);
                jb.out[(long long)(nv - 1 - iy) * nu + ix] = make_double2(zr, zi);
                zmax = fmax(zmax, sqrt(zr * zr + zi * zi));
            }
        }
        zmax = warp_max(zmax);
        if (lane == 0) sm.sred[warp] = zmax;
        __syncthreads();
        if (tid == 0 && !jb.acc && jb.nsplit <= 1) {
            double m = 0.0;
            for (int w = 0; w < kConsumerWarps; ++w) m = fmax(m, sm.sred[w]);
            atomicMax(&jb.sc->maxabs, (unsigned long long)__double_as_longlong(m));
        }
        if (!persistent) break;
    }
}

// MINB: CTAs per SM the register allocation targets (2 or 3).  The role
// test reads the thread index through a shuffle from lane 0 so the compiler
// sees a warp-uniform branch and allocates the two roles' registers apart.
template <int TX, int TY, int MINB>
__global__ void __launch_bounds__(kThreads, MINB) bp_tile_kernel(const DevJob *__restrict__ jobs,
                                                                 const WorkItem *__restrict__ items,
                                                                 int nitems, int *__restrict__ counter,
                                                                 int stage_cap, int cmax, int persistent) {
    static_assert(TX * TY % (2 * kConsumers) == 0, "tile must give each consumer pairs of pixels");
    extern __shared__ float4 smem[];
    __shared__ double sred[kConsumerWarps];
    __shared__ int s_item, s_mode[2];
    __shared__ uint64_t mbar[4];
    TileSmem sm;
    sm.stage = smem;
    sm.raw = reinterpret_cast<PulseRec *>(smem + 2 * stage_cap);
    sm.rec2 = smem + 2 * stage_cap + 2 * cmax;
    sm.mbar_rec = mbar;
    sm.mbar_win = mbar + 2;
    sm.sred = sred;
    sm.s_item = &s_item;
    sm.s_mode = s_mode;
    if (threadIdx.x == kConsumers) {
        for (int i = 0; i < 4; ++i)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[i])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (__shfl_sync(0xffffffffu, (int)threadIdx.x, 0) >= kConsumers)
        producer_loop(jobs, items, nitems, stage_cap, cmax, persistent, sm);
    else
        consumer_loop<TX, TY, (MINB >= 3)>(jobs, items, nitems, counter, stage_cap, cmax, persistent, sm);
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
        // pair l holds (m, d) of bins (l, l+1); below the profile it is (Q[0], 0)
        const float4 md = __ldg(&jb.Qp[(size_t)p * (N + 1) + (l < 0 ? N : min(l, N - 1))]);
        const float vr = fmaf(w - 0.5f, md.z, md.x), vi = fmaf(w - 0.5f, md.w, md.y);
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
    double m = sqrt(zr * zr + zi * zi);
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(__activemask(), m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&jb.sc->maxabs, (unsigned long long)__double_as_longlong(m));
}

template <int TX, int TY, int MINB>
cudaError_t set_attr(size_t smem) {
    return cudaFuncSetAttribute(bp_tile_kernel<TX, TY, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem);
}

template <int TX, int TY, int MINB>
int active_blocks(size_t smem) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, bp_tile_kernel<TX, TY, MINB>, kThreads, smem) !=
        cudaSuccess)
        return 0;
    return n;
}

}  // namespace

// (tile width, tile height, CTAs per SM) instantiations of bp_tile_kernel
// tiles of an even number of pixels per consumer thread (pairs)
#define SARBP_BP_TILES(X)                                                                  \
    X(32, 16, 2) X(32, 32, 2) X(32, 64, 2) X(64, 16, 2) X(64, 32, 2) X(16, 32, 2) X(16, 64, 2) \
    X(32, 16, 3) X(32, 32, 3) X(64, 16, 3) X(16, 32, 3)

bool bp_tile_supported(int tx, int ty, int minb) {
#define X(a, b, m) \
    if (tx == a && ty == b && minb == m) return true;
    SARBP_BP_TILES(X)
#undef X
    return false;
}

size_t bp_smem_bytes(const BpLaunch &L) {
    return 2 * (size_t)L.stage_cap * sizeof(float4) + (size_t)L.cmax * sizeof(PulseRec) +
           8 * (size_t)L.cmax * sizeof(float4);
}

cudaError_t init_backproject_attributes() {
    const size_t maxs = 220 * 1024;
    cudaError_t e = cudaSuccess;
#define X(a, b, m) \
    if (e == cudaSuccess) e = set_attr<a, b, m>(maxs);
    SARBP_BP_TILES(X)
#undef X
    return e;
}

int bp_max_active_blocks(const BpLaunch &L) {
    const size_t smem = bp_smem_bytes(L);
#define X(a, b, m) \
    if (L.tile_x == a && L.tile_y == b && L.minb == m) return active_blocks<a, b, m>(smem);
    SARBP_BP_TILES(X)
#undef X
    return 0;
}

cudaError_t launch_backproject(const BpLaunch &L, const DevJob *d_jobs, const WorkItem *d_items,
                               int nitems, int *d_counter, cudaStream_t st) {
    const size_t smem = bp_smem_bytes(L);
    const int grid = L.persistent ? L.grid : nitems;
    if (grid <= 0) return cudaSuccess;
#define X(a, b, m)                                                                                \
    if (L.tile_x == a && L.tile_y == b && L.minb == m) {                                          \
        bp_tile_kernel<a, b, m><<<grid, kThreads, smem, st>>>(d_jobs, d_items, nitems, d_counter, \
                                                              L.stage_cap, L.cmax, L.persistent); \
        return cudaGetLastError();                                                                \
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
