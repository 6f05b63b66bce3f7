// range_compress.cu -- fused range compression, one kernel per N_fft.
//
// Replaces backprojection.cpp:79-104 and the FFTW extern (dft.cpp:40-79):
// for each output pulse row p of each job
//   src     = (p + 2*ceil(P/2)) mod P     (fftshift over the pulse axis,
//                                          applied twice: :98 and :104;
//                                          src = p for a pulse chunk, whose
//                                          rows come in phase-history order)
//   x[n]    = phs[src][s] * |k_r[s]| * wS[s] * wP[src],
//             s = ((n + N/2) mod N) - (N - S)/2, zero outside [0, S)
//                                         (window, filter, pad, fftshift)
//   X       = forward DFT of x             (FFTW_FORWARD, dft.cpp:26)
//   Q[p][k] = X[(k + N/2) mod N]           (fftshift on store)
//
// The DFT is a Stockham auto-sort FFT: N/16 threads per row, 16 complex
// values per thread in registers, radix-16 passes (one leading radix-2/4/8
// pass when log2 N is not a multiple of 4), rows exchanged through padded
// shared memory between passes.  Twiddles come from a per-N table laid out
// [r-1][j mod Ns] per pass so a warp's loads are contiguous.
#include "internal.h"
#include "kernels.h"

namespace sarbp {

namespace {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

// W_16^j = exp(-2 pi i j / 16), j in [0, 8)
__device__ __forceinline__ float2 w16(int j) {
    constexpr float c1 = 0.92387953251128674f, s1 = 0.38268343236508977f,
                    h = 0.70710678118654752f;
    switch (j) {
        case 0: return make_float2(1.f, 0.f);
        case 1: return make_float2(c1, -s1);
        case 2: return make_float2(h, -h);
        case 3: return make_float2(s1, -c1);
        case 4: return make_float2(0.f, -1.f);
        case 5: return make_float2(-s1, -c1);
        case 6: return make_float2(-h, -h);
        default: return make_float2(-c1, -s1);
    }
}

__host__ __device__ constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n >> 1); }

// In-register forward DFT of R points v[B..B+R), natural order in and out:
// log2(R) self-sorting (Stockham) radix-2 stages, every index an affine
// function of unrolled loop counters so the values stay in registers.
template <int R, int B>
__device__ __forceinline__ void dft_reg(float2 (&v)[16]) {
    float2 x[R], y[R];
#pragma unroll
    for (int i = 0; i < R; ++i) x[i] = v[B + i];
#pragma unroll
    for (int ns = 1; ns < R; ns <<= 1) {
#pragma unroll
        for (int j = 0; j < R / 2; ++j) {
            const int k = j & (ns - 1);
            const int tw = k * (8 / ns);  // W_{2ns}^k = W_16^(8k/ns)
            const float2 a = x[j];
            float2 b = x[j + R / 2];
            if (tw == 4) {
                b = make_float2(b.y, -b.x);  // * (-i)
            } else if (tw != 0) {
                b = cmul(b, w16(tw));
            }
            const int o = (j / ns) * 2 * ns + k;
            y[o] = make_float2(a.x + b.x, a.y + b.y);
            y[o + ns] = make_float2(a.x - b.x, a.y - b.y);
        }
#pragma unroll
        for (int i = 0; i < R; ++i) x[i] = y[i];
    }
#pragma unroll
    for (int i = 0; i < R; ++i) v[B + i] = x[i];
}

__device__ __forceinline__ int pad_idx(int i) { return i + (i >> 4); }

template <int N, int R, int NS>
struct Pass {
    static constexpr int T = N / 16;   // threads per row
    static constexpr int NB = 16 / R;  // butterflies per thread
};

// twiddle + butterflies of one pass on a thread's 16 values
template <int N, int R, int NS>
__device__ __forceinline__ void pass_compute(float2 (&v)[16], int t, const float2 *__restrict__ tw) {
    constexpr int T = Pass<N, R, NS>::T, NB = Pass<N, R, NS>::NB;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        if constexpr (NS > 1) {
            const int jm = (t + b * T) & (NS - 1);
#pragma unroll
            for (int r = 1; r < R; ++r) v[b * R + r] = cmul(v[b * R + r], __ldg(&tw[(r - 1) * NS + jm]));
        }
    }
    if constexpr (NB == 1) {
        dft_reg<R, 0>(v);
    } else if constexpr (NB == 2) {
        dft_reg<R, 0>(v); dft_reg<R, R>(v);
    } else if constexpr (NB == 4) {
        dft_reg<R, 0>(v); dft_reg<R, R>(v); dft_reg<R, 2 * R>(v); dft_reg<R, 3 * R>(v);
    } else {
        dft_reg<R, 0>(v); dft_reg<R, 2>(v); dft_reg<R, 4>(v); dft_reg<R, 6>(v);
        dft_reg<R, 8>(v); dft_reg<R, 10>(v); dft_reg<R, 12>(v); dft_reg<R, 14>(v);
    }
}

template <int N, int R, int NS>
__device__ __forceinline__ void pass_store_smem(const float2 (&v)[16], int t, float2 *sm) {
    constexpr int T = Pass<N, R, NS>::T, NB = Pass<N, R, NS>::NB;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        const int j = t + b * T;
        const int base = (j / NS) * NS * R + (j & (NS - 1));
#pragma unroll
        for (int r = 0; r < R; ++r) sm[pad_idx(base + r * NS)] = v[b * R + r];
    }
}

template <int N, int R>
__device__ __forceinline__ void pass_load_smem(float2 (&v)[16], int t, const float2 *sm) {
    constexpr int T = N / 16, NB = 16 / R;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        const int j = t + b * T;
#pragma unroll
        for (int r = 0; r < R; ++r) v[b * R + r] = sm[pad_idx(j + r * (N / R))];
    }
}

// Radix schedule: R0 = 2^(log2 N mod 4) first (if not 1), then radix 16.
template <int N>
struct Plan {
    static constexpr int L = ilog2(N);
    static constexpr int R0 = 1 << (L % 4);  // 1 means no leading pass
};

// Recursive radix-16 passes; pass index K has NS = R0 * 16^K.  The last
// pass stores with the fftshift, either the profile itself (qrow) or, with
// `pairs`, the interpolation pairs (m, d) = ((Q[k] + Q[k+1]) / 2,
// Q[k+1] - Q[k]) with Q[N] read as Q[N-1] (the reference's index clamp),
// followed by (Q[0], 0) at index N.
template <int N, int NS>
__device__ __forceinline__ void passes16(float2 (&v)[16], int t, float2 *sm, const float2 *tw_base,
                                         int tw_off, float2 *__restrict__ qrow, float4 *__restrict__ prow,
                                         bool pairs) {
    constexpr int R = 16;
    const float2 *tw = tw_base + tw_off;
    pass_compute<N, R, NS>(v, t, tw);
    if constexpr (NS * R == N) {
        // last pass: j < NS, out index k = j + r*NS, stored with fftshift
        const int j = t;
        if (pairs) {
            __syncthreads();
#pragma unroll
            for (int r = 0; r < R; ++r) sm[pad_idx((j + r * NS + N / 2) & (N - 1))] = v[r];
            __syncthreads();
            if (prow != nullptr) {
#pragma unroll
                for (int u = 0; u < R; ++u) {
                    const int k = t + u * NS;
                    const float2 a = sm[pad_idx(k)];
                    const float2 b = sm[pad_idx(k + 1 < N ? k + 1 : N - 1)];
                    prow[k] = make_float4(0.5f * (a.x + b.x), 0.5f * (a.y + b.y), b.x - a.x, b.y - a.y);
                }
                if (t == 0) {
                    const float2 a = sm[pad_idx(0)];
                    prow[N] = make_float4(a.x, a.y, 0.f, 0.f);
                }
            }
        } else if (qrow != nullptr) {
#pragma unroll
            for (int r = 0; r < R; ++r) qrow[(j + r * NS + N / 2) & (N - 1)] = v[r];
        }
    } else {
        __syncthreads();
        pass_store_smem<N, R, NS>(v, t, sm);
        __syncthreads();
        pass_load_smem<N, R>(v, t, sm);
        passes16<N, NS * R>(v, t, sm, tw_base, tw_off + (NS > 1 ? (R - 1) * NS : 0), qrow, prow, pairs);
    }
}

template <int LOGN>
__global__ void __launch_bounds__((1 << LOGN) / 16 > 256 ? (1 << LOGN) / 16 : 256)
range_compress_kernel(const DevJob *__restrict__ jobs, const RowItem *__restrict__ rows, int nrows,
                      const float2 *__restrict__ tw, int pairs) {
    constexpr int N = 1 << LOGN;
    constexpr int T = N / 16;
    constexpr int RPB = T >= 256 ? 1 : 256 / T;
    constexpr int R0 = Plan<N>::R0;
    extern __shared__ float2 smem_all[];
    const int lrow = threadIdx.x / T;
    const int t = threadIdx.x % T;
    const int grow = blockIdx.x * RPB + lrow;
    const bool live = grow < nrows;
    float2 *sm = smem_all + lrow * (N + N / 16);

    RowItem it = live ? rows[grow] : RowItem{0, 0};
    const DevJob &jb = jobs[it.job];
    const int S = jb.S, P = jb.P, p = it.pulse;
    const int pm = P / 2 + P % 2;
    const int src = jb.chunked ? p : (int)(((long long)p + 2 * pm) % P);
    const int x_pad = (N - S) >> 1;  // floor division by 2
    const float2 *__restrict__ ph = jb.phs + (size_t)src * S;
    const float wp = live ? jb.wP[src] : 0.f;

    // first pass input: radix R1 (R0, or 16 when R0 == 1) with NS = 1
    constexpr int R1 = R0 > 1 ? R0 : 16;
    constexpr int NB1 = 16 / R1;
    float2 v[16];
#pragma unroll
    for (int b = 0; b < NB1; ++b) {
        const int j = t + b * T;
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            const int n = j + r * (N / R1);
            const int s = ((n + N / 2) & (N - 1)) - x_pad;
            float2 x = make_float2(0.f, 0.f);
            if (live && s >= 0 && s < S) {
                const float2 a = __ldg(&ph[s]);
                const float f = __ldg(&jb.filt[s]);
                const float w = __ldg(&jb.wS[s]) * wp;
                x = make_float2((a.x * f) * w, (a.y * f) * w);
            }
            v[b * R1 + r] = x;
        }
    }
    float2 *__restrict__ qrow = (live && !pairs) ? jb.Q + (size_t)p * N : nullptr;
    float4 *__restrict__ prow = (live && pairs) ? jb.Qp + (size_t)p * (N + 1) : nullptr;
    if constexpr (R0 > 1) {
        pass_compute<N, R0, 1>(v, t, tw);
        __syncthreads();
        pass_store_smem<N, R0, 1>(v, t, sm);
        __syncthreads();
        pass_load_smem<N, 16>(v, t, sm);
        passes16<N, R0>(v, t, sm, tw, 0, qrow, prow, pairs != 0);
    } else {
        // first radix-16 pass has NS = 1 and no twiddles
        passes16<N, 1>(v, t, sm, tw, 0, qrow, prow, pairs != 0);
    }
}

}  // namespace

// Twiddle table of one N: for each pass with NS > 1, entries
// W_{NS*R}^{jm*r} at [(r-1)*NS + jm], passes concatenated in order.
int twiddle_table_size(int logN) {
    const int N = 1 << logN;
    const int R0 = 1 << (logN % 4);
    int ns = R0 > 1 ? R0 : 1;
    int total = 0;
    if (R0 == 1) ns = 16;  // first radix-16 pass has no table
    while (ns < N) {
        total += 15 * ns;
        ns *= 16;
    }
    return total;
}

void fill_twiddle_table(int logN, float2 *host) {
    const int N = 1 << logN;
    const int R0 = 1 << (logN % 4);
    int ns = R0 > 1 ? R0 : 16;
    int off = 0;
    while (ns < N) {
        const int R = 16;
        for (int r = 1; r < R; ++r)
            for (int jm = 0; jm < ns; ++jm) {
                const long long e = (long long)jm * r;
                const double a = -2.0 * 3.14159265358979323846 * (double)e / (double)(ns * R);
                host[off + (r - 1) * ns + jm] = make_float2((float)cos(a), (float)sin(a));
            }
        off += 15 * ns;
        ns *= 16;
    }
}

template <int LOGN>
static cudaError_t launch_rc(const DevJob *d_jobs, const RowItem *d_rows, int nrows, int pairs,
                             const float2 *d_tw, cudaStream_t st) {
    constexpr int N = 1 << LOGN;
    constexpr int T = N / 16;
    constexpr int RPB = T >= 256 ? 1 : 256 / T;
    const int threads = RPB * T;
    const size_t smem = (size_t)RPB * (N + N / 16) * sizeof(float2);
    const int blocks = (nrows + RPB - 1) / RPB;
    range_compress_kernel<LOGN><<<blocks, threads, smem, st>>>(d_jobs, d_rows, nrows, d_tw, pairs);
    return cudaGetLastError();
}

template <int LOGN>
static cudaError_t rc_attr() {
    constexpr int N = 1 << LOGN;
    constexpr int T = N / 16;
    constexpr int RPB = T >= 256 ? 1 : 256 / T;
    const size_t smem = (size_t)RPB * (N + N / 16) * sizeof(float2);
    return cudaFuncSetAttribute(range_compress_kernel<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem);
}

cudaError_t init_range_compress_attributes() {
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = rc_attr<4>();
    if (e == cudaSuccess) e = rc_attr<5>();
    if (e == cudaSuccess) e = rc_attr<6>();
    if (e == cudaSuccess) e = rc_attr<7>();
    if (e == cudaSuccess) e = rc_attr<8>();
    if (e == cudaSuccess) e = rc_attr<9>();
    if (e == cudaSuccess) e = rc_attr<10>();
    if (e == cudaSuccess) e = rc_attr<11>();
    if (e == cudaSuccess) e = rc_attr<12>();
    if (e == cudaSuccess) e = rc_attr<13>();
    if (e == cudaSuccess) e = rc_attr<14>();
    return e;
}

cudaError_t launch_range_compress(int logN, const DevJob *d_jobs, const RowItem *d_rows, int nrows, int pairs,
                                  const float2 *d_tw, cudaStream_t st) {
    switch (logN) {
        case 4: return launch_rc<4>(d_jobs, d_rows, nrows, pairs, d_tw, st);
        case 5: return launch_rc<5>(d_jobs, d_rows, nrows, pairs, d_tw, st);
        case 6: return launch_rc<6>(d_jobs, d_rows, nrows, pairs, d_tw, st);
        case 7: return launch_rc<7>(d_jobs, d_rows, nrows, pairs, d_tw, st);
        case 8: return launch_rc<8>(d_jobs, d_rows, nrows, pairs, d_tw, st);
        case 9: return launch_rc<9>(d_jobs, d_rows, nrows, pairs, d_tw, st);
        case 10: return launch_rc<10>(d_jobs, d_rows, nrows, pairs, d_tw, st);
        case 11: return launch_rc<11>(d_jobs, d_rows, nrows, pairs, d_tw, st);
        case 12: return launch_rc<12>(d_jobs, d_rows, nrows, pairs, d_tw, st);
        case 13: return launch_rc<13>(d_jobs, d_rows, nrows, pairs, d_tw, st);
        case 14: return launch_rc<14>(d_jobs, d_rows, nrows, pairs, d_tw, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace sarbp
