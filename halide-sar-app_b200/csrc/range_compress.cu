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
// [r-1][j mod Ns] per pass so a warp's loads are contiguous.  Up to
// N = 2^kMaxLogNSmem one CTA holds a whole row; above it (the reference
// sizes N_fft = 2^(floor(log2(S * upsample)) + 1), sarbp.cpp:258, so 8192
// samples at -u 2 need 32768) the DFT is a four-step FFT of two such
// sub-DFTs through a work buffer (see rc_cols_kernel / rc_rows_kernel).
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

// ---- N_fft above 2^kMaxLogNSmem: four-step FFT through a work buffer ----
// With N = N1 N2, n = N2 n1 + n2 and k = k1 + N1 k2 (Cooley-Tukey):
//   Y[n2][k1]     = W_N^(n2 k1) * DFT_N1 over n1 of x[N2 n1 + n2]  (columns)
//   X[k1 + N1 k2] = DFT_N2 over n2 of Y[n2][k1]                     (rows)
// The columns kernel writes Y to work[row][k1][n2]; the rows kernel stores
// with the fftshift, Q[j] = X[(j + N/2) mod N] at j = k1 + N1 k2',
// k2' = (k2 + N2/2) mod N2.  Both sub-DFTs run the radix-16 passes above on
// rows of shared memory, one CTA holding several columns (stride STR, one
// float2 more than a padded row so that neighbouring columns fall in other
// banks).

// The passes of one sub-DFT; on return thread t holds X[t + r N/16] in v[r].
template <int N, int NS>
__device__ __forceinline__ void passes16_regs(float2 (&v)[16], int t, float2 *sm, const float2 *tw_base,
                                              int tw_off) {
    pass_compute<N, 16, NS>(v, t, tw_base + tw_off);
    if constexpr (NS * 16 < N) {
        __syncthreads();
        pass_store_smem<N, 16, NS>(v, t, sm);
        __syncthreads();
        pass_load_smem<N, 16>(v, t, sm);
        passes16_regs<N, NS * 16>(v, t, sm, tw_base, tw_off + (NS > 1 ? 15 * NS : 0));
    }
}

// Loads a sub-DFT's first-pass inputs from its shared row (as the single-row
// kernel loads them from global memory) and runs all passes.
template <int N>
__device__ __forceinline__ void fft_row_regs(float2 (&v)[16], int t, float2 *sm, const float2 *tw) {
    constexpr int T = N / 16, R0 = Plan<N>::R0, R1 = R0 > 1 ? R0 : 16, NB1 = 16 / R1;
#pragma unroll
    for (int b = 0; b < NB1; ++b)
#pragma unroll
        for (int r = 0; r < R1; ++r) v[b * R1 + r] = sm[pad_idx(t + b * T + r * (N / R1))];
    if constexpr (R0 > 1) {
        pass_compute<N, R0, 1>(v, t, tw);
        __syncthreads();
        pass_store_smem<N, R0, 1>(v, t, sm);
        __syncthreads();
        pass_load_smem<N, 16>(v, t, sm);
        passes16_regs<N, R0>(v, t, sm, tw, 0);
    } else {
        __syncthreads();  // every thread has read its inputs before the first store
        passes16_regs<N, 1>(v, t, sm, tw, 0);
    }
}

template <int L1>
struct ColsShape {
    static constexpr int N1 = 1 << L1, T = N1 / 16, C = 256 / T, STR = N1 + N1 / 16 + 1;
};
template <int L2>
struct RowsShape {
    static constexpr int N2 = 1 << L2, T = N2 / 16, C = 256 / T, STR = N2 + N2 / 16 + 1;
};

// Columns: one CTA per (row, C consecutive n2); rows [row0, row0 + grid/groups).
template <int L1>
__global__ void __launch_bounds__(256)
rc_cols_kernel(const DevJob *__restrict__ jobs, const RowItem *__restrict__ rows, int row0, int logN,
               const float2 *__restrict__ tw1, const float2 *__restrict__ twN, float2 *__restrict__ work) {
    using Sh = ColsShape<L1>;
    constexpr int N1 = Sh::N1, T = Sh::T, C = Sh::C, STR = Sh::STR;
    extern __shared__ float2 smem_all[];
    const int N = 1 << logN, N2 = N >> L1, groups = N2 / C;
    const int rb = blockIdx.x / groups, n2_0 = (blockIdx.x % groups) * C;
    const RowItem it = rows[row0 + rb];
    const DevJob &jb = jobs[it.job];
    const int S = jb.S, P = jb.P, p = it.pulse;
    const int pm = P / 2 + P % 2;
    const int src = jb.chunked ? p : (int)(((long long)p + 2 * pm) % P);
    const int x_pad = (N - S) >> 1;
    const float2 *__restrict__ ph = jb.phs + (size_t)src * S;
    const float wp = jb.wP[src];
    // window * filter * pad * fftshift of x[N2 n1 + n2], lanes along n2
    for (int i = threadIdx.x; i < N1 * C; i += blockDim.x) {
        const int c = i % C, n1 = i / C;
        const int s = ((n1 * N2 + n2_0 + c + N / 2) & (N - 1)) - x_pad;
        float2 x = make_float2(0.f, 0.f);
        if (s >= 0 && s < S) {
            const float2 a = __ldg(&ph[s]);
            const float f = __ldg(&jb.filt[s]);
            const float w = __ldg(&jb.wS[s]) * wp;
            x = make_float2((a.x * f) * w, (a.y * f) * w);
        }
        smem_all[c * STR + pad_idx(n1)] = x;
    }
    __syncthreads();
    const int c = threadIdx.x / T, t = threadIdx.x % T;
    float2 *sm = smem_all + c * STR;
    float2 v[16];
    fft_row_regs<N1>(v, t, sm, tw1);
    const int n2 = n2_0 + c;
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = cmul(v[r], __ldg(&twN[n2 * (t + r * T)]));
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 16; ++r) sm[pad_idx(t + r * T)] = v[r];
    __syncthreads();
    float2 *__restrict__ wrow = work + (size_t)rb * N;
    for (int i = threadIdx.x; i < N1 * C; i += blockDim.x) {
        const int cc = i % C, k1 = i / C;
        wrow[(size_t)k1 * N2 + n2_0 + cc] = smem_all[cc * STR + pad_idx(k1)];
    }
}

// Rows: one CTA per (row, C consecutive k1), plus the next column k1_0 + C
// (column 0 after the last group) for the pairs' right neighbours:
// Q[j + 1] is column k1 + 1 at the same k2', or column 0 at k2' + 1 when
// k1 = N1 - 1, and Q[N] is read as Q[N - 1] (the reference's clamp).
template <int L2>
__global__ void __launch_bounds__(288)
rc_rows_kernel(const DevJob *__restrict__ jobs, const RowItem *__restrict__ rows, int row0, int logN,
               const float2 *__restrict__ tw2, const float2 *__restrict__ work, int pairs) {
    using Sh = RowsShape<L2>;
    constexpr int N2 = Sh::N2, T = Sh::T, C = Sh::C, STR = Sh::STR;
    extern __shared__ float2 smem_all[];
    const int N = 1 << logN, N1 = N >> L2, groups = N1 / C;
    const int rb = blockIdx.x / groups, k1_0 = (blockIdx.x % groups) * C;
    const RowItem it = rows[row0 + rb];
    const DevJob &jb = jobs[it.job];
    const int p = it.pulse;
    const float2 *__restrict__ wrow = work + (size_t)rb * N;
    for (int i = threadIdx.x; i < (C + 1) * N2; i += blockDim.x) {
        const int c = i / N2, n2 = i % N2;
        const int k1 = (k1_0 + c) & (N1 - 1);
        smem_all[c * STR + pad_idx(n2)] = wrow[(size_t)k1 * N2 + n2];
    }
    __syncthreads();
    const int c = threadIdx.x / T, t = threadIdx.x % T;
    float2 *sm = smem_all + c * STR;
    float2 v[16];
    fft_row_regs<N2>(v, t, sm, tw2);
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 16; ++r) sm[pad_idx((t + r * T + N2 / 2) & (N2 - 1))] = v[r];
    __syncthreads();
    if (pairs) {
        float4 *__restrict__ prow = jb.Qp + (size_t)p * (N + 1);
        for (int i = threadIdx.x; i < C * N2; i += blockDim.x) {
            const int cc = i % C, k2 = i / C, k1 = k1_0 + cc;
            const float2 a = smem_all[cc * STR + pad_idx(k2)];
            float2 b = a;
            if (k1 + 1 < N1) b = smem_all[(cc + 1) * STR + pad_idx(k2)];
            else if (k2 + 1 < N2) b = smem_all[C * STR + pad_idx(k2 + 1)];
            prow[(size_t)k1 + (size_t)N1 * k2] =
                make_float4(0.5f * (a.x + b.x), 0.5f * (a.y + b.y), b.x - a.x, b.y - a.y);
        }
        if (k1_0 == 0 && threadIdx.x == 0) {
            const float2 a = smem_all[pad_idx(0)];
            prow[N] = make_float4(a.x, a.y, 0.f, 0.f);
        }
    } else {
        float2 *__restrict__ qrow = jb.Q + (size_t)p * N;
        for (int i = threadIdx.x; i < C * N2; i += blockDim.x) {
            const int cc = i % C, k2 = i / C;
            qrow[(size_t)(k1_0 + cc) + (size_t)N1 * k2] = smem_all[cc * STR + pad_idx(k2)];
        }
    }
}

template <int L1, int L2>
cudaError_t launch_four_step(int logN, const DevJob *d_jobs, const RowItem *d_rows, int nrows, int pairs,
                             const float2 *tw1, const float2 *tw2, const float2 *twN, float2 *work,
                             int rb, cudaStream_t st) {
    using A = ColsShape<L1>;
    using B = RowsShape<L2>;
    static_assert(L1 + L2 >= 15 && (1 << L2) >= A::C && (1 << L1) >= B::C, "four-step split");
    const size_t smem_a = (size_t)A::C * A::STR * sizeof(float2);
    const size_t smem_b = (size_t)(B::C + 1) * B::STR * sizeof(float2);
    for (int r0 = 0; r0 < nrows; r0 += rb) {
        const int nb = nrows - r0 < rb ? nrows - r0 : rb;
        rc_cols_kernel<L1><<<nb * ((1 << L2) / A::C), A::C * A::T, smem_a, st>>>(d_jobs, d_rows, r0, logN, tw1,
                                                                               twN, work);
        rc_rows_kernel<L2><<<nb * ((1 << L1) / B::C), (B::C + 1) * B::T, smem_b, st>>>(d_jobs, d_rows, r0, logN,
                                                                                     tw2, work, pairs);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace

// Twiddle table of one N: for each pass with NS > 1, entries
// W_{NS*R}^{jm*r} at [(r-1)*NS + jm], passes concatenated in order.  Above
// 2^kMaxLogNSmem (four-step FFTs) the table is W_N^m, m in [0, N).
int twiddle_table_size(int logN) {
    const int N = 1 << logN;
    if (logN > kMaxLogNSmem) return N;
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
    if (logN > kMaxLogNSmem) {
        for (int m = 0; m < N; ++m) {
            const double a = -2.0 * 3.14159265358979323846 * (double)m / (double)N;
            host[m] = make_float2((float)cos(a), (float)sin(a));
        }
        return;
    }
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

int rc_work_rows(int logN) {
    // about 256 MB of work buffer (2^25 complex values)
    return logN > kMaxLogNSmem ? (logN >= 25 ? 1 : 1 << (25 - logN)) : 0;
}

size_t rc_work_bytes(int logN) {
    return logN > kMaxLogNSmem ? (size_t)rc_work_rows(logN) * ((size_t)1 << logN) * sizeof(float2) : 0;
}

cudaError_t launch_range_compress_large(int logN, const DevJob *d_jobs, const RowItem *d_rows, int nrows,
                                        int pairs, const float2 *tw1, const float2 *tw2, const float2 *twN,
                                        float2 *work, int work_rows, cudaStream_t st) {
    if (nrows <= 0) return cudaSuccess;
    if (!tw1 || !tw2 || !twN || !work || work_rows < 1) return cudaErrorInvalidValue;
    const int rb = work_rows;
    switch (logN) {
        case 15: return launch_four_step<7, 8>(logN, d_jobs, d_rows, nrows, pairs, tw1, tw2, twN, work, rb, st);
        case 16: return launch_four_step<8, 8>(logN, d_jobs, d_rows, nrows, pairs, tw1, tw2, twN, work, rb, st);
        case 17: return launch_four_step<8, 9>(logN, d_jobs, d_rows, nrows, pairs, tw1, tw2, twN, work, rb, st);
        default: return cudaErrorInvalidValue;
    }
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
