// resize.cu -- resampling of platform arrays on the device: the computation
// the reference's data/resize.py applies to phs, pos and k_r to change the
// pulse and sample counts of a recorded phase history
// (data/resize.py:14-70, `skimage.transform.resize(a, shape,
// preserve_range=True)` with its defaults: linear interpolation, mode
// 'reflect', anti-aliasing when an axis shrinks, output clipped to the input
// range).  scikit-image is not part of the reference (an unpinned
// third-party dependency, absent here); the steps below restate its
// published algorithm (skimage >= 0.19 `resize`, built on scipy.ndimage):
//
//   1. anti-aliasing, on every axis with factor f = in / out > 1: a Gaussian
//      of sigma (f - 1) / 2, truncated at 4 sigma (radius int(4 sigma + 0.5)),
//      weights exp(-x^2 / (2 sigma^2)) normalised to sum 1, applied along
//      axis 0 then axis 1 as a correlation with mirrored edges
//      (x[-k] = x[k], x[n-1+k] = x[n-1-k]), each pass accumulated in f64 as
//      x[i] w0 + sum_{k = r..1} (x[i-k] + x[i+k]) w_k and rounded to the
//      array's type;
//   2. zoom to the output shape, grid-aligned: output index o of an axis
//      samples input coordinate c = (o + 0.5) (in / out) - 0.5, mirrored
//      into [0, n-1]; linear weights (1 - t, t) of the two neighbours
//      floor(c), floor(c) + 1 (mirrored at the edge); the four neighbours of
//      a 2-D sample summed in f64 in row-major order, each value times its
//      axis-0 weight then its axis-1 weight; rounded to the array's type;
//   3. clipped to [min, max] of the unfiltered input.
// Arrays are [rows][cols][ncomp] of f32 or f64; each of the ncomp
// interleaved components (re, im of a complex array) is resampled on its
// own, as the reference does with np.real and np.imag.
#include <algorithm>
#include <cfloat>
#include <cstdint>

#include "internal.h"
#include "kernels.h"

namespace sarbp {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ long long mirror_index(long long m, long long n) {
    if (m >= 0 && m < n) return m;  // inside: no reflection
    if (n <= 1) return 0;
    const long long period = 2 * n - 2;
    if (m < 0) m = -m;
    m %= period;
    return m >= n ? period - m : m;
}

// Launch shape of the per-column kernels: x over the columns of a row, y
// over rows (strided; gridDim.y <= 65535), about 32 blocks per SM in all.
struct RowGrid {
    dim3 grid;
};
inline RowGrid row_grid(long long rows, long long cols) {
    long long gx = (cols + kThreads - 1) / kThreads;
    long long gy = rows;
    const long long target = 148LL * 32;
    if (gx >= target) gy = 1;
    else gy = std::min<long long>(gy, std::max<long long>(1, target / gx));
    gy = std::min<long long>(gy, 65535);
    return RowGrid{dim3((unsigned)std::max<long long>(1, gx), (unsigned)std::max<long long>(1, gy))};
}

// Components per element: NC > 0 fixed at compile time (1, or 2 for the
// real and imaginary parts of a complex array), NC == 0 taken from nc.
template <int NC>
__device__ __forceinline__ int ncomp(int nc) {
    return NC > 0 ? NC : nc;
}

// One correlation pass along `axis` (0: rows, 1: cols) of [rows][cols][nc]
// with symmetric weights w[0..r] (w[0] the centre).  Thread: one column of
// a row (all its components), rows strided over y.
template <typename T, int NC>
__global__ void gauss_pass_kernel(const T *__restrict__ in, T *__restrict__ out, int rows, int cols, int nc_,
                                  int axis, const double *__restrict__ w, int r) {
    const int nc = ncomp<NC>(nc_);
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < cols; c += gridDim.x * blockDim.x) {
        for (int row = blockIdx.y; row < rows; row += gridDim.y) {
            const int pos = axis == 0 ? row : c, len = axis == 0 ? rows : cols;
            // first value of the element at position m along the axis
            auto base = [&](long long m) -> long long {
                const long long mm = mirror_index(m, len);
                return (axis == 0 ? mm * cols + c : (long long)row * cols + mm) * nc;
            };
            const long long b0 = base(pos);
            T *o = out + ((long long)row * cols + c) * nc;
            if constexpr (NC > 0) {
                // the components side by side, the taps unrolled, so that
                // the loads of several taps are in flight together
                double acc[NC];
#pragma unroll
                for (int k = 0; k < NC; ++k) acc[k] = (double)in[b0 + k] * w[0];
#pragma unroll 4
                for (int t = r; t >= 1; --t) {
                    const long long bm = base((long long)pos - t), bp = base((long long)pos + t);
                    const double wt = w[t];
#pragma unroll
                    for (int k = 0; k < NC; ++k) acc[k] += ((double)in[bm + k] + (double)in[bp + k]) * wt;
                }
#pragma unroll
                for (int k = 0; k < NC; ++k) o[k] = (T)acc[k];
            } else {
                for (int kk = 0; kk < nc; ++kk) {
                    double acc = (double)in[b0 + kk] * w[0];
                    for (int t = r; t >= 1; --t)
                        acc += ((double)in[base((long long)pos - t) + kk] + (double)in[base((long long)pos + t) + kk]) *
                               w[t];
                    o[kk] = (T)acc;
                }
            }
        }
    }
}

// sample coordinate of output index o on an axis of in -> out points
__device__ __forceinline__ double grid_coord(int o, double zoom, long long len) {
    double cc = ((double)o + 0.5) * zoom - 0.5;
    if (len <= 1) return 0.0;
    const double sz2 = (double)(2 * len - 2);
    if (cc < 0) cc = -cc;
    cc = cc - sz2 * (double)(long long)(cc / sz2);
    if (cc >= (double)len) cc = sz2 - cc;
    return cc;
}

// The two neighbours (mirrored) and linear weights of output index o.
struct Taps {
    long long i0, i1;
    double w0, w1;
};
__device__ __forceinline__ Taps taps_of(int o, double zoom, long long len) {
    const double c = grid_coord(o, zoom, len);
    const double f = floor(c);
    const double t = c - f;
    const long long a = (long long)f;
    return Taps{mirror_index(a, len), mirror_index(a + 1, len), 1.0 - t, t};
}

// taps[0 .. orows) of the output rows, taps[orows .. orows + ocols) of the
// output columns
__global__ void taps_kernel(Taps *__restrict__ taps, int orows, int ocols, double z0, double z1, int rows,
                            int cols) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < orows) taps[i] = taps_of(i, z0, rows);
    else if (i < orows + ocols) taps[i] = taps_of(i - orows, z1, cols);
}

// Thread: one output column (all its components), output rows strided
// over y; the four neighbours summed in f64 in row-major order, each value
// times its row weight then its column weight.
template <typename T, int NC>
__global__ void zoom_kernel(const T *__restrict__ in, T *__restrict__ out, int rows, int cols, int nc_,
                            int orows, int ocols, const Taps *__restrict__ taps, const double *__restrict__ bounds) {
    const int nc = ncomp<NC>(nc_);
    for (int oc = blockIdx.x * blockDim.x + threadIdx.x; oc < ocols; oc += gridDim.x * blockDim.x) {
        const Taps tc = taps[orows + oc];
#pragma unroll 4
        for (int orow = blockIdx.y; orow < orows; orow += gridDim.y) {
            const Taps tr = taps[orow];
            const T *p00 = in + (tr.i0 * cols + tc.i0) * nc, *p01 = in + (tr.i0 * cols + tc.i1) * nc;
            const T *p10 = in + (tr.i1 * cols + tc.i0) * nc, *p11 = in + (tr.i1 * cols + tc.i1) * nc;
            T *o = out + ((long long)orow * ocols + oc) * nc;
#pragma unroll
            for (int k = 0; k < (NC > 0 ? NC : 1); ++k) {
                for (int kk = k; kk < nc; kk += (NC > 0 ? NC : 1)) {
                    double t = 0.0, coeff;
                    coeff = (double)p00[kk];
                    coeff *= tr.w0;
                    coeff *= tc.w0;
                    t += coeff;
                    coeff = (double)p01[kk];
                    coeff *= tr.w0;
                    coeff *= tc.w1;
                    t += coeff;
                    coeff = (double)p10[kk];
                    coeff *= tr.w1;
                    coeff *= tc.w0;
                    t += coeff;
                    coeff = (double)p11[kk];
                    coeff *= tr.w1;
                    coeff *= tc.w1;
                    t += coeff;
                    o[kk] = (T)fmin(fmax(t, bounds[2 * kk]), bounds[2 * kk + 1]);  // the bounds are values of type T
                }
            }
        }
    }
}

// [min, max] of each component: partial bounds of kBoundBlocks slices of
// the array (part[b][k] = (lo, hi)), then one block per component reduces
// them (fmin / fmax: the order does not change the result)
constexpr int kBoundBlocks = 148 * 4;

template <typename T, int NC>
__global__ void __launch_bounds__(kThreads) bounds_partial_kernel(const T *__restrict__ in, long long count, int nc_,
                                                                  double *__restrict__ part) {
    // NC > 0: the NC components in one sweep; NC == 0: one sweep per component
    constexpr int KB = NC > 0 ? NC : 1;
    const int nc = NC > 0 ? NC : nc_;
    __shared__ double slo[KB][kThreads / 32], shi[KB][kThreads / 32];
    for (int k0 = 0; k0 < nc; k0 += KB) {
        double lo[KB], hi[KB];
#pragma unroll
        for (int k = 0; k < KB; ++k) {
            lo[k] = DBL_MAX;
            hi[k] = -DBL_MAX;
        }
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count;
             i += (long long)gridDim.x * blockDim.x) {
#pragma unroll
            for (int k = 0; k < KB; ++k) {
                const double v = (double)in[i * nc + k0 + k];
                lo[k] = fmin(lo[k], v);
                hi[k] = fmax(hi[k], v);
            }
        }
#pragma unroll
        for (int k = 0; k < KB; ++k) {
            for (int o = 16; o > 0; o >>= 1) {
                lo[k] = fmin(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
                hi[k] = fmax(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
            }
            if ((threadIdx.x & 31) == 0) {
                slo[k][threadIdx.x >> 5] = lo[k];
                shi[k][threadIdx.x >> 5] = hi[k];
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
#pragma unroll
            for (int k = 0; k < KB; ++k) {
                double l = slo[k][0], h = shi[k][0];
                for (int w = 1; w < kThreads / 32; ++w) {
                    l = fmin(l, slo[k][w]);
                    h = fmax(h, shi[k][w]);
                }
                part[((long long)blockIdx.x * nc + k0 + k) * 2] = l;
                part[((long long)blockIdx.x * nc + k0 + k) * 2 + 1] = h;
            }
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kThreads) bounds_final_kernel(const double *__restrict__ part, int nparts, int nc,
                                                                double *__restrict__ bounds) {
    const int k = blockIdx.x;
    double lo = DBL_MAX, hi = -DBL_MAX;
    for (int b = threadIdx.x; b < nparts; b += blockDim.x) {
        lo = fmin(lo, part[((long long)b * nc + k) * 2]);
        hi = fmax(hi, part[((long long)b * nc + k) * 2 + 1]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    __shared__ double slo[kThreads / 32], shi[kThreads / 32];
    if ((threadIdx.x & 31) == 0) {
        slo[threadIdx.x >> 5] = lo;
        shi[threadIdx.x >> 5] = hi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kThreads / 32; ++w) {
            lo = fmin(lo, slo[w]);
            hi = fmax(hi, shi[w]);
        }
        bounds[2 * k] = lo;
        bounds[2 * k + 1] = hi;
    }
}

template <typename T>
cudaError_t resize_t(const ResizePlan &p, const void *in, void *out, void *tmp_a, void *tmp_b, double *bounds,
                     cudaStream_t st) {
    const T *src = static_cast<const T *>(in);
    T *a = static_cast<T *>(tmp_a), *b = static_cast<T *>(tmp_b);
    // bounds[0 .. 2 nc) the result, bounds + 2 nc the partials
    const long long count = (long long)p.rows * p.cols;
    const int nparts = (int)std::min<long long>(kBoundBlocks, (count + kThreads - 1) / kThreads);
    if (p.nc == 1)
        bounds_partial_kernel<T, 1><<<nparts, kThreads, 0, st>>>(src, count, 1, bounds + 2);
    else if (p.nc == 2)
        bounds_partial_kernel<T, 2><<<nparts, kThreads, 0, st>>>(src, count, 2, bounds + 4);
    else
        bounds_partial_kernel<T, 0><<<nparts, kThreads, 0, st>>>(src, count, p.nc, bounds + 2 * p.nc);
    bounds_final_kernel<<<p.nc, kThreads, 0, st>>>(bounds + 2 * p.nc, nparts, p.nc, bounds);
    // anti-aliasing passes, axis 0 then axis 1
    const T *cur = src;
    for (int axis = 0; axis < 2; ++axis) {
        if (p.radius[axis] < 0) continue;
        T *dst = (cur == a) ? b : a;
        const dim3 g = row_grid(p.rows, p.cols).grid;
        const double *w = p.d_weights + p.woff[axis];
        if (p.nc == 1)
            gauss_pass_kernel<T, 1><<<g, kThreads, 0, st>>>(cur, dst, p.rows, p.cols, 1, axis, w, p.radius[axis]);
        else if (p.nc == 2)
            gauss_pass_kernel<T, 2><<<g, kThreads, 0, st>>>(cur, dst, p.rows, p.cols, 2, axis, w, p.radius[axis]);
        else
            gauss_pass_kernel<T, 0><<<g, kThreads, 0, st>>>(cur, dst, p.rows, p.cols, p.nc, axis, w, p.radius[axis]);
        cur = dst;
    }
    Taps *taps = static_cast<Taps *>(p.d_taps);
    const int ntaps = p.orows + p.ocols;
    taps_kernel<<<(ntaps + kThreads - 1) / kThreads, kThreads, 0, st>>>(taps, p.orows, p.ocols, p.zoom[0],
                                                                       p.zoom[1], p.rows, p.cols);
    const dim3 g = row_grid(p.orows, p.ocols).grid;
    T *o = static_cast<T *>(out);
    if (p.nc == 1)
        zoom_kernel<T, 1><<<g, kThreads, 0, st>>>(cur, o, p.rows, p.cols, 1, p.orows, p.ocols, taps, bounds);
    else if (p.nc == 2)
        zoom_kernel<T, 2><<<g, kThreads, 0, st>>>(cur, o, p.rows, p.cols, 2, p.orows, p.ocols, taps, bounds);
    else
        zoom_kernel<T, 0><<<g, kThreads, 0, st>>>(cur, o, p.rows, p.cols, p.nc, p.orows, p.ocols, taps, bounds);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_resize(const ResizePlan &p, const void *in, void *out, void *tmp_a, void *tmp_b,
                          double *bounds, cudaStream_t st) {
    if (p.elem_bytes == 4) return resize_t<float>(p, in, out, tmp_a, tmp_b, bounds, st);
    if (p.elem_bytes == 8) return resize_t<double>(p, in, out, tmp_a, tmp_b, bounds, st);
    return cudaErrorInvalidValue;
}

}  // namespace sarbp
