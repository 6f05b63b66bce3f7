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
#include <cfloat>
#include <cstdint>

#include "internal.h"
#include "kernels.h"

namespace sarbp {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ long long mirror_index(long long m, long long n) {
    if (n <= 1) return 0;
    const long long period = 2 * n - 2;
    if (m < 0) m = -m;
    m %= period;
    return m >= n ? period - m : m;
}

// One correlation pass along `axis` (0: rows, 1: cols) of [rows][cols][nc]
// with symmetric weights w[0..r] (w[0] the centre).
template <typename T>
__global__ void gauss_pass_kernel(const T *__restrict__ in, T *__restrict__ out, int rows, int cols, int nc,
                                  int axis, const double *__restrict__ w, int r) {
    const long long n = (long long)rows * cols * nc;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(i % nc);
        const long long rc = i / nc;
        const int c = (int)(rc % cols), row = (int)(rc / cols);
        const int pos = axis == 0 ? row : c, len = axis == 0 ? rows : cols;
        auto at = [&](long long m) -> double {
            const long long mm = mirror_index(m, len);
            const long long idx = axis == 0 ? (mm * cols + c) * nc + k : ((long long)row * cols + mm) * nc + k;
            return (double)in[idx];
        };
        double acc = at(pos) * w[0];
        for (int j = r; j >= 1; --j) acc += (at((long long)pos - j) + at((long long)pos + j)) * w[j];
        out[i] = (T)acc;
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

template <typename T>
__global__ void zoom_kernel(const T *__restrict__ in, T *__restrict__ out, int rows, int cols, int nc,
                            int orows, int ocols, double z0, double z1, const double *__restrict__ bounds) {
    const long long n = (long long)orows * ocols * nc;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(i % nc);
        const long long rc = i / nc;
        const int oc = (int)(rc % ocols), orow = (int)(rc / ocols);
        const double c0 = grid_coord(orow, z0, rows), c1 = grid_coord(oc, z1, cols);
        const double f0 = floor(c0), f1 = floor(c1);
        const double t0 = c0 - f0, t1 = c1 - f1;
        const double w0[2] = {1.0 - t0, t0}, w1[2] = {1.0 - t1, t1};
        const long long a0 = (long long)f0, a1 = (long long)f1;
        double t = 0.0;
        for (int h0 = 0; h0 < 2; ++h0) {
            const long long r0 = mirror_index(a0 + h0, rows);
            for (int h1 = 0; h1 < 2; ++h1) {
                const long long r1 = mirror_index(a1 + h1, cols);
                double coeff = (double)in[(r0 * cols + r1) * nc + k];
                coeff *= w0[h0];
                coeff *= w1[h1];
                t += coeff;
            }
        }
        const double lo = bounds[2 * k], hi = bounds[2 * k + 1];
        out[i] = (T)fmin(fmax(t, lo), hi);  // the bounds are values of type T
    }
}

// [min, max] of each component (one block per component)
template <typename T>
__global__ void bounds_kernel(const T *__restrict__ in, long long count, int nc, double *__restrict__ bounds) {
    const int k = blockIdx.x;
    double lo = DBL_MAX, hi = -DBL_MAX;
    for (long long i = threadIdx.x; i < count; i += blockDim.x) {
        const double v = (double)in[i * nc + k];
        lo = fmin(lo, v);
        hi = fmax(hi, v);
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

int grid_of(long long n) {
    long long b = (n + kThreads - 1) / kThreads;
    if (b > 148LL * 16) b = 148LL * 16;
    return (int)(b < 1 ? 1 : b);
}

template <typename T>
cudaError_t resize_t(const ResizePlan &p, const void *in, void *out, void *tmp_a, void *tmp_b, double *bounds,
                     cudaStream_t st) {
    const T *src = static_cast<const T *>(in);
    T *a = static_cast<T *>(tmp_a), *b = static_cast<T *>(tmp_b);
    const long long n_in = (long long)p.rows * p.cols * p.nc;
    bounds_kernel<T><<<p.nc, kThreads, 0, st>>>(src, (long long)p.rows * p.cols, p.nc, bounds);
    // anti-aliasing passes, axis 0 then axis 1
    const T *cur = src;
    for (int axis = 0; axis < 2; ++axis) {
        if (p.radius[axis] < 0) continue;
        T *dst = (cur == a) ? b : a;
        gauss_pass_kernel<T><<<grid_of(n_in), kThreads, 0, st>>>(cur, dst, p.rows, p.cols, p.nc, axis,
                                                                 p.d_weights + p.woff[axis], p.radius[axis]);
        cur = dst;
    }
    const long long n_out = (long long)p.orows * p.ocols * p.nc;
    zoom_kernel<T><<<grid_of(n_out), kThreads, 0, st>>>(cur, static_cast<T *>(out), p.rows, p.cols, p.nc, p.orows,
                                                        p.ocols, p.zoom[0], p.zoom[1], bounds);
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
