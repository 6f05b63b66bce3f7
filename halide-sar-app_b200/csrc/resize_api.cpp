// resize_api.cpp -- sarbp_resize*: the array resampling of the reference's
// data/resize.py (see resize.cu for the algorithm), host planning.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "context.h"
#include "kernels.h"
#include "runner.h"
#include "sarbp_b200.h"

using namespace sarbp;

namespace {

size_t a256(size_t x) { return (x + 255) / 256 * 256; }

// The sum numpy's ndarray.sum gives a float64 vector (pairwise summation:
// eight running sums for 8..128 elements, a plain loop below 8).
double numpy_sum(const std::vector<double> &a) {
    const size_t n = a.size();
    if (n < 8) {
        double s = 0.0;
        for (double v : a) s += v;
        return s;
    }
    if (n > 128) {  // halves, recursively
        std::vector<double> lo(a.begin(), a.begin() + (n / 2 - (n / 2) % 8)), hi(a.begin() + lo.size(), a.end());
        return numpy_sum(lo) + numpy_sum(hi);
    }
    double r[8];
    for (int j = 0; j < 8; ++j) r[j] = a[j];
    size_t i = 8;
    for (; i < n - (n % 8); i += 8)
        for (int j = 0; j < 8; ++j) r[j] += a[i + j];
    double s = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
    for (; i < n; ++i) s += a[i];
    return s;
}

// Gaussian weights of scipy.ndimage.gaussian_filter1d (order 0, truncate
// 4): w[j] for j = 0..radius, w[0] the centre.
std::vector<double> gauss_weights(double sigma, int *radius) {
    const int r = (int)(4.0 * sigma + 0.5);
    const double a = -0.5 / (sigma * sigma);
    std::vector<double> phi(2 * r + 1);
    for (int x = -r; x <= r; ++x) phi[x + r] = std::exp(a * (double)((long long)x * x));
    const double s = numpy_sum(phi);
    std::vector<double> w(r + 1);
    for (int j = 0; j <= r; ++j) w[j] = phi[r + j] / s;
    *radius = r;
    return w;
}

int resize_enqueue(sarbp_ctx *ctx, int elem_bytes, int ncomp, const void *in, int rows, int cols, int orows,
                   int ocols, void *out) {
    if (elem_bytes != 4 && elem_bytes != 8) return fail(SARBP_ERR_INVALID, "resize: elements of 4 or 8 bytes");
    if (ncomp < 1 || rows < 1 || cols < 1 || orows < 1 || ocols < 1 || !in || !out)
        return fail(SARBP_ERR_INVALID, "resize: sizes must be >= 1 and arrays non-NULL");
    ResizePlan p{};
    p.elem_bytes = elem_bytes;
    p.nc = ncomp;
    p.rows = rows;
    p.cols = cols;
    p.orows = orows;
    p.ocols = ocols;
    const int in_ext[2] = {rows, cols}, out_ext[2] = {orows, ocols};
    // anti-aliasing when any axis shrinks; sigma (f - 1) / 2 on each axis
    const bool aa = orows < rows || ocols < cols;
    std::vector<double> weights;
    for (int ax = 0; ax < 2; ++ax) {
        const double f = (double)in_ext[ax] / (double)out_ext[ax];
        p.zoom[ax] = (double)in_ext[ax] / (double)out_ext[ax];
        p.radius[ax] = -1;
        const double sigma = std::max(0.0, (f - 1.0) / 2.0);
        if (aa && sigma > 1e-15) {
            int r = 0;
            std::vector<double> w = gauss_weights(sigma, &r);
            p.radius[ax] = r;
            p.woff[ax] = (int)weights.size();
            weights.insert(weights.end(), w.begin(), w.end());
        }
    }
    const size_t n_in = (size_t)rows * cols * ncomp * elem_bytes;
    // bounds: the result (2 ncomp) and the partials of up to 148 * 4 blocks
    const size_t b_w = a256(std::max<size_t>(1, weights.size()) * sizeof(double)),
                 b_b = a256((size_t)(1 + 148 * 4) * 2 * ncomp * sizeof(double));
    const size_t b_t = a256(((size_t)orows + ocols) * 32);
    cudaError_t e = ctx->resize_buf.ensure(b_w + b_b + 2 * a256(n_in) + b_t, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "resize: scratch");
    char *base = static_cast<char *>(ctx->resize_buf.ptr);
    double *d_w = reinterpret_cast<double *>(base), *d_b = reinterpret_cast<double *>(base + b_w);
    if (!weights.empty())
        e = cudaMemcpyAsync(d_w, weights.data(), weights.size() * sizeof(double), cudaMemcpyHostToDevice,
                            ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "resize: weights");
    p.d_weights = d_w;
    p.d_taps = base + b_w + b_b + 2 * a256(n_in);
    e = launch_resize(p, in, out, base + b_w + b_b, base + b_w + b_b + a256(n_in), d_b, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "resize launch");
    ctx->dev.launches += 4 + (p.radius[0] >= 0) + (p.radius[1] >= 0);
    return SARBP_OK;
}

}  // namespace

extern "C" {

int sarbp_resize_device(sarbp_ctx *ctx, int elem_bytes, int ncomp, const void *in, int rows, int cols,
                        int out_rows, int out_cols, void *out) {
    int rc = ctx_set_device(ctx);
    if (rc) return rc;
    return resize_enqueue(ctx, elem_bytes, ncomp, in, rows, cols, out_rows, out_cols, out);
}

int sarbp_resize(sarbp_ctx *ctx, int elem_bytes, int ncomp, const void *in, int rows, int cols, int out_rows,
                 int out_cols, void *out) {
    int rc = ctx_set_device(ctx);
    if (rc) return rc;
    if (elem_bytes != 4 && elem_bytes != 8) return fail(SARBP_ERR_INVALID, "resize: elements of 4 or 8 bytes");
    if (ncomp < 1 || rows < 1 || cols < 1 || out_rows < 1 || out_cols < 1 || !in || !out)
        return fail(SARBP_ERR_INVALID, "resize: sizes must be >= 1 and arrays non-NULL");
    const size_t n_in = (size_t)rows * cols * ncomp * elem_bytes;
    const size_t n_out = (size_t)out_rows * out_cols * ncomp * elem_bytes;
    cudaError_t e = ctx->io.ensure(a256(n_in) + a256(n_out), ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "resize: device arrays");
    char *d_in = static_cast<char *>(ctx->io.ptr), *d_out = d_in + a256(n_in);
    e = cudaMemcpyAsync(d_in, in, n_in, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "resize: copying the array in");
    rc = resize_enqueue(ctx, elem_bytes, ncomp, d_in, rows, cols, out_rows, out_cols, d_out);
    if (rc) return rc;
    e = cudaMemcpyAsync(out, d_out, n_out, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "resize: copying the array out");
    return SARBP_OK;
}

}  // extern "C"
