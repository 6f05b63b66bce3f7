// prep.cu -- per-job set-up kernel: Taylor windows, |k_r| filter and the
// per-pulse geometry table, for every job of a batch in one launch.
//
// grid = (njobs, 3): y == 0 sample window + filter (+ clears the job's
// max|z| and status words), y == 1 pulse window, y == 2 pulse geometry.
#include "internal.h"
#include "kernels.h"

namespace sarbp {

namespace {

constexpr int kPrepThreads = 256;

__device__ double block_max(double v, double *sred) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) sred[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = lane < (blockDim.x >> 5) ? sred[lane] : -INFINITY;
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0) sred[0] = v;
    }
    __syncthreads();
    v = sred[0];
    __syncthreads();
    return v;
}

// Taylor window before normalisation, signal.h:43-45:
// w(x) = 1 + sum_r F_m(r) cos(2 pi (r+1) xi), xi = linspace(-0.5, 0.5, num)
__device__ double taylor_w(const DevJob &jb, int num, int x) {
    const double step = (0.5 - (-0.5)) / (double)(num - 1);
    double xi = -0.5 + (double)x * step;
    xi = fmin(fmax(xi, -0.5), 0.5);
    double w = 1.0;
    for (int r = 0; r < jb.n_taylor; ++r)
        w = w + jb.taylor_F[r] * cos((2.0 * 3.14159265358979323846) * (double)(r + 1) * xi);
    return w;
}

// An orthonormal frame (rows of E) for the tiles' window bound: the image
// plane the reference builds by default, u_hat along the ground projection
// of the mid-aperture position, v_hat = z x u_hat, n_hat = z
// (img_plane.cpp:56-75 with n_hat = (0, 0, 1)); the x, y, z axes when that
// projection vanishes.  It depends on the antenna positions only, so the
// r-array and axes forms of a job get the same frame.  Any orthonormal frame
// keeps the bound valid; the image plane's own makes it tight.
__device__ void image_frame(const DevJob &jb, double (&E)[3][3]) {
    for (int i = 0; i < 3; ++i)
        for (int c = 0; c < 3; ++c) E[i][c] = i == c ? 1.0 : 0.0;
    const int m = jb.P / 2;
    double x, y;
    if (jb.precision == SARBP_PREC_PRECISE_ && jb.pos64) {
        x = jb.pos64[3 * m];
        y = jb.pos64[3 * m + 1];
    } else {
        x = jb.pos32[3 * m];
        y = jb.pos32[3 * m + 1];
    }
    const double n = sqrt(x * x + y * y);
    if (!(n > 0.0) || !isfinite(n)) return;
    E[0][0] = x / n;
    E[0][1] = y / n;
    E[0][2] = 0.0;
    E[1][0] = -y / n;
    E[1][1] = x / n;
    E[1][2] = 0.0;
}

__global__ void __launch_bounds__(kPrepThreads) prep_kernel(const DevJob *__restrict__ jobs) {
    __shared__ double sred[32];
    const DevJob &jb = jobs[blockIdx.x];
    const int what = blockIdx.y;
    if (what == 0 || what == 1) {
        const int num = what == 0 ? jb.S : jb.P;
        float *dst = what == 0 ? jb.wS : jb.wP;
        double m = -INFINITY;
        for (int x = threadIdx.x; x < num; x += blockDim.x) m = fmax(m, taylor_w(jb, num, x));
        m = block_max(m, sred);
        for (int x = threadIdx.x; x < num; x += blockDim.x)
            dst[x] = (float)(taylor_w(jb, num, x) / m);
        if (what == 0) {
            for (int s = threadIdx.x; s < jb.S; s += blockDim.x) {
                float f;
                if (jb.precision == SARBP_PREC_PRECISE_ && jb.k_r64)
                    f = (float)fabs(jb.k_r64[s]);
                else
                    f = fabsf(jb.k_r32[s]);
                jb.filt[s] = f;
            }
            if (threadIdx.x == 0) {
                jb.sc->maxabs = 0ull;
                jb.sc->status = 0;
                const int h = jb.S / 2;  // k_c = k_r[S/2] (backprojection.cpp:123)
                jb.sc->k_c = (jb.precision == SARBP_PREC_PRECISE_ && jb.k_r64) ? jb.k_r64[h]
                                                                               : (double)jb.k_r32[h];
            }
        }
    } else {
        double E[3][3];
        image_frame(jb, E);
        double la[3] = {0.0, 0.0, 0.0}, nmin = INFINITY;
        for (int p = threadIdx.x; p < jb.P; p += blockDim.x) {
            double4 g;
            if (jb.precision == SARBP_PREC_PRECISE_) {
                double x, y, z;
                if (jb.pos64) {
                    x = jb.pos64[3 * p]; y = jb.pos64[3 * p + 1]; z = jb.pos64[3 * p + 2];
                } else {
                    x = jb.pos32[3 * p]; y = jb.pos32[3 * p + 1]; z = jb.pos32[3 * p + 2];
                }
                double s = __dmul_rn(x, x);
                s = __dadd_rn(s, __dmul_rn(y, y));
                s = __dadd_rn(s, __dmul_rn(z, z));
                g = make_double4(x, y, z, sqrt(s));
            } else {
                // norm_r0 of the reference: f32 (x*x + y*y) + z*z, no fused
                // multiply-add, correctly rounded sqrt (backprojection.cpp:108,
                // util.h:67-71 on the f32 pos buffer).
                const float x = jb.pos32[3 * p], y = jb.pos32[3 * p + 1], z = jb.pos32[3 * p + 2];
                float s = __fmul_rn(x, x);
                s = __fadd_rn(s, __fmul_rn(y, y));
                s = __fadd_rn(s, __fmul_rn(z, z));
                g = make_double4(x, y, z, (double)__fsqrt_rn(s));
            }
            jb.pulse[p] = g;
            const double n = sqrt(g.x * g.x + g.y * g.y + g.z * g.z);
            if (n > 0.0 && isfinite(n)) {
                for (int i = 0; i < 3; ++i)
                    la[i] = fmax(la[i], fabs(g.x * E[i][0] + g.y * E[i][1] + g.z * E[i][2]) / n);
                nmin = fmin(nmin, n);
            } else {
                nmin = 0.0;  // no bound from this job's positions
            }
        }
        for (int i = 0; i < 3; ++i) la[i] = block_max(la[i], sred);
        nmin = -block_max(-nmin, sred);
        if (threadIdx.x == 0) {
            for (int i = 0; i < 3; ++i) {
                jb.sc->los_abs[i] = la[i];
                for (int c = 0; c < 3; ++c) jb.sc->frame[i][c] = E[i][c];
            }
            jb.sc->pos_min = nmin;
        }
    }
}

}  // namespace

void launch_prep(const DevJob *d_jobs, int njobs, cudaStream_t st) {
    prep_kernel<<<dim3(njobs, 3), kPrepThreads, 0, st>>>(d_jobs);
}

}  // namespace sarbp
