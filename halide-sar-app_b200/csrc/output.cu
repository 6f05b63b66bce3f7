// output.cu -- dB and u8 output stages (img_output.cpp:10-52).
//
//   m   = max |z| over the image               (img_output.cpp:23-24)
//   dB  = 10 * log(|z| / m) / log(10)          (img_output.cpp:26, util.h:56-58;
//         log(Expr(10)) has an integer argument, so Halide takes it in f32)
//   u8  = trunc(clamp((clamp(dB, lo, hi) - lo) / (hi - lo) * 255, 0, 255))
//                                              (img_output.cpp:48-51, signal.h:55-57)
// All HBM-bound; the fused form reads the complex image once and writes the
// u8 (and optionally the f64 dB) image, using the max|z| that the
// backprojection epilogue already reduced.
#include <algorithm>
#include <cstdint>

#include "internal.h"
#include "kernels.h"

namespace sarbp {

namespace {

constexpr double kLn10F32 = 2.302585124969482421875;  // logf(10.0f)

__device__ __forceinline__ uint8_t to_u8(double v, double lo, double hi) {
    if (v != v) v = lo;
    v = fmin(fmax(v, lo), hi);
    double n = (v - lo) / (hi - lo) * 255.0;
    n = fmin(fmax(n, 0.0), 255.0);
    return (uint8_t)n;
}

// u8 of one pixel.  The value is decided in f32 (|z|^2 rounded to f32, the
// accurate logf), whose error is far below 1e-4 of a grey level for display
// ranges of 0.1 dB and wider; a pixel whose f32 level lands within that
// margin of an integer, of the clamps, or is not finite, is recomputed with
// the reference's f64 formula.  Only the f64 path runs where dB itself is
// written.
struct U8Scale {
    double m, lo, hi;
    float inv_m2, k, q0, eps;  // q = k ln(|z|^2 / m^2) + q0 (grey levels)
};

__device__ __forceinline__ U8Scale u8_scale(double m, double lo, double hi) {
    U8Scale u;
    u.m = m;
    u.lo = lo;
    u.hi = hi;
    const double g = 255.0 / (hi - lo);               // grey levels per dB
    u.inv_m2 = (float)(1.0 / (m * m));
    u.k = (float)(5.0 / kLn10F32 * g);                // 10 log10(a/m) = 5 ln(a^2/m^2) / ln 10
    u.q0 = (float)(-lo * g);
    u.eps = (float)(2e-5 * g + 1e-4);
    return u;
}

__device__ __forceinline__ uint8_t u8_of(double2 z, const U8Scale &u) {
    const double a2 = z.x * z.x + z.y * z.y;
    const float q = fmaf(u.k, logf((float)a2 * u.inv_m2), u.q0);
    const float f = q - floorf(q);
    if (q > u.eps && q < 255.0f - u.eps && f > u.eps && f < 1.0f - u.eps) return (uint8_t)q;
    return to_u8(10.0 * (log(sqrt(a2) / u.m) / kLn10F32), u.lo, u.hi);
}

// max |z|: four independent 16-byte loads in flight per thread and step (a
// warp's loads stay contiguous), the maximum taken on |z|^2 and one square
// root at the end -- the same value, as the square root is monotonic and
// correctly rounded.
__global__ void maxabs_kernel(const double2 *__restrict__ img, long long n,
                              unsigned long long *__restrict__ out) {
    double m2 = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    for (; i + 3 * stride < n; i += 4 * stride) {
        double2 z[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) z[k] = img[i + k * stride];
#pragma unroll
        for (int k = 0; k < 4; ++k) m2 = fmax(m2, z[k].x * z[k].x + z[k].y * z[k].y);
    }
    for (; i < n; i += stride) {
        const double2 z = img[i];
        m2 = fmax(m2, z.x * z.x + z.y * z.y);
    }
    double m = sqrt(m2);
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ double s[32];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, s[w]);
        atomicMax(out, (unsigned long long)__double_as_longlong(m));
    }
}

__global__ void db_u8_kernel(const double2 *__restrict__ img, long long n,
                             const unsigned long long *__restrict__ maxbits, double *__restrict__ dB,
                             uint8_t *__restrict__ u8, double lo, double hi) {
    const double m = __longlong_as_double((long long)*maxbits);
    const U8Scale us = u8_scale(m, lo, hi);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double2 z = img[i];
        if (!dB) {
            u8[i] = u8_of(z, us);
            continue;
        }
        const double a = sqrt(z.x * z.x + z.y * z.y);
        const double d = 10.0 * (log(a / m) / kLn10F32);
        dB[i] = d;
        if (u8) u8[i] = to_u8(d, lo, hi);
    }
}

__global__ void u8_from_db_kernel(const double *__restrict__ dB, long long n, double lo, double hi,
                                  uint8_t *__restrict__ u8) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        u8[i] = to_u8(dB[i], lo, hi);
}

// u8 of the four neighbouring pixels [i0, i0 + 4) of an image of n pixels:
// 64 B of complex f64 in, one 32-bit word of u8 out when the destination is
// 4-byte aligned (vec).
__device__ __forceinline__ void u8_quad(const double2 *__restrict__ img, long long n, long long i0,
                                        uint8_t *__restrict__ u8, bool vec, const U8Scale &us) {
    if (vec && i0 + 4 <= n) {
        double2 z[4];  // the four loads first, then the conversions
#pragma unroll
        for (int k = 0; k < 4; ++k) z[k] = img[i0 + k];
        uint32_t w = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) w |= (uint32_t)u8_of(z[k], us) << (8 * k);
        *reinterpret_cast<uint32_t *>(u8 + i0) = w;
    } else {
        for (long long i = i0; i < n && i < i0 + 4; ++i) u8[i] = u8_of(img[i], us);
    }
}

// blockIdx.y = job; jobs without an u8 output return at once.  Each thread
// converts four neighbouring pixels at a time.
__global__ void batch_u8_kernel(const DevJob *__restrict__ jobs) {
    const DevJob &jb = jobs[blockIdx.y];
    if (!jb.out_u8) return;
    const double m = __longlong_as_double((long long)jb.sc->maxabs);
    const long long n = (long long)jb.nu * jb.nv;
    const U8Scale us = u8_scale(m, jb.dB_min, jb.dB_max);
    const bool vec = ((reinterpret_cast<uintptr_t>(jb.out_u8) & 3) == 0);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; 4 * q < n; q += stride)
        u8_quad(jb.out, n, 4 * q, jb.out_u8, vec, us);
}

// The same conversion for one image given by its pointer and a max|z| from
// maxabs_kernel.
__global__ void img_u8_kernel(const double2 *__restrict__ img, long long n,
                              const unsigned long long *__restrict__ maxbits, uint8_t *__restrict__ u8,
                              double lo, double hi) {
    const U8Scale us = u8_scale(__longlong_as_double((long long)*maxbits), lo, hi);
    const bool vec = ((reinterpret_cast<uintptr_t>(u8) & 3) == 0);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; 4 * q < n; q += stride)
        u8_quad(img, n, 4 * q, u8, vec, us);
}

int grid_for(long long n) {
    long long b = (n + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    if (b < 1) b = 1;
    return (int)b;
}

// CTAs of 256 threads that the device holds at once for `kernel` (one wave
// of a grid-stride loop: no partial last wave); looked up once per kernel.
template <typename K>
long long resident_ctas(K kernel, int *cache) {
    if (*cache > 0) return *cache;
    int dev = 0, sms = 148, occ = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, 256, 0) != cudaSuccess || occ < 1) occ = 4;
    *cache = occ * sms;
    return *cache;
}
int g_maxabs_ctas = 0, g_img_u8_ctas = 0, g_batch_u8_ctas = 0;

}  // namespace

cudaError_t launch_maxabs(const double2 *img, long long n, unsigned long long *d_max, cudaStream_t st) {
    // at least eight pixels a thread (two steps of four loads), at most one
    // wave of resident CTAs
    const long long b = std::max<long long>(
        1, std::min<long long>((n + 2047) / 2048, resident_ctas(maxabs_kernel, &g_maxabs_ctas)));
    maxabs_kernel<<<(unsigned)b, 256, 0, st>>>(img, n, d_max);
    return cudaGetLastError();
}

cudaError_t launch_db_u8(const double2 *img, long long n, const unsigned long long *d_max, double *dB,
                         uint8_t *u8, double lo, double hi, cudaStream_t st) {
    db_u8_kernel<<<grid_for(n), 256, 0, st>>>(img, n, d_max, dB, u8, lo, hi);
    return cudaGetLastError();
}

cudaError_t launch_u8_from_db(const double *dB, long long n, double lo, double hi, uint8_t *u8,
                              cudaStream_t st) {
    u8_from_db_kernel<<<grid_for(n), 256, 0, st>>>(dB, n, lo, hi, u8);
    return cudaGetLastError();
}

cudaError_t launch_img_u8(const double2 *img, long long n, const unsigned long long *d_max, uint8_t *u8,
                          double lo, double hi, cudaStream_t st) {
    // one wave of resident CTAs, four pixels per thread and step
    const long long bx = std::max<long long>(
        1, std::min<long long>((n / 4 + 255) / 256, resident_ctas(img_u8_kernel, &g_img_u8_ctas)));
    img_u8_kernel<<<(unsigned)bx, 256, 0, st>>>(img, n, d_max, u8, lo, hi);
    return cudaGetLastError();
}

cudaError_t launch_batch_u8(const DevJob *d_jobs, int njobs, long long max_pixels, cudaStream_t st) {
    // one wave of resident CTAs over the whole batch
    long long bx = (max_pixels / 4 + 255) / 256;
    const long long cap =
        std::max<long long>(1, (resident_ctas(batch_u8_kernel, &g_batch_u8_ctas) + njobs - 1) / njobs);
    bx = std::max<long long>(1, std::min(bx, cap));
    batch_u8_kernel<<<dim3((unsigned)bx, njobs), 256, 0, st>>>(d_jobs);
    return cudaGetLastError();
}

}  // namespace sarbp
