// accum_kernels.cu -- kernels of pulse-chunked image formation (see accum.cpp).
//
// A pulse-chunked job forms its image from consecutive groups of phase-
// history rows.  The descriptor kept on the device is rewritten in stream
// order for each launch (store_job_kernel takes it as a kernel parameter,
// so no host synchronisation is needed between chunks); per chunk:
//   chunk_tables_kernel  the chunk's pulse window and pulse table, gathered
//                        from the whole aperture's (the reference pairs
//                        phase-history row q with antenna position
//                        (q - P mod 2) mod P: the pulse axis is fftshifted
//                        twice, backprojection.cpp:98,104)
//   range compression, tile records, backprojection (adds to acc)
// and once at the end
//   finalize_kernel      out[nv-1-y][x] = acc[y][x] * fin[y][x]
//                        (backprojection.cpp:130-135), max |z| for dB/u8.
// The combine kernel does the same for one-shot jobs formed in pulse parts
// (each part's sums in its own slice; see DevJob::nsplit).
#include <cstdint>

#include "internal.h"
#include "kernels.h"

namespace sarbp {

namespace {

constexpr int kThreads = 256;

__global__ void store_job_kernel(DevJob dj, DevJob *dst) { *dst = dj; }

__global__ void chunk_tables_kernel(const double4 *__restrict__ pulse, const float *__restrict__ wP, int P,
                                    int q0, int n, double4 *__restrict__ pulse_c, float *__restrict__ wP_c) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int q = q0 + i;
    const int p = (q - (P & 1) + P) % P;
    wP_c[i] = wP[q];
    pulse_c[i] = pulse[p];
}

__global__ void __launch_bounds__(kThreads) finalize_kernel(const DevJob *__restrict__ jobs) {
    const DevJob &jb = jobs[0];
    const long long n = (long long)jb.nu * jb.nv;
    double zmax = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int iy = (int)(i / jb.nu), ix = (int)(i - (long long)iy * jb.nu);
        const float2 a = jb.acc[i], f = jb.fin[i];
        // the same arithmetic as the backprojection kernel's epilogue
        const double zr = (double)fmaf(a.x, f.x, -a.y * f.y);
        const double zi = (double)fmaf(a.x, f.y, a.y * f.x);
        jb.out[(long long)(jb.nv - 1 - iy) * jb.nu + ix] = make_double2(zr, zi);
        zmax = fmax(zmax, sqrt(zr * zr + zi * zi));
    }
    for (int o = 16; o > 0; o >>= 1) zmax = fmax(zmax, __shfl_xor_sync(0xffffffffu, zmax, o));
    __shared__ double s[kThreads / 32];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = zmax;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kThreads / 32; ++w) zmax = fmax(zmax, s[w]);
        atomicMax(&jb.sc->maxabs, (unsigned long long)__double_as_longlong(zmax));
    }
}

// Jobs formed in pulse parts: out[nv-1-y][x] = (sum of the nsplit slices,
// in slice order) * fin[y][x], the same arithmetic as the backprojection
// kernel's epilogue; max |z| for dB/u8.  blockIdx.y: entry of the job list.
__global__ void __launch_bounds__(kThreads) combine_parts_kernel(const DevJob *__restrict__ jobs,
                                                                 const int *__restrict__ list) {
    const DevJob &jb = jobs[list[blockIdx.y]];
    const long long n = (long long)jb.nu * jb.nv;
    const int ns = jb.nsplit;
    double zmax = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int iy = (int)(i / jb.nu), ix = (int)(i - (long long)iy * jb.nu);
        float2 a = jb.parts[i];
        for (int k = 1; k < ns; ++k) {
            const float2 b = jb.parts[(long long)k * n + i];
            a.x += b.x;
            a.y += b.y;
        }
        const float2 f = jb.fin[i];
        const double zr = (double)fmaf(a.x, f.x, -a.y * f.y);
        const double zi = (double)fmaf(a.x, f.y, a.y * f.x);
        jb.out[(long long)(jb.nv - 1 - iy) * jb.nu + ix] = make_double2(zr, zi);
        zmax = fmax(zmax, sqrt(zr * zr + zi * zi));
    }
    for (int o = 16; o > 0; o >>= 1) zmax = fmax(zmax, __shfl_xor_sync(0xffffffffu, zmax, o));
    __shared__ double s[kThreads / 32];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = zmax;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kThreads / 32; ++w) zmax = fmax(zmax, s[w]);
        atomicMax(&jb.sc->maxabs, (unsigned long long)__double_as_longlong(zmax));
    }
}

__global__ void fill_items_kernel(WorkItem *items, int ntiles, RowItem *rows, int nrows) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < ntiles) items[t] = WorkItem{0, t, 0};
    if (t < nrows) rows[t] = RowItem{0, t};
}

int blocks_for(long long n) {
    long long b = (n + kThreads - 1) / kThreads;
    return (int)(b < 1 ? 1 : b);
}

}  // namespace

cudaError_t launch_store_job(const DevJob &dj, DevJob *d_dst, cudaStream_t st) {
    store_job_kernel<<<1, 1, 0, st>>>(dj, d_dst);
    return cudaGetLastError();
}

cudaError_t launch_chunk_tables(const double4 *pulse, const float *wP, int P, int q0, int n, double4 *pulse_c,
                                float *wP_c, cudaStream_t st) {
    chunk_tables_kernel<<<blocks_for(n), kThreads, 0, st>>>(pulse, wP, P, q0, n, pulse_c, wP_c);
    return cudaGetLastError();
}

cudaError_t launch_finalize(const DevJob *d_job, long long npix, int num_sms, cudaStream_t st) {
    long long b = (npix + kThreads - 1) / kThreads;
    if (b > (long long)num_sms * 8) b = (long long)num_sms * 8;
    finalize_kernel<<<(int)(b < 1 ? 1 : b), kThreads, 0, st>>>(d_job);
    return cudaGetLastError();
}

cudaError_t launch_combine_parts(const DevJob *d_jobs, const int *d_list, int nlist, long long max_pixels,
                                 int num_sms, cudaStream_t st) {
    if (nlist <= 0) return cudaSuccess;
    long long b = (max_pixels + kThreads - 1) / kThreads;
    const long long cap = ((long long)num_sms * 8 + nlist - 1) / nlist;
    if (b > cap) b = cap;
    combine_parts_kernel<<<dim3((unsigned)(b < 1 ? 1 : b), (unsigned)nlist), kThreads, 0, st>>>(d_jobs, d_list);
    return cudaGetLastError();
}

cudaError_t launch_fill_items(WorkItem *items, int ntiles, RowItem *rows, int nrows, cudaStream_t st) {
    fill_items_kernel<<<blocks_for(ntiles > nrows ? ntiles : nrows), kThreads, 0, st>>>(items, ntiles, rows,
                                                                                        nrows);
    return cudaGetLastError();
}

}  // namespace sarbp
