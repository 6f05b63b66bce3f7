// peaks.cu -- FP32-pipe and SFU throughput of the device, measured.
//
// The backprojection kernel is bound by FP32 instructions and SFU (MUFU)
// operations, whose peaks are not among the copy / GEMM peaks usually
// measured for a node.  These two kernels time long chains of independent
// FFMA (8 chains per thread) and of sin.approx (MUFU.SIN plus its FMUL
// range scaling) so the roofline fraction can be stated against numbers
// measured on the same GPU and clock.
#include "kernels.h"

namespace sarbp {

namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(256) ffma_kernel(float *out, int iters, float a, float b) {
    float x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = threadIdx.x * 1e-3f + c;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = fmaf(x[c], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    if (s == 1234.5f) out[0] = s;  // keeps the chains live
}

__global__ void __launch_bounds__(256) mufu_kernel(float *out, int iters) {
    float x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = threadIdx.x * 1e-3f + c * 0.1f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) asm volatile("sin.approx.f32 %0, %0;" : "+f"(x[c]));
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    if (s == 1234.5f) out[0] = s;
}

}  // namespace

// Returns FFMA instructions/s and MUFU ops/s (per GPU).
cudaError_t measure_peaks(int num_sms, cudaStream_t st, double *ffma_per_s, double *mufu_per_s) {
    float *d = nullptr;
    cudaError_t e = cudaMalloc(&d, 256);
    if (e != cudaSuccess) return e;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int blocks = num_sms * 8, threads = 256;
    const int it_f = 1 << 14, it_m = 1 << 11;
    // warm-up
    ffma_kernel<<<blocks, threads, 0, st>>>(d, 256, 0.999f, 1e-3f);
    mufu_kernel<<<blocks, threads, 0, st>>>(d, 64);
    float best_f = 1e30f, best_m = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
        cudaEventRecord(a, st);
        ffma_kernel<<<blocks, threads, 0, st>>>(d, it_f, 0.999f, 1e-3f);
        cudaEventRecord(b, st);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        best_f = ms < best_f ? ms : best_f;
        cudaEventRecord(a, st);
        mufu_kernel<<<blocks, threads, 0, st>>>(d, it_m);
        cudaEventRecord(b, st);
        cudaEventSynchronize(b);
        cudaEventElapsedTime(&ms, a, b);
        best_m = ms < best_m ? ms : best_m;
    }
    e = cudaGetLastError();
    const double n_thr = (double)blocks * threads;
    *ffma_per_s = n_thr * kChains * it_f / (best_f * 1e-3);
    *mufu_per_s = n_thr * kChains * it_m / (best_m * 1e-3);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(d);
    return e;
}

}  // namespace sarbp
