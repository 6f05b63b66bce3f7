// kernels.h -- launch wrappers of the device kernels (host-callable).
#pragma once

#include <cuda_runtime.h>

#include "internal.h"
#include "sarbp_b200.h"

#define SARBP_PREC_COMPAT_ SARBP_PREC_COMPAT
#define SARBP_PREC_PRECISE_ SARBP_PREC_PRECISE
#define SARBP_PREC_NAIVE_ SARBP_PREC_NAIVE

namespace sarbp {

// prep.cu
void launch_prep(const DevJob *d_jobs, int njobs, cudaStream_t st);

// range_compress.cu
int twiddle_table_size(int logN);
void fill_twiddle_table(int logN, float2 *host);
cudaError_t launch_range_compress(int logN, const DevJob *d_jobs, const RowItem *d_rows, int nrows, int pairs,
                                  const float2 *d_tw, cudaStream_t st);
cudaError_t init_range_compress_attributes();
// N_fft above 2^kMaxLogNSmem: a four-step FFT through `work`, which holds
// work_rows rows of N_fft complex values (rows go through it work_rows at a
// time; rc_work_rows(logN) rows, rc_work_bytes(logN) bytes, is about
// 256 MB); tw1 and tw2 are the tables of logN / 2 and logN - logN / 2, twN
// the W_N table.
int rc_work_rows(int logN);
size_t rc_work_bytes(int logN);
cudaError_t launch_range_compress_large(int logN, const DevJob *d_jobs, const RowItem *d_rows, int nrows,
                                        int pairs, const float2 *tw1, const float2 *tw2, const float2 *twN,
                                        float2 *work, int work_rows, cudaStream_t st);

// backproject.cu
struct BpLaunch {
    int tile_x, tile_y;
    int minb;        // CTAs per SM the kernel's registers are sized for (2 or 3)
    int stage_cap;   // float4 entries of each half of the staging double buffer
    int cmax;        // max pulses per chunk
    int persistent;  // 1: grid = resident CTAs pulling items from *counter
    int grid;        // CTAs when persistent
    int parts;       // requested pulse parts per tile (sarbp_opts::pulse_parts)
};
bool bp_tile_supported(int tile_x, int tile_y, int minb);
size_t bp_smem_bytes(const BpLaunch &L);
int bp_max_active_blocks(const BpLaunch &L);
cudaError_t init_backproject_attributes();
cudaError_t launch_backproject(const BpLaunch &L, const DevJob *d_jobs, const WorkItem *d_items,
                               int nitems, int *d_counter, cudaStream_t st);
cudaError_t launch_backproject_naive(const DevJob *d_jobs, int job, int nu, int nv, cudaStream_t st);

// geometry.cu
// records = 0: tile table and final phases only (pulse-chunked jobs)
cudaError_t launch_tile_setup(const DevJob *d_jobs, const WorkItem *d_items, int nitems, int tile_pixels,
                              cudaStream_t st, int records = 1);
// per-(tile, pulse) records of one pulse chunk over an existing tile table
cudaError_t launch_tile_records(const DevJob *d_jobs, const WorkItem *d_items, int nitems, cudaStream_t st);


// accum_kernels.cu (pulse-chunked jobs)
cudaError_t launch_store_job(const DevJob &dj, DevJob *d_dst, cudaStream_t st);
cudaError_t launch_chunk_tables(const double4 *pulse, const float *wP, int P, int q0, int n, double4 *pulse_c,
                                float *wP_c, cudaStream_t st);
cudaError_t launch_finalize(const DevJob *d_job, long long npix, int num_sms, cudaStream_t st);
cudaError_t launch_fill_items(WorkItem *items, int ntiles, RowItem *rows, int nrows, cudaStream_t st);
// jobs d_list[0 .. nlist) of d_jobs, formed in pulse parts: sum of the parts
// times the final phase into out (row flip), max |z|
cudaError_t launch_combine_parts(const DevJob *d_jobs, const int *d_list, int nlist, long long max_pixels,
                                 int num_sms, cudaStream_t st);

// resize.cu (the reference's data/resize.py resampling)
struct ResizePlan {
    int elem_bytes;        // 4 (f32) or 8 (f64)
    int nc;                // interleaved components resampled independently
    int rows, cols, orows, ocols;
    double zoom[2];        // input / output extent per axis
    int radius[2];         // Gaussian radius per axis; -1: axis not filtered
    int woff[2];           // offset of each axis's weights w[0..radius] in d_weights
    const double *d_weights;
    void *d_taps;          // (orows + ocols) * 32 bytes of scratch: the zoom's taps per index
};
cudaError_t launch_resize(const ResizePlan &p, const void *in, void *out, void *tmp_a, void *tmp_b,
                          double *bounds, cudaStream_t st);

// peaks.cu
cudaError_t measure_peaks(int num_sms, cudaStream_t st, double *ffma_per_s, double *mufu_per_s);

// output.cu
cudaError_t launch_maxabs(const double2 *img, long long n, unsigned long long *d_max, cudaStream_t st);
cudaError_t launch_db_u8(const double2 *img, long long n, const unsigned long long *d_max,
                         double *dB, uint8_t *u8, double dB_min, double dB_max, cudaStream_t st);
cudaError_t launch_u8_from_db(const double *dB, long long n, double dB_min, double dB_max,
                              uint8_t *u8, cudaStream_t st);
// u8 image straight from a complex image and its max|z| (no f64 dB image)
cudaError_t launch_img_u8(const double2 *img, long long n, const unsigned long long *d_max, uint8_t *u8,
                          double lo, double hi, cudaStream_t st);
// u8 images of every job of a batch that asked for one (uses DevJob::maxabs)
cudaError_t launch_batch_u8(const DevJob *d_jobs, int njobs, long long max_pixels, cudaStream_t st);

}  // namespace sarbp
