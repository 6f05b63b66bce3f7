// runner.h -- enqueues one batch of image-formation jobs on a stream.
//
// A Runner owns the device memory a batch needs besides the caller's
// arrays: the job descriptors, row and work-item lists, and a grow-only
// scratch arena for range profiles, windows and per-pulse geometry.  One
// Runner serves one stream; the serving loop keeps several.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "internal.h"
#include "kernels.h"
#include "sarbp_b200.h"

namespace sarbp {

void set_error(const std::string &msg);
const char *last_error_cstr();
int fail(int code, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);

struct DeviceBuffer {
    void *ptr = nullptr;
    size_t cap = 0;
    // Grows to at least `bytes`; synchronises `st` before freeing the old one.
    cudaError_t ensure(size_t bytes, cudaStream_t st);
    // Frees any previous buffer (the caller makes sure it is idle) and
    // allocates exactly `bytes`, rounded up to 256.
    cudaError_t alloc_exact(size_t bytes);
    void release();
};

struct PinnedBuffer {
    void *ptr = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes);
    void release();
};

// Per-device constants shared by all runners of a context.
struct DeviceInfo {
    int device = 0;
    int num_sms = 148;
    std::map<int, float2 *> twiddles;  // logN -> device table (guarded by mu)
    std::mutex mu;
    std::atomic<long long> launches{0};
    // stage timing: events [0] before set-up, [1] after set-up, [2] after
    // range compression, [3] after tile geometry, [4] after backprojection,
    // [5] after u8
    static constexpr int kEvents = 6;
    bool timing = false;
    cudaEvent_t ev[kEvents] = {};
    bool ev_recorded[kEvents] = {};
    cudaError_t record(int i, cudaStream_t st);
    cudaError_t twiddle(int logN, float2 **out);
    bool has_twiddle(int logN);
    void release();
};

// Range compression of rows of one N_fft on st: the single-row kernel up to
// 2^kMaxLogNSmem, above it the four-step FFT through `work`, which holds
// work_rows rows of N_fft complex values (reused from launch to launch).
cudaError_t range_compress_rows(DeviceInfo *dev, int logN, const DevJob *d_jobs, const RowItem *d_rows, int nrows,
                                int pairs, float2 *work, int work_rows, cudaStream_t st);

// Row slabs of a single job, for overlapping its host<->device copies with
// compute: slab g covers tile rows [row0[g], row0[g + 1]).
// After prep and range compression (on the main stream), slab g's tile
// geometry and backprojection run on the main stream (g even) or `aux`
// (g odd) once `ready[g]` has fired (when set), and `done[g]` is recorded
// when its pixels are final; the main stream joins every slab at the end.
// Consecutive slabs sit on different streams so that one slab's CTAs fill
// the SMs while the previous slab's last tiles finish.
struct SlabSpec {
    int nslabs = 0;
    const int *row0 = nullptr;  // [nslabs + 1] tile-row boundaries, ascending
    cudaStream_t aux = nullptr;
    const cudaEvent_t *ready = nullptr;  // [nslabs] or NULL
    const cudaEvent_t *done = nullptr;   // [nslabs]
    // Called once the descriptors and the range compression are enqueued and
    // before any slab waits on `ready`: the place to issue the slabs' input
    // copies and record `ready`.  Host-to-device copies of all streams share
    // the copy engine in issue order, so copies issued earlier would hold
    // back the batch's own descriptor upload.
    std::function<cudaError_t()> before_slabs;
    // When set, the batch's descriptors are uploaded on this stream (where
    // the caller has already queued the phase-history copies) and the
    // kernels wait for them there: the copy engine runs one stream's queue
    // ahead of another's, so a descriptor copy on the compute stream could
    // wait behind every queued input copy.
    cudaStream_t copy_stream = nullptr;
};

class Runner {
public:
    explicit Runner(DeviceInfo *dev) : dev_(dev) {}
    ~Runner();
    // Validates and enqueues jobs on st.  Returns SARBP_OK or an error code
    // (no device work is enqueued on a validation error).
    // With q_out set, only range compression runs and job 0's profiles are
    // copied there.
    // With for_graph set the call is being captured into a CUDA graph: no
    // stage events, no wait on the previous descriptor copy (the captured
    // copy re-reads this Runner's pinned descriptors at every replay, so the
    // Runner must not enqueue anything else afterwards), and every buffer
    // must already be large enough (an uncaptured enqueue of the same jobs
    // comes first).
    // With resident_qp, job i whose resident_qp[i] is non-NULL uses those
    // range profiles (interpolation pairs [P][N+1], formed beforehand) and
    // needs no phase history: its range compression is skipped.
    int enqueue(const sarbp_job *jobs, int njobs, const sarbp_opts *opts, cudaStream_t st,
                void *q_out = nullptr, bool for_graph = false, const SlabSpec *slabs = nullptr,
                const float4 *const *resident_qp = nullptr);
    // tile size the next enqueue with these options uses
    static void tile_shape(const sarbp_opts *opts, int *tile_x, int *tile_y);
    // Waits for the last batch and reads the kernels' status words.
    int check_status(cudaStream_t st);
    // Device footprint of the library scratch a job needs (bytes) on a GPU
    // of num_sms SMs.
    static size_t job_scratch_bytes(const sarbp_job &j, const sarbp_opts *opts = nullptr,
                                    bool resident_profiles = false, int num_sms = 148);
    // Frees the scratch (the Runner must be idle).
    void release_scratch() { scratch_.release(); }
    // Take each batch's scratch from `pool` (stream-ordered) instead of the
    // grow-only buffer; not for graph capture.
    void use_pool(cudaMemPool_t pool) { pool_ = pool; }
    // Scratch currently held (grow-only).
    size_t scratch_capacity() const { return scratch_.cap + meta_.cap; }
    // false: never record the context's stage-timing events (runners driven
    // from another thread, e.g. the serving loop's lanes)
    bool stage_events = true;

private:
    DeviceInfo *dev_;
    DeviceBuffer scratch_, meta_;
    PinnedBuffer host_meta_;
    cudaEvent_t meta_done_ = nullptr;  // host_meta_ may be rewritten after this
    cudaEvent_t front_done_ = nullptr; // range compression done (slabbed runs)
    // Range compression runs on side_ beside the tile geometry on the main
    // stream (both only read the set-up's tables); fork_/join_ order them.
    cudaStream_t side_ = nullptr;
    cudaEvent_t fork_ = nullptr, join_ = nullptr;
    int last_njobs_ = 0;
    PinnedBuffer status_pin_;          // JobScalars of the last batch, copied behind it
    cudaMemPool_t pool_ = nullptr;
};

BpLaunch default_launch(const sarbp_opts *opts, int num_sms);
// default_launch with the CTAs per SM the enqueue uses: a tile shape without
// a 3-CTA/SM build runs at 2 unless the caller asked
BpLaunch resolved_launch(const sarbp_opts *opts, int num_sms);

// Pulse parts per tile of a one-shot job (DevJob::nsplit): L.parts when the
// caller set it (at most one part per pulse); otherwise 1 for images of
// 2^18 pixels and more and for jobs whose tiles fill more than half of the
// resident CTAs, and else the part count with the best estimated use of
// the SMs (whole waves of equal items, a fixed cost per item), each part at
// least 32 pulses, at most 16 parts, and 1 unless that beats one item per
// tile by 15 %.  Depends only on the job's sizes, the launch shape and the
// SM count, so a job splits the same way alone and in any batch.
int pulse_parts(int nu, int nv, int P, const BpLaunch &L, int num_sms);

// Checks a job's sizes, pointers and Taylor level (SARBP_OK or an error code
// with the message set); need_phs = false for pulse-chunked jobs, whose
// phase history comes chunk by chunk.
int validate_job(const sarbp_job &j, int prec, int idx, bool rc_only, bool need_phs);
// Fills the sizes, Taylor coefficients, caller pointers, range-axis
// constants and outputs of a job's descriptor (not its scratch pointers).
void describe_job(const sarbp_job &j, int prec, int tile_x, int tile_y, DevJob &dj);

}  // namespace sarbp

struct sarbp_ctx;
struct sarbp_accum;
namespace sarbp {
// sarbp_accum_create on the given compute and copy streams instead of the
// context's (the serving loop's streaming apertures); NULL: the context's.
int accum_create_on(sarbp_ctx *ctx, const sarbp_job *job, const sarbp_opts *opts, int max_chunk,
                    cudaStream_t stream, cudaStream_t copy_stream, sarbp_accum **out);
// Device bytes of a job's inputs other than its phase history, and its
// outputs (the host-buffer paths' device copies).
size_t job_io_bytes(const sarbp_job &j, bool with_phs);

}  // namespace sarbp
