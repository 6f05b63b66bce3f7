/*
 * sarbp_b200.h -- C ABI of the B200 SAR backprojection library
 * (libsarbp_b200.so).
 *
 * Drop-in for the `-s cuda` path of ISI-apex/halide-sar-app: the same
 * inputs as the reference's Halide pipeline `backprojection_cuda`
 * (backprojection.cpp:35-46, called at sarbp.cpp:277), as plain pointers
 * and sizes, plus the dB / u8 output stages (img_output.cpp:10-52).
 *
 * Conventions
 *  - Every function returns an int status: SARBP_OK (0) or a negative
 *    SARBP_ERR_* code; sarbp_last_error() gives a message for the calling
 *    thread.  Nothing aborts and no kernel traps.
 *  - Layouts follow the reference's Halide buffers:
 *      phs        complex64 [npulses][nsamples]   (Halide {2, S, P})
 *      k_r        [nsamples]
 *      pos        [npulses][3]                    (Halide {3, P})
 *      r          SoA [3][nu*nv], pixel i at u index i % nu, v index i / nu
 *                                                 (Halide {nu*nv, 3})
 *      output_img complex128 [nv][nu], rows flipped as in
 *                 backprojection.cpp:130          (Halide {2, nu, nv})
 *  - Functions named *_device take device pointers and enqueue on the
 *    context's stream without synchronising; the others take host pointers
 *    and return when the result is in host memory.
 *  - A context is used by one host thread at a time.
 */
#ifndef SARBP_B200_H
#define SARBP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SARBP_OK 0
#define SARBP_ERR_INVALID (-1)     /* bad argument, shape or size */
#define SARBP_ERR_UNSUPPORTED (-2) /* e.g. N_fft not a power of two in [16, 131072] */
#define SARBP_ERR_NOMEM (-3)       /* device or host allocation failed */
#define SARBP_ERR_CUDA (-4)        /* a CUDA runtime call failed */
#define SARBP_ERR_GEOMETRY (-5)    /* non-finite geometry, or a pixel tile whose
                                      range window does not fit on chip */
#define SARBP_ERR_TIMEOUT (-6)     /* a bounded wait gave up */
#define SARBP_ERR_ADMISSION (-7)   /* serving: job exceeds the HBM cap */
#define SARBP_ERR_STATE (-8)       /* call not valid in the current state */

/* Precision of the pulse-accumulation kernel. */
#define SARBP_PREC_COMPAT 0  /* the reference's semantics: f32 pos, f32 |pos|
                                (norm_r0), f32 k_c; split-precision kernel */
#define SARBP_PREC_PRECISE 1 /* f64 per-pulse geometry (positions, |pos|, k_c);
                                split-precision kernel */
#define SARBP_PREC_NAIVE 2   /* plain FP32 range and phase per pixel*pulse
                                (precision-study baseline) */

/* Taylor window of range compression (signal.h:14-51). */
#define SARBP_TAYLOR_REF 0   /* the reference's expression as Halide types it:
                                the F_m denominator term (m+1)^2/(r+1)^2 is an
                                Int32 division (signal.h:40), which is zero-
                                divided, so undefined, above 30 dB; such levels
                                are rejected with SARBP_ERR_INVALID */
#define SARBP_TAYLOR_FLOAT 1 /* the same window with that quotient taken in
                                floating point (the published RITSAR taylor()
                                the reference restates); defined at every level.
                                A deviation from the reference, chosen per job. */

typedef struct sarbp_ctx sarbp_ctx;

/* Kernel tuning; a zero field means "library default / autotuned". */
typedef struct sarbp_opts {
    int precision;   /* SARBP_PREC_* */
    int tile_x;      /* pixel tile width  (16, 32 or 64) */
    int tile_y;      /* pixel tile height (tile_x*tile_y in {512, 1024, 2048}) */
    int pulse_chunk; /* pulses staged per chunk (4..256) */
    int persistent;  /* 0 or 1: persistent work-list launch; 2: one CTA per tile */
    int stage_cap;   /* float4 entries of each half of the range-window staging buffer */
    int min_blocks;  /* CTAs per SM the kernel's registers are sized for (2 or 3) */
    int pulse_parts; /* work items per pixel tile over consecutive pulse ranges: 0 = chosen
                        per job (images below 2^18 pixels whose tiles leave resident CTAs
                        idle are split; the parts' sums are added in a fixed order, so a
                        job forms the same image alone and in any batch), 1 = one item
                        per tile, 2..16 = that many parts (at most one per pulse) */
} sarbp_opts;

/*
 * One image-formation job with all arrays device-resident.  Exactly one of
 * (r) or (u, v, u_hat, v_hat) describes the pixel positions: when r is
 * NULL, pixel (ix, iy) sits at u_hat*u[ix] + v_hat*v[iy]
 * (img_plane.cpp:92-102) and no nu*nv*3 position array is read.
 */
typedef struct sarbp_job {
    int nsamples, npulses, n_fft, taylor_s_l, nu, nv;
    double delta_r;
    const float *phs;    /* complex64 [P][S] */
    const float *k_r;    /* [S] f32, used in COMPAT / NAIVE */
    const double *k_r64; /* [S] f64, used in PRECISE (may be NULL -> k_r) */
    const float *pos;    /* [P][3] f32, used in COMPAT / NAIVE */
    const double *pos64; /* [P][3] f64, used in PRECISE (may be NULL -> pos) */
    const double *r;     /* SoA [3][nu*nv] or NULL */
    const double *u;     /* [nu], when r == NULL */
    const double *v;     /* [nv], when r == NULL */
    double u_hat[3], v_hat[3];
    double *output_img;  /* complex128 [nv][nu] (device) */
    uint8_t *out_u8;     /* optional: u8 image [nv][nu] (device), or NULL */
    double dB_min, dB_max; /* used when out_u8 != NULL */
    int precision;       /* SARBP_PREC_*; overrides opts->precision when >= 0 */
    int taylor_mode;     /* SARBP_TAYLOR_REF (0) or SARBP_TAYLOR_FLOAT */
} sarbp_job;

/* ---- context ---- */
int sarbp_ctx_create(int device, sarbp_ctx **out);
int sarbp_ctx_destroy(sarbp_ctx *ctx);
/* Launch on a caller-owned cudaStream_t (NULL = the context's own stream). */
int sarbp_ctx_set_stream(sarbp_ctx *ctx, void *cuda_stream);
void *sarbp_ctx_stream(sarbp_ctx *ctx);
int sarbp_ctx_synchronize(sarbp_ctx *ctx);
/* Kernels this context has launched so far (all entry points). */
long long sarbp_ctx_launch_count(sarbp_ctx *ctx);
/* Record CUDA events around each stage of every batch (on = 1). */
int sarbp_ctx_set_timing(sarbp_ctx *ctx, int on);
/* Device time (ms) of the last batch's stages: [0] set-up kernel, [1] range
 * compression, [2] tile geometry, [3] backprojection, [4] u8 output; -1 for
 * a stage that did not run.  Waits for the batch. */
int sarbp_ctx_last_stage_ms(sarbp_ctx *ctx, float *ms5);
/* Measured FP32 FFMA instructions/s and SFU (MUFU) operations/s of the
 * context's device, from two chain microkernels. */
int sarbp_measure_peaks(sarbp_ctx *ctx, double *ffma_per_s, double *mufu_per_s);
const char *sarbp_last_error(void);
const char *sarbp_version(void);

/*
 * Backprojection with host buffers: replaces the Halide pipeline
 * `int backprojection_cuda(phs, k_r, taylor_s_l, N_fft, delta_r, u, v, pos,
 * r, output_img)` (backprojection.cpp:35-46, sarbp.cpp:277).  Range
 * compression (the FFTW extern call_dft, dft.cpp:40-79) runs on the device.
 * opts may be NULL (SARBP_PREC_COMPAT, autotuned tiles).
 */
int sarbp_backprojection(sarbp_ctx *ctx, const float *phs, int nsamples,
                         int npulses, const float *k_r, int taylor_s_l,
                         int n_fft, double delta_r, const double *u, int nu,
                         const double *v, int nv, const float *pos,
                         const double *r, double *output_img,
                         const sarbp_opts *opts);

/*
 * The same image from the image-plane axes instead of pixel_locs: pixel
 * (i, j) is u_hat * u[i] + v_hat * v[j] (img_plane.cpp:92-102, the r array
 * img_plane_create builds, ImgPlane.cpp:16-63), formed on the device in the
 * same f64 arithmetic, so the nu*nv*3 f64 positions are neither built on the
 * host nor copied.  Used by the sarbp CLI.
 */
int sarbp_backprojection_plane(sarbp_ctx *ctx, const float *phs, int nsamples,
                               int npulses, const float *k_r, int taylor_s_l,
                               int n_fft, double delta_r, const double *u,
                               int nu, const double *v, int nv,
                               const double u_hat[3], const double v_hat[3],
                               const float *pos, double *output_img,
                               const sarbp_opts *opts);

/* The same with f64 positions and k_r (SARBP_PREC_PRECISE by default). */
int sarbp_backprojection_f64(sarbp_ctx *ctx, const float *phs, int nsamples,
                             int npulses, const double *k_r, int taylor_s_l,
                             int n_fft, double delta_r, const double *u,
                             int nu, const double *v, int nv,
                             const double *pos, const double *r,
                             double *output_img, const sarbp_opts *opts);

/* Device-resident single job (enqueued, not synchronised). */
int sarbp_backprojection_device(sarbp_ctx *ctx, const sarbp_job *job,
                                const sarbp_opts *opts);

/*
 * Range compression only (backprojection.cpp:79-104 with the FFT extern
 * call_dft, dft.cpp:40-79): writes the complex64 range profiles Q
 * [npulses][n_fft] of `job` to the device buffer q_out.  The pixel and
 * output fields of `job` are not used.
 */
int sarbp_range_compress_device(sarbp_ctx *ctx, const sarbp_job *job,
                                const sarbp_opts *opts, float *q_out);

/*
 * Many jobs of uneven size in one batch: one window kernel, one range
 * compression launch per distinct N_fft, and one persistent backprojection
 * launch over a (job, pixel tile, pulse part) work list ordered
 * longest-first (small jobs split their tiles' pulses into parts, see
 * sarbp_opts.pulse_parts), then one combine launch for the jobs formed in
 * parts.  Enqueued on the context's stream, not synchronised.
 */
int sarbp_batch_device(sarbp_ctx *ctx, const sarbp_job *jobs, int njobs,
                       const sarbp_opts *opts);

/*
 * A batch captured as a CUDA graph (no counterpart in the reference, which
 * forms one image per call).  sarbp_plan_create runs the batch once (this
 * writes the jobs' outputs and sizes the plan's own scratch), then captures
 * the same launch sequence into a graph on a stream of the plan.
 * sarbp_plan_launch replays it on cuda_stream (NULL: the plan's stream);
 * the job arrays may hold new data between replays but keep their device
 * addresses and shapes, and one replay must finish before the next starts
 * (replays share the plan's scratch).  sarbp_plan_wait synchronises the
 * last replay's stream and returns its status (as sarbp_ctx_synchronize).
 */
typedef struct sarbp_plan sarbp_plan;
int sarbp_plan_create(sarbp_ctx *ctx, const sarbp_job *jobs, int njobs,
                      const sarbp_opts *opts, sarbp_plan **out);
int sarbp_plan_launch(sarbp_plan *plan, void *cuda_stream);
int sarbp_plan_wait(sarbp_plan *plan);
/* kernel nodes in the plan's graph (launches per replay) */
int sarbp_plan_kernel_count(const sarbp_plan *plan);
int sarbp_plan_destroy(sarbp_plan *plan);

/*
 * Serving loop (no counterpart in the reference): continuous batching of
 * image-formation requests under a device-memory budget.  A request is a
 * sarbp_job whose pointers are HOST memory (output_img and out_u8, each
 * optional, receive the complex128 and u8 images); the caller keeps them
 * valid until the request is done.  A scheduler thread admits queued
 * requests in arrival order while their device footprint (inputs, outputs,
 * and their batch's scratch) fits hbm_cap_bytes, uploads each phase history
 * once, and launches them as one batch on the first free of `lanes` streams
 * (default 3), at most max_batch requests (default 32) and max_batch_work
 * pixel*pulses (default 6e9, about 5 ms of work) per batch; batches of
 * different lanes overlap on the device and complete in whichever order
 * they finish.  A request that cannot fit an idle
 * server fails with SARBP_ERR_ADMISSION.  `launch` (may be NULL) fixes the
 * precision and launch shape of every batch, so a request's image does not
 * depend on what it was batched with.
 */
typedef struct sarbp_server sarbp_server;
int sarbp_server_create(sarbp_ctx *ctx, const sarbp_opts *launch,
                        double hbm_cap_bytes, int lanes, int max_batch,
                        double max_batch_work, sarbp_server **out);
int sarbp_server_submit(sarbp_server *server, const sarbp_job *host_job,
                        long long *id);
/* Waits up to timeout_s (< 0: no limit) for request id; returns its status,
 * or SARBP_ERR_TIMEOUT while it is still queued or running. */
int sarbp_server_wait(sarbp_server *server, long long id, double timeout_s);
/* Seconds since the server started: submission, admission (batch launch),
 * completion (images on the host; -1 while in flight). */
int sarbp_server_times(sarbp_server *server, long long id, double *submit_s,
                       double *start_s, double *done_s);
/* Forgets a finished request. */
int sarbp_server_release(sarbp_server *server, long long id);
int sarbp_server_stats(sarbp_server *server, long long *submitted,
                       long long *completed, long long *batches,
                       double *in_use_bytes, double *peak_bytes);
/* Finishes every queued and running request, then frees the server. */
int sarbp_server_destroy(sarbp_server *server);

/*
 * Registered apertures: the phase history of `host_aperture` (HOST
 * pointers: phs, k_r and/or k_r64, pos and/or pos64; sizes, n_fft, Taylor
 * level and mode, delta_r, precision -- <0: the server's) is uploaded and
 * range-compressed ONCE, on the calling thread, and stays resident on the
 * device as interpolation pairs (16 B x npulses x (n_fft + 1)) with its k_r
 * and positions, charged to the server's budget until unregistered
 * (SARBP_ERR_ADMISSION when it does not fit).  Requests submitted on it
 * with sarbp_server_submit_on bring only their image plane (nu, nv, and r or
 * u/v/u_hat/v_hat) and outputs (output_img, out_u8 with dB_min/dB_max), all
 * host memory; the rest of host_job is ignored.  Their batches neither
 * upload nor range-compress the phase history.  An aperture can be
 * unregistered once none of its requests is queued or running.
 */
int sarbp_server_register(sarbp_server *server, const sarbp_job *host_aperture,
                          long long *aperture);
int sarbp_server_submit_on(sarbp_server *server, long long aperture,
                           const sarbp_job *host_job, long long *id);
int sarbp_server_unregister(sarbp_server *server, long long aperture);
/*
 * Streaming apertures: a partial image kept on the device while an
 * aperture's phase history arrives in pulse chunks (a pulse-chunked
 * accumulator, sarbp_accum_*, under the server's budget and beside its
 * batches).  sarbp_server_open_stream takes a job of HOST pointers (k_r,
 * antenna positions of all npulses pulses, image plane, output_img and
 * optional out_u8; phs is not read), charges its device footprint
 * (sarbp_job_device_bytes with max_chunk) to the budget
 * (SARBP_ERR_ADMISSION when it does not fit) and uploads those inputs;
 * sarbp_server_stream_add range-compresses host phase-history rows
 * [pulse0, pulse0 + count) and adds them to the partial image on the
 * stream's own streams, overlapped with the lanes' batches (the rows may be
 * reused once the next add or the finish returns); sarbp_server_stream_finish
 * applies the final phase and row flip, copies the image(s) to the host,
 * waits, frees the stream and returns its status.  Calls on one stream
 * from several host threads are serialised (an add after the finish
 * returns SARBP_ERR_INVALID); different streams proceed independently.
 */
int sarbp_server_open_stream(sarbp_server *server, const sarbp_job *host_job,
                             int max_chunk, long long *stream_id);
int sarbp_server_stream_add(sarbp_server *server, long long stream_id, int pulse0,
                            int count, const float *phs_rows_host);
int sarbp_server_stream_finish(sarbp_server *server, long long stream_id);

/* Bytes the server copied host -> device, pulses it range-compressed, and
 * requests it served from registered apertures, since it started. */
int sarbp_server_counters(sarbp_server *server, double *h2d_bytes,
                          long long *rc_pulses, long long *resident_requests);

/*
 * Pulse-chunked image formation (no counterpart in the reference, which
 * range-compresses and backprojects all pulses of a job in one call,
 * backprojection.cpp:67-138): a device-resident partial image that
 * accumulates the aperture's pulses chunk by chunk, for apertures whose
 * phase history arrives over time or whose one-shot scratch (16 B x P x
 * n_fft of range profiles and 32 B x P per 32x32-pixel tile of pulse
 * geometry) does not fit.  The image is the reference's: a sum over pulses
 * followed by the final phase of pulse P/2 and the row flip
 * (backprojection.cpp:126-135), with the reference's pulse pairing
 * (phase-history row q weighs w_P[q] and meets antenna position
 * (q - P mod 2) mod P, from the double fftshift of backprojection.cpp:98,104).
 *
 * sarbp_accum_create: `job` holds device pointers and the WHOLE aperture's
 *   sizes (npulses = P), k_r, antenna positions of all P pulses, Taylor
 *   level, pixel positions (r, or u/v/u_hat/v_hat) and outputs (output_img,
 *   optional out_u8); job->phs is not read.  The pointers must stay valid
 *   until destroy.  Device memory: the windows, pulse and tile tables, the
 *   final phase and a complex f32 partial image (8 B per pixel each), plus
 *   scratch for one chunk of up to max_chunk pulses.  Enqueues its set-up
 *   on the context's stream.  SARBP_PREC_COMPAT or SARBP_PREC_PRECISE.
 * sarbp_accum_add_device: range-compresses phase-history rows
 *   [pulse0, pulse0 + count) (phs_rows: complex64 [count][nsamples] on the
 *   device, count <= max_chunk) and adds them to the partial image.
 *   Chunks may come in any order; each pulse exactly once (again:
 *   SARBP_ERR_STATE).  Enqueued on the context's stream.
 * sarbp_accum_add: the same from host memory: the rows go up on the
 *   context's copy stream into one of two staging buffers while the
 *   previous chunk computes.  With pinned memory the copy is asynchronous:
 *   keep the rows unchanged until the next sarbp_accum_add or
 *   sarbp_accum_wait returns.
 * sarbp_accum_finalize: once all P pulses are in, enqueues the final phase
 *   and row flip into output_img (and the u8 image).
 * sarbp_accum_wait: waits for the accumulator's work; after finalize,
 *   returns the kernels' status as sarbp_ctx_synchronize does.
 * sarbp_accum_reset: zeroes the partial image for a new aperture on the
 *   same geometry (same positions, pixels and sizes).
 */
typedef struct sarbp_accum sarbp_accum;
int sarbp_accum_create(sarbp_ctx *ctx, const sarbp_job *job,
                       const sarbp_opts *opts, int max_chunk,
                       sarbp_accum **out);
int sarbp_accum_add_device(sarbp_accum *acc, int pulse0, int count,
                           const float *phs_rows);
int sarbp_accum_add(sarbp_accum *acc, int pulse0, int count,
                    const float *phs_rows_host);
int sarbp_accum_finalize(sarbp_accum *acc);
int sarbp_accum_wait(sarbp_accum *acc);
int sarbp_accum_reset(sarbp_accum *acc);
/* device bytes the accumulator holds (with its staging buffers) */
double sarbp_accum_device_bytes(const sarbp_accum *acc);
int sarbp_accum_destroy(sarbp_accum *acc);

/*
 * Device bytes a job needs: its inputs and outputs plus the library's
 * scratch, formed in one call (chunk_pulses <= 0) or through a pulse-chunked
 * accumulator with chunks of min(chunk_pulses, npulses) pulses and two
 * staging buffers (the phase history itself then never resides whole).
 */
int sarbp_job_device_bytes(const sarbp_job *job, const sarbp_opts *opts,
                           int chunk_pulses, double *bytes);

/*
 * A job with HOST pointers (as for the serving loop) formed under a device
 * memory cap: picks the largest pulse chunk whose footprint
 * (sarbp_job_device_bytes) fits max_device_bytes, evens the chunks out,
 * uploads the inputs other than the phase history, streams the phase
 * history chunk by chunk (each upload overlapped with the previous chunk's
 * kernels) through a pulse-chunked accumulator, and copies the image (and
 * u8 image) back.  *chunk_pulses and *device_bytes (either may be NULL)
 * receive the chunk size used and the device memory held.  Returns when the
 * image is on the host.
 */
int sarbp_backprojection_streamed(sarbp_ctx *ctx, const sarbp_job *host_job,
                                  const sarbp_opts *opts,
                                  double max_device_bytes, int *chunk_pulses,
                                  double *device_bytes);

/*
 * Launch-shape autotuner: runs the batch with each candidate pixel tile
 * (32x32, 32x16, 64x16, 16x32 at 3 CTAs/SM; 32x32, 32x64, 64x32, 16x64 at
 * 2, with the staging buffer grown into the third CTA's shared memory) and
 * pulse-chunk depth (32, 64, 128), times set-up through backprojection
 * with CUDA events, re-times the three fastest, and writes the fastest
 * tile_x, tile_y, min_blocks, pulse_chunk and stage_cap into *inout (other
 * fields kept).  The result is cached in the context under the batch's
 * shape signature (sizes and precision), so a later call with the same
 * shapes returns at once (*best_ms = -1 then).  Writes the jobs' outputs.
 */
int sarbp_autotune(sarbp_ctx *ctx, const sarbp_job *jobs, int njobs,
                   sarbp_opts *inout, float *best_ms);

/*
 * Backprojection of one device-resident job that allocates nothing (no
 * counterpart in the reference).  For callers that must not allocate device
 * memory when they need an image: processes whose device memory is handed
 * out up front by a pool they do not own (a cudaMalloc there fails, or
 * fragments and bypasses the pool), and real-time loops that cannot take
 * cudaMalloc's latency and implicit device synchronisation on the path that
 * forms each image.  Runs the same kernels as sarbp_backprojection_device on
 * `cuda_stream`, with all scratch in one static 64 MiB device array of the
 * library:
 *  - jobs needing more scratch than that, or an N_fft above 16384, return
 *    SARBP_ERR_UNSUPPORTED
 *    (roughly: 256 KiB of twiddle tables + 16 B x npulses x n_fft + 32 B x
 *    npulses x tiles of 32x32 pixels + 8 B x pixels);
 *  - every call shares the array and it keeps the last call's contents, so
 *    calls that overlap on the GPU race: serialise them;
 *  - the first call on a device looks up the array, sets kernel attributes
 *    and fills the twiddle tables, then waits for `cuda_stream`; make it
 *    before any stream capture.  That set-up is kept until the process
 *    exits: after cudaDeviceReset the entry point must not be used again;
 *  - precision SARBP_PREC_COMPAT or SARBP_PREC_PRECISE only;
 *  - `status` (device int) receives the kernels' status bits (0 = fine;
 *    1 = a pixel tile too spread out, left at zero; 2 = non-finite geometry;
 *    8 = a bounded wait for a copy gave up).  It may be NULL, but then
 *    those conditions go unreported: the call returns SARBP_OK and the image
 *    may be wrong.
 * The array stays allocated on every GPU that loads the library until exit.
 */
int sarbp_backprojection_noalloc(const sarbp_job *job, void *cuda_stream, int *status);

/* ---- dB / u8 output stages (img_output.cpp:10-52) ---- */
/* dB = 10*log10(|z| / max|z|) for a complex128 [nv][nu] image. */
int sarbp_img_output_to_dB(sarbp_ctx *ctx, const double *img, int nu, int nv,
                           double *dB);
/* u8 = trunc(clamp((clamp(dB,min,max)-min)/(max-min)*255, 0, 255)). */
int sarbp_img_output_u8(sarbp_ctx *ctx, const double *dB, int nu, int nv,
                        double dB_min, double dB_max, uint8_t *out);
int sarbp_img_output_to_dB_device(sarbp_ctx *ctx, const double *img, int nu,
                                  int nv, double *dB);
int sarbp_img_output_u8_device(sarbp_ctx *ctx, const double *dB, int nu,
                               int nv, double dB_min, double dB_max,
                               uint8_t *out);

/* img_output_to_dB then img_output_u8 (sarbp.cpp:299-316) in one device
 * pass that writes only the u8 image (no f64 dB image): a max|z| reduction,
 * then the per-pixel grey levels.  The same conversion as the u8 output of a
 * job (sarbp_job.out_u8).  Enqueued, not synchronised. */
int sarbp_img_output_u8_from_img_device(sarbp_ctx *ctx, const double *img, int nu,
                                        int nv, double dB_min, double dB_max,
                                        uint8_t *out);

/*
 * Resampling of platform arrays to other pulse / sample counts: the
 * computation of the reference's data/resize.py (data/resize.py:14-70),
 * skimage.transform.resize(a, (out_rows, out_cols), preserve_range=True)
 * with its defaults -- linear interpolation on grid-aligned sample
 * positions, mirrored edges, a Gaussian anti-aliasing filter of sigma
 * (in/out - 1)/2 on the axes that shrink (when any axis shrinks), output
 * clipped to the input's range -- restated on the device.  `in`/`out` are
 * [rows][cols][ncomp] arrays of f32 (elem_bytes 4) or f64 (8); the ncomp
 * interleaved components (re, im of a complex array) are resampled
 * independently.  A 1-D array is rows = 1.  The _device form takes device
 * pointers and is enqueued on the context's stream; sarbp_resize takes host
 * pointers and returns when `out` is written.
 */
int sarbp_resize_device(sarbp_ctx *ctx, int elem_bytes, int ncomp, const void *in,
                        int rows, int cols, int out_rows, int out_cols, void *out);
int sarbp_resize(sarbp_ctx *ctx, int elem_bytes, int ncomp, const void *in, int rows,
                 int cols, int out_rows, int out_cols, void *out);

/* ---- host helpers used by the CLI and the harness ---- */
/* Taylor window (signal.h:14-51), f64 [num]. */
int sarbp_taylor(int num, double S_L, double *out);
/* The same with a SARBP_TAYLOR_* mode (no counterpart in the reference). */
int sarbp_taylor_mode(int num, double S_L, int mode, double *out);
/* nu/nv of img_plane_create (ImgPlane.cpp:20-28). */
int sarbp_img_plane_dims(int nsamples, int npulses, int upsample, int *nu,
                         int *nv);
/* img_plane_create (ImgPlane.cpp:16-63): u[nu], v[nv], k_u, k_v, u_hat[3],
 * v_hat[3], and pixel_locs SoA [3][nu*nv] when non-NULL. */
int sarbp_img_plane(int nsamples, int npulses, double delta_r,
                    const float *R_c, const float *n_hat, double res_factor,
                    double aspect, int upsample, double *d_u, double *d_v,
                    double *u, double *v, double *k_u, double *k_v,
                    double *u_hat, double *v_hat, double *pixel_locs);

/*
 * Seeded synthetic stepped-frequency phase history (the harness's stand-in
 * for the AFRL / Sandia data): circular aperture of npulses positions at
 * slant range R0, depression dep_deg, azimuth span span_deg, centred on the
 * scene origin; scatterers (x, y, z, amplitude re, im) summed as
 * S(f,p) = sum_i a_i exp(+j 4 pi f/c (|p| - |p - x_i|)), plus complex
 * Gaussian noise at snr_db (no noise when snr_db >= 300).
 * Outputs: phs complex64 [P][S], pos f64 [P][3], k_r f64 [S].
 */
int sarbp_synth_phase_history(int nsamples, int npulses, double f0, double df,
                              double R0, double dep_deg, double span_deg,
                              const double *scat, int nscat, double snr_db,
                              uint64_t seed, float *phs, double *pos,
                              double *k_r, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
