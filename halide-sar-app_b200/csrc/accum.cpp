// accum.cpp -- pulse-chunked image formation: a device-resident partial
// image that accumulates the aperture's pulses chunk by chunk (no
// counterpart in the reference, which range-compresses and backprojects all
// pulses in one call, backprojection.cpp:67-138).
//
// The image of backprojection.cpp:126-135 is a sum over pulses followed by
// one per-pixel phase:
//     out[nv-1-y][x] = exp(+j k_c dr(pixel, P/2)) * sum_p Qhat(pixel, p) exp(-j k_c dr(pixel, p))
// so the sum can be formed over any partition of the pulses.  An sarbp_accum
// holds, for one job (pixel positions, antenna positions of all P pulses,
// k_r, Taylor level): the windows and the pulse table of the whole aperture,
// the tile table and the final phase per pixel (formed once, at create), the
// partial image acc (complex f32 per pixel), and scratch for ONE chunk of up
// to max_chunk pulses (its range profiles as (m, d) pairs and its
// per-(tile, pulse) records).  Each add() range-compresses its phase-history
// rows and adds their contribution to acc; finalize() applies the final
// phase and the row flip.  The footprint is thus bounded by max_chunk instead
// of P: at 4096^2 x 4000 with N_fft 8192 the one-shot scratch is 2.7 GB
// (0.5 GB of pairs, 2.1 GB of records), and a 500-pulse chunk needs 0.33 GB.
//
// The reference's pulse pairing is kept: the pulse axis is fftshifted twice
// (backprojection.cpp:98,104), so phase-history row q carries Taylor weight
// w_P[q] and meets antenna position (q - P mod 2) mod P.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "context.h"
#include "internal.h"
#include "kernels.h"
#include "runner.h"
#include "sarbp_b200.h"

using namespace sarbp;

namespace {

size_t a256(size_t x) { return (x + 255) / 256 * 256; }

struct AccumLayout {
    size_t sc, job, items, rows, cnt, filt, wS, wP, pulse, tiles, fin, acc, Qp, recs, pulse_c, wP_c, work, end;
    int work_rows;  // rows of the four-step range compression's work buffer (0: none)
};

int log2_of(int n) {
    int l = 0;
    while ((1 << l) < n) ++l;
    return l;
}

AccumLayout accum_layout(const sarbp_job &j, int tile_x, int tile_y, int C) {
    const size_t P = (size_t)j.npulses, S = (size_t)j.nsamples, N = (size_t)j.n_fft;
    const size_t ntiles = (size_t)((j.nu + tile_x - 1) / tile_x) * (size_t)((j.nv + tile_y - 1) / tile_y);
    const size_t npix = (size_t)j.nu * j.nv;
    AccumLayout L;
    size_t o = 0;
    L.sc = o;      o = a256(o + sizeof(JobScalars));
    L.job = o;     o = a256(o + sizeof(DevJob));
    L.items = o;   o = a256(o + ntiles * sizeof(WorkItem));
    L.rows = o;    o = a256(o + (size_t)C * sizeof(RowItem));
    L.cnt = o;     o = a256(o + sizeof(int));
    L.filt = o;    o = a256(o + S * sizeof(float));
    L.wS = o;      o = a256(o + S * sizeof(float));
    L.wP = o;      o = a256(o + P * sizeof(float));
    L.pulse = o;   o = a256(o + P * sizeof(double4));
    L.tiles = o;   o = a256(o + ntiles * sizeof(TileInfo));
    L.fin = o;     o = a256(o + npix * sizeof(float2));
    L.acc = o;     o = a256(o + npix * sizeof(float2));
    L.Qp = o;      o = a256(o + (size_t)C * (N + 1) * sizeof(float4));
    L.recs = o;    o = a256(o + ntiles * (size_t)C * sizeof(PulseRec));
    L.pulse_c = o; o = a256(o + (size_t)C * sizeof(double4));
    L.wP_c = o;    o = a256(o + (size_t)C * sizeof(float));
    const int logN = log2_of(j.n_fft);
    L.work_rows = logN > kMaxLogNSmem ? std::min(C, rc_work_rows(logN)) : 0;
    L.work = o;    o = a256(o + (size_t)L.work_rows * N * sizeof(float2));
    L.end = o;
    return L;
}

int precision_for(const sarbp_job &j, const sarbp_opts *o) {
    if (j.precision >= 0) return j.precision;
    return o ? o->precision : SARBP_PREC_COMPAT;
}

BpLaunch launch_for(const sarbp_opts *opts, int num_sms) {
    BpLaunch L = default_launch(opts, num_sms);
    if (!bp_tile_supported(L.tile_x, L.tile_y, L.minb) && !(opts && opts->min_blocks)) L.minb = 2;
    return L;
}

}  // namespace

size_t sarbp::job_io_bytes(const sarbp_job &j, bool with_phs) {
    const size_t P = (size_t)j.npulses, S = (size_t)j.nsamples, npix = (size_t)j.nu * j.nv;
    size_t b = with_phs ? a256(P * S * 8) : 0;
    b += j.k_r ? a256(S * 4) : 0;
    b += j.k_r64 ? a256(S * 8) : 0;
    b += j.pos ? a256(P * 12) : 0;
    b += j.pos64 ? a256(P * 24) : 0;
    b += j.r ? a256(npix * 24) : a256((size_t)j.nu * 8) + a256((size_t)j.nv * 8);
    b += a256(npix * 16);
    b += j.out_u8 ? a256(npix) : 0;
    return b;
}

namespace {
size_t io_bytes(const sarbp_job &j, bool with_phs) { return job_io_bytes(j, with_phs); }
}  // namespace

struct sarbp_accum {
    sarbp_ctx *ctx = nullptr;
    sarbp_job job{};
    int prec = 0;
    BpLaunch L{};
    int P = 0, S = 0, N = 0, logN = 0, C = 0, ntiles = 0;
    long long npix = 0;
    AccumLayout lay{};
    DeviceBuffer mem;
    DeviceBuffer stage;  // two staging buffers of C phase-history rows (host path)
    PinnedBuffer status_pin;
    DevJob base{};       // host copy of the whole job's descriptor
    std::vector<unsigned char> added;
    long long nadded = 0;
    long long nhost = 0;  // host-path chunks so far
    cudaEvent_t copied[2] = {nullptr, nullptr}, consumed[2] = {nullptr, nullptr};
    bool finalized = false;

    // streams of the serving loop's streaming apertures (NULL: the context's)
    cudaStream_t own_st = nullptr, own_cin = nullptr;

    char *dptr(size_t off) const { return static_cast<char *>(mem.ptr) + off; }
    DevJob *d_job() const { return reinterpret_cast<DevJob *>(dptr(lay.job)); }
    cudaStream_t st() const { return own_st ? own_st : ctx->stream; }
    cudaStream_t cin() const { return own_cin ? own_cin : ctx->copy_in; }
    int start();
    int check_chunk(int q0, int n) const;
    int add(int q0, int n, const float *phs_rows, cudaEvent_t rc_done);
};

int sarbp_accum::check_chunk(int q0, int n) const {
    if (finalized) return fail(SARBP_ERR_STATE, "pulse-chunked job: finalized (reset it for a new aperture)");
    if (n < 1 || n > C)
        return fail(SARBP_ERR_INVALID, "pulse-chunked job: a chunk holds 1.." + std::to_string(C) +
                                           " pulses, got " + std::to_string(n));
    if (q0 < 0 || (long long)q0 + n > P)
        return fail(SARBP_ERR_INVALID, "pulse-chunked job: pulses [" + std::to_string(q0) + ", " +
                                           std::to_string((long long)q0 + n) + ") outside [0, " +
                                           std::to_string(P) + ")");
    for (int q = q0; q < q0 + n; ++q)
        if (added[q])
            return fail(SARBP_ERR_STATE, "pulse-chunked job: pulse " + std::to_string(q) + " was already added");
    return SARBP_OK;
}

int sarbp_accum::start() {
    cudaStream_t s = st();
    DevJob &b = base;
    describe_job(job, prec, L.tile_x, L.tile_y, b);
    b.phs = nullptr;
    b.Q = nullptr;
    b.sc = reinterpret_cast<JobScalars *>(dptr(lay.sc));
    b.filt = reinterpret_cast<float *>(dptr(lay.filt));
    b.wS = reinterpret_cast<float *>(dptr(lay.wS));
    b.wP = reinterpret_cast<float *>(dptr(lay.wP));
    b.pulse = reinterpret_cast<double4 *>(dptr(lay.pulse));
    b.tiles = reinterpret_cast<TileInfo *>(dptr(lay.tiles));
    b.fin = reinterpret_cast<float2 *>(dptr(lay.fin));
    b.Qp = reinterpret_cast<float4 *>(dptr(lay.Qp));
    b.recs = reinterpret_cast<PulseRec *>(dptr(lay.recs));
    b.acc = nullptr;
    b.chunked = 0;
    cudaError_t e = launch_store_job(b, d_job(), s);
    // windows, filter, pulse table, k_c (clears max|z| and status)
    if (e == cudaSuccess) {
        launch_prep(d_job(), 1, s);
        e = cudaGetLastError();
    }
    auto *items = reinterpret_cast<WorkItem *>(dptr(lay.items));
    auto *rows = reinterpret_cast<RowItem *>(dptr(lay.rows));
    if (e == cudaSuccess) e = launch_fill_items(items, ntiles, rows, C, s);
    // tile table and final phase per pixel (no records: those come per chunk)
    if (e == cudaSuccess) e = launch_tile_setup(d_job(), items, ntiles, L.tile_x * L.tile_y, s, 0);
    if (e == cudaSuccess) e = cudaMemsetAsync(dptr(lay.acc), 0, (size_t)npix * sizeof(float2), s);
    if (e != cudaSuccess) return cuda_fail(e, "pulse-chunked job: set-up launches");
    ctx->dev.launches += 4;
    return SARBP_OK;
}

int sarbp_accum::add(int q0, int n, const float *phs_rows, cudaEvent_t rc_done) {
    if (!phs_rows) return fail(SARBP_ERR_INVALID, "pulse-chunked job: phase-history rows are NULL");
    int rc = check_chunk(q0, n);
    if (rc) return rc;
    cudaStream_t s = st();
    DevJob c = base;
    c.P = n;
    c.phs = reinterpret_cast<const float2 *>(phs_rows);
    c.chunked = 1;
    c.acc = reinterpret_cast<float2 *>(dptr(lay.acc));
    c.pulse = reinterpret_cast<double4 *>(dptr(lay.pulse_c));
    c.wP = reinterpret_cast<float *>(dptr(lay.wP_c));
    auto *items = reinterpret_cast<const WorkItem *>(dptr(lay.items));
    auto *rows = reinterpret_cast<const RowItem *>(dptr(lay.rows));
    int *cnt = reinterpret_cast<int *>(dptr(lay.cnt));
    cudaError_t e = launch_chunk_tables(base.pulse, base.wP, P, q0, n, c.pulse, c.wP, s);
    if (e == cudaSuccess) e = launch_store_job(c, d_job(), s);
    if (e == cudaSuccess)
        e = range_compress_rows(&ctx->dev, logN, d_job(), rows, n, 1, reinterpret_cast<float2 *>(dptr(lay.work)),
                                lay.work_rows, s);
    if (e == cudaSuccess && rc_done) e = cudaEventRecord(rc_done, s);
    if (e == cudaSuccess) e = launch_tile_records(d_job(), items, ntiles, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(cnt, 0, sizeof(int), s);
    if (e != cudaSuccess) return cuda_fail(e, "pulse-chunked job: chunk launches");
    BpLaunch Lc = L;
    const int occ = bp_max_active_blocks(Lc);
    if (occ < 1) return fail(SARBP_ERR_CUDA, "backprojection kernel does not fit on an SM");
    Lc.grid = (int)std::min<long long>((long long)occ * ctx->dev.num_sms, (long long)ntiles);
    e = launch_backproject(Lc, d_job(), items, ntiles, cnt, s);
    if (e != cudaSuccess) return cuda_fail(e, "pulse-chunked job: backprojection launch");
    ctx->dev.launches += 5;
    for (int q = q0; q < q0 + n; ++q) added[q] = 1;
    nadded += n;
    return SARBP_OK;
}

int sarbp::accum_create_on(sarbp_ctx *ctx, const sarbp_job *job, const sarbp_opts *opts, int max_chunk,
                           cudaStream_t stream, cudaStream_t copy_stream, sarbp_accum **out) {
    int rc = ctx_set_device(ctx);
    if (rc) return rc;
    if (!job || !out) return fail(SARBP_ERR_INVALID, "job and out must be non-NULL");
    *out = nullptr;
    const int prec = precision_for(*job, opts);
    if (prec == SARBP_PREC_NAIVE)
        return fail(SARBP_ERR_UNSUPPORTED, "pulse-chunked jobs run the split-precision kernel only");
    rc = validate_job(*job, prec, 0, false, false);
    if (rc) return rc;
    if (max_chunk < 1) return fail(SARBP_ERR_INVALID, "max_chunk must be >= 1");
    std::unique_ptr<sarbp_accum> a(new sarbp_accum());
    a->ctx = ctx;
    a->own_st = stream;
    a->own_cin = copy_stream;
    a->job = *job;
    a->prec = prec;
    a->L = launch_for(opts, ctx->dev.num_sms);
    if (!bp_tile_supported(a->L.tile_x, a->L.tile_y, a->L.minb))
        return fail(SARBP_ERR_INVALID, "unsupported pixel tile");
    a->P = job->npulses;
    a->S = job->nsamples;
    a->N = job->n_fft;
    while ((1 << a->logN) < a->N) ++a->logN;
    a->C = std::min(max_chunk, a->P);
    a->ntiles = ((job->nu + a->L.tile_x - 1) / a->L.tile_x) * ((job->nv + a->L.tile_y - 1) / a->L.tile_y);
    a->npix = (long long)job->nu * job->nv;
    a->lay = accum_layout(*job, a->L.tile_x, a->L.tile_y, a->C);
    a->added.assign(a->P, 0);
    cudaError_t e = a->mem.alloc_exact(a->lay.end);
    if (e != cudaSuccess) return cuda_fail(e, "pulse-chunked job: device memory");
    // the twiddle tables now (one-time synchronous uploads), not at an add
    float2 *tw = nullptr;
    e = ctx->dev.twiddle(a->logN, &tw);
    if (e == cudaSuccess && a->logN > kMaxLogNSmem) e = ctx->dev.twiddle(a->logN / 2, &tw);
    if (e == cudaSuccess && a->logN > kMaxLogNSmem) e = ctx->dev.twiddle(a->logN - a->logN / 2, &tw);
    if (e != cudaSuccess) return cuda_fail(e, "twiddle table");
    e = a->status_pin.ensure(sizeof(JobScalars));
    if (e != cudaSuccess) return cuda_fail(e, "pinned status word");
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
        e = cudaEventCreateWithFlags(&a->copied[b], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&a->consumed[b], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        sarbp_accum_destroy(a.release());
        return cuda_fail(e, "creating events");
    }
    rc = a->start();
    if (rc) {
        sarbp_accum_destroy(a.release());
        return rc;
    }
    *out = a.release();
    return SARBP_OK;
}

extern "C" {

int sarbp_accum_create(sarbp_ctx *ctx, const sarbp_job *job, const sarbp_opts *opts, int max_chunk,
                       sarbp_accum **out) {
    return accum_create_on(ctx, job, opts, max_chunk, nullptr, nullptr, out);
}

int sarbp_accum_add_device(sarbp_accum *acc, int pulse0, int count, const float *phs_rows) {
    if (!acc) return fail(SARBP_ERR_INVALID, "accumulator is NULL");
    int rc = ctx_set_device(acc->ctx);
    if (rc) return rc;
    return acc->add(pulse0, count, phs_rows, nullptr);
}

int sarbp_accum_add(sarbp_accum *acc, int pulse0, int count, const float *phs_rows_host) {
    if (!acc) return fail(SARBP_ERR_INVALID, "accumulator is NULL");
    int rc = ctx_set_device(acc->ctx);
    if (rc) return rc;
    if (!phs_rows_host) return fail(SARBP_ERR_INVALID, "pulse-chunked job: phase-history rows are NULL");
    rc = acc->check_chunk(pulse0, count);
    if (rc) return rc;
    const size_t row_bytes = (size_t)acc->S * 8, half = a256((size_t)acc->C * row_bytes);
    cudaError_t e = acc->stage.cap >= 2 * half ? cudaSuccess : acc->stage.alloc_exact(2 * half);
    if (e != cudaSuccess) return cuda_fail(e, "pulse-chunked job: staging buffers");
    const int b = (int)(acc->nhost & 1);
    char *dst = static_cast<char *>(acc->stage.ptr) + b * half;
    cudaStream_t cin = acc->cin();
    // the chunk that used this staging buffer two adds ago must be range-compressed
    if (acc->nhost >= 2 && (e = cudaStreamWaitEvent(cin, acc->consumed[b], 0)) != cudaSuccess)
        return cuda_fail(e, "cudaStreamWaitEvent");
    e = cudaMemcpyAsync(dst, phs_rows_host, (size_t)count * row_bytes, cudaMemcpyHostToDevice, cin);
    if (e == cudaSuccess) e = cudaEventRecord(acc->copied[b], cin);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(acc->st(), acc->copied[b], 0);
    if (e != cudaSuccess) return cuda_fail(e, "pulse-chunked job: copying phase-history rows");
    rc = acc->add(pulse0, count, reinterpret_cast<const float *>(dst), acc->consumed[b]);
    if (rc) {
        cudaStreamSynchronize(cin);  // the copy may still read the caller's rows
        return rc;
    }
    // the previous chunk's rows have left the caller's memory when this returns
    if (acc->nhost >= 1 && (e = cudaEventSynchronize(acc->copied[b ^ 1])) != cudaSuccess)
        return cuda_fail(e, "cudaEventSynchronize");
    acc->nhost++;
    return SARBP_OK;
}

int sarbp_accum_finalize(sarbp_accum *acc) {
    if (!acc) return fail(SARBP_ERR_INVALID, "accumulator is NULL");
    int rc = ctx_set_device(acc->ctx);
    if (rc) return rc;
    if (acc->finalized) return fail(SARBP_ERR_STATE, "pulse-chunked job: already finalized");
    if (acc->nadded != acc->P)
        return fail(SARBP_ERR_STATE, "pulse-chunked job: " + std::to_string(acc->nadded) + " of " +
                                         std::to_string(acc->P) + " pulses added");
    cudaStream_t s = acc->st();
    DevJob f = acc->base;
    f.acc = reinterpret_cast<float2 *>(acc->dptr(acc->lay.acc));
    JobScalars *sc = reinterpret_cast<JobScalars *>(acc->dptr(acc->lay.sc));
    cudaError_t e = launch_store_job(f, acc->d_job(), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(&sc->maxabs, 0, sizeof(sc->maxabs), s);
    if (e == cudaSuccess) e = launch_finalize(acc->d_job(), acc->npix, acc->ctx->dev.num_sms, s);
    int nl = 2;
    if (e == cudaSuccess && acc->job.out_u8) {
        e = launch_batch_u8(acc->d_job(), 1, acc->npix, s);
        ++nl;
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(acc->status_pin.ptr, sc, sizeof(JobScalars), cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return cuda_fail(e, "pulse-chunked job: finalize launches");
    acc->ctx->dev.launches += nl;
    acc->finalized = true;
    return SARBP_OK;
}

int sarbp_accum_wait(sarbp_accum *acc) {
    if (!acc) return fail(SARBP_ERR_INVALID, "accumulator is NULL");
    int rc = ctx_set_device(acc->ctx);
    if (rc) return rc;
    cudaError_t e = cudaStreamSynchronize(acc->st());
    if (e == cudaSuccess) e = cudaStreamSynchronize(acc->cin());
    if (e != cudaSuccess) return cuda_fail(e, "synchronising the stream");
    if (!acc->finalized) return SARBP_OK;
    const int s = static_cast<const JobScalars *>(acc->status_pin.ptr)->status;
    if (s & kStatusNonFinite)
        return fail(SARBP_ERR_GEOMETRY, "non-finite pixel or antenna position (those pixels or pulses were left out)");
    if (s & kStatusTimeout) return fail(SARBP_ERR_TIMEOUT, "a bounded wait for a range-profile copy gave up");
    if (s & kStatusTileTooWide)
        return fail(SARBP_ERR_GEOMETRY, "a pixel tile spans more range bins than fit on chip; those tiles "
                                        "were left at zero");
    return SARBP_OK;
}

int sarbp_accum_reset(sarbp_accum *acc) {
    if (!acc) return fail(SARBP_ERR_INVALID, "accumulator is NULL");
    int rc = ctx_set_device(acc->ctx);
    if (rc) return rc;
    cudaStream_t s = acc->st();
    JobScalars *sc = reinterpret_cast<JobScalars *>(acc->dptr(acc->lay.sc));
    cudaError_t e = cudaMemsetAsync(acc->dptr(acc->lay.acc), 0, (size_t)acc->npix * sizeof(float2), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(&sc->status, 0, sizeof(sc->status), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(&sc->maxabs, 0, sizeof(sc->maxabs), s);
    if (e != cudaSuccess) return cuda_fail(e, "pulse-chunked job: reset");
    std::fill(acc->added.begin(), acc->added.end(), 0);
    acc->nadded = 0;
    acc->finalized = false;
    return SARBP_OK;
}

double sarbp_accum_device_bytes(const sarbp_accum *acc) {
    return acc ? (double)(acc->mem.cap + acc->stage.cap) : 0.0;
}

int sarbp_accum_destroy(sarbp_accum *acc) {
    if (!acc) return SARBP_OK;
    cudaSetDevice(acc->ctx->dev.device);
    cudaStreamSynchronize(acc->st());
    cudaStreamSynchronize(acc->cin());
    acc->mem.release();
    acc->stage.release();
    acc->status_pin.release();
    for (int b = 0; b < 2; ++b) {
        if (acc->copied[b]) cudaEventDestroy(acc->copied[b]);
        if (acc->consumed[b]) cudaEventDestroy(acc->consumed[b]);
    }
    delete acc;
    return SARBP_OK;
}

int sarbp_job_device_bytes(const sarbp_job *job, const sarbp_opts *opts, int chunk_pulses, double *bytes) {
    if (!job || !bytes) return fail(SARBP_ERR_INVALID, "job and bytes must be non-NULL");
    if (job->npulses < 1 || job->nsamples < 1 || job->nu < 1 || job->nv < 1 || job->n_fft < 1)
        return fail(SARBP_ERR_INVALID, "sizes must be >= 1");
    const BpLaunch L = launch_for(opts, 148);
    if (chunk_pulses <= 0) {
        sarbp_job j = *job;
        j.precision = precision_for(*job, opts);
        *bytes = (double)(io_bytes(*job, true) + Runner::job_scratch_bytes(j, opts));
        return SARBP_OK;
    }
    const int C = std::min(chunk_pulses, job->npulses);
    const size_t stage = 2 * a256((size_t)C * job->nsamples * 8);
    *bytes = (double)(io_bytes(*job, false) + accum_layout(*job, L.tile_x, L.tile_y, C).end + stage);
    return SARBP_OK;
}

int sarbp_backprojection_streamed(sarbp_ctx *ctx, const sarbp_job *host_job, const sarbp_opts *opts,
                                  double max_device_bytes, int *chunk_pulses, double *device_bytes) {
    int rc = ctx_set_device(ctx);
    if (rc) return rc;
    if (!host_job) return fail(SARBP_ERR_INVALID, "job is NULL");
    const sarbp_job &h = *host_job;
    const int prec = precision_for(h, opts);
    rc = validate_job(h, prec, 0, false, true);
    if (rc) return rc;
    // the largest chunk whose footprint fits, then chunks of even size
    const BpLaunch L = launch_for(opts, ctx->dev.num_sms);
    auto footprint = [&](int c) {
        return (double)(io_bytes(h, false) + accum_layout(h, L.tile_x, L.tile_y, c).end +
                        2 * a256((size_t)c * h.nsamples * 8));
    };
    int lo = 0, hi = h.npulses;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (footprint(mid) <= max_device_bytes) lo = mid;
        else hi = mid - 1;
    }
    if (lo < 1)
        return fail(SARBP_ERR_NOMEM, "pulse-chunked job: even one pulse per chunk needs " +
                                         std::to_string((long long)footprint(1)) + " device bytes, over the cap");
    const int nchunks = (h.npulses + lo - 1) / lo;
    const int C = (h.npulses + nchunks - 1) / nchunks;
    // inputs other than the phase history, and the outputs
    const size_t P = (size_t)h.npulses, S = (size_t)h.nsamples, npix = (size_t)h.nu * h.nv;
    DeviceBuffer io;
    cudaError_t e = io.alloc_exact(io_bytes(h, false));
    if (e != cudaSuccess) return cuda_fail(e, "pulse-chunked job: device inputs");
    struct Guard {
        DeviceBuffer *b;
        sarbp_accum *a = nullptr;
        ~Guard() {
            if (a) sarbp_accum_destroy(a);
            b->release();
        }
    } guard{&io};
    char *base = static_cast<char *>(io.ptr);
    size_t o = 0;
    sarbp_job d = h;
    struct Copy { const void *src; size_t n; const void **dst; };
    const void *dk32 = nullptr, *dk64 = nullptr, *dp32 = nullptr, *dp64 = nullptr, *dr = nullptr, *du = nullptr,
               *dv = nullptr;
    const Copy copies[] = {{h.k_r, S * 4, &dk32},           {h.k_r64, S * 8, &dk64},
                           {h.pos, P * 12, &dp32},          {h.pos64, P * 24, &dp64},
                           {h.r, npix * 24, &dr},           {h.r ? nullptr : h.u, (size_t)h.nu * 8, &du},
                           {h.r ? nullptr : h.v, (size_t)h.nv * 8, &dv}};
    for (const Copy &c : copies) {
        if (!c.src) continue;
        *c.dst = base + o;
        e = cudaMemcpyAsync(base + o, c.src, c.n, cudaMemcpyHostToDevice, ctx->stream);
        if (e != cudaSuccess) return cuda_fail(e, "pulse-chunked job: copying inputs");
        o += a256(c.n);
    }
    d.k_r = static_cast<const float *>(dk32);
    d.k_r64 = static_cast<const double *>(dk64);
    d.pos = static_cast<const float *>(dp32);
    d.pos64 = static_cast<const double *>(dp64);
    d.r = static_cast<const double *>(dr);
    d.u = static_cast<const double *>(du);
    d.v = static_cast<const double *>(dv);
    d.phs = nullptr;
    d.output_img = reinterpret_cast<double *>(base + o);
    o += a256(npix * 16);
    d.out_u8 = h.out_u8 ? reinterpret_cast<uint8_t *>(base + o) : nullptr;
    d.precision = prec;
    rc = sarbp_accum_create(ctx, &d, opts, C, &guard.a);
    if (rc) return rc;
    for (int q0 = 0; q0 < h.npulses; q0 += C) {
        const int n = std::min(C, h.npulses - q0);
        rc = sarbp_accum_add(guard.a, q0, n, h.phs + (size_t)q0 * S * 2);
        if (rc) return rc;
    }
    rc = sarbp_accum_finalize(guard.a);
    if (rc) return rc;
    if (h.output_img) e = cudaMemcpyAsync(h.output_img, d.output_img, npix * 16, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess && h.out_u8)
        e = cudaMemcpyAsync(h.out_u8, d.out_u8, npix, cudaMemcpyDeviceToHost, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "pulse-chunked job: copying the image to the host");
    rc = sarbp_accum_wait(guard.a);
    if (chunk_pulses) *chunk_pulses = C;
    if (device_bytes) *device_bytes = (double)io.cap + sarbp_accum_device_bytes(guard.a);
    return rc;
}

}  // extern "C"
