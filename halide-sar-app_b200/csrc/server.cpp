// server.cpp -- the serving loop: continuous batching of image-formation
// requests under an HBM budget (no counterpart in the reference, which forms
// one image per process run).
//
// A request is a sarbp_job whose pointers are HOST memory.  submit() only
// queues it.  A scheduler thread forms batches: whenever one of the lanes
// (a stream with its own Runner) is free it takes queued requests in arrival
// order while their device footprint fits the budget, uploads each one's
// phase history, k_r, positions and image-plane axes once into memory from
// the server's pool, enqueues the batch (one persistent backprojection over
// all the batch's tiles) and the copies of the images back to the host, and
// frees the request memory stream-ordered behind them.  Requests that arrive
// while other batches are on the GPU go into the next free lane, so batches
// of different lanes overlap on the device.  A completion thread picks up
// the lanes' batches in whichever order they finish, stamps the requests
// done and returns their budget.  A batch holds at most max_batch requests
// and max_work pixel*pulses, which bounds how long a small request can wait
// for the large ones it shares a batch with.
//
// Footprint of a request: its device inputs and outputs plus its share of
// its batch's scratch, all taken from the server's memory pool when the
// batch launches and returned stream-ordered behind it; the budget is
// charged from admission to completion.  A request larger than the whole
// budget fails with SARBP_ERR_ADMISSION.
//
// Registered apertures: sarbp_server_register uploads a phase history, k_r
// and antenna positions once and range-compresses them once into resident
// interpolation pairs; requests submitted on the aperture
// (sarbp_server_submit_on) bring only their image plane and outputs, and
// their batches skip the upload and the range compression of that aperture.
// The resident bytes are charged to the budget from registration to
// sarbp_server_unregister.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "context.h"
#include "runner.h"
#include "sarbp_b200.h"

using namespace sarbp;

namespace {

using Clock = std::chrono::steady_clock;

size_t a256(size_t x) { return (x + 255) / 256 * 256; }

// A registered aperture: device copies of k_r and the antenna positions and
// the range profiles as interpolation pairs [P][N_fft + 1] (one block).
struct Aperture {
    long long id = 0;
    sarbp_job shape{};  // sizes, Taylor, delta_r and precision of the aperture
    void *mem = nullptr;
    size_t bytes = 0;
    const float *k32 = nullptr, *p32 = nullptr;
    const double *k64 = nullptr, *p64 = nullptr;
    const float4 *qp = nullptr;
    int refs = 0;  // queued or running requests on it
};

// A streaming aperture: a device-resident partial image (pulse-chunked
// accumulator) with its own compute and copy streams, and the device copies
// of the job's inputs other than the phase history, and of its outputs.
// Calls on one stream hold `mu`; `closed` is set by the finish, so an add
// that raced with it (and still held the pointer) sees a closed stream.
struct StreamAp {
    std::mutex mu;
    bool closed = false;
    sarbp_job host{};      // the caller's job (host outputs)
    sarbp_job dev{};       // device copies
    DeviceBuffer io;
    sarbp_accum *acc = nullptr;
    size_t bytes = 0;      // charged to the budget
    cudaStream_t st = nullptr, cin = nullptr;
    void release() {
        if (acc) sarbp_accum_destroy(acc);
        acc = nullptr;
        if (st) cudaStreamSynchronize(st);
        io.release();
        if (st) cudaStreamDestroy(st);
        if (cin) cudaStreamDestroy(cin);
        st = cin = nullptr;
    }
};

struct Request {
    long long id = 0;
    Aperture *ap = nullptr;  // registered aperture, or NULL (the request brings its phase history)
    sarbp_job host{};  // the caller's job, host pointers
    size_t io_bytes = 0, scratch_bytes = 0;
    double work = 0.0;  // pixel*pulses
    double t_submit = 0.0, t_start = 0.0, t_done = 0.0;
    bool done = false;
    int status = SARBP_OK;
    std::string error;
    void *dmem = nullptr;
};

// Device layout of a request's inputs and outputs (one pool allocation).
struct IoLayout {
    size_t phs, k32, k64, p32, p64, r, u, v, out, u8, end;
};

IoLayout io_layout(const sarbp_job &j) {
    const size_t P = (size_t)j.npulses, S = (size_t)j.nsamples, npix = (size_t)j.nu * j.nv;
    IoLayout L{};
    size_t o = 0;
    L.phs = o; o += j.phs ? a256(P * S * 8) : 0;
    L.k32 = o; o += j.k_r ? a256(S * 4) : 0;
    L.k64 = o; o += j.k_r64 ? a256(S * 8) : 0;
    L.p32 = o; o += j.pos ? a256(P * 12) : 0;
    L.p64 = o; o += j.pos64 ? a256(P * 24) : 0;
    L.r = o; o += j.r ? a256(npix * 24) : 0;
    L.u = o; o += (!j.r && j.u) ? a256((size_t)j.nu * 8) : 0;
    L.v = o; o += (!j.r && j.v) ? a256((size_t)j.nv * 8) : 0;
    L.out = o; o += a256(npix * 16);
    L.u8 = o; o += j.out_u8 ? a256(npix) : 0;
    L.end = o;
    return L;
}

}  // namespace

struct sarbp_server {
    struct Lane {
        cudaStream_t st = nullptr;
        std::unique_ptr<Runner> runner;
        cudaEvent_t done = nullptr;
        std::vector<Request *> batch;
        bool busy = false;
        size_t charged = 0;  // budget charged for the batch in flight
    };

    sarbp_ctx *ctx = nullptr;
    sarbp_opts launch{};
    size_t cap = 0;
    int max_batch = 32;
    double max_work = 6e9;  // pixel*pulses per batch (bounds a batch's latency)
    cudaMemPool_t pool = nullptr;
    Clock::time_point t0 = Clock::now();

    std::mutex mu;
    std::condition_variable cv;
    std::deque<Request *> queue;
    std::map<long long, std::unique_ptr<Request>> reqs;
    long long next_id = 1;
    size_t in_use = 0, peak = 0;
    long long submitted = 0, completed = 0, batches = 0;
    std::vector<Lane> lanes;
    std::deque<Lane *> inflight;
    bool stop = false, sched_exited = false;
    std::thread sched, comp;
    // registered apertures (guarded by mu) and their set-up stream
    std::map<long long, std::unique_ptr<Aperture>> apertures;
    // streaming apertures: partial images accumulating pulse chunks
    std::map<long long, std::shared_ptr<StreamAp>> streams;
    long long next_stream = 1;
    long long next_ap = 1;
    cudaStream_t reg_st = nullptr;
    // counters: bytes copied host -> device, pulses range-compressed,
    // requests served from a registered aperture
    std::atomic<long long> h2d_bytes{0}, rc_pulses{0}, resident_requests{0};

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }

    void scheduler();
    void completer();
    void launch_batch(Lane &L);
};

void sarbp_server::launch_batch(Lane &L) {
    cudaSetDevice(ctx->dev.device);
    std::vector<sarbp_job> jobs;
    std::vector<const float4 *> resident;
    jobs.reserve(L.batch.size());
    int rc = SARBP_OK;
    std::string err;
    long long up = 0, rcp = 0, res = 0;
    for (Request *q : L.batch) {
        const sarbp_job &h = q->host;
        const IoLayout lay = io_layout(h);
        cudaError_t e = cudaMallocFromPoolAsync(&q->dmem, lay.end, pool, L.st);
        if (e != cudaSuccess) {
            rc = cuda_fail(e, "serving: device memory for a request");
            err = last_error_cstr();
            q->dmem = nullptr;
            break;
        }
        char *b = static_cast<char *>(q->dmem);
        const size_t P = (size_t)h.npulses, S = (size_t)h.nsamples, npix = (size_t)h.nu * h.nv;
        struct Copy { size_t off; const void *src; size_t n; };
        const Copy in[] = {{lay.phs, h.phs, P * S * 8},     {lay.k32, h.k_r, S * 4},
                           {lay.k64, h.k_r64, S * 8},       {lay.p32, h.pos, P * 12},
                           {lay.p64, h.pos64, P * 24},      {lay.r, h.r, npix * 24},
                           {lay.u, h.r ? nullptr : h.u, (size_t)h.nu * 8},
                           {lay.v, h.r ? nullptr : h.v, (size_t)h.nv * 8}};
        for (const Copy &c : in)
            if (c.src && e == cudaSuccess) {
                e = cudaMemcpyAsync(b + c.off, c.src, c.n, cudaMemcpyHostToDevice, L.st);
                up += (long long)c.n;
            }
        if (e != cudaSuccess) {
            rc = cuda_fail(e, "serving: uploading a request");
            err = last_error_cstr();
            break;
        }
        sarbp_job d = h;
        if (q->ap) {  // resident phase history: no upload, no range compression
            d.phs = nullptr;
            d.k_r = q->ap->k32;
            d.k_r64 = q->ap->k64;
            d.pos = q->ap->p32;
            d.pos64 = q->ap->p64;
            ++res;
        } else {
            d.phs = reinterpret_cast<const float *>(b + lay.phs);
            d.k_r = h.k_r ? reinterpret_cast<const float *>(b + lay.k32) : nullptr;
            d.k_r64 = h.k_r64 ? reinterpret_cast<const double *>(b + lay.k64) : nullptr;
            d.pos = h.pos ? reinterpret_cast<const float *>(b + lay.p32) : nullptr;
            d.pos64 = h.pos64 ? reinterpret_cast<const double *>(b + lay.p64) : nullptr;
            rcp += h.npulses;
        }
        resident.push_back(q->ap ? q->ap->qp : nullptr);
        d.r = h.r ? reinterpret_cast<const double *>(b + lay.r) : nullptr;
        d.u = (!h.r && h.u) ? reinterpret_cast<const double *>(b + lay.u) : nullptr;
        d.v = (!h.r && h.v) ? reinterpret_cast<const double *>(b + lay.v) : nullptr;
        d.output_img = reinterpret_cast<double *>(b + lay.out);
        d.out_u8 = h.out_u8 ? reinterpret_cast<uint8_t *>(b + lay.u8) : nullptr;
        jobs.push_back(d);
    }
    if (rc == SARBP_OK) {
        rc = L.runner->enqueue(jobs.data(), (int)jobs.size(), &launch, L.st, nullptr, false, nullptr,
                               resident.data());
        if (rc) err = last_error_cstr();
    }
    h2d_bytes += up;
    rc_pulses += rcp;
    resident_requests += res;
    if (rc == SARBP_OK) {
        for (size_t i = 0; i < jobs.size() && rc == SARBP_OK; ++i) {
            const sarbp_job &h = L.batch[i]->host;
            const size_t npix = (size_t)h.nu * h.nv;
            cudaError_t e = cudaSuccess;
            if (h.output_img)
                e = cudaMemcpyAsync(h.output_img, jobs[i].output_img, npix * 16, cudaMemcpyDeviceToHost, L.st);
            if (e == cudaSuccess && h.out_u8)
                e = cudaMemcpyAsync(h.out_u8, jobs[i].out_u8, npix, cudaMemcpyDeviceToHost, L.st);
            if (e != cudaSuccess) {
                rc = cuda_fail(e, "serving: copying an image to the host");
                err = last_error_cstr();
            }
        }
    }
    for (Request *q : L.batch) {
        if (q->dmem) cudaFreeAsync(q->dmem, L.st);
        q->dmem = nullptr;
        if (rc) {
            q->status = rc;
            q->error = err;
        }
    }
    cudaEventRecord(L.done, L.st);
}

void sarbp_server::scheduler() {
    cudaSetDevice(ctx->dev.device);
    std::unique_lock<std::mutex> lk(mu);
    auto free_lane = [&]() -> Lane * {
        for (Lane &L : lanes)
            if (!L.busy) return &L;
        return nullptr;
    };
    for (;;) {
        cv.wait(lk, [&] { return (stop && queue.empty()) || (!queue.empty() && free_lane()); });
        if (queue.empty()) {
            sched_exited = true;
            cv.notify_all();
            return;
        }
        Lane &L = *free_lane();
        // admission: arrival order, while the batch fits the budget
        std::vector<Request *> batch;
        size_t bytes = 0;
        double work = 0.0;
        while (!queue.empty() && (int)batch.size() < max_batch) {
            Request *q = queue.front();
            const size_t need = q->io_bytes + q->scratch_bytes;
            if (!batch.empty() && work + q->work > max_work) break;
            if (in_use + bytes + need > cap) {
                if (need > cap) {  // cannot fit even an idle server
                    queue.pop_front();
                    q->status = SARBP_ERR_ADMISSION;
                    q->error = "request needs " + std::to_string(need >> 20) +
                               " MiB of device memory, more than the server budget of " +
                               std::to_string(cap >> 20) + " MiB";
                    q->done = true;
                    q->t_done = now();
                    if (q->ap) --q->ap->refs;
                    ++completed;
                    cv.notify_all();
                    continue;
                }
                break;  // wait for memory to free up
            }
            queue.pop_front();
            batch.push_back(q);
            bytes += need;
            work += q->work;
        }
        if (batch.empty()) {
            // the head request waits for memory: sleep until a batch completes
            if (!inflight.empty()) {
                const long long before = completed;
                cv.wait(lk, [&] { return stop || completed != before; });
            }
            continue;
        }
        in_use += bytes;
        L.charged = bytes;
        peak = std::max(peak, in_use);
        const double t = now();
        for (Request *q : batch) q->t_start = t;
        L.batch = std::move(batch);
        L.busy = true;
        ++batches;
        lk.unlock();
        launch_batch(L);
        lk.lock();
        inflight.push_back(&L);
        cv.notify_all();
    }
}

void sarbp_server::completer() {
    cudaSetDevice(ctx->dev.device);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        cv.wait(lk, [&] { return !inflight.empty() || sched_exited; });
        if (inflight.empty()) return;
        // the first lane whose batch is done (batches of different lanes
        // finish out of launch order: a small one need not wait for a large one)
        Lane *L = nullptr;
        for (Lane *c : inflight)
            if (cudaEventQuery(c->done) != cudaErrorNotReady) {
                L = c;
                break;
            }
        if (!L) {
            cv.wait_for(lk, std::chrono::microseconds(50));
            continue;
        }
        lk.unlock();
        cudaError_t e = cudaEventSynchronize(L->done);
        int rc = e == cudaSuccess ? L->runner->check_status(L->st) : cuda_fail(e, "serving: waiting for a batch");
        std::string err = rc ? last_error_cstr() : std::string();
        const double t = now();
        lk.lock();
        for (Request *q : L->batch) {
            if (q->status == SARBP_OK && rc) {
                q->status = rc;
                q->error = err;
            }
            if (q->ap) --q->ap->refs;
            q->t_done = t;
            q->done = true;
            ++completed;
        }
        in_use -= L->charged;
        L->charged = 0;
        L->batch.clear();
        L->busy = false;
        inflight.erase(std::find(inflight.begin(), inflight.end(), L));
        cv.notify_all();
    }
}

extern "C" {

int sarbp_server_create(sarbp_ctx *ctx, const sarbp_opts *launch, double hbm_cap_bytes, int lanes,
                        int max_batch, double max_batch_work, sarbp_server **out) {
    int rc = ctx_set_device(ctx);
    if (rc) return rc;
    if (!out) return fail(SARBP_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!(hbm_cap_bytes > 0)) return fail(SARBP_ERR_INVALID, "the HBM budget must be positive");
    auto s = std::make_unique<sarbp_server>();
    s->ctx = ctx;
    if (launch) s->launch = *launch;
    s->cap = (size_t)hbm_cap_bytes;
    s->max_batch = max_batch > 0 ? max_batch : 32;
    if (max_batch_work > 0) s->max_work = max_batch_work;
    const int nl = lanes > 0 ? std::min(lanes, 8) : 3;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = ctx->dev.device;
    cudaError_t e = cudaMemPoolCreate(&s->pool, &props);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemPoolCreate");
    unsigned long long keep = (unsigned long long)s->cap;
    cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    s->lanes.resize(nl);
    for (auto &L : s->lanes) {
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&L.st, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming);
        L.runner = std::make_unique<Runner>(&ctx->dev);
        L.runner->stage_events = false;
        L.runner->use_pool(s->pool);
    }
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->reg_st, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
        // back the pool with memory up front so that first batches do not
        // pay for physical allocation (kept: the release threshold is the cap)
        const size_t warm = std::min<size_t>(s->cap, (size_t)8 << 30);
        void *p = nullptr;
        e = cudaMallocFromPoolAsync(&p, warm, s->pool, s->lanes[0].st);
        if (e == cudaSuccess) e = cudaFreeAsync(p, s->lanes[0].st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->lanes[0].st);
    }
    if (e != cudaSuccess) {
        for (auto &L : s->lanes) {
            if (L.st) cudaStreamDestroy(L.st);
            if (L.done) cudaEventDestroy(L.done);
        }
        if (s->reg_st) cudaStreamDestroy(s->reg_st);
        cudaMemPoolDestroy(s->pool);
        return cuda_fail(e, "creating serving lanes");
    }
    sarbp_server *p = s.release();
    p->sched = std::thread([p] { p->scheduler(); });
    p->comp = std::thread([p] { p->completer(); });
    *out = p;
    return SARBP_OK;
}

int sarbp_server_submit(sarbp_server *s, const sarbp_job *host_job, long long *id) {
    if (!s || !host_job || !id) return fail(SARBP_ERR_INVALID, "bad submit arguments");
    const sarbp_job &j = *host_job;
    if (j.nsamples < 1 || j.npulses < 1 || j.nu < 1 || j.nv < 1 || !j.phs ||
        !(j.k_r || j.k_r64) || !(j.pos || j.pos64) || !(j.r || (j.u && j.v)))
        return fail(SARBP_ERR_INVALID, "request: sizes, phs, k_r, pos and pixel positions are required");
    auto q = std::make_unique<Request>();
    q->host = j;
    q->io_bytes = io_layout(j).end;
    q->scratch_bytes = Runner::job_scratch_bytes(j, &s->launch) + (64u << 10);
    q->work = (double)j.nu * j.nv * j.npulses;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return fail(SARBP_ERR_STATE, "server is shutting down");
    q->id = s->next_id++;
    q->t_submit = s->now();
    *id = q->id;
    s->queue.push_back(q.get());
    s->reqs[q->id] = std::move(q);
    ++s->submitted;
    s->cv.notify_all();
    return SARBP_OK;
}

int sarbp_server_wait(sarbp_server *s, long long id, double timeout_s) {
    if (!s) return fail(SARBP_ERR_INVALID, "server is NULL");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail(SARBP_ERR_INVALID, "unknown request id");
    Request *q = it->second.get();
    const auto until = Clock::now() + std::chrono::duration<double>(timeout_s < 0 ? 1e9 : timeout_s);
    if (!s->cv.wait_until(lk, until, [&] { return q->done; }))
        return fail(SARBP_ERR_TIMEOUT, "request " + std::to_string(id) + " not finished yet");
    if (q->status) set_error(q->error);
    return q->status;
}

int sarbp_server_times(sarbp_server *s, long long id, double *submit_s, double *start_s, double *done_s) {
    if (!s) return fail(SARBP_ERR_INVALID, "server is NULL");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail(SARBP_ERR_INVALID, "unknown request id");
    const Request &q = *it->second;
    if (submit_s) *submit_s = q.t_submit;
    if (start_s) *start_s = q.t_start;
    if (done_s) *done_s = q.done ? q.t_done : -1.0;
    return SARBP_OK;
}

int sarbp_server_release(sarbp_server *s, long long id) {
    if (!s) return fail(SARBP_ERR_INVALID, "server is NULL");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail(SARBP_ERR_INVALID, "unknown request id");
    if (!it->second->done) return fail(SARBP_ERR_STATE, "request still in flight");
    s->reqs.erase(it);
    return SARBP_OK;
}

int sarbp_server_stats(sarbp_server *s, long long *submitted, long long *completed, long long *batches,
                       double *in_use_bytes, double *peak_bytes) {
    if (!s) return fail(SARBP_ERR_INVALID, "server is NULL");
    std::lock_guard<std::mutex> lk(s->mu);
    if (submitted) *submitted = s->submitted;
    if (completed) *completed = s->completed;
    if (batches) *batches = s->batches;
    if (in_use_bytes) *in_use_bytes = (double)s->in_use;
    if (peak_bytes) *peak_bytes = (double)s->peak;
    return SARBP_OK;
}

int sarbp_server_destroy(sarbp_server *s) {
    if (!s) return SARBP_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv.notify_all();
    }
    if (s->sched.joinable()) s->sched.join();  // drains the queue
    if (s->comp.joinable()) s->comp.join();    // waits for the lanes
    cudaSetDevice(s->ctx->dev.device);
    for (auto &L : s->lanes) {
        if (L.st) cudaStreamSynchronize(L.st);
        L.runner.reset();
        if (L.st) cudaStreamDestroy(L.st);
        if (L.done) cudaEventDestroy(L.done);
    }
    for (auto &kv : s->streams) kv.second->release();
    s->streams.clear();
    for (auto &kv : s->apertures) cudaFreeAsync(kv.second->mem, s->reg_st);
    s->apertures.clear();
    if (s->reg_st) {
        cudaStreamSynchronize(s->reg_st);
        cudaStreamDestroy(s->reg_st);
    }
    if (s->pool) cudaMemPoolDestroy(s->pool);
    delete s;
    return SARBP_OK;
}

int sarbp_server_register(sarbp_server *s, const sarbp_job *host_aperture, long long *aperture) {
    if (!s || !host_aperture || !aperture) return fail(SARBP_ERR_INVALID, "bad register arguments");
    int rc = ctx_set_device(s->ctx);
    if (rc) return rc;
    sarbp_job h = *host_aperture;
    if (h.precision < 0) h.precision = s->launch.precision;
    if (h.precision != SARBP_PREC_COMPAT && h.precision != SARBP_PREC_PRECISE)
        return fail(SARBP_ERR_UNSUPPORTED, "registered apertures run SARBP_PREC_COMPAT or SARBP_PREC_PRECISE");
    // the image plane is the requests' business: check the rest with a stand-in one
    sarbp_job chk = h;
    chk.nu = chk.nv = 1;
    chk.r = nullptr;
    chk.u = chk.v = reinterpret_cast<const double *>(&h);
    chk.output_img = reinterpret_cast<double *>(&chk);
    chk.out_u8 = nullptr;
    rc = validate_job(chk, h.precision, 0, false, true);
    if (rc) return rc;
    const size_t P = (size_t)h.npulses, S = (size_t)h.nsamples, N = (size_t)h.n_fft;
    // resident block [k32][k64][p32][p64][pairs]; set-up block
    // [phs][scalars][descriptor][filt][wS][wP][pulse][rows][four-step work]
    const size_t b_k32 = h.k_r ? a256(S * 4) : 0, b_k64 = h.k_r64 ? a256(S * 8) : 0;
    const size_t b_p32 = h.pos ? a256(P * 12) : 0, b_p64 = h.pos64 ? a256(P * 24) : 0;
    const size_t b_qp = a256(P * (N + 1) * sizeof(float4));
    const size_t res_bytes = b_k32 + b_k64 + b_p32 + b_p64 + b_qp;
    const size_t o_sc = a256(P * S * 8), o_job = o_sc + a256(sizeof(JobScalars));
    const size_t o_filt = o_job + a256(sizeof(DevJob)), o_ws = o_filt + a256(S * 4), o_wp = o_ws + a256(S * 4);
    const size_t o_pulse = o_wp + a256(P * 4), o_rows = o_pulse + a256(P * sizeof(double4));
    int logN = 0;
    while (((size_t)1 << logN) < N) ++logN;
    const size_t o_work = o_rows + a256(P * sizeof(RowItem));
    const size_t tmp_bytes = o_work + a256(rc_work_bytes(logN));
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->in_use + res_bytes + tmp_bytes > s->cap)
            return fail(SARBP_ERR_ADMISSION, "registering needs " + std::to_string((res_bytes + tmp_bytes) >> 20) +
                                                 " MiB of device memory; the budget has " +
                                                 std::to_string((s->cap - std::min(s->cap, s->in_use)) >> 20) +
                                                 " MiB free");
        s->in_use += res_bytes + tmp_bytes;
        s->peak = std::max(s->peak, s->in_use);
    }
    auto uncharge = [&](size_t bytes) {
        std::lock_guard<std::mutex> lk(s->mu);
        s->in_use -= bytes;
        s->cv.notify_all();
    };
    cudaStream_t st = s->reg_st;
    auto ap = std::make_unique<Aperture>();
    void *tmp = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&ap->mem, res_bytes, s->pool, st);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(&tmp, tmp_bytes, s->pool, st);
    if (e != cudaSuccess) {
        if (ap->mem) cudaFreeAsync(ap->mem, st);
        cudaStreamSynchronize(st);
        uncharge(res_bytes + tmp_bytes);
        return cuda_fail(e, "registering an aperture: device memory");
    }
    char *rb = static_cast<char *>(ap->mem), *tb = static_cast<char *>(tmp);
    size_t o = 0;
    struct Copy { const void *src; size_t n, b; char *dst; };
    const Copy in[] = {{h.k_r, S * 4, b_k32, nullptr}, {h.k_r64, S * 8, b_k64, nullptr},
                       {h.pos, P * 12, b_p32, nullptr}, {h.pos64, P * 24, b_p64, nullptr}};
    char *dst[4] = {};
    for (int i = 0; i < 4 && e == cudaSuccess; ++i) {
        if (!in[i].src) continue;
        dst[i] = rb + o;
        e = cudaMemcpyAsync(dst[i], in[i].src, in[i].n, cudaMemcpyHostToDevice, st);
        o += in[i].b;
    }
    ap->k32 = reinterpret_cast<const float *>(dst[0]);
    ap->k64 = reinterpret_cast<const double *>(dst[1]);
    ap->p32 = reinterpret_cast<const float *>(dst[2]);
    ap->p64 = reinterpret_cast<const double *>(dst[3]);
    ap->qp = reinterpret_cast<const float4 *>(rb + o);
    if (e == cudaSuccess) e = cudaMemcpyAsync(tb, h.phs, P * S * 8, cudaMemcpyHostToDevice, st);
    // range compression into the resident pairs (prep kernel: windows, filter)
    sarbp_job d = h;
    d.phs = reinterpret_cast<const float *>(tb);
    d.k_r = ap->k32;
    d.k_r64 = ap->k64;
    d.pos = ap->p32;
    d.pos64 = ap->p64;
    DevJob dj{};
    describe_job(d, h.precision, 32, 32, dj);
    dj.Qp = const_cast<float4 *>(ap->qp);
    dj.sc = reinterpret_cast<JobScalars *>(tb + o_sc);
    dj.filt = reinterpret_cast<float *>(tb + o_filt);
    dj.wS = reinterpret_cast<float *>(tb + o_ws);
    dj.wP = reinterpret_cast<float *>(tb + o_wp);
    dj.pulse = reinterpret_cast<double4 *>(tb + o_pulse);
    DevJob *d_job = reinterpret_cast<DevJob *>(tb + o_job);
    auto *rows = reinterpret_cast<RowItem *>(tb + o_rows);
    if (e == cudaSuccess) e = launch_store_job(dj, d_job, st);
    if (e == cudaSuccess) {
        launch_prep(d_job, 1, st);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = launch_fill_items(nullptr, 0, rows, (int)P, st);
    if (e == cudaSuccess)
        e = range_compress_rows(&s->ctx->dev, dj.logN, d_job, rows, (int)P, 1, reinterpret_cast<float2 *>(tb + o_work),
                                rc_work_rows(dj.logN), st);
    if (e == cudaSuccess) e = cudaFreeAsync(tmp, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cudaStreamSynchronize(st);
        cudaFreeAsync(ap->mem, st);
        cudaStreamSynchronize(st);
        uncharge(res_bytes + tmp_bytes);
        return cuda_fail(e, "registering an aperture: upload and range compression");
    }
    s->ctx->dev.launches += 4;
    s->h2d_bytes += (long long)(P * S * 8 + (h.k_r ? S * 4 : 0) + (h.k_r64 ? S * 8 : 0) + (h.pos ? P * 12 : 0) +
                                (h.pos64 ? P * 24 : 0));
    s->rc_pulses += (long long)P;
    ap->shape = h;
    ap->shape.phs = nullptr;
    ap->bytes = res_bytes;
    std::lock_guard<std::mutex> lk(s->mu);
    s->in_use -= tmp_bytes;
    ap->id = s->next_ap++;
    *aperture = ap->id;
    s->apertures[ap->id] = std::move(ap);
    s->cv.notify_all();
    return SARBP_OK;
}

int sarbp_server_submit_on(sarbp_server *s, long long aperture, const sarbp_job *host_job, long long *id) {
    if (!s || !host_job || !id) return fail(SARBP_ERR_INVALID, "bad submit arguments");
    const sarbp_job &j = *host_job;
    if (j.nu < 1 || j.nv < 1 || !(j.r || (j.u && j.v)))
        return fail(SARBP_ERR_INVALID, "request: nu, nv and pixel positions are required");
    auto q = std::make_unique<Request>();
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return fail(SARBP_ERR_STATE, "server is shutting down");
    auto it = s->apertures.find(aperture);
    if (it == s->apertures.end()) return fail(SARBP_ERR_INVALID, "unknown aperture id");
    Aperture *ap = it->second.get();
    sarbp_job h = ap->shape;  // sizes, Taylor, delta_r, precision
    h.phs = nullptr;
    h.k_r = nullptr;
    h.k_r64 = nullptr;
    h.pos = nullptr;
    h.pos64 = nullptr;
    h.nu = j.nu;
    h.nv = j.nv;
    h.r = j.r;
    h.u = j.u;
    h.v = j.v;
    for (int k = 0; k < 3; ++k) {
        h.u_hat[k] = j.u_hat[k];
        h.v_hat[k] = j.v_hat[k];
    }
    h.output_img = j.output_img;
    h.out_u8 = j.out_u8;
    h.dB_min = j.dB_min;
    h.dB_max = j.dB_max;
    q->host = h;
    q->ap = ap;
    q->io_bytes = io_layout(h).end;
    q->scratch_bytes = Runner::job_scratch_bytes(h, &s->launch, true) + (64u << 10);
    q->work = (double)h.nu * h.nv * h.npulses;
    ++ap->refs;
    q->id = s->next_id++;
    q->t_submit = s->now();
    *id = q->id;
    s->queue.push_back(q.get());
    s->reqs[q->id] = std::move(q);
    ++s->submitted;
    s->cv.notify_all();
    return SARBP_OK;
}

int sarbp_server_unregister(sarbp_server *s, long long aperture) {
    if (!s) return fail(SARBP_ERR_INVALID, "server is NULL");
    std::unique_ptr<Aperture> ap;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->apertures.find(aperture);
        if (it == s->apertures.end()) return fail(SARBP_ERR_INVALID, "unknown aperture id");
        if (it->second->refs > 0)
            return fail(SARBP_ERR_STATE, "aperture still has queued or running requests");
        ap = std::move(it->second);
        s->apertures.erase(it);
    }
    cudaSetDevice(s->ctx->dev.device);
    cudaError_t e = cudaFreeAsync(ap->mem, s->reg_st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->reg_st);
    std::lock_guard<std::mutex> lk(s->mu);
    s->in_use -= ap->bytes;
    s->cv.notify_all();
    if (e != cudaSuccess) return cuda_fail(e, "unregistering an aperture");
    return SARBP_OK;
}

int sarbp_server_open_stream(sarbp_server *s, const sarbp_job *host_job, int max_chunk, long long *stream_id) {
    if (!s || !host_job || !stream_id) return fail(SARBP_ERR_INVALID, "bad open_stream arguments");
    int rc = ctx_set_device(s->ctx);
    if (rc) return rc;
    sarbp_job h = *host_job;
    if (h.precision < 0) h.precision = s->launch.precision;
    if (h.precision != SARBP_PREC_COMPAT && h.precision != SARBP_PREC_PRECISE)
        return fail(SARBP_ERR_UNSUPPORTED, "streaming apertures run SARBP_PREC_COMPAT or SARBP_PREC_PRECISE");
    rc = validate_job(h, h.precision, 0, false, false);
    if (rc) return rc;
    if (max_chunk < 1) return fail(SARBP_ERR_INVALID, "max_chunk must be >= 1");
    double need = 0;
    rc = sarbp_job_device_bytes(&h, &s->launch, max_chunk, &need);
    if (rc) return rc;
    auto sa = std::make_shared<StreamAp>();
    sa->bytes = (size_t)need;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->in_use + sa->bytes > s->cap)
            return fail(SARBP_ERR_ADMISSION, "streaming aperture needs " + std::to_string(sa->bytes >> 20) +
                                                 " MiB of device memory; the budget has " +
                                                 std::to_string((s->cap - std::min(s->cap, s->in_use)) >> 20) +
                                                 " MiB free");
        s->in_use += sa->bytes;
        s->peak = std::max(s->peak, s->in_use);
    }
    auto undo = [&](int code) {
        sa->release();
        std::lock_guard<std::mutex> lk(s->mu);
        s->in_use -= sa->bytes;
        s->cv.notify_all();
        return code;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&sa->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sa->cin, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = sa->io.alloc_exact(job_io_bytes(h, false));
    if (e != cudaSuccess) return undo(cuda_fail(e, "streaming aperture: streams and device memory"));
    // inputs other than the phase history, and the outputs, on the device
    const size_t P = (size_t)h.npulses, S = (size_t)h.nsamples, npix = (size_t)h.nu * h.nv;
    char *b = static_cast<char *>(sa->io.ptr);
    size_t o = 0;
    sarbp_job d = h;
    auto put = [&](const void *src, size_t n) -> const void * {
        if (!src) return nullptr;
        void *p = b + o;
        o += (n + 255) / 256 * 256;
        if (e == cudaSuccess) e = cudaMemcpyAsync(p, src, n, cudaMemcpyHostToDevice, sa->st);
        return p;
    };
    d.k_r = static_cast<const float *>(put(h.k_r, S * 4));
    d.k_r64 = static_cast<const double *>(put(h.k_r64, S * 8));
    d.pos = static_cast<const float *>(put(h.pos, P * 12));
    d.pos64 = static_cast<const double *>(put(h.pos64, P * 24));
    d.r = static_cast<const double *>(put(h.r, npix * 24));
    d.u = h.r ? nullptr : static_cast<const double *>(put(h.u, (size_t)h.nu * 8));
    d.v = h.r ? nullptr : static_cast<const double *>(put(h.v, (size_t)h.nv * 8));
    d.phs = nullptr;
    d.output_img = reinterpret_cast<double *>(b + o);
    o += (npix * 16 + 255) / 256 * 256;
    d.out_u8 = h.out_u8 ? reinterpret_cast<uint8_t *>(b + o) : nullptr;
    if (e != cudaSuccess) return undo(cuda_fail(e, "streaming aperture: copying inputs"));
    s->h2d_bytes += (long long)o;
    rc = accum_create_on(s->ctx, &d, &s->launch, max_chunk, sa->st, sa->cin, &sa->acc);
    if (rc) {
        const std::string msg = last_error_cstr();
        undo(rc);
        return fail(rc, msg);
    }
    sa->host = h;
    sa->dev = d;
    std::lock_guard<std::mutex> lk(s->mu);
    *stream_id = s->next_stream++;
    s->streams[*stream_id] = std::move(sa);
    return SARBP_OK;
}

int sarbp_server_stream_add(sarbp_server *s, long long stream_id, int pulse0, int count,
                            const float *phs_rows_host) {
    if (!s) return fail(SARBP_ERR_INVALID, "server is NULL");
    std::shared_ptr<StreamAp> sa;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->streams.find(stream_id);
        if (it == s->streams.end()) return fail(SARBP_ERR_INVALID, "unknown stream id");
        sa = it->second;
    }
    std::lock_guard<std::mutex> slk(sa->mu);
    if (sa->closed) return fail(SARBP_ERR_INVALID, "unknown stream id (finished)");
    const int rc = sarbp_accum_add(sa->acc, pulse0, count, phs_rows_host);
    if (rc == SARBP_OK) {
        s->h2d_bytes += (long long)count * sa->host.nsamples * 8;
        s->rc_pulses += count;
    }
    return rc;
}

int sarbp_server_stream_finish(sarbp_server *s, long long stream_id) {
    if (!s) return fail(SARBP_ERR_INVALID, "server is NULL");
    std::shared_ptr<StreamAp> sa;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->streams.find(stream_id);
        if (it == s->streams.end()) return fail(SARBP_ERR_INVALID, "unknown stream id");
        sa = std::move(it->second);
        s->streams.erase(it);
    }
    std::lock_guard<std::mutex> slk(sa->mu);  // after any add in flight
    sa->closed = true;
    int rc = ctx_set_device(s->ctx);
    if (rc == SARBP_OK) rc = sarbp_accum_finalize(sa->acc);
    if (rc == SARBP_OK) {
        const size_t npix = (size_t)sa->host.nu * sa->host.nv;
        cudaError_t e = cudaSuccess;
        if (sa->host.output_img)
            e = cudaMemcpyAsync(sa->host.output_img, sa->dev.output_img, npix * 16, cudaMemcpyDeviceToHost, sa->st);
        if (e == cudaSuccess && sa->host.out_u8)
            e = cudaMemcpyAsync(sa->host.out_u8, sa->dev.out_u8, npix, cudaMemcpyDeviceToHost, sa->st);
        rc = e == cudaSuccess ? sarbp_accum_wait(sa->acc) : cuda_fail(e, "streaming aperture: copying the image");
    }
    const std::string msg = rc ? last_error_cstr() : std::string();
    sa->release();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->in_use -= sa->bytes;
        s->cv.notify_all();
    }
    return rc ? fail(rc, msg) : SARBP_OK;
}

int sarbp_server_counters(sarbp_server *s, double *h2d_bytes, long long *rc_pulses,
                          long long *resident_requests) {
    if (!s) return fail(SARBP_ERR_INVALID, "server is NULL");
    if (h2d_bytes) *h2d_bytes = (double)s->h2d_bytes.load();
    if (rc_pulses) *rc_pulses = s->rc_pulses.load();
    if (resident_requests) *resident_requests = s->resident_requests.load();
    return SARBP_OK;
}

}  // extern "C"
