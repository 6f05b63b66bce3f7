// runner.cpp -- validation, scratch layout and launch sequence of a batch.
#include "runner.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

#include "host_math.h"

namespace sarbp {

namespace {
thread_local std::string g_error;

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
bool is_pow2(long long n) { return n > 0 && (n & (n - 1)) == 0; }
int ilog2i(long long n) {
    int l = 0;
    while ((1ll << l) < n) ++l;
    return l;
}

struct JobLayout {
    size_t Q, Qp, filt, wS, wP, pulse, tiles, recs, fin, parts, end;
};

// Scratch of one job: profiles (pairs for the tile kernel, plain Q for the
// range-compression-only entry point), windows, pulse table, and for the
// tile kernel the tile table, per-(tile, pulse) records and final phases,
// and for a job formed in nsplit > 1 pulse parts one partial image per part.
JobLayout layout_of(const sarbp_job &j, size_t base, int tile_x, int tile_y, bool rc_only, bool naive,
                    bool resident = false, int nsplit = 1) {
    JobLayout L;
    const size_t P = (size_t)j.npulses, N = (size_t)j.n_fft, S = (size_t)j.nsamples;
    const bool tiles = !rc_only && !naive;
    const size_t ntiles =
        tiles ? (size_t)((j.nu + tile_x - 1) / tile_x) * (size_t)((j.nv + tile_y - 1) / tile_y) : 0;
    size_t o = base;
    L.Q = o;      o = align_up(o + (rc_only ? P * N * sizeof(float2) : 0), 256);
    L.Qp = o;     o = align_up(o + (rc_only || resident ? 0 : P * (N + 1) * sizeof(float4)), 256);
    L.filt = o;   o = align_up(o + S * sizeof(float), 256);
    L.wS = o;     o = align_up(o + S * sizeof(float), 256);
    L.wP = o;     o = align_up(o + P * sizeof(float), 256);
    L.pulse = o;  o = align_up(o + P * sizeof(double4), 256);
    L.tiles = o;  o = align_up(o + ntiles * sizeof(TileInfo), 256);
    L.recs = o;   o = align_up(o + ntiles * P * sizeof(PulseRec), 256);
    L.fin = o;    o = align_up(o + (tiles ? (size_t)j.nu * j.nv * sizeof(float2) : 0), 256);
    L.parts = o;  o = align_up(o + (tiles && nsplit > 1 ? (size_t)nsplit * j.nu * j.nv * sizeof(float2) : 0), 256);
    L.end = o;
    return L;
}

int precision_of(const sarbp_job &j, const sarbp_opts *o) {
    if (j.precision >= 0) return j.precision;
    return o ? o->precision : SARBP_PREC_COMPAT;
}

}  // namespace

int validate_job(const sarbp_job &j, int prec, int idx, bool rc_only, bool need_phs) {
    auto bad = [&](const std::string &what) {
        return fail(SARBP_ERR_INVALID, "job " + std::to_string(idx) + ": " + what);
    };
    if (j.nsamples < 1 || j.npulses < 1) return bad("nsamples and npulses must be >= 1");
    if (!rc_only && (j.nu < 1 || j.nv < 1)) return bad("image extents nu and nv must be >= 1");
    if ((long long)j.nu * j.nv > (1ll << 31)) return bad("image larger than 2^31 pixels");
    if (!is_pow2(j.n_fft) || j.n_fft < (1 << kMinLogN) || j.n_fft > (1 << kMaxLogN))
        return fail(SARBP_ERR_UNSUPPORTED, "job " + std::to_string(idx) +
                                               ": N_fft must be a power of two in [16, 131072], got " +
                                               std::to_string(j.n_fft));
    if (j.taylor_s_l < 1) return bad("taylor must be >= 1");
    if (!(std::isfinite(j.delta_r))) return bad("delta_r must be finite");
    if (prec != SARBP_PREC_COMPAT && prec != SARBP_PREC_PRECISE && prec != SARBP_PREC_NAIVE)
        return bad("unknown precision mode");
    if (need_phs && !j.phs) return bad("phs is NULL");
    if (!j.k_r && !(prec == SARBP_PREC_PRECISE && j.k_r64)) return bad("k_r is NULL");
    if (!j.pos && !(prec == SARBP_PREC_PRECISE && j.pos64)) return bad("pos is NULL");
    if (!rc_only && !j.r && !(j.u && j.v)) return bad("pixel positions: r, or u and v, are required");
    if (!rc_only && !j.output_img) return bad("output_img is NULL");
    if (j.out_u8 && !(j.dB_min < j.dB_max)) return bad("dB_min < dB_max is required for the u8 image");
    if (j.taylor_mode != SARBP_TAYLOR_REF && j.taylor_mode != SARBP_TAYLOR_FLOAT)
        return bad("unknown taylor_mode");
    const std::vector<double> F = taylor_coefficients(j.taylor_s_l, j.taylor_mode);
    if ((int)F.size() > kMaxTaylorTerms) return bad("taylor side-lobe level too large (n_bar > 65)");
    for (double f : F)
        if (!std::isfinite(f))
            return bad("taylor " + std::to_string(j.taylor_s_l) +
                       " dB: the window formula of signal.h:39-41 divides by zero for side-lobe "
                       "levels above 30 dB (its F_m denominator uses Int32 division); "
                       "SARBP_TAYLOR_FLOAT takes that quotient in floating point");
    const double lsa = std::floor((double)(-j.nsamples) * j.delta_r / 2);
    const double lsb = std::floor((double)j.nsamples * j.delta_r / 2);
    if (!(lsb > lsa)) return bad("range axis is empty: floor(S*delta_r/2) <= floor(-S*delta_r/2)");
    return SARBP_OK;
}

void describe_job(const sarbp_job &j, int prec, int tile_x, int tile_y, DevJob &dj) {
    dj.S = j.nsamples;
    dj.P = j.npulses;
    dj.N = j.n_fft;
    dj.nu = j.nu;
    dj.nv = j.nv;
    dj.precision = prec;
    dj.tile_x = tile_x;
    dj.tile_y = tile_y;
    dj.tiles_x = (j.nu + tile_x - 1) / tile_x;
    dj.tiles_y = (j.nv + tile_y - 1) / tile_y;
    dj.logN = ilog2i(j.n_fft);
    dj.n_taylor = taylor_coefficients_into(j.taylor_s_l, dj.taylor_F, kMaxTaylorTerms, j.taylor_mode);
    dj.phs = reinterpret_cast<const float2 *>(j.phs);
    dj.k_r32 = j.k_r;
    dj.k_r64 = j.k_r64;
    dj.pos32 = j.pos;
    dj.pos64 = j.pos64;
    dj.r = j.r;
    dj.u = j.u;
    dj.v = j.v;
    for (int k = 0; k < 3; ++k) {
        dj.uh[k] = j.u_hat[k];
        dj.vh[k] = j.v_hat[k];
    }
    dj.delta_r = j.delta_r;
    // backprojection.cpp:120 and :53: lsa = floor(-S*dr/2), lsb = floor(S*dr/2),
    // lsr = (lsb - lsa) / (N_fft - 1)
    dj.lsa = std::floor((double)(-j.nsamples) * j.delta_r / 2);
    const double lsb = std::floor((double)j.nsamples * j.delta_r / 2);
    dj.lsr = (lsb - dj.lsa) / (double)(j.n_fft - 1);
    dj.inv_lsr = 1.0 / dj.lsr;
    dj.out = reinterpret_cast<double2 *>(j.output_img);
    dj.out_u8 = j.out_u8;
    dj.dB_min = j.dB_min;
    dj.dB_max = j.dB_max;
    dj.chunked = 0;
    dj.acc = nullptr;
    dj.nsplit = 1;
    dj.parts = nullptr;
}

void set_error(const std::string &msg) { g_error = msg; }
int fail(int code, const std::string &msg) {
    g_error = msg;
    return code;
}
int cuda_fail(cudaError_t e, const char *what) {
    g_error = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? SARBP_ERR_NOMEM : SARBP_ERR_CUDA;
}
const char *last_error_cstr() { return g_error.c_str(); }

cudaError_t DeviceBuffer::ensure(size_t bytes, cudaStream_t st) {
    if (bytes <= cap) return cudaSuccess;
    if (ptr) {
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return e;
        cudaFree(ptr);
        ptr = nullptr;
        cap = 0;
    }
    const size_t want = align_up(bytes + bytes / 8, 1 << 20);
    cudaError_t e = cudaMalloc(&ptr, want);
    if (e != cudaSuccess) {
        ptr = nullptr;
        return e;
    }
    cap = want;
    return cudaSuccess;
}
cudaError_t DeviceBuffer::alloc_exact(size_t bytes) {
    release();
    const size_t want = align_up(bytes > 0 ? bytes : 1, 256);
    cudaError_t e = cudaMalloc(&ptr, want);
    if (e != cudaSuccess) {
        ptr = nullptr;
        return e;
    }
    cap = want;
    return cudaSuccess;
}
void DeviceBuffer::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
}

cudaError_t PinnedBuffer::ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    cap = 0;
    const size_t want = align_up(bytes + bytes / 4, 1 << 16);
    cudaError_t e = cudaMallocHost(&ptr, want);
    if (e != cudaSuccess) {
        ptr = nullptr;
        return e;
    }
    cap = want;
    return cudaSuccess;
}
void PinnedBuffer::release() {
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    cap = 0;
}

bool DeviceInfo::has_twiddle(int logN) {
    std::lock_guard<std::mutex> lk(mu);
    return twiddles.count(logN) != 0;
}

cudaError_t DeviceInfo::twiddle(int logN, float2 **out) {
    std::lock_guard<std::mutex> lk(mu);
    auto it = twiddles.find(logN);
    if (it != twiddles.end()) {
        *out = it->second;
        return cudaSuccess;
    }
    const int n = std::max(1, twiddle_table_size(logN));
    std::vector<float2> h(n);
    fill_twiddle_table(logN, h.data());
    float2 *d = nullptr;
    cudaError_t e = cudaMalloc(&d, n * sizeof(float2));
    if (e != cudaSuccess) return e;
    e = cudaMemcpy(d, h.data(), n * sizeof(float2), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(d);
        return e;
    }
    twiddles[logN] = d;
    *out = d;
    return cudaSuccess;
}
cudaError_t range_compress_rows(DeviceInfo *dev, int logN, const DevJob *d_jobs, const RowItem *d_rows, int nrows,
                                int pairs, float2 *work, int work_rows, cudaStream_t st) {
    float2 *tw = nullptr;
    cudaError_t e = dev->twiddle(logN, &tw);
    if (e != cudaSuccess) return e;
    if (logN <= kMaxLogNSmem) return launch_range_compress(logN, d_jobs, d_rows, nrows, pairs, tw, st);
    float2 *tw1 = nullptr, *tw2 = nullptr;
    if ((e = dev->twiddle(logN / 2, &tw1)) != cudaSuccess) return e;
    if ((e = dev->twiddle(logN - logN / 2, &tw2)) != cudaSuccess) return e;
    return launch_range_compress_large(logN, d_jobs, d_rows, nrows, pairs, tw1, tw2, tw, work, work_rows, st);
}

cudaError_t DeviceInfo::record(int i, cudaStream_t st) {
    if (!timing) return cudaSuccess;
    if (!ev[i]) {
        cudaError_t e = cudaEventCreate(&ev[i]);
        if (e != cudaSuccess) return e;
    }
    ev_recorded[i] = true;
    return cudaEventRecord(ev[i], st);
}

void DeviceInfo::release() {
    for (int i = 0; i < kEvents; ++i)
        if (ev[i]) cudaEventDestroy(ev[i]);
    for (auto &kv : twiddles) cudaFree(kv.second);
    twiddles.clear();
}

BpLaunch default_launch(const sarbp_opts *opts, int num_sms) {
    BpLaunch L;
    L.tile_x = 32;
    L.tile_y = 32;
    L.minb = 3;
    L.stage_cap = 2048;
    L.cmax = 64;
    L.persistent = 1;
    L.parts = 0;
    if (opts) {
        if (opts->tile_x > 0 && opts->tile_y > 0) {
            L.tile_x = opts->tile_x;
            L.tile_y = opts->tile_y;
        }
        if (opts->pulse_chunk > 0) L.cmax = std::min(256, std::max(4, opts->pulse_chunk));
        L.persistent = opts->persistent == 2 ? 0 : 1;
        if (opts->stage_cap > 0) L.stage_cap = std::max(64, std::min(4096, opts->stage_cap)) & ~1;
        if (opts->min_blocks == 2 || opts->min_blocks == 3) L.minb = opts->min_blocks;
        L.parts = std::max(0, std::min(16, opts->pulse_parts));
    }
    L.cmax = (L.cmax + 3) / 4 * 4;
    L.grid = num_sms;
    return L;
}

BpLaunch resolved_launch(const sarbp_opts *opts, int num_sms) {
    BpLaunch L = default_launch(opts, num_sms);
    if (!bp_tile_supported(L.tile_x, L.tile_y, L.minb) && !(opts && opts->min_blocks)) L.minb = 2;
    return L;
}

int pulse_parts(int nu, int nv, int P, const BpLaunch &L, int num_sms) {
    constexpr int kMaxParts = 16, kMinPartPulses = 32;
    constexpr double kItemCost = 16.0;  // fixed cost of an item, in pulses of its tile
    const long long ntiles = (long long)((nu + L.tile_x - 1) / L.tile_x) * ((nv + L.tile_y - 1) / L.tile_y);
    const int sms = std::max(1, num_sms), minb = std::max(1, L.minb);
    const long long R = (long long)minb * sms;  // resident CTAs
    if (L.parts >= 1) return std::max(1, std::min(L.parts, P));
    if ((long long)nu * nv >= (1ll << 18) || 2 * ntiles > R || ntiles < 1) return 1;
    // Estimated time of s parts per tile, in pulse times of a CTA on a full
    // SM: an SM running k CTAs does f(k) of a full SM's work (fewer warps
    // hide less latency; measured on 256^2, 512^2 and 2048^2 images alone),
    // and the SMs with the most items set the time.
    auto f = [](long long k) { return k == 1 ? 0.80 : k == 2 ? 0.95 : 1.0; };
    auto time_of = [&](int s) {
        const long long items = ntiles * s;
        const double item = (double)P / s + kItemCost;
        if (items <= R) {
            const long long k = (items + sms - 1) / sms;
            return (double)k * item / f(k);
        }
        return (double)((items + R - 1) / R) * minb * item / f(minb);
    };
    int best = 1;
    double best_t = time_of(1) / 1.15;
    for (int s = 2; s <= kMaxParts && P / s >= kMinPartPulses; ++s) {
        const double t = time_of(s);
        if (t < best_t) {
            best = s;
            best_t = t;
        }
    }
    return best;
}

size_t Runner::job_scratch_bytes(const sarbp_job &j, const sarbp_opts *opts, bool resident_profiles, int num_sms) {
    const BpLaunch L = resolved_launch(opts, num_sms);
    const bool naive = j.precision == SARBP_PREC_NAIVE;
    const int ns = naive ? 1 : pulse_parts(j.nu, j.nv, j.npulses, L, num_sms);
    const size_t work = resident_profiles ? 0 : align_up(rc_work_bytes(ilog2i(j.n_fft)), 256);
    return layout_of(j, 0, L.tile_x, L.tile_y, false, naive, resident_profiles, ns).end + work;
}

Runner::~Runner() {
    if (side_) cudaStreamSynchronize(side_);
    scratch_.release();
    meta_.release();
    host_meta_.release();
    status_pin_.release();
    if (meta_done_) cudaEventDestroy(meta_done_);
    if (front_done_) cudaEventDestroy(front_done_);
    if (side_) cudaStreamDestroy(side_);
    if (fork_) cudaEventDestroy(fork_);
    if (join_) cudaEventDestroy(join_);
}

void Runner::tile_shape(const sarbp_opts *opts, int *tile_x, int *tile_y) {
    const BpLaunch L = default_launch(opts, 148);
    *tile_x = L.tile_x;
    *tile_y = L.tile_y;
}

int Runner::enqueue(const sarbp_job *jobs, int njobs, const sarbp_opts *opts, cudaStream_t st,
                    void *q_out, bool for_graph, const SlabSpec *slabs, const float4 *const *resident_qp) {
    const bool rc_only = q_out != nullptr;
    if (rc_only) resident_qp = nullptr;
    auto resident = [&](int i) { return resident_qp && resident_qp[i]; };
    if (slabs && slabs->nslabs > 0) {
        if (njobs != 1 || rc_only || for_graph || !slabs->row0 || !slabs->aux || !slabs->done)
            return fail(SARBP_ERR_INVALID, "row slabs need one job, a second stream and done events");
        if (!front_done_) {
            cudaError_t e = cudaEventCreateWithFlags(&front_done_, cudaEventDisableTiming);
            if (e != cudaSuccess) return cuda_fail(e, "cudaEventCreate");
        }
    } else {
        slabs = nullptr;
    }
    auto rec = [&](int i) { return (for_graph || !stage_events) ? cudaSuccess : dev_->record(i, st); };
    if (njobs < 1 || !jobs) return fail(SARBP_ERR_INVALID, "no jobs");
    BpLaunch L = resolved_launch(opts, dev_->num_sms);
    if (!bp_tile_supported(L.tile_x, L.tile_y, L.minb))
        return fail(SARBP_ERR_INVALID, "unsupported pixel tile " + std::to_string(L.tile_x) + "x" +
                                           std::to_string(L.tile_y) + " at " + std::to_string(L.minb) +
                                           " CTAs/SM");
    std::vector<int> prec(njobs);
    for (int i = 0; i < njobs; ++i) {
        prec[i] = precision_of(jobs[i], opts);
        int rc = validate_job(jobs[i], prec[i], i, rc_only, !resident(i));
        if (rc) return rc;
    }
    if (!meta_done_) {
        cudaError_t e = cudaEventCreateWithFlags(&meta_done_, cudaEventDisableTiming);
        if (e != cudaSuccess) return cuda_fail(e, "cudaEventCreate");
    }
    // ---- pulse parts (row slabs come only for images of 2^18 pixels and
    // more without a requested part count, which pulse_parts never splits) ----
    std::vector<int> nsplit(njobs, 1);
    for (int i = 0; i < njobs; ++i)
        if (!rc_only && !slabs && prec[i] != SARBP_PREC_NAIVE)
            nsplit[i] = pulse_parts(jobs[i].nu, jobs[i].nv, jobs[i].npulses, L, dev_->num_sms);
    // ---- scratch layout: JobScalars block first, then per-job arrays ----
    size_t off = align_up((size_t)njobs * sizeof(JobScalars), 256);
    std::vector<JobLayout> lay(njobs);
    for (int i = 0; i < njobs; ++i) {
        lay[i] = layout_of(jobs[i], off, L.tile_x, L.tile_y, rc_only, prec[i] == SARBP_PREC_NAIVE, resident(i),
                           nsplit[i]);
        off = lay[i].end;
    }
    // work buffer of the four-step range compression (N_fft above
    // 2^kMaxLogNSmem), shared by the batch's row groups one after another
    size_t work_off = 0, work_bytes = 0;
    for (int i = 0; i < njobs; ++i)
        if (!resident(i)) work_bytes = std::max(work_bytes, rc_work_bytes(ilog2i(jobs[i].n_fft)));
    if (work_bytes) {
        work_off = off;
        off = align_up(off + work_bytes, 256);
    }
    if (for_graph && (scratch_.cap < off || pool_ || status_pin_.cap < njobs * sizeof(JobScalars)))
        return fail(SARBP_ERR_STATE, "graph capture needs a prior run of the same jobs");
    cudaError_t e;
    char *sbase = nullptr;
    // pool mode: this batch's scratch comes from the pool and goes back to it
    // stream-ordered behind the batch (on every exit path)
    struct PoolBlock {
        void *p = nullptr;
        cudaStream_t st = nullptr;
        ~PoolBlock() {
            if (p) cudaFreeAsync(p, st);
        }
    } pooled;
    if (pool_) {
        pooled.st = st;
        e = cudaMallocFromPoolAsync(&pooled.p, off, pool_, st);
        if (e != cudaSuccess) {
            pooled.p = nullptr;
            return cuda_fail(e, "allocating scratch");
        }
        sbase = static_cast<char *>(pooled.p);
    } else {
        e = scratch_.ensure(off, st);
        if (e != cudaSuccess) return cuda_fail(e, "allocating scratch");
        sbase = static_cast<char *>(scratch_.ptr);
    }
    // status words come back through a pinned copy enqueued behind the batch
    if (status_pin_.cap < njobs * sizeof(JobScalars)) {
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "synchronising the stream");
        if ((e = status_pin_.ensure(njobs * sizeof(JobScalars))) != cudaSuccess)
            return cuda_fail(e, "allocating pinned status words");
    }
    auto copy_status = [&]() -> cudaError_t {
        last_njobs_ = njobs;
        return cudaMemcpyAsync(status_pin_.ptr, sbase, njobs * sizeof(JobScalars), cudaMemcpyDeviceToHost, st);
    };

    // ---- rows grouped by N_fft, work items longest first, one tile-geometry
    // item per tile, the jobs formed in pulse parts ----
    std::map<int, std::vector<RowItem>> rows;
    std::vector<WorkItem> items, tiles;
    std::vector<int> naive, split;
    for (int i = 0; i < njobs; ++i) {
        if (!resident(i)) {  // resident profiles were range-compressed before
            auto &v = rows[ilog2i(jobs[i].n_fft)];
            for (int p = 0; p < jobs[i].npulses; ++p) v.push_back(RowItem{i, p});
        }
        if (rc_only) continue;
        if (prec[i] == SARBP_PREC_NAIVE) {
            naive.push_back(i);
            continue;
        }
        const int tx = (jobs[i].nu + L.tile_x - 1) / L.tile_x;
        const int ty = (jobs[i].nv + L.tile_y - 1) / L.tile_y;
        for (int s = 0; s < nsplit[i]; ++s)
            for (int t = 0; t < tx * ty; ++t) items.push_back(WorkItem{i, t, s});
        if (nsplit[i] > 1) split.push_back(i);
    }
    auto item_pulses = [&](const WorkItem &w) {
        int p0, p1;
        part_range(jobs[w.job].npulses, nsplit[w.job], w.part, p0, p1);
        return p1 - p0;
    };
    std::stable_sort(items.begin(), items.end(),
                     [&](const WorkItem &a, const WorkItem &b) { return item_pulses(a) > item_pulses(b); });
    if (!split.empty())
        for (const WorkItem &w : items)
            if (w.part == 0) tiles.push_back(w);
    size_t nrows_total = 0;
    for (auto &kv : rows) nrows_total += kv.second.size();

    // ---- meta block: [DevJob][RowItem...][WorkItem...][tile WorkItem...]
    // [split job...][counter] (the tile list only when a job is split: the
    // work items are then not one per tile) ----
    const size_t o_jobs = 0;
    const size_t o_rows = align_up(o_jobs + (size_t)njobs * sizeof(DevJob), 256);
    const size_t o_items = align_up(o_rows + nrows_total * sizeof(RowItem), 256);
    const size_t o_tiles = align_up(o_items + items.size() * sizeof(WorkItem), 256);
    const size_t o_split = align_up(o_tiles + tiles.size() * sizeof(WorkItem), 256);
    const size_t o_cnt = align_up(o_split + split.size() * sizeof(int), 256);
    const size_t meta_bytes = o_cnt + 256 * (size_t)(slabs ? slabs->nslabs : 1);
    if (for_graph && (host_meta_.cap < meta_bytes || meta_.cap < meta_bytes))
        return fail(SARBP_ERR_STATE, "graph capture needs a prior run of the same jobs");
    // the previous batch's descriptor copy must have left host_meta_
    e = for_graph ? cudaSuccess : cudaEventSynchronize(meta_done_);
    if (e != cudaSuccess) return cuda_fail(e, "waiting for the previous batch");
    e = host_meta_.ensure(meta_bytes);
    if (e != cudaSuccess) return cuda_fail(e, "allocating pinned descriptors");
    e = meta_.ensure(meta_bytes, st);
    if (e != cudaSuccess) return cuda_fail(e, "allocating device descriptors");
    char *h = static_cast<char *>(host_meta_.ptr);
    char *d = static_cast<char *>(meta_.ptr);
    std::memset(h, 0, meta_bytes);

    DevJob *hj = reinterpret_cast<DevJob *>(h + o_jobs);
    for (int i = 0; i < njobs; ++i) {
        const sarbp_job &j = jobs[i];
        DevJob &dj = hj[i];
        describe_job(j, prec[i], L.tile_x, L.tile_y, dj);
        dj.Q = reinterpret_cast<float2 *>(sbase + lay[i].Q);
        dj.Qp = rc_only ? nullptr
                : resident(i) ? const_cast<float4 *>(resident_qp[i])
                              : reinterpret_cast<float4 *>(sbase + lay[i].Qp);
        dj.tiles = reinterpret_cast<TileInfo *>(sbase + lay[i].tiles);
        dj.recs = reinterpret_cast<PulseRec *>(sbase + lay[i].recs);
        dj.fin = reinterpret_cast<float2 *>(sbase + lay[i].fin);
        dj.filt = reinterpret_cast<float *>(sbase + lay[i].filt);
        dj.wS = reinterpret_cast<float *>(sbase + lay[i].wS);
        dj.wP = reinterpret_cast<float *>(sbase + lay[i].wP);
        dj.pulse = reinterpret_cast<double4 *>(sbase + lay[i].pulse);
        dj.sc = reinterpret_cast<JobScalars *>(sbase) + i;
        dj.nsplit = nsplit[i];
        dj.parts = nsplit[i] > 1 ? reinterpret_cast<float2 *>(sbase + lay[i].parts) : nullptr;
    }
    RowItem *hr = reinterpret_cast<RowItem *>(h + o_rows);
    std::vector<std::pair<int, size_t>> row_groups;  // (logN, first row)
    size_t rpos = 0;
    for (auto &kv : rows) {
        row_groups.push_back({kv.first, rpos});
        std::memcpy(hr + rpos, kv.second.data(), kv.second.size() * sizeof(RowItem));
        rpos += kv.second.size();
    }
    std::memcpy(h + o_items, items.data(), items.size() * sizeof(WorkItem));
    std::memcpy(h + o_tiles, tiles.data(), tiles.size() * sizeof(WorkItem));
    std::memcpy(h + o_split, split.data(), split.size() * sizeof(int));

    cudaStream_t ms = (slabs && slabs->copy_stream) ? slabs->copy_stream : st;
    e = cudaMemcpyAsync(d, h, meta_bytes, cudaMemcpyHostToDevice, ms);
    if (e != cudaSuccess) return cuda_fail(e, "copying descriptors");
    e = for_graph ? cudaSuccess : cudaEventRecord(meta_done_, ms);
    if (e == cudaSuccess && ms != st) e = cudaStreamWaitEvent(st, meta_done_, 0);
    if (e != cudaSuccess) return cuda_fail(e, "ordering the descriptor copy");

    const DevJob *d_jobs = reinterpret_cast<const DevJob *>(d + o_jobs);
    const RowItem *d_rows = reinterpret_cast<const RowItem *>(d + o_rows);
    const WorkItem *d_items = reinterpret_cast<const WorkItem *>(d + o_items);
    const WorkItem *d_tiles = split.empty() ? d_items : reinterpret_cast<const WorkItem *>(d + o_tiles);
    const int ntile_items = split.empty() ? (int)items.size() : (int)tiles.size();
    const int *d_split = reinterpret_cast<const int *>(d + o_split);
    int *d_cnt = reinterpret_cast<int *>(d + o_cnt);

    // twiddle tables first (a one-time synchronous upload per N_fft; a
    // four-step N_fft also needs the tables of its two sub-lengths)
    for (size_t g = 0; g < row_groups.size(); ++g) {
        const int l = row_groups[g].first;
        const int need[3] = {l, l > kMaxLogNSmem ? l / 2 : l, l > kMaxLogNSmem ? l - l / 2 : l};
        for (int n : need) {
            float2 *tw = nullptr;
            if (for_graph && !dev_->has_twiddle(n))
                return fail(SARBP_ERR_STATE, "graph capture needs a prior run of the same jobs");
            e = dev_->twiddle(n, &tw);
            if (e != cudaSuccess) return cuda_fail(e, "twiddle table");
        }
    }
    if (stage_events)
        for (int k = 0; k < DeviceInfo::kEvents; ++k) dev_->ev_recorded[k] = false;
    if ((e = rec(0)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
    launch_prep(d_jobs, njobs, st);
    dev_->launches++;
    if ((e = rec(1)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
    const bool slabbed = slabs && !items.empty() && prec[0] != SARBP_PREC_NAIVE;
    // Range compression beside the tile geometry: both read only the
    // set-up's tables, and the backprojection waits for both.  Each kernel
    // fills the SMs on its own, so they mostly fill each other's tails
    // (5.988 -> 5.979 ms per 2048^2 x 1999 step).  Not while the context
    // times its stages (each stage then runs alone), and not for row slabs
    // (their geometry already runs beside the backprojection).
    const bool side = !rc_only && !slabbed && !items.empty() && !row_groups.empty() &&
                      !(stage_events && dev_->timing && !for_graph);
    cudaStream_t rs = st;
    if (side) {
        if (!side_ && (e = cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking)) != cudaSuccess)
            return cuda_fail(e, "creating a stream");
        if (!fork_ && (e = cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming)) != cudaSuccess)
            return cuda_fail(e, "cudaEventCreate");
        if (!join_ && (e = cudaEventCreateWithFlags(&join_, cudaEventDisableTiming)) != cudaSuccess)
            return cuda_fail(e, "cudaEventCreate");
        if ((e = cudaEventRecord(fork_, st)) != cudaSuccess || (e = cudaStreamWaitEvent(side_, fork_, 0)) != cudaSuccess)
            return cuda_fail(e, "ordering range compression");
        rs = side_;
    }
    // the main stream waits for the side stream before the backprojection,
    // and on every return in between (nothing may outlive the batch there)
    struct Join {
        cudaStream_t st = nullptr, side = nullptr;
        cudaEvent_t ev = nullptr;
        cudaError_t now() {
            cudaError_t r = cudaSuccess;
            if (ev && (r = cudaEventRecord(ev, side)) == cudaSuccess) r = cudaStreamWaitEvent(st, ev, 0);
            ev = nullptr;
            return r;
        }
        ~Join() { now(); }
    } join{st, side_, side ? join_ : nullptr};
    for (size_t g = 0; g < row_groups.size(); ++g) {
        const int logN = row_groups[g].first;
        const size_t first = row_groups[g].second;
        const size_t count = rows[logN].size();
        float2 *work = work_bytes ? reinterpret_cast<float2 *>(sbase + work_off) : nullptr;
        e = range_compress_rows(dev_, logN, d_jobs, d_rows + first, (int)count, rc_only ? 0 : 1, work,
                                rc_work_rows(logN), rs);
        if (e != cudaSuccess) return cuda_fail(e, "range compression launch");
        dev_->launches++;
    }
    if ((e = rec(2)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
    if (rc_only) {
        e = cudaMemcpyAsync(q_out, hj[0].Q, (size_t)jobs[0].npulses * jobs[0].n_fft * sizeof(float2),
                            cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return cuda_fail(e, "copying range profiles");
        if ((e = copy_status()) != cudaSuccess) return cuda_fail(e, "copying job status");
        return SARBP_OK;
    }
    if (slabs && slabs->before_slabs && (e = slabs->before_slabs()) != cudaSuccess)
        return cuda_fail(e, "slab input copies");
    if (slabbed) {
        // ---- row slabs: geometry + backprojection per slab, two streams ----
        // (stage events: the slabs' geometry counts with the backprojection)
        if ((e = rec(3)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
        if ((e = cudaEventRecord(front_done_, st)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
        const int tiles_x = (jobs[0].nu + L.tile_x - 1) / L.tile_x;
        if (bp_max_active_blocks(L) < 1) return fail(SARBP_ERR_CUDA, "backprojection kernel does not fit on an SM");
        for (int g = 0; g < slabs->nslabs; ++g) {
            const size_t first = std::min(items.size(), (size_t)slabs->row0[g] * tiles_x);
            const size_t last = std::min(items.size(), (size_t)std::max(slabs->row0[g], slabs->row0[g + 1]) * tiles_x);
            cudaStream_t sg = (g & 1) ? slabs->aux : st;
            if ((g & 1) && (e = cudaStreamWaitEvent(sg, front_done_, 0)) != cudaSuccess)
                return cuda_fail(e, "cudaStreamWaitEvent");
            if (slabs->ready && (e = cudaStreamWaitEvent(sg, slabs->ready[g], 0)) != cudaSuccess)
                return cuda_fail(e, "cudaStreamWaitEvent");
            if (last > first) {
                const int n = (int)(last - first);
                e = launch_tile_setup(d_jobs, d_items + first, n, L.tile_x * L.tile_y, sg);
                // one CTA per tile: the block scheduler then starts the next
                // slab's CTAs (other stream) as this slab's last tiles finish
                // (persistent CTAs per slab, pulling the slab's tiles from its
                // own counter, measured 6.58 against 6.49 ms per 2048^2 x
                // 1999 host-buffer call)
                BpLaunch Lg = L;
                Lg.persistent = 0;
                Lg.grid = n;
                if (e == cudaSuccess) e = launch_backproject(Lg, d_jobs, d_items + first, n, d_cnt + 64 * g, sg);
                if (e != cudaSuccess) return cuda_fail(e, "slab launch");
                dev_->launches += 2;
            }
            if ((e = cudaEventRecord(slabs->done[g], sg)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
        }
        for (int g = 1; g < slabs->nslabs; g += 2)
            if ((e = cudaStreamWaitEvent(st, slabs->done[g], 0)) != cudaSuccess)
                return cuda_fail(e, "cudaStreamWaitEvent");
        items.clear();  // formed above
    }
    if (!items.empty()) {
        e = launch_tile_setup(d_jobs, d_tiles, ntile_items, L.tile_x * L.tile_y, st);
        if (e != cudaSuccess) return cuda_fail(e, "tile geometry launch");
        dev_->launches += 1;
    }
    if ((e = join.now()) != cudaSuccess) return cuda_fail(e, "ordering range compression");
    if (!slabbed && (e = rec(3)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
    if (!items.empty()) {
        if (L.persistent) {
            const int occ = bp_max_active_blocks(L);
            if (occ < 1) return fail(SARBP_ERR_CUDA, "backprojection kernel does not fit on an SM");
            L.grid = std::min<long long>((long long)occ * dev_->num_sms, (long long)items.size());
        }
        e = launch_backproject(L, d_jobs, d_items, (int)items.size(), d_cnt, st);
        if (e != cudaSuccess) return cuda_fail(e, "backprojection launch");
        dev_->launches++;
    }
    if (!split.empty()) {
        long long px = 0;
        for (int i : split) px = std::max(px, (long long)jobs[i].nu * jobs[i].nv);
        e = launch_combine_parts(d_jobs, d_split, (int)split.size(), px, dev_->num_sms, st);
        if (e != cudaSuccess) return cuda_fail(e, "pulse-part combine launch");
        dev_->launches++;
    }
    for (int i : naive) {
        e = launch_backproject_naive(d_jobs, i, jobs[i].nu, jobs[i].nv, st);
        if (e != cudaSuccess) return cuda_fail(e, "naive backprojection launch");
        dev_->launches++;
    }
    if (slabs && !slabbed)  // the whole image is final here
        for (int g = 0; g < slabs->nslabs; ++g)
            if ((e = cudaEventRecord(slabs->done[g], st)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
    if ((e = rec(4)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
    bool any_u8 = false;
    long long max_px = 0;
    for (int i = 0; i < njobs; ++i) {
        any_u8 = any_u8 || jobs[i].out_u8;
        max_px = std::max(max_px, (long long)jobs[i].nu * jobs[i].nv);
    }
    if (any_u8) {
        e = launch_batch_u8(d_jobs, njobs, max_px, st);
        if (e != cudaSuccess) return cuda_fail(e, "u8 launch");
        dev_->launches++;
        if ((e = rec(5)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
    }
    if ((e = copy_status()) != cudaSuccess) return cuda_fail(e, "copying job status");
    return SARBP_OK;
}

int Runner::check_status(cudaStream_t st) {
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "synchronising the stream");
    if (last_njobs_ == 0 || !status_pin_.ptr) return SARBP_OK;
    const JobScalars *sc = static_cast<const JobScalars *>(status_pin_.ptr);
    for (int i = 0; i < last_njobs_; ++i) {
        const int s = sc[i].status;
        if (s & kStatusNonFinite)
            return fail(SARBP_ERR_GEOMETRY, "job " + std::to_string(i) +
                                                ": non-finite pixel or antenna position (those "
                                                "pixels or pulses were left out)");
        if (s & kStatusTimeout)
            return fail(SARBP_ERR_TIMEOUT, "job " + std::to_string(i) +
                                               ": a bounded wait for a range-profile copy gave up");
        if (s & kStatusTileTooWide)
            return fail(SARBP_ERR_GEOMETRY,
                        "job " + std::to_string(i) +
                            ": a pixel tile spans more range bins than fit on chip (pixel positions "
                            "are not spatially compact); those tiles were left at zero");
    }
    return SARBP_OK;
}

}  // namespace sarbp
