// plan.cpp -- CUDA-graph plans of a job batch and the launch-shape autotuner.
//
// A plan is one batch of device-resident jobs (uneven sizes allowed)
// enqueued once for real, which sizes every scratch buffer and builds the
// twiddle tables, and then captured into a CUDA graph: prep, one range
// compression launch per FFT length, tile geometry, the persistent
// backprojection over the (job, tile, pulse part) work list (and the combine
// of pulse parts) and the u8 stage.  Each
// replay re-reads the job descriptors from the plan's own pinned copy, so the
// input arrays may hold new data between replays but must keep their
// addresses and shapes.
//
// The autotuner times the whole batch (set-up through backprojection) over
// a set of pixel-tile shapes, CTAs per SM and pulse-chunk depths, keeps the
// fastest and caches it in the context under the batch's shape signature.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <memory>
#include <string>
#include <vector>

#include "context.h"
#include "kernels.h"
#include "runner.h"
#include "sarbp_b200.h"

using namespace sarbp;

struct sarbp_plan {
    sarbp_ctx *ctx = nullptr;
    std::unique_ptr<Runner> runner;
    cudaStream_t cap = nullptr;  // the plan's own stream (capture and default replay)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t last = nullptr;  // stream of the latest replay
    int kernels = 0;

    ~sarbp_plan() {
        if (last) cudaStreamSynchronize(last);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        runner.reset();
        if (cap) cudaStreamDestroy(cap);
    }
};

namespace {

std::string shape_key(const sarbp_job *jobs, int njobs, int precision) {
    std::vector<std::string> parts;
    parts.reserve(njobs);
    char b[96];
    for (int i = 0; i < njobs; ++i) {
        const sarbp_job &j = jobs[i];
        std::snprintf(b, sizeof(b), "%dx%dp%ds%dn%d", j.nu, j.nv, j.npulses, j.nsamples, j.n_fft);
        parts.emplace_back(b);
    }
    std::sort(parts.begin(), parts.end());
    std::string k = "prec" + std::to_string(precision);
    for (const auto &p : parts) k += "|" + p;
    return k;
}

struct Candidate {
    int tx, ty, minb;
};

}  // namespace

extern "C" {

int sarbp_plan_create(sarbp_ctx *ctx, const sarbp_job *jobs, int njobs, const sarbp_opts *opts,
                      sarbp_plan **out) {
    int rc = ctx_set_device(ctx);
    if (rc) return rc;
    if (!out || !jobs || njobs < 1) return fail(SARBP_ERR_INVALID, "bad plan arguments");
    *out = nullptr;
    auto p = std::make_unique<sarbp_plan>();
    p->ctx = ctx;
    p->runner = std::make_unique<Runner>(&ctx->dev);
    cudaError_t e = cudaStreamCreateWithFlags(&p->cap, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
    // one real run: sizes the scratch, uploads twiddles, checks the jobs
    rc = p->runner->enqueue(jobs, njobs, opts, p->cap);
    if (rc) return rc;
    rc = p->runner->check_status(p->cap);
    if (rc) return rc;
    e = cudaStreamBeginCapture(p->cap, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamBeginCapture");
    rc = p->runner->enqueue(jobs, njobs, opts, p->cap, nullptr, true);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(p->cap, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    p->graph = g;
    e = cudaGraphInstantiate(&p->exec, g, 0);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
    size_t n = 0;
    e = cudaGraphGetNodes(g, nullptr, &n);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphGetNodes");
    std::vector<cudaGraphNode_t> nodes(n);
    if (n && (e = cudaGraphGetNodes(g, nodes.data(), &n)) != cudaSuccess)
        return cuda_fail(e, "cudaGraphGetNodes");
    for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++p->kernels;
    }
    *out = p.release();
    return SARBP_OK;
}

int sarbp_plan_launch(sarbp_plan *plan, void *cuda_stream) {
    if (!plan) return fail(SARBP_ERR_INVALID, "plan is NULL");
    int rc = ctx_set_device(plan->ctx);
    if (rc) return rc;
    cudaStream_t st = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : plan->cap;
    cudaError_t e = cudaGraphLaunch(plan->exec, st);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphLaunch");
    plan->last = st;
    plan->ctx->dev.launches += plan->kernels;
    return SARBP_OK;
}

int sarbp_plan_wait(sarbp_plan *plan) {
    if (!plan) return fail(SARBP_ERR_INVALID, "plan is NULL");
    int rc = ctx_set_device(plan->ctx);
    if (rc) return rc;
    return plan->runner->check_status(plan->last ? plan->last : plan->cap);
}

int sarbp_plan_kernel_count(const sarbp_plan *plan) { return plan ? plan->kernels : -1; }

int sarbp_plan_destroy(sarbp_plan *plan) {
    if (!plan) return SARBP_OK;
    int rc = ctx_set_device(plan->ctx);
    delete plan;
    return rc;
}

int sarbp_autotune(sarbp_ctx *ctx, const sarbp_job *jobs, int njobs, sarbp_opts *inout,
                   float *best_ms) {
    int rc = ctx_set_device(ctx);
    if (rc) return rc;
    if (!inout || !jobs || njobs < 1) return fail(SARBP_ERR_INVALID, "bad autotune arguments");
    if (best_ms) *best_ms = -1.0f;
    const std::string key = shape_key(jobs, njobs, inout->precision);
    auto hit = ctx->tuned.find(key);
    if (hit != ctx->tuned.end()) {
        const int prec = inout->precision;
        *inout = hit->second;
        inout->precision = prec;
        return SARBP_OK;
    }
    static const Candidate kCands[] = {{32, 32, 3}, {32, 16, 3}, {64, 16, 3}, {16, 32, 3},
                                       {32, 32, 2}, {32, 64, 2}, {64, 32, 2}, {16, 64, 2}};
    static const int kChunks[] = {32, 64, 128};
    DeviceInfo &d = ctx->dev;
    const bool timing_was = d.timing;
    d.timing = true;
    auto time_once = [&](const sarbp_opts &o, float *ms) -> int {
        int r = ctx->runner->enqueue(jobs, njobs, &o, ctx->stream);
        if (r) return r;
        r = ctx->runner->check_status(ctx->stream);
        if (r) return r;
        cudaError_t e = cudaEventElapsedTime(ms, d.ev[0], d.ev[4]);
        return e == cudaSuccess ? SARBP_OK : cuda_fail(e, "cudaEventElapsedTime");
    };
    struct Trial {
        sarbp_opts o;
        float ms;
    };
    std::vector<Trial> trials;
    float warm = 0.0f;
    rc = time_once(*inout, &warm);  // sizes the scratch before anything is timed
    for (const Candidate &c : kCands) {
        if (rc) break;
        if (!bp_tile_supported(c.tx, c.ty, c.minb)) continue;
        for (int chunk : kChunks) {
            sarbp_opts o = *inout;
            o.tile_x = c.tx;
            o.tile_y = c.ty;
            o.min_blocks = c.minb;
            o.pulse_chunk = chunk;
            // at 2 CTAs/SM the staging buffer takes the shared memory the
            // third CTA would have had (longer chunks for wide windows):
            // half of 228 KB less 2 KB of reserve and the chunk's records
            // (32 + 128 B per pulse), in 32-byte pairs of halves
            o.stage_cap = c.minb == 2 ? (int)(((228 << 10) / 2 - 2048 - 160 * chunk) / 32) & ~1 : 0;
            float ms = 0.0f;
            rc = time_once(o, &ms);
            if (rc) break;
            trials.push_back({o, ms});
        }
    }
    if (!rc && !trials.empty()) {
        // re-time the three fastest twice more and keep each one's best
        std::sort(trials.begin(), trials.end(), [](const Trial &a, const Trial &b) { return a.ms < b.ms; });
        const size_t top = std::min<size_t>(3, trials.size());
        for (size_t i = 0; i < top && !rc; ++i)
            for (int r = 0; r < 2 && !rc; ++r) {
                float ms = 0.0f;
                rc = time_once(trials[i].o, &ms);
                trials[i].ms = std::min(trials[i].ms, ms);
            }
        std::sort(trials.begin(), trials.begin() + top,
                  [](const Trial &a, const Trial &b) { return a.ms < b.ms; });
    }
    d.timing = timing_was;
    if (rc) return rc;
    if (trials.empty()) return fail(SARBP_ERR_UNSUPPORTED, "no launch shape to tune");
    *inout = trials[0].o;
    if (best_ms) *best_ms = trials[0].ms;
    ctx->tuned[key] = trials[0].o;
    return SARBP_OK;
}

}  // extern "C"
