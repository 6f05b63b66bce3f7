// api.cpp -- the extern "C" entry points of include/sarbp_b200.h.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "context.h"
#include "host_math.h"
#include "kernels.h"
#include "runner.h"
#include "sarbp_b200.h"

namespace sarbp {
const char *last_error_cstr();
}

using namespace sarbp;

int sarbp::ctx_set_device(sarbp_ctx *ctx) {
    if (!ctx) return fail(SARBP_ERR_INVALID, "context is NULL");
    cudaError_t e = cudaSetDevice(ctx->dev.device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    return SARBP_OK;
}

namespace {

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

int set_device(sarbp_ctx *ctx) { return ctx_set_device(ctx); }

// An image plane given by its axes instead of pixel_locs: pixel (i, j) sits
// at u_hat * u[i] + v_hat * v[j] (img_plane.cpp:92-102), formed on the device.
struct PlaneAxes {
    const double *u, *v, *u_hat, *v_hat;
};

// Row slabs for a host-buffer call on one image of 2^18 pixels or more, so
// that the positions go up and the image comes down slab by slab while
// other slabs compute: row0[0..nslabs] are tile-row boundaries.  The first
// slab is small (1/32 of the tile rows) so that backprojection starts once
// the phase history and a few position rows are up, the second twice that,
// the last as small as the first so that little of the image is still to
// come down when the kernels end; the rest in equal slabs of at least 8
// tile rows, at most kMaxSlabs slabs in all.  None when the caller asked for
// pulse parts (slabs run one item per tile).
void slab_plan(const sarbp_opts *opts, int precision, int nu, int nv, int *tile_x, int *tile_y,
               int *nslabs, int (&row0)[sarbp_ctx::kMaxSlabs + 1]) {
    Runner::tile_shape(opts, tile_x, tile_y);
    const int tiles_y = (nv + *tile_y - 1) / *tile_y;
    *nslabs = 0;
    if (precision == SARBP_PREC_NAIVE || (size_t)nu * nv < ((size_t)1 << 18) || tiles_y < 16) return;
    if (opts && opts->pulse_parts >= 2) return;
    const int h0 = std::max(1, tiles_y / 32);
    const int rest = tiles_y - 4 * h0;  // after the first, second and last slabs
    const int nbody = std::max(1, std::min(sarbp_ctx::kMaxSlabs - 3, rest / 8));
    const int hb = (rest + nbody - 1) / nbody;
    int n = 0, y = 0;
    row0[n++] = 0;
    row0[n++] = y += h0;
    row0[n++] = y += 2 * h0;
    for (int b = 0; b < nbody && y < tiles_y - h0; ++b) row0[n++] = y = std::min(tiles_y - h0, y + hb);
    row0[n++] = tiles_y;
    *nslabs = n - 1;
}

// Copies host arrays to one device block, runs one job, copies the image back.
int run_host_job(sarbp_ctx *ctx, const float *phs, int S, int P, const float *k_r32,
                 const double *k_r64, int taylor, int n_fft, double delta_r, int nu, int nv,
                 const float *pos32, const double *pos64, const double *r, double *out,
                 const sarbp_opts *opts, int precision, const PlaneAxes *plane = nullptr) {
    int rc = set_device(ctx);
    if (rc) return rc;
    if (!phs || !out) return fail(SARBP_ERR_INVALID, "phs and output_img must be non-NULL");
    if (!r && !(plane && plane->u && plane->v && plane->u_hat && plane->v_hat))
        return fail(SARBP_ERR_INVALID, "r (pixel_locs) must be non-NULL");
    if (S < 1 || P < 1 || nu < 1 || nv < 1) return fail(SARBP_ERR_INVALID, "sizes must be >= 1");
    const size_t npix = (size_t)nu * nv;
    const size_t b_phs = align256((size_t)S * P * 2 * sizeof(float));
    const size_t b_k32 = k_r32 ? align256((size_t)S * sizeof(float)) : 0;
    const size_t b_k64 = k_r64 ? align256((size_t)S * sizeof(double)) : 0;
    const size_t b_p32 = pos32 ? align256((size_t)P * 3 * sizeof(float)) : 0;
    const size_t b_p64 = pos64 ? align256((size_t)P * 3 * sizeof(double)) : 0;
    const size_t b_r = r ? align256(npix * 3 * sizeof(double)) : 0;
    const size_t b_u = r ? 0 : align256((size_t)nu * sizeof(double));
    const size_t b_v = r ? 0 : align256((size_t)nv * sizeof(double));
    const size_t b_out = align256(npix * 2 * sizeof(double));
    const size_t total = b_phs + b_k32 + b_k64 + b_p32 + b_p64 + b_r + b_u + b_v + b_out;
    cudaError_t e = ctx->io.ensure(total, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "allocating device inputs");
    char *base = static_cast<char *>(ctx->io.ptr);
    size_t o = 0;
    float *d_phs = reinterpret_cast<float *>(base + o); o += b_phs;
    float *d_k32 = k_r32 ? reinterpret_cast<float *>(base + o) : nullptr; o += b_k32;
    double *d_k64 = k_r64 ? reinterpret_cast<double *>(base + o) : nullptr; o += b_k64;
    float *d_p32 = pos32 ? reinterpret_cast<float *>(base + o) : nullptr; o += b_p32;
    double *d_p64 = pos64 ? reinterpret_cast<double *>(base + o) : nullptr; o += b_p64;
    double *d_r = r ? reinterpret_cast<double *>(base + o) : nullptr; o += b_r;
    double *d_u = r ? nullptr : reinterpret_cast<double *>(base + o); o += b_u;
    double *d_v = r ? nullptr : reinterpret_cast<double *>(base + o); o += b_v;
    double *d_out = reinterpret_cast<double *>(base + o);
    cudaStream_t st = ctx->stream;
    // Row slabs: the pixel positions go up and the image comes down slab by
    // slab while other slabs compute (images of 2^18 pixels and more).
    int tile_x = 0, tile_y = 0, nslabs = 0, row0[sarbp_ctx::kMaxSlabs + 1] = {};
    slab_plan(opts, precision, nu, nv, &tile_x, &tile_y, &nslabs, row0);
    cudaStream_t cin = nslabs ? ctx->copy_in : st;
    struct Copy { void *dst; const void *src; size_t n; };
    const Copy copies[] = {
        {d_phs, phs, (size_t)S * P * 2 * sizeof(float)},
        {d_k32, k_r32, (size_t)S * sizeof(float)},
        {d_k64, k_r64, (size_t)S * sizeof(double)},
        {d_p32, pos32, (size_t)P * 3 * sizeof(float)},
        {d_p64, pos64, (size_t)P * 3 * sizeof(double)},
        {d_r, nslabs ? nullptr : r, npix * 3 * sizeof(double)},
        {d_u, r ? nullptr : plane->u, (size_t)nu * sizeof(double)},
        {d_v, r ? nullptr : plane->v, (size_t)nv * sizeof(double)},
    };
    for (const Copy &c : copies) {
        if (!c.src) continue;
        e = cudaMemcpyAsync(c.dst, c.src, c.n, cudaMemcpyHostToDevice, cin);
        if (e != cudaSuccess) return cuda_fail(e, "copying inputs to the device");
    }
    SlabSpec spec;
    if (nslabs) {
        spec.copy_stream = cin;  // descriptors after the phase history, before the positions
        // the pixel positions go up slab by slab once the batch's descriptors
        // and range compression are enqueued (see SlabSpec::before_slabs)
        spec.before_slabs = [&]() -> cudaError_t {
            for (int g = 0; g < nslabs && r; ++g) {
                const size_t y0 = std::min((size_t)nv, (size_t)row0[g] * tile_y);
                const size_t y1 = std::min((size_t)nv, (size_t)row0[g + 1] * tile_y);
                for (int c = 0; c < 3 && y1 > y0; ++c) {
                    const size_t off = (size_t)c * npix + y0 * (size_t)nu;
                    cudaError_t ce = cudaMemcpyAsync(d_r + off, r + off, (y1 - y0) * (size_t)nu * sizeof(double),
                                                     cudaMemcpyHostToDevice, cin);
                    if (ce != cudaSuccess) return ce;
                }
                cudaError_t ce = cudaEventRecord(ctx->ev_ready[g], cin);
                if (ce != cudaSuccess) return ce;
            }
            return cudaSuccess;
        };
        spec.nslabs = nslabs;
        spec.row0 = row0;
        spec.aux = ctx->aux;
        spec.ready = r ? ctx->ev_ready : nullptr;
        spec.done = ctx->ev_done;
    }
    sarbp_job j;
    std::memset(&j, 0, sizeof(j));
    j.nsamples = S;
    j.npulses = P;
    j.n_fft = n_fft;
    j.taylor_s_l = taylor;
    j.nu = nu;
    j.nv = nv;
    j.delta_r = delta_r;
    j.phs = d_phs;
    j.k_r = d_k32;
    j.k_r64 = d_k64;
    j.pos = d_p32;
    j.pos64 = d_p64;
    j.r = d_r;
    if (!r) {
        j.u = d_u;
        j.v = d_v;
        for (int d = 0; d < 3; ++d) {
            j.u_hat[d] = plane->u_hat[d];
            j.v_hat[d] = plane->v_hat[d];
        }
    }
    j.output_img = d_out;
    j.precision = precision;
    rc = ctx->runner->enqueue(&j, 1, opts, st, nullptr, false, nslabs ? &spec : nullptr);
    if (rc) {
        // the copies may still read the caller's buffers
        cudaStreamSynchronize(cin);
        return rc;
    }
    if (!nslabs) {
        e = cudaMemcpyAsync(out, d_out, npix * 2 * sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) return cuda_fail(e, "copying the image to the host");
        return ctx->runner->check_status(st);
    }
    // output rows are flipped (backprojection.cpp:130): pixel rows [y0, y1)
    // are image rows [nv - y1, nv - y0)
    for (int g = 0; g < nslabs; ++g) {
        const size_t y0 = std::min((size_t)nv, (size_t)row0[g] * tile_y);
        const size_t y1 = std::min((size_t)nv, (size_t)row0[g + 1] * tile_y);
        if ((e = cudaStreamWaitEvent(ctx->copy_out, ctx->ev_done[g], 0)) != cudaSuccess)
            return cuda_fail(e, "cudaStreamWaitEvent");
        const size_t off = ((size_t)nv - y1) * (size_t)nu * 2;
        e = cudaMemcpyAsync(out + off, d_out + off, (y1 - y0) * (size_t)nu * 2 * sizeof(double),
                            cudaMemcpyDeviceToHost, ctx->copy_out);
        if (e != cudaSuccess) return cuda_fail(e, "copying the image to the host");
    }
    if ((e = cudaEventRecord(ctx->ev_out, ctx->copy_out)) != cudaSuccess ||
        (e = cudaStreamWaitEvent(st, ctx->ev_out, 0)) != cudaSuccess)
        return cuda_fail(e, "ordering output copies");
    return ctx->runner->check_status(st);
}

int effective_precision(const sarbp_opts *opts, int dflt) {
    return opts ? opts->precision : dflt;
}

}  // namespace

extern "C" {

const char *sarbp_last_error(void) { return last_error_cstr(); }
const char *sarbp_version(void) { return "sarbp_b200 0.1 (sm_100a)"; }

int sarbp_ctx_create(int device, sarbp_ctx **out) {
    if (!out) return fail(SARBP_ERR_INVALID, "out is NULL");
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceCount");
    if (device < 0 || device >= ndev)
        return fail(SARBP_ERR_INVALID, "device " + std::to_string(device) + " out of range");
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    cudaDeviceProp prop;
    e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceProperties");
    if (prop.major < 10)
        return fail(SARBP_ERR_UNSUPPORTED, std::string("device is sm_") + std::to_string(prop.major) +
                                               std::to_string(prop.minor) +
                                               "; this build targets sm_100a (B200)");
    e = init_range_compress_attributes();
    if (e == cudaSuccess) e = init_backproject_attributes();
    if (e != cudaSuccess) return cuda_fail(e, "setting kernel attributes");
    auto *ctx = new sarbp_ctx();
    ctx->dev.device = device;
    ctx->dev.num_sms = prop.multiProcessorCount;
    ctx->runner.reset(new Runner(&ctx->dev));
    e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete ctx;
        return cuda_fail(e, "cudaStreamCreate");
    }
    ctx->stream = ctx->own_stream;
    for (cudaStream_t *sp : {&ctx->copy_in, &ctx->aux, &ctx->copy_out})
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(sp, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_out, cudaEventDisableTiming);
    for (int g = 0; g < sarbp_ctx::kMaxSlabs && e == cudaSuccess; ++g) {
        e = cudaEventCreateWithFlags(&ctx->ev_ready[g], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_done[g], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        sarbp_ctx_destroy(ctx);
        return cuda_fail(e, "creating streams and events");
    }
    *out = ctx;
    return SARBP_OK;
}

int sarbp_ctx_destroy(sarbp_ctx *ctx) {
    if (!ctx) return SARBP_OK;
    cudaSetDevice(ctx->dev.device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    ctx->runner.reset();
    ctx->io.release();
    ctx->out_aux.release();
    ctx->resize_buf.release();
    ctx->dev.release();
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    for (cudaStream_t sp : {ctx->copy_in, ctx->aux, ctx->copy_out})
        if (sp) cudaStreamDestroy(sp);
    if (ctx->ev_out) cudaEventDestroy(ctx->ev_out);
    for (int g = 0; g < sarbp_ctx::kMaxSlabs; ++g) {
        if (ctx->ev_ready[g]) cudaEventDestroy(ctx->ev_ready[g]);
        if (ctx->ev_done[g]) cudaEventDestroy(ctx->ev_done[g]);
    }
    delete ctx;
    return SARBP_OK;
}

int sarbp_ctx_set_stream(sarbp_ctx *ctx, void *cuda_stream) {
    int rc = set_device(ctx);
    if (rc) return rc;
    ctx->stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : ctx->own_stream;
    return SARBP_OK;
}

void *sarbp_ctx_stream(sarbp_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int sarbp_ctx_synchronize(sarbp_ctx *ctx) {
    int rc = set_device(ctx);
    if (rc) return rc;
    return ctx->runner->check_status(ctx->stream);
}

long long sarbp_ctx_launch_count(sarbp_ctx *ctx) { return ctx ? ctx->dev.launches.load() : -1; }

int sarbp_ctx_set_timing(sarbp_ctx *ctx, int on) {
    int rc = set_device(ctx);
    if (rc) return rc;
    ctx->dev.timing = on != 0;
    return SARBP_OK;
}

int sarbp_ctx_last_stage_ms(sarbp_ctx *ctx, float *ms5) {
    int rc = set_device(ctx);
    if (rc) return rc;
    if (!ms5) return fail(SARBP_ERR_INVALID, "ms5 is NULL");
    DeviceInfo &d = ctx->dev;
    constexpr int kStages = DeviceInfo::kEvents - 1;
    for (int i = 0; i < kStages; ++i) ms5[i] = -1.0f;
    if (!d.ev_recorded[0]) return fail(SARBP_ERR_STATE, "no timed batch (enable sarbp_ctx_set_timing)");
    for (int i = 0; i < DeviceInfo::kEvents; ++i)
        if (d.ev_recorded[i]) {
            cudaError_t e = cudaEventSynchronize(d.ev[i]);
            if (e != cudaSuccess) return cuda_fail(e, "cudaEventSynchronize");
        }
    for (int i = 0; i < kStages; ++i)
        if (d.ev_recorded[i] && d.ev_recorded[i + 1]) {
            cudaError_t e = cudaEventElapsedTime(&ms5[i], d.ev[i], d.ev[i + 1]);
            if (e != cudaSuccess) return cuda_fail(e, "cudaEventElapsedTime");
        }
    return SARBP_OK;
}

int sarbp_measure_peaks(sarbp_ctx *ctx, double *ffma_per_s, double *mufu_per_s) {
    int rc = set_device(ctx);
    if (rc) return rc;
    if (!ffma_per_s || !mufu_per_s) return fail(SARBP_ERR_INVALID, "outputs are NULL");
    cudaError_t e = measure_peaks(ctx->dev.num_sms, ctx->stream, ffma_per_s, mufu_per_s);
    if (e != cudaSuccess) return cuda_fail(e, "peak microkernels");
    ctx->dev.launches += 8;
    return SARBP_OK;
}

int sarbp_backprojection(sarbp_ctx *ctx, const float *phs, int nsamples, int npulses,
                         const float *k_r, int taylor_s_l, int n_fft, double delta_r,
                         const double *u, int nu, const double *v, int nv, const float *pos,
                         const double *r, double *output_img, const sarbp_opts *opts) {
    (void)u;
    (void)v;  // the reference reads only their extents (backprojection.cpp:71-72)
    if (!k_r || !pos) return fail(SARBP_ERR_INVALID, "k_r and pos must be non-NULL");
    return run_host_job(ctx, phs, nsamples, npulses, k_r, nullptr, taylor_s_l, n_fft, delta_r, nu,
                        nv, pos, nullptr, r, output_img, opts,
                        effective_precision(opts, SARBP_PREC_COMPAT));
}

int sarbp_backprojection_plane(sarbp_ctx *ctx, const float *phs, int nsamples, int npulses,
                               const float *k_r, int taylor_s_l, int n_fft, double delta_r,
                               const double *u, int nu, const double *v, int nv,
                               const double u_hat[3], const double v_hat[3], const float *pos,
                               double *output_img, const sarbp_opts *opts) {
    if (!k_r || !pos) return fail(SARBP_ERR_INVALID, "k_r and pos must be non-NULL");
    if (!u || !v || !u_hat || !v_hat)
        return fail(SARBP_ERR_INVALID, "u, v, u_hat and v_hat must be non-NULL");
    const PlaneAxes plane{u, v, u_hat, v_hat};
    return run_host_job(ctx, phs, nsamples, npulses, k_r, nullptr, taylor_s_l, n_fft, delta_r, nu,
                        nv, pos, nullptr, nullptr, output_img, opts,
                        effective_precision(opts, SARBP_PREC_COMPAT), &plane);
}

int sarbp_backprojection_f64(sarbp_ctx *ctx, const float *phs, int nsamples, int npulses,
                             const double *k_r, int taylor_s_l, int n_fft, double delta_r,
                             const double *u, int nu, const double *v, int nv, const double *pos,
                             const double *r, double *output_img, const sarbp_opts *opts) {
    (void)u;
    (void)v;
    if (!k_r || !pos) return fail(SARBP_ERR_INVALID, "k_r and pos must be non-NULL");
    if (nsamples < 1 || npulses < 1) return fail(SARBP_ERR_INVALID, "sizes must be >= 1");
    const int prec = effective_precision(opts, SARBP_PREC_PRECISE);
    if (prec == SARBP_PREC_PRECISE)
        return run_host_job(ctx, phs, nsamples, npulses, nullptr, k_r, taylor_s_l, n_fft, delta_r,
                            nu, nv, nullptr, pos, r, output_img, opts, prec);
    // f32 semantics from f64 inputs: the loader's downcast (PlatformData.cpp:138-149, :219-231)
    std::vector<float> k32(nsamples), p32((size_t)npulses * 3);
    for (int i = 0; i < nsamples; ++i) k32[i] = (float)k_r[i];
    for (size_t i = 0; i < p32.size(); ++i) p32[i] = (float)pos[i];
    return run_host_job(ctx, phs, nsamples, npulses, k32.data(), nullptr, taylor_s_l, n_fft, delta_r,
                        nu, nv, p32.data(), nullptr, r, output_img, opts, prec);
}

int sarbp_backprojection_device(sarbp_ctx *ctx, const sarbp_job *job, const sarbp_opts *opts) {
    int rc = set_device(ctx);
    if (rc) return rc;
    // one persistent launch: row slabs (as the host-buffer calls use to
    // overlap their copies) measured 1 % slower with the inputs resident
    return ctx->runner->enqueue(job, 1, opts, ctx->stream);
}

int sarbp_range_compress_device(sarbp_ctx *ctx, const sarbp_job *job, const sarbp_opts *opts,
                                float *q_out) {
    int rc = set_device(ctx);
    if (rc) return rc;
    if (!q_out) return fail(SARBP_ERR_INVALID, "q_out is NULL");
    return ctx->runner->enqueue(job, 1, opts, ctx->stream, q_out);
}

int sarbp_batch_device(sarbp_ctx *ctx, const sarbp_job *jobs, int njobs, const sarbp_opts *opts) {
    int rc = set_device(ctx);
    if (rc) return rc;
    return ctx->runner->enqueue(jobs, njobs, opts, ctx->stream);
}

int sarbp_img_output_to_dB_device(sarbp_ctx *ctx, const double *img, int nu, int nv, double *dB) {
    int rc = set_device(ctx);
    if (rc) return rc;
    if (!img || !dB || nu < 1 || nv < 1) return fail(SARBP_ERR_INVALID, "bad dB arguments");
    cudaError_t e = ctx->out_aux.ensure(256, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "allocating");
    auto *m = static_cast<unsigned long long *>(ctx->out_aux.ptr);
    e = cudaMemsetAsync(m, 0, sizeof(unsigned long long), ctx->stream);
    if (e == cudaSuccess) e = launch_maxabs(reinterpret_cast<const double2 *>(img), (long long)nu * nv, m, ctx->stream);
    if (e == cudaSuccess)
        e = launch_db_u8(reinterpret_cast<const double2 *>(img), (long long)nu * nv, m, dB, nullptr, 0, 1,
                         ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "dB launch");
    ctx->dev.launches += 2;
    return SARBP_OK;
}

int sarbp_img_output_u8_device(sarbp_ctx *ctx, const double *dB, int nu, int nv, double dB_min,
                               double dB_max, uint8_t *out) {
    int rc = set_device(ctx);
    if (rc) return rc;
    if (!dB || !out || nu < 1 || nv < 1) return fail(SARBP_ERR_INVALID, "bad u8 arguments");
    if (!(dB_min < dB_max)) return fail(SARBP_ERR_INVALID, "Constraint failed: dB_min < dB_max");
    cudaError_t e = launch_u8_from_db(dB, (long long)nu * nv, dB_min, dB_max, out, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "u8 launch");
    ctx->dev.launches += 1;
    return SARBP_OK;
}

int sarbp_img_output_u8_from_img_device(sarbp_ctx *ctx, const double *img, int nu, int nv,
                                        double dB_min, double dB_max, uint8_t *out) {
    int rc = set_device(ctx);
    if (rc) return rc;
    if (!img || !out || nu < 1 || nv < 1) return fail(SARBP_ERR_INVALID, "bad u8 arguments");
    if (!(dB_min < dB_max)) return fail(SARBP_ERR_INVALID, "Constraint failed: dB_min < dB_max");
    cudaError_t e = ctx->out_aux.ensure(256, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "allocating");
    auto *m = static_cast<unsigned long long *>(ctx->out_aux.ptr);
    const long long n = (long long)nu * nv;
    e = cudaMemsetAsync(m, 0, sizeof(unsigned long long), ctx->stream);
    if (e == cudaSuccess) e = launch_maxabs(reinterpret_cast<const double2 *>(img), n, m, ctx->stream);
    if (e == cudaSuccess)
        e = launch_img_u8(reinterpret_cast<const double2 *>(img), n, m, out, dB_min, dB_max, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "u8 launch");
    ctx->dev.launches += 2;
    return SARBP_OK;
}

int sarbp_img_output_to_dB(sarbp_ctx *ctx, const double *img, int nu, int nv, double *dB) {
    int rc = set_device(ctx);
    if (rc) return rc;
    if (!img || !dB || nu < 1 || nv < 1) return fail(SARBP_ERR_INVALID, "bad dB arguments");
    const size_t n = (size_t)nu * nv;
    cudaError_t e = ctx->io.ensure(align256(n * 16) + align256(n * 8), ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "allocating");
    double *d_img = static_cast<double *>(ctx->io.ptr);
    double *d_db = reinterpret_cast<double *>(static_cast<char *>(ctx->io.ptr) + align256(n * 16));
    e = cudaMemcpyAsync(d_img, img, n * 16, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "copy");
    rc = sarbp_img_output_to_dB_device(ctx, d_img, nu, nv, d_db);
    if (rc) return rc;
    e = cudaMemcpyAsync(dB, d_db, n * 8, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "copy");
    return SARBP_OK;
}

int sarbp_img_output_u8(sarbp_ctx *ctx, const double *dB, int nu, int nv, double dB_min,
                        double dB_max, uint8_t *out) {
    int rc = set_device(ctx);
    if (rc) return rc;
    if (!dB || !out || nu < 1 || nv < 1) return fail(SARBP_ERR_INVALID, "bad u8 arguments");
    if (!(dB_min < dB_max)) return fail(SARBP_ERR_INVALID, "Constraint failed: dB_min < dB_max");
    const size_t n = (size_t)nu * nv;
    cudaError_t e = ctx->io.ensure(align256(n * 8) + align256(n), ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "allocating");
    double *d_db = static_cast<double *>(ctx->io.ptr);
    uint8_t *d_u8 = static_cast<uint8_t *>(ctx->io.ptr) + align256(n * 8);
    e = cudaMemcpyAsync(d_db, dB, n * 8, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "copy");
    rc = sarbp_img_output_u8_device(ctx, d_db, nu, nv, dB_min, dB_max, d_u8);
    if (rc) return rc;
    e = cudaMemcpyAsync(out, d_u8, n, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "copy");
    return SARBP_OK;
}

int sarbp_taylor(int num, double S_L, double *out) {
    if (num < 2 || !out) return fail(SARBP_ERR_INVALID, "taylor: num >= 2 and out required");
    if (!(S_L >= 1.0)) return fail(SARBP_ERR_INVALID, "taylor: S_L >= 1 required");
    taylor_window(num, S_L, out);
    return SARBP_OK;
}

int sarbp_taylor_mode(int num, double S_L, int mode, double *out) {
    if (mode != SARBP_TAYLOR_REF && mode != SARBP_TAYLOR_FLOAT) return fail(SARBP_ERR_INVALID, "taylor: unknown mode");
    if (num < 2 || !out) return fail(SARBP_ERR_INVALID, "taylor: num >= 2 and out required");
    if (!(S_L >= 1.0)) return fail(SARBP_ERR_INVALID, "taylor: S_L >= 1 required");
    taylor_window(num, S_L, out, mode);
    return SARBP_OK;
}

int sarbp_img_plane_dims(int nsamples, int npulses, int upsample, int *nu, int *nv) {
    if (nsamples < 1 || npulses < 1 || !nu || !nv) return fail(SARBP_ERR_INVALID, "bad sizes");
    *nu = upsample ? ip_upsample(nsamples) : nsamples;
    *nv = upsample ? ip_upsample(npulses) : npulses;
    return SARBP_OK;
}

int sarbp_img_plane(int nsamples, int npulses, double delta_r, const float *R_c,
                    const float *n_hat, double res_factor, double aspect, int upsample,
                    double *d_u, double *d_v, double *u, double *v, double *k_u, double *k_v,
                    double *u_hat, double *v_hat, double *pl) {
    if (nsamples < 1 || npulses < 1 || !R_c) return fail(SARBP_ERR_INVALID, "bad image-plane inputs");
    static const float kNHat[3] = {0, 0, 1};  // ImgPlane.h:35
    ImgPlane ip = img_plane_create(nsamples, npulses, delta_r, R_c, n_hat ? n_hat : kNHat,
                                   res_factor, aspect, upsample != 0);
    if (d_u) *d_u = ip.d_u;
    if (d_v) *d_v = ip.d_v;
    if (u) std::memcpy(u, ip.u.data(), ip.u.size() * sizeof(double));
    if (v) std::memcpy(v, ip.v.data(), ip.v.size() * sizeof(double));
    if (k_u) std::memcpy(k_u, ip.k_u.data(), ip.k_u.size() * sizeof(double));
    if (k_v) std::memcpy(k_v, ip.k_v.data(), ip.k_v.size() * sizeof(double));
    if (u_hat) std::memcpy(u_hat, ip.u_hat, sizeof(ip.u_hat));
    if (v_hat) std::memcpy(v_hat, ip.v_hat, sizeof(ip.v_hat));
    if (pl) pixel_locs(ip, pl);
    return SARBP_OK;
}

}  // extern "C"
