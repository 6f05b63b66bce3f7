// noalloc.cu -- backprojection of one job without any memory allocation.
//
// Some callers must not allocate device memory at the time they want an
// image: processes whose device memory is handed out up front by a pool or
// an allocator they do not own (a cudaMalloc there fails, or fragments and
// bypasses the pool), and real-time loops that cannot take cudaMalloc's
// latency and its implicit device synchronisation on the path that forms
// each image.  For them this file gives one more entry point,
// sarbp_backprojection_noalloc, that runs the same kernels as
// sarbp_backprojection_device but keeps every scratch array (range-profile
// pairs, windows, pulse table, tile table, per-(tile, pulse) records, final
// phases, descriptors, work list) in one file-scope device array of
// kScratchBytes, whose first kTwiddleBytes hold the FFT twiddle tables of
// every supported N_fft, filled once per device.  No context is created and
// nothing is allocated, on the device or on the host.
//
// Consequences a caller must know:
//  - every GPU on which this library's module is loaded holds the array
//    (64 MiB) until the process exits;
//  - a job whose scratch exceeds the array is rejected (SARBP_ERR_UNSUPPORTED);
//  - all calls share the array: calls that overlap on the GPU (two streams,
//    or two host threads) race and corrupt each other -- serialise them;
//  - the first call on a device looks up the array's device address, sets
//    kernel attributes and fills the twiddle tables (then waits for its
//    stream); make that first call before any stream capture;
//  - the per-device set-up is kept for the life of the process: after a
//    cudaDeviceReset (or any teardown of the primary context) the cached
//    address is stale, so the entry point must not be used again.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "host_math.h"
#include "internal.h"
#include "kernels.h"
#include "runner.h"
#include "sarbp_b200.h"

namespace sarbp {

namespace {

constexpr size_t kScratchBytes = size_t(64) << 20;  // 64 MiB
constexpr int kMaxDevices = 64;

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Fixed offsets of the twiddle tables of logN = kMinLogN..kMaxLogNSmem at the
// start of the scratch (256-byte aligned each).
constexpr size_t twiddle_offset(int logN) {
    size_t o = 0;
    for (int l = kMinLogN; l < logN; ++l) {
        const int N = 1 << l, R0 = 1 << (l % 4);
        size_t n = 0;
        for (int ns = R0 > 1 ? R0 : 16; ns < N; ns *= 16) n += 15 * (size_t)ns;
        o = (o + (n + 1) * 8 + 255) / 256 * 256;  // float2 entries
    }
    return o;
}
constexpr size_t kTwiddleBytes = twiddle_offset(kMaxLogNSmem + 1);

// The scratch.  Host code must not use this symbol as an address: the device
// address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_setup_mutex;
void *g_scratch_addr[kMaxDevices] = {};
int g_num_sms[kMaxDevices] = {};

// Twiddle table of one N (same layout as fill_twiddle_table): for each pass
// with NS > 1, exp(-2 pi i jm r / (NS 16)) at [(r-1) NS + jm].
__global__ void twiddle_kernel(float2 *tw, int logN) {
    const int N = 1 << logN;
    const int R0 = 1 << (logN % 4);
    int ns = R0 > 1 ? R0 : 16, off = 0;
    while (ns < N) {
        for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < 15 * ns; k += gridDim.x * blockDim.x) {
            const int r = k / ns + 1, jm = k % ns;
            const double a = -2.0 * 3.14159265358979323846 * (double)((long long)jm * r) / (double)(ns * 16);
            tw[off + k] = make_float2((float)cos(a), (float)sin(a));
        }
        off += 15 * ns;
        ns *= 16;
    }
}

// Looks up the scratch address on the current device and fills the twiddle
// tables (once per device, on `st`, waiting for it).
int scratch_for_device(int dev, cudaStream_t st, void **addr, int *num_sms) {
    if (dev < 0 || dev >= kMaxDevices) return fail(SARBP_ERR_UNSUPPORTED, "device index too large");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
        int sms = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
        e = init_range_compress_attributes();
        if (e == cudaSuccess) e = init_backproject_attributes();
        if (e != cudaSuccess) return cuda_fail(e, "setting kernel attributes");
        for (int l = kMinLogN; l <= kMaxLogNSmem; ++l)
            twiddle_kernel<<<64, 256, 0, st>>>(reinterpret_cast<float2 *>(static_cast<char *>(p) +
                                                                          twiddle_offset(l)), l);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(e, "no-alloc: filling the twiddle tables");
        g_num_sms[dev] = sms;
        g_scratch_addr[dev] = p;
    }
    *addr = g_scratch_addr[dev];
    *num_sms = g_num_sms[dev];
    return SARBP_OK;
}

__global__ void store_job_kernel(DevJob dj, DevJob *dst) { *dst = dj; }

// work items (0, t, s) for the job's tiles and pulse parts (part 0 of every
// tile first, which the tile-geometry kernel takes as its tile list),
// range-compression rows (0, p), the persistent launch counter and the
// combine kernel's job list
__global__ void init_items_kernel(WorkItem *items, int ntiles, int nitems, RowItem *rows, int npulses,
                                  int *counter, int *split_list) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nitems) items[t] = WorkItem{0, t % ntiles, t / ntiles};
    if (t < npulses) rows[t] = RowItem{0, t};
    if (t == 0) {
        *counter = 0;
        *split_list = 0;
    }
}

__global__ void status_kernel(const JobScalars *sc, int *status) { *status = sc->status; }

}  // namespace

}  // namespace sarbp

using namespace sarbp;

extern "C" int sarbp_backprojection_noalloc(const sarbp_job *job, void *cuda_stream, int *status) {
    if (!job) return fail(SARBP_ERR_INVALID, "job is NULL");
    const sarbp_job &j = *job;
    const int prec = j.precision >= 0 ? j.precision : SARBP_PREC_COMPAT;
    // ---- validation (host only) ----
    auto bad = [](const char *what) { return fail(SARBP_ERR_INVALID, std::string("no-alloc: ") + what); };
    if (j.nsamples < 1 || j.npulses < 1 || j.nu < 1 || j.nv < 1) return bad("sizes must be >= 1");
    if ((long long)j.nu * j.nv > (1ll << 31)) return bad("image larger than 2^31 pixels");
    if (j.n_fft < (1 << kMinLogN) || j.n_fft > (1 << kMaxLogNSmem) || (j.n_fft & (j.n_fft - 1)))
        return fail(SARBP_ERR_UNSUPPORTED, "no-alloc: N_fft must be a power of two in [16, 16384]");
    if (prec != SARBP_PREC_COMPAT && prec != SARBP_PREC_PRECISE)
        return bad("precision must be SARBP_PREC_COMPAT or SARBP_PREC_PRECISE");
    if (j.taylor_s_l < 1 || !std::isfinite(j.delta_r)) return bad("taylor >= 1 and a finite delta_r required");
    if (!j.phs || !j.output_img || !(j.r || (j.u && j.v))) return bad("phs, output_img and pixel positions required");
    if (!j.k_r && !(prec == SARBP_PREC_PRECISE && j.k_r64)) return bad("k_r is NULL");
    if (!j.pos && !(prec == SARBP_PREC_PRECISE && j.pos64)) return bad("pos is NULL");
    if (j.out_u8 && !(j.dB_min < j.dB_max)) return bad("dB_min < dB_max is required for the u8 image");
    DevJob dj;
    std::memset(&dj, 0, sizeof(dj));
    if (j.taylor_mode != SARBP_TAYLOR_REF && j.taylor_mode != SARBP_TAYLOR_FLOAT) return bad("unknown taylor_mode");
    dj.n_taylor = taylor_coefficients_into(j.taylor_s_l, dj.taylor_F, kMaxTaylorTerms, j.taylor_mode);
    if (dj.n_taylor > kMaxTaylorTerms) return bad("taylor side-lobe level too large");
    for (int k = 0; k < dj.n_taylor; ++k)
        if (!std::isfinite(dj.taylor_F[k]))
            return bad("taylor levels above 30 dB have no defined window (use SARBP_TAYLOR_FLOAT)");
    const double lsa = std::floor((double)(-j.nsamples) * j.delta_r / 2);
    const double lsb = std::floor((double)j.nsamples * j.delta_r / 2);
    if (!(lsb > lsa)) return bad("range axis is empty");

    // ---- scratch layout inside the static array ----
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    const BpLaunch L0 = resolved_launch(nullptr, sms);
    const size_t P = (size_t)j.npulses, N = (size_t)j.n_fft, S = (size_t)j.nsamples;
    const int tiles_x = (j.nu + L0.tile_x - 1) / L0.tile_x, tiles_y = (j.nv + L0.tile_y - 1) / L0.tile_y;
    const size_t ntiles = (size_t)tiles_x * tiles_y;
    // the pulse parts of the device entry point, so that both form the same image
    const int nsplit = pulse_parts(j.nu, j.nv, j.npulses, L0, sms);
    const size_t nitems = ntiles * (size_t)nsplit;
    int logN = 0;
    while ((1 << logN) < j.n_fft) ++logN;
    size_t o = kTwiddleBytes;  // the twiddle tables come first
    const size_t o_sc = o;    o = align_up(o + sizeof(JobScalars), 256);
    const size_t o_job = o;   o = align_up(o + sizeof(DevJob), 256);
    const size_t o_items = o; o = align_up(o + nitems * sizeof(WorkItem), 256);
    const size_t o_split = o; o = align_up(o + sizeof(int), 256);
    const size_t o_rows = o;  o = align_up(o + P * sizeof(RowItem), 256);
    const size_t o_cnt = o;   o = align_up(o + sizeof(int), 256);
    const size_t o_qp = o;    o = align_up(o + P * (N + 1) * sizeof(float4), 256);
    const size_t o_filt = o;  o = align_up(o + S * sizeof(float), 256);
    const size_t o_ws = o;    o = align_up(o + S * sizeof(float), 256);
    const size_t o_wp = o;    o = align_up(o + P * sizeof(float), 256);
    const size_t o_pulse = o; o = align_up(o + P * sizeof(double4), 256);
    const size_t o_tiles = o; o = align_up(o + ntiles * sizeof(TileInfo), 256);
    const size_t o_recs = o;  o = align_up(o + ntiles * P * sizeof(PulseRec), 256);
    const size_t o_fin = o;   o = align_up(o + (size_t)j.nu * j.nv * sizeof(float2), 256);
    const size_t o_parts = o; o = align_up(o + (nsplit > 1 ? (size_t)nsplit * j.nu * j.nv * sizeof(float2) : 0), 256);
    if (o > kScratchBytes)
        return fail(SARBP_ERR_UNSUPPORTED,
                    "no-alloc: the job needs " + std::to_string(o >> 20) + " MiB of scratch, more than the " +
                        std::to_string(kScratchBytes >> 20) + " MiB static array");

    void *base = nullptr;
    int num_sms = 0;
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    int rc = scratch_for_device(dev, st, &base, &num_sms);
    if (rc) return rc;
    char *sb = static_cast<char *>(base);

    // ---- descriptor ----
    dj.S = j.nsamples;
    dj.P = j.npulses;
    dj.N = j.n_fft;
    dj.nu = j.nu;
    dj.nv = j.nv;
    dj.precision = prec;
    dj.tile_x = L0.tile_x;
    dj.tile_y = L0.tile_y;
    dj.tiles_x = tiles_x;
    dj.tiles_y = tiles_y;
    dj.logN = logN;
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
    dj.Q = nullptr;
    dj.Qp = reinterpret_cast<float4 *>(sb + o_qp);
    dj.filt = reinterpret_cast<float *>(sb + o_filt);
    dj.wS = reinterpret_cast<float *>(sb + o_ws);
    dj.wP = reinterpret_cast<float *>(sb + o_wp);
    dj.pulse = reinterpret_cast<double4 *>(sb + o_pulse);
    dj.tiles = reinterpret_cast<TileInfo *>(sb + o_tiles);
    dj.recs = reinterpret_cast<PulseRec *>(sb + o_recs);
    dj.fin = reinterpret_cast<float2 *>(sb + o_fin);
    dj.sc = reinterpret_cast<JobScalars *>(sb + o_sc);
    dj.delta_r = j.delta_r;
    dj.lsa = lsa;
    dj.lsr = (lsb - lsa) / (double)(j.n_fft - 1);
    dj.inv_lsr = 1.0 / dj.lsr;
    dj.out = reinterpret_cast<double2 *>(j.output_img);
    dj.out_u8 = j.out_u8;
    dj.dB_min = j.dB_min;
    dj.dB_max = j.dB_max;
    dj.nsplit = nsplit;
    dj.parts = nsplit > 1 ? reinterpret_cast<float2 *>(sb + o_parts) : nullptr;

    DevJob *d_job = reinterpret_cast<DevJob *>(sb + o_job);
    WorkItem *d_items = reinterpret_cast<WorkItem *>(sb + o_items);
    int *d_cnt = reinterpret_cast<int *>(sb + o_cnt);
    const float2 *d_tw = reinterpret_cast<const float2 *>(sb + twiddle_offset(logN));
    RowItem *d_rows = reinterpret_cast<RowItem *>(sb + o_rows);
    int *d_split = reinterpret_cast<int *>(sb + o_split);

    // ---- launches (the prep kernel clears the job's scalars) ----
    store_job_kernel<<<1, 1, 0, st>>>(dj, d_job);
    const size_t nfill = nitems > P ? nitems : P;
    init_items_kernel<<<(int)((nfill + 255) / 256), 256, 0, st>>>(d_items, (int)ntiles, (int)nitems, d_rows,
                                                                  j.npulses, d_cnt, d_split);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "no-alloc set-up launches");
    launch_prep(d_job, 1, st);
    e = launch_range_compress(logN, d_job, d_rows, j.npulses, 1, d_tw, st);
    if (e == cudaSuccess) e = launch_tile_setup(d_job, d_items, (int)ntiles, L0.tile_x * L0.tile_y, st);
    if (e != cudaSuccess) return cuda_fail(e, "no-alloc range compression / geometry launch");
    BpLaunch L = L0;
    const int occ = bp_max_active_blocks(L);
    if (occ < 1) return fail(SARBP_ERR_CUDA, "no-alloc: backprojection kernel does not fit on an SM");
    L.grid = (int)std::min<long long>((long long)occ * num_sms, (long long)nitems);
    e = launch_backproject(L, d_job, d_items, (int)nitems, d_cnt, st);
    if (e == cudaSuccess && nsplit > 1) e = launch_combine_parts(d_job, d_split, 1, (long long)j.nu * j.nv, num_sms, st);
    if (e == cudaSuccess && j.out_u8) e = launch_batch_u8(d_job, 1, (long long)j.nu * j.nv, st);
    if (e == cudaSuccess && status) {
        status_kernel<<<1, 1, 0, st>>>(dj.sc, status);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return cuda_fail(e, "no-alloc backprojection launch");
    return SARBP_OK;
}
