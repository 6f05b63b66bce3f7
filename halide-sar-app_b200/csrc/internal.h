// internal.h -- descriptors shared by the host pipeline and the kernels.
//
// One DevJob describes one image-formation job in device memory: the
// caller's inputs, the library's per-job scratch (range profiles, windows,
// per-pulse and per-tile geometry) and the outputs.  The host builds an
// array of them, copies it to the device, and every kernel of a batch
// indexes it by job.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sarbp {

constexpr int kMaxTaylorTerms = 64;  // n_bar - 1 <= 64  (S_L up to ~150 dB)
constexpr int kMinLogN = 4;          // N_fft in [16, 131072]
constexpr int kMaxLogN = 17;
constexpr int kMaxLogNSmem = 14;     // up to here one CTA holds a whole row

// status bits written by kernels into JobScalars::status
constexpr int kStatusTileTooWide = 1;   // range window of a tile exceeds smem
constexpr int kStatusNonFinite = 2;     // non-finite pixel or pulse geometry
constexpr int kStatusNearField = 4;     // pulse closer than the tile radius
constexpr int kStatusTimeout = 8;       // a bounded wait on an async copy gave up

// per-job words the kernels write; kept contiguous for one status read-back
struct JobScalars {
    unsigned long long maxabs;  // bits of max |z| (f64, non-negative)
    double k_c;                 // k_r[S/2] by precision mode (prep kernel)
    int status;                 // kStatus* bits
    int pad[3];
    // prep kernel, f64: an orthonormal frame E of the job's image plane
    // (rows; the grid axes, or the first pixels of r), and over the job's
    // antenna positions max |pos . E_i| / |pos| and min |pos|, which bound
    // the tiles' line-of-sight components and so their range windows
    double frame[3][3];
    double los_abs[3];
    double pos_min;
};

// Tiles wider than this many radians of k_c * (half-diagonal) are "wide":
// FP32 rounding of w_hat . d (about |d| * 2^-24) would exceed the phase
// budget, so the linear phase toward a reference direction w0 is taken out
// of the pulse loop and applied in f64 through the final phase.
constexpr double kWideRad = 1024.0;
constexpr int kOrderInvalid = 7;

// Geometry of one pixel tile (tile-set-up kernel -> backprojection).
struct __align__(16) TileInfo {
    double rc[3];  // centre of the tile's bounding box
    float rho;     // max |r - rc| over the tile, padded (m)
    int K;         // range window half-width (bins): W = 2K + 1
    int planar;    // 1 when every pixel has r.z == rc.z
    int wide;      // 1: records hold w_hat - w0, fin carries exp(-j w0 . d)
    float w0[3];   // unit direction from rc to the mid-aperture antenna (wide tiles)
    int transposed;  // 1: consumer lanes run along y (square tiles; see tile set-up)
};

// Per-(tile, pulse) constants (tile geometry kernel -> backprojection):
//   a = (w_hat.x, w_hat.y, w_hat.z, e = 1/(2 k_c R)); wide tiles: w_hat - w0
//   b = (c0 - theta*inv_lsr/k_c, theta, k_c R, int bits: 8*base + series order)
// series order 0..3 (see the backprojection kernel); kOrderInvalid marks a
// pulse that contributes nothing (non-finite geometry).
struct __align__(16) PulseRec {
    float4 a;
    float4 b;
};

struct DevJob {
    // sizes
    int S, P, N, nu, nv;
    int precision;
    int tiles_x, tiles_y;
    int tile_x, tile_y;
    int logN;
    int n_taylor;  // n_bar - 1 coefficients (same for both axes)
    // caller inputs (device)
    const float2 *phs;    // [P][S]
    const float *k_r32;   // [S]
    const double *k_r64;  // [S] or null
    const float *pos32;   // [P][3]
    const double *pos64;  // [P][3] or null
    const double *r;      // SoA [3][nu*nv] or null (grid form)
    const double *u, *v;  // grid form
    double uh[3], vh[3];
    // library scratch (device)
    float2 *Q;            // [P][N] range profiles (only when Qp is null)
    float4 *Qp;           // [P][N+1] interpolation pairs (m, d) + (Q[0], 0) at N
    float *filt;          // [S]  |k_r|
    float *wS;            // [S]  sample window
    float *wP;            // [P]  pulse window
    double4 *pulse;       // [P]  (x, y, z, |pos|) by precision mode
    TileInfo *tiles;      // [tiles_x * tiles_y]
    PulseRec *recs;       // [tiles][P]
    float2 *fin;          // [nv][nu] exp(+j k_c dr(pixel, P/2)), r-space order
    JobScalars *sc;       // max|z|, k_c, status (written by the kernels)
    // constants
    double delta_r, lsa, lsr, inv_lsr;
    double taylor_F[kMaxTaylorTerms];
    // outputs
    double2 *out;         // [nv][nu]
    uint8_t *out_u8;      // [nv][nu] or null
    double dB_min, dB_max;
    // pulse-chunked jobs: the descriptor of one chunk has P = the chunk's
    // pulses, phs its phase-history rows in order (no fftshift rotation:
    // wP and pulse are the chunk's gathered window and pulse table), and
    // the backprojection adds its sums into acc instead of writing out
    int chunked;
    float2 *acc;          // [nv][nu] partial image (pixel-row order) or null
    // pulse parts: a job whose tiles leave resident CTAs idle has each tile
    // formed as nsplit items over consecutive pulse ranges (part_range);
    // each item stores its sums into slice `part` of parts ([nsplit][nv][nu],
    // pixel-row order), and the combine kernel adds the slices in order and
    // applies the final phase.  nsplit <= 1: one item per tile.
    int nsplit;
    float2 *parts;
};

// (job, tile, pulse part) work item of the per-tile kernels
struct WorkItem {
    int job;
    int tile;
    int part;  // 0 .. nsplit - 1 (0 for the tile-geometry kernels)
};

// Pulses [p0, p1) of part `part` of nsplit near-equal parts of P.
__host__ __device__ inline void part_range(int P, int nsplit, int part, int &p0, int &p1) {
    if (nsplit <= 1) {
        p0 = 0;
        p1 = P;
        return;
    }
    p0 = (int)((long long)part * P / nsplit);
    p1 = (int)((long long)(part + 1) * P / nsplit);
}

// one row of a batched range-compression launch
struct RowItem {
    int job;
    int pulse;
};

}  // namespace sarbp
