/*
 * sarbp_oracle.h -- CPU oracle for the SAR backprojection hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm (ISI-apex/halide-sar-app) used as the parity checker for the CUDA
 * path and as the timed CPU baseline.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline / reference arm may load it.  The product
 * library never links it.
 *
 * Parity status: pinned at the helper level (Taylor window table, norm,
 * cross, linspace, arange known answers from the reference's test/ folder,
 * and the reference's AFRL image-plane fixtures data/AFRL/pass1/HH_ip_npy).
 * The backprojected image itself is NOT pinned: the reference ships no
 * golden image and cannot be built here (Halide, FFTW, cnpy, libpng are all
 * absent), so the image-level oracle is this restatement.  The FFT stage is
 * pinned to the DFT definition (checked against numpy.fft in the tests).
 *
 * Two precisions:
 *   ORC_MODE_REF  -- the reference's precision as written: f32 pos, f32 k_r,
 *                    f32 |pos| (norm_r0), f32 phs*filt, f64 everything else.
 *   ORC_MODE_FP64 -- the same algorithm entirely in f64 (f64 positions,
 *                    f64 k_r, f64 |pos|, f64 filter).
 */
#ifndef SARBP_ORACLE_H
#define SARBP_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MODE_REF 0
#define ORC_MODE_FP64 1
/* flag or'ed into the mode of orc_range_compress / orc_backprojection: the
 * Taylor window's F_m denominator quotient in floating point instead of the
 * reference's Int32 division (see orc_taylor_mode) */
#define ORC_TAYLOR_FLOAT 16

/* ---- helper-level restatements (util.h, signal.h, img_plane.cpp) ---- */
int orc_ip_upsample(int n);
void orc_taylor(int num, double S_L, double *out);
void orc_taylor_mode(int num, double S_L, int float_den, double *out);
void orc_linspace_f32(float start, float stop, int num, float *out);
void orc_linspace_f64(double start, double stop, int num, double *out);
void orc_arange_f32(float start, float step, int n, float *out);
float orc_norm_f32(const float *in, int n);
void orc_cross3_f32(const float *a, const float *b, float *out);
float orc_norm3d_f32(const float *xyz);

/* Image plane, ImgPlane.cpp:16-63.  Writes u[nu], v[nv], k_u[nu], k_v[nv],
 * u_hat[3], v_hat[3]; pixel_locs (SoA, [3][nu*nv]) when non-NULL. */
void orc_img_plane(int nsamples, int npulses, double delta_r, const float *R_c,
                   const float *n_hat, double res_factor, double aspect,
                   int upsample, int *nu, int *nv, double *d_u, double *d_v,
                   double *u, double *v, double *k_u, double *k_v,
                   double *u_hat, double *v_hat, double *pixel_locs);
/* pixel_locs from u, v, u_hat, v_hat (img_plane.cpp:77-103), SoA [3][nu*nv] */
void orc_pixel_locs(const double *u, int nu, const double *v, int nv,
                    const double *u_hat, const double *v_hat, double *out);

/* ---- the hot path ---- */
/* Forward, unnormalised complex DFT in place (interleaved re/im), f64. */
void orc_fft_forward(double *data, int n);

/* Range compression, backprojection.cpp:79-104.  phs is complex64 [P][S];
 * k_r is f64 [S] (rounded to f32 first in ORC_MODE_REF).  Q is complex f64
 * [P][N_fft]. */
int orc_range_compress(const float *phs, int S, int P, const double *k_r,
                       int taylor_s_l, int N_fft, int mode, double *Q,
                       int nthreads);

/* |pos_p| per pulse (norm_r0, backprojection.cpp:108): f32 in REF mode with
 * the op order (x*x + y*y) + z*z, no fused multiply-add; f64 in FP64 mode.
 * pos is f64 [P][3] (in REF mode its values are first rounded to f32). */
void orc_norm_r0(const double *pos, int P, int mode, double *nr0);
/* backprojection.cpp:52-65: complex samples q[lsn][2] on linspace(lsa, lsb,
 * lsn), interpolated at xs[nx] with the reference's clamps -> out[nx][2]. */
void orc_interp_linspace(const double *xs, long long nx, double lsa, double lsb, int lsn,
                         const double *q, double *out);

/* Per-pixel pulse accumulation, backprojection.cpp:110-138.  Evaluates the
 * output image at the n_out output pixels listed in out_idx (y*nu + x, in
 * output-image coordinates; NULL = all nu*nv in order).  out is complex f64
 * [n_out].  pos is f64 [P][3] (rounded to f32 in REF mode), r is SoA
 * [3][nu*nv] f64, k_r as above (k_c = k_r[S/2]).  Loop order follows the
 * reference CPU schedule (backprojection.cpp:296-314): pixels in x-vectors
 * of 4, parallel over vectors, pulse loop inside. */
int orc_backproject(const double *Q, int P, int N_fft, int S, double delta_r,
                    const double *k_r, const double *pos, const double *r,
                    int nu, int nv, const long long *out_idx, long long n_out,
                    int mode, double *out, int nthreads);

/* Whole pipeline: range compression + backprojection for all pixels. */
int orc_backprojection(const float *phs, int S, int P, const double *k_r,
                       int taylor_s_l, int N_fft, double delta_r,
                       const double *pos, const double *r, int nu, int nv,
                       int mode, double *out_img, int nthreads);

/* dB and u8 output stages, img_output.cpp:18-51 */
void orc_img_output_to_dB(const double *img, long long npix, double *dB);
void orc_img_output_u8(const double *dB, long long npix, double dB_min,
                       double dB_max, unsigned char *out);

int orc_max_threads(void);

/* Seeded synthetic phase history (the benchmark's CPU arm generates its
 * inputs with this, without the product library): phs complex64 [P][S],
 * pos f64 [P][3], k_r f64 [S]; scat is [nscat][5] (x, y, z, Re a, Im a). */
int orc_synth_phase_history(int S, int P, double f0, double df, double R0, double dep_deg,
                            double span_deg, const double *scat, int nscat, double snr_db,
                            unsigned long long seed, float *phs, double *pos, double *k_r,
                            int nthreads);

#ifdef __cplusplus
}
#endif
#endif
