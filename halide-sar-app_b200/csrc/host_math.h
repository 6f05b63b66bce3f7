// host_math.h -- small host-side computations of the reference pipeline.
#pragma once

#include <vector>

namespace sarbp {

// Taylor window coefficients F_m (signal.h:28-41) for side-lobe level S_L;
// returns n_bar - 1 values.  mode: SARBP_TAYLOR_REF (the reference's Int32
// division in the F_m denominator) or SARBP_TAYLOR_FLOAT (a float quotient).
std::vector<double> taylor_coefficients(double S_L, int mode = 0);
// The same coefficients written into out[0..cap) without allocating; returns
// their count (n_bar - 1), which may exceed cap (then only cap are written).
int taylor_coefficients_into(double S_L, double *out, int cap, int mode = 0);
// Full Taylor window (signal.h:14-51), normalised to its maximum.
void taylor_window(int num, double S_L, double *out, int mode = 0);

// ImgPlane.cpp:20-28 / ip.h:5-9
int ip_upsample(int n);

struct ImgPlane {
    int nu = 0, nv = 0;
    double d_u = 0, d_v = 0;
    std::vector<double> u, v, k_u, k_v;
    double u_hat[3] = {0, 0, 0}, v_hat[3] = {0, 0, 0};
};
// img_plane_create without the pixel_locs array (ImgPlane.cpp:16-63).
ImgPlane img_plane_create(int nsamples, int npulses, double delta_r, const float *R_c,
                          const float *n_hat, double res_factor, double aspect, bool upsample);
// pixel_locs SoA [3][nu*nv] (img_plane.cpp:77-103)
void pixel_locs(const ImgPlane &ip, double *out);

}  // namespace sarbp
