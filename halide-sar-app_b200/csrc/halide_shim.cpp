// halide_shim.cpp -- halide_buffer_t entry points over the C ABI (see
// include/sarbp_halide.h): each checks the shape and type the generator
// declares (backprojection.cpp:35-46, img_output.cpp:15-16, :43-46), maps the
// dense host data onto the matching sarbp_* call and marks the output
// buffer host-dirty, as a Halide pipeline that wrote host memory does.
#include "sarbp_halide.h"

#include <cstdlib>
#include <mutex>
#include <string>

#include "sarbp_b200.h"

namespace {

constexpr uint8_t kUInt = 1, kFloat = 2;  // halide_type_t codes
constexpr uint64_t kHostDirty = 1, kDeviceDirty = 2;

sarbp_ctx *shared_ctx(int *status) {
    static std::once_flag once;
    static sarbp_ctx *ctx = nullptr;
    static int rc = 0;
    std::call_once(once, [] {
        const char *e = std::getenv("SARBP_DEVICE");
        rc = sarbp_ctx_create(e ? std::atoi(e) : 0, &ctx);
    });
    *status = rc;
    return ctx;
}

// A dense buffer of `dims` dimensions, element type (code, bits), extents
// read back through `ext`; the first dimension has stride 1 and each next
// one the product of the previous extents (Halide's default layout).
bool dense(const halide_buffer_t *b, int dims, uint8_t code, int bits, int *ext) {
    if (!b || !b->host || (b->flags & kDeviceDirty)) return false;
    if (b->dimensions != dims || b->type.code != code || b->type.bits != bits || b->type.lanes != 1)
        return false;
    long long stride = 1;
    for (int d = 0; d < dims; ++d) {
        if (b->dim[d].extent < 1 || b->dim[d].stride != stride) return false;
        ext[d] = b->dim[d].extent;
        stride *= b->dim[d].extent;
    }
    return true;
}

}  // namespace

int backprojection_cuda(halide_buffer_t *phs, halide_buffer_t *k_r, int32_t taylor_s_l, int32_t N_fft,
                        double delta_r, halide_buffer_t *u, halide_buffer_t *v, halide_buffer_t *pos,
                        halide_buffer_t *r, halide_buffer_t *output_img) {
    int e_phs[3], e_k[1], e_u[1], e_v[1], e_pos[2], e_r[2], e_out[3];
    if (!dense(phs, 3, kFloat, 32, e_phs) || e_phs[0] != 2 || !dense(k_r, 1, kFloat, 32, e_k) ||
        !dense(u, 1, kFloat, 64, e_u) || !dense(v, 1, kFloat, 64, e_v) ||
        !dense(pos, 2, kFloat, 32, e_pos) || e_pos[0] != 3 || !dense(r, 2, kFloat, 64, e_r) ||
        !dense(output_img, 3, kFloat, 64, e_out) || e_out[0] != 2)
        return SARBP_ERR_INVALID;
    const int S = e_phs[1], P = e_phs[2], nu = e_u[0], nv = e_v[0];
    if (e_k[0] != S || e_pos[1] != P || e_r[0] != nu * nv || e_r[1] != 3 || e_out[1] != nu ||
        e_out[2] != nv)
        return SARBP_ERR_INVALID;
    int rc = 0;
    sarbp_ctx *ctx = shared_ctx(&rc);
    if (rc) return rc;
    rc = sarbp_backprojection(ctx, reinterpret_cast<const float *>(phs->host), S, P,
                              reinterpret_cast<const float *>(k_r->host), taylor_s_l, N_fft, delta_r,
                              reinterpret_cast<const double *>(u->host), nu,
                              reinterpret_cast<const double *>(v->host), nv,
                              reinterpret_cast<const float *>(pos->host),
                              reinterpret_cast<const double *>(r->host),
                              reinterpret_cast<double *>(output_img->host), nullptr);
    if (rc == 0) output_img->flags |= kHostDirty;
    return rc;
}

void dft_init_fftw(size_t) {}
void dft_destroy_fftw(void) {}

extern "C" {

int img_output_to_dB(halide_buffer_t *img, halide_buffer_t *out) {
    int e_in[3], e_out[2];
    if (!dense(img, 3, kFloat, 64, e_in) || e_in[0] != 2 || !dense(out, 2, kFloat, 64, e_out) ||
        e_out[0] != e_in[1] || e_out[1] != e_in[2])
        return SARBP_ERR_INVALID;
    int rc = 0;
    sarbp_ctx *ctx = shared_ctx(&rc);
    if (rc) return rc;
    rc = sarbp_img_output_to_dB(ctx, reinterpret_cast<const double *>(img->host), e_in[1], e_in[2],
                                reinterpret_cast<double *>(out->host));
    if (rc == 0) out->flags |= kHostDirty;
    return rc;
}

int img_output_u8(halide_buffer_t *dB, double dB_min, double dB_max, halide_buffer_t *out) {
    int e_in[2], e_out[2];
    if (!dense(dB, 2, kFloat, 64, e_in) || !dense(out, 2, kUInt, 8, e_out) || e_out[0] != e_in[0] ||
        e_out[1] != e_in[1])
        return SARBP_ERR_INVALID;
    int rc = 0;
    sarbp_ctx *ctx = shared_ctx(&rc);
    if (rc) return rc;
    rc = sarbp_img_output_u8(ctx, reinterpret_cast<const double *>(dB->host), e_in[0], e_in[1], dB_min,
                             dB_max, reinterpret_cast<uint8_t *>(out->host));
    if (rc == 0) out->flags |= kHostDirty;
    return rc;
}

}  // extern "C"
