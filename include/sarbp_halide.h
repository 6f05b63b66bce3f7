/*
 * sarbp_halide.h -- link-compatible replacements for the Halide AOT entry
 * points the reference CLI calls on its `-s cuda` path, so that code written
 * against the generated headers links against libsarbp_halide.so unchanged.
 *
 *   backprojection_cuda   C++ linkage (the generator is built with
 *                         c_plus_plus_name_mangling, CMakeLists.txt:77-84);
 *                         arguments as in backprojection.cpp:35-46
 *   img_output_to_dB      C linkage (CMakeLists.txt:105-106), img_output.cpp:10-39
 *   img_output_u8         C linkage (CMakeLists.txt:107-108), img_output.cpp:41-52
 *   dft_init_fftw / dft_destroy_fftw   C++ linkage (dft.h); no-ops here, the
 *                         FFT runs on the device inside backprojection_cuda
 *
 * Buffers are halide_buffer_t with host memory.  The struct below is the
 * public, stable layout of Halide's runtime ABI, declared here only when
 * HalideRuntime.h has not been included first.  Buffers whose device copy is
 * newer than the host copy (device_dirty) or without host memory (bounds
 * queries) are refused with a negative status.  All calls share one
 * process-wide context on CUDA device 0 (SARBP_DEVICE selects another).
 */
#ifndef SARBP_HALIDE_H
#define SARBP_HALIDE_H

#include <stddef.h>
#include <stdint.h>

#ifndef HALIDE_HALIDERUNTIME_H
struct halide_device_interface_t;
struct halide_type_t {
    uint8_t code; /* 0 int, 1 uint, 2 float, 3 handle, 4 bfloat */
    uint8_t bits;
    uint16_t lanes;
};
struct halide_dimension_t {
    int32_t min, extent, stride;
    uint32_t flags;
};
struct halide_buffer_t {
    uint64_t device;
    const struct halide_device_interface_t *device_interface;
    uint8_t *host;
    uint64_t flags; /* bit 0 host_dirty, bit 1 device_dirty */
    struct halide_type_t type;
    int32_t dimensions;
    struct halide_dimension_t *dim;
    void *padding;
};
#endif

#ifdef __cplusplus
/* phs f32 {2,S,P}, k_r f32 {S}, u f64 {nu}, v f64 {nv}, pos f32 {3,P},
 * r f64 {nu*nv,3}, output_img f64 {2,nu,nv}; returns 0 or a negative
 * sarbp status. */
int backprojection_cuda(struct halide_buffer_t *phs, struct halide_buffer_t *k_r,
                        int32_t taylor_s_l, int32_t N_fft, double delta_r,
                        struct halide_buffer_t *u, struct halide_buffer_t *v,
                        struct halide_buffer_t *pos, struct halide_buffer_t *r,
                        struct halide_buffer_t *output_img);
void dft_init_fftw(size_t N_fft);
void dft_destroy_fftw(void);
extern "C" {
#endif

/* img f64 {2,nu,nv} -> out f64 {nu,nv} */
int img_output_to_dB(struct halide_buffer_t *img, struct halide_buffer_t *out);
/* dB f64 {nu,nv} -> out u8 {nu,nv} */
int img_output_u8(struct halide_buffer_t *dB, double dB_min, double dB_max,
                  struct halide_buffer_t *out);

#ifdef __cplusplus
}
#endif

#endif /* SARBP_HALIDE_H */
