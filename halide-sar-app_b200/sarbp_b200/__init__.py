"""sarbp_b200 -- SAR backprojection on B200 (sm_100a), Python side.

Mirrors the reference application's operator interface for the `-s cuda`
path (ISI-apex/halide-sar-app):

  backprojection_cuda(phs, k_r, taylor_s_l, N_fft, delta_r, u, v, pos, r)
        -> output_img            (backprojection.cpp:35-46, sarbp.cpp:277)
  img_output_to_dB(img) -> dB    (img_output.cpp:10-39)
  img_output_u8(dB, dB_min, dB_max) -> u8   (img_output.cpp:41-52)
  img_plane_create(...)          (ImgPlane.cpp:16-63)
  taylor(num, S_L)               (signal.h:14-51)

Arrays use the reference's memory layouts (see include/sarbp_b200.h); the
image comes back as complex128 [nv, nu] with the reference's row flip.
All compute runs through libsarbp_b200.so; there is no CPU path.
"""
import collections
import ctypes
import math

import numpy as np

from ._lib import (ERR_ADMISSION, ERR_CUDA, ERR_GEOMETRY, ERR_INVALID, ERR_NOMEM, ERR_STATE,
                   ERR_TIMEOUT, ERR_UNSUPPORTED, OK, PREC_COMPAT, PREC_NAIVE, PREC_PRECISE,
                   TAYLOR_FLOAT, TAYLOR_REF, Job, Opts, SarbpError, check, lib)

__all__ = [
    "Context", "Job", "Opts", "SarbpError", "PREC_COMPAT", "PREC_PRECISE", "PREC_NAIVE",
    "TAYLOR_REF", "TAYLOR_FLOAT", "Accumulator", "Server", "Plan", "make_job", "job_device_bytes",
    "backprojection_streamed", "n_fft_for", "taylor", "img_plane_create", "img_plane_dims", "pixel_locs",
    "version",
]


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else ctypes.c_void_p(0)


def last_error():
    """Message of the calling thread's last failed call."""
    return lib().sarbp_last_error().decode()


def version():
    return lib().sarbp_version().decode()


def n_fft_for(nsamples, upsample):
    """FFT width of sarbp.cpp:258: 2^(floor(log2(nsamples*upsample)) + 1)."""
    return int(math.pow(2, int(math.log2(nsamples * upsample)) + 1))


def taylor(num, S_L, mode=TAYLOR_REF):
    """Taylor window (signal.h:14-51); mode TAYLOR_FLOAT takes the F_m
    denominator quotient in floating point instead of Int32."""
    out = np.empty(num, np.float64)
    if mode == TAYLOR_REF:
        check(lib().sarbp_taylor(int(num), float(S_L), _ptr(out)))
    else:
        check(lib().sarbp_taylor_mode(int(num), float(S_L), int(mode), _ptr(out)))
    return out


def img_plane_dims(nsamples, npulses, upsample=True):
    nu, nv = ctypes.c_int(), ctypes.c_int()
    check(lib().sarbp_img_plane_dims(int(nsamples), int(npulses), int(bool(upsample)),
                                     ctypes.byref(nu), ctypes.byref(nv)))
    return nu.value, nv.value


def img_plane_create(nsamples, npulses, delta_r, R_c, n_hat=(0.0, 0.0, 1.0), res_factor=1.0,
                     aspect=1.0, upsample=True, with_pixel_locs=True):
    """ImgPlane.cpp:16-63; returns dict(nu, nv, d_u, d_v, u, v, k_u, k_v, u_hat,
    v_hat[, pixel_locs SoA [3, nu*nv]])."""
    nu, nv = img_plane_dims(nsamples, npulses, upsample)
    R_c = np.ascontiguousarray(R_c, np.float32)
    n_hat = np.ascontiguousarray(n_hat, np.float32)
    o = {k: np.empty(n, np.float64) for k, n in
         (("u", nu), ("v", nv), ("k_u", nu), ("k_v", nv), ("u_hat", 3), ("v_hat", 3))}
    pl = np.empty((3, nu * nv), np.float64) if with_pixel_locs else None
    du, dv = ctypes.c_double(), ctypes.c_double()
    check(lib().sarbp_img_plane(int(nsamples), int(npulses), float(delta_r), _ptr(R_c), _ptr(n_hat),
                                float(res_factor), float(aspect), int(bool(upsample)),
                                ctypes.cast(ctypes.byref(du), ctypes.c_void_p),
                                ctypes.cast(ctypes.byref(dv), ctypes.c_void_p),
                                *[_ptr(o[k]) for k in ("u", "v", "k_u", "k_v", "u_hat", "v_hat")],
                                _ptr(pl)))
    o.update(nu=nu, nv=nv, d_u=du.value, d_v=dv.value)
    if pl is not None:
        o["pixel_locs"] = pl
    return o


def pixel_locs(u, v, u_hat, v_hat):
    """img_plane.cpp:92-102: SoA [3, nu*nv], pixel i at u[i % nu], v[i // nu]."""
    u = np.asarray(u, np.float64)
    v = np.asarray(v, np.float64)
    out = np.empty((3, u.size * v.size), np.float64)
    for d in range(3):
        out[d] = np.add.outer(v_hat[d] * v, u_hat[d] * u).ravel()
    return out


def _opts(precision=None, tile=None, pulse_chunk=0, persistent=0, stage_cap=0, min_blocks=0, pulse_parts=0):
    o = Opts()
    o.precision = PREC_COMPAT if precision is None else int(precision)
    if tile:
        o.tile_x, o.tile_y = int(tile[0]), int(tile[1])
    o.pulse_chunk = int(pulse_chunk)
    o.persistent = int(persistent)
    o.stage_cap = int(stage_cap)
    o.min_blocks = int(min_blocks)
    o.pulse_parts = int(pulse_parts)
    return o


class Context:
    """One device context (device memory, stream, kernel launch counter)."""

    def __init__(self, device=0):
        self._h = ctypes.c_void_p()
        check(lib().sarbp_ctx_create(int(device), ctypes.byref(self._h)))

    def close(self):
        if self._h:
            lib().sarbp_ctx_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_stream(self, cuda_stream_handle):
        check(lib().sarbp_ctx_set_stream(self._h, ctypes.c_void_p(cuda_stream_handle or 0)))

    def synchronize(self):
        check(lib().sarbp_ctx_synchronize(self._h))

    def launch_count(self):
        return int(lib().sarbp_ctx_launch_count(self._h))

    def set_timing(self, on=True):
        check(lib().sarbp_ctx_set_timing(self._h, int(bool(on))))

    def last_stage_ms(self):
        """(set-up, range compression, tile geometry, backprojection, u8) ms
        of the last batch."""
        ms = (ctypes.c_float * 5)()
        check(lib().sarbp_ctx_last_stage_ms(self._h, ms))
        return tuple(float(x) for x in ms)

    def measure_peaks(self):
        """(FFMA instructions/s, MUFU ops/s) measured on this device."""
        f, m = ctypes.c_double(), ctypes.c_double()
        check(lib().sarbp_measure_peaks(self._h, ctypes.byref(f), ctypes.byref(m)))
        return f.value, m.value

    # ---- the reference's operators, host arrays ----
    def backprojection_cuda(self, phs, k_r, taylor_s_l, N_fft, delta_r, u, v, pos, r,
                            precision=None, **tune):
        """Drop-in for the Halide pipeline backprojection_cuda.  phs complex64
        [P, S]; k_r [S]; pos [P, 3]; r SoA [3, nu*nv]; returns complex128
        [nv, nu].  f32 pos/k_r run with the reference's semantics
        (PREC_COMPAT); f64 pos/k_r default to PREC_PRECISE."""
        phs = np.ascontiguousarray(phs, np.complex64)
        P, S = phs.shape
        u = np.ascontiguousarray(u, np.float64)
        v = np.ascontiguousarray(v, np.float64)
        nu, nv = u.size, v.size
        r = np.ascontiguousarray(r, np.float64)
        if r.size != 3 * nu * nv:
            raise SarbpError(ERR_INVALID, "r must hold 3*nu*nv values")
        out = np.empty((nv, nu), np.complex128)
        wide = np.asarray(pos).dtype == np.float64 or np.asarray(k_r).dtype == np.float64
        if wide:
            pos = np.ascontiguousarray(pos, np.float64)
            k_r = np.ascontiguousarray(k_r, np.float64)
            o = _opts(PREC_PRECISE if precision is None else precision, **tune)
            fn = lib().sarbp_backprojection_f64
        else:
            pos = np.ascontiguousarray(pos, np.float32)
            k_r = np.ascontiguousarray(k_r, np.float32)
            o = _opts(PREC_COMPAT if precision is None else precision, **tune)
            fn = lib().sarbp_backprojection
        if pos.size != 3 * P or k_r.size != S:
            raise SarbpError(ERR_INVALID, "pos must be [P, 3] and k_r [S]")
        check(fn(self._h, _ptr(phs), S, P, _ptr(k_r), int(taylor_s_l), int(N_fft), float(delta_r),
                 _ptr(u), nu, _ptr(v), nv, _ptr(pos), _ptr(r), _ptr(out), ctypes.byref(o)))
        return out

    def backprojection_plane(self, phs, k_r, taylor_s_l, N_fft, delta_r, u, v, u_hat, v_hat, pos,
                             precision=None, **tune):
        """backprojection_cuda with pixel_locs given by the image-plane axes:
        pixel (i, j) = u_hat * u[i] + v_hat * v[j], formed on the device."""
        phs = np.ascontiguousarray(phs, np.complex64)
        P, S = phs.shape
        u = np.ascontiguousarray(u, np.float64)
        v = np.ascontiguousarray(v, np.float64)
        uh = np.ascontiguousarray(u_hat, np.float64)
        vh = np.ascontiguousarray(v_hat, np.float64)
        pos = np.ascontiguousarray(pos, np.float32)
        k_r = np.ascontiguousarray(k_r, np.float32)
        if pos.size != 3 * P or k_r.size != S or uh.size != 3 or vh.size != 3:
            raise SarbpError(ERR_INVALID, "pos must be [P, 3], k_r [S], u_hat and v_hat [3]")
        nu, nv = u.size, v.size
        out = np.empty((nv, nu), np.complex128)
        o = _opts(PREC_COMPAT if precision is None else precision, **tune)
        check(lib().sarbp_backprojection_plane(
            self._h, _ptr(phs), S, P, _ptr(k_r), int(taylor_s_l), int(N_fft), float(delta_r),
            _ptr(u), nu, _ptr(v), nv, _ptr(uh), _ptr(vh), _ptr(pos), _ptr(out), ctypes.byref(o)))
        return out

    def img_output_to_dB(self, img):
        img = np.ascontiguousarray(img, np.complex128)
        nv, nu = img.shape
        out = np.empty((nv, nu), np.float64)
        check(lib().sarbp_img_output_to_dB(self._h, _ptr(img), nu, nv, _ptr(out)))
        return out

    def img_output_u8(self, dB, dB_min, dB_max):
        dB = np.ascontiguousarray(dB, np.float64)
        nv, nu = dB.shape
        out = np.empty((nv, nu), np.uint8)
        check(lib().sarbp_img_output_u8(self._h, _ptr(dB), nu, nv, float(dB_min), float(dB_max),
                                        _ptr(out)))
        return out

    def img_output_u8_from_img_device(self, img_ptr, nu, nv, dB_min, dB_max, out_ptr):
        """u8 image [nv, nu] from a device complex128 image in one pass (max|z|
        reduction + grey levels), enqueued on the context's stream."""
        check(lib().sarbp_img_output_u8_from_img_device(self._h, ctypes.c_void_p(img_ptr), int(nu), int(nv),
                                                        float(dB_min), float(dB_max), ctypes.c_void_p(out_ptr)))

    def resize(self, a, shape):
        """skimage.transform.resize(a, shape, preserve_range=True) as the
        reference's data/resize.py uses it, on the device (sarbp_resize):
        a 1-D or 2-D f32 / f64 array; a complex array is resampled as its
        real and imaginary parts."""
        a = np.asarray(a)
        shape = tuple(int(x) for x in shape)
        if a.ndim not in (1, 2) or len(shape) != a.ndim:
            raise SarbpError(ERR_INVALID, "resize: 1-D or 2-D arrays, and a shape of the same rank")
        cplx = np.iscomplexobj(a)
        if cplx:
            real = np.float32 if a.dtype == np.complex64 else np.float64
            src = np.ascontiguousarray(a).view(real)
        else:
            if a.dtype not in (np.float32, np.float64):
                a = a.astype(np.float64)
            real = a.dtype.type
            src = np.ascontiguousarray(a)
        rows, cols = (1, a.shape[0]) if a.ndim == 1 else a.shape
        orows, ocols = (1, shape[0]) if a.ndim == 1 else shape
        nc = 2 if cplx else 1
        out = np.empty((orows, ocols * nc), real)
        check(lib().sarbp_resize(self._h, np.dtype(real).itemsize, nc, _ptr(src), rows, cols, orows, ocols,
                                 _ptr(out)))
        if cplx:
            out = out.view(np.complex64 if real == np.float32 else np.complex128)
        return out.reshape(shape)

    def range_compress_device(self, job, q_out_ptr, precision=None):
        """Writes the complex64 range profiles [P, N_fft] of `job` to q_out_ptr."""
        o = _opts(precision)
        check(lib().sarbp_range_compress_device(self._h, ctypes.byref(job), ctypes.byref(o),
                                                ctypes.c_void_p(q_out_ptr)))

    # ---- device-resident jobs (pointers from torch tensors or raw ints) ----
    def run_jobs(self, jobs, precision=None, **tune):
        """Enqueues a list of Job structs (device pointers) as one batch."""
        arr = (Job * len(jobs))(*jobs)
        o = _opts(precision, **tune)
        if len(jobs) == 1:
            check(lib().sarbp_backprojection_device(self._h, arr, ctypes.byref(o)))
        else:
            check(lib().sarbp_batch_device(self._h, arr, len(jobs), ctypes.byref(o)))

    def autotune(self, jobs, precision=None):
        """Fastest launch shape for this batch (sarbp_autotune); returns
        (tune dict for run_jobs / plan, best ms or -1 when cached)."""
        arr = (Job * len(jobs))(*jobs)
        o = _opts(precision)
        ms = ctypes.c_float()
        check(lib().sarbp_autotune(self._h, arr, len(jobs), ctypes.byref(o), ctypes.byref(ms)))
        tune = dict(tile=(o.tile_x, o.tile_y), pulse_chunk=o.pulse_chunk, min_blocks=o.min_blocks,
                    stage_cap=o.stage_cap, pulse_parts=o.pulse_parts)
        return tune, ms.value

    def plan(self, jobs, precision=None, **tune):
        """The batch captured as a CUDA graph (sarbp_plan_create)."""
        return Plan(self, jobs, precision, **tune)


class Accumulator:
    """Pulse-chunked image formation (sarbp_accum_*): a device-resident
    partial image that takes the aperture's phase-history rows chunk by
    chunk.  `job` is a Job of device pointers for the whole aperture (its
    phs field is not read); add_device(pulse0, count, ptr) takes device rows,
    add(pulse0, rows) host rows (complex64 [count, S]); finalize() writes the
    job's output image; wait() returns once done (raises on a kernel error)."""

    def __init__(self, ctx, job, max_chunk, precision=None, **tune):
        self._job = job
        o = _opts(precision, **tune)
        self._h = ctypes.c_void_p()
        check(lib().sarbp_accum_create(ctx._h, ctypes.byref(job), ctypes.byref(o), int(max_chunk),
                                       ctypes.byref(self._h)))
        self._rows = []

    def add_device(self, pulse0, count, phs_rows_ptr):
        check(lib().sarbp_accum_add_device(self._h, int(pulse0), int(count), ctypes.c_void_p(phs_rows_ptr)))

    def add(self, pulse0, rows):
        rows = np.ascontiguousarray(rows, np.complex64)
        check(lib().sarbp_accum_add(self._h, int(pulse0), int(rows.shape[0]), _ptr(rows)))
        self._rows = self._rows[-1:] + [rows]  # the copy may still read them

    def finalize(self):
        check(lib().sarbp_accum_finalize(self._h))

    def wait(self):
        check(lib().sarbp_accum_wait(self._h))
        self._rows = []

    def reset(self):
        check(lib().sarbp_accum_reset(self._h))

    @property
    def device_bytes(self):
        return float(lib().sarbp_accum_device_bytes(self._h))

    def close(self):
        if self._h:
            lib().sarbp_accum_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def job_device_bytes(job, chunk_pulses=0, precision=None, **tune):
    """Device bytes of a job formed in one call, or in chunks of chunk_pulses."""
    b = ctypes.c_double()
    o = _opts(precision, **tune)
    check(lib().sarbp_job_device_bytes(ctypes.byref(job), ctypes.byref(o), int(chunk_pulses), ctypes.byref(b)))
    return b.value


def backprojection_streamed(ctx, host_job, max_device_bytes, precision=None, **tune):
    """A Job of HOST pointers formed in pulse chunks under a device-memory
    cap (sarbp_backprojection_streamed); returns (chunk pulses, device bytes)."""
    o = _opts(precision, **tune)
    c, b = ctypes.c_int(), ctypes.c_double()
    check(lib().sarbp_backprojection_streamed(ctx._h, ctypes.byref(host_job), ctypes.byref(o),
                                              float(max_device_bytes), ctypes.byref(c), ctypes.byref(b)))
    return c.value, b.value


class Server:
    """The serving loop (sarbp_server_*): submit(job) queues a Job whose
    pointers are host memory and returns its id; wait(id) returns its status
    (ERR_TIMEOUT while in flight); times(id) gives (submit, start, done)
    seconds on the server's clock."""

    def __init__(self, ctx, hbm_cap_bytes=150e9, lanes=3, max_batch=32, max_batch_work=0.0,
                 precision=None, **tune):
        o = _opts(precision, **tune)
        self._h = ctypes.c_void_p()
        check(lib().sarbp_server_create(ctx._h, ctypes.byref(o), float(hbm_cap_bytes), int(lanes),
                                        int(max_batch), float(max_batch_work), ctypes.byref(self._h)))
        self._keep = {}

    def submit(self, job, keep=None):
        rid = ctypes.c_longlong()
        check(lib().sarbp_server_submit(self._h, ctypes.byref(job), ctypes.byref(rid)))
        self._keep[rid.value] = (job, keep)
        return rid.value

    def register(self, job):
        """Uploads and range-compresses an aperture (a Job of host pointers)
        once; returns its id for submit_on."""
        aid = ctypes.c_longlong()
        check(lib().sarbp_server_register(self._h, ctypes.byref(job), ctypes.byref(aid)))
        return aid.value

    def submit_on(self, aperture, job, keep=None):
        """Queues a request on a registered aperture: `job` supplies the image
        plane (nu, nv, r or u/v/u_hat/v_hat) and outputs, host memory."""
        rid = ctypes.c_longlong()
        check(lib().sarbp_server_submit_on(self._h, int(aperture), ctypes.byref(job), ctypes.byref(rid)))
        self._keep[rid.value] = (job, keep)
        return rid.value

    def unregister(self, aperture):
        check(lib().sarbp_server_unregister(self._h, int(aperture)))

    def open_stream(self, job, max_chunk):
        """A streaming aperture (partial image on the device) for a Job of host
        pointers whose phase history will arrive in chunks; returns its id."""
        sid = ctypes.c_longlong()
        check(lib().sarbp_server_open_stream(self._h, ctypes.byref(job), int(max_chunk), ctypes.byref(sid)))
        self._keep[("stream", sid.value)] = [job, collections.deque(maxlen=8)]
        return sid.value

    def stream_add(self, stream, pulse0, rows):
        """Adds host phase-history rows (complex64 [count, S]) starting at pulse0."""
        rows = np.ascontiguousarray(rows, np.complex64)
        check(lib().sarbp_server_stream_add(self._h, int(stream), int(pulse0), int(rows.shape[0]), _ptr(rows)))
        # these rows may still be read by their copy until the next add on the
        # stream returns; adds from several threads append in any order, so
        # the last few are kept
        self._keep[("stream", stream)][1].append(rows)

    def stream_finish(self, stream):
        """Writes the stream's image into its output buffer(s) and frees it."""
        try:
            check(lib().sarbp_server_stream_finish(self._h, int(stream)))
        finally:
            self._keep.pop(("stream", stream), None)

    def counters(self):
        """(bytes copied host -> device, pulses range-compressed, requests
        served from registered apertures) since the server started."""
        b, p, r = ctypes.c_double(), ctypes.c_longlong(), ctypes.c_longlong()
        check(lib().sarbp_server_counters(self._h, ctypes.byref(b), ctypes.byref(p), ctypes.byref(r)))
        return dict(h2d_bytes=b.value, rc_pulses=p.value, resident_requests=r.value)

    def wait(self, rid, timeout=-1.0):
        return int(lib().sarbp_server_wait(self._h, int(rid), float(timeout)))

    def times(self, rid):
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        check(lib().sarbp_server_times(self._h, int(rid), ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def release(self, rid):
        check(lib().sarbp_server_release(self._h, int(rid)))
        self._keep.pop(rid, None)

    def stats(self):
        s, c, b = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        u, p = ctypes.c_double(), ctypes.c_double()
        check(lib().sarbp_server_stats(self._h, ctypes.byref(s), ctypes.byref(c), ctypes.byref(b),
                                       ctypes.byref(u), ctypes.byref(p)))
        return dict(submitted=s.value, completed=c.value, batches=b.value, in_use_bytes=u.value,
                    peak_bytes=p.value)

    def close(self):
        if self._h:
            lib().sarbp_server_destroy(self._h)
            self._h = ctypes.c_void_p()
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Plan:
    """A CUDA-graph batch: launch(stream) replays it, wait() synchronises and
    checks status, kernels is the kernel count per replay."""

    def __init__(self, ctx, jobs, precision=None, **tune):
        self._jobs = (Job * len(jobs))(*jobs)
        o = _opts(precision, **tune)
        self._h = ctypes.c_void_p()
        check(lib().sarbp_plan_create(ctx._h, self._jobs, len(jobs), ctypes.byref(o),
                                      ctypes.byref(self._h)))
        self.kernels = lib().sarbp_plan_kernel_count(self._h)

    def launch(self, stream=None):
        check(lib().sarbp_plan_launch(self._h, stream))

    def wait(self):
        check(lib().sarbp_plan_wait(self._h))

    def close(self):
        if self._h:
            lib().sarbp_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_job(nsamples, npulses, n_fft, taylor_s_l, nu, nv, delta_r, phs, k_r, pos, output_img,
             r=0, u=0, v=0, u_hat=(0, 0, 0), v_hat=(0, 0, 0), k_r64=0, pos64=0, out_u8=0,
             dB_min=0.0, dB_max=0.0, precision=-1, taylor_mode=TAYLOR_REF):
    """Builds a Job from device addresses (ints, e.g. tensor.data_ptr())."""
    j = Job()
    j.nsamples, j.npulses, j.n_fft, j.taylor_s_l = int(nsamples), int(npulses), int(n_fft), int(taylor_s_l)
    j.nu, j.nv, j.delta_r = int(nu), int(nv), float(delta_r)
    j.phs, j.k_r, j.k_r64, j.pos, j.pos64 = phs or None, k_r or None, k_r64 or None, pos or None, pos64 or None
    j.r, j.u, j.v = r or None, u or None, v or None
    for i in range(3):
        j.u_hat[i] = float(u_hat[i])
        j.v_hat[i] = float(v_hat[i])
    j.output_img, j.out_u8 = output_img or None, out_u8 or None
    j.dB_min, j.dB_max = float(dB_min), float(dB_max)
    j.precision = int(precision)
    j.taylor_mode = int(taylor_mode)
    return j
