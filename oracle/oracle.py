"""ctypes wrapper of the CPU oracle (liboracle: sarbp_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference arm as the parity checker and CPU
baseline.  The product library never imports it.

See sarbp_oracle.h for what is pinned (helper-level known answers and the
reference's AFRL image-plane fixtures) and what is not (the backprojected
image: the reference ships no golden image and cannot be built here).
"""
import ctypes
import os

import numpy as np

MODE_REF = 0
MODE_FP64 = 1
TAYLOR_FLOAT = 16  # mode flag: Taylor F_m denominator quotient in floating point

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libsarbp_oracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)


def build():
    import subprocess
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_taylor.argtypes = [ctypes.c_int, ctypes.c_double, _dp]
        L.orc_taylor_mode.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, _dp]
        L.orc_linspace_f32.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.c_int, _fp]
        L.orc_arange_f32.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.c_int, _fp]
        L.orc_norm_f32.argtypes = [_fp, ctypes.c_int]
        L.orc_norm_f32.restype = ctypes.c_float
        L.orc_cross3_f32.argtypes = [_fp, _fp, _fp]
        L.orc_ip_upsample.argtypes = [ctypes.c_int]
        L.orc_img_plane.argtypes = [
            ctypes.c_int, ctypes.c_int, ctypes.c_double, _fp, _fp, ctypes.c_double,
            ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
            ctypes.POINTER(ctypes.c_int), _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.orc_pixel_locs.argtypes = [_dp, ctypes.c_int, _dp, ctypes.c_int, _dp, _dp, _dp]
        L.orc_fft_forward.argtypes = [_dp, ctypes.c_int]
        L.orc_range_compress.argtypes = [_fp, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int]
        L.orc_norm_r0.argtypes = [_dp, ctypes.c_int, ctypes.c_int, _dp]
        L.orc_interp_linspace.argtypes = [_dp, ctypes.c_longlong, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_int, _dp, _dp]
        L.orc_backproject.argtypes = [
            _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp, _dp, _dp,
            ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong), ctypes.c_longlong,
            ctypes.c_int, _dp, ctypes.c_int]
        L.orc_img_output_to_dB.argtypes = [_dp, ctypes.c_longlong, _dp]
        L.orc_img_output_u8.argtypes = [_dp, ctypes.c_longlong, ctypes.c_double,
                                        ctypes.c_double, ctypes.POINTER(ctypes.c_ubyte)]
        L.orc_max_threads.restype = ctypes.c_int
        L.orc_synth_phase_history.argtypes = [
            ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
            ctypes.c_double, _dp, ctypes.c_int, ctypes.c_double, ctypes.c_ulonglong, _fp, _dp, _dp, ctypes.c_int]
        _lib = L
    return _lib


def _ptr(a, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct))


def max_threads():
    return lib().orc_max_threads()


def taylor(num, s_l, taylor_mode=0):
    """Taylor window; taylor_mode 1 takes the F_m denominator quotient in
    floating point (the float-division variant) instead of Int32."""
    out = np.empty(num, np.float64)
    lib().orc_taylor_mode(int(num), float(s_l), int(bool(taylor_mode)), _ptr(out, ctypes.c_double))
    return out


def linspace_f32(start, stop, num):
    out = np.empty(num, np.float32)
    lib().orc_linspace_f32(start, stop, num, _ptr(out, ctypes.c_float))
    return out


def arange_f32(start, step, n):
    out = np.empty(n, np.float32)
    lib().orc_arange_f32(start, step, n, _ptr(out, ctypes.c_float))
    return out


def norm_f32(v):
    v = np.ascontiguousarray(v, np.float32)
    return lib().orc_norm_f32(_ptr(v, ctypes.c_float), v.size)


def cross3_f32(a, b):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    out = np.empty(3, np.float32)
    lib().orc_cross3_f32(_ptr(a, ctypes.c_float), _ptr(b, ctypes.c_float), _ptr(out, ctypes.c_float))
    return out


def ip_upsample(n):
    return lib().orc_ip_upsample(int(n))


def img_plane(nsamples, npulses, delta_r, R_c, n_hat=(0.0, 0.0, 1.0), res_factor=1.0,
              aspect=1.0, upsample=True, pixel_locs=True):
    """ImgPlane.cpp:16-63; returns a dict of nu, nv, d_u, d_v, u, v, k_u, k_v,
    u_hat, v_hat and (optionally) pixel_locs as SoA [3, nu*nv]."""
    L = lib()
    R_c = np.ascontiguousarray(R_c, np.float32)
    n_hat = np.ascontiguousarray(n_hat, np.float32)
    nu, nv = ctypes.c_int(), ctypes.c_int()
    du, dv = ctypes.c_double(), ctypes.c_double()
    null = ctypes.POINTER(ctypes.c_double)()
    L.orc_img_plane(nsamples, npulses, delta_r, _ptr(R_c, ctypes.c_float),
                    _ptr(n_hat, ctypes.c_float), res_factor, aspect, int(bool(upsample)),
                    ctypes.byref(nu), ctypes.byref(nv), ctypes.byref(du), ctypes.byref(dv),
                    null, null, null, null, null, null, null)
    nu, nv = nu.value, nv.value
    out = {k: np.empty(n, np.float64) for k, n in
           (("u", nu), ("v", nv), ("k_u", nu), ("k_v", nv), ("u_hat", 3), ("v_hat", 3))}
    pl = np.empty((3, nu * nv), np.float64) if pixel_locs else None
    L.orc_img_plane(nsamples, npulses, delta_r, _ptr(R_c, ctypes.c_float),
                    _ptr(n_hat, ctypes.c_float), res_factor, aspect, int(bool(upsample)),
                    ctypes.byref(ctypes.c_int()), ctypes.byref(ctypes.c_int()),
                    ctypes.byref(du), ctypes.byref(dv),
                    *[_ptr(out[k], ctypes.c_double) for k in ("u", "v", "k_u", "k_v", "u_hat", "v_hat")],
                    _ptr(pl, ctypes.c_double) if pl is not None else null)
    out.update(nu=nu, nv=nv, d_u=du.value, d_v=dv.value)
    if pl is not None:
        out["pixel_locs"] = pl
    return out


def pixel_locs(u, v, u_hat, v_hat):
    u = np.ascontiguousarray(u, np.float64)
    v = np.ascontiguousarray(v, np.float64)
    uh = np.ascontiguousarray(u_hat, np.float64)
    vh = np.ascontiguousarray(v_hat, np.float64)
    out = np.empty((3, u.size * v.size), np.float64)
    lib().orc_pixel_locs(_ptr(u, ctypes.c_double), u.size, _ptr(v, ctypes.c_double), v.size,
                         _ptr(uh, ctypes.c_double), _ptr(vh, ctypes.c_double),
                         _ptr(out, ctypes.c_double))
    return out


def fft_forward(x):
    a = np.ascontiguousarray(x, np.complex128).copy()
    lib().orc_fft_forward(a.view(np.float64).ctypes.data_as(_dp), a.size)
    return a


def interp_linspace(xs, lsa, lsb, lsn, fp):
    """The interp of backprojection.cpp:52-65: complex fp sampled on
    linspace(lsa, lsb, lsn), evaluated at xs (clamped like the reference)."""
    xs = np.ascontiguousarray(xs, np.float64)
    q = np.ascontiguousarray(np.asarray(fp, np.complex128)).view(np.float64)
    out = np.zeros(2 * xs.size, np.float64)
    lib().orc_interp_linspace(_ptr(xs, ctypes.c_double), xs.size, float(lsa), float(lsb), int(lsn),
                              _ptr(q, ctypes.c_double), _ptr(out, ctypes.c_double))
    return out.view(np.complex128)


def range_compress(phs, k_r, taylor_s_l, n_fft, mode=MODE_REF, nthreads=0, taylor_mode=0):
    """phs complex64 [P, S] -> Q complex128 [P, N_fft]; taylor_mode 1 selects
    the float-division Taylor window."""
    if taylor_mode:
        mode |= TAYLOR_FLOAT
    phs = np.ascontiguousarray(phs, np.complex64)
    P, S = phs.shape
    k_r = np.ascontiguousarray(k_r, np.float64)
    Q = np.empty((P, n_fft), np.complex128)
    rc = lib().orc_range_compress(phs.view(np.float32).ctypes.data_as(_fp), S, P,
                                  _ptr(k_r, ctypes.c_double), int(taylor_s_l), int(n_fft),
                                  int(mode), Q.view(np.float64).ctypes.data_as(_dp), int(nthreads))
    if rc:
        raise ValueError("orc_range_compress failed: %d" % rc)
    return Q


def backproject(Q, S, delta_r, k_r, pos, r, nu, nv, out_idx=None, mode=MODE_REF, nthreads=0):
    """Evaluates output pixels (y*nu + x) listed in out_idx (None = all);
    returns complex128 [n_out] (or [nv, nu] when out_idx is None)."""
    Q = np.ascontiguousarray(Q, np.complex128)
    P, N = Q.shape
    k_r = np.ascontiguousarray(k_r, np.float64)
    pos = np.ascontiguousarray(pos, np.float64)
    r = np.ascontiguousarray(r, np.float64)
    assert r.shape == (3, nu * nv)
    if out_idx is None:
        n_out = nu * nv
        idx_p = ctypes.POINTER(ctypes.c_longlong)()
    else:
        out_idx = np.ascontiguousarray(out_idx, np.int64)
        n_out = out_idx.size
        idx_p = out_idx.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))
    out = np.empty(n_out, np.complex128)
    rc = lib().orc_backproject(Q.view(np.float64).ctypes.data_as(_dp), P, N, int(S), float(delta_r),
                               _ptr(k_r, ctypes.c_double), _ptr(pos, ctypes.c_double),
                               _ptr(r, ctypes.c_double), int(nu), int(nv), idx_p, n_out, int(mode),
                               out.view(np.float64).ctypes.data_as(_dp), int(nthreads))
    if rc:
        raise ValueError("orc_backproject failed: %d" % rc)
    return out.reshape(nv, nu) if out_idx is None else out


def backprojection(phs, k_r, taylor_s_l, n_fft, delta_r, pos, r, nu, nv, mode=MODE_REF,
                   out_idx=None, nthreads=0, taylor_mode=0):
    Q = range_compress(phs, k_r, taylor_s_l, n_fft, mode, nthreads, taylor_mode)
    return backproject(Q, phs.shape[1], delta_r, k_r, pos, r, nu, nv, out_idx, mode, nthreads)


def img_output_to_dB(img):
    img = np.ascontiguousarray(img, np.complex128)
    out = np.empty(img.shape, np.float64)
    lib().orc_img_output_to_dB(img.view(np.float64).ctypes.data_as(_dp), img.size,
                               _ptr(out, ctypes.c_double))
    return out


def img_output_u8(dB, dB_min, dB_max):
    dB = np.ascontiguousarray(dB, np.float64)
    out = np.empty(dB.shape, np.uint8)
    lib().orc_img_output_u8(_ptr(dB, ctypes.c_double), dB.size, float(dB_min), float(dB_max),
                            _ptr(out, ctypes.c_ubyte))
    return out


C_LIGHT = 299792458.0


def synth_phase_history(S, P, f0, df, R0, dep, span, scat, snr_db, seed, nthreads=0):
    """Seeded synthetic phase history (orc_synth_phase_history): returns
    (phs complex64 [P, S], pos f64 [P, 3], k_r f64 [S])."""
    scat = np.ascontiguousarray(scat, np.float64)
    phs = np.empty((P, S), np.complex64)
    pos = np.empty((P, 3), np.float64)
    k_r = np.empty(S, np.float64)
    rc = lib().orc_synth_phase_history(int(S), int(P), float(f0), float(df), float(R0), float(dep), float(span),
                                       _ptr(scat, ctypes.c_double), int(scat.shape[0]), float(snr_db),
                                       int(seed), phs.view(np.float32).ctypes.data_as(_fp),
                                       _ptr(pos, ctypes.c_double), _ptr(k_r, ctypes.c_double), int(nthreads))
    if rc:
        raise ValueError("orc_synth_phase_history failed: %d" % rc)
    return phs, pos, k_r


def make_workload(cfg, scat, seed, with_r=True, nthreads=0):
    """A benchmark workload from its configuration dict (P, S, f0, df, R0,
    dep, span, snr, n, extent, taylor, upsample, db) and scene, with the
    oracle alone: phase history, positions, k_r, delta_r, N_fft, and a
    square n x n image plane over `extent` metres whose axes come from the
    reference's image-plane construction with R_c the mid-aperture position
    (ImgPlane.cpp:16-63), pixel positions SoA [3, n*n]."""
    S, P = cfg["S"], cfg["P"]
    phs, pos, k_r = synth_phase_history(S, P, cfg["f0"], cfg["df"], cfg["R0"], cfg["dep"], cfg["span"], scat,
                                        cfg["snr"], seed, nthreads)
    delta_r = C_LIGHT / (2.0 * S * cfg["df"])
    ip = img_plane(S, P, delta_r, pos[P // 2].astype(np.float32), pixel_locs=False)
    n = cfg["n"]
    d = cfg["extent"] / n
    u = (np.arange(n) - n // 2) * d
    v = (np.arange(n) - n // 2) * d
    out = dict(cfg=cfg, phs=phs, pos=pos, k_r=k_r, delta_r=delta_r, S=S, P=P, nu=n, nv=n, u=u, v=v,
               u_hat=ip["u_hat"], v_hat=ip["v_hat"], taylor=cfg["taylor"], db=cfg["db"],
               N_fft=int(2 ** (int(np.log2(S * cfg["upsample"])) + 1)))
    if with_r:
        out["r"] = pixel_locs(u, v, ip["u_hat"], ip["v_hat"])
    return out
