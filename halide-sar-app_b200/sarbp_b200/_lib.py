"""ctypes binding of libsarbp_b200.so (include/sarbp_b200.h).

The library is required: importing this module on a machine where it has
not been built raises, and every compute entry point runs the CUDA kernels.
There is no CPU fallback.
"""
import ctypes
import os

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libsarbp_b200.so")

OK = 0
ERR_INVALID = -1
ERR_UNSUPPORTED = -2
ERR_NOMEM = -3
ERR_CUDA = -4
ERR_GEOMETRY = -5
ERR_TIMEOUT = -6
ERR_ADMISSION = -7
ERR_STATE = -8

PREC_COMPAT = 0
PREC_PRECISE = 1
PREC_NAIVE = 2

TAYLOR_REF = 0
TAYLOR_FLOAT = 1

_c_int_p = ctypes.POINTER(ctypes.c_int)
_dp = ctypes.c_void_p


class SarbpError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("sarbp error %d: %s" % (code, msg))
        self.code = code


class Opts(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("tile_x", ctypes.c_int), ("tile_y", ctypes.c_int),
                ("pulse_chunk", ctypes.c_int), ("persistent", ctypes.c_int),
                ("stage_cap", ctypes.c_int), ("min_blocks", ctypes.c_int), ("pulse_parts", ctypes.c_int)]


class Job(ctypes.Structure):
    _fields_ = [("nsamples", ctypes.c_int), ("npulses", ctypes.c_int), ("n_fft", ctypes.c_int),
                ("taylor_s_l", ctypes.c_int), ("nu", ctypes.c_int), ("nv", ctypes.c_int),
                ("delta_r", ctypes.c_double),
                ("phs", _dp), ("k_r", _dp), ("k_r64", _dp), ("pos", _dp), ("pos64", _dp),
                ("r", _dp), ("u", _dp), ("v", _dp),
                ("u_hat", ctypes.c_double * 3), ("v_hat", ctypes.c_double * 3),
                ("output_img", _dp), ("out_u8", _dp),
                ("dB_min", ctypes.c_double), ("dB_max", ctypes.c_double),
                ("precision", ctypes.c_int), ("taylor_mode", ctypes.c_int)]


# name -> (restype, argtypes); every symbol declared in include/sarbp_b200.h
SIGNATURES = {
    "sarbp_ctx_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "sarbp_ctx_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "sarbp_ctx_set_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "sarbp_ctx_stream": (ctypes.c_void_p, [ctypes.c_void_p]),
    "sarbp_ctx_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "sarbp_ctx_launch_count": (ctypes.c_longlong, [ctypes.c_void_p]),
    "sarbp_ctx_set_timing": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "sarbp_ctx_last_stage_ms": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)]),
    "sarbp_measure_peaks": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                           ctypes.POINTER(ctypes.c_double)]),
    "sarbp_last_error": (ctypes.c_char_p, []),
    "sarbp_version": (ctypes.c_char_p, []),
    "sarbp_backprojection": (ctypes.c_int, [
        ctypes.c_void_p, _dp, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
        ctypes.c_double, _dp, ctypes.c_int, _dp, ctypes.c_int, _dp, _dp, _dp,
        ctypes.POINTER(Opts)]),
    "sarbp_backprojection_plane": (ctypes.c_int, [
        ctypes.c_void_p, _dp, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
        ctypes.c_double, _dp, ctypes.c_int, _dp, ctypes.c_int, _dp, _dp, _dp, _dp,
        ctypes.POINTER(Opts)]),
    "sarbp_backprojection_f64": (ctypes.c_int, [
        ctypes.c_void_p, _dp, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
        ctypes.c_double, _dp, ctypes.c_int, _dp, ctypes.c_int, _dp, _dp, _dp,
        ctypes.POINTER(Opts)]),
    "sarbp_plan_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Job), ctypes.c_int,
                                         ctypes.POINTER(Opts), ctypes.POINTER(ctypes.c_void_p)]),
    "sarbp_plan_launch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "sarbp_plan_wait": (ctypes.c_int, [ctypes.c_void_p]),
    "sarbp_plan_kernel_count": (ctypes.c_int, [ctypes.c_void_p]),
    "sarbp_plan_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "sarbp_server_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Opts), ctypes.c_double,
                                           ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                           ctypes.POINTER(ctypes.c_void_p)]),
    "sarbp_server_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Job),
                                           ctypes.POINTER(ctypes.c_longlong)]),
    "sarbp_server_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_double]),
    "sarbp_server_times": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.POINTER(ctypes.c_double),
                                          ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    "sarbp_server_release": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong]),
    "sarbp_server_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong),
                                          ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong),
                                          ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    "sarbp_server_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "sarbp_server_register": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Job),
                                             ctypes.POINTER(ctypes.c_longlong)]),
    "sarbp_server_submit_on": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.POINTER(Job),
                                              ctypes.POINTER(ctypes.c_longlong)]),
    "sarbp_server_unregister": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong]),
    "sarbp_server_open_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Job), ctypes.c_int,
                                                ctypes.POINTER(ctypes.c_longlong)]),
    "sarbp_server_stream_add": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int, ctypes.c_int,
                                               _dp]),
    "sarbp_server_stream_finish": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong]),
    "sarbp_server_counters": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                             ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]),
    "sarbp_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Job), ctypes.c_int,
                                      ctypes.POINTER(Opts), ctypes.POINTER(ctypes.c_float)]),
    "sarbp_backprojection_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Job),
                                                   ctypes.POINTER(Opts)]),
    "sarbp_batch_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Job), ctypes.c_int,
                                          ctypes.POINTER(Opts)]),
    "sarbp_range_compress_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Job),
                                                   ctypes.POINTER(Opts), _dp]),
    "sarbp_backprojection_noalloc": (ctypes.c_int, [ctypes.POINTER(Job), ctypes.c_void_p, _dp]),
    "sarbp_accum_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Job), ctypes.POINTER(Opts),
                                          ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "sarbp_accum_add_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp]),
    "sarbp_accum_add": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp]),
    "sarbp_accum_finalize": (ctypes.c_int, [ctypes.c_void_p]),
    "sarbp_accum_wait": (ctypes.c_int, [ctypes.c_void_p]),
    "sarbp_accum_reset": (ctypes.c_int, [ctypes.c_void_p]),
    "sarbp_accum_device_bytes": (ctypes.c_double, [ctypes.c_void_p]),
    "sarbp_accum_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "sarbp_job_device_bytes": (ctypes.c_int, [ctypes.POINTER(Job), ctypes.POINTER(Opts), ctypes.c_int,
                                              ctypes.POINTER(ctypes.c_double)]),
    "sarbp_backprojection_streamed": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Job), ctypes.POINTER(Opts),
                                                     ctypes.c_double, ctypes.POINTER(ctypes.c_int),
                                                     ctypes.POINTER(ctypes.c_double)]),
    "sarbp_img_output_to_dB": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_int, ctypes.c_int, _dp]),
    "sarbp_img_output_u8": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_double, ctypes.c_double, _dp]),
    "sarbp_img_output_to_dB_device": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_int,
                                                     ctypes.c_int, _dp]),
    "sarbp_img_output_u8_device": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_double, ctypes.c_double, _dp]),
    "sarbp_img_output_u8_from_img_device": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_int, ctypes.c_int,
                                                           ctypes.c_double, ctypes.c_double, _dp]),
    "sarbp_resize_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp]),
    "sarbp_resize": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp]),
    "sarbp_taylor": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, _dp]),
    "sarbp_taylor_mode": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, ctypes.c_int, _dp]),
    "sarbp_img_plane_dims": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _c_int_p,
                                            _c_int_p]),
    "sarbp_img_plane": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp, _dp,
                                       ctypes.c_double, ctypes.c_double, ctypes.c_int, _dp, _dp,
                                       _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
    "sarbp_synth_phase_history": (ctypes.c_int, [
        ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
        ctypes.c_double, ctypes.c_double, _dp, ctypes.c_int, ctypes.c_double, ctypes.c_uint64,
        _dp, _dp, _dp, ctypes.c_int]),
}

_lib = None


def lib():
    """Loads the library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libsarbp_b200.so not found at %s; build it with "
                              "`make -C halide-sar-app_b200` (or __graft_entry__.build())" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc):
    if rc != OK:
        msg = lib().sarbp_last_error()
        raise SarbpError(rc, msg.decode() if msg else "")
    return rc
