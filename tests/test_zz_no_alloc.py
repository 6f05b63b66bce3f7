"""sarbp_backprojection_noalloc: the backprojection entry point that
allocates nothing.

It exists for callers that must not allocate device memory when they want
an image: processes whose device memory is handed out up front by a pool
they do not own (a cudaMalloc there fails or fragments the pool), and
real-time loops that cannot afford cudaMalloc's latency and implicit
synchronisation on the path that forms each image.  Its scratch lives in
one static 64 MiB device array of the library that every call reuses.

The test runs three different jobs, twice each, back to back (stale
contents of one call must not leak into the next):
  * COMPAT precision with a pixel-position array (r),
  * COMPAT with the image-plane axes (u, v, u_hat, v_hat) and a u8 image,
  * PRECISE with f64 positions and k_r,
and checks each image against the ordinary device entry point (relative
L2 <= 1e-4, the tolerance of the other GPU parity tests; the u8 images must
be equal) and against the CPU oracle at sampled pixels (reference
precision, or FP64 for PRECISE: relative L2 <= 1e-4).

The file is named to be collected last: if it fails, a run that stops at
the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-4


def _cases(sb, torch):
    from sarbp_b200 import synth
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    cases = []
    # COMPAT, r array
    d = synth.make("plain_small", seed=1, overrides=dict(n=256, extent=25.0))
    t = dict(phs=dev(d["phs"].view(np.float32)), k=dev(d["k_r"].astype(np.float32)),
             pos=dev(d["pos"].astype(np.float32)), r=dev(d["r"]))
    kw = dict(r=t["r"].data_ptr())
    cases.append(("compat_r", d, t, sb.PREC_COMPAT, kw, False))
    # COMPAT, image-plane axes, u8 image
    d = synth.make("plain_small", seed=5, with_r=True,
                   overrides=dict(P=333, S=300, n=200, extent=30.0, taylor=20))
    t = dict(phs=dev(d["phs"].view(np.float32)), k=dev(d["k_r"].astype(np.float32)),
             pos=dev(d["pos"].astype(np.float32)), u=dev(d["u"]), v=dev(d["v"]))
    kw = dict(u=t["u"].data_ptr(), v=t["v"].data_ptr(), u_hat=d["u_hat"], v_hat=d["v_hat"],
              dB_min=d["db"][0], dB_max=d["db"][1])
    cases.append(("compat_grid_u8", d, t, sb.PREC_COMPAT, kw, True))
    # PRECISE, f64 k_r and positions
    d = synth.make("plain_small", seed=9, overrides=dict(P=400, S=424, n=192, extent=20.0))
    t = dict(phs=dev(d["phs"].view(np.float32)), k=dev(d["k_r"].astype(np.float32)),
             pos=dev(d["pos"].astype(np.float32)), k64=dev(d["k_r"]), pos64=dev(d["pos"]), r=dev(d["r"]))
    kw = dict(r=t["r"].data_ptr(), k_r64=t["k64"].data_ptr(), pos64=t["pos64"].data_ptr())
    cases.append(("precise_r", d, t, sb.PREC_PRECISE, kw, False))
    return cases


def _job(sb, d, t, prec, kw, out, u8):
    return sb.make_job(d["S"], d["P"], d["N_fft"], d["taylor"], d["nu"], d["nv"], d["delta_r"],
                       t["phs"].data_ptr(), t["k"].data_ptr(), t["pos"].data_ptr(), out.data_ptr(),
                       out_u8=u8.data_ptr() if u8 is not None else 0, precision=prec, **kw)


def _image(t):
    return t.cpu().numpy().view(np.complex128)[..., 0]


def test_noalloc_matches_device_entry_point_and_oracle(sb, ctx, oracle):
    import torch
    from sarbp_b200 import _lib
    L = _lib.lib()
    status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(4)
    cases = _cases(sb, torch)
    oracle_ref = {}
    results = []
    for name, d, t, prec, kw, want_u8 in cases * 2:  # each job twice, interleaved
        nu, nv = d["nu"], d["nv"]
        ref = torch.zeros((nv, nu, 2), dtype=torch.float64, device="cuda")
        ref_u8 = torch.zeros((nv, nu), dtype=torch.uint8, device="cuda") if want_u8 else None
        ctx.run_jobs([_job(sb, d, t, prec, kw, ref, ref_u8)])
        ctx.synchronize()
        got = torch.full((nv, nu, 2), float("nan"), dtype=torch.float64, device="cuda")
        got_u8 = torch.zeros((nv, nu), dtype=torch.uint8, device="cuda") if want_u8 else None
        job = _job(sb, d, t, prec, kw, got, got_u8)
        torch.cuda.synchronize()
        rc = L.sarbp_backprojection_noalloc(ctypes.byref(job), ctypes.c_void_p(stream),
                                            ctypes.c_void_p(status.data_ptr()))
        assert rc == 0, L.sarbp_last_error()
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        a, b = _image(got), _image(ref)
        assert np.all(np.isfinite(a))
        e_dev = rel_l2(a, b)
        assert e_dev < TOL, (name, e_dev)
        if want_u8:
            assert np.array_equal(got_u8.cpu().numpy(), ref_u8.cpu().numpy()), name
        # the CPU oracle at sampled pixels (output-image coordinates)
        if name not in oracle_ref:
            idx = rng.choice(nu * nv, 2000, replace=False)
            r = d["r"] if "r" in d else oracle.pixel_locs(d["u"], d["v"], d["u_hat"], d["v_hat"])
            if prec == sb.PREC_PRECISE:
                want = oracle.backprojection(d["phs"], d["k_r"], d["taylor"], d["N_fft"], d["delta_r"],
                                             d["pos"], r, nu, nv, mode=oracle.MODE_FP64, out_idx=idx)
            else:
                want = oracle.backprojection(d["phs"], d["k_r"].astype(np.float32), d["taylor"], d["N_fft"],
                                             d["delta_r"], d["pos"].astype(np.float32), r, nu, nv,
                                             mode=oracle.MODE_REF, out_idx=idx)
            oracle_ref[name] = (idx, want)
        idx, want = oracle_ref[name]
        e_orc = rel_l2(a.ravel()[idx], want)
        assert e_orc < TOL, (name, e_orc)
        results.append((name, e_dev, e_orc))
    print("no-alloc rel-L2 (vs device entry point, vs oracle):",
          ["%s %.1e %.1e" % r for r in results])


def test_noalloc_rejects_jobs_larger_than_its_scratch(sb):
    from sarbp_b200 import _lib
    L = _lib.lib()
    # 4000 pulses x 8192 bins of (m, d) pairs alone need 500 MiB
    job = sb.make_job(2048, 4000, 8192, 17, 4096, 4096, 0.25, 16, 16, 16, 16, r=16)
    rc = L.sarbp_backprojection_noalloc(ctypes.byref(job), None, None)
    assert rc == _lib.ERR_UNSUPPORTED
    assert b"MiB" in L.sarbp_last_error()
    # N_fft above 16384 (the four-step FFT's work buffer) is not taken either
    job = sb.make_job(64, 8, 32768, 17, 32, 32, 0.25, 16, 16, 16, 16, r=16)
    assert L.sarbp_backprojection_noalloc(ctypes.byref(job), None, None) == _lib.ERR_UNSUPPORTED
