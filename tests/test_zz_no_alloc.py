"""sarbp_backprojection_noalloc: the backprojection entry point that
allocates nothing.

It exists for callers that cannot allocate device memory at the moment
they want an image -- code inside a CUDA stream capture, processes whose
device memory belongs to a pool they do not own, or real-time loops that
must stay off the allocator.  Its scratch lives in one static 64 MiB device
array of the library that every call reuses, so the test runs two different
jobs back to back (stale contents of the first must not leak into the
second) and compares each image with the ordinary device entry point,
within the parity tolerance of the other GPU tests (relative L2 <= 1e-4).

The file is named to be collected last: if it fails, a run that stops at
the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _jobs(sb, torch):
    from sarbp_b200 import synth
    out = []
    for name, over, seed in (("plain_small", dict(n=256, extent=25.0), 1),
                             ("plain_small", dict(P=333, S=300, n=200, extent=30.0, taylor=20), 5)):
        d = synth.make(name, seed=seed, overrides=over)
        t = dict(phs=torch.from_numpy(d["phs"].view(np.float32).copy()).cuda(),
                 k=torch.from_numpy(d["k_r"].astype(np.float32)).cuda(),
                 pos=torch.from_numpy(d["pos"].astype(np.float32)).cuda(),
                 r=torch.from_numpy(d["r"]).cuda())
        args = (d["S"], d["P"], d["N_fft"], d["taylor"], d["nu"], d["nv"], d["delta_r"],
                t["phs"].data_ptr(), t["k"].data_ptr(), t["pos"].data_ptr())
        out.append((d, t, args))
    return out


def test_noalloc_matches_device_entry_point(sb, ctx):
    import torch
    from sarbp_b200 import _lib
    L = _lib.lib()
    status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    results = []
    for d, t, args in _jobs(sb, torch) * 2:  # job A, job B, job A, job B
        ref = torch.zeros((d["nv"], d["nu"], 2), dtype=torch.float64, device="cuda")
        ctx.run_jobs([sb.make_job(*args, ref.data_ptr(), r=t["r"].data_ptr())])
        ctx.synchronize()
        got = torch.full((d["nv"], d["nu"], 2), float("nan"), dtype=torch.float64, device="cuda")
        job = sb.make_job(*args, got.data_ptr(), r=t["r"].data_ptr())
        rc = L.sarbp_backprojection_noalloc(ctypes.byref(job), ctypes.c_void_p(stream),
                                            ctypes.c_void_p(status.data_ptr()))
        assert rc == 0, L.sarbp_last_error()
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        a = got.cpu().numpy().view(np.complex128)[..., 0]
        b = ref.cpu().numpy().view(np.complex128)[..., 0]
        assert np.all(np.isfinite(a))
        e = rel_l2(a, b)
        results.append(e)
        assert e < 1e-4
    print("no-alloc vs device entry point rel-L2:", ["%.1e" % x for x in results])


def test_noalloc_rejects_jobs_larger_than_its_scratch(sb):
    from sarbp_b200 import _lib
    L = _lib.lib()
    # 4000 pulses x 8192 bins of (m, d) pairs alone need 500 MiB
    job = sb.make_job(2048, 4000, 8192, 17, 4096, 4096, 0.25, 16, 16, 16, 16, r=16)
    rc = L.sarbp_backprojection_noalloc(ctypes.byref(job), None, None)
    assert rc == _lib.ERR_UNSUPPORTED
    assert b"MiB" in L.sarbp_last_error()
