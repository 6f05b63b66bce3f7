"""Pulse-chunked image formation (sarbp_accum_*, sarbp_backprojection_streamed).

* The image formed from K chunks, added in any order, equals the one-shot
  image of the same job to relative L2 <= 1e-5 (only the f32 summation
  order differs) and the CPU oracle to <= 1e-4, for odd and even pulse
  counts (the reference's double fftshift pairs phase-history row q with
  antenna position (q - P mod 2) mod P), narrow and wide tiles, COMPAT and
  PRECISE.
* Host rows (pageable or pinned) give the same image bit for bit as device
  rows; reset() starts a new aperture (twice the phase history gives
  exactly twice the image).
* Misuse is an error code: a pulse added twice, finalize before all pulses,
  a chunk over max_chunk or outside the aperture.
* A 4096^2 x 4000 job (N_fft 8192) is formed under a 1.25 GB device cap,
  under half its one-shot footprint, and matches the one-shot image.
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL_ONE_SHOT = 1e-5
TOL_ORACLE = 1e-4


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _setup(sb, torch, d, prec, u8=False):
    """Device arrays of a synthetic job and two Jobs over them: one-shot
    (output o1) and chunked (output o2)."""
    t = dict(phs=_dev(torch, d["phs"].view(np.float32)), k=_dev(torch, d["k_r"].astype(np.float32)),
             pos=_dev(torch, d["pos"].astype(np.float32)), k64=_dev(torch, d["k_r"]), pos64=_dev(torch, d["pos"]),
             u=_dev(torch, d["u"]), v=_dev(torch, d["v"]))
    nu, nv = d["nu"], d["nv"]
    outs = [torch.zeros((nv, nu, 2), dtype=torch.float64, device="cuda") for _ in range(2)]
    u8s = [torch.zeros((nv, nu), dtype=torch.uint8, device="cuda") if u8 else None for _ in range(2)]
    jobs = []
    for o, q in zip(outs, u8s):
        jobs.append(sb.make_job(d["S"], d["P"], d["N_fft"], d["taylor"], nu, nv, d["delta_r"], t["phs"].data_ptr(),
                                t["k"].data_ptr(), t["pos"].data_ptr(), o.data_ptr(), u=t["u"].data_ptr(),
                                v=t["v"].data_ptr(), u_hat=d["u_hat"], v_hat=d["v_hat"], k_r64=t["k64"].data_ptr(),
                                pos64=t["pos64"].data_ptr(), out_u8=q.data_ptr() if q is not None else 0,
                                dB_min=d["db"][0], dB_max=d["db"][1], precision=prec,
                                taylor_mode=d.get("taylor_mode", 0)))
    return t, outs, u8s, jobs


def _img(t):
    return t.cpu().numpy().view(np.complex128)[..., 0]


def _chunks(P, sizes):
    out, q = [], 0
    for s in sizes:
        if q >= P:
            break
        out.append((q, min(s, P - q)))
        q += s
    if q < P:
        out.append((q, P - q))
    return out


def _oracle(oracle, d, prec, idx):
    r = oracle.pixel_locs(d["u"], d["v"], d["u_hat"], d["v_hat"])
    if prec == 1:
        return oracle.backprojection(d["phs"], d["k_r"], d["taylor"], d["N_fft"], d["delta_r"], d["pos"], r,
                                     d["nu"], d["nv"], mode=oracle.MODE_FP64, out_idx=idx)
    return oracle.backprojection(d["phs"], d["k_r"].astype(np.float32), d["taylor"], d["N_fft"], d["delta_r"],
                                 d["pos"].astype(np.float32), r, d["nu"], d["nv"], mode=oracle.MODE_REF,
                                 out_idx=idx)


CASES = [
    # name, synth overrides, precision, chunk sizes (added in reverse order)
    ("odd_P_compat", dict(n=256, extent=25.0), 0, (100, 150, 219)),
    ("even_P_precise", dict(P=400, n=200, extent=20.0), 1, (64, 64, 64, 64, 64, 64, 16)),
    ("wide_tiles", dict(P=301, S=256, n=128, extent=80.0, R0=3000.0), 0, (120, 120, 61)),
    # N_fft 32768: each chunk range-compressed by the four-step FFT
    ("four_step_fft", dict(P=97, S=8192, df=1.5e6 * 424 / 8192, n=128, extent=20.0), 0, (40, 40, 17)),
]


@pytest.mark.parametrize("name,over,prec,sizes", CASES)
def test_chunks_equal_one_shot_and_oracle(sb, ctx, oracle, name, over, prec, sizes):
    import torch
    from sarbp_b200 import synth
    d = synth.make("plain_small", seed=3, with_r=False, overrides=over)
    t, outs, u8s, jobs = _setup(sb, torch, d, prec, u8=True)
    ctx.run_jobs([jobs[0]])
    ctx.synchronize()
    chunks = _chunks(d["P"], sizes)
    acc = sb.Accumulator(ctx, jobs[1], max(sizes))
    try:
        for q0, n in reversed(chunks):
            acc.add_device(q0, n, t["phs"].data_ptr() + q0 * d["S"] * 8)
        acc.finalize()
        acc.wait()
    finally:
        acc.close()
    one, chk = _img(outs[0]), _img(outs[1])
    assert np.all(np.isfinite(chk))
    e1 = rel_l2(chk, one)
    idx = np.random.default_rng(2).choice(d["nu"] * d["nv"], 2000, replace=False)
    e2 = rel_l2(chk.ravel()[idx], _oracle(oracle, d, prec, idx))
    print("%s: %d chunks, rel-L2 vs one-shot %.2e, vs oracle %.2e" % (name, len(chunks), e1, e2))
    assert e1 < TOL_ONE_SHOT
    assert e2 < TOL_ORACLE
    # u8 of the chunked image is the reference's u8 of that image
    want = oracle.img_output_u8(oracle.img_output_to_dB(chk), d["db"][0], d["db"][1])
    assert np.array_equal(u8s[1].cpu().numpy(), want)


def test_host_rows_match_device_rows_and_reset(sb, ctx):
    import torch
    from sarbp_b200 import synth
    d = synth.make("plain_small", seed=6, with_r=False, overrides=dict(P=333, S=300, n=160, extent=20.0))
    t, outs, _, jobs = _setup(sb, torch, d, 0)
    chunks = _chunks(d["P"], (90, 90, 90))
    acc = sb.Accumulator(ctx, jobs[0], 90)
    try:
        for q0, n in chunks:
            acc.add_device(q0, n, t["phs"].data_ptr() + q0 * d["S"] * 8)
        acc.finalize()
        acc.wait()
        dev_img = _img(outs[0]).copy()
        # pageable host rows
        acc.reset()
        for q0, n in chunks:
            acc.add(q0, d["phs"][q0:q0 + n])
        acc.finalize()
        acc.wait()
        assert np.array_equal(_img(outs[0]), dev_img)
        # pinned host rows, twice the phase history
        pinned = torch.from_numpy((2 * d["phs"]).view(np.float32).copy()).pin_memory().numpy().view(np.complex64)
        acc.reset()
        for q0, n in chunks:
            acc.add(q0, pinned[q0:q0 + n])
        acc.finalize()
        acc.wait()
        assert np.array_equal(_img(outs[0]), 2.0 * dev_img)
    finally:
        acc.close()


def test_misuse_is_an_error_code(sb, ctx):
    import torch
    from sarbp_b200 import _lib, synth
    d = synth.make("plain_small", seed=7, with_r=False, overrides=dict(P=100, S=128, n=64, extent=10.0))
    t, outs, _, jobs = _setup(sb, torch, d, 0)
    acc = sb.Accumulator(ctx, jobs[0], 40)
    p = t["phs"].data_ptr()
    try:
        with pytest.raises(sb.SarbpError) as e:
            acc.add_device(0, 41, p)
        assert e.value.code == _lib.ERR_INVALID
        with pytest.raises(sb.SarbpError) as e:
            acc.add_device(80, 30, p)
        assert e.value.code == _lib.ERR_INVALID
        acc.add_device(0, 40, p)
        with pytest.raises(sb.SarbpError) as e:
            acc.add_device(30, 20, p)
        assert e.value.code == _lib.ERR_STATE
        with pytest.raises(sb.SarbpError) as e:
            acc.finalize()
        assert e.value.code == _lib.ERR_STATE
        acc.add_device(40, 40, p)
        acc.add_device(80, 20, p)
        acc.finalize()
        acc.wait()
        with pytest.raises(sb.SarbpError) as e:
            acc.add_device(0, 10, p)
        assert e.value.code == _lib.ERR_STATE
    finally:
        acc.close()
    jobs[1].precision = sb.PREC_NAIVE
    with pytest.raises(sb.SarbpError) as e:
        sb.Accumulator(ctx, jobs[1], 10)
    assert e.value.code == _lib.ERR_UNSUPPORTED


def test_large_job_under_a_device_memory_cap(sb, ctx, oracle):
    """4096^2 x 4000 pulses x 2048 samples (N_fft 8192) at 20 km: the
    one-shot footprint is several GB; streamed under a 1.25 GB cap the image
    equals the one-shot image and the FP64 oracle at sampled pixels."""
    import torch
    from sarbp_b200 import synth
    from sarbp_b200.batch import HostJob
    cfg = dict(synth.CONFIGS["precision"], nscat=40, clutter=0)
    d = synth.make("precision", seed=5, with_r=False, overrides=cfg)
    hj = HostJob(dict(cfg, seed=5), data=d)
    out_s = np.zeros((d["nv"], d["nu"]), np.complex128)
    job_h = hj.job(out_s, precision=sb.PREC_PRECISE)
    cap = 1.25e9
    one_shot = sb.job_device_bytes(job_h, precision=sb.PREC_PRECISE)
    assert one_shot > 2 * cap
    C, used = sb.backprojection_streamed(ctx, job_h, cap, precision=sb.PREC_PRECISE)
    assert used <= cap and C < d["P"]
    assert sb.job_device_bytes(job_h, chunk_pulses=C, precision=sb.PREC_PRECISE) <= cap
    # one-shot on the device for comparison
    t, outs, _, jobs = _setup(sb, torch, d, sb.PREC_PRECISE)
    ctx.run_jobs([jobs[0]])
    ctx.synchronize()
    one = _img(outs[0])
    e1 = rel_l2(out_s, one)
    idx = np.random.default_rng(11).choice(d["nu"] * d["nv"], 1000, replace=False)
    e2 = rel_l2(out_s.ravel()[idx], _oracle(oracle, d, 1, idx))
    print("streamed 4096^2 x 4000: chunk %d pulses, %.2f GB held (one-shot %.2f GB); rel-L2 vs one-shot %.2e, "
          "vs FP64 oracle %.2e" % (C, used / 1e9, one_shot / 1e9, e1, e2))
    assert e1 < TOL_ONE_SHOT
    assert e2 < TOL_ORACLE
