"""Batched uneven jobs: one batch call, the CUDA-graph plan and the launch
autotuner (the batched form of the hot path).

* Every job of a mixed batch gives the same image batched as alone (same
  launch shape: bit-identical, each pixel tile is formed by one CTA in the
  same order whatever else is in the work list).
* A plan replays the captured batch and re-reads the input arrays at each
  replay: doubling a phase history doubles that job's image exactly (the
  range compression and the accumulation are linear and a factor of 2 is
  exact in floating point) and leaves the other jobs unchanged.
* The autotuner returns a supported launch shape, caches it per shape
  signature, and the tuned batch matches the oracle (reference semantics,
  relative L2 <= 1e-4 on sampled pixels of every job).
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mixed_jobs():
    import torch
    from sarbp_b200 import synth
    from sarbp_b200.batch import DeviceJob
    cfgs = synth.batch_jobs(njobs=7, seed=11, sizes=(64, 128, 256), pulses=(64, 300),
                            samples=(128, 256))
    return [DeviceJob(c, torch, "cuda", u8=True) for c in cfgs]


def _images(jobs):
    return [j.image().copy() for j in jobs]


def _zero(jobs):
    import torch
    for j in jobs:
        j.out.zero_()
    torch.cuda.synchronize()  # the library's streams do not order after torch's


def test_batch_equals_alone(ctx, mixed_jobs):
    alone = []
    for j in mixed_jobs:
        ctx.run_jobs([j.job])
        ctx.synchronize()
        alone.append(j.image().copy())
    _zero(mixed_jobs)
    ctx.run_jobs([j.job for j in mixed_jobs])
    ctx.synchronize()
    for a, b in zip(alone, _images(mixed_jobs)):
        assert np.array_equal(a, b)


def test_plan_replays_reread_inputs(ctx, sb, mixed_jobs):
    import torch
    J = [j.job for j in mixed_jobs]
    ctx.run_jobs(J)
    ctx.synchronize()
    base = _images(mixed_jobs)
    u8_base = [j.out_u8.cpu().numpy().copy() for j in mixed_jobs]
    plan = sb.Plan(ctx, J)
    try:
        assert plan.kernels >= 5
        _zero(mixed_jobs)
        plan.launch()
        plan.wait()
        for a, b in zip(base, _images(mixed_jobs)):
            assert np.array_equal(a, b)
        for a, j in zip(u8_base, mixed_jobs):
            assert np.array_equal(a, j.out_u8.cpu().numpy())
        k = 2
        mixed_jobs[k].phs.mul_(2.0)
        torch.cuda.synchronize()
        plan.launch()
        plan.wait()
        got = _images(mixed_jobs)
        for i, (a, b) in enumerate(zip(base, got)):
            assert np.array_equal(b, 2.0 * a if i == k else a), i
    finally:
        mixed_jobs[2].phs.mul_(0.5)
        torch.cuda.synchronize()
        plan.close()


def test_autotune_and_oracle(ctx, oracle, mixed_jobs):
    from sarbp_b200 import _lib
    J = [j.job for j in mixed_jobs]
    tune, ms = ctx.autotune(J)
    assert ms > 0
    assert _lib.lib().sarbp_ctx_launch_count(ctx._h) > 0
    tune2, ms2 = ctx.autotune(J)
    assert tune2 == tune and ms2 == -1.0
    _zero(mixed_jobs)
    ctx.run_jobs(J, **tune)
    ctx.synchronize()
    rng = np.random.default_rng(5)
    for j in mixed_jobs:
        d = j.data
        r = oracle.pixel_locs(d["u"], d["v"], d["u_hat"], d["v_hat"])
        idx = rng.choice(j.nu * j.nv, size=min(2000, j.nu * j.nv), replace=False)
        want = oracle.backprojection(d["phs"], d["k_r"].astype(np.float32), d["taylor"], d["N_fft"],
                                     d["delta_r"], d["pos"].astype(np.float32), r, j.nu, j.nv,
                                     out_idx=idx, taylor_mode=d["taylor_mode"])
        got = j.image().ravel()[idx]
        assert rel_l2(got, want) < 1e-4, (j.nu, j.P, j.S)


@pytest.mark.parametrize("lo,hi", [(-40.0, 0.0), (-3.0, -1.0), (-80.0, 10.0)])
def test_u8_stage_equals_reference_formula(ctx, oracle, mixed_jobs, lo, hi):
    """The fused u8 stage (f32 decision with an f64 fallback near grey-level
    edges) gives exactly the reference's u8 (img_output.cpp:18-51 through the
    oracle) of the image it wrote, for wide and narrow display ranges."""
    import torch
    for j in mixed_jobs:
        j.job.dB_min, j.job.dB_max = lo, hi
    _zero(mixed_jobs)
    ctx.run_jobs([j.job for j in mixed_jobs])
    ctx.synchronize()
    for j in mixed_jobs:
        img = j.image()
        want = oracle.img_output_u8(oracle.img_output_to_dB(img), lo, hi)
        got = j.out_u8.cpu().numpy()
        assert np.array_equal(got, want), (j.nu, int((got != want).sum()))
    d = mixed_jobs[0].data.get("db", (-40.0, 0.0))
    for j in mixed_jobs:
        j.job.dB_min, j.job.dB_max = d


def test_taylor_above_30_db_float_window_matches_oracle(ctx, sb, oracle):
    """Side-lobe levels 31-35 dB (where the reference's Int32-division window
    is undefined) run with the float-quotient window (TAYLOR_FLOAT) and match
    the oracle's float-division window at reference precision; the same jobs
    with the reference's window are rejected."""
    import torch
    from sarbp_b200 import synth
    from sarbp_b200.batch import DeviceJob
    cfgs = synth.batch_jobs(njobs=5, seed=17, sizes=(128, 256), pulses=(150, 400), samples=(256, 512),
                            taylors=(31, 35))
    jobs = [DeviceJob(c, torch, "cuda") for c in cfgs]
    assert all(j.data["taylor_mode"] == sb.TAYLOR_FLOAT for j in jobs)
    ctx.run_jobs([j.job for j in jobs])
    ctx.synchronize()
    rng = np.random.default_rng(8)
    for j in jobs:
        d = j.data
        r = oracle.pixel_locs(d["u"], d["v"], d["u_hat"], d["v_hat"])
        idx = rng.choice(j.nu * j.nv, size=1500, replace=False)
        want = oracle.backprojection(d["phs"], d["k_r"].astype(np.float32), d["taylor"], d["N_fft"],
                                     d["delta_r"], d["pos"].astype(np.float32), r, j.nu, j.nv,
                                     out_idx=idx, taylor_mode=1)
        assert rel_l2(j.image().ravel()[idx], want) < 1e-4, (d["taylor"], j.nu, j.P)
    ref_job = jobs[0].job
    ref_job.taylor_mode = sb.TAYLOR_REF
    with pytest.raises(sb.SarbpError) as e:
        ctx.run_jobs([ref_job])
    assert e.value.code == sb.ERR_INVALID and b"30 dB" in str(e.value).encode()
    ref_job.taylor_mode = sb.TAYLOR_FLOAT
