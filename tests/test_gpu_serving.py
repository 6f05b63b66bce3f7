"""The serving loop (continuous batching under an HBM budget).

* A request's image is the same alone and in a mix (bit for bit): the
  server fixes the launch shape, and each pixel tile is formed by one CTA
  whatever else shares the batch.
* Served images in PREC_PRECISE agree with the FP64 oracle to relative L2
  <= 1e-3 (the serving target) on a 5 % sample of the requests, at
  sampled pixels.
* Admission by footprint: requests that cannot fit the budget of an idle
  server fail with ERR_ADMISSION; the others are served with the budget
  never exceeded; overlapping submissions are batched.
"""
import time

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pool():
    from sarbp_b200 import synth
    from sarbp_b200.batch import HostJob
    cfgs = synth.batch_jobs(njobs=6, seed=21, sizes=(128, 256), pulses=(100, 400), samples=(256, 512))
    return [HostJob(c) for c in cfgs]


def _submit(srv, hj, precision):
    out, u8 = hj.new_outputs()
    job = hj.job(out, u8, precision=precision)
    rid = srv.submit(job, keep=(out, u8))
    return rid, out


def test_same_alone_and_in_mix(ctx, sb, pool):
    srv = sb.Server(ctx, hbm_cap_bytes=8e9, lanes=2, max_batch=8, precision=sb.PREC_PRECISE)
    try:
        rid, alone = _submit(srv, pool[0], sb.PREC_PRECISE)
        assert srv.wait(rid, 60.0) == 0
        mix = []
        for i in range(24):
            hj = pool[(i * 5) % len(pool)]
            mix.append((hj, *_submit(srv, hj, sb.PREC_PRECISE)))
        for hj, r, out in mix:
            assert srv.wait(r, 60.0) == 0
        twins = [out for hj, r, out in mix if hj is pool[0]]
        assert twins
        for out in twins:
            assert np.array_equal(out, alone)
        st = srv.stats()
        assert st["completed"] == 25 and st["batches"] >= 2
        assert st["peak_bytes"] <= 8e9
        for hj, r, out in mix:
            s, a, d = srv.times(r)
            assert 0 <= s <= a <= d
    finally:
        srv.close()


def test_served_vs_fp64_sample(ctx, sb, oracle, pool):
    srv = sb.Server(ctx, hbm_cap_bytes=8e9, lanes=2, max_batch=8, precision=sb.PREC_PRECISE)
    try:
        reqs = []
        for i in range(40):
            hj = pool[i % len(pool)]
            reqs.append((hj, *_submit(srv, hj, sb.PREC_PRECISE)))
        for _, r, _ in reqs:
            assert srv.wait(r, 120.0) == 0
    finally:
        srv.close()
    rng = np.random.default_rng(3)
    sample = rng.choice(len(reqs), size=max(2, len(reqs) // 20), replace=False)
    for k in sample:
        hj, _, out = reqs[k]
        d = hj.data
        r = oracle.pixel_locs(d["u"], d["v"], d["u_hat"], d["v_hat"])
        idx = rng.choice(hj.nu * hj.nv, 1500, replace=False)
        ref = oracle.backprojection(d["phs"], d["k_r"], d["taylor"], d["N_fft"], d["delta_r"], d["pos"], r,
                                    hj.nu, hj.nv, mode=oracle.MODE_FP64, out_idx=idx,
                                    taylor_mode=d["taylor_mode"])
        e = rel_l2(out.ravel()[idx], ref)
        print("served request %d (%dx%d, %d pulses): rel-L2 vs FP64 %.2e" % (k, hj.nu, hj.nv, hj.P, e))
        assert e < 1e-3


def test_admission_by_footprint(ctx, sb, pool):
    from sarbp_b200 import _lib, synth
    from sarbp_b200.batch import HostJob
    cap = 256e6
    srv = sb.Server(ctx, hbm_cap_bytes=cap, lanes=2, max_batch=4, precision=sb.PREC_COMPAT)
    try:
        big = HostJob(synth.batch_jobs(njobs=1, seed=2, sizes=(2048,), pulses=(1500, 1600),
                                       samples=(1024,))[0])
        rid_big, _ = _submit(srv, big, sb.PREC_COMPAT)
        rids = [_submit(srv, pool[i % len(pool)], sb.PREC_COMPAT)[0] for i in range(12)]
        assert srv.wait(rid_big, 60.0) == _lib.ERR_ADMISSION
        for r in rids:
            assert srv.wait(r, 60.0) == 0
        st = srv.stats()
        assert 0 < st["peak_bytes"] <= cap
        assert st["completed"] == 13
    finally:
        srv.close()


def test_wait_times_out_while_queued(ctx, sb, pool):
    from sarbp_b200 import _lib
    srv = sb.Server(ctx, hbm_cap_bytes=8e9, lanes=1, max_batch=1)
    try:
        rids = [_submit(srv, pool[i % len(pool)], sb.PREC_COMPAT)[0] for i in range(6)]
        last = rids[-1]
        # the last of six one-request batches on one lane cannot be done at once
        t0 = time.perf_counter()
        rc = srv.wait(last, 0.0)
        assert rc in (0, _lib.ERR_TIMEOUT)
        assert time.perf_counter() - t0 < 1.0
        for r in rids:
            assert srv.wait(r, 60.0) == 0
    finally:
        srv.close()


def test_registered_aperture_skips_upload_and_range_compression(ctx, sb, pool):
    """A phase history registered once stays resident: requests on it give
    the same image, bit for bit, as requests that bring the phase history,
    the server copies only their image-plane axes, and no pulse is
    range-compressed after the registration."""
    from sarbp_b200 import _lib
    srv = sb.Server(ctx, hbm_cap_bytes=8e9, lanes=2, max_batch=8, precision=sb.PREC_PRECISE)
    try:
        hj = pool[1]
        rid, direct = _submit(srv, hj, sb.PREC_PRECISE)
        assert srv.wait(rid, 60.0) == 0
        base_use = srv.stats()["in_use_bytes"]
        dummy = hj.new_outputs()[0]
        ap = srv.register(hj.job(dummy, precision=sb.PREC_PRECISE))
        c0 = srv.counters()
        assert srv.stats()["in_use_bytes"] > base_use  # resident profiles are charged
        outs = []
        for _ in range(6):
            out = hj.new_outputs()[0]
            outs.append((srv.submit_on(ap, hj.job(out), keep=out), out))
        for r, out in outs:
            assert srv.wait(r, 60.0) == 0
            assert np.array_equal(out, direct)
        c1 = srv.counters()
        assert c1["rc_pulses"] == c0["rc_pulses"]
        assert c1["resident_requests"] - c0["resident_requests"] == 6
        assert c1["h2d_bytes"] - c0["h2d_bytes"] == 6 * (hj.u.nbytes + hj.v.nbytes)
        with pytest.raises(sb.SarbpError) as e:
            srv.submit_on(ap + 100, hj.job(dummy))
        assert e.value.code == _lib.ERR_INVALID
        srv.unregister(ap)
        assert srv.stats()["in_use_bytes"] == base_use
        with pytest.raises(sb.SarbpError):
            srv.unregister(ap)
    finally:
        srv.close()


def test_registered_aperture_with_four_step_fft(ctx, sb):
    """An aperture whose N_fft (32768: 8192 samples at -u 2) takes the
    four-step range compression, registered once: its requests give the
    same image bit for bit as a request that brings the phase history."""
    from sarbp_b200 import synth
    from sarbp_b200.batch import HostJob
    cfg = dict(synth.batch_jobs(njobs=1, seed=31)[0], P=120, S=8192, df=1.5e6 * 424 / 8192, n=128,
               extent=20.0, upsample=2, taylor=20, taylor_mode=0)
    hj = HostJob(cfg)
    assert hj.data["N_fft"] == 32768
    srv = sb.Server(ctx, hbm_cap_bytes=8e9, lanes=2, max_batch=4, precision=sb.PREC_PRECISE)
    try:
        rid, direct = _submit(srv, hj, sb.PREC_PRECISE)
        assert srv.wait(rid, 60.0) == 0
        ap = srv.register(hj.job(hj.new_outputs()[0], precision=sb.PREC_PRECISE))
        out = hj.new_outputs()[0]
        r = srv.submit_on(ap, hj.job(out), keep=out)
        assert srv.wait(r, 60.0) == 0
        assert np.array_equal(out, direct) and np.all(np.isfinite(out))
        srv.unregister(ap)
    finally:
        srv.close()


def test_register_over_budget_is_an_admission_error(ctx, sb):
    from sarbp_b200 import _lib, synth
    from sarbp_b200.batch import HostJob
    srv = sb.Server(ctx, hbm_cap_bytes=64e6, lanes=1, max_batch=2, precision=sb.PREC_COMPAT)
    try:
        big = HostJob(synth.batch_jobs(njobs=1, seed=4, sizes=(256,), pulses=(1900, 2000), samples=(1024,))[0])
        with pytest.raises(sb.SarbpError) as e:
            srv.register(big.job(big.new_outputs()[0]))
        assert e.value.code == _lib.ERR_ADMISSION
        assert srv.stats()["in_use_bytes"] == 0
    finally:
        srv.close()


def test_streaming_aperture_beside_batches(ctx, sb, pool):
    """A streaming aperture (partial image on the device, phase history
    arriving in chunks) under the server's budget, while requests run: its
    image equals the stand-alone pulse-chunked accumulator's bit for bit and
    the one-shot image to 1e-5; its device memory is charged while open and
    returned at finish; one that does not fit is an admission error."""
    import torch
    from sarbp_b200 import _lib
    hj = pool[2]
    d = hj.data
    srv = sb.Server(ctx, hbm_cap_bytes=8e9, lanes=2, max_batch=8, precision=sb.PREC_PRECISE)
    try:
        base = srv.stats()["in_use_bytes"]
        out_s = hj.new_outputs()[0]
        sid = srv.open_stream(hj.job(out_s, precision=sb.PREC_PRECISE), 64)
        assert srv.stats()["in_use_bytes"] > base
        rids = [_submit(srv, pool[i % len(pool)], sb.PREC_PRECISE)[0] for i in range(6)]
        chunks = [(q, min(64, hj.P - q)) for q in range(0, hj.P, 64)]
        for q0, n in chunks:
            srv.stream_add(sid, q0, d["phs"][q0:q0 + n])
        srv.stream_finish(sid)
        for r in rids:
            assert srv.wait(r, 60.0) == 0
        assert srv.stats()["in_use_bytes"] == base
        with pytest.raises(sb.SarbpError) as e:
            srv.stream_add(sid, 0, d["phs"][:1])
        assert e.value.code == _lib.ERR_INVALID
    finally:
        srv.close()
    # the stand-alone accumulator and the one-shot image on the same data
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    t = dict(phs=dev(d["phs"].view(np.float32)), k=dev(d["k_r"].astype(np.float32)), k64=dev(d["k_r"]),
             pos=dev(d["pos"].astype(np.float32)), pos64=dev(d["pos"]), u=dev(d["u"]), v=dev(d["v"]))
    outs = [torch.zeros((hj.nv, hj.nu, 2), dtype=torch.float64, device="cuda") for _ in range(2)]
    jobs = [sb.make_job(hj.S, hj.P, d["N_fft"], d["taylor"], hj.nu, hj.nv, d["delta_r"], t["phs"].data_ptr(),
                        t["k"].data_ptr(), t["pos"].data_ptr(), o.data_ptr(), u=t["u"].data_ptr(),
                        v=t["v"].data_ptr(), u_hat=d["u_hat"], v_hat=d["v_hat"], k_r64=t["k64"].data_ptr(),
                        pos64=t["pos64"].data_ptr(), precision=sb.PREC_PRECISE, taylor_mode=d["taylor_mode"])
            for o in outs]
    acc = sb.Accumulator(ctx, jobs[0], 64)
    try:
        for q0, n in chunks:
            acc.add_device(q0, n, t["phs"].data_ptr() + q0 * hj.S * 8)
        acc.finalize()
        acc.wait()
    finally:
        acc.close()
    ctx.run_jobs([jobs[1]])
    ctx.synchronize()
    alone = outs[0].cpu().numpy().view(np.complex128)[..., 0]
    one = outs[1].cpu().numpy().view(np.complex128)[..., 0]
    assert np.array_equal(out_s, alone)
    assert rel_l2(out_s, one) < 1e-5
    small = sb.Server(ctx, hbm_cap_bytes=1e6, lanes=1, max_batch=1, precision=sb.PREC_PRECISE)
    try:
        with pytest.raises(sb.SarbpError) as e:
            small.open_stream(hj.job(hj.new_outputs()[0], precision=sb.PREC_PRECISE), 64)
        assert e.value.code == _lib.ERR_ADMISSION
    finally:
        small.close()


@pytest.mark.gpu
def test_streaming_aperture_from_two_threads(ctx, sb, pool):
    """Two host threads add interleaved pulse chunks to one streaming
    aperture at once (the library serialises calls on a stream): the image
    equals the one-thread image to 1e-6 (the chunks' partial sums are added
    in another order); an add racing the finish either lands before it or is
    refused as a finished stream."""
    import threading
    from sarbp_b200 import _lib
    hj = pool[3]
    d = hj.data
    chunks = [(q, min(48, hj.P - q)) for q in range(0, hj.P, 48)]
    srv = sb.Server(ctx, hbm_cap_bytes=8e9, lanes=2, max_batch=8, precision=sb.PREC_PRECISE)
    try:
        out1 = hj.new_outputs()[0]
        sid = srv.open_stream(hj.job(out1, precision=sb.PREC_PRECISE), 48)
        for q0, n in chunks:
            srv.stream_add(sid, q0, d["phs"][q0:q0 + n])
        srv.stream_finish(sid)

        out2 = hj.new_outputs()[0]
        sid = srv.open_stream(hj.job(out2, precision=sb.PREC_PRECISE), 48)
        errors = []

        def worker(part):
            try:
                for q0, n in part:
                    srv.stream_add(sid, q0, d["phs"][q0:q0 + n])
            except Exception as exc:  # reported below
                errors.append(exc)

        threads = [threading.Thread(target=worker, args=(chunks[k::2],)) for k in range(2)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        assert not errors
        srv.stream_finish(sid)
        assert rel_l2(out2, out1) < 1e-6

        # an add racing the finish: lands first (then the finish sees one
        # pulse chunk missing) or is refused as a finished stream
        out3 = hj.new_outputs()[0]
        sid = srv.open_stream(hj.job(out3, precision=sb.PREC_PRECISE), 48)
        for q0, n in chunks[:-1]:
            srv.stream_add(sid, q0, d["phs"][q0:q0 + n])
        q0, n = chunks[-1]
        codes = []

        def late_add():
            try:
                srv.stream_add(sid, q0, d["phs"][q0:q0 + n])
                codes.append(0)
            except sb.SarbpError as exc:
                codes.append(exc.code)

        t = threading.Thread(target=late_add)
        t.start()
        try:
            srv.stream_finish(sid)
            fin = 0
        except sb.SarbpError as exc:
            fin = exc.code
        t.join()
        assert (codes, fin) in (([0], 0), ([_lib.ERR_INVALID], _lib.ERR_STATE))
        if fin == 0:
            assert np.array_equal(out3, out1) or rel_l2(out3, out1) < 1e-6
        assert srv.stats()["in_use_bytes"] == 0
    finally:
        srv.close()
