"""CUDA path against the CPU oracle (needs a B200).

Tolerances (stated per test):
  * COMPAT precision vs the reference-precision oracle: complex-image
    relative L2 <= 1e-4 and dB max |diff| <= 0.05 dB over the pixels the
    oracle shows within the display range (dB >= dB_min).
  * PRECISE precision vs the FP64 oracle: relative L2 <= 1e-4 (the target
    is 1e-3).
  * range profiles (FP32 FFT) vs the f64 oracle: relative L2 <= 2e-6.
"""
import numpy as np
import pytest

from conftest import db_max_diff, rel_l2

pytestmark = pytest.mark.gpu

REL_COMPAT = 1e-4
REL_PRECISE = 1e-4
DB_TOL = 0.05


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


@pytest.fixture(scope="module")
def cfg1():
    from sarbp_b200 import synth
    return synth.make("plain_small", seed=1)


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _job_for_rc(sb, torch, phs, k_r, taylor, N, pos):
    P, S = phs.shape
    t_phs = _dev(torch, phs.view(np.float32))
    t_k = _dev(torch, np.asarray(k_r, np.float32))
    t_pos = _dev(torch, np.asarray(pos, np.float32))
    j = sb.make_job(S, P, N, taylor, 0, 0, 1.0, t_phs.data_ptr(), t_k.data_ptr(), t_pos.data_ptr(), 0)
    return j, (t_phs, t_k, t_pos)


@pytest.mark.parametrize("P,S,N", [(469, 424, 1024), (470, 424, 1024), (33, 100, 16), (9, 7, 32),
                                   (65, 300, 512), (17, 1000, 2048), (1999, 1024, 4096),
                                   (5, 2048, 8192), (3, 4000, 16384), (12, 64, 128), (7, 120, 256),
                                   (31, 33, 64), (5, 8192, 32768), (4, 10000, 65536), (3, 6000, 131072),
                                   (1100, 64, 32768), (3, 40000, 32768)])
def test_range_compress_matches_oracle(sb, ctx, oracle, torch, P, S, N):
    """Fused window/filter/pad/shift + Stockham FFT + shift vs the f64
    oracle for every radix schedule (N = 16 .. 16384), the four-step FFT
    above that (N = 32768 .. 131072; 1100 rows go through its work buffer in
    two batches), odd and even P, and N < S (the centre of the pulse is
    kept)."""
    rng = np.random.default_rng(P * 7 + S)
    phs = (rng.normal(size=(P, S)) + 1j * rng.normal(size=(P, S))).astype(np.complex64)
    k_r = rng.uniform(350, 400, size=S).astype(np.float32)
    pos = np.zeros((P, 3), np.float32)
    j, keep = _job_for_rc(sb, torch, phs, k_r, 17, N, pos)
    q = torch.empty((P, N, 2), dtype=torch.float32, device="cuda")
    ctx.range_compress_device(j, q.data_ptr())
    ctx.synchronize()
    Q = q.cpu().numpy().view(np.complex64)[..., 0]
    ref = oracle.range_compress(phs, k_r.astype(np.float64), 17, N, mode=oracle.MODE_REF)
    assert rel_l2(Q, ref) < 2e-6
    # row by row too (rows of very different energy)
    for p in range(0, P, max(1, P // 7)):
        assert rel_l2(Q[p], ref[p]) < 5e-6


@pytest.mark.parametrize("P,S,u", [(65, 8192, 2), (64, 3000, 6), (33, 12000, 6)])
def test_four_step_fft_full_image(ctx, oracle, sb, P, S, u):
    """N_fft above 16384 by the reference's rule (sarbp.cpp:258): S = 8192
    at -u 2 (the reference's Sandia runs) and S >= 2731 at the default -u 6
    give 32768 and more, range-compressed by the four-step FFT into the
    interpolation pairs; whole 128^2 image against the reference-precision
    oracle, compat tolerance."""
    from sarbp_b200 import synth
    d = synth.make("plain_small", seed=6,
                   overrides=dict(P=P, S=S, df=1.5e6 * 424 / S, n=128, extent=20.0, upsample=u))
    assert d["N_fft"] == sb.n_fft_for(S, u) and d["N_fft"] > 16384
    pos32, k32 = d["pos"].astype(np.float32), d["k_r"].astype(np.float32)
    img = ctx.backprojection_cuda(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], d["u"], d["v"],
                                  pos32, d["r"])
    ref = oracle.backprojection(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], pos32, d["r"],
                                d["nu"], d["nv"], mode=oracle.MODE_REF)
    e = rel_l2(img, ref)
    print("N_fft %d (S %d, -u %d): rel-L2 %.3e" % (d["N_fft"], S, u, e))
    assert e < REL_COMPAT
    assert db_max_diff(img, ref, d["db"][0]) < DB_TOL


def test_sandia_shape_sampled(ctx, oracle):
    """The reference's Sandia GPU runs' range axis (8192 samples, -u 2 ->
    N_fft 32768) on 2048 of its 8192 pulses and a 4096^2 image over 200 m:
    whole image on the GPU, 2048 sampled pixels against the oracle."""
    from sarbp_b200 import synth
    d = synth.make("sandia_8192", seed=7, overrides=dict(P=2048, n=4096, extent=200.0))
    assert d["N_fft"] == 32768
    pos32, k32 = d["pos"].astype(np.float32), d["k_r"].astype(np.float32)
    img = ctx.backprojection_cuda(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], d["u"], d["v"],
                                  pos32, d["r"])
    rng = np.random.default_rng(8)
    idx = rng.choice(d["nu"] * d["nv"], 2048, replace=False)
    ref = oracle.backproject(oracle.range_compress(d["phs"], k32, d["taylor"], d["N_fft"]), d["S"],
                             d["delta_r"], k32, pos32, d["r"], d["nu"], d["nv"], out_idx=idx)
    e = rel_l2(img.ravel()[idx], ref)
    print("sandia shape (2048 pulses) sampled rel-L2 %.3e" % e)
    assert e < REL_COMPAT


def test_compat_plain_small_full_image(ctx, oracle, cfg1):
    """plain_small (469 x 424 -> 512^2, Taylor 17): whole image, reference
    semantics (f32 pos, k_r) against the reference-precision oracle."""
    d = cfg1
    pos32 = d["pos"].astype(np.float32)
    k32 = d["k_r"].astype(np.float32)
    img = ctx.backprojection_cuda(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], d["u"], d["v"],
                                  pos32, d["r"])
    ref = oracle.backprojection(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], pos32, d["r"],
                                d["nu"], d["nv"], mode=oracle.MODE_REF)
    e = rel_l2(img, ref)
    dbd = db_max_diff(img, ref, d["db"][0])
    print("compat plain_small rel-L2 %.3e  dB max diff %.4f" % (e, dbd))
    assert e < REL_COMPAT
    assert dbd < DB_TOL


@pytest.mark.parametrize("R0,extent,n,u,az", [
    (400.0, 120.0, 256, 2, 0.0),    # near field: closed form (series order 3), wide tiles
    (2000.0, 80.0, 256, 2, 0.0),    # four-term series, wide tiles
    (10e3, 150.0, 256, 2, 0.0),     # far, coarse pixels (0.59 m): wide tiles, low orders
    (10e3, 20.0, 256, 2, 0.0),      # far, fine pixels: narrow tiles, two-term series
    (10e3, 60.0, 256, 6, 35.0),     # -u 6, pixels at the range resolution, plane turned 35 deg
    (3000.0, 60.0, 256, 6, -60.0),  # the same nearer, turned the other way
])
def test_geometry_regimes(ctx, oracle, R0, extent, n, u, az):
    """Standoff, pixel size, upsampling and image-plane orientation across
    the kernel's regimes (which series order a pulse needs, whether a tile is
    wide, how narrow a window the tile's line-of-sight extent allows)
    against the reference-precision oracle, whole image, compat tolerance."""
    from sarbp_b200 import synth
    d = synth.make("plain_small", seed=3, overrides=dict(R0=R0, extent=extent, n=n, upsample=u, az=az))
    pos32 = d["pos"].astype(np.float32)
    k32 = d["k_r"].astype(np.float32)
    img = ctx.backprojection_cuda(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], d["u"], d["v"],
                                  pos32, d["r"])
    ref = oracle.backprojection(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], pos32, d["r"],
                                d["nu"], d["nv"], mode=oracle.MODE_REF)
    e = rel_l2(img, ref)
    dbd = db_max_diff(img, ref, d["db"][0])
    print("R0 %.0f m, pixel %.3f m, -u %d, az %.0f: rel-L2 %.3e  dB max diff %.4f" % (R0, extent / n, u, az, e, dbd))
    assert e < REL_COMPAT
    assert dbd < DB_TOL


def test_precise_plain_small_vs_fp64(ctx, oracle, cfg1):
    d = cfg1
    img = ctx.backprojection_cuda(d["phs"], d["k_r"], d["taylor"], d["N_fft"], d["delta_r"], d["u"],
                                  d["v"], d["pos"], d["r"])
    ref = oracle.backprojection(d["phs"], d["k_r"], d["taylor"], d["N_fft"], d["delta_r"], d["pos"],
                                d["r"], d["nu"], d["nv"], mode=oracle.MODE_FP64)
    e = rel_l2(img, ref)
    print("precise plain_small rel-L2 vs FP64 %.3e" % e)
    assert e < REL_PRECISE
    assert db_max_diff(img, ref, d["db"][0]) < DB_TOL


def test_afrl_real_data(sb, ctx, oracle, afrl_input):
    """The reference's own AFRL input through img_plane_create, as in
    `sarbp -p HH_npy -d -30 -D 0 -t 17 -u 2 -s cuda` (README.md:55)."""
    a = afrl_input
    S, P = int(a["nsamples"][0]), int(a["npulses"][0])
    ip = sb.img_plane_create(S, P, float(a["delta_r"][0]), a["R_c"])
    N = sb.n_fft_for(S, 2)
    img = ctx.backprojection_cuda(a["phs"], a["k_r"], 17, N, float(a["delta_r"][0]), ip["u"], ip["v"],
                                  a["pos"], ip["pixel_locs"])
    ref = oracle.backprojection(a["phs"], a["k_r"].astype(np.float64), 17, N, float(a["delta_r"][0]),
                                a["pos"].astype(np.float64), ip["pixel_locs"], ip["nu"], ip["nv"],
                                mode=oracle.MODE_REF)
    e = rel_l2(img, ref)
    print("AFRL rel-L2 %.3e" % e)
    assert e < REL_COMPAT
    assert db_max_diff(img, ref, -30.0) < DB_TOL
    u8 = ctx.img_output_u8(ctx.img_output_to_dB(img), -30.0, 0.0)
    u8r = oracle.img_output_u8(oracle.img_output_to_dB(ref), -30.0, 0.0)
    assert np.mean(u8.astype(int) != u8r) < 0.01 and np.abs(u8.astype(int) - u8r).max() <= 1


def test_plain_large_full_size_sampled(ctx, oracle):
    """plain_large at full size (1999 x 1024 -> 2048^2, Taylor 30): the whole
    image on the GPU, 4096 sampled pixels from the oracle."""
    from sarbp_b200 import synth
    d = synth.make("plain_large", seed=2)
    pos32, k32 = d["pos"].astype(np.float32), d["k_r"].astype(np.float32)
    img = ctx.backprojection_cuda(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], d["u"], d["v"],
                                  pos32, d["r"])
    rng = np.random.default_rng(0)
    idx = rng.choice(d["nu"] * d["nv"], 4096, replace=False)
    ref = oracle.backproject(oracle.range_compress(d["phs"], k32, d["taylor"], d["N_fft"]), d["S"],
                             d["delta_r"], k32, pos32, d["r"], d["nu"], d["nv"], out_idx=idx)
    got = img.ravel()[idx]
    e = rel_l2(got, ref)
    print("plain_large sampled rel-L2 %.3e" % e)
    assert e < REL_COMPAT
    assert np.all(np.isfinite(img))


def test_largest_image_32768_squared_sampled(sb, torch, oracle):
    """A 32768^2 image (2^30 pixels, the size of the reference's largest
    Sandia runs) from plain_large's aperture in one device call on one GPU:
    pixel positions from the image-plane axes, the 17 GB image and ~75 GB
    of scratch on the device (its own context, released afterwards); 4096
    sampled pixels against the oracle at the reference's precision."""
    from sarbp_b200 import synth
    d = synth.make("plain_large", seed=4, with_r=False, overrides=dict(n=32768, extent=200.0))
    nu, nv = d["nu"], d["nv"]
    assert nu * nv == 1 << 30
    dev = torch.device("cuda", 0)
    pos32, k32 = d["pos"].astype(np.float32), d["k_r"].astype(np.float32)
    c = sb.Context(0)
    try:
        t = dict(phs=torch.from_numpy(d["phs"].view(np.float32).copy()).to(dev), k=torch.from_numpy(k32).to(dev),
                 pos=torch.from_numpy(pos32).to(dev), u=torch.from_numpy(d["u"]).to(dev),
                 v=torch.from_numpy(d["v"]).to(dev))
        out = torch.empty((nv, nu, 2), dtype=torch.float64, device=dev)
        job = sb.make_job(d["S"], d["P"], d["N_fft"], d["taylor"], nu, nv, d["delta_r"], t["phs"].data_ptr(),
                          t["k"].data_ptr(), t["pos"].data_ptr(), out.data_ptr(), u=t["u"].data_ptr(),
                          v=t["v"].data_ptr(), u_hat=d["u_hat"], v_hat=d["v_hat"])
        c.run_jobs([job])
        c.synchronize()
        rng = np.random.default_rng(5)
        ix, iy = rng.integers(0, nu, 4096), rng.integers(0, nv, 4096)
        rows = torch.from_numpy(nv - 1 - iy).to(dev)
        got = out[rows, torch.from_numpy(ix).to(dev)].cpu().numpy().view(np.complex128)[:, 0]
        del out, t
    finally:
        c.close()
        torch.cuda.empty_cache()
    # the sampled pixels' positions as img_plane.cpp:92-102 forms them
    uh, vh = np.asarray(d["u_hat"], np.float64), np.asarray(d["v_hat"], np.float64)
    r = np.stack([(uh[k] * d["u"][ix]) + (vh[k] * d["v"][iy]) for k in range(3)])
    ref = oracle.backproject(oracle.range_compress(d["phs"], k32, d["taylor"], d["N_fft"]), d["S"],
                             d["delta_r"], k32, pos32, r, r.shape[1], 1)[0]
    e = rel_l2(got, ref)
    print("32768^2 sampled rel-L2 %.3e" % e)
    assert e < REL_COMPAT
    assert np.all(np.isfinite(got))


def test_linearity_full_size(ctx):
    """BP(a x + b y) = a BP(x) + b BP(y) at plain_large size."""
    from sarbp_b200 import synth
    d = synth.make("plain_large", seed=3)
    rng = np.random.default_rng(1)
    y = (rng.normal(size=d["phs"].shape) + 1j * rng.normal(size=d["phs"].shape)).astype(np.complex64)
    a, b = 0.75 - 0.25j, 1.5j
    run = lambda ph: ctx.backprojection_cuda(ph, d["k_r"].astype(np.float32), d["taylor"], d["N_fft"],
                                             d["delta_r"], d["u"], d["v"], d["pos"].astype(np.float32),
                                             d["r"])
    lhs = run((a * d["phs"] + b * y).astype(np.complex64))
    rhs = a * run(d["phs"]) + b * run(y)
    assert rel_l2(lhs, rhs) < 2e-5


def test_point_target_focus(ctx):
    from sarbp_b200 import synth
    scat = np.array([[6.0, -9.0, 0.0, 1.0, 0.0]])
    phs, pos, k_r = synth.phase_history(1024, 999, 16.7e9, 0.59e6, 8e3, 45, 3, scat, 400, 1)
    dr = synth.C / (2 * 1024 * 0.59e6)
    g = synth.grid_plane(1024, 40.0, pos, dr, 1024, 999)
    r = synth.pixel_locs(g["u"], g["v"], g["u_hat"], g["v_hat"])
    img = ctx.backprojection_cuda(phs, k_r.astype(np.float32), 30, 4096, dr, g["u"], g["v"],
                                  pos.astype(np.float32), r)
    aimg = np.abs(img)
    y, x = np.unravel_index(aimg.argmax(), aimg.shape)
    loc = r[:, 1024 * (1024 - y - 1) + x]
    assert np.hypot(loc[0] - 6.0, loc[1] + 9.0) < 1.0
    assert aimg.max() > 1000 * np.median(aimg)


@pytest.mark.parametrize("tile", [(32, 16), (32, 64), (64, 16), (64, 32), (16, 32), (16, 64)])
def test_tile_shapes_agree(ctx, oracle, cfg1, tile):
    d = cfg1
    pos32, k32 = d["pos"].astype(np.float32), d["k_r"].astype(np.float32)
    img = ctx.backprojection_cuda(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], d["u"], d["v"],
                                  pos32, d["r"], tile=tile)
    ref = oracle.backprojection(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], pos32, d["r"],
                                d["nu"], d["nv"], mode=oracle.MODE_REF)
    assert rel_l2(img, ref) < REL_COMPAT


@pytest.mark.parametrize("parts", [0, 3, 7, 16])
def test_pulse_parts_match_one_item_per_tile(ctx, oracle, parts):
    """Tiles formed as several (tile, pulse part) work items, each part's
    sums stored in its own partial image and added in part order by the
    combine kernel (0: the part count chosen for the job, here 4 for 64
    tiles and 469 pulses).  Near field (400 m): wide tiles, series orders 1
    to 3, odd P (the fftshifted pulse axis), P not a multiple of the part
    count.  Against one item per tile: relative L2 <= 1e-5 (the same terms
    summed in another order, and a chunk's series order taken over other
    pulses); against the oracle at the compat tolerance."""
    from sarbp_b200 import synth
    d = synth.make("plain_small", seed=3, overrides=dict(R0=400.0, extent=120.0, n=256, upsample=2))
    pos32, k32 = d["pos"].astype(np.float32), d["k_r"].astype(np.float32)
    run = lambda **kw: ctx.backprojection_cuda(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], d["u"],
                                               d["v"], pos32, d["r"], **kw)
    one = run(pulse_parts=1)
    img = run(pulse_parts=parts)
    assert np.array_equal(img, run(pulse_parts=parts))  # deterministic
    ref = oracle.backprojection(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], pos32, d["r"],
                                d["nu"], d["nv"], mode=oracle.MODE_REF)
    e_one, e_ref = rel_l2(img, one), rel_l2(img, ref)
    print("pulse parts %d: rel-L2 vs one item per tile %.3e, vs oracle %.3e" % (parts, e_one, e_ref))
    assert 0 < e_one < 1e-5
    assert e_ref < REL_COMPAT
    assert db_max_diff(img, ref, d["db"][0]) < DB_TOL


@pytest.mark.parametrize("chunk,persistent", [(4, 0), (16, 2), (64, 2), (256, 1)])
def test_pulse_chunk_and_launch_modes(ctx, oracle, cfg1, chunk, persistent):
    d = cfg1
    pos32, k32 = d["pos"].astype(np.float32), d["k_r"].astype(np.float32)
    img = ctx.backprojection_cuda(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], d["u"], d["v"],
                                  pos32, d["r"], pulse_chunk=chunk, persistent=persistent)
    ref = oracle.backprojection(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], pos32, d["r"],
                                d["nu"], d["nv"], mode=oracle.MODE_REF)
    assert rel_l2(img, ref) < REL_COMPAT


@pytest.mark.parametrize("tile,chunk,stage", [((32, 32), 64, 3264), ((32, 64), 32, 3424), ((16, 64), 128, 2944)])
def test_two_ctas_with_grown_staging(ctx, oracle, cfg1, tile, chunk, stage):
    """2 CTAs/SM with the staging buffer grown into the third CTA's shared
    memory (the autotuner's 2-CTA candidates): same tolerance as above."""
    d = cfg1
    pos32, k32 = d["pos"].astype(np.float32), d["k_r"].astype(np.float32)
    img = ctx.backprojection_cuda(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], d["u"], d["v"],
                                  pos32, d["r"], tile=tile, pulse_chunk=chunk, min_blocks=2, stage_cap=stage)
    ref = oracle.backprojection(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], pos32, d["r"],
                                d["nu"], d["nv"], mode=oracle.MODE_REF)
    assert rel_l2(img, ref) < REL_COMPAT


@pytest.mark.parametrize("P,S,nu,nv", [(2, 2, 1, 1), (3, 17, 7, 13), (64, 100, 33, 65), (200, 50, 100, 3)])
def test_ragged_sizes(ctx, oracle, P, S, nu, nv):
    """Tiny and ragged shapes: edge tiles, P and S far from powers of two,
    N_fft below S (the pulse centre is kept); also with 16 pulse parts per
    tile requested (one part per pulse when P < 16)."""
    from sarbp_b200 import synth
    scat = synth.scene(4, 5.0, 0, seed=P)
    phs, pos, k_r = synth.phase_history(S, P, 9.3e9, 2e6, 9e3, 35, 3, scat, 30.0, P + S)
    dr = synth.C / (2 * S * 2e6)
    g = synth.grid_plane(max(nu, nv), 12.0, pos, dr, S, P)
    u, v = g["u"][:nu], g["v"][:nv]
    r = synth.pixel_locs(u, v, g["u_hat"], g["v_hat"])
    for N in (16, 64):
        ref = oracle.backprojection(phs, k_r.astype(np.float32), 17, N, dr, pos.astype(np.float32), r,
                                    nu, nv, mode=oracle.MODE_REF)
        for parts in (0, 16):
            img = ctx.backprojection_cuda(phs, k_r.astype(np.float32), 17, N, dr, u, v, pos.astype(np.float32), r,
                                          pulse_parts=parts)
            assert img.shape == (nv, nu)
            assert rel_l2(img, ref) < 5 * REL_COMPAT


def test_scattered_pixels(ctx, oracle, cfg1):
    """Pixel positions that are not a grid (a random shuffle of the plane):
    each tile spans the whole 50 m scene, so the per-pixel offsets are tens
    of metres and the closed-form range path keeps only f32 relative
    precision on them (~|offset| * 6e-8 m, ~1e-3 rad of phase at X band).
    Tolerance here: relative L2 <= 1e-3 -- or the call is rejected with
    SARBP_ERR_GEOMETRY when a tile's range window exceeds the staging
    buffer; never a silently wrong image."""
    d = cfg1
    rng = np.random.default_rng(5)
    n = 64
    perm = rng.permutation(d["nu"] * d["nv"])[: n * n]
    r = np.ascontiguousarray(d["r"][:, perm])
    pos32, k32 = d["pos"].astype(np.float32), d["k_r"].astype(np.float32)
    try:
        img = ctx.backprojection_cuda(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"],
                                      np.zeros(n), np.zeros(n), pos32, r)
    except Exception as ex:  # documented: tiles wider than the staging buffer are rejected
        assert getattr(ex, "code", None) == -5
        return
    ref = oracle.backprojection(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], pos32, r, n, n,
                                mode=oracle.MODE_REF)
    assert rel_l2(img, ref) < 1e-3


def test_batch_matches_single_bitwise(sb, ctx, torch):
    """Uneven jobs in one persistent launch give bit-identical images to
    the same jobs run one by one."""
    from sarbp_b200 import synth
    params = synth.batch_jobs(njobs=5, seed=3, sizes=(64, 128, 256), pulses=(100, 400),
                              samples=(256, 512), taylors=(17, 30))
    datas = [synth.make_from(p) for p in params]
    keep, jobs, outs = [], [], []
    for dd in datas:
        t = dict(phs=_dev(torch, dd["phs"].view(np.float32)), k=_dev(torch, dd["k_r"].astype(np.float32)),
                 pos=_dev(torch, dd["pos"].astype(np.float32)), u=_dev(torch, dd["u"]),
                 v=_dev(torch, dd["v"]))
        out = torch.zeros((dd["nv"], dd["nu"], 2), dtype=torch.float64, device="cuda")
        keep.append(t)
        outs.append(out)
        jobs.append(sb.make_job(dd["S"], dd["P"], dd["N_fft"], dd["taylor"], dd["nu"], dd["nv"],
                                dd["delta_r"], t["phs"].data_ptr(), t["k"].data_ptr(), t["pos"].data_ptr(),
                                out.data_ptr(), u=t["u"].data_ptr(), v=t["v"].data_ptr(),
                                u_hat=dd["u_hat"], v_hat=dd["v_hat"]))
    ctx.run_jobs(jobs)
    ctx.synchronize()
    batched = [o.cpu().numpy().copy() for o in outs]
    for j, o, b in zip(jobs, outs, batched):
        o.zero_()
        ctx.run_jobs([j])
        ctx.synchronize()
        np.testing.assert_array_equal(o.cpu().numpy(), b)


def test_grid_form_equals_r_array(sb, ctx, torch, cfg1):
    """Pixel positions generated on the device from (u, v, u_hat, v_hat) are
    the same numbers as the reference's pixel_locs array."""
    d = cfg1
    t_phs = _dev(torch, d["phs"].view(np.float32))
    t_k = _dev(torch, d["k_r"].astype(np.float32))
    t_pos = _dev(torch, d["pos"].astype(np.float32))
    t_r = _dev(torch, d["r"])
    t_u, t_v = _dev(torch, d["u"]), _dev(torch, d["v"])
    o1 = torch.zeros((d["nv"], d["nu"], 2), dtype=torch.float64, device="cuda")
    o2 = torch.zeros_like(o1)
    common = (d["S"], d["P"], d["N_fft"], d["taylor"], d["nu"], d["nv"], d["delta_r"], t_phs.data_ptr(),
              t_k.data_ptr(), t_pos.data_ptr())
    ctx.run_jobs([sb.make_job(*common, o1.data_ptr(), r=t_r.data_ptr())])
    ctx.run_jobs([sb.make_job(*common, o2.data_ptr(), u=t_u.data_ptr(), v=t_v.data_ptr(),
                              u_hat=d["u_hat"], v_hat=d["v_hat"])])
    ctx.synchronize()
    np.testing.assert_array_equal(o1.cpu().numpy(), o2.cpu().numpy())
    # the host-buffer entry point pipelines the image in row slabs (copies
    # overlapped with compute on two streams); every tile is still formed by
    # the same kernel, so the image is the same bit for bit
    h = ctx.backprojection_cuda(d["phs"], d["k_r"].astype(np.float32), d["taylor"], d["N_fft"],
                                d["delta_r"], d["u"], d["v"], d["pos"].astype(np.float32), d["r"])
    np.testing.assert_array_equal(h, o1.cpu().numpy().view(np.complex128)[..., 0])


@pytest.mark.parametrize("nu,nv", [(2048, 1024), (1000, 1500), (640, 2000)])
def test_host_pipeline_row_slabs(ctx, oracle, nu, nv):
    """Host-buffer calls on images large enough to be pipelined in row slabs
    (ragged last slab, non-square images): the same image as the
    device-resident call, and the oracle's on sampled pixels."""
    import torch
    import sarbp_b200 as sb
    from sarbp_b200 import synth
    d = synth.make("plain_small", seed=4, with_r=False,
                   overrides=dict(P=200, S=256, n=max(nu, nv), extent=60.0))
    u, v = d["u"][:nu], d["v"][:nv]
    r = synth.pixel_locs(u, v, d["u_hat"], d["v_hat"])
    k32, pos32 = d["k_r"].astype(np.float32), d["pos"].astype(np.float32)
    h = ctx.backprojection_cuda(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], u, v, pos32, r)
    t = [_dev(torch, a) for a in (d["phs"].view(np.float32), k32, pos32, r)]
    o = torch.zeros((nv, nu, 2), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ctx.run_jobs([sb.make_job(d["S"], d["P"], d["N_fft"], d["taylor"], nu, nv, d["delta_r"], t[0].data_ptr(),
                              t[1].data_ptr(), t[2].data_ptr(), o.data_ptr(), r=t[3].data_ptr())])
    ctx.synchronize()
    np.testing.assert_array_equal(h, o.cpu().numpy().view(np.complex128)[..., 0])
    idx = np.random.default_rng(1).choice(nu * nv, 3000, replace=False)
    ref = oracle.backprojection(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], pos32, r, nu, nv,
                                out_idx=idx)
    assert rel_l2(h.ravel()[idx], ref) < REL_COMPAT


def test_db_u8_kernels_match_oracle(ctx, oracle, cfg1):
    rng = np.random.default_rng(9)
    img = (rng.normal(size=(300, 257)) + 1j * rng.normal(size=(300, 257))) * rng.uniform(0, 5, (300, 257))
    img[3, 4] = 0.0
    dB = ctx.img_output_to_dB(img)
    dBr = oracle.img_output_to_dB(img)
    fin = np.isfinite(dBr)
    assert np.array_equal(np.isfinite(dB), fin)
    np.testing.assert_allclose(dB[fin], dBr[fin], rtol=0, atol=1e-12)
    u8 = ctx.img_output_u8(dB, -30.0, 0.0)
    np.testing.assert_array_equal(u8, oracle.img_output_u8(dBr, -30.0, 0.0))


@pytest.mark.parametrize("shape", [(300, 257), (512, 512), (1, 3)])
def test_u8_from_image_in_one_pass_matches_oracle(ctx, oracle, torch, shape):
    """sarbp_img_output_u8_from_img_device (max|z| then grey levels, no f64
    dB image) gives exactly the reference's u8 of the image
    (img_output.cpp:18-51 through the oracle), also for ragged sizes."""
    rng = np.random.default_rng(11)
    img = (rng.normal(size=shape) + 1j * rng.normal(size=shape)) * rng.uniform(0, 5, shape)
    nv, nu = shape
    for lo, hi in ((-30.0, 0.0), (-3.0, -1.0)):
        d_img = torch.from_numpy(img.view(np.float64).reshape(nv, nu, 2).copy()).cuda()
        d_u8 = torch.zeros((nv, nu), dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        ctx.img_output_u8_from_img_device(d_img.data_ptr(), nu, nv, lo, hi, d_u8.data_ptr())
        ctx.synchronize()
        want = oracle.img_output_u8(oracle.img_output_to_dB(img), lo, hi)
        assert np.array_equal(d_u8.cpu().numpy(), want), (shape, lo, hi)


def test_naive_mode_is_worse_but_finite(ctx, oracle, cfg1):
    d = cfg1
    ref = oracle.backprojection(d["phs"], d["k_r"], d["taylor"], d["N_fft"], d["delta_r"], d["pos"],
                                d["r"], d["nu"], d["nv"], mode=oracle.MODE_FP64)
    naive = ctx.backprojection_cuda(d["phs"], d["k_r"], d["taylor"], d["N_fft"], d["delta_r"], d["u"],
                                    d["v"], d["pos"], d["r"], precision=2)
    split = ctx.backprojection_cuda(d["phs"], d["k_r"], d["taylor"], d["N_fft"], d["delta_r"], d["u"],
                                    d["v"], d["pos"], d["r"], precision=1)
    en, es = rel_l2(naive, ref), rel_l2(split, ref)
    print("naive %.3e split %.3e" % (en, es))
    assert np.all(np.isfinite(naive)) and es < en


def test_errors_are_codes(sb, ctx, cfg1):
    d = cfg1
    pos32, k32 = d["pos"].astype(np.float32), d["k_r"].astype(np.float32)
    call = lambda **kw: ctx.backprojection_cuda(
        kw.get("phs", d["phs"]), k32, kw.get("taylor", 17), kw.get("N", d["N_fft"]), d["delta_r"],
        d["u"], d["v"], kw.get("pos", pos32), d["r"])
    with pytest.raises(sb.SarbpError) as e:
        call(N=1000)
    assert e.value.code == sb._lib.ERR_UNSUPPORTED
    with pytest.raises(sb.SarbpError) as e:
        call(N=1 << 18)  # above the four-step FFT's 131072
    assert e.value.code == sb._lib.ERR_UNSUPPORTED
    with pytest.raises(sb.SarbpError) as e:
        call(taylor=0)
    assert e.value.code == sb._lib.ERR_INVALID
    with pytest.raises(sb.SarbpError) as e:
        call(taylor=35)
    assert e.value.code == sb._lib.ERR_INVALID
    bad = pos32.copy()
    bad[10, 1] = np.nan
    with pytest.raises(sb.SarbpError) as e:
        call(pos=bad)
    assert e.value.code == sb._lib.ERR_GEOMETRY
    # the context still works afterwards
    img = call()
    assert np.all(np.isfinite(img))


def test_bad_pixels_and_sizes_are_codes(sb, ctx, cfg1):
    """A non-finite pixel position is SARBP_ERR_GEOMETRY (one NaN in one
    coordinate, and an infinity), empty image or pulse extents are
    SARBP_ERR_INVALID; the context keeps working and gives the same image
    as before."""
    d = cfg1
    pos32, k32 = d["pos"].astype(np.float32), d["k_r"].astype(np.float32)
    good = ctx.backprojection_cuda(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], d["u"], d["v"],
                                   pos32, d["r"])
    for coord, val in ((2, np.nan), (0, np.inf)):
        r = d["r"].copy()
        r[coord, 777] = val
        with pytest.raises(sb.SarbpError) as e:
            ctx.backprojection_cuda(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], d["u"], d["v"],
                                    pos32, r)
        assert e.value.code == sb._lib.ERR_GEOMETRY
    with pytest.raises(sb.SarbpError) as e:
        ctx.backprojection_cuda(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], d["u"][:0], d["v"],
                                pos32, d["r"][:, :0])
    assert e.value.code == sb._lib.ERR_INVALID
    with pytest.raises(sb.SarbpError) as e:
        ctx.backprojection_cuda(d["phs"][:0], k32, d["taylor"], d["N_fft"], d["delta_r"], d["u"], d["v"],
                                pos32[:0], d["r"])
    assert e.value.code == sb._lib.ERR_INVALID
    again = ctx.backprojection_cuda(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], d["u"], d["v"],
                                    pos32, d["r"])
    assert np.array_equal(again, good)


def test_kernels_are_launched(ctx, cfg1):
    d = cfg1
    before = ctx.launch_count()
    ctx.backprojection_cuda(d["phs"], d["k_r"].astype(np.float32), d["taylor"], d["N_fft"], d["delta_r"],
                            d["u"], d["v"], d["pos"].astype(np.float32), d["r"])
    # set-up and range compression, then tile geometry (with the pulse
    # records) and backprojection per row slab: 512 x 512 in 32-row tiles is
    # 16 tile rows, pipelined as 4 slabs of 1, 2, 12 and 1 tile rows
    assert ctx.launch_count() - before == 2 + 2 * 4
