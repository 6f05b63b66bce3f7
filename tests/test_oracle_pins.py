"""The CPU oracle pinned against the reference's own known answers and
fixtures (CPU only)."""
import numpy as np
import pytest

from conftest import rel_l2


def test_taylor_table(oracle, known_answers):
    ka = known_answers["taylor"]  # test/taylor_test.cpp:14-31
    out = oracle.taylor(ka["num"], ka["S_L"])
    assert np.all(np.abs(out - np.array(ka["expected"])) < ka["tol"])


def test_taylor_symmetric_normalised(oracle):
    for n, sl in ((1999, 30), (424, 17), (469, 17), (1024, 20), (256, 1)):
        w = oracle.taylor(n, sl)
        assert w.max() == 1.0
        np.testing.assert_allclose(w, w[::-1], rtol=0, atol=1e-12)
        assert np.all(w > 0)


def test_taylor_integer_division_quirk(oracle):
    """pow(m+1, 2) / pow(r+1, 2) is an Int32 division in Halide
    (signal.h:40), so F_m's denominator hits 0 once n_bar >= 5, i.e. for
    side-lobe levels of 31 dB and up: the reference's window is undefined
    there.  Up to 30 dB it is finite."""
    assert np.all(np.isfinite(oracle.taylor(64, 30)))
    assert not np.all(np.isfinite(oracle.taylor(64, 31)))


def test_norm(oracle, known_answers):
    ka = known_answers["norm"]  # test/norm_test.cpp:15-46
    assert oracle.norm_f32(ka["in1"]) == ka["expected1"]
    in2 = np.array(ka["in2"], np.float32).reshape(2, 2)
    assert [oracle.norm_f32(row) for row in in2] == ka["expected2"]


def test_cross(oracle, known_answers):
    ka = known_answers["cross"]  # test/cross_test.cpp:14-31
    out = oracle.cross3_f32(ka["a"], ka["b"])
    assert np.all(np.abs(out - np.array(ka["expected"])) < ka["tol"])


def test_linspace(oracle, known_answers):
    ka = known_answers["linspace"]  # test/linspace_test.cpp:15-37
    out = oracle.linspace_f32(ka["start"], ka["stop"], ka["num"])
    step = np.float32((np.float32(ka["stop"]) - np.float32(ka["start"])) / np.float32(ka["num"] - 1))
    ref = np.float32(ka["start"]) + np.arange(ka["num"], dtype=np.float32) * step
    ref[-1] = ka["stop"]
    assert np.all(np.abs(ref - out) < ka["tol"])
    assert out[-1] == np.float32(ka["stop"]) and out[0] == np.float32(ka["start"])


def test_interp_known_answer(oracle, known_answers):
    """The linspace interpolation of backprojection.cpp:52-65 (clamped below
    the first and above the last sample) against the reference's interp
    known answers (test/interp_test.cpp:15-26), on the real and imaginary
    parts."""
    ka = known_answers["interp"]
    xp = np.array(ka["xp"])
    assert np.allclose(np.diff(xp), xp[1] - xp[0])  # a linspace axis
    fp = np.array(ka["fp"])
    out = oracle.interp_linspace(ka["xs"], xp[0], xp[-1], xp.size, fp - 2j * fp)
    exp = np.array(ka["expected"])
    assert np.all(np.abs(out.real - exp) < ka["tol"])
    assert np.all(np.abs(out.imag + 2 * exp) < 2 * ka["tol"])


def test_arange(oracle, known_answers):
    ka = known_answers["arange"]  # test/arange_test.cpp:18-40
    n = int(np.ceil((ka["stop"] - ka["start"]) / ka["step"]))
    out = oracle.arange_f32(ka["start"], ka["step"], n)
    assert np.all(np.abs(out - np.array(ka["expected"])) < ka["tol"])


def test_afrl_image_plane(oracle, afrl_input, afrl_img_plane):
    """ImgPlane.cpp against the RITSAR image-plane outputs shipped in
    data/AFRL/pass1/HH_ip_npy.  u, v, k_u, k_v, du, dv agree exactly; u_hat
    and v_hat carry the reference's f32 v_hat (img_plane.cpp:61)."""
    ip = oracle.img_plane(int(afrl_input["nsamples"][0]), int(afrl_input["npulses"][0]),
                          float(afrl_input["delta_r"][0]), afrl_input["R_c"], pixel_locs=False)
    g = afrl_img_plane
    for k in ("u", "v", "k_u", "k_v"):
        np.testing.assert_array_equal(ip[k], g[k])
    assert ip["d_u"] == g["du"][0] and ip["d_v"] == g["dv"][0]
    np.testing.assert_allclose(ip["u_hat"], g["u_hat"], rtol=0, atol=2e-9)
    np.testing.assert_allclose(ip["v_hat"], g["v_hat"], rtol=0, atol=1e-7)
    assert list(g["n_hat"]) == [0, 0, 1]


@pytest.mark.parametrize("n", [16, 64, 1000, 1024, 4096])
def test_fft_is_forward_dft(oracle, n):
    """dft.cpp:26 plans FFTW_FORWARD: X[k] = sum x[n] exp(-2 pi i n k / N)."""
    rng = np.random.default_rng(n)
    x = rng.normal(size=n) + 1j * rng.normal(size=n)
    np.testing.assert_allclose(oracle.fft_forward(x), np.fft.fft(x), rtol=0,
                               atol=1e-11 * np.sqrt(n) * np.abs(x).max() * np.log2(n))


def _naive_range_compress(phs, k_r, taylor_s_l, N, taylor_fn):
    """Straight numpy statement of backprojection.cpp:79-104 in f64
    (both fftshifts over both axes)."""
    P, S = phs.shape
    win = np.outer(taylor_fn(P, taylor_s_l), taylor_fn(S, taylor_s_l))
    x = phs.astype(np.complex128) * np.abs(k_r)[None, :] * win
    pad = np.zeros((P, N), np.complex128)
    xp = (N - S) // 2
    for n in range(N):
        s = n - xp
        if 0 <= s < S:
            pad[:, n] = x[:, s]
    sh = lambda a: np.roll(a, (-(N // 2 + N % 2), -(P // 2 + P % 2)), axis=(1, 0))
    return sh(np.fft.fft(sh(pad), axis=1))


@pytest.mark.parametrize("P,S,N", [(7, 10, 32), (8, 10, 32), (5, 40, 32), (33, 100, 256)])
def test_range_compress_matches_numpy_statement(oracle, P, S, N):
    rng = np.random.default_rng(P * S)
    phs = (rng.normal(size=(P, S)) + 1j * rng.normal(size=(P, S))).astype(np.complex64)
    k_r = rng.uniform(300, 400, size=S)
    Q = oracle.range_compress(phs, k_r, 17, N, mode=oracle.MODE_FP64)
    ref = _naive_range_compress(phs, k_r, 17, N, oracle.taylor)
    assert rel_l2(Q, ref) < 1e-12


def test_odd_pulse_count_rotates_rows(oracle):
    """fftshift over the pulse axis twice (backprojection.cpp:98, :104):
    odd P rotates the range profiles by one pulse, even P does not."""
    rng = np.random.default_rng(3)
    for P in (5, 6):
        phs = (rng.normal(size=(P, 12)) + 1j * rng.normal(size=(P, 12))).astype(np.complex64)
        k_r = np.full(12, 350.0)
        Q = oracle.range_compress(phs, k_r, 17, 32, mode=oracle.MODE_FP64)
        single = []
        for p in range(P):
            only = np.zeros_like(phs)
            only[p] = phs[p]
            single.append(np.abs(oracle.range_compress(only, k_r, 17, 32, mode=oracle.MODE_FP64)).sum(1))
        src_of_row0 = int(np.argmax([s[0] for s in single]))
        assert src_of_row0 == (1 if P % 2 else 0)


def test_ref_and_fp64_modes_close(oracle):
    """The reference-precision oracle and the FP64 oracle differ mainly by
    the f32 |pos| (norm_r0); at 10 km that is a visible but bounded error."""
    import sarbp_b200.synth as synth
    d = synth.make("plain_small", overrides=dict(n=64, extent=20.0))
    ref = oracle.backprojection(d["phs"], d["k_r"], 17, d["N_fft"], d["delta_r"], d["pos"], d["r"],
                                64, 64, mode=oracle.MODE_REF)
    f64 = oracle.backprojection(d["phs"], d["k_r"], 17, d["N_fft"], d["delta_r"], d["pos"], d["r"],
                                64, 64, mode=oracle.MODE_FP64)
    e = rel_l2(ref, f64)
    assert 1e-6 < e < 0.5


def test_point_target_focuses(oracle):
    """A single scatterer focuses to one bright pixel near its position
    (the reference's range axis floor(+-S*dr/2) shifts it by < 1 m)."""
    import sarbp_b200.synth as synth
    scat = np.array([[3.0, -4.0, 0.0, 1.0, 0.0]])
    phs, pos, k_r = synth.phase_history(424, 469, 9.29e9, 1.5e6, 10e3, 30, 4, scat, 400, 1)
    delta_r = synth.C / (2 * 424 * 1.5e6)
    g = synth.grid_plane(128, 25.0, pos, delta_r, 424, 469)
    r = synth.pixel_locs(g["u"], g["v"], g["u_hat"], g["v_hat"])
    img = oracle.backprojection(phs, k_r, 17, 1024, delta_r, pos, r, 128, 128)
    a = np.abs(img)
    y, x = np.unravel_index(a.argmax(), a.shape)
    pix = 128 * (128 - y - 1) + x
    loc = r[:, pix]
    assert abs(loc[0] - 3.0) < 1.0 and abs(loc[1] + 4.0) < 0.5
    assert a.max() > 100 * np.median(a)


def test_db_u8_semantics(oracle):
    img = np.array([[3 + 4j, 0.5, 0.0], [1e-3, 2.5j, -5.0]], np.complex128)
    dB = oracle.img_output_to_dB(img)
    assert dB[0, 0] == 0.0 and dB[1, 2] == 0.0 and np.isneginf(dB[0, 2])
    np.testing.assert_allclose(dB[0, 1], 10 * np.log10(0.1), rtol=1e-7)
    u8 = oracle.img_output_u8(dB, -30.0, 0.0)
    assert u8[0, 0] == 255 and u8[0, 2] == 0 and u8.dtype == np.uint8
    assert u8[0, 1] == int((10 * np.log10(0.1) + 30) / 30 * 255)


def test_oracle_generator_equals_the_library_generator(oracle, sb):
    """The benchmark's CPU arm builds its inputs with the oracle's generator
    (no product code in that arm): the same phase history, positions, k_r
    and pixel positions, bit for bit, as the product library's generator."""
    from sarbp_b200 import synth
    cfg = dict(synth.CONFIGS["plain_small"], P=97, S=130, n=48, nscat=7, clutter=3)
    d = synth.make("plain_small", seed=4, overrides=cfg)
    w = oracle.make_workload(cfg, synth.scene(cfg["nscat"], cfg["half"], cfg["clutter"], 4), 4)
    for k in ("phs", "pos", "k_r", "u", "v", "u_hat", "v_hat", "r"):
        assert np.array_equal(d[k], w[k]), k
    assert d["delta_r"] == w["delta_r"] and d["N_fft"] == w["N_fft"]
