"""The C ABI library: loads, exports every declared symbol, host helpers
(CPU only; no kernel is launched here)."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def _declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        if 'extern "C"' not in src:
            continue
        for m in re.finditer(r"\b(sarbp_\w+)\s*\(", src):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol(sb):
    from sarbp_b200 import _lib
    L = _lib.lib()
    declared = _declared_functions()
    assert len(declared) >= 15
    missing = [n for n in declared if not hasattr(L, n)]
    assert not missing, missing
    # and the Python binding covers all of them
    assert declared <= set(_lib.SIGNATURES), declared - set(_lib.SIGNATURES)


def test_version(sb):
    assert "sm_100a" in sb.version()


def test_taylor_matches_oracle(sb, oracle, known_answers):
    ka = known_answers["taylor"]
    np.testing.assert_array_equal(sb.taylor(ka["num"], ka["S_L"]), oracle.taylor(ka["num"], ka["S_L"]))
    for n, sl in ((1999, 30), (424, 17), (1024, 20)):
        np.testing.assert_array_equal(sb.taylor(n, sl), oracle.taylor(n, sl))


def test_taylor_float_mode_matches_oracle_and_is_defined_above_30_db(sb, oracle):
    """TAYLOR_FLOAT (the F_m denominator quotient in floating point) equals
    the oracle's float-division window at every level; the reference's
    Int32-division window is only defined up to 30 dB."""
    for n, sl in ((1999, 17), (424, 30), (1024, 31), (777, 35), (2000, 45)):
        w = sb.taylor(n, sl, sb.TAYLOR_FLOAT)
        np.testing.assert_array_equal(w, oracle.taylor(n, sl, taylor_mode=1))
        assert np.all(np.isfinite(w)) and abs(w.max() - 1.0) < 1e-15
    # both variants agree where no Int32 quotient rounds (n_bar <= 3)
    np.testing.assert_array_equal(sb.taylor(500, 17, sb.TAYLOR_FLOAT), sb.taylor(500, 17))
    # above 30 dB the reference's window is 0/0 somewhere
    assert not np.all(np.isfinite(oracle.taylor(500, 31)))
    with pytest.raises(sb.SarbpError):
        sb.taylor(500, 20, 7)


def test_img_plane_matches_fixture(sb, afrl_input, afrl_img_plane):
    ip = sb.img_plane_create(int(afrl_input["nsamples"][0]), int(afrl_input["npulses"][0]),
                             float(afrl_input["delta_r"][0]), afrl_input["R_c"])
    for k in ("u", "v", "k_u", "k_v"):
        np.testing.assert_array_equal(ip[k], afrl_img_plane[k])
    np.testing.assert_allclose(ip["v_hat"], afrl_img_plane["v_hat"], atol=1e-7, rtol=0)
    assert ip["pixel_locs"].shape == (3, 512 * 512)


def test_img_plane_and_pixel_locs_match_oracle(sb, oracle):
    R_c = np.array([1234.5, -3000.25, 4000.0], np.float32)
    for up in (True, False):
        a = sb.img_plane_create(300, 129, 0.3, R_c, res_factor=0.7, aspect=1.3, upsample=up)
        b = oracle.img_plane(300, 129, 0.3, R_c, res_factor=0.7, aspect=1.3, upsample=up)
        for k in ("u", "v", "k_u", "k_v", "u_hat", "v_hat", "pixel_locs"):
            np.testing.assert_array_equal(a[k], b[k])
        np.testing.assert_array_equal(sb.pixel_locs(a["u"], a["v"], a["u_hat"], a["v_hat"]),
                                      b["pixel_locs"])


def test_n_fft_rule(sb):
    # sarbp.cpp:258
    assert sb.n_fft_for(424, 2) == 1024
    assert sb.n_fft_for(1024, 2) == 4096
    assert sb.n_fft_for(2048, 2) == 8192
    assert sb.n_fft_for(424, 6) == 4096
    assert sb.n_fft_for(1800, 6) == 16384


def test_synth_deterministic_and_threads_independent(sb):
    from sarbp_b200 import synth
    scat = synth.scene(5, 10.0, 3, seed=4)
    a = synth.phase_history(64, 33, 9.3e9, 1.5e6, 10e3, 30, 4, scat, 20.0, 11, nthreads=1)
    b = synth.phase_history(64, 33, 9.3e9, 1.5e6, 10e3, 30, 4, scat, 20.0, 11, nthreads=5)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    phs, pos, k_r = a
    assert phs.dtype == np.complex64 and phs.shape == (33, 64)
    np.testing.assert_allclose(np.linalg.norm(pos, axis=1), 10e3, rtol=1e-12)


def test_synth_matches_direct_sum(sb):
    from sarbp_b200 import synth
    scat = np.array([[1.0, 2.0, 0.0, 0.7, -0.2], [-3.0, 0.5, 0.0, 0.1, 0.4]])
    phs, pos, k_r = synth.phase_history(100, 7, 9.3e9, 1.5e6, 10e3, 30, 4, scat, 400, 1)
    D = np.linalg.norm(pos, axis=1)[:, None] - np.linalg.norm(pos[:, None, :] - scat[None, :, :3], axis=2)
    a = scat[:, 3] + 1j * scat[:, 4]
    ref = (a[None, None, :] * np.exp(1j * k_r[None, :, None] * D[:, None, :])).sum(-1)
    np.testing.assert_allclose(phs, ref, rtol=0, atol=2e-6)


def test_errors_without_gpu_are_codes(sb):
    """Creating a context on a machine without a usable B200 returns an
    error code and a message instead of crashing."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(sb.SarbpError) as ei:
        sb.Context(0)
    assert ei.value.code in (sb._lib.ERR_CUDA, sb._lib.ERR_INVALID)


def test_pulse_parts_in_the_job_footprint(sb):
    """Small one-shot jobs are formed in pulse parts (one partial image per
    part in the footprint); images of 2^18 pixels and more are not unless
    asked; an explicit part count applies to any image."""
    def fp(nu, nv, P, **tune):
        job = sb.make_job(1024, P, 4096, 30, nu, nv, 0.2, 0, 0, 0, 0, r=1)
        return sb.job_device_bytes(job, precision=sb.PREC_COMPAT, **tune)
    # 256^2: 64 tiles of 32x32 for 148 SMs x 3 resident CTAs -> 4 parts of
    # 125 pulses (two items on each of 128 SMs)
    assert fp(256, 256, 500) - fp(256, 256, 500, pulse_parts=1) == 4 * 256 * 256 * 8
    # 100 pulses: 2 parts (one item on each of 128 SMs); 40: no part of 32
    # pulses pays for its fixed cost
    assert fp(256, 256, 100) - fp(256, 256, 100, pulse_parts=1) == 2 * 256 * 256 * 8
    assert fp(256, 256, 40) == fp(256, 256, 40, pulse_parts=1)
    # 2048^2 (4096 tiles) and 512^2 (2^18 pixels): one item per tile
    assert fp(2048, 2048, 1999) == fp(2048, 2048, 1999, pulse_parts=1)
    assert fp(512, 512, 469) == fp(512, 512, 469, pulse_parts=1)
    # explicit parts: 4 partial images of 2048^2, capped at one part per pulse
    assert fp(2048, 2048, 1999, pulse_parts=4) - fp(2048, 2048, 1999) == 4 * 2048 * 2048 * 8
    assert fp(64, 64, 3, pulse_parts=16) - fp(64, 64, 3, pulse_parts=1) == 3 * 64 * 64 * 8
