"""Resampling of platform data (the reference's data/resize.py) on the
device, against the CPU restatement of skimage.transform.resize on
scipy.ndimage (oracle/resize_oracle.py):

* 2-D arrays shrinking on both axes, growing, and shrinking on one axis
  only (pos: (P, 3) -> (p, 3)); 1-D arrays (k_r); f32 and f64; complex
  arrays resampled as real and imaginary parts.  The f64 accumulation runs
  in scipy's order, so the results agree to the last bits: relative
  1e-6 of the array's range for f32, 1e-12 for f64.
* The resize tool on the AFRL platform files writes the same arrays, with
  the reference's dtypes, as the restated tool.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _check(got, want):
    assert got.shape == want.shape and got.dtype == want.dtype, (got.shape, want.shape, got.dtype, want.dtype)
    tol = (1e-6 if want.real.dtype == np.float32 else 1e-12) * max(1e-30, float(np.abs(want).max()))
    np.testing.assert_allclose(got, want, rtol=0, atol=tol)


@pytest.mark.parametrize("shape_in,shape_out", [
    ((469, 424), (300, 256)),   # both axes shrink
    ((97, 130), (200, 333)),    # both grow
    ((469, 424), (469, 212)),   # one axis
    ((1999, 3), (777, 3)),      # pos
    ((40, 7), (13, 2)),
])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_resize_2d_matches_oracle(ctx, shape_in, shape_out, dtype):
    from resize_oracle import sk_resize
    a = np.random.default_rng(3).normal(size=shape_in).astype(dtype)
    _check(ctx.resize(a, shape_out), sk_resize(a, shape_out))


@pytest.mark.parametrize("n_in,n_out", [(424, 212), (424, 1000), (1024, 333), (5, 1)])
def test_resize_1d_matches_oracle(ctx, n_in, n_out):
    from resize_oracle import sk_resize
    k = np.linspace(380.0, 395.0, n_in).astype(np.float32)
    _check(ctx.resize(k, (n_out,)), sk_resize(k, (n_out,)))
    _check(ctx.resize(k.astype(np.float64) * 0.5, (n_out,)), sk_resize(k.astype(np.float64) * 0.5, (n_out,)))


def test_resize_complex_is_real_and_imaginary_parts(ctx):
    from resize_oracle import sk_resize
    rng = np.random.default_rng(5)
    z = (rng.normal(size=(123, 77)) + 1j * rng.normal(size=(123, 77))).astype(np.complex64)
    want = sk_resize(np.real(z), (50, 90)) + 1j * sk_resize(np.imag(z), (50, 90))
    _check(ctx.resize(z, (50, 90)), want)


def test_resize_tool_on_afrl_files(ctx, afrl_input, tmp_path):
    from resize_oracle import resize_platform
    from sarbp_b200.resize import resize
    src = tmp_path / "in"
    src.mkdir()
    for k in ("delta_r", "k_r", "npulses", "nsamples", "phs", "pos", "R_c"):
        np.save(str(src / (k + ".npy")), afrl_input[k])
    for p, s, sp, ss, name in ((300, 256, 1.0, 1.0, "a"), (None, None, 0.5, 1.5, "b")):
        dst = str(tmp_path / name)
        resize(str(src), dst, p, s, scale_p=sp, scale_s=ss, ctx=ctx)
        d_r, k_r, P, S, phs, pos = resize_platform(afrl_input["delta_r"], afrl_input["k_r"],
                                                   afrl_input["npulses"], afrl_input["nsamples"],
                                                   afrl_input["phs"], afrl_input["pos"], p, s, sp, ss)
        got = {k: np.load(os.path.join(dst, k + ".npy")) for k in
               ("delta_r", "k_r", "npulses", "nsamples", "phs", "pos", "R_c")}
        assert np.array_equal(got["delta_r"], d_r) and got["delta_r"].dtype == d_r.dtype
        assert int(got["npulses"]) == P and int(got["nsamples"]) == S
        assert np.array_equal(got["R_c"], afrl_input["R_c"])
        _check(got["k_r"], k_r)
        _check(got["phs"], phs)
        _check(got["pos"], pos)
