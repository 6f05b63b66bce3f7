"""The sarbp CLI and the halide_buffer_t shim, on the CPU: argument checks,
the platform loader (shapes, word sizes, downcasts, PlatformData.cpp:21-256)
and the image-plane sizes it prints, up to the point where it needs a GPU;
and the shim library's exported names (sarbp.cpp-style callers link against
them).  The GPU half is in test_gpu_cli.py."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG

SARBP = os.path.join(PKG, "bin", "sarbp")
SHIM = os.path.join(PKG, "lib", "libsarbp_halide.so")


def _run(*args, cwd=None):
    p = subprocess.run([SARBP, *args], capture_output=True, text=True, timeout=120, cwd=cwd)
    return p.returncode, p.stdout, p.stderr


def write_platform(d, pd, wide=False, int32=False, extra=None):
    """A platform directory in the reference's .npy layout from fixture
    arrays (phs [P, S], pos [P, 3], k_r [S], R_c [3], delta_r, sizes)."""
    os.makedirs(d, exist_ok=True)
    P, S = pd["phs"].shape
    it = np.int32 if int32 else np.int64
    np.save(os.path.join(d, "nsamples.npy"), np.array(S, it))
    np.save(os.path.join(d, "npulses.npy"), np.array(P, it))
    np.save(os.path.join(d, "delta_r.npy"), np.array(float(np.ravel(pd["delta_r"])[0])))
    ft, ct = (np.float64, np.complex128) if wide else (np.float32, np.complex64)
    np.save(os.path.join(d, "phs.npy"), pd["phs"].astype(ct))
    np.save(os.path.join(d, "pos.npy"), pd["pos"].astype(ft))
    np.save(os.path.join(d, "k_r.npy"), pd["k_r"].astype(ft))
    np.save(os.path.join(d, "R_c.npy"), np.asarray(pd["R_c"]).astype(ft))
    for k, v in (extra or {}).items():
        np.save(os.path.join(d, k + ".npy"), v)
    return d


@pytest.fixture(scope="module")
def cli_built():
    if not os.path.exists(SARBP):
        pytest.fail("sarbp CLI not built (make -C halide-sar-app_b200)")
    return SARBP


def test_help_and_constraints(cli_built):
    rc, out, _ = _run("-h")
    assert rc == 0 and "--platform-dir" in out and "--num-iters" in out
    rc, _, err = _run("-o", "x.png")
    assert rc != 0 and "Missing required parameters" in err
    rc, _, err = _run("-p", "d", "-o", "x.png")  # dB_min = dB_max = 0 by default
    assert rc != 0 and "dB_min < dB_max" in err
    for flag, val, msg in (("-t", "0", "taylor >= 1"), ("-u", "0", "upsample >= 1"),
                           ("-r", "0", "res-factor > 0"), ("-a", "-1", "aspect > 0")):
        rc, _, err = _run("-p", "d", "-o", "x.png", "-d", "-30", flag, val)
        assert rc != 0 and msg in err, (flag, err)


def test_schedules(cli_built, tmp_path):
    rc, _, err = _run("-p", str(tmp_path), "-o", "x.png", "-d", "-30", "-s", "cpu")
    assert rc != 0 and "not provided by this build" in err
    rc, _, err = _run("-p", str(tmp_path), "-o", "x.png", "-d", "-30", "-s", "bogus")
    assert rc != 0 and "Unknown schedule" in err


def test_loader_reports_sizes_and_image_plane(cli_built, tmp_path, afrl_input):
    d = write_platform(str(tmp_path / "afrl"), afrl_input)
    rc, out, err = _run("-p", d, "-o", str(tmp_path / "o.png"), "-d", "-30", "-t", "17", "-u", "2")
    assert "Number of pulses: 469" in out and "Pulse sample size: 424" in out
    # ImgPlane.cpp:20-23 / ip.h:5-9: nu = 2^ceil(log2 S), nv = 2^ceil(log2 P)
    assert "X length: 512" in out and "Y length: 512" in out
    assert "downcasting" not in out
    if rc != 0:  # no GPU here: the context is the first thing that needs one
        assert "device" in err.lower() or "cuda" in err.lower(), err


def test_loader_downcasts_like_the_reference(cli_built, tmp_path, afrl_input):
    d = write_platform(str(tmp_path / "wide"), afrl_input, wide=True, int32=True)
    _, out, _ = _run("-p", d, "-o", str(tmp_path / "o.png"), "-d", "-30")
    for name in ("k_r", "R_c", "pos"):
        assert "PlatformData: downcasting %s from double to float" % name in out
    assert "PlatformData: downcasting phs from complex<double> to complex<float>" in out
    assert "Number of pulses: 469" in out


@pytest.mark.parametrize("bad,msg", [
    (dict(pos=np.zeros((10, 3), np.float32)), "Bad shape: pos"),
    (dict(k_r=np.zeros(7, np.float32)), "Bad shape: k_r"),
    (dict(R_c=np.zeros(3, np.int16)), "Bad word size: R_c"),
    (dict(delta_r=np.float32(0.3)), "Bad word size: delta_r"),
    (dict(n_hat=np.zeros(3, np.float64)), "Bad word size: n_hat"),
    (dict(t=np.zeros(5, np.float64)), "Bad shape: t"),
    (dict(B=np.float32(1.0)), "Bad word size: B"),
])
def test_loader_errors(cli_built, tmp_path, afrl_input, bad, msg):
    d = write_platform(str(tmp_path / "bad"), afrl_input)
    for k, v in bad.items():
        np.save(os.path.join(d, k + ".npy"), v)
    rc, out, err = _run("-p", d, "-o", str(tmp_path / "o.png"), "-d", "-30")
    assert rc != 0 and msg in err, (out, err)
    assert "Number of pulses" not in out or msg.endswith(("pos", "k_r", "R_c", "n_hat", "t"))


def test_halide_shim_exports():
    if not os.path.exists(SHIM):
        pytest.fail("libsarbp_halide.so not built")
    L = ctypes.CDLL(SHIM)
    for name in ("_Z19backprojection_cudaP15halide_buffer_tS0_iidS0_S0_S0_S0_S0_",
                 "img_output_to_dB", "img_output_u8",
                 "_Z13dft_init_fftwm", "_Z16dft_destroy_fftwv"):
        assert hasattr(L, name), name
    # the FFTW plan calls are no-ops and need no device
    L._Z13dft_init_fftwm(ctypes.c_size_t(4096))
    L._Z16dft_destroy_fftwv()


def test_halide_shim_refuses_bad_buffers():
    from halide_buffers import HalideBuffer
    L = ctypes.CDLL(SHIM)
    img = HalideBuffer(np.zeros((4, 4, 2)))          # {2, 4, 4} f64
    bad_out = HalideBuffer(np.zeros((4, 5)))         # extents differ
    assert L.img_output_to_dB(img.ptr(), bad_out.ptr()) < 0
    wrong_type = HalideBuffer(np.zeros((4, 4), np.float32))
    assert L.img_output_to_dB(img.ptr(), wrong_type.ptr()) < 0
    img.buf.flags = 2                                 # device_dirty
    assert L.img_output_to_dB(img.ptr(), HalideBuffer(np.zeros((4, 4))).ptr()) < 0


def test_loader_rejects_a_truncated_payload(cli_built, tmp_path, afrl_input):
    """A phase history whose payload ends early (the threaded read of the
    payload in pieces) is an error naming the file, not a partial array."""
    d = write_platform(str(tmp_path / "cut"), afrl_input, wide=True)
    path = os.path.join(d, "phs.npy")
    size = os.path.getsize(path)
    with open(path, "r+b") as f:
        f.truncate(size - 12345)
    rc, out, err = _run("-p", d, "-o", str(tmp_path / "o.png"), "-d", "-30")
    assert rc != 0 and "phs.npy" in err and "truncated data" in err, (out, err)
    assert "Loaded platform data" not in out
