"""The sarbp CLI, the image-plane entry point and the halide_buffer_t shim on
the GPU.

* The CLI run on the AFRL pass-1 platform data (469 pulses x 424 samples,
  512 x 512 image, Taylor 17, upsample 2, -30..0 dB) writes a PNG whose
  pixels equal the oracle's u8 image (sarbp.cpp:250-324 step by step) up to
  one grey level on fewer than 1 % of the pixels: u8 = 8.5 levels per dB
  here, and the complex image agrees to the compat tolerance (relative
  L2 <= 1e-4, dB within 0.05).
* A complex128 / float64 platform directory (the downcast path) gives the
  identical PNG.
* sarbp_backprojection_plane (pixel positions formed on the device from the
  image-plane axes) equals sarbp_backprojection with host pixel_locs bit for
  bit: both evaluate (0 + u_hat*u) + v_hat*v in f64 without contraction.
* The shim's backprojection_cuda / img_output_to_dB / img_output_u8 equal
  the C ABI calls they wrap.
"""
import ctypes
import math
import os
import struct
import subprocess
import zlib

import numpy as np
import pytest

from conftest import PKG, rel_l2
from halide_buffers import HalideBuffer
from test_cli import SARBP, SHIM, write_platform

pytestmark = pytest.mark.gpu

TAYLOR, UPS, DB_MIN, DB_MAX = 17, 2, -30.0, 0.0


def read_png_gray8(path):
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, w = 8, b"", None
    while pos < len(data):
        n, typ = struct.unpack(">I4s", data[pos:pos + 8])
        body = data[pos + 8:pos + 8 + n]
        crc = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0]
        assert zlib.crc32(typ + body) & 0xffffffff == crc
        if typ == b"IHDR":
            w, h, depth, ctype = struct.unpack(">IIBB", body[:10])
            assert depth == 8 and ctype == 0
        elif typ == b"IDAT":
            idat += body
        pos += 12 + n
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, w + 1)
    assert np.all(raw[:, 0] == 0)  # filter type None on every row
    return raw[:, 1:].copy()


@pytest.fixture(scope="module")
def afrl_reference(afrl_input, oracle):
    pd = afrl_input
    P, S = pd["phs"].shape
    dr = float(np.ravel(pd["delta_r"])[0])
    ip = oracle.img_plane(S, P, dr, pd["R_c"], upsample=True)
    n_fft = int(math.pow(2, int(math.log2(S * UPS)) + 1))
    img = oracle.backprojection(pd["phs"], pd["k_r"], TAYLOR, n_fft, dr, pd["pos"],
                                ip["pixel_locs"], ip["nu"], ip["nv"])
    u8 = oracle.img_output_u8(oracle.img_output_to_dB(img), DB_MIN, DB_MAX)
    return dict(ip=ip, n_fft=n_fft, img=img, u8=u8, dr=dr)


def _cli(d, out_png):
    p = subprocess.run([SARBP, "-p", d, "-o", out_png, "-t", str(TAYLOR), "-u", str(UPS),
                        "-d", str(DB_MIN), "-D", str(DB_MAX), "-n", "2"],
                       capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    return p.stdout


def test_cli_png_matches_oracle(tmp_path, afrl_input, afrl_reference):
    d = write_platform(str(tmp_path / "afrl"), afrl_input)
    out = _cli(d, str(tmp_path / "afrl.png"))
    # the reference's progress lines, verbatim (sarbp.cpp:275-326)
    for line in ("(1) Halide backprojection start", "(2) Halide backprojection returned 0",
                 "Halide dB conversion returned 0", "Halide PNG production returned 0", "Wrote "):
        assert line in out, line
    got = read_png_gray8(str(tmp_path / "afrl.png"))
    ref = afrl_reference["u8"]
    assert got.shape == ref.shape == (512, 512)
    diff = np.abs(got.astype(int) - ref.astype(int))
    print("u8 mismatches: %d of %d, max %d" % ((diff > 0).sum(), diff.size, diff.max()))
    assert diff.max() <= 1 and (diff > 0).mean() < 0.01

    wide = write_platform(str(tmp_path / "wide"), afrl_input, wide=True, int32=True)
    out = _cli(wide, str(tmp_path / "wide.png"))
    assert "downcasting phs" in out
    assert np.array_equal(read_png_gray8(str(tmp_path / "wide.png")), got)


def test_plane_entry_point_equals_pixel_locs(ctx, afrl_input, afrl_reference):
    pd, R = afrl_input, afrl_reference
    ip = R["ip"]
    a = ctx.backprojection_cuda(pd["phs"], pd["k_r"], TAYLOR, R["n_fft"], R["dr"], ip["u"], ip["v"],
                                pd["pos"], ip["pixel_locs"])
    b = ctx.backprojection_plane(pd["phs"], pd["k_r"], TAYLOR, R["n_fft"], R["dr"], ip["u"], ip["v"],
                                 ip["u_hat"], ip["v_hat"], pd["pos"])
    assert np.array_equal(a, b)
    assert rel_l2(a, R["img"]) < 1e-4


def test_halide_shim_matches_c_abi(ctx, afrl_input, afrl_reference):
    L = ctypes.CDLL(SHIM)
    pd, R = afrl_input, afrl_reference
    ip = R["ip"]
    nu, nv = ip["nu"], ip["nv"]
    phs = HalideBuffer(pd["phs"].view(np.float32).reshape(pd["phs"].shape + (2,)))  # {2, S, P}
    k_r = HalideBuffer(pd["k_r"].astype(np.float32))
    u, v = HalideBuffer(ip["u"]), HalideBuffer(ip["v"])
    pos = HalideBuffer(pd["pos"].astype(np.float32))                                # {3, P}
    r = HalideBuffer(ip["pixel_locs"])                                              # {nu*nv, 3}
    out = HalideBuffer(np.zeros((nv, nu, 2)))                                       # {2, nu, nv}
    L._Z13dft_init_fftwm(ctypes.c_size_t(R["n_fft"]))
    bp = L._Z19backprojection_cudaP15halide_buffer_tS0_iidS0_S0_S0_S0_S0_
    bp.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_double] + \
        [ctypes.c_void_p] * 5
    rc = bp(ctypes.addressof(phs.buf), ctypes.addressof(k_r.buf), TAYLOR, R["n_fft"], R["dr"],
            ctypes.addressof(u.buf), ctypes.addressof(v.buf), ctypes.addressof(pos.buf),
            ctypes.addressof(r.buf), ctypes.addressof(out.buf))
    L._Z16dft_destroy_fftwv()
    assert rc == 0
    assert out.buf.flags & 1  # host_dirty
    img = out.arr.view(np.complex128)[..., 0]
    want = ctx.backprojection_cuda(pd["phs"], pd["k_r"], TAYLOR, R["n_fft"], R["dr"], ip["u"], ip["v"],
                                   pd["pos"], ip["pixel_locs"])
    assert np.array_equal(img, want)

    dB = HalideBuffer(np.zeros((nv, nu)))
    assert L.img_output_to_dB(ctypes.byref(out.buf), dB.ptr()) == 0
    assert np.array_equal(dB.arr, ctx.img_output_to_dB(img))
    u8 = HalideBuffer(np.zeros((nv, nu), np.uint8))
    L.img_output_u8.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_void_p]
    assert L.img_output_u8(ctypes.addressof(dB.buf), DB_MIN, DB_MAX, ctypes.addressof(u8.buf)) == 0
    assert np.array_equal(u8.arr, ctx.img_output_u8(dB.arr, DB_MIN, DB_MAX))


@pytest.mark.parametrize("form", ["r", "plane"])
def test_row_blocks_on_gpu_reassemble_the_image(ctx, afrl_input, afrl_reference, form):
    """The per-rank work of the distributed mode (sarbp_b200.distributed),
    run rank by rank on this GPU: each of three ranks' kernels write its
    block of output rows straight into its device send buffer
    (DeviceCompute, form_block), and the buffers assembled in rank order (as
    rank 0 does after the NCCL gather) give the whole image.  Block edges
    that do not fall on 32-row tile edges give tiles with other centres, so
    the match is to rounding (relative L2 < 1e-5), and to the oracle within
    the compat tolerance.  Pixel positions as the r array and as the
    image-plane axes."""
    import torch
    from sarbp_b200.distributed import DeviceCompute, assemble, form_block
    pd, R = afrl_input, afrl_reference
    ip = R["ip"]
    nu, nv = ip["nu"], ip["nv"]
    kw = dict(r=ip["pixel_locs"]) if form == "r" else dict(u_hat=ip["u_hat"], v_hat=ip["v_hat"])
    compute = DeviceCompute(ctx, pd["phs"], pd["k_r"], TAYLOR, R["n_fft"], R["dr"], ip["u"], ip["v"], pd["pos"],
                            **kw)
    sends = [form_block(compute, nu, nv, 3, k, device="cuda") for k in range(3)]
    assert all(s.is_cuda for s in sends)
    out = assemble(sends, nu, nv)
    whole = assemble([form_block(compute, nu, nv, 1, 0, device="cuda")], nu, nv)
    assert rel_l2(out, whole) < 1e-5
    assert rel_l2(out, R["img"]) < 1e-4
