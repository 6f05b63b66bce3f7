"""The CLI's PNG writer (cli/png_write.cpp, the image output of sarbp.cpp:324)
on the CPU: a small harness compiled against it writes seeded 8-bit images,
which are decoded here with zlib and compared pixel for pixel.  Sizes cover
a 1 x 1 image, ragged rows, and images large enough that the zlib stream is
deflated in several pieces on several threads (pieces of at least 256 KB),
including highly compressible ones (long runs)."""
import os
import struct
import subprocess
import zlib

import numpy as np
import pytest

from conftest import PKG

HARNESS = r"""
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "png_write.h"
int main(int argc, char **argv) {
    const int w = std::atoi(argv[2]), h = std::atoi(argv[3]);
    std::vector<uint8_t> px((size_t)w * h);
    FILE *f = std::fopen(argv[4], "rb");
    if (!f || std::fread(px.data(), 1, px.size(), f) != px.size()) return 2;
    std::fclose(f);
    sarbp_cli::png_write_gray8(argv[1], px.data(), w, h);
    return 0;
}
"""


def read_png_gray8(path):
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, w = 8, b"", None
    while pos < len(data):
        n, = struct.unpack(">I", data[pos:pos + 4])
        typ, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        crc, = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])
        assert zlib.crc32(typ + body) & 0xffffffff == crc, typ
        if typ == b"IHDR":
            w, h, depth, ctype, comp, filt, inter = struct.unpack(">IIBBBBB", body)
            assert (depth, ctype, comp, filt, inter) == (8, 0, 0, 0, 0)
        elif typ == b"IDAT":
            idat += body
        pos += 12 + n
    raw = zlib.decompress(idat)  # checks the Adler-32 of the rows
    rows = np.frombuffer(raw, np.uint8).reshape(h, w + 1)
    assert np.all(rows[:, 0] == 0)
    return rows[:, 1:]


@pytest.fixture(scope="module")
def writer(tmp_path_factory):
    d = tmp_path_factory.mktemp("png")
    src = d / "harness.cpp"
    src.write_text(HARNESS)
    exe = str(d / "harness")
    cli = os.path.join(PKG, "cli")
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", cli, str(src), os.path.join(cli, "png_write.cpp"),
                    "-lz", "-o", exe], check=True)
    return exe, d


@pytest.mark.parametrize("w,h,kind", [(1, 1, "noise"), (7, 13, "noise"), (2048, 2048, "noise"),
                                      (2048, 2048, "runs"), (4099, 1037, "noise"), (512, 512, "constant")])
def test_png_round_trip(writer, w, h, kind):
    exe, d = writer
    rng = np.random.default_rng(w * 7 + h)
    if kind == "noise":
        px = rng.integers(0, 256, (h, w), dtype=np.uint8)
    elif kind == "runs":
        px = np.repeat(rng.integers(0, 256, (h, w // 64 + 1), dtype=np.uint8), 64, axis=1)[:, :w].copy()
    else:
        px = np.full((h, w), 77, np.uint8)
    raw, png = d / ("px_%d_%d_%s.bin" % (w, h, kind)), d / ("img_%d_%d_%s.png" % (w, h, kind))
    px.tofile(raw)
    subprocess.run([exe, str(png), str(w), str(h), str(raw)], check=True)
    got = read_png_gray8(str(png))
    assert got.shape == (h, w)
    assert np.array_equal(got, px)
