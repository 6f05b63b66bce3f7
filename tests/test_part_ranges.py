"""Pulse parts of the work items (part_range, csrc/internal.h) on the CPU:
for every pulse count and part count the parts are consecutive, cover
[0, P) exactly once, differ in length by at most one pulse, and one part
is the whole aperture.  A small harness is compiled against the header."""
import os
import subprocess

import pytest

from conftest import PKG

HARNESS = r"""
#include <cstdio>
#include "internal.h"
int main() {
    for (int P = 1; P <= 700; ++P)
        for (int ns = 0; ns <= 16; ++ns) {
            if (ns > P) continue;
            int prev = 0, lo = 1 << 30, hi = 0;
            const int parts = ns < 1 ? 1 : ns;
            for (int s = 0; s < parts; ++s) {
                int p0, p1;
                sarbp::part_range(P, ns, s, p0, p1);
                if (p0 != prev || p1 <= p0) { std::printf("bad P=%d ns=%d s=%d [%d,%d)\n", P, ns, s, p0, p1); return 1; }
                lo = p1 - p0 < lo ? p1 - p0 : lo;
                hi = p1 - p0 > hi ? p1 - p0 : hi;
                prev = p1;
            }
            if (prev != P || hi - lo > 1) { std::printf("bad cover P=%d ns=%d\n", P, ns); return 1; }
        }
    int p0, p1;
    sarbp::part_range(2000000000, 16, 15, p0, p1);  // no overflow at large P
    if (p1 != 2000000000 || p0 != 1875000000) { std::printf("overflow\n"); return 1; }
    std::printf("ok\n");
    return 0;
}
"""


def test_part_ranges_cover_the_aperture(tmp_path):
    src = tmp_path / "parts.cpp"
    src.write_text(HARNESS)
    exe = str(tmp_path / "parts")
    cuda_inc = "/usr/local/cuda/include"
    if not os.path.isdir(cuda_inc):
        pytest.skip("CUDA headers not found")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(PKG, "csrc"), "-I", cuda_inc, str(src), "-o", exe],
                   check=True)
    p = subprocess.run([exe], capture_output=True, text=True)
    assert p.returncode == 0 and p.stdout.strip() == "ok", p.stdout
