import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "halide-sar-app_b200")
for p in (PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA kernels)")


@pytest.fixture(scope="session")
def known_answers():
    with open(os.path.join(GOLDEN, "reference_known_answers.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def afrl_input():
    return dict(np.load(os.path.join(GOLDEN, "afrl_input.npz"), allow_pickle=False))


@pytest.fixture(scope="session")
def afrl_img_plane():
    return dict(np.load(os.path.join(GOLDEN, "afrl_img_plane.npz"), allow_pickle=False))


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def sb():
    import sarbp_b200
    return sarbp_b200


@pytest.fixture(scope="session")
def ctx(sb):
    c = sb.Context(0)
    yield c
    c.close()


def rel_l2(a, b):
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def db_image(img):
    a = np.abs(np.asarray(img, np.complex128))
    with np.errstate(divide="ignore"):
        return 10.0 * np.log10(a / a.max())


def db_max_diff(img, ref, floor_db):
    """max |dB(img) - dB(ref)| over the pixels that ref shows above floor_db
    (the displayed dynamic range; both images scaled by their own max)."""
    d1, d2 = db_image(img), db_image(ref)
    m = d2 >= floor_db
    return float(np.abs(d1[m] - d2[m]).max())
