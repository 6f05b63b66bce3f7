"""Regenerates the golden fixtures in this folder from the reference checkout.

Run where the reference checkout is readable, passing its directory:
    python tests/golden/make_golden.py REF      (or SARBP_REFERENCE=REF)

Writes
  reference_known_answers.json  known-answer values of the reference's own
                                unit tests (test/taylor_test.cpp,
                                test/norm_test.cpp, test/cross_test.cpp,
                                test/linspace_test.cpp, test/arange_test.cpp,
                                test/interp_test.cpp),
                                parsed from the test sources
  afrl_img_plane.npz            RITSAR image-plane outputs for AFRL pass 1
                                (data/AFRL/pass1/HH_ip_npy/*.npy)
  afrl_input.npz                the AFRL pass-1 HH platform data
                                (data/AFRL/pass1/HH_npy/*.npy), the reference's
                                real-data input (469 pulses x 424 samples)
Only plain .npy arrays are read (allow_pickle=False); the *_npy_txt folders
hold pickled objects and are never opened.
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _read(ref, rel):
    with open(os.path.join(ref, rel)) as f:
        return f.read()


def _floats(s):
    return [float(x) for x in re.findall(r"-?\d+(?:\.\d+)?(?:e-?\d+)?", s)]


def known_answers(ref):
    out = {}
    src = _read(ref, "test/taylor_test.cpp")
    n = int(re.search(r"#define\s+INPUT_NUM\s+(\d+)", src).group(1))
    table = _floats(re.search(r"reference\[INPUT_NUM\]\s*=\s*\{([^}]*)\}", src).group(1))
    sl = float(re.search(r"taylor\(INPUT_NUM,\s*([\d.]+)\s*,", src).group(1))
    tol = float(re.search(r">=\s*([\d.]+)f?\)", src).group(1))
    assert len(table) == n
    out["taylor"] = {"num": n, "S_L": sl, "expected": table, "tol": tol,
                     "source": "test/taylor_test.cpp:11-31"}

    src = _read(ref, "test/norm_test.cpp")
    in1 = _floats(re.search(r"float in\[X_LEN\]\s*=\s*\{([^}]*)\}", src).group(1))
    exp1 = float(re.search(r"out_buf\(\)\s*!=\s*([\d.]+)", src).group(1))
    in2 = _floats(re.search(r"float in\[X_LEN \* Y_LEN\]\s*=\s*\{([^}]*)\}", src).group(1))
    exp2 = [float(x) for x in re.findall(r"out_buf\((\d)\)\s*!=\s*([\d.]+)", src) and
            [m[1] for m in re.findall(r"out_buf\((\d)\)\s*!=\s*([\d.]+)", src)]]
    out["norm"] = {"in1": in1, "expected1": exp1, "in2": in2, "expected2": exp2,
                   "source": "test/norm_test.cpp:15-46"}

    src = _read(ref, "test/cross_test.cpp")
    a = _floats(re.search(r"float a\[N\]\s*=\s*\{([^}]*)\}", src).group(1))
    b = _floats(re.search(r"float b\[N\]\s*=\s*\{([^}]*)\}", src).group(1))
    exp = []
    for i, sign, val in re.findall(r"abs\(obuf\[(\d)\]\s*([+-])\s*([\d.]+)\)", src):
        exp.append(-float(val) if sign == "+" else float(val))
    tol = float(re.search(r">=\s*([\d.]+)f", src).group(1))
    out["cross"] = {"a": a, "b": b, "expected": exp, "tol": tol, "source": "test/cross_test.cpp:14-31"}

    src = _read(ref, "test/linspace_test.cpp")
    out["linspace"] = {
        "num": int(re.search(r"#define\s+INPUT_NUM\s+(\d+)", src).group(1)),
        "start": float(re.search(r"#define\s+START\s+(-?[\d.]+)f", src).group(1)),
        "stop": float(re.search(r"#define\s+STOP\s+(-?[\d.]+)f", src).group(1)),
        "tol": float(re.search(r">=\s*([\d.]+)f", src).group(1)),
        "source": "test/linspace_test.cpp:15-37 (expected: start + i*step, last = stop)"}

    src = _read(ref, "test/arange_test.cpp")
    start = float(re.search(r"#define\s+START\s+(-?[\d.]+)f", src).group(1))
    stop = float(re.search(r"#define\s+STOP\s+(-?[\d.]+)f", src).group(1))
    step = float(re.search(r"#define\s+STEP\s+(-?[\d.]+)f", src).group(1))
    listed = _floats(re.search(r"output should be:\s*\[([^\]]*)\]", src).group(1))
    out["arange"] = {"start": start, "stop": stop, "step": step, "expected": listed,
                     "tol": float(re.search(r">=\s*([\d.]+)f", src).group(1)),
                     "source": "test/arange_test.cpp:18-40"}

    src = _read(ref, "test/interp_test.cpp")
    arr = lambda name: _floats(re.search(r"float %s\[\w+\]\s*=\s*\{([^}]*)\}" % name, src).group(1))
    out["interp"] = {"xs": arr("xs"), "xp": arr("xp"), "fp": arr("fp"),
                     "expected": _floats(re.search(r"output should be:\s*\[([^\]]*)\]", src).group(1)),
                     "tol": float(re.search(r">=\s*([\d.]+)f", src).group(1)),
                     "source": "test/interp_test.cpp:15-26"}
    return out


def main():
    # the reference checkout: the first argument, else $SARBP_REFERENCE
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SARBP_REFERENCE")
    if not ref:
        sys.exit("usage: make_golden.py REFERENCE_DIR (or set SARBP_REFERENCE)")
    ka = known_answers(ref)
    with open(os.path.join(HERE, "reference_known_answers.json"), "w") as f:
        json.dump(ka, f, indent=1)
    ip_dir = os.path.join(ref, "data/AFRL/pass1/HH_ip_npy")
    ip = {k: np.load(os.path.join(ip_dir, k + ".npy"), allow_pickle=False)
          for k in ("u", "v", "k_u", "k_v", "du", "dv", "u_hat", "v_hat", "n_hat")}
    np.savez_compressed(os.path.join(HERE, "afrl_img_plane.npz"), **ip)
    pd_dir = os.path.join(ref, "data/AFRL/pass1/HH_npy")
    pd = {k: np.load(os.path.join(pd_dir, k + ".npy"), allow_pickle=False)
          for k in ("phs", "pos", "k_r", "delta_r", "R_c", "nsamples", "npulses", "freq")}
    np.savez_compressed(os.path.join(HERE, "afrl_input.npz"), **pd)
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    main()
