"""Times the reference's own GPU implementation (oracle/_ref, built from its sources) on the
Kelvin-Helmholtz benchmark workload: 256^3 periodic, HLLC, MC limiter, CFL 0.4, gamma 5/3.
Test infrastructure: prints one JSON line; the figure is recorded in profiles/ next to ours.

Usage: python oracle/ref_harness/time_reference.py [--n 256] [--warmup 3] [--iters 20]
"""
import argparse
import ctypes
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from gpuimogen_b200 import problems  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--iters", type=int, default=20)
    ap.add_argument("--limiter", default="mc")
    a = ap.parse_args()
    L = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libimogen_ref_%s.so" % a.limiter))
    dp = ctypes.POINTER(ctypes.c_double)
    L.ref_time.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int64, ctypes.c_double,
                           ctypes.c_int, dp, ctypes.c_double, ctypes.c_int, ctypes.c_int, dp]
    shape = (a.n, a.n, a.n)
    q = problems.kelvin_helmholtz(shape, gamma=5 / 3.0, seed=12345)
    h = np.array([1.0 / a.n] * 3)
    ms = ctypes.c_double(0)
    rc = L.ref_time(q.ctypes.data_as(dp), a.n, a.n, a.n, q.shape[1], 5 / 3.0, 2, h.ctypes.data_as(dp), 0.4,
                    a.warmup, a.iters, ctypes.byref(ms))
    cells = a.n ** 3
    print(json.dumps({"impl": "reference_gpu", "rc": rc, "grid": list(shape), "iterations": a.iters,
                      "ms_per_iteration": ms.value / a.iters,
                      "mcell_updates_per_s": cells * a.iters / (ms.value / 1e3) / 1e6,
                      "limiter": a.limiter, "method": "HLLC"}))


if __name__ == "__main__":
    main()
