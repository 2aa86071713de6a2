"""Measurement studies for the benchmark configurations beyond the headline bench.

  python -m gpuimogen_b200.studies precision [--shape 512,512,256] [--steps 200]
      Kelvin-Helmholtz with the HLLC flux and MC limiter run twice from the same seeded state:
      FP64 throughout, and the FP32-flux form (flux and limiter arithmetic in FP32, conserved
      accumulation, CFL reduction and floors in FP64).  Prints one JSON line with both
      throughputs (Mcell-updates/s, CUDA events) and the relative L1 difference per field of
      the FP32-flux result against the FP64 result.

Every number comes from the library (no CPU path).
"""
import argparse
import json
import sys

import numpy as np
import torch

from . import imogen as ib
from . import problems
from .timestep import TimeManager, run_iteration


def _run(q0, shape, steps, precision, warmup=2):
    fl = ib.Fluid(shape, q=torch.from_numpy(q0).cuda(), gamma=5 / 3.0)
    geo = ib.Geometry(shape)
    num = ib.numerics(slope="mc", precision=precision)
    tm = TimeManager(cfl=0.4)
    # warm-up on a scratch copy so that the measured run starts from the seeded state
    if warmup:
        scratch = ib.Fluid(shape, q=fl.q.clone(), gamma=5 / 3.0)
        t2 = TimeManager(cfl=0.4)
        for _ in range(warmup):
            run_iteration([scratch], geo, t2, 2, num)
        del scratch
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        run_iteration([fl], geo, tm, 2, num)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    n = shape[0] * shape[1] * shape[2]
    return fl, n * steps / (ms / 1e3) / 1e6, tm.time


def precision(shape, steps, seed=12345):
    q0 = problems.kelvin_helmholtz(shape, gamma=5 / 3.0, seed=seed)
    n = shape[0] * shape[1] * shape[2]
    f64, v64, t64 = _run(q0, shape, steps, "fp64")
    f32, v32, t32 = _run(q0, shape, steps, "fp32flux")
    a, b = f32.q[:, :n], f64.q[:, :n]
    den = b.abs().sum(dim=1)
    rel = ((a - b).abs().sum(dim=1) / den).cpu().numpy()
    mom = float(((a[2:] - b[2:]).abs().sum() / b[2:].abs().sum()).item())
    return {
        "study": "precision", "workload": "kelvin_helmholtz_hllc_mc", "grid": list(shape), "steps": steps,
        "fp64_mcell_updates_per_s": v64, "fp32flux_mcell_updates_per_s": v32, "speedup": v32 / v64,
        "rel_l1_vs_fp64": {"rho": float(rel[0]), "E": float(rel[1]), "px": float(rel[2]), "py": float(rel[3]),
                           "pz": float(rel[4]), "momentum": mom},
        "time_fp64": t64, "time_fp32flux": t32,
    }


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("study", choices=["precision"])
    ap.add_argument("--shape", default="512,512,256")
    ap.add_argument("--steps", type=int, default=200)
    a = ap.parse_args(argv)
    shape = tuple(int(s) for s in a.shape.split(","))
    ib.load("product")
    if a.study == "precision":
        print(json.dumps(precision(shape, a.steps)), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
