"""Per-direction sweep timing with CUDA events.

Times one `cudaFluidStep` sweep along each axis (x, y, z; an axis shorter than 3 cells is
skipped) on the Kelvin-Helmholtz state, after one untimed sweep, as the mean of --reps launches.
Usage:
  python -m gpuimogen_b200.time_sweeps --shape 256,256,256 [--method 3] [--fluxlim vanleer]
                                       [--slope mc] [--precision fp64] [--reps 5]
Prints one line per shape: shape, method and the three times in ms.
"""
import argparse

import torch

import gpuimogen_b200 as ib
from gpuimogen_b200 import problems


def time_directions(shape, method, num, reps=5, gamma=5 / 3.0):
    q = problems.kelvin_helmholtz(shape, seed=1)
    fl = ib.Fluid(shape, q=torch.from_numpy(q).cuda(), gamma=gamma)
    geo = ib.Geometry(shape)
    out = []
    for d in (1, 2, 3):
        if shape[d - 1] < 3:
            out.append(None)
            continue
        params = [1e-5, 1, gamma, 1e-5, method, d]
        ib.cudaFluidStep(fl, geo, params, num)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            ib.cudaFluidStep(fl, geo, params, num)
        b.record()
        torch.cuda.synchronize()
        out.append(round(a.elapsed_time(b) / reps, 3))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--shape", action="append", required=True, help="nx,ny,nz (repeatable)")
    ap.add_argument("--method", type=int, default=2)
    ap.add_argument("--slope", default="mc")
    ap.add_argument("--fluxlim", default="vanleer")
    ap.add_argument("--precision", default="fp64")
    ap.add_argument("--reps", type=int, default=5)
    a = ap.parse_args()
    ib.load("product")
    num = ib.numerics(slope=a.slope, fluxlim=a.fluxlim, precision=a.precision)
    for s in a.shape:
        shape = tuple(int(v) for v in s.split(","))
        print(shape, "method", a.method, "ms x/y/z", time_directions(shape, a.method, num, a.reps), flush=True)


if __name__ == "__main__":
    main()
