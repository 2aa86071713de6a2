"""Small-case driver for profiling the sweep kernels with Nsight Compute.

Runs one warm-up iteration of the Kelvin-Helmholtz problem, then one launch of each sweep
kernel (x, y, z; a sweep along an axis of extent 1 launches nothing) and one CFL reduction on a
grid whose state (5 FP64 slabs) exceeds the 126 MB L2: n^3, or --shape nx,ny,nz.  Usage:
  python -m gpuimogen_b200.profile_sweeps [--n 192 | --shape 2048,2048,1] [--precision fp64|fp32flux]
                                         [--method 2]
"""
import argparse

import torch

import gpuimogen_b200 as ib
from gpuimogen_b200 import problems


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=192)
    ap.add_argument("--shape", default=None, help="nx,ny,nz instead of n^3")
    ap.add_argument("--precision", default="fp64")
    ap.add_argument("--method", type=int, default=2)
    ap.add_argument("--slope", default="mc")
    a = ap.parse_args()
    shape = tuple(int(v) for v in a.shape.split(",")) if a.shape else (a.n, a.n, a.n)
    q = problems.kelvin_helmholtz(shape, seed=1)
    fl = ib.Fluid(shape, q=torch.from_numpy(q).cuda(), gamma=5 / 3.0)
    geo = ib.Geometry(shape)
    num = ib.numerics(slope=a.slope, precision=a.precision)
    tm = ib.TimeManager(cfl=0.4)
    ib.run_iteration([fl], geo, tm, a.method, num)        # warm-up: 1 CFL + 6 sweeps
    dt = tm.dTime
    for d in (1, 2, 3):
        ib.cudaFluidStep(fl, geo, [dt, 1, 5 / 3.0, 1e-5, a.method, d], num)
    ib.cflTimestepFused(fl, 5 / 3.0, geo, a.method)
    torch.cuda.synchronize()
    print("profile_sweeps done", shape, a.precision)


if __name__ == "__main__":
    main()
