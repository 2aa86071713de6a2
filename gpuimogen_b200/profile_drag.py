"""Small-case driver for profiling the drag kernels with Nsight Compute.

Builds the 2-D gas-dust state of gpuimogen_b200.dusty on an n x n grid, trains a small drag model
(200k exact labels, 2 epochs), then runs one exact LogTrap2 drag call (logtrap_kernel) and one
learned call (mlp_tc_kernel<1>).  Usage:
  python -m gpuimogen_b200.profile_drag [--n 1024]
"""
import argparse

import torch

import gpuimogen_b200 as ib
from gpuimogen_b200 import dusty
from gpuimogen_b200 import learned_drag as ld


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1024)
    a = ap.parse_args()
    ib.load("product")
    model, _ = ld.train(n_samples=200_000, epochs=2, seed=3, batch=8192)
    exact = dusty.DustyRun(a.n)
    learned = dusty.DustyRun(a.n, model=model)
    dt = 4e-5
    exact.drag([exact.gas, exact.dust], dt)
    learned.drag([learned.gas, learned.dust], dt)
    torch.cuda.synchronize()
    print("profile_drag done", a.n, "fallbacks", int(learned.fallbacks.item()))


if __name__ == "__main__":
    main()
