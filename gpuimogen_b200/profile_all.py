"""Small-case driver that launches every kind of kernel of the library once, for an Nsight Compute
launch table (duration, DRAM bytes, FP64 and tensor pipes) covering the whole library.

Cases: the Kelvin-Helmholtz state at --n^3 (default 160^3: 164 MB of state, above the 126 MB L2)
for the fluid kernels; KH on 512 x 512 x 8 (z sweeps of 2 MB planes: the wide-block kernels) and
on 2048 x 2048 x 1 (x and y pencils of 2048 cells: the chunked pipeline and its halo copy); the
2-D gas-dust state at --m^2 (default 1024^2) for the drag kernels (ETDRK2 included); a
592-problem Riemann ensemble (4 iterations) for the ensemble kernel; a 65536-sample batch for the
MLP training kernels.  Usage:
  python -m gpuimogen_b200.profile_all [--n 160] [--m 1024]
"""
import argparse

import torch

import gpuimogen_b200 as ib
from gpuimogen_b200 import dusty, ensemble, problems
from gpuimogen_b200 import learned_drag as ld


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=160)
    ap.add_argument("--m", type=int, default=1024)
    a = ap.parse_args()
    ib.load("product")
    shape = (a.n, a.n, a.n)
    q = problems.kelvin_helmholtz(shape, seed=1)
    geo = ib.Geometry(shape)
    dt = 1e-5
    # HLLC FP64 / FP32 flux, HLL, Xin-Jin sweeps (x, y, z each)
    for method, prec in ((2, "fp64"), (2, "fp32flux"), (1, "fp64"), (3, "fp64")):
        fl = ib.Fluid(shape, q=torch.from_numpy(q).cuda(), gamma=5 / 3.0)
        num = ib.numerics(slope="mc", precision=prec)
        for d in (1, 2, 3):
            ib.cudaFluidStep(fl, geo, [dt, 1, 5 / 3.0, 1e-5, method, d], num)
    # z sweeps of large x-y planes (FP64 4-column blocks, FP32 flux 8-column wide blocks)
    shp = (512, 512, 8)
    qw = problems.kelvin_helmholtz(shp, seed=2)
    for prec in ("fp64", "fp32flux"):
        fw = ib.Fluid(shp, q=torch.from_numpy(qw).cuda(), gamma=5 / 3.0)
        ib.cudaFluidStep(fw, ib.Geometry(shp), [dt, 1, 5 / 3.0, 1e-5, 2, 3], ib.numerics(slope="mc", precision=prec))
    del fw
    # pencils of 2048 cells: chunked pipeline (x and y), each after its halo copy
    shp = (2048, 2048, 1)
    fc = ib.Fluid(shp, q=torch.from_numpy(problems.kelvin_helmholtz(shp, seed=3)).cuda(), gamma=5 / 3.0)
    for d in (1, 2):
        ib.cudaFluidStep(fc, ib.Geometry(shp), [dt, 1, 5 / 3.0, 1e-5, 2, d], ib.numerics(slope="mc"))
    del fc
    # CFL (fused soundspeed), freezeAndPtot, boundary fill (outflow), statics-free
    fl = ib.Fluid(shape, q=torch.from_numpy(q).cuda(), gamma=5 / 3.0, bc="outflow")
    ib.cflTimestepFused(fl, 5 / 3.0, geo, 2)
    ib.freezeAndPtot(fl, 5 / 3.0, 1, 0.0)
    ib.setFluidBoundary(fl, 1)
    # drag integrators on the 2-D gas-dust state
    run = dusty.DustyRun(a.m)
    for method in ("logtrap2", "rk4", "etdrk1", "etdrk2"):
        run.reset()
        ib.cudaSource2FluidDrag(run.gas, run.dust, run.tg, run.td, run.geo, [4e-5, ib.DRAG[method]])
    # learned drag (small model) and the MLP training kernels
    model, _ = ld.train(n_samples=65536 * 4, epochs=1, seed=3, batch=65536)
    run.reset()
    ld.drag_step(run.gas, run.dust, model, 4e-5)
    # ensemble
    ens = ensemble.RiemannEnsemble.random(592, seed=2)
    ens.run(t_end=0.1, itermax=4, tuning={"threads": 512, "chunk": 504})
    torch.cuda.synchronize()
    print("profile_all done")


if __name__ == "__main__":
    main()
