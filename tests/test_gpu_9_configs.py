"""Parity at the sizes of the benchmark configurations.

* Kelvin-Helmholtz 256^3, HLLC, MC limiter, 100 iterations (the FP64 drop-in's headline case),
  against the reference's own GPU kernels (its gpuclass sources built for sm_100a into
  oracle/_ref by oracle/ref_harness/Makefile; the test is skipped where that build is absent):
  the strict builds of both (every operation as the source writes it) agree bit for bit, every
  dt included; the library as built (FMA contraction) agrees with the reference as it builds
  itself within 1e-12 relative L1 per field, and every dt within 1e-13.
* The Sod shock tube as configured: 1024 cells on [0, 1], gamma 1.4, (1, 0, 1) | (0.125, 0, 0.1),
  CFL 0.4, to t = 0.2, Xin-Jin and HLL, outflow and const boundaries: the same iteration count
  and state as the oracle (1e-12 relative L1 per field), and the density's L1 distance to the
  exact solution (run/test_suite/tsSod.m:40-77).
* The precision form at its size: 512 x 512 x 256 Kelvin-Helmholtz, 200 iterations, the FP32-flux
  run within 1e-5 relative L1 of the FP64 run in density, energy and momentum.
"""
import ctypes
import os

import numpy as np
import pytest
import torch

import riemann_exact as rx
from gpuimogen_b200 import problems
from helpers import bits_equal, first_diff, host, rel_l1, to_fluid

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")


def _ref_lib(strict):
    path = os.path.join(REF, "libimogen_ref_mc%s.so" % ("_strict" if strict else ""))
    if not os.path.exists(path):
        pytest.skip("the reference's kernels are not built (oracle/ref_harness)")
    L = ctypes.CDLL(path)
    dp = ctypes.POINTER(ctypes.c_double)
    L.ref_run.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int64, ctypes.c_double,
                          ctypes.c_double, ctypes.c_double, ctypes.c_int, dp, ctypes.POINTER(ctypes.c_int),
                          ctypes.c_double, ctypes.c_int, dp]
    return L


@pytest.mark.parametrize("variant", ["strict", "product"])
def test_kh256_100_iterations_vs_reference_kernels(cuda, ib, variant):
    shape = (256, 256, 256)
    n = 256 ** 3
    niter = 100
    q0 = problems.kelvin_helmholtz(shape, gamma=5 / 3.0, seed=12345)
    # the reference's kernels, strict or as the reference builds itself
    L = _ref_lib(variant == "strict")
    ref = q0.copy()
    dts_ref = np.zeros(niter)
    h = np.array([1.0 / 256] * 3)
    bc = (ctypes.c_int * 6)(*[0] * 6)
    dp = ctypes.POINTER(ctypes.c_double)
    rc = L.ref_run(ref.ctypes.data_as(dp), 256, 256, 256, ref.shape[1], 5 / 3.0, 1e-5, -1.0, 2,
                   h.ctypes.data_as(dp), bc, 0.4, niter, dts_ref.ctypes.data_as(dp))
    assert rc == 0
    torch.cuda.synchronize()
    # the library
    ib.use_variant(variant)
    try:
        fl = to_fluid(q0, shape, gamma=5 / 3.0)
        geo = ib.Geometry(shape)
        tm = ib.TimeManager(cfl=0.4)
        num = ib.numerics(slope="mc")
        dts = np.array([ib.run_iteration([fl], geo, tm, 2, num) for _ in range(niter)])
        out = host(fl)
    finally:
        ib.use_variant("product")
    assert ib.device_wait_status() == 0
    err = rel_l1(out, ref, n)
    print("KH 256^3 x 100 (%s): rel L1 per field vs reference kernels %s, max dt rel diff %.3g"
          % (variant, np.array2string(err), np.max(np.abs(dts - dts_ref) / dts_ref)))
    if variant == "strict":
        assert np.array_equal(dts, dts_ref), np.max(np.abs(dts - dts_ref))
        assert bits_equal(out, ref, n), first_diff(out, ref, n)
    else:
        assert np.all(np.abs(dts - dts_ref) <= 1e-13 * dts_ref), np.max(np.abs(dts - dts_ref) / dts_ref)
        assert np.all(err <= 1e-12), err
    assert not np.array_equal(out[0, :n], q0[0, :n])


@pytest.mark.parametrize("bc", ["outflow", "const"])
@pytest.mark.parametrize("method", [3, 1])
def test_sod_1024_to_t02_matches_oracle_and_exact(cuda, ib, po, method, bc):
    n = 1024
    shape = (n, 1, 1)
    q0 = problems.sod(n)
    fl = to_fluid(q0, shape, bc=bc, gamma=1.4)
    geo = ib.Geometry(shape)
    tm = ib.TimeManager(cfl=0.4, tmax=0.2)
    while tm.running:
        ib.run_iteration([fl], geo, tm, method)
    out = host(fl)
    assert abs(tm.time - 0.2) < 1e-14
    # the oracle, with the reference's time bookkeeping (TimeManager.m:124-186, 270-277)
    ref = q0.copy()
    sp = po.step_params(0.0, geo.h, 1.4, method=method)
    t, it, kc = 0.0, 0, 0.0
    while t < 0.2 * (1 - 1e-14):
        dt = 0.4 * po.cfl_timestep(ref, shape, 1.4, geo.h, method)
        if t + 2 * dt > 0.2:
            dt = .5 * (0.2 - t)
        sp.dt = dt
        po.fluid_step_3d(ref, shape, sp, [bc] * 6, 1, it)
        po.fluid_step_3d(ref, shape, sp, [bc] * 6, -1, it)
        y = 2 * dt - kc
        tn = t + y
        kc = (tn - t) - y
        t = tn
        it += 1
    assert it == tm.iteration, (it, tm.iteration)
    err = rel_l1(out, ref, n)
    assert np.all(err <= 1e-12), err
    # the exact Riemann solution (tsSod.m compares the density): L1 over the cells
    x = (np.arange(n) + 0.5) / n
    ex = rx.sample(x, tm.time, 0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1), 1.4)
    l1 = float(np.mean(np.abs(out[0, :n] - ex[0])))
    print("Sod 1024 method %d %s: %d iterations, L1(rho) vs exact %.3e" % (method, bc, tm.iteration, l1))
    # the reference's outflow condition writes rho * 1.05 into the transverse momentum of inflow
    # boundary cells (cudaStatics.cu:379-384, 469-474), which the scheme carries into the grid:
    # the oracle's own L1 is 3.3e-3 (Xin-Jin) and 2.9e-3 (HLL) there against 1.0e-3 and 0.8e-3
    # with const boundaries
    assert l1 < (4.0e-3 if bc == "outflow" else 1.5e-3), l1


def test_kh_precision_form_512x512x256_200_steps(cuda, ib):
    shape = (512, 512, 256)
    n = shape[0] * shape[1] * shape[2]
    q0 = torch.from_numpy(problems.kelvin_helmholtz(shape, gamma=5 / 3.0, seed=12345)).cuda()
    geo = ib.Geometry(shape)
    final = {}
    for prec in ("fp64", "fp32flux"):
        fl = ib.Fluid(shape, q=q0.clone(), gamma=5 / 3.0)
        tm = ib.TimeManager(cfl=0.4)
        num = ib.numerics(slope="mc", precision=prec)
        for _ in range(200):
            ib.run_iteration([fl], geo, tm, 2, num)
        final[prec] = fl.q[:, :n]
    a, b = final["fp32flux"], final["fp64"]
    rel = ((a - b).abs().sum(dim=1) / b.abs().sum(dim=1)).cpu().numpy()
    mom = float(((a[2:] - b[2:]).abs().sum() / b[2:].abs().sum()).item())
    print("KH 512x512x256 x 200, FP32 flux vs FP64: rel L1 rho %.3g E %.3g momentum %.3g" % (rel[0], rel[1], mom))
    assert rel[0] <= 1e-5 and rel[1] <= 1e-5 and mom <= 1e-5, (rel, mom)
    assert ib.device_wait_status() == 0
