"""CPU-only checks of the oracle: known-answer problems of the reference's test suite.

The reference pins its fluid path with the Sod shock tube against the exact Riemann solution
(run/test_suite/tsSod.m:40-77, experiment/RiemannProblem/analysis/SodShockSolution.m) and its
closed-form unit tests (gpuclass/unitTest.m: soundspeed :409-453, freezeAndPtot :647-680).
"""
import math

import numpy as np
import pytest

import riemann_exact as rx
from gpuimogen_b200 import problems


def run_sod_oracle(po, n, method, bc, T=0.2, cfl=0.4, gamma=1.4):
    q = problems.sod(n, gamma)
    h = 1.0 / n
    sp = po.step_params(0.0, (h, 1.0, 1.0), gamma, rho_min=1e-5, method=method)
    t, it, kc = 0.0, 0, 0.0
    while t < T * (1 - 1e-14):
        tau = po.cfl_timestep(q, (n, 1, 1), gamma, (h, 1.0, 1.0), method)
        dt = cfl * tau
        if t + 2 * dt > T:
            dt = .5 * (T - t)
        sp.dt = dt
        po.fluid_step_3d(q, (n, 1, 1), sp, [bc, bc, "circular", "circular", "circular", "circular"], 1, it)
        po.fluid_step_3d(q, (n, 1, 1), sp, [bc, bc, "circular", "circular", "circular", "circular"], -1, it)
        y = 2 * dt - kc
        tn = t + y
        kc = (tn - t) - y
        t = tn
        it += 1
    return q, t, it


@pytest.mark.parametrize("method,l1max", [(2, 1.5e-3), (1, 1.5e-3), (3, 2.0e-3)])
def test_sod_const_matches_exact(po, method, l1max):
    n = 256
    q, t, it = run_sod_oracle(po, n, method, "const")
    x = (np.arange(n) + 0.5) / n
    ex = rx.sample(x, t, 0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1), 1.4)
    l1 = np.mean(np.abs(q[0, :n] - ex[0]))
    assert abs(t - 0.2) < 1e-14
    assert l1 < 4 * l1max, l1   # coarse grid: 4x the 1024-cell bound
    assert np.all(q[0, :n] > 0)


def test_sod_convergence_first_order_or_better(po):
    errs = []
    for n in (128, 256, 512):
        q, t, _ = run_sod_oracle(po, n, 2, "const")
        x = (np.arange(n) + 0.5) / n
        ex = rx.sample(x, t, 0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1), 1.4)
        errs.append(np.mean(np.abs(q[0, :n] - ex[0])))
    rate = math.log(errs[0] / errs[2], 4.0)
    assert rate > 0.6, errs   # shocks limit Sod to ~first order in L1 (tsSod.m reports the same)


def test_soundspeed_closed_form(po):
    shape = (13, 7, 5)
    q = problems.random_smooth(shape, gamma=5 / 3.0, seed=3)
    n = 13 * 7 * 5
    cs = po.soundspeed(q, shape, 5 / 3.0)
    rho, E, px, py, pz = (q[k, :n] for k in range(5))
    e = E - 0.5 * (px ** 2 + py ** 2 + pz ** 2) / rho
    ref = np.sqrt(np.maximum(0, 5 / 3.0 * (2 / 3.0) * e / rho))
    assert np.allclose(cs, ref, rtol=1e-10, atol=0)   # unitTest.m:409-453 tolerance


def test_freeze_and_ptot_closed_form(po):
    shape = (16, 6, 3)
    q = problems.random_smooth(shape, gamma=1.4, seed=5)
    n = 16 * 6 * 3
    rho, E, px, py, pz = (q[k, :n].copy() for k in range(5))
    ptot, freeze = po.freeze_and_ptot(q, shape, 1.4, 0.0)
    P = 0.4 * (E - 0.5 * (px ** 2 + py ** 2 + pz ** 2) / rho)
    cf = (np.sqrt(1.4 * P / rho) + np.abs(px / rho)).reshape(3, 6, 16).max(axis=2).reshape(-1)
    assert np.allclose(ptot, P, rtol=1e-10)
    assert np.allclose(freeze, cf, rtol=1e-10)      # unitTest.m:647-680 tolerance


def test_hllc_direction_symmetry_bitexact(po):
    """A y (z) sweep equals an x sweep of the transposed array with the momenta relabelled,
    bit for bit: the per-direction slab maps are the only direction dependence."""
    nx, ny, nz = 12, 10, 9
    q = problems.random_jumpy((nx, ny, nz), seed=21)
    n = nx * ny * nz
    sp = po.step_params(2e-3, (0.1, 0.1, 0.1), 1.4, method=2, slope="mc")
    a = q.copy()
    po.fluid_sweep(a, (nx, ny, nz), sp, 2)
    # transpose x<->y and swap px<->py
    f = q[:, :n].reshape(5, nz, ny, nx).transpose(0, 1, 3, 2).copy()
    f = f[[0, 1, 3, 2, 4]]
    b = problems.pack((ny, nx, nz), *[f[k] for k in range(5)])
    po.fluid_sweep(b, (ny, nx, nz), sp, 1)
    bb = b[:, :n].reshape(5, nz, nx, ny)[[0, 1, 3, 2, 4]].transpose(0, 1, 3, 2).reshape(5, n)
    assert np.array_equal(a[:, :n], bb)


def test_drag_dustybox_conserves_momentum_energy(po):
    """Drag exchanges momentum and heats the gas but conserves total momentum and energy
    (DustyBox, experiment/Advection/DustyBoxAnalyzer.m)."""
    shape = (8, 4, 1)
    n = 32
    gas = problems.pack(shape, 1.0, 1.0 / (5 / 3.0 - 1) + 0.5 * 0.01, 0.1, 0.0, 0.0)
    dust = problems.pack(shape, np.linspace(0.05, 1.0, n).reshape(1, 4, 8), 0.0, 0.0, 0.0, 0.0)
    dust[1, :n] = 0.5 * 0.0 + 1e-4 * dust[0, :n]
    tg = [5 / 3.0, 3.3e-27, 8.4e-6, 0.7, 2.4e-19, 0.2, 1.381e-23, -1]
    td = [1.01, 3e-11, 0, 0, math.pi * 25e-12, 0, 1.381e-23, 0.1]
    p0 = gas[2, :n] + dust[2, :n]
    e0 = gas[1, :n] + 0.5 * dust[2, :n] ** 2 / dust[0, :n]
    po.drag_2fluid(gas, dust, shape, tg, td, 1e-3, 4)
    assert np.allclose(gas[2, :n] + dust[2, :n], p0, rtol=1e-13, atol=1e-15)
    assert np.allclose(gas[1, :n] + 0.5 * dust[2, :n] ** 2 / dust[0, :n], e0, rtol=1e-12)
    assert np.all(np.abs(gas[2, :n] / gas[0, :n] - dust[2, :n] / dust[0, :n]) < 0.1)
