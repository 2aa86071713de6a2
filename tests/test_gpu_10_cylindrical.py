"""Cylindrical geometry on the GPU (x = r, y = theta, z = z): radial and theta sweeps of HLLC, HLL
(adiabatic and isothermal) and Xin-Jin in both theta memory layouts, with the reference's radius
arithmetic and with the geometric radius, the cylindrical CFL and the complete timestep with the
cylinder source terms (alone and split around the two-fluid drag), against the CPU oracle: bit for
bit in the strict build, within 1e-12 relative L1 as built.  Where the golden vectors of the
reference's own kernels exist, the strict build must reproduce them too.
"""
import json
import os

import numpy as np
import pytest

from gpuimogen_b200 import dusty, problems
from helpers import bits_equal, first_diff, host, oracle_cyl_loop, rel_l1, to_fluid

pytestmark = pytest.mark.gpu

H = [0.05, 0.04, 0.1]
RIN = 1.0
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cylindrical.npz")
SWEEPS = [(1, 0), (2, 0), (2, 1)]


def _n(shape):
    return shape[0] * shape[1] * shape[2]


@pytest.mark.parametrize("variant", ["strict", "product"])
@pytest.mark.parametrize("geometric", [False, True])
# radial rows up to 512 cells take the row kernel, theta pencils of at least 64 cells with x even
# the pencil-pair kernels ((12, 72, 3)); shorter theta pencils, or x odd, the tile kernel (or the
# Xin-Jin pencil kernel); (520, 6, 1) sends the radial rows to the tile kernel, (256, 4, 2) to the
# 256-cell row kernel
@pytest.mark.parametrize("shape", [(32, 24, 6), (32, 24, 1), (20, 9, 5), (21, 9, 5), (520, 6, 1), (12, 72, 3),
                                   (256, 4, 2)])
@pytest.mark.parametrize("method,c_iso", [(2, -1.0), (1, -1.0), (1, 0.8), (3, -1.0)])
def test_cyl_sweeps_vs_oracle(cuda, ib, po, variant, geometric, shape, method, c_iso):
    n = _n(shape)
    q0 = problems.rotating_annulus(shape, r_inner=RIN, dr=H[0], seed=13)
    geo = ib.Geometry(shape, h=H, cylindrical=True, r_inner=RIN)
    num = ib.numerics(slope="mc", geometric_radius=geometric)
    gamma = 1.4
    ib.use_variant(variant)
    try:
        for d, form in SWEEPS:
            fl = to_fluid(q0.copy(), shape, gamma=gamma, c_iso=c_iso)
            ib.cudaFluidStep(fl, geo, [0.004, 1, gamma, 1e-5, method, d, c_iso, form], num)
            out = host(fl)
            ref = q0.copy()
            sp = po.step_params(0.004, H, 2.0 if c_iso != -1 else gamma, c_iso=c_iso, method=method, slope="mc",
                                cylindrical=True, r_inner=RIN, theta_form=form, geometric_radius=geometric)
            po.fluid_sweep(ref, shape, sp, d)
            assert not np.array_equal(ref[:, :n], q0[:, :n])
            if variant == "strict":
                assert bits_equal(out, ref, n), (d, form, first_diff(out, ref, n))
            else:
                err = rel_l1(out, ref, n)
                assert np.all(err <= 1e-12), (d, form, err)
    finally:
        ib.use_variant("product")
    assert ib.device_wait_status() == 0


@pytest.mark.parametrize("shape", [(24, 20, 6), (24, 20, 1), (24, 1, 1)])
@pytest.mark.parametrize("method", [1, 2, 3])
def test_cyl_cfl_vs_oracle(cuda, ib, po, shape, method):
    q = problems.rotating_annulus(shape, r_inner=RIN, dr=H[0], seed=43)
    geo = ib.Geometry(shape, h=H, cylindrical=True, r_inner=RIN)
    fl = to_fluid(q.copy(), shape, gamma=1.4)
    t = ib.cflTimestepFused(fl, 1.4, geo, method)
    ref = po.cfl_timestep(q, shape, 1.4, H, method, cylindrical=True, r_inner=RIN)
    assert abs(t - ref) <= 1e-15 * ref, (t, ref)


CASES = [
    # shape, method, gamma, c_iso, bc, niter
    ((24, 20, 6), 2, 1.4, -1.0, ["const", "const"] + ["circular"] * 4, 6),
    ((24, 32, 1), 1, 1.4, -1.0, ["const", "const"] + ["circular"] * 4, 6),
    ((24, 32, 1), 2, 5 / 3.0, -1.0, ["mirror", "const"] + ["circular"] * 4, 6),
    ((24, 32, 1), 1, 1.4, 0.8, ["const", "const"] + ["circular"] * 4, 6),
    ((32, 32, 3), 3, 1.4, -1.0, ["const", "const"] + ["circular"] * 4, 6),
    ((20, 16, 8), 3, 1.4, -1.0, ["outflow", "mirror"] + ["circular"] * 4, 4),
]


@pytest.mark.parametrize("variant", ["strict", "product"])
@pytest.mark.parametrize("case", CASES, ids=lambda c: "%dx%dx%d_m%d" % (c[0] + (c[1],)))
def test_cyl_main_loop_vs_oracle(cuda, ib, po, variant, case):
    shape, method, gamma, c_iso, bc, niter = case
    n = _n(shape)
    cfl = 0.4 if method != 3 else 0.3
    q0 = problems.rotating_annulus(shape, r_inner=RIN, dr=H[0], gamma=gamma, seed=47)
    geo = ib.Geometry(shape, h=H, cylindrical=True, r_inner=RIN)
    ib.use_variant(variant)
    try:
        fl = to_fluid(q0.copy(), shape, bc=bc, gamma=gamma, c_iso=c_iso)
        tm = ib.TimeManager(cfl=cfl)
        dts = np.array([ib.run_iteration([fl], geo, tm, method) for _ in range(niter)])
        out = host(fl)
    finally:
        ib.use_variant("product")
    ref = q0.copy()
    dref = oracle_cyl_loop(po, ref, shape, H, RIN, method, gamma, c_iso, bc, cfl, niter)
    if variant == "strict":
        assert np.array_equal(dts, dref), np.max(np.abs(dts - dref))
        assert bits_equal(out, ref, n), first_diff(out, ref, n)
    else:
        assert np.all(np.abs(dts - dref) <= 1e-13 * dref)
        assert np.all(rel_l1(out, ref, n) <= 1e-12), rel_l1(out, ref, n)


@pytest.mark.parametrize("variant", ["strict", "product"])
def test_cyl_two_fluid_drag_vs_oracle(cuda, ib, po, variant):
    """Gas + dust in cylindrical geometry: the source is cylinder dt/2, drag dt, cylinder dt/2
    (srcC__D) around and between the fluid steps."""
    shape = (24, 20, 1)
    n = _n(shape)
    gas = problems.rotating_annulus(shape, r_inner=RIN, dr=H[0], gamma=5 / 3.0, seed=51)
    dust = problems.rotating_annulus(shape, r_inner=RIN, dr=H[0], gamma=5 / 3.0, seed=52)
    dust[0] *= 0.3
    for k in (2, 3, 4):
        dust[k] *= 0.3
    dust[1, :n] = 0.5 * (dust[2, :n] ** 2 + dust[3, :n] ** 2 + dust[4, :n] ** 2) / dust[0, :n] + 1e-4 * dust[0, :n]
    tg, td = dusty.ld.THERMO_GAS, dusty.ld.THERMO_DUST
    bc = ["const", "const"] + ["circular"] * 4
    geo = ib.Geometry(shape, h=H, cylindrical=True, r_inner=RIN)
    num = ib.numerics(slope="ospre")
    ib.use_variant(variant)
    try:
        g = to_fluid(gas.copy(), shape, bc=bc, gamma=tg[0])
        d = to_fluid(dust.copy(), shape, bc=bc, gamma=td[0], c_iso=td[7])
        tm = ib.TimeManager(cfl=0.4)
        dts = np.array([ib.run_iteration([g, d], geo, tm, 2, num, drag=(tg, td, "logtrap2")) for _ in range(5)])
        og, od = host(g), host(d)
    finally:
        ib.use_variant("product")
    rg, rd = gas.copy(), dust.copy()
    dref = oracle_cyl_loop(po, rg, shape, H, RIN, 2, tg[0], -1.0, bc, 0.4, 5, drag=(tg, td, 4), dust=rd)
    if variant == "strict":
        assert np.array_equal(dts, dref)
        assert bits_equal(og, rg, n), first_diff(og, rg, n)
        assert bits_equal(od, rd, n), first_diff(od, rd, n)
    else:
        assert np.all(rel_l1(og, rg, n) <= 1e-12) and np.all(rel_l1(od, rd, n) <= 1e-12)
    assert not np.array_equal(od[2, :n], dust[2, :n])


def test_cyl_golden_reference_kernels(cuda, ib):
    """The strict build against the reference's own kernels (strict): single sweeps and loops."""
    if not os.path.exists(GOLD):
        pytest.skip("cylindrical golden vectors not generated")
    z = np.load(GOLD)
    meta = json.loads(str(z["meta"]))
    h, rin = meta["h"], meta["r_inner"]
    ib.use_variant("strict")
    try:
        for case in meta["sweeps"]:
            shape = tuple(case["shape"])
            n = _n(shape)
            geo = ib.Geometry(shape, h=h, cylindrical=True, r_inner=rin)
            for d, form in SWEEPS:
                fl = to_fluid(z["in_" + case["name"]].copy(), shape, gamma=1.4, c_iso=case["c_iso"])
                ib.cudaFluidStep(fl, geo, [meta["dt"], 1, 1.4, 1e-5, case["method"], d, case["c_iso"], form])
                ref = z["out_%s_d%d_f%d_strict" % (case["name"], d, form)]
                out = host(fl)
                assert bits_equal(out, ref, n), (case["name"], d, form, first_diff(out, ref, n))
        for case in meta["runs"]:
            shape = tuple(case["shape"])
            n = _n(shape)
            geo = ib.Geometry(shape, h=h, cylindrical=True, r_inner=rin)
            fl = to_fluid(z["run_in_" + case["name"]].copy(), shape, bc=case["bc"], gamma=case["gamma"],
                          c_iso=case["c_iso"])
            tm = ib.TimeManager(cfl=case["cfl"])
            dts = np.array([ib.run_iteration([fl], geo, tm, case["method"]) for _ in range(case["niter"])])
            assert np.array_equal(dts, z["run_dts_%s_strict" % case["name"]]), case["name"]
            out, ref = host(fl), z["run_out_%s_strict" % case["name"]]
            assert bits_equal(out, ref, n), (case["name"], first_diff(out, ref, n))
    finally:
        ib.use_variant("product")
