"""The oracle against golden vectors produced by the reference's own GPU code.

tests/golden/*.npz were generated by tests/golden/make_golden.py, which runs imogenproject/gpuImogen's
gpuclass sources (compiled unchanged for sm_100a by oracle/ref_harness/Makefile) on seeded inputs.
The reference built with -fmad=false ("strict") performs exactly the IEEE operations its source
writes, so the oracle (-ffp-contract=off) must reproduce it bit for bit; the reference as it builds
itself (FMA contraction on) must agree within 1e-12 relative L1 per field.
"""
import glob
import json
import os

import numpy as np
import pytest

from helpers import bits_equal, first_diff, rel_l1

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FLUID = sorted(p for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
               if os.path.basename(p) not in ("cfl.npz", "drag.npz", "drag_etdrk2.npz", "cylindrical.npz"))


def load(path):
    z = np.load(path)
    return json.loads(str(z["meta"])), z


def run_oracle(po, meta, q):
    shape = tuple(meta["shape"])
    h = [1.0 / s for s in shape]
    gamma = meta["gamma"]
    c_iso = meta["c_iso"]
    g_eff = 2.0 if c_iso != -1 else gamma
    sp = po.step_params(0.0, h, g_eff, rho_min=meta["rho_min"], c_iso=c_iso, method=meta["method"],
                        slope=meta["limiter"])
    dts = []
    for it in range(meta["niter"]):
        tau = po.cfl_timestep(q, shape, gamma, h, meta["method"])
        sp.dt = meta["cfl"] * tau
        dts.append(sp.dt)
        po.fluid_step_3d(q, shape, sp, meta["bc"], 1, it)
        po.fluid_step_3d(q, shape, sp, meta["bc"], -1, it)
    return np.array(dts)


def test_golden_vectors_present():
    assert len(FLUID) >= 8, "golden vectors missing: run tests/golden/make_golden.py on a GPU machine"


@pytest.mark.parametrize("path", FLUID, ids=[os.path.basename(p)[:-4] for p in FLUID])
def test_oracle_matches_reference_gpu(po, path):
    meta, z = load(path)
    shape = tuple(meta["shape"])
    n = shape[0] * shape[1] * shape[2]
    q = np.array(z["input"])
    dts = run_oracle(po, meta, q)
    assert np.array_equal(dts, z["dts_strict"]), (dts, z["dts_strict"])
    assert bits_equal(q, z["out_strict"], n), first_diff(q, z["out_strict"], n)
    err = rel_l1(q, z["out_fast"], n)
    assert np.all(err <= 1e-12), err


def test_oracle_cfl_matches_reference_gpu(po):
    from gpuimogen_b200 import problems
    path = os.path.join(GOLDEN, "cfl.npz")
    vals = json.loads(str(np.load(path)["values"]))
    gens = {"jumpy": ((17, 13, 9), 1.4, lambda s, g: problems.random_jumpy(s, gamma=g, seed=29)),
            "smooth": ((40, 30, 1), 5 / 3.0, lambda s, g: problems.random_smooth(s, gamma=g, seed=23, amp=0.3)),
            "sod": ((300, 1, 1), 1.4, lambda s, g: problems.sod(s[0], g))}
    for gen, (shape, gamma, make) in gens.items():
        q = make(shape, gamma)
        for method in (1, 2, 3):
            t = po.cfl_timestep(q, shape, gamma, (0.02, 0.03, 0.05), method)
            assert t == vals["%s_m%d_strict" % (gen, method)]
            assert abs(t - vals["%s_m%d_fast" % (gen, method)]) <= 1e-15 * t


@pytest.mark.parametrize("case", ["", "stiff_"])
@pytest.mark.parametrize("method", [0, 1, 2, 4, 5])
def test_oracle_drag_matches_reference_gpu(po, method, case):
    """EMP, RK4, ETDRK1, LogTrap2 and LogTrap3 against the reference's own kernels, weak drag
    (k dt ~ 1e-4) and stiff drag (k dt ~ 1)."""
    z = np.load(os.path.join(GOLDEN, "drag.npz"))
    meta = json.loads(str(z["meta"]))
    shape = tuple(meta["shape"])
    n = shape[0] * shape[1] * shape[2]
    g, d = np.array(z["gas"]), np.array(z["dust"])
    td = meta["td_stiff"] if case else meta["td"]
    po.drag_2fluid(g, d, shape, meta["tg"], td, meta["dt"], method)
    for tag in ("strict", "fast"):
        # pow/exp/expm1: glibc here, CUDA's math library in the reference
        for mine, ref in ((g, z["gas_%sm%d_%s" % (case, method, tag)]),
                          (d, z["dust_%sm%d_%s" % (case, method, tag)])):
            # the explicit EMP and RK4 integrators are unstable at k dt ~ 1 and produce NaN there;
            # the oracle must produce NaN in exactly the same cells
            bad = np.isnan(ref[:, :n])
            assert np.array_equal(np.isnan(mine[:, :n]), bad), tag
            a, b = np.where(bad, 0.0, mine[:, :n]), np.where(bad, 0.0, ref[:, :n])
            err = rel_l1(a, b, n)
            assert np.all(err <= 1e-12), (tag, err)


ETDRK2_SHAPES = [(16, 8, 1), (8, 6, 5), (12, 1, 6), (32, 1, 1)]


@pytest.mark.parametrize("case", ["", "stiff_"])
@pytest.mark.parametrize("shape", ETDRK2_SHAPES, ids=lambda s: "%dx%dx%d" % s)
def test_oracle_etdrk2_matches_reference_gpu(po, shape, case):
    """ETDRK2 (exponential midpoint with the finite-difference pressure gradient) against the
    reference's kernels, one state per gradient layout (x-y, 3-D, x-z, 1-D), weak and stiff drag."""
    z = np.load(os.path.join(GOLDEN, "drag_etdrk2.npz"))
    meta = json.loads(str(z["meta"]))
    key = "%dx%dx%d" % shape
    n = shape[0] * shape[1] * shape[2]
    g, d = np.array(z["gas_" + key]), np.array(z["dust_" + key])
    td = meta["td_stiff"] if case else meta["td"]
    po.drag_2fluid(g, d, shape, meta["tg"], td, meta["dt"], 3, h=[1.0 / s for s in shape])
    for tag in ("strict", "fast"):
        for mine, ref in ((g, z["gas_out_%s%s_%s" % (case, key, tag)]), (d, z["dust_out_%s%s_%s" % (case, key, tag)])):
            assert not np.any(np.isnan(ref[:, :n]))
            err = rel_l1(mine[:, :n], ref[:, :n], n)
            assert np.all(err <= 1e-12), (tag, err)
