"""Cylindrical geometry (x = r, y = theta, z = z) in the CPU oracle.

Pinned against the reference's own kernels: tests/golden/cylindrical.npz holds the outputs of
the reference's gpuclass sources (built for sm_100a by oracle/ref_harness, run on a GPU by
tests/golden/make_golden.py --cyl-only) for single radial and theta sweeps of HLLC, HLL
(adiabatic and isothermal) and Xin-Jin in both theta memory layouts, the geometric source terms
(including the pressure reset of a cold gas), the cylindrical CFL timesteps of 1-, 2- and 3-D
grids, and whole main loops with the cylinder source between and around the fluid steps.  The
reference built with -fmad=false must agree with the oracle bit for bit.

Properties that hold whatever the reference: a gas at rest at uniform pressure stays at rest
through a radial sweep to rounding (the geometric pressure term balances the difference of the
face areas), and a theta sweep of a theta-independent state changes nothing.
"""
import json
import os

import numpy as np
import pytest

from gpuimogen_b200 import problems
from helpers import bits_equal, first_diff, oracle_cyl_loop

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cylindrical.npz")


def _gold():
    if not os.path.exists(GOLD):
        pytest.skip("cylindrical golden vectors not generated")
    z = np.load(GOLD)
    return z, json.loads(str(z["meta"]))


def _n(shape):
    return shape[0] * shape[1] * shape[2]


def test_cyl_sweeps_match_reference(po):
    z, meta = _gold()
    h = meta["h"]
    for case in meta["sweeps"]:
        shape = tuple(case["shape"])
        for d, form in ((1, 0), (2, 0), (2, 1)):
            q = z["in_" + case["name"]].copy()
            gamma = 2.0 if case["c_iso"] != -1 else 1.4
            sp = po.step_params(meta["dt"], h, gamma, c_iso=case["c_iso"], method=case["method"], cylindrical=True,
                                r_inner=meta["r_inner"], theta_form=form)
            po.fluid_sweep(q, shape, sp, d)
            ref = z["out_%s_d%d_f%d_strict" % (case["name"], d, form)]
            assert bits_equal(q, ref, _n(shape)), (case["name"], d, form, first_diff(q, ref, _n(shape)))


def test_cyl_source_and_cfl_match_reference(po):
    z, meta = _gold()
    h = meta["h"]
    shape = (24, 20, 6)
    for key in ("src", "src_cold"):
        q = z[key + "_in"].copy()
        po.cyl_source(q, shape, 0.05, h[0], meta["r_inner"])
        ref = z[key + "_out_strict"]
        assert bits_equal(q, ref, _n(shape)), (key, first_diff(q, ref, _n(shape)))
    # the cold copy hits the pressure reset somewhere, and the reset changed E there
    assert not np.array_equal(z["src_cold_out_strict"][1], z["src_cold_in"][1])
    for shape in ((24, 20, 6), (24, 20, 1), (24, 1, 1)):
        qs = z["cfl_in_%dx%dx%d" % shape]
        for method in (1, 2, 3):
            t = po.cfl_timestep(qs, shape, 1.4, h, method, cylindrical=True, r_inner=meta["r_inner"])
            assert t == float(z["cfl_%dx%dx%d_m%d_strict" % (shape + (method,))]), (shape, method)


def test_cyl_main_loops_match_reference(po):
    z, meta = _gold()
    for case in meta["runs"]:
        shape = tuple(case["shape"])
        q = z["run_in_" + case["name"]].copy()
        dts = oracle_cyl_loop(po, q, shape, meta["h"], meta["r_inner"], case["method"], case["gamma"], case["c_iso"],
                              case["bc"], case["cfl"], case["niter"])
        assert np.array_equal(dts, z["run_dts_%s_strict" % case["name"]]), case["name"]
        ref = z["run_out_%s_strict" % case["name"]]
        assert bits_equal(q, ref, _n(shape)), (case["name"], first_diff(q, ref, _n(shape)))


@pytest.mark.parametrize("method", [1, 2, 3])
def test_radial_sweep_keeps_gas_at_rest(po, method):
    shape = (32, 6, 4)
    n = _n(shape)
    q = problems.pack(shape, 1.0, 1.0 / 0.4, 0.0, 0.0, 0.0)
    h = [0.05, 0.04, 0.1]
    sp = po.step_params(0.01, h, 1.4, method=method, cylindrical=True, r_inner=0.3)
    po.fluid_sweep(q, shape, sp, 1)
    assert np.max(np.abs(q[2, :n])) < 1e-13, np.max(np.abs(q[2, :n]))
    assert np.max(np.abs(q[0, :n] - 1.0)) < 1e-13


@pytest.mark.parametrize("method", [1, 2, 3])
@pytest.mark.parametrize("form", [0, 1])
def test_theta_sweep_of_axisymmetric_state_is_identity(po, method, form):
    shape = (16, 12, 3)
    q0 = problems.rotating_annulus((16, 1, 3), r_inner=1.0, dr=0.05, seed=5)
    n1 = 16 * 3
    q = np.zeros((5, problems.slab_pitch(*shape)))
    for k in range(5):   # the same value along theta
        q[k, :_n(shape)] = np.repeat(q0[k, :n1].reshape(3, 1, 16), 12, axis=1).ravel()
    ref = q.copy()
    sp = po.step_params(0.002, [0.05, 0.04, 0.1], 1.4, method=method, cylindrical=True, r_inner=1.0,
                        theta_form=form)
    po.fluid_sweep(q, shape, sp, 2)
    assert bits_equal(q, ref, _n(shape)), first_diff(q, ref, _n(shape))


def test_theta_forms_follow_the_sweep_index(po):
    # sweep index (iteration + 3 [forward]) mod 6 = 0 or 5 puts r third in memory (theta,z,r)
    forms = [[po.theta_form(d, it) for it in range(6)] for d in (1, -1)]
    assert forms[0] == [0, 0, 1, 1, 0, 0]   # forward: sweep indices 3, 4, 5, 0, 1, 2
    assert forms[1] == [1, 0, 0, 0, 0, 1]   # backward: 0, 1, 2, 3, 4, 5
