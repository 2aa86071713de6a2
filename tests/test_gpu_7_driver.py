"""The standalone C++ driver against the Python main loop: same library, same initial state, so
the final states, the simulated time and the iteration count must agree bit for bit (the driver
restates TimeManager.m's bookkeeping and imogen.m's Strang composition in C++)."""
import json
import math
import subprocess

import numpy as np
import pytest
import torch

import gpuimogen_b200 as ibm
from gpuimogen_b200 import build as bld
from gpuimogen_b200 import dusty, problems
from helpers import bits_equal, first_diff, host, to_fluid

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def exe():
    return bld.build_driver()


def drive(exe, *args):
    r = subprocess.run([exe, *args], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_driver_kh_matches_python_loop(cuda, ib, exe, tmp_path):
    shape = (24, 20, 16)
    n = shape[0] * shape[1] * shape[2]
    q = problems.kelvin_helmholtz(shape, seed=9)
    q.tofile(tmp_path / "in.bin")
    out = drive(exe, "--problem", "kh", "--grid", "24,20,16", "--input", str(tmp_path / "in.bin"), "--steps", "4",
                "--output", str(tmp_path / "out.bin"))
    fl = to_fluid(q, shape, gamma=5 / 3.0)
    tm = ib.TimeManager(cfl=0.4)
    for _ in range(4):
        ib.run_iteration([fl], ib.Geometry(shape), tm, 2, ib.numerics(slope="mc"))
    ref = host(fl)
    got = np.fromfile(tmp_path / "out.bin").reshape(5, -1)
    assert out["iterations"] == 4 and out["time"] == tm.time
    assert bits_equal(got, ref, n), first_diff(got, ref, n)


def test_driver_sod_to_tmax_matches_python_loop(cuda, ib, exe, tmp_path):
    shape = (256, 1, 1)
    q = problems.sod(256, 1.4)
    q.tofile(tmp_path / "sod.bin")
    out = drive(exe, "--problem", "sod", "--grid", "256,1,1", "--method", "hll", "--limiter", "ospre",
                "--tmax", "0.2", "--input", str(tmp_path / "sod.bin"), "--output", str(tmp_path / "sod_out.bin"))
    fl = to_fluid(q, shape, bc="const", gamma=1.4)
    tm = ib.TimeManager(cfl=0.4, tmax=0.2)
    while tm.running:
        ib.run_iteration([fl], ib.Geometry(shape), tm, 1, ib.numerics(slope="ospre"))
    got = np.fromfile(tmp_path / "sod_out.bin").reshape(5, -1)
    assert out["iterations"] == tm.iteration and out["time"] == tm.time
    assert math.isclose(tm.time, 0.2, rel_tol=1e-13)
    assert bits_equal(got, host(fl), 256), first_diff(got, host(fl), 256)


def test_driver_gas_dust_matches_python_loop(cuda, ib, exe, tmp_path):
    n = 64
    shape, g, d = dusty.initial_state(n, seed=5)
    g.tofile(tmp_path / "g.bin")
    d.tofile(tmp_path / "d.bin")
    out = drive(exe, "--problem", "dusty", "--grid", "64,64,1", "--input", str(tmp_path / "g.bin"),
                "--dust-input", str(tmp_path / "d.bin"), "--steps", "3", "--output", str(tmp_path / "g_out.bin"),
                "--dust-output", str(tmp_path / "d_out.bin"))
    run = dusty.DustyRun(n, seed=5)
    tm = run.run(3)
    N = n * n
    G, D = run.gas.q.cpu().numpy(), run.dust.q.cpu().numpy()
    got_g = np.fromfile(tmp_path / "g_out.bin").reshape(5, -1)
    got_d = np.fromfile(tmp_path / "d_out.bin").reshape(5, -1)
    assert out["iterations"] == 3 and out["time"] == tm.time
    assert bits_equal(got_g, G, N), first_diff(got_g, G, N)
    assert bits_equal(got_d, D, N), first_diff(got_d, D, N)
