"""The main loop with its timestep on the device, replayed from CUDA graphs (GraphLoop).

Each iteration is the CFL reduction into a device time state, ib_timeUpdate, the complete
timestep reading dt from device memory and ib_timeAdvance; six graphs (one per iteration index
modulo 6) are replayed with no host read between iterations.  The kernels compute lambda = dt / h
from the device dt as the host path computes it, so the loop must reproduce run_iteration (the
host loop of imogen.m:115-139 with TimeManager.m's bookkeeping) bit for bit: the state, the
simulated time and the iteration count, for a 3-D problem, for Sod run to t = 0.2 (where the
last-step clip and the loop's end matter) and for gas + dust with the drag source.  Replays past
the end time must change nothing.
"""
import numpy as np
import pytest

import gpuimogen_b200 as ib
from gpuimogen_b200 import dusty, problems
from helpers import bits_equal, first_diff, host, to_fluid

pytestmark = pytest.mark.gpu


def test_graph_loop_kh_matches_host_loop(cuda):
    shape = (32, 24, 20)
    n = shape[0] * shape[1] * shape[2]
    q0 = problems.kelvin_helmholtz(shape, seed=4)
    geo = ib.Geometry(shape)
    num = ib.numerics(slope="mc")
    a = to_fluid(q0.copy(), shape, gamma=5 / 3.0)
    tm = ib.TimeManager(cfl=0.4)
    for _ in range(14):
        ib.run_iteration([a], geo, tm, 2, num)
    b = to_fluid(q0.copy(), shape, gamma=5 / 3.0)
    loop = ib.GraphLoop([b], geo, 2, num, cfl=0.4)     # six eager iterations
    loop.run(8)                                         # eight replays
    s = loop.state()
    qa, qb = host(a), host(b)
    assert s.iteration == tm.iteration == 14
    assert s.time == tm.time
    assert bits_equal(qa, qb, n), first_diff(qa, qb, n)


@pytest.mark.parametrize("method", [3, 2])
def test_graph_loop_sod_to_tmax_matches_host_loop(cuda, method):
    n = 1024
    shape = (n, 1, 1)
    q0 = problems.sod(n)
    geo = ib.Geometry(shape)
    a = to_fluid(q0.copy(), shape, bc="const", gamma=1.4)
    tm = ib.TimeManager(cfl=0.4, tmax=0.2)
    while tm.running:
        ib.run_iteration([a], geo, tm, method)
    b = to_fluid(q0.copy(), shape, bc="const", gamma=1.4)
    loop = ib.GraphLoop([b], geo, method, cfl=0.4, tmax=0.2).run(check_every=32)
    s = loop.state()
    assert s.iteration == tm.iteration, (s.iteration, tm.iteration)
    assert s.time == tm.time and abs(s.time - 0.2) < 1e-14
    qa, qb = host(a), host(b)
    assert bits_equal(qa, qb, n), first_diff(qa, qb, n)
    # replays past the end change nothing
    loop.run(6)
    assert bits_equal(host(b), qb, n)
    assert loop.state().iteration == s.iteration and loop.state().time == s.time


def test_graph_loop_two_fluid_drag_matches_host_loop(cuda):
    nn = 64
    shape, gas, dust = dusty.initial_state(nn, seed=9)
    N = nn * nn
    drag = (dusty.ld.THERMO_GAS, dusty.ld.THERMO_DUST, "logtrap2")
    geo = ib.Geometry(shape)
    num = ib.numerics(slope="mc")
    mk = lambda: (to_fluid(gas.copy(), shape, gamma=5 / 3.0),
                  to_fluid(dust.copy(), shape, gamma=2.0, c_iso=dusty.C_DUST))
    ga, da = mk()
    tm = ib.TimeManager(cfl=0.4)
    for _ in range(10):
        ib.run_iteration([ga, da], geo, tm, 2, num, drag=drag)
    gb, db = mk()
    loop = ib.GraphLoop([gb, db], geo, 2, num, drag=drag, cfl=0.4)
    loop.run(4)
    assert loop.state().iteration == 10 and loop.state().time == tm.time
    for x, y in ((ga, gb), (da, db)):
        qx, qy = host(x), host(y)
        assert bits_equal(qx, qy, N), first_diff(qx, qy, N)
    assert not np.array_equal(host(db)[2, :N], dust[2, :N])  # the drag acted
