"""Batched ensemble of independent 1-D Riemann problems (ib_riemannEnsemble) against the oracle.

Each problem of the ensemble must come out exactly as if it had been run alone: the oracle runs
it with the reference's main loop (CFL tau, dt = CFL tau clipped at t_end, forward and backward
1-D fluid step with the boundary fill, Kahan t += 2 dt).  Strict build: bit for bit, same dt
sequence (same final time and iteration count).  Product build: 1e-12 relative L1."""
import numpy as np
import pytest
import torch

import gpuimogen_b200 as ib
from gpuimogen_b200 import ensemble as en
from helpers import bits_equal, first_diff, product_close

pytestmark = pytest.mark.gpu

SIZES = [9, 13, 40, 120, 255, 256, 300, 600, 1000, 2049, 4096]


def oracle_problem(po, q, h, gamma, cfl, t_end, itermax, method, slope, bc):
    n = q.shape[1]
    shape = (n, 1, 1)
    hh = [h, 1.0, 1.0]
    sp = po.step_params(0.0, hh, gamma, rho_min=1e-5, method=method, slope=slope)
    bcs = [bc, bc, "circular", "circular", "circular", "circular"]
    tm = ib.TimeManager(cfl=cfl, tmax=t_end, itermax=itermax)
    while tm.running:
        tau = po.cfl_timestep(q, shape, gamma, hh, method)
        sp.dt = tm.update(tau)
        po.fluid_step_3d(q, shape, sp, bcs, 1, tm.iteration)
        po.fluid_step_3d(q, shape, sp, bcs, -1, tm.iteration)
        tm.step()
    return tm


def make(sizes, seed, bc="outflow"):
    _, states = en.riemann_states(len(sizes), seed)
    q, off, h = en.pack_problems(np.array(sizes), states, 1.4)
    return q, off, h, en.RiemannEnsemble(q, off, h, gamma=1.4, bc=(bc, bc))


@pytest.mark.parametrize("method,bc", [(2, "outflow"), (2, "const"), (1, "outflow"), (2, "mirror")])
def test_ensemble_matches_oracle_per_problem(cuda, ib, po, method, bc):
    q, off, h, ens = make(SIZES, seed=11 + method, bc=bc)
    t_end, itermax = 0.04, 12
    ref = []
    for p in range(len(SIZES)):
        qp = np.ascontiguousarray(q[:, off[p]:off[p + 1]])
        tm = oracle_problem(po, qp, h[p], 1.4, 0.4, t_end, itermax, method, "mc", bc)
        ref.append((qp, tm))
    ib.use_variant("strict")
    try:
        ens.run(t_end=t_end, method=method, slope="mc", itermax=itermax)
        torch.cuda.synchronize()
    finally:
        ib.use_variant("product")
    t_out, iters = ens.t_out.cpu().numpy(), ens.iters.cpu().numpy()
    for p, (qp, tm) in enumerate(ref):
        got = ens.host_problem(p)
        assert iters[p] == tm.iteration, (p, iters[p], tm.iteration)
        assert t_out[p] == tm.time, (p, t_out[p], tm.time)
        assert bits_equal(got, qp, qp.shape[1]), (p, first_diff(got, qp, qp.shape[1]))
    # product build: same problems, FMA-contracted arithmetic
    ens.reset()
    ens.run(t_end=t_end, method=method, slope="mc", itermax=itermax)
    torch.cuda.synchronize()
    for p, (qp, tm) in enumerate(ref):
        ok, info = product_close(ens.host_problem(p), qp, qp.shape[1], l1=1e-12, scale=1e-10)
        assert ok, (p, info)


def test_ensemble_launch_shapes_and_graph_agree(cuda, ib):
    """Results do not depend on the launch shape, and a captured graph replays the same launch."""
    _, _, _, ens = make([256, 4096, 700, 1500, 333, 2048, 260, 999] * 5, seed=3)
    kw = dict(t_end=0.02, slope="mc", itermax=0)
    outs = []
    for tune in en.CANDIDATES:
        ens.reset()
        ens.run(tuning=tune, **kw)
        torch.cuda.synchronize()
        outs.append((ens.q.clone(), ens.iters.clone(), ens.t_out.clone()))
    for q, it, t in outs[1:]:
        assert torch.equal(q, outs[0][0]) and torch.equal(it, outs[0][1]) and torch.equal(t, outs[0][2])
    g = ens.capture(tuning=en.CANDIDATES[2], **kw)
    ens.q.zero_()
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(ens.q, outs[0][0])
    assert torch.all(torch.abs(ens.t_out - 0.02) <= 1e-15)


def test_ensemble_fp32_flux_close_to_fp64(cuda, ib):
    _, _, _, ens = make(list(range(256, 4097, 64)), seed=5)
    kw = dict(t_end=0.02, slope="mc")
    ens.run(precision="fp64", **kw)
    torch.cuda.synchronize()
    q64 = ens.q.clone()
    ens.reset()
    ens.run(precision="fp32flux", **kw)
    torch.cuda.synchronize()
    n = ens.cells
    err = float(((ens.q[0, :n] - q64[0, :n]).abs().sum() / q64[0, :n].abs().sum()).item())
    assert 0 < err <= 1e-5, err


def test_ensemble_autotune_and_invalid_inputs(cuda, ib):
    _, _, _, ens = make([9, 8, 256], seed=9)
    ens.run(t_end=0.01)
    torch.cuda.synchronize()
    it = ens.iters.cpu().numpy()
    assert it[1] == -1 and it[0] > 0 and it[2] > 0  # 8 cells: too short for the 4-cell boundary fill
    with pytest.raises(ib.ImogenError):
        ens.run(t_end=0.01, tuning={"threads": 100})
    with pytest.raises(ib.ImogenError):
        ens.run(t_end=0.01, method=3)
    _, _, _, big = make([256, 512, 4096, 1024] * 40, seed=2)
    tune = en.autotune(big, t_end=0.1, iters=4)
    assert tune in en.CANDIDATES
