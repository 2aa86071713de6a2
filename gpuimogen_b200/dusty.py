"""Two-fluid gas-dust run in 2-D: the library's fluid step for both fluids, Strang-composed with the
drag source (exact LogTrap2 or the learned surrogate), as the reference's main loop composes them
(imogen.m:115-139 / flux_multi.cu:174-272: drag(dt/2), fluid forward, drag(dt), fluid backward,
drag(dt/2)).

Workload: n x n periodic unit box.  Gas: gamma 5/3, rho = 1, P = 1, velocity = 1e-3 sin(2 pi x) in
y plus seeded uniform 1e-3 perturbations.  Dust: pressureless in the reference's sense (an
isothermal fluid with c_s = 0.1, fluidDetailModel.m), at rest, rho_dust / rho_gas log-uniform in
[0.01, 1] per cell, E = p^2/2rho + 1e-4 rho.  HLLC with the MC limiter for both fluids, CFL 0.4.

    python -m gpuimogen_b200.dusty [--n 2048] [--steps 500]
prints one JSON line: both runs' time per iteration (CUDA events), the drag calls alone, the
learned run's error against the exact run (relative L1 per field) and its fallback count.
"""
import json
import math

import numpy as np
import torch

from . import imogen as ib
from . import learned_drag as ld
from .timestep import TimeManager, run_iteration

GAMMA_GAS = 5 / 3.0
C_DUST = 0.1


def initial_state(n, seed=5):
    rng = np.random.Generator(np.random.Philox(seed))
    shape = (n, n, 1)
    x = (np.arange(n) + 0.5) / n
    X = np.broadcast_to(x[None, :], (n, n))
    vx = rng.uniform(-1e-3, 1e-3, (n, n))
    vy = 1e-3 * np.sin(2 * np.pi * X) + rng.uniform(-1e-3, 1e-3, (n, n))
    rho = np.ones((n, n))
    P = np.ones((n, n))
    S = ib.slab_pitch(n, n, 1)
    gas = np.zeros((5, S))
    N = n * n
    gas[0, :N] = rho.ravel()
    gas[2, :N] = (rho * vx).ravel()
    gas[3, :N] = (rho * vy).ravel()
    gas[1, :N] = (P / (GAMMA_GAS - 1) + 0.5 * rho * (vx ** 2 + vy ** 2)).ravel()
    rd = rho.ravel() * np.exp(rng.uniform(math.log(0.01), 0.0, N))
    dust = np.zeros((5, S))
    dust[0, :N] = rd
    dust[1, :N] = 1e-4 * rd
    return shape, gas, dust


class DustyRun:
    def __init__(self, n=2048, seed=5, model=None, tg=ld.THERMO_GAS, td=ld.THERMO_DUST):
        self.shape, g, d = initial_state(n, seed)
        self.g0 = torch.from_numpy(g).cuda()
        self.d0 = torch.from_numpy(d).cuda()
        self.gas = ib.Fluid(self.shape, bc="circular", q=self.g0.clone(), gamma=GAMMA_GAS)
        self.dust = ib.Fluid(self.shape, bc="circular", q=self.d0.clone(), gamma=2.0, c_isothermal=C_DUST)
        self.geo = ib.Geometry(self.shape)
        self.num = ib.numerics(slope="mc")
        self.model = model
        self.tg, self.td = tg, td
        self.fallbacks = torch.zeros(1, dtype=torch.int64, device="cuda")

    def reset(self):
        self.gas.q.copy_(self.g0)
        self.dust.q.copy_(self.d0)
        self.fallbacks.zero_()

    def drag(self, fluids, dt):
        gas, dust = fluids
        if self.model is None:
            ib.cudaSource2FluidDrag(gas, dust, self.tg, self.td, self.geo, [dt, ib.DRAG["logtrap2"]])
        else:
            ld.drag_step(gas, dust, self.model, dt, self.tg, self.td, fallback_counter=self.fallbacks)

    def run(self, steps):
        tm = TimeManager(cfl=0.4)
        for _ in range(steps):
            run_iteration([self.gas, self.dust], self.geo, tm, 2, self.num, source=self.drag)
        return tm


def time_run(run, steps, warm=2):
    run.reset()
    run.run(warm)
    run.reset()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    tm = run.run(steps)
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b), tm


def time_drag(run, reps=10):
    """Mean time of one drag call on the initial state (each call on a fresh copy of it; only the
    calls are inside the CUDA-event intervals)."""
    dt = 4e-5
    fl = [run.gas, run.dust]
    total = 0.0
    for r in range(reps + 1):
        run.reset()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        run.drag(fl, dt)
        b.record()
        torch.cuda.synchronize()
        if r:
            total += a.elapsed_time(b)
    run.reset()
    return total / reps


def study(n=2048, steps=500, samples=10_000_000, epochs=10, seed=5, verbose=False):
    model, hist = ld.train(n_samples=samples, epochs=epochs, seed=2024, verbose=verbose)
    ev = ld.evaluate(model, n=2_000_000)
    exact = DustyRun(n, seed)
    learned = DustyRun(n, seed, model=model)
    cells = n * n
    out = {"study": "dusty_2d", "grid": [n, n], "steps": steps, "training": hist, "evaluation": ev}
    for name, r in (("exact", exact), ("learned", learned)):
        ms, tm = time_run(r, steps)
        out[name] = {"ms": ms, "ms_per_iteration": ms / steps, "mcell_updates_per_s": cells * steps / (ms / 1e3) / 1e6,
                     "time": tm.time, "drag_call_ms": time_drag(r)}
    # learned vs exact after the same number of steps (states from time_run, drag timing restored)
    exact.reset(); learned.reset()
    exact.run(steps); learned.run(steps)
    torch.cuda.synchronize()
    N = cells
    def rel(a, b):
        return [float((a[k, :N] - b[k, :N]).abs().sum() / max(float(b[k, :N].abs().sum()), 1e-300)) for k in range(5)]
    out["learned_vs_exact_rel_l1"] = {"gas": rel(learned.gas.q, exact.gas.q), "dust": rel(learned.dust.q, exact.dust.q)}
    out["learned_fallback_cells"] = int(learned.fallbacks.item())
    out["speedup_learned_step"] = out["exact"]["ms"] / out["learned"]["ms"]
    out["speedup_drag_call"] = out["exact"]["drag_call_ms"] / out["learned"]["drag_call_ms"]
    return out


def main(argv=None):
    import argparse
    import sys
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--samples", type=int, default=10_000_000)
    ap.add_argument("--epochs", type=int, default=10)
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args(argv)
    ib.load("product")
    print(json.dumps(study(a.n, a.steps, a.samples, a.epochs, verbose=a.verbose)), flush=True)
    return 0


if __name__ == "__main__":
    import sys
    sys.exit(main())
