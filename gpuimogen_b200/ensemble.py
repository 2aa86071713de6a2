"""Batched ensembles of independent 1-D Riemann problems on one GPU.

Every problem is a 1-D fluid on [0, 1] with its own cell count, its own CFL timestep and its own
clock; the library's ib_riemannEnsemble runs all of them to their end time in one persistent
kernel launch (CTAs take problems from a device work counter, longest first).  This module
builds the packed device layout, generates the seeded Riemann-problem workload, picks the
launch shape with a small autotuner, and captures the launch in a CUDA graph for repeated runs.

    ens = RiemannEnsemble.random(4096, seed=1)            # N_i ~ U{256..4096}, outflow ends
    tune = autotune(ens, t_end=0.1)                        # timed trial runs, best launch shape
    ens.run(t_end=0.1, tuning=tune)                        # or: g = ens.capture(...); g.replay()
"""
import ctypes
import json
import math
import os

import numpy as np
import torch

from . import imogen as ib


def riemann_states(nprob, seed, nmin=256, nmax=4096, gamma=1.4):
    """Seeded workload: N ~ U{nmin..nmax}; left/right rho and P log-uniform in [0.1, 10], u uniform
    in [-2, 2]; the discontinuity at mid-domain.  Returns (sizes, states[nprob, 2, 3]) with the
    (rho, u, P) of the left and right side."""
    rng = np.random.Generator(np.random.Philox(seed))
    sizes = rng.integers(nmin, nmax, size=nprob, endpoint=True)
    rho = np.exp(rng.uniform(math.log(0.1), math.log(10.0), size=(nprob, 2)))
    P = np.exp(rng.uniform(math.log(0.1), math.log(10.0), size=(nprob, 2)))
    u = rng.uniform(-2.0, 2.0, size=(nprob, 2))
    return sizes.astype(np.int64), np.stack([rho, u, P], axis=2)


def pack_problems(sizes, states, gamma=1.4):
    """Host arrays: q (5, pitch) with problem p in cells offsets[p]..offsets[p+1]-1, offsets, h."""
    sizes = np.asarray(sizes, dtype=np.int64)
    offsets = np.zeros(len(sizes) + 1, dtype=np.int64)
    offsets[1:] = np.cumsum(sizes)
    total = int(offsets[-1])
    pitch = ((total + 31) // 32) * 32
    q = np.zeros((5, pitch))
    for p, n in enumerate(sizes):
        n = int(n)
        x = (np.arange(n) + 0.5) / n
        left = x < 0.5
        (rl, ul, pl), (rr, ur, pr) = states[p]
        rho = np.where(left, rl, rr)
        u = np.where(left, ul, ur)
        P = np.where(left, pl, pr)
        o = int(offsets[p])
        q[0, o:o + n] = rho
        q[1, o:o + n] = P / (gamma - 1) + 0.5 * rho * u * u
        q[2, o:o + n] = rho * u
    h = 1.0 / sizes.astype(np.float64)
    return q, offsets, h


class RiemannEnsemble:
    """Device-resident ensemble: q (5, pitch) float64, offsets, h, processing order, outputs."""

    def __init__(self, q, offsets, h, gamma=1.4, rho_min=1e-5, bc=("outflow", "outflow"), device=None,
                 longest_first=True):
        dev = device or torch.device("cuda", torch.cuda.current_device())
        self.q0 = torch.as_tensor(np.ascontiguousarray(q), dtype=torch.float64).to(dev)  # pristine copy
        self.q = self.q0.clone()
        self.offsets = torch.as_tensor(np.asarray(offsets, dtype=np.int64)).to(dev)
        self.h = torch.as_tensor(np.asarray(h, dtype=np.float64)).to(dev)
        sizes = np.diff(np.asarray(offsets, dtype=np.int64))
        self.sizes = sizes
        order = np.argsort(-sizes, kind="stable") if longest_first else np.arange(len(sizes))
        self.order = torch.as_tensor(order.astype(np.int32)).to(dev)
        self.nproblems = len(sizes)
        self.t_out = torch.zeros(self.nproblems, dtype=torch.float64, device=dev)
        self.iters = torch.zeros(self.nproblems, dtype=torch.int32, device=dev)
        self.gamma = gamma
        self.rho_min = rho_min
        self.bc = tuple(ib.BC[b] if isinstance(b, str) else int(b) for b in bc)
        self.cells = int(sizes.sum())

    @classmethod
    def random(cls, nprob, seed=1, nmin=256, nmax=4096, gamma=1.4, **kw):
        sizes, states = riemann_states(nprob, seed, nmin, nmax, gamma)
        q, offsets, h = pack_problems(sizes, states, gamma)
        return cls(q, offsets, h, gamma=gamma, **kw)

    def reset(self):
        """Back to the initial state (device-to-device copy, stream-ordered, capturable)."""
        self.q.copy_(self.q0)

    def _struct(self):
        e = ib.IbEnsemble()
        e.q = self.q.data_ptr()
        e.slab_pitch = self.q.shape[1]
        e.offsets = self.offsets.data_ptr()
        e.h = self.h.data_ptr()
        e.order = self.order.data_ptr()
        e.t_out = self.t_out.data_ptr()
        e.iters_out = self.iters.data_ptr()
        e.nproblems = self.nproblems
        e.bc[0], e.bc[1] = self.bc
        return e

    def run(self, t_end=0.1, cfl=0.4, method=2, slope="mc", precision="fp64", tuning=None, itermax=0):
        """One launch: every problem to t_end (stream-ordered, does not synchronise)."""
        e = self._struct()
        th = ib.IbFluidThermo(self.gamma, self.rho_min, -1.0)
        num = ib.numerics(slope=slope, precision=precision)
        tu = None
        if tuning is not None:
            tu = ib.IbEnsembleTuning(int(tuning.get("threads", 0)), int(tuning.get("chunk", 0)),
                                     int(tuning.get("ctas_per_sm", 0)), 0)
        rc = ib._lib().ib_riemannEnsemble(ctypes.byref(e), ctypes.byref(th), int(method), float(cfl), float(t_end),
                                          int(itermax), ctypes.byref(num),
                                          ctypes.byref(tu) if tu is not None else None, ib._stream())
        ib._check("ib_riemannEnsemble", rc)

    def host_problem(self, p):
        """(5, N_p) numpy copy of problem p."""
        o0, o1 = int(self.offsets[p]), int(self.offsets[p + 1])
        return self.q[:, o0:o1].cpu().numpy()

    def cell_updates(self):
        """Cell-iterations of the last run (sum over problems of cells x iterations)."""
        return int((self.iters.to(torch.int64).cpu() * torch.as_tensor(self.sizes)).sum())

    def capture(self, **runkw):
        """CUDA graph of (reset to the initial state, one ensemble launch).  A first launch runs
        outside the capture so the library sets up its work counter and kernel attributes."""
        self.run(**runkw)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.reset()
            self.run(**runkw)
        torch.cuda.synchronize()
        return g


# ------------------------------------------------------------------------------------------------
# Autotuner: launch shapes are timed on a seeded sample of the ensemble with an iteration cap, and
# the fastest (cell-iterations per second) is kept per (device, method, precision, limiter).
# ------------------------------------------------------------------------------------------------
CANDIDATES = [
    {"threads": 128, "chunk": 120, "ctas_per_sm": 0},
    {"threads": 256, "chunk": 120, "ctas_per_sm": 0},
    {"threads": 256, "chunk": 248, "ctas_per_sm": 0},
    {"threads": 512, "chunk": 248, "ctas_per_sm": 0},
    {"threads": 512, "chunk": 504, "ctas_per_sm": 0},
    {"threads": 256, "chunk": 248, "ctas_per_sm": 2},
]
_TUNED = {}


def autotune(ens, t_end=0.1, cfl=0.4, method=2, slope="mc", precision="fp64", sample=None, iters=16,
             cache_file=None, candidates=None, verbose=False):
    """Returns the fastest launch shape for this ensemble's kind of workload.  The trial runs use
    a seeded sample of the ensemble's problems (default: 4 per SM) for `iters` iterations each."""
    dev = torch.cuda.current_device()
    key = "%s|m%d|%s|%s" % (torch.cuda.get_device_name(dev), method, precision, slope)
    if key in _TUNED:
        return dict(_TUNED[key])
    if cache_file and os.path.exists(cache_file):
        with open(cache_file) as f:
            saved = json.load(f)
        if key in saved:
            _TUNED[key] = saved[key]
            return dict(saved[key])
    nsm = torch.cuda.get_device_properties(dev).multi_processor_count
    k = min(ens.nproblems, sample or 4 * nsm)
    rng = np.random.Generator(np.random.Philox(7))
    pick = np.sort(rng.choice(ens.nproblems, size=k, replace=False))
    offs = ens.offsets.cpu().numpy()
    q_full = ens.q0.cpu().numpy()
    sizes = ens.sizes[pick]
    new_off = np.zeros(k + 1, dtype=np.int64)
    new_off[1:] = np.cumsum(sizes)
    pitch = ((int(new_off[-1]) + 31) // 32) * 32
    q = np.zeros((5, pitch))
    for j, p in enumerate(pick):
        q[:, new_off[j]:new_off[j + 1]] = q_full[:, offs[p]:offs[p + 1]]
    sub = RiemannEnsemble(q, new_off, 1.0 / sizes.astype(np.float64), gamma=ens.gamma, rho_min=ens.rho_min,
                          bc=ens.bc)
    results = []
    for cand in (candidates or CANDIDATES):
        runkw = dict(t_end=t_end, cfl=cfl, method=method, slope=slope, precision=precision, tuning=cand,
                     itermax=iters)
        try:
            sub.reset()
            sub.run(**runkw)  # warm-up (and validity of the shape)
            torch.cuda.synchronize()
        except ib.ImogenError:
            continue
        best = math.inf
        for _ in range(2):
            sub.reset()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            sub.run(**runkw)
            b.record()
            torch.cuda.synchronize()
            best = min(best, a.elapsed_time(b))
        rate = sub.cell_updates() / (best / 1e3) / 1e6
        results.append((rate, cand))
        if verbose:
            print("autotune", cand, "%.1f Mcell-updates/s" % rate, flush=True)
    if not results:
        raise RuntimeError("autotune: no launch shape ran")
    rate, cand = max(results, key=lambda r: r[0])
    _TUNED[key] = dict(cand)
    if cache_file:
        saved = {}
        if os.path.exists(cache_file):
            with open(cache_file) as f:
                saved = json.load(f)
        saved[key] = dict(cand)
        with open(cache_file, "w") as f:
            json.dump(saved, f, indent=1)
    return dict(cand)


def study(nprob=4096, seed=1, t_end=0.1, cfl=0.4, slope="mc", reps=2, verbose=False):
    """Config: 4096 HLLC Riemann problems, N ~ U{256..4096}, outflow ends, each to t_end.  Times
    the graph-captured launch in FP64 and in the FP32-flux form; reports cell-iterations per
    second and the FP32-flux density error against the FP64 run (relative L1 over all cells)."""
    ens = RiemannEnsemble.random(nprob, seed=seed)
    out = {"study": "riemann_ensemble", "problems": nprob, "cells": ens.cells, "t_end": t_end, "cfl": cfl,
           "method": "HLLC", "limiter": slope, "boundaries": "outflow"}
    final = {}
    for prec in ("fp64", "fp32flux"):
        tune = autotune(ens, t_end=t_end, cfl=cfl, slope=slope, precision=prec, verbose=verbose)
        g = ens.capture(t_end=t_end, cfl=cfl, slope=slope, precision=prec, tuning=tune)
        times = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            g.replay()
            b.record()
            torch.cuda.synchronize()
            times.append(a.elapsed_time(b))
        ms = min(times)
        upd = ens.cell_updates()
        it = ens.iters.cpu().numpy()
        tt = ens.t_out.cpu().numpy()
        final[prec] = ens.q[0, :ens.cells].clone()
        out[prec] = {"tuning": tune, "ms": ms, "cell_updates": upd,
                     "mcell_updates_per_s": upd / (ms / 1e3) / 1e6,
                     "iterations": {"min": int(it.min()), "max": int(it.max()), "mean": float(it.mean())},
                     "all_reached_t_end": bool(np.all(np.abs(tt - t_end) <= 1e-12 * t_end))}
        del g
    a, b = final["fp32flux"], final["fp64"]
    out["fp32flux_rel_l1_rho_vs_fp64"] = float(((a - b).abs().sum() / b.abs().sum()).item())
    out["speedup_fp32flux"] = out["fp32flux"]["mcell_updates_per_s"] / out["fp64"]["mcell_updates_per_s"]
    return out


def main(argv=None):
    import argparse
    import sys
    ap = argparse.ArgumentParser()
    ap.add_argument("--nprob", type=int, default=4096)
    ap.add_argument("--t-end", type=float, default=0.1)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args(argv)
    ib.load("product")
    print(json.dumps(study(a.nprob, a.seed, a.t_end, verbose=a.verbose)), flush=True)
    return 0


if __name__ == "__main__":
    import sys
    sys.exit(main())
