#!/usr/bin/env python
"""Benchmark of the Imogen fluid step on B200.

Workload (one GPU): the 3-D Kelvin-Helmholtz problem, plain HLLC FP64 drop-in, MC limiter:
256^3 periodic unit cube, gamma = 5/3, P = 2.5, rho = 2 / v_x = +0.5 in the |y-1/2| < 1/4 band
and rho = 1 / v_x = -0.5 elsewhere, seeded U(+-1e-2) velocity perturbations, CFL 0.4.
One step = one main-loop iteration of the reference (imogen.m:115-139): CFL reduction, forward
3-sweep fluid step, backward 3-sweep fluid step; the state advances by 2*dt.  The timed loop is
the library's device-side main loop (GraphLoop: the time state in device memory, each iteration a
replayed CUDA graph, with no host read between iterations); the end-to-end leg runs every step as
a separate job through run_iteration with host buffers.
Metric: Mcell-updates/s = cells x iterations / seconds / 1e6 (whole job over all ranks).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: each rank runs an independent replica of the workload (the single-GPU fluid step has
no inter-GPU exchange), scaling "weak"; the time is the maximum over ranks.
--impl reference times the reference's CPU path, which for this hot path is the oracle's C
restatement of the reference kernels (the reference itself has no CPU implementation), on all
host cores, on a bounded sample of the same workload.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SHAPE = (256, 256, 256)
GAMMA = 5.0 / 3.0
CFL = 0.4
METHOD = 2  # HLLC
METRIC = "Mcell-updates/s"
# device copies of the state in the end-to-end leg: a buffer holds a step's upload, compute and
# download in turn, so with three the upload of step i+1 never waits for step i-1's download
E2E_BUFFERS = int(os.environ.get("IMOGEN_BENCH_E2E_BUFFERS", "3"))
# DRAM bytes per cell of one sweep launch (dram__bytes_read.sum + dram__bytes_write.sum / cells),
# from the ncu capture of this workload's three sweep kernels summarised in
# profiles/sweep_kernels_kh256_fp64.md (KH 256^3, state larger than L2).
TRAFFIC_B_PER_CELL = {"x_row": (671.35 + 617.76) * 1e6 / 256 ** 3,
                      "y_pair": (671.32 + 623.59) * 1e6 / 256 ** 3,
                      "z_pair": (671.30 + 625.57) * 1e6 / 256 ** 3}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--shape", default=None, help="override grid, e.g. 128,128,128 (not the benchmark config)")
    ap.add_argument("--case", default="bench", choices=["bench"] + sorted(CASES),
                    help="bench (default): the benchmark line; the others are small cases for ncu "
                         "captures and per-kernel timings (one GPU, no JSON bench line)")
    ap.add_argument("--n", type=int, default=None, help="cases: cube edge (sweeps, all) or 2-D edge (drag)")
    ap.add_argument("--m", type=int, default=1024, help="case all: 2-D gas-dust edge")
    ap.add_argument("--method", type=int, default=2, help="cases: 1 HLL, 2 HLLC, 3 Xin-Jin")
    ap.add_argument("--slope", default="mc")
    ap.add_argument("--fluxlim", default="vanleer")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32flux"])
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--cyl", action="store_true", help="case time-sweeps: cylindrical geometry")
    ap.add_argument("--t-end", type=float, default=0.01, help="case ensemble: end time")
    return ap.parse_args()


# ------------------------------------------------------------------------------------------------
# Small cases for Nsight Compute captures and per-kernel timings (one GPU).  Each launches the
# kernels it names a few times on a state larger than the 126 MB L2 and prints one line.
# ------------------------------------------------------------------------------------------------
def _case_shape(args, default_n):
    if args.shape:
        return tuple(int(v) for v in args.shape.split(","))
    n = args.n or default_n
    return (n, n, n)


def case_sweeps(args):
    """One warm-up iteration of Kelvin-Helmholtz, then one launch of each sweep kernel (x, y, z;
    an axis of extent 1 launches nothing) and one CFL reduction: n^3 (default 192) or --shape."""
    import torch
    import gpuimogen_b200 as ib
    from gpuimogen_b200 import problems
    shape = _case_shape(args, 192)
    q = problems.kelvin_helmholtz(shape, seed=1)
    fl = ib.Fluid(shape, q=torch.from_numpy(q).cuda(), gamma=GAMMA)
    geo = ib.Geometry(shape)
    num = ib.numerics(slope=args.slope, fluxlim=args.fluxlim, precision=args.precision)
    tm = ib.TimeManager(cfl=CFL)
    ib.run_iteration([fl], geo, tm, args.method, num)
    for d in (1, 2, 3):
        ib.cudaFluidStep(fl, geo, [tm.dTime, 1, GAMMA, 1e-5, args.method, d], num)
    ib.cflTimestepFused(fl, GAMMA, geo, args.method)
    torch.cuda.synchronize()
    print("case sweeps done", shape, args.precision, "method", args.method)


def case_time_sweeps(args):
    """Per-direction sweep time (CUDA events, mean of --reps launches after one untimed launch)
    of cudaFluidStep on the Kelvin-Helmholtz state: n^3 (default 256) or --shape.  --cyl: the
    rotating annulus in cylindrical geometry instead (x = r, y = theta)."""
    import torch
    import gpuimogen_b200 as ib
    from gpuimogen_b200 import problems
    shape = _case_shape(args, 256)
    num = ib.numerics(slope=args.slope, fluxlim=args.fluxlim, precision=args.precision)
    if args.cyl:
        h = [1.0 / shape[0], 2 * math.pi / shape[1], 1.0 / shape[2]]
        q = problems.rotating_annulus(shape, r_inner=1.0, dr=h[0], gamma=GAMMA, seed=1)
        geo = ib.Geometry(shape, h=h, cylindrical=True, r_inner=1.0)
    else:
        q = problems.kelvin_helmholtz(shape, seed=1)
        geo = ib.Geometry(shape)
    fl = ib.Fluid(shape, q=torch.from_numpy(q).cuda(), gamma=GAMMA)
    out = []
    for d in (1, 2, 3):
        if shape[d - 1] < 3:
            out.append(None)
            continue
        params = [1e-5, 1, GAMMA, 1e-5, args.method, d]
        ib.cudaFluidStep(fl, geo, params, num)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(args.reps):
            ib.cudaFluidStep(fl, geo, params, num)
        b.record()
        torch.cuda.synchronize()
        out.append(round(a.elapsed_time(b) / args.reps, 4))
    print(json.dumps({"case": "time-sweeps", "shape": list(shape), "method": args.method, "slope": args.slope,
                      "fluxlim": args.fluxlim, "precision": args.precision, "cylindrical": bool(args.cyl),
                      "ms_x_y_z": out}))


def case_ensemble(args):
    """One launch of the 4096-problem Riemann ensemble (the batching form's problems, HLLC MC,
    FP64 or --precision) to --t-end (default 0.01, a tenth of the form's end time: a short launch
    for an ncu capture), after one untimed launch; prints its CUDA-event time and throughput."""
    import torch
    from gpuimogen_b200 import ensemble
    ens = ensemble.RiemannEnsemble.random(4096, seed=1)
    kw = dict(t_end=args.t_end, cfl=CFL, slope="mc", precision=args.precision,
              tuning={"threads": 256, "chunk": 248, "ctas_per_sm": 0})
    ens.run(**kw)
    ens.reset()
    torch.cuda.synchronize()
    ms = _events_ms(lambda: ens.run(**kw))
    print(json.dumps({"case": "ensemble", "problems": 4096, "t_end": args.t_end, "precision": args.precision,
                      "ms": ms, "mcell_updates_per_s": ens.cell_updates() / (ms / 1e3) / 1e6}))


def case_cfl(args):
    """CUDA-event time of the two device-result CFL entry points (ib_cflTimestepFused with its
    allocated scratch, ib_cflTimestepNoAlloc with the built-in array) on 512^2 and 256^3."""
    import ctypes
    import torch
    import gpuimogen_b200 as ib
    from gpuimogen_b200 import imogen, problems
    L = imogen.load("product")
    res = {}
    for shape in ((512, 512, 1), (256, 256, 256)):
        fl = ib.Fluid(shape, q=torch.from_numpy(problems.kelvin_helmholtz(shape, seed=1)).cuda(), gamma=GAMMA)
        geo = ib.Geometry(shape)
        tau = torch.zeros(2, dtype=torch.float64, device="cuda")
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        f, g = fl.c_struct(), geo.c_struct()
        times = {}
        for name in ("fused", "noalloc"):
            def call():
                if name == "fused":
                    return L.ib_cflTimestepFused(ctypes.byref(f), GAMMA, ctypes.byref(g), 2, None,
                                                 ctypes.c_void_p(tau.data_ptr()), st)
                return L.ib_cflTimestepNoAlloc(ctypes.byref(f), GAMMA, ctypes.byref(g), 2,
                                               ctypes.c_void_p(tau.data_ptr() + 8), st)
            assert call() == 0
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(args.reps):
                assert call() == 0
            b.record()
            torch.cuda.synchronize()
            times[name] = round(a.elapsed_time(b) / args.reps, 4)
        assert tau[0].item() == tau[1].item()
        res["x".join(str(v) for v in shape)] = times
    print(json.dumps({"case": "cfl", "ms": res}))


def case_drag(args):
    """The 2-D gas-dust state on n x n (default 1024): one exact LogTrap2 drag call
    (logtrap_kernel) and one learned call (mlp_tc_kernel<1>) after training a small model
    (200k exact labels, 2 epochs)."""
    import torch
    import gpuimogen_b200 as ib
    from gpuimogen_b200 import dusty
    from gpuimogen_b200 import learned_drag as ld
    n = args.n or 1024
    model, _ = ld.train(n_samples=200_000, epochs=2, seed=3, batch=8192)
    exact = dusty.DustyRun(n)
    learned = dusty.DustyRun(n, model=model)
    exact.drag([exact.gas, exact.dust], 4e-5)
    learned.drag([learned.gas, learned.dust], 4e-5)
    torch.cuda.synchronize()
    print("case drag done", n, "fallbacks", int(learned.fallbacks.item()))


def case_all(args):
    """Every kind of kernel of the library once: KH at n^3 (default 160^3, 164 MB of state) for
    the sweeps of every method and precision, CFL, freezeAndPtot and the outflow fill; the
    rotating annulus at the same size in cylindrical geometry (one complete HLLC iteration, the r
    and theta sweeps of HLL and Xin-Jin); KH on
    512 x 512 x 8 (z sweeps of 2 MB planes: the wide-block kernels) and 2048 x 2048 x 1 (the
    chunked pipeline and its halo copy); the 2-D gas-dust state at --m^2 for the drag kernels
    (ETDRK2 included) and the learned drag; a 592-problem Riemann ensemble (4 iterations); the
    MLP training kernels on a 65536-sample batch."""
    import torch
    import gpuimogen_b200 as ib
    from gpuimogen_b200 import dusty, ensemble, problems
    from gpuimogen_b200 import learned_drag as ld
    shape = _case_shape(args, 160)
    q = problems.kelvin_helmholtz(shape, seed=1)
    geo = ib.Geometry(shape)
    dt = 1e-5
    for method, prec in ((2, "fp64"), (2, "fp32flux"), (1, "fp64"), (3, "fp64")):
        fl = ib.Fluid(shape, q=torch.from_numpy(q).cuda(), gamma=GAMMA)
        num = ib.numerics(slope="mc", precision=prec)
        for d in (1, 2, 3):
            ib.cudaFluidStep(fl, geo, [dt, 1, GAMMA, 1e-5, method, d], num)
    # cylindrical geometry (x = r, y = theta) on the rotating annulus: one complete HLLC iteration
    # (cylindrical CFL, cylinder source, radial, theta and z sweeps), then the r and theta sweeps of
    # HLL and Xin-Jin
    hc = [1.0 / shape[0], 2 * math.pi / shape[1], 1.0 / shape[2]]
    qc = problems.rotating_annulus(shape, r_inner=1.0, dr=hc[0], gamma=GAMMA, seed=1)
    gc = ib.Geometry(shape, h=hc, cylindrical=True, r_inner=1.0)
    fcyl = ib.Fluid(shape, q=torch.from_numpy(qc).cuda(), gamma=GAMMA)
    ib.run_iteration([fcyl], gc, ib.TimeManager(cfl=CFL), 2)
    for method in (1, 3):
        fcyl = ib.Fluid(shape, q=torch.from_numpy(qc).cuda(), gamma=GAMMA)
        for d in (1, 2):
            ib.cudaFluidStep(fcyl, gc, [dt, 1, GAMMA, 1e-5, method, d], ib.numerics(slope="mc"))
    del fcyl
    shp = (512, 512, 8)
    qw = problems.kelvin_helmholtz(shp, seed=2)
    for prec in ("fp64", "fp32flux"):
        fw = ib.Fluid(shp, q=torch.from_numpy(qw).cuda(), gamma=GAMMA)
        ib.cudaFluidStep(fw, ib.Geometry(shp), [dt, 1, GAMMA, 1e-5, 2, 3], ib.numerics(slope="mc", precision=prec))
    del fw
    shp = (2048, 2048, 1)
    fc = ib.Fluid(shp, q=torch.from_numpy(problems.kelvin_helmholtz(shp, seed=3)).cuda(), gamma=GAMMA)
    for d in (1, 2):
        ib.cudaFluidStep(fc, ib.Geometry(shp), [dt, 1, GAMMA, 1e-5, 2, d], ib.numerics(slope="mc"))
    del fc
    fl = ib.Fluid(shape, q=torch.from_numpy(q).cuda(), gamma=GAMMA, bc="outflow")
    ib.cflTimestepFused(fl, GAMMA, geo, 2)
    ib.freezeAndPtot(fl, GAMMA, 1, 0.0)
    ib.setFluidBoundary(fl, 1)
    run = dusty.DustyRun(args.m)
    for method in ("logtrap2", "rk4", "etdrk1", "etdrk2"):
        run.reset()
        ib.cudaSource2FluidDrag(run.gas, run.dust, run.tg, run.td, run.geo, [4e-5, ib.DRAG[method]])
    model, _ = ld.train(n_samples=65536 * 4, epochs=1, seed=3, batch=65536)
    run.reset()
    ld.drag_step(run.gas, run.dust, model, 4e-5)
    ens = ensemble.RiemannEnsemble.random(592, seed=2)
    ens.run(t_end=0.1, itermax=4, tuning={"threads": 256, "chunk": 248})
    torch.cuda.synchronize()
    print("case all done")


def graph_loop_timing(n_sod=1024, n_dust=2048, dust_iters=40):
    """Per-iteration time of the host loop (run_iteration: the CFL time read to the host every
    iteration) and of the device-time loop replayed from CUDA graphs (GraphLoop), CUDA events:
    Sod 1024 cells, Xin-Jin, to t = 0.2 (launch- and latency-bound), and 2-D gas + dust with
    exact LogTrap2 drag on n_dust^2 for dust_iters iterations after the graphs' six warm-up
    iterations."""
    import torch
    import gpuimogen_b200 as ib
    from gpuimogen_b200 import dusty, problems
    out = {}
    shape = (n_sod, 1, 1)
    geo = ib.Geometry(shape)
    for name in ("host_loop", "graph_loop"):
        fl = ib.Fluid(shape, bc="const", q=torch.from_numpy(problems.sod(n_sod)).cuda(), gamma=1.4)
        if name == "host_loop":
            tm = ib.TimeManager(cfl=CFL, tmax=0.2)

            def go():
                while tm.running:
                    ib.run_iteration([fl], geo, tm, 3)
            ms = _events_ms(go)
            iters = tm.iteration
        else:
            loop = ib.GraphLoop([fl], geo, 3, cfl=CFL, tmax=0.2)   # 6 eager iterations, then capture
            it0 = loop.iteration
            ms = _events_ms(lambda: loop.run(check_every=64))
            iters = loop.iteration - it0
        out.setdefault("sod_1024_xj", {})[name] = {"us_per_iteration": 1e3 * ms / iters, "iterations": iters}
    drag = (dusty.ld.THERMO_GAS, dusty.ld.THERMO_DUST, "logtrap2")
    num = ib.numerics(slope="mc")
    for name in ("host_loop", "graph_loop"):
        run = dusty.DustyRun(n_dust)
        fl = [run.gas, run.dust]
        if name == "host_loop":
            tm = ib.TimeManager(cfl=CFL)
            for _ in range(6):
                ib.run_iteration(fl, run.geo, tm, 2, num, drag=drag)
            ms = _events_ms(lambda: [ib.run_iteration(fl, run.geo, tm, 2, num, drag=drag) for _ in range(dust_iters)])
        else:
            loop = ib.GraphLoop(fl, run.geo, 2, num, drag=drag, cfl=CFL)
            ms = _events_ms(lambda: loop.run(dust_iters, check_every=dust_iters + 1))
        out.setdefault("gas_dust_%d_exact_drag" % n_dust, {})[name] = {"ms_per_iteration": ms / dust_iters}
        del run
    return out


def case_graph(args):
    """Host loop against the device-time CUDA-graph loop (graph_loop_timing)."""
    print(json.dumps({"case": "graph", **graph_loop_timing()}))


CASES = {"ensemble": case_ensemble, "graph": case_graph, "sweeps": case_sweeps, "time-sweeps": case_time_sweeps, "cfl": case_cfl, "drag": case_drag,
         "all": case_all}


def dist_init(n_gpus):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        dist.init_process_group("nccl" if torch.cuda.is_available() else "gloo",
                                timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def max_over_ranks(ms, world, device):
    """The slowest rank's time: every rank contributes its own and all get the maximum."""
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(world, cells, steps, ms_max):
    """Whole-job Mcell-updates/s of `world` replicas that each advanced `cells` for `steps`."""
    return world * cells * steps / (ms_max / 1e3) / 1e6


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ["index", "clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.active",
              "clocks_event_reasons.hw_slowdown", "clocks_event_reasons.hw_thermal_slowdown",
              "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap"]

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self, wait_s=10.0):
        """Starts nvidia-smi (20 ms interval) and waits for its first sample, so that the timed
        region that follows is covered from its beginning."""
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=" + ",".join(self.FIELDS), "--format=csv,noheader,nounits",
                 "-lms", "20", "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
            return
        t0 = time.time()
        while not self.lines and time.time() - t0 < wait_s:
            time.sleep(0.01)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def mark(self):
        """Host time stamp for the window of samples kept (begin and end of the timed region)."""
        return time.time()

    def stop(self, begin=None, end=None):
        """Stops sampling; summarises the samples taken between begin and end (host times of the
        timed region; the sample after end is kept too, as it covers the region's last interval)."""
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.05)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = list(self.lines)
        if begin is not None and end is not None:
            inside = [l for t, l in lines if begin <= t <= end]
            after = [l for t, l in lines if t > end][:1]
            lines = inside + after
        else:
            lines = [l for _, l in lines]
        for l in lines:
            p = [x.strip() for x in l.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
                power.append(float(p[3]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": max(power) if power else None}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def cpu_reference_sample(shape, iterations=1):
    """Time the oracle (C restatement of the reference kernels, OpenMP on all host threads) on
    `iterations` iterations of the workload; returns (Mcell-updates/s, seconds, threads)."""
    from oracle import pyoracle as po
    from gpuimogen_b200 import problems
    po.lib()
    q = problems.kelvin_helmholtz(shape, gamma=GAMMA, seed=12345)
    h = [1.0 / s for s in shape]
    sp = po.step_params(0.0, h, GAMMA, rho_min=1e-5, method=METHOD, slope="mc")
    bc = ["circular"] * 6
    t0 = time.perf_counter()
    for it in range(iterations):
        tau = po.cfl_timestep(q, shape, GAMMA, h, METHOD)
        sp.dt = CFL * tau
        po.fluid_step_3d(q, shape, sp, bc, 1, it)
        po.fluid_step_3d(q, shape, sp, bc, -1, it)
    sec = time.perf_counter() - t0
    cells = shape[0] * shape[1] * shape[2]
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return cells * iterations / sec / 1e6, sec, threads


def bench_config(shape, world):
    """The workload's config dict, the same for both arms of the benchmark."""
    return {"workload": "kelvin_helmholtz_3d_hllc_fp64", "grid": list(shape), "gamma": GAMMA, "cfl": CFL,
            "limiter": "MC", "method": "HLLC", "time_scheme": "SSPRK2", "boundaries": "periodic",
            "parallelism": "replicas" if world > 1 else "single",
            "l2_policy": "state %.0f MB > 126 MB L2, no flush needed"
                         % (5 * 8 * ((shape[0] * shape[1] * shape[2] + 31) // 32 * 32) / 1e6)}


def _stats(xs):
    """Median and spread of repeated measurements."""
    xs = sorted(xs)
    return {"median": float(np.median(xs)), "min": float(xs[0]), "max": float(xs[-1]), "n": len(xs)}


def _events_ms(fn, stream=None):
    """CUDA-event time of fn() on the current stream (synchronised on both sides)."""
    import torch
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    fn()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b)


def form_fp32_flux(reps=5, iters=10, l1_steps=200, shape=(512, 512, 256)):
    """Precision form, KH 512 x 512 x 256 HLLC MC: FP64 and FP32-flux throughput (median of `reps`
    timings of `iters` iterations each, after warm-up) and the FP32-flux result's relative L1 error
    against the FP64 run after `l1_steps` iterations from the same seeded state."""
    import torch
    import gpuimogen_b200 as ib
    from gpuimogen_b200 import problems
    q0 = torch.from_numpy(problems.kelvin_helmholtz(shape, gamma=GAMMA, seed=12345)).cuda()
    cells = shape[0] * shape[1] * shape[2]
    geo = ib.Geometry(shape)
    out = {"workload": "kelvin_helmholtz_3d_hllc_mc", "grid": list(shape), "iterations_per_timing": iters}
    finals = {}
    for prec in ("fp64", "fp32flux"):
        num = ib.numerics(slope="mc", precision=prec)
        fl = ib.Fluid(shape, q=q0.clone(), gamma=GAMMA)
        tm = ib.TimeManager(cfl=CFL)
        for _ in range(3):
            ib.run_iteration([fl], geo, tm, METHOD, num)
        vals = []
        for _ in range(reps):
            ms = _events_ms(lambda: [ib.run_iteration([fl], geo, tm, METHOD, num) for _ in range(iters)])
            vals.append(cells * iters / (ms / 1e3) / 1e6)
        out[prec] = {"mcell_updates_per_s": _stats(vals)}
        fl.q.copy_(q0)
        tm = ib.TimeManager(cfl=CFL)
        for _ in range(l1_steps):
            ib.run_iteration([fl], geo, tm, METHOD, num)
        finals[prec] = fl.q[:, :cells].clone()
        del fl
    a, b = finals["fp32flux"], finals["fp64"]
    rel = ((a - b).abs().sum(dim=1) / b.abs().sum(dim=1)).cpu().numpy()
    mom = float(((a[2:] - b[2:]).abs().sum() / b[2:].abs().sum()).item())
    out["rel_l1_vs_fp64_after_%d" % l1_steps] = {"rho": float(rel[0]), "E": float(rel[1]), "momentum": mom}
    out["speedup_fp32flux"] = (out["fp32flux"]["mcell_updates_per_s"]["median"] /
                               out["fp64"]["mcell_updates_per_s"]["median"])
    return out


def form_ensemble(reps=5, nprob=4096):
    """Batching form: 4096 HLLC Riemann problems, N ~ U{256..4096}, each to t = 0.1 in one
    persistent graph-captured launch (autotuned shape), FP64 and FP32 flux: Mcell-updates/s as the
    median of `reps` graph replays, and the FP32-flux density error against FP64."""
    import torch
    from gpuimogen_b200 import ensemble
    ens = ensemble.RiemannEnsemble.random(nprob, seed=1)
    out = {"workload": "riemann_ensemble_hllc", "problems": nprob, "cells": ens.cells, "t_end": 0.1}
    final = {}
    for prec in ("fp64", "fp32flux"):
        tune = ensemble.autotune(ens, t_end=0.1, cfl=CFL, slope="mc", precision=prec)
        g = ens.capture(t_end=0.1, cfl=CFL, slope="mc", precision=prec, tuning=tune)
        vals = []
        for _ in range(reps):
            ms = _events_ms(g.replay)
            vals.append(ens.cell_updates() / (ms / 1e3) / 1e6)
        final[prec] = ens.q[0, :ens.cells].clone()
        out[prec] = {"mcell_updates_per_s": _stats(vals), "tuning": tune, "cell_updates": ens.cell_updates()}
        del g
    a, b = final["fp32flux"], final["fp64"]
    out["fp32flux_rel_l1_rho_vs_fp64"] = float(((a - b).abs().sum() / b.abs().sum()).item())
    out["speedup_fp32flux"] = (out["fp32flux"]["mcell_updates_per_s"]["median"] /
                               out["fp64"]["mcell_updates_per_s"]["median"])
    return out


def form_two_fluid(reps=5, iters=10, l1_steps=500, n=2048):
    """Learned-drag form, 2-D gas + dust on 2048^2: a drag model trained on 1e7 exact samples (the
    library's training kernels), then exact LogTrap2 vs learned drag: one drag call (median of
    `reps`, each on the initial state), one two-fluid iteration (median of `reps` timings of
    `iters` iterations) and the learned run's relative L1 against the exact run after `l1_steps`."""
    import torch
    from gpuimogen_b200 import dusty
    from gpuimogen_b200 import learned_drag as ld
    model, hist = ld.train(n_samples=10_000_000, epochs=10, seed=2024)
    runs = {"exact": dusty.DustyRun(n), "learned": dusty.DustyRun(n, model=model)}
    cells = n * n
    out = {"workload": "gas_dust_2d", "grid": [n, n], "training_val_rmse_log_s": hist["val_rmse_log_s"][-1]}
    for name, r in runs.items():
        call = []
        for _ in range(reps + 1):
            r.reset()
            call.append(_events_ms(lambda: r.drag([r.gas, r.dust], 4e-5)))
        r.reset()
        r.run(2)
        it = []
        for _ in range(reps):
            it.append(_events_ms(lambda: r.run(iters)) / iters)
        out[name] = {"drag_call_ms": _stats(call[1:]), "iteration_ms": _stats(it),
                     "mcell_updates_per_s": cells / (float(np.median(it)) / 1e3) / 1e6}
    for r in runs.values():
        r.reset()
        r.run(l1_steps)
    torch.cuda.synchronize()
    ex, le = runs["exact"], runs["learned"]

    def rel(a, b):
        return [float((a[k, :cells] - b[k, :cells]).abs().sum() / max(float(b[k, :cells].abs().sum()), 1e-300))
                for k in range(5)]
    out["learned_vs_exact_rel_l1_after_%d" % l1_steps] = {"gas": rel(le.gas.q, ex.gas.q),
                                                          "dust": rel(le.dust.q, ex.dust.q)}
    out["learned_fallback_cells"] = int(le.fallbacks.item())
    out["speedup_drag_call"] = out["exact"]["drag_call_ms"]["median"] / out["learned"]["drag_call_ms"]["median"]
    out["speedup_iteration"] = out["exact"]["iteration_ms"]["median"] / out["learned"]["iteration_ms"]["median"]
    return out


def reference_gpu_sample(shape, warmup=3, iters=20, reps=3):
    """The reference's own GPU kernels (its gpuclass sources compiled for sm_100a into oracle/_ref,
    MC limiter) on the same workload and GPU: Mcell-updates/s, median of `reps` timings of `iters`
    iterations (the reference's host-side timing of its own loop, which allocates temporaries every
    call).  None when the reference build is absent."""
    import ctypes
    from gpuimogen_b200 import problems
    path = os.path.join(ROOT, "oracle", "_ref", "libimogen_ref_mc.so")
    if not os.path.exists(path):
        return None
    L = ctypes.CDLL(path)
    dp = ctypes.POINTER(ctypes.c_double)
    L.ref_time.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int64, ctypes.c_double,
                           ctypes.c_int, dp, ctypes.c_double, ctypes.c_int, ctypes.c_int, dp]
    q = problems.kelvin_helmholtz(shape, gamma=GAMMA, seed=12345)
    h = np.array([1.0 / s for s in shape])
    cells = shape[0] * shape[1] * shape[2]
    vals = []
    for _ in range(reps):
        ms = ctypes.c_double(0)
        qq = q.copy()
        rc = L.ref_time(qq.ctypes.data_as(dp), shape[0], shape[1], shape[2], q.shape[1], GAMMA, METHOD,
                        h.ctypes.data_as(dp), CFL, warmup, iters, ctypes.byref(ms))
        if rc != 0:
            return {"error": "reference returned %d" % rc}
        vals.append(cells * iters / (ms.value / 1e3) / 1e6)
    return {"mcell_updates_per_s": _stats(vals), "iterations": iters,
            "build": "reference gpuclass sources, MC limiter, nvcc -O2 sm_100a (oracle/ref_harness)"}


def run_reference(args, world, rank):
    if rank != 0:
        return 0
    shape = tuple(int(s) for s in args.shape.split(",")) if args.shape else SHAPE
    # bounded sample: one iteration of the full 256^3 workload per timed step
    for _ in range(max(0, min(args.warmup, 1))):
        cpu_reference_sample((64, 64, 64), 1)
    vals, secs = [], []
    for _ in range(args.steps):
        v, s, thr = cpu_reference_sample(shape, 1)
        vals.append(v)
        secs.append(s)
    total = sum(secs)
    value = shape[0] * shape[1] * shape[2] * args.steps / total / 1e6
    line = {
        "metric": METRIC, "value": value, "unit": "Mcell-updates/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": bench_config(shape, world),
        "cpu_baseline": {"value": value, "unit": "Mcell-updates/s", "cores": thr, "kind": "port",
                         "sample": "%d iteration(s) of the %dx%dx%d workload per step, oracle C restatement of the "
                                   "reference kernels (the reference has no CPU implementation of this path)"
                                   % (1, *shape)},
        "e2e": {"value": value, "unit": "Mcell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.case != "bench":
        import torch
        import gpuimogen_b200 as ib
        torch.cuda.set_device(0)
        ib.load("product")
        CASES[args.case](args)
        return 0
    world, rank, local = dist_init(args.gpus)
    if args.impl == "reference":
        rc = run_reference(args, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return rc

    import torch
    import torch.distributed as dist
    import gpuimogen_b200 as ib
    from gpuimogen_b200 import problems

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ib.load("product")
    shape = tuple(int(s) for s in args.shape.split(",")) if args.shape else SHAPE
    cells = shape[0] * shape[1] * shape[2]
    q0 = problems.kelvin_helmholtz(shape, gamma=GAMMA, seed=12345 + rank)
    slab = q0.shape[1]
    fl = ib.Fluid(shape, bc="circular", q=torch.from_numpy(q0).to(dev), gamma=GAMMA)
    geo = ib.Geometry(shape)
    num = ib.numerics(slope="mc")
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()

    # The main loop runs through GraphLoop (timestep.py): the time state stays on the device and
    # every iteration -- CFL reduction, time update, forward and backward fluid steps, time advance
    # -- is one replayed CUDA graph; its construction runs six eager iterations (setting up scratch
    # memory and capturing), then W warm-up replays.
    loop = ib.GraphLoop([fl], geo, METHOD, num, cfl=CFL)
    loop.run(args.warmup, check_every=args.warmup + 1)
    torch.cuda.synchronize()

    # ---------------- device-resident timed region ----------------
    sampler = ClockSampler(torch.cuda.current_device() if "CUDA_VISIBLE_DEVICES" not in os.environ
                           else int(os.environ["CUDA_VISIBLE_DEVICES"].split(",")[local]))
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    ph0 = loop.phase
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    t_begin = sampler.mark()
    e0.record(stream)
    loop.run(args.steps, check_every=args.steps + 1)
    e1.record(stream)
    torch.cuda.synchronize()
    t_end = sampler.mark()
    # the library kernels the replayed graphs launched (each phase's count from its eager run)
    launches = sum(loop.launches[(ph0 + k) % 6] for k in range(args.steps))
    clocks = sampler.stop(t_begin, t_end)
    tm = ib.TimeManager(cfl=CFL)
    tm.dTime = loop.state().dt
    ms = e0.elapsed_time(e1)
    barrier()
    ms_max = max_over_ranks(ms, world, dev)
    value = job_value(world, cells, args.steps, ms_max)

    # ---------------- per-kernel roofline (same stream, CUDA events) ----------------
    peak, peak_kind = measured_peaks()
    kern = {}
    reps = max(3, min(10, args.steps))
    for d, name in ((1, "x_row"), (2, "y_pair"), (3, "z_pair")):
        dt = tm.dTime
        ib.cudaFluidStep(fl, geo, [dt, 1, GAMMA, 1e-5, METHOD, d], num)  # warm
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        for _ in range(reps):
            ib.cudaFluidStep(fl, geo, [dt, 1, GAMMA, 1e-5, METHOD, d], num)
        b.record(stream)
        torch.cuda.synchronize()
        kern[name] = a.elapsed_time(b) / reps
    # CFL reduction
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    tau_dev = torch.zeros(1, dtype=torch.float64, device=dev)
    a.record(stream)
    for _ in range(reps):
        ib.cflTimestepFused(fl, GAMMA, geo, METHOD, tau_device=tau_dev)
    b.record(stream)
    torch.cuda.synchronize()
    kern["cfl"] = a.elapsed_time(b) / reps
    # share per iteration: 2 x-row launches, 2 y, 2 z, 1 cfl
    share = {"x_row": 2 * kern["x_row"], "y_pair": 2 * kern["y_pair"], "z_pair": 2 * kern["z_pair"],
             "cfl": kern["cfl"]}
    dom = max(share, key=share.get)
    alg_bytes = (80 if dom != "cfl" else 40) * cells
    achieved = alg_bytes / (kern[dom] / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": (TRAFFIC_B_PER_CELL.get(dom, 0) * cells) or None, "kernel": dom, "peak_source": peak_kind,
                "per_kernel_ms": kern, "step_alg_bytes_per_cell": 480 + 40,
                "step_frac": (520 * cells) / (ms_max / args.steps / 1e3) / 1e9 / peak}

    # ---------------- end to end through the public API with host buffers ----------------
    # Every step is one job: its input state is copied in from pinned host memory, the step runs
    # through the public API (run_iteration: CFL timestep read to the host, six sweeps), and its
    # result state is copied back out.  Uploads and downloads have their own streams and the
    # device state has E2E_BUFFERS copies, so step i's compute overlaps step i+1's upload and
    # step i-1's download (the copy engines and the SMs work at once).  Timed from the first upload's
    # start to the last download's end (CUDA events; all streams of this device).
    # at least 20 steps, so that the first upload and the last download (not overlapped with
    # anything) weigh as little as in a long run of the same pipeline
    e2e_steps = max(20, min(args.steps, 40))
    NB = E2E_BUFFERS
    pinned_in = torch.from_numpy(q0).pin_memory()
    pinned_out = [torch.empty_like(pinned_in).pin_memory() for _ in range(NB)]
    bufs = [fl] + [ib.Fluid(shape, q=torch.empty_like(fl.q), gamma=GAMMA) for _ in range(NB - 1)]
    s_up, s_down = torch.cuda.Stream(), torch.cuda.Stream()
    up_done = [torch.cuda.Event() for _ in range(NB)]
    comp_done = [torch.cuda.Event() for _ in range(NB)]
    down_done = [torch.cuda.Event() for _ in range(NB)]
    tm2 = ib.TimeManager(cfl=CFL)
    torch.cuda.synchronize()
    barrier()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)

    def upload(i):
        k = i % NB
        with torch.cuda.stream(s_up):
            if i >= NB:
                s_up.wait_event(down_done[k])   # buffer k's previous result has been read out
            bufs[k].q.copy_(pinned_in, non_blocking=True)
            up_done[k].record(s_up)

    a.record(s_up)
    upload(0)
    for i in range(e2e_steps):
        k = i % NB
        if i + 1 < e2e_steps:
            upload(i + 1)                       # queued before this step's compute blocks the host
        stream.wait_event(up_done[k])
        ib.run_iteration([bufs[k]], geo, tm2, METHOD, num)
        comp_done[k].record(stream)
        with torch.cuda.stream(s_down):
            s_down.wait_event(comp_done[k])
            pinned_out[k].copy_(bufs[k].q, non_blocking=True)
            down_done[k].record(s_down)
    s_down.wait_stream(s_up)
    b.record(s_down)
    torch.cuda.synchronize()
    e2e_ms = a.elapsed_time(b)
    e2e_val = job_value(world, cells, e2e_steps, max_over_ranks(e2e_ms, world, dev))
    nbytes = 5 * slab * 8

    # ---------------- the FP32-flux, batched-ensemble and learned-drag forms (rank 0, N = 1 only) ----
    forms = None
    if rank == 0 and world == 1 and os.environ.get("IMOGEN_BENCH_SKIP_FORMS") != "1":
        forms = {"fp32_flux": form_fp32_flux(), "ensemble": form_ensemble(), "two_fluid": form_two_fluid()}

    # ---------------- baselines (rank 0, N = 1 only) ----------------
    cpu = None
    if rank == 0 and world == 1 and os.environ.get("IMOGEN_BENCH_SKIP_CPU") != "1":
        v, s, thr = cpu_reference_sample(shape, 1)
        cpu = {"value": v, "unit": "Mcell-updates/s", "cores": thr, "kind": "port",
               "sample": "1 iteration of the %dx%dx%d workload (%.1f s), oracle C restatement, OpenMP" % (*shape, s),
               "reference_gpu": reference_gpu_sample(shape)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Mcell-updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(shape, world),
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_val, "unit": "Mcell-updates/s", "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": nbytes + 8, "steps": e2e_steps,
                    "copies": "own streams, %d device copies of the state (upload i+1 and download i-1 "
                              "overlap step i)" % NB},
            "gpu_launches": launches,
            "clocks": clocks,
            "forms": forms,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
