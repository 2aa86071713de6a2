"""Time bookkeeping and the complete fluid iteration.

TimeManager restates time/TimeManager.m:124-186 (dt = CFL * tau, last-step clip so that
t + 2 dt <= TIMEMAX) and :270-277 (iteration += 1, Kahan-compensated t += 2 dt).  run_iteration
is the main loop body of imogen.m:115-139 / performCompleteTimestep (flux_multi.cu:174-272):
source half step, forward fluid step, full source step, backward fluid step, source half step.
"""
import math

import torch

from . import imogen as ib


class TimeManager:
    def __init__(self, cfl=0.4, tmax=math.inf, itermax=None):
        self.CFL = cfl
        self.TIMEMAX = tmax
        self.ITERMAX = itermax
        self.time = 0.0
        self.iteration = 0
        self.dTime = 0.0
        self._kahan_c = 0.0

    def update(self, tau):
        self.dTime = self.CFL * tau
        if self.time + 2 * self.dTime > self.TIMEMAX:
            self.dTime = .5 * (self.TIMEMAX - self.time)
        return self.dTime

    def step(self):
        self.iteration += 1
        y = (2 * self.dTime) - self._kahan_c
        t = self.time + y
        self._kahan_c = (t - self.time) - y
        self.time = t

    @property
    def running(self):
        if self.ITERMAX is not None and self.iteration >= self.ITERMAX:
            return False
        return self.time < self.TIMEMAX * (1 - 1e-14) if math.isfinite(self.TIMEMAX) else True


def cfl_tau(fluids, geometry, method):
    """Minimum over fluids of the CFL time (TimeManager.update loop)."""
    tau = 1e38
    for f in fluids:
        t = ib.cflTimestepFused(f, f.gamma, geometry, method)
        if not math.isfinite(t):
            raise ib.ImogenError("cflTimestep: non-finite timestep", -101)
        tau = min(tau, t)
    return tau


def run_iteration(fluids, geometry, tm, method, num=None, source=None, drag=None):
    """One main-loop iteration; `source(fluids, dt_fraction)` applies the sources if given
    (forward and backward fluid steps through fluidstep, as the Matlab loop calls them);
    otherwise the complete timestep runs through completeTimestep (performCompleteTimestep), with
    the two-fluid drag between the steps when drag = (thermo_gas, thermo_dust, method)."""
    tau = cfl_tau(fluids, geometry, method)
    dt = tm.update(tau)
    if source is not None:
        source(fluids, 0.5 * dt)
        ib.fluidstep(fluids, geometry, [dt, 1, 1, tm.iteration, method], num)
        source(fluids, dt)
        ib.fluidstep(fluids, geometry, [dt, 1, -1, tm.iteration, method], num)
        source(fluids, 0.5 * dt)
    else:
        ib.completeTimestep(fluids, geometry, [dt, 1, tm.iteration, method], num, drag=drag)
    tm.step()
    return dt


class GraphLoop:
    """The main loop with its timestep on the device, replayed from CUDA graphs.

    Each iteration is the CFL reduction of every fluid into an ib_time_state in device memory,
    ib_timeUpdate (dt = CFL * min tau with the end-time clip), ib_completeTimestepDeviceDt (sources
    and both fluid steps reading dt from the device) and ib_timeAdvance (compensated time sum).  No
    host value depends on dt, so the first six iterations run eagerly (they set up the library's
    scratch memory and kernel attributes for every sweep order) and are then captured as six
    graphs, one per iteration index modulo 6; run() replays them and reads the time state back
    every `check_every` iterations.  Past the end time dt is 0 and every kernel returns at once, so
    replays beyond it change nothing.  Results are bit for bit those of run_iteration.
    drag = (thermo_gas, thermo_dust, method) for gas + dust (fluids [gas, dust])."""

    def __init__(self, fluids, geometry, method, num=None, drag=None, cfl=0.4, tmax=math.inf):
        if isinstance(fluids, ib.Fluid):
            fluids = [fluids]
        assert 1 <= len(fluids) <= 4
        self.fluids, self.geometry, self.method, self.num, self.drag = fluids, geometry, method, num, drag
        dev = fluids[0].q.device
        st = ib.IbTimeState()
        st.cfl, st.tmax, st.nfluids = float(cfl), float(tmax), len(fluids)
        raw = bytes(st)
        self._ts = torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(dev)
        self.ts_ptr = self._ts.data_ptr()
        self._dt_ptr = self.ts_ptr + ib.IbTimeState.dt.offset
        self._graphs = []
        self.phase = 0
        # the library's kernel launches of each phase's iteration (what a replay of its graph runs)
        self.launches = []
        for _ in range(6):
            l0 = ib.launch_count()
            self._iteration(self.phase)
            self.launches.append(ib.launch_count() - l0)
            self.phase += 1
        torch.cuda.synchronize()
        for p in range(6):
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, capture_error_mode="thread_local"):
                self._iteration(p)
            self._graphs.append(g)
        torch.cuda.synchronize()

    def _iteration(self, phase):
        for k, f in enumerate(self.fluids):
            ib.cflTimestepFused(f, f.gamma, self.geometry, self.method,
                                tau_device=_DevAddr(self.ts_ptr + 8 * k))
        ib.timeUpdate(self.ts_ptr)
        ib.completeTimestepDeviceDt(self.fluids, self.geometry, self._dt_ptr, [1, phase, self.method], self.num,
                                    drag=self.drag)
        ib.timeAdvance(self.ts_ptr)

    def state(self):
        """The device time state as a ctypes ib_time_state (synchronises)."""
        return ib.IbTimeState.from_buffer_copy(bytes(self._ts.cpu().numpy()))

    @property
    def time(self):
        return self.state().time

    @property
    def iteration(self):
        return self.state().iteration

    def done(self):
        s = self.state()
        if s.status:
            raise ib.ImogenError("cflTimestep: non-finite timestep", -101)
        return math.isfinite(s.tmax) and not (s.time < s.tmax * (1 - 1e-14))

    def run(self, iterations=None, check_every=16):
        """Replays iterations until the end time (checked every `check_every` replays) or until
        `iterations` more have been replayed."""
        k = 0
        while iterations is None or k < iterations:
            self._graphs[self.phase % 6].replay()
            self.phase += 1
            k += 1
            if k % check_every == 0 and self.done():
                break
        return self


class _DevAddr:
    """A device address where ib.cflTimestepFused expects a tensor (it reads .data_ptr())."""

    def __init__(self, addr):
        self.addr = addr

    def data_ptr(self):
        return self.addr
