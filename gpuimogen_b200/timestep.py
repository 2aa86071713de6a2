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
