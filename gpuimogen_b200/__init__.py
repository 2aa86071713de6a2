"""gpuimogen_b200: B200-native (sm_100a) fluid-step hot path of the Imogen hydrodynamics code.

The compiled library (libimogen_b200.so, C ABI in include/imogen_b200.h) implements the
dimensionally split HLL / HLLC / Xin-Jin sweeps with their limiters, the CFL reduction, boundary
fill, the pressure/freeze pass and the two-fluid drag source; this package binds it with the
call forms of the reference's mex functions.
"""
from .imogen import (BC, DRAG, FLUXLIM, METHOD, PRECISION, SLOPE, Fluid, Geometry, ImogenError,  # noqa: F401
                     cflTimestep, cflTimestepFused, cudaFluidStep, cudaSoundspeed, cudaSource2FluidDrag,
                     cudaStatics, completeTimestep, device_wait_status, fluidstep, freezeAndPtot, load, numerics,
                     setFluidBoundary,
                     slab_pitch, use_variant)
from .timestep import GraphLoop, TimeManager, cfl_tau, run_iteration  # noqa: F401

__all__ = [
    "Fluid", "Geometry", "ImogenError", "TimeManager", "cudaFluidStep", "fluidstep", "cflTimestep",
    "cflTimestepFused", "cudaSoundspeed", "freezeAndPtot", "cudaStatics", "setFluidBoundary",
    "cudaSource2FluidDrag", "numerics", "load", "use_variant", "run_iteration", "cfl_tau", "device_wait_status",
    "completeTimestep", "GraphLoop",
]
