"""ctypes binding of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by bench.py's CPU
baseline leg, as the checker.  The product package never imports it.

Arrays are numpy float64 of shape (5, slab) holding [rho, E, px, py, pz] with x fastest in each
slab (slab >= nx*ny*nz), the same layout the library uses in device memory.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

SLOPE = {"ospre": 0, "mc": 1, "vanleer": 2, "minmod": 3, "superbee": 4, "vanalbada": 5, "zero": 6}
FLUXLIM = {"ospre": 0, "vanleer": 1, "minmod": 2, "superbee": 3, "zero": 4}
BC = {"circular": 0, "mirror": 1, "wall": 2, "stationary": 3, "const": 4, "linear": 5,
      "outflow": 6, "freebalance": 7}


class Grid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
                ("pad_", ctypes.c_int32), ("slab", ctypes.c_int64)]


class Step(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_double), ("h", ctypes.c_double * 3), ("gamma", ctypes.c_double),
                ("rho_min", ctypes.c_double), ("c_iso", ctypes.c_double),
                ("method", ctypes.c_int32), ("slope_limiter", ctypes.c_int32),
                ("flux_limiter", ctypes.c_int32), ("geometry", ctypes.c_int32),
                ("r_inner", ctypes.c_double), ("theta_form", ctypes.c_int32),
                ("cyl_flags", ctypes.c_int32)]

GEO_SQUARE, GEO_CYLINDRICAL = 0, 1
THETA_213, THETA_231 = 0, 1
CYL_GEOMETRIC_RADIUS = 1


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        L.or_fluid_sweep.argtypes = [dp, ctypes.POINTER(Grid), ctypes.POINTER(Step), ctypes.c_int]
        L.or_fluid_boundary.argtypes = [dp, ctypes.POINTER(Grid), ctypes.POINTER(ctypes.c_int32),
                                        ctypes.c_int, ctypes.c_int]
        L.or_fluid_step_3d.argtypes = [dp, ctypes.POINTER(Grid), ctypes.POINTER(Step),
                                       ctypes.POINTER(ctypes.c_int32), ctypes.c_int, ctypes.c_int]
        L.or_soundspeed.argtypes = [dp, ctypes.POINTER(Grid), ctypes.c_double, dp]
        L.or_cfl_timestep.argtypes = [dp, dp, ctypes.POINTER(Grid), dp,
                                      ctypes.POINTER(ctypes.c_int32), ctypes.c_int]
        L.or_cfl_timestep.restype = ctypes.c_double
        L.or_cfl_timestep_geo.argtypes = [dp, dp, ctypes.POINTER(Grid), dp,
                                          ctypes.POINTER(ctypes.c_int32), ctypes.c_int, ctypes.c_int,
                                          ctypes.c_double]
        L.or_cfl_timestep_geo.restype = ctypes.c_double
        L.or_cyl_source.argtypes = [dp, ctypes.POINTER(Grid), ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double]
        L.or_theta_form.argtypes = [ctypes.c_int, ctypes.c_int]
        L.or_theta_form.restype = ctypes.c_int
        L.or_freeze_and_ptot.argtypes = [dp, ctypes.POINTER(Grid), ctypes.c_double,
                                         ctypes.c_double, dp, dp]
        L.or_array_boundary.argtypes = [dp, ctypes.POINTER(Grid), ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.or_statics_fade.argtypes = [dp, dp, ctypes.c_int64, ctypes.c_int64]
        L.or_drag_2fluid.argtypes = [dp, dp, ctypes.POINTER(Grid), dp, dp, ctypes.c_double,
                                     ctypes.c_int, dp]
        L.or_drag_params.argtypes = [dp, dp, ctypes.c_double, dp]
        L.or_drag_logtrap_cells.argtypes = [dp, dp, ctypes.c_int64, ctypes.c_int64, dp,
                                            ctypes.c_double, ctypes.c_int]
        _LIB = L
    return _LIB


def _p(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def grid(shape, slab=None):
    nx, ny, nz = shape
    return Grid(nx, ny, nz, 0, slab if slab is not None else nx * ny * nz)


def step_params(dt, h, gamma, rho_min=1e-5, c_iso=-1.0, method=2, slope="ospre", fluxlim="ospre",
                cylindrical=False, r_inner=0.0, theta_form=THETA_213, geometric_radius=False):
    return Step(dt, (ctypes.c_double * 3)(*h), gamma, rho_min, c_iso, method,
                SLOPE[slope], FLUXLIM[fluxlim], GEO_CYLINDRICAL if cylindrical else GEO_SQUARE,
                r_inner, theta_form, CYL_GEOMETRIC_RADIUS if geometric_radius else 0)


def _bcarr(bc):
    arr = (ctypes.c_int32 * 6)(*[BC[b] if isinstance(b, str) else int(b) for b in bc])
    return arr


def fluid_sweep(q, shape, sp, direction):
    g = grid(shape, q.shape[1])
    rc = lib().or_fluid_sweep(_p(q), ctypes.byref(g), ctypes.byref(sp), direction)
    if rc:
        raise RuntimeError("or_fluid_sweep rc=%d" % rc)


def fluid_boundary(q, shape, bc, direction, depth=4):
    g = grid(shape, q.shape[1])
    rc = lib().or_fluid_boundary(_p(q), ctypes.byref(g), _bcarr(bc), direction, depth)
    if rc:
        raise RuntimeError("or_fluid_boundary rc=%d" % rc)


def fluid_step_3d(q, shape, sp, bc, sweep_dir, step_number):
    g = grid(shape, q.shape[1])
    rc = lib().or_fluid_step_3d(_p(q), ctypes.byref(g), ctypes.byref(sp), _bcarr(bc),
                                sweep_dir, step_number)
    if rc:
        raise RuntimeError("or_fluid_step_3d rc=%d" % rc)


def soundspeed(q, shape, gamma):
    g = grid(shape, q.shape[1])
    cs = np.zeros(shape[0] * shape[1] * shape[2])
    lib().or_soundspeed(_p(q), ctypes.byref(g), gamma, _p(cs))
    return cs


def cfl_timestep(q, shape, gamma, h, method, cs=None, cylindrical=False, r_inner=0.0):
    if cs is None:
        cs = soundspeed(q, shape, gamma)
    g = grid(shape, q.shape[1])
    hh = np.ascontiguousarray(h, dtype=np.float64)
    rez = (ctypes.c_int32 * 3)(*shape)
    return lib().or_cfl_timestep_geo(_p(q), _p(cs), ctypes.byref(g), _p(hh), rez, method,
                                     GEO_CYLINDRICAL if cylindrical else GEO_SQUARE, r_inner)


def cyl_source(q, shape, dt, dr, r_inner):
    """Cylindrical geometric source terms over dt, in place."""
    g = grid(shape, q.shape[1])
    lib().or_cyl_source(_p(q), ctypes.byref(g), dt, dr, r_inner)


def theta_form(sweep_dir, step_number):
    return lib().or_theta_form(sweep_dir, step_number)


def freeze_and_ptot(q, shape, gamma, cs_min):
    g = grid(shape, q.shape[1])
    nx, ny, nz = shape
    ptot = np.zeros(nx * ny * nz)
    freeze = np.zeros(ny * nz)
    lib().or_freeze_and_ptot(_p(q), ctypes.byref(g), gamma, cs_min, _p(ptot), _p(freeze))
    return ptot, freeze


def array_boundary(phi, shape, mode, direction, side, vec_component=0, depth=4):
    g = grid(shape)
    m = BC[mode] if isinstance(mode, str) else int(mode)
    return lib().or_array_boundary(_p(phi), ctypes.byref(g), m, direction, side,
                                   vec_component, depth)


def statics_fade(phi, statics):
    """statics: float64 array (3, n) of [linear index; value; coefficient]."""
    st = np.ascontiguousarray(statics, dtype=np.float64)
    lib().or_statics_fade(_p(phi), _p(st), st.shape[1], st.shape[1])


def drag_params(thermo_gas, thermo_dust, dt):
    out = np.zeros(11)
    tg = np.ascontiguousarray(thermo_gas, dtype=np.float64)
    td = np.ascontiguousarray(thermo_dust, dtype=np.float64)
    lib().or_drag_params(_p(tg), _p(td), dt, _p(out))
    return out


def drag_2fluid(gas, dust, shape, thermo_gas, thermo_dust, dt, method, h=None):
    """Drag over dt in place; h = cell sizes (default 1/n per axis), used by ETDRK2 only."""
    g = grid(shape, gas.shape[1])
    tg = np.ascontiguousarray(thermo_gas, dtype=np.float64)
    td = np.ascontiguousarray(thermo_dust, dtype=np.float64)
    hh = np.ascontiguousarray([1.0 / s for s in shape] if h is None else h, dtype=np.float64)
    rc = lib().or_drag_2fluid(_p(gas), _p(dust), ctypes.byref(g), _p(tg), _p(td), dt, method, _p(hh))
    if rc:
        raise RuntimeError("or_drag_2fluid rc=%d" % rc)
