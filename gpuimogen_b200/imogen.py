"""Python binding of libimogen_b200.so with the reference's mex call forms.

Each function below mirrors one mex entry point of the reference's fluid-step hot path
(imogenproject/gpuImogen, gpuclass/): same name, same parameter-vector layout, same in-place
semantics and the same error behaviour (a non-zero status raises ImogenError, where the mex glue
calls mexErrMsgTxt).  Device memory is held in torch tensors; every call runs on the current
torch CUDA stream.  There is no CPU fallback: without the compiled library or a GPU every call
raises.
"""
import ctypes
import os

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))

SUCCESSFUL = 0
METHOD = {"hll": 1, "hllc": 2, "xinjin": 3}
SLOPE = {"ospre": 0, "mc": 1, "vanleer": 2, "minmod": 3, "superbee": 4, "vanalbada": 5, "zero": 6}
FLUXLIM = {"ospre": 0, "vanleer": 1, "minmod": 2, "superbee": 3, "zero": 4}
PRECISION = {"fp64": 0, "fp32flux": 1}
BC = {"circular": 0, "mirror": 1, "wall": 2, "stationary": 3, "const": 4, "linear": 5,
      "outflow": 6, "freebalance": 7}
DRAG = {"emp": 0, "rk4": 1, "etdrk1": 2, "etdrk2": 3, "logtrap2": 4, "logtrap3": 5}


class ImogenError(RuntimeError):
    def __init__(self, where, status):
        name = "UNKNOWN"
        try:
            name = _lib().ib_status_string(status).decode()
        except Exception:
            pass
        extra = ""
        if status == -1000:
            try:
                extra = " (cudaError %d)" % _lib().ib_last_cuda_error()
            except Exception:
                pass
        super().__init__("%s returned %d %s%s" % (where, status, name, extra))
        self.status = status


# ---------------------------------------------------------------------------------------------
# C structures (include/imogen_b200.h)
# ---------------------------------------------------------------------------------------------
class IbGrid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
                ("reserved", ctypes.c_int32), ("slab_pitch", ctypes.c_int64)]


class IbStatics(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("count", ctypes.c_int64), ("pitch", ctypes.c_int64)]


class IbFluid(ctypes.Structure):
    _fields_ = [("q", ctypes.c_void_p), ("grid", IbGrid), ("bc", ctypes.c_int32 * 6),
                ("halo", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("statics", IbStatics * 5)]


class IbFluidThermo(ctypes.Structure):
    _fields_ = [("gamma", ctypes.c_double), ("rho_min", ctypes.c_double),
                ("c_isothermal", ctypes.c_double)]


class IbGeometry(ctypes.Structure):
    _fields_ = [("h", ctypes.c_double * 3), ("r_inner", ctypes.c_double), ("shape", ctypes.c_int32),
                ("global_rez", ctypes.c_int32 * 3)]


class IbNumerics(ctypes.Structure):
    _fields_ = [("slope_limiter", ctypes.c_int32), ("flux_limiter", ctypes.c_int32),
                ("precision", ctypes.c_int32), ("flags", ctypes.c_int32)]


class IbThermo(ctypes.Structure):
    _fields_ = [("gamma", ctypes.c_double), ("mass", ctypes.c_double), ("mu0", ctypes.c_double),
                ("mu_t_index", ctypes.c_double), ("sigma0", ctypes.c_double),
                ("sigma_t_index", ctypes.c_double), ("k_bolt", ctypes.c_double),
                ("c_isothermal", ctypes.c_double)]


class IbDragSource(ctypes.Structure):
    _fields_ = [("thermo_gas", IbThermo), ("thermo_dust", IbThermo), ("method", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class IbTimeState(ctypes.Structure):
    _fields_ = [("tau", ctypes.c_double * 4), ("dt", ctypes.c_double), ("time", ctypes.c_double),
                ("kahan", ctypes.c_double), ("cfl", ctypes.c_double), ("tmax", ctypes.c_double),
                ("iteration", ctypes.c_int64), ("nfluids", ctypes.c_int32), ("status", ctypes.c_int32)]


class IbDragModel(ctypes.Structure):
    _fields_ = [("params", ctypes.c_void_p), ("feature_shift", ctypes.c_float * 5),
                ("feature_scale", ctypes.c_float * 5), ("out_shift", ctypes.c_float), ("out_scale", ctypes.c_float),
                ("domain_lo", ctypes.c_float * 5), ("domain_hi", ctypes.c_float * 5)]


# drag-decay MLP parameter layout (include/imogen_b200.h, IB_MLP_*)
MLP_IN, MLP_HID, MLP_NPARAM = 16, 64, 9473
MLP_OFF = {"W1": 0, "B1": 1024, "W2": 1088, "B2": 5184, "W3": 5248, "B3": 9344, "W4": 9408, "B4": 9472}


class IbEnsemble(ctypes.Structure):
    _fields_ = [("q", ctypes.c_void_p), ("slab_pitch", ctypes.c_int64), ("offsets", ctypes.c_void_p),
                ("h", ctypes.c_void_p), ("order", ctypes.c_void_p), ("t_out", ctypes.c_void_p),
                ("iters_out", ctypes.c_void_p), ("nproblems", ctypes.c_int32), ("bc", ctypes.c_int32 * 2),
                ("reserved", ctypes.c_int32)]


class IbEnsembleTuning(ctypes.Structure):
    _fields_ = [("threads", ctypes.c_int32), ("chunk", ctypes.c_int32), ("ctas_per_sm", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


EXPORTS = {
    "ib_slab_pitch": (ctypes.c_int64, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
    "ib_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "ib_last_cuda_error": (ctypes.c_int, []),
    "ib_launch_count": (ctypes.c_longlong, []),
    "ib_cudaFluidStep": (ctypes.c_int, [ctypes.POINTER(IbFluid), ctypes.POINTER(IbGeometry),
                                        ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                                        ctypes.POINTER(IbNumerics), ctypes.c_void_p]),
    "ib_fluidstep": (ctypes.c_int, [ctypes.POINTER(IbFluid), ctypes.POINTER(IbFluidThermo), ctypes.c_int,
                                    ctypes.POINTER(IbGeometry), ctypes.POINTER(ctypes.c_double),
                                    ctypes.c_int, ctypes.POINTER(IbNumerics), ctypes.c_void_p]),
    "ib_completeTimestep": (ctypes.c_int, [ctypes.POINTER(IbFluid), ctypes.POINTER(IbFluidThermo), ctypes.c_int,
                                           ctypes.POINTER(IbGeometry), ctypes.POINTER(ctypes.c_double),
                                           ctypes.c_int, ctypes.POINTER(IbNumerics), ctypes.POINTER(IbDragSource),
                                           ctypes.c_void_p]),
    "ib_completeTimestepDeviceDt": (ctypes.c_int, [ctypes.POINTER(IbFluid), ctypes.POINTER(IbFluidThermo),
                                                   ctypes.c_int, ctypes.POINTER(IbGeometry), ctypes.c_void_p,
                                                   ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                                                   ctypes.POINTER(IbNumerics), ctypes.POINTER(IbDragSource),
                                                   ctypes.c_void_p]),
    "ib_timeUpdate": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "ib_timeAdvance": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "ib_cudaSoundspeed": (ctypes.c_int, [ctypes.POINTER(IbFluid), ctypes.c_double, ctypes.c_void_p,
                                         ctypes.c_void_p]),
    "ib_cflTimestep": (ctypes.c_int, [ctypes.POINTER(IbFluid), ctypes.c_void_p, ctypes.POINTER(IbGeometry),
                                      ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]),
    "ib_cflTimestepFused": (ctypes.c_int, [ctypes.POINTER(IbFluid), ctypes.c_double,
                                           ctypes.POINTER(IbGeometry), ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_double), ctypes.c_void_p,
                                           ctypes.c_void_p]),
    "ib_device_wait_status": (ctypes.c_int, [ctypes.c_int]),
    "ib_setTileWaitLimit": (ctypes.c_int, [ctypes.c_longlong]),
    "ib_mlpWorkspaceFloats": (ctypes.c_int64, [ctypes.c_int64]),
    "ib_mlpLossGrad": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "ib_mlpForward": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                     ctypes.c_void_p]),
    "ib_mlpInferTC": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                     ctypes.c_void_p]),
    "ib_mlpAdam": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                  ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                                  ctypes.c_void_p]),
    "ib_dragDecayExact": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(IbThermo),
                                         ctypes.POINTER(IbThermo), ctypes.c_void_p, ctypes.c_void_p]),
    "ib_cudaSource2FluidDragLearned": (ctypes.c_int, [ctypes.POINTER(IbFluid), ctypes.POINTER(IbFluid),
                                                      ctypes.POINTER(IbThermo), ctypes.POINTER(IbThermo),
                                                      ctypes.POINTER(IbDragModel), ctypes.c_double, ctypes.c_void_p,
                                                      ctypes.c_void_p]),
    "ib_riemannEnsemble": (ctypes.c_int, [ctypes.POINTER(IbEnsemble), ctypes.POINTER(IbFluidThermo), ctypes.c_int,
                                          ctypes.c_double, ctypes.c_double, ctypes.c_int32,
                                          ctypes.POINTER(IbNumerics), ctypes.POINTER(IbEnsembleTuning),
                                          ctypes.c_void_p]),
    "ib_cflTimestepNoAlloc": (ctypes.c_int, [ctypes.POINTER(IbFluid), ctypes.c_double,
                                             ctypes.POINTER(IbGeometry), ctypes.c_int, ctypes.c_void_p,
                                             ctypes.c_void_p]),
    "ib_bcModeFromString": (ctypes.c_int, [ctypes.c_char_p]),
    "ib_arrayFromGpuTag": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p),
                                          ctypes.POINTER(IbGrid), ctypes.POINTER(ctypes.c_int32),
                                          ctypes.POINTER(ctypes.c_int32)]),
    "ib_fluidFromGpuTags": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_int32),
                                           ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(IbFluid)]),
    "ib_freezeAndPtot": (ctypes.c_int, [ctypes.POINTER(IbFluid), ctypes.c_double, ctypes.c_int,
                                        ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p]),
    "ib_cudaStatics": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(IbGrid), ctypes.POINTER(ctypes.c_int32),
                                      ctypes.c_int, ctypes.c_int, ctypes.POINTER(IbStatics), ctypes.c_int,
                                      ctypes.c_void_p]),
    "ib_setFluidBoundary": (ctypes.c_int, [ctypes.POINTER(IbFluid), ctypes.c_int, ctypes.c_void_p]),
    "ib_cudaSource2FluidDrag": (ctypes.c_int, [ctypes.POINTER(IbFluid), ctypes.POINTER(IbFluid),
                                               ctypes.POINTER(IbThermo), ctypes.POINTER(IbThermo),
                                               ctypes.POINTER(IbGeometry), ctypes.POINTER(ctypes.c_double),
                                               ctypes.c_int, ctypes.c_void_p]),
}

_LIBS = {}
_VARIANT = os.environ.get("IMOGEN_B200_VARIANT", "product")


def library_path(variant=None):
    """Path of the product or strict build; IMOGEN_B200_LIB overrides the product path."""
    variant = variant or _VARIANT
    if variant == "product" and os.environ.get("IMOGEN_B200_LIB"):
        return os.environ["IMOGEN_B200_LIB"]
    name = "libimogen_b200.so" if variant == "product" else "libimogen_b200_strict.so"
    return os.path.join(HERE, name)


def load(variant=None):
    """Load (once) and return the compiled library; raises if it is missing."""
    variant = variant or _VARIANT
    if variant not in _LIBS:
        path = library_path(variant)
        if not os.path.exists(path):
            raise ImportError("libimogen_b200 is not built (%s); run python -m gpuimogen_b200.build" % path)
        L = ctypes.CDLL(path)
        for name, (res, args) in EXPORTS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIBS[variant] = L
    return _LIBS[variant]


def use_variant(variant):
    """Select 'product' (default) or 'strict' (-fmad=false) for subsequent calls."""
    global _VARIANT
    assert variant in ("product", "strict")
    _VARIANT = variant


def _lib():
    return load(_VARIANT)


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _check(where, status):
    if status != SUCCESSFUL:
        raise ImogenError(where, status)


def launch_count():
    """Kernels launched through the library so far in this process."""
    return int(_lib().ib_launch_count())


def device_wait_status(clear=False):
    """0 when no bounded device wait of the TMA-fed sweeps has run out since the last clear."""
    return int(_lib().ib_device_wait_status(1 if clear else 0))


def slab_pitch(nx, ny, nz):
    n = nx * ny * nz
    return ((n + 31) // 32) * 32


# ---------------------------------------------------------------------------------------------
# Host-side objects mirroring FluidManager / GeometryManager
# ---------------------------------------------------------------------------------------------
def _bc_codes(bc):
    if isinstance(bc, str):
        bc = [bc] * 6
    if len(bc) == 2:
        bc = list(bc) * 3
    return [BC[b] if isinstance(b, str) else int(b) for b in bc]


class Fluid:
    """One fluid: a (5, slab_pitch) float64 device tensor [rho, E, px, py, pz], x fastest.

    Mirrors the reference's FluidManager canister (mass, ener, mom(1..3)) plus its boundary
    settings, halo depth and statics lists.
    """

    def __init__(self, shape, bc="circular", halo=4, device="cuda", q=None, statics=None,
                 gamma=5.0 / 3.0, rho_min=1e-5, c_isothermal=-1.0):
        self.shape = tuple(int(s) for s in shape)
        nx, ny, nz = self.shape
        self.slab = slab_pitch(nx, ny, nz)
        if q is None:
            q = torch.zeros((5, self.slab), dtype=torch.float64, device=device)
        assert q.dtype == torch.float64 and q.is_contiguous() and q.shape == (5, self.slab)
        self.q = q
        self.bc = _bc_codes(bc)
        self.halo = halo
        self.statics = statics or [None] * 5  # per slab: (3, n) float64 device tensor or None
        self.gamma = gamma
        self.rho_min = rho_min
        self.c_isothermal = c_isothermal

    @property
    def numel(self):
        nx, ny, nz = self.shape
        return nx * ny * nz

    def field(self, k):
        """View of slab k as a (nz, ny, nx) tensor."""
        nx, ny, nz = self.shape
        return self.q[k, : self.numel].view(nz, ny, nx)

    def set_state(self, rho, E, px, py, pz):
        for k, a in enumerate((rho, E, px, py, pz)):
            t = torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64).reshape(-1))
            self.q[k, : self.numel].copy_(t.to(self.q.device, non_blocking=False))

    def to_numpy(self):
        return self.q.detach().cpu().numpy()

    def c_struct(self):
        f = IbFluid()
        f.q = self.q.data_ptr()
        nx, ny, nz = self.shape
        f.grid = IbGrid(nx, ny, nz, 0, self.slab)
        for i in range(6):
            f.bc[i] = self.bc[i]
        f.halo = self.halo
        for k in range(5):
            s = self.statics[k]
            if s is not None:
                f.statics[k] = IbStatics(s.data_ptr(), s.shape[1], s.shape[1])
        return f

    def thermo(self):
        return IbFluidThermo(self.gamma, self.rho_min, self.c_isothermal)


class Geometry:
    """GeometryManager subset: cell sizes, shape and global resolution.

    Square (default): h = [dx, dy, dz].  Cylindrical (geometryCylindrical, GeometryManager.m:
    300-311): x = r, y = theta, z = z, h = [dr, dtheta, dz] and r_inner = the radius of the centre
    of radial cell 0."""

    def __init__(self, shape, h=None, cylindrical=False, r_inner=0.0):
        self.shape = tuple(int(s) for s in shape)
        if h is None:
            h = [1.0 / s for s in self.shape]
        self.h = [float(x) for x in h]
        self.cylindrical = bool(cylindrical)
        self.r_inner = float(r_inner)

    def c_struct(self):
        g = IbGeometry()
        for i in range(3):
            g.h[i] = self.h[i]
            g.global_rez[i] = self.shape[i]
        g.r_inner = self.r_inner
        g.shape = 1 if self.cylindrical else 0
        return g


FLAG_CYL_GEOMETRIC_RADIUS = 1


def numerics(slope="ospre", fluxlim="ospre", precision="fp64", geometric_radius=False):
    """Numerical switches; geometric_radius: cylindrical theta sweeps use the cell centre radius
    instead of the reference's radius arithmetic."""
    return IbNumerics(SLOPE[slope] if isinstance(slope, str) else slope,
                      FLUXLIM[fluxlim] if isinstance(fluxlim, str) else fluxlim,
                      PRECISION[precision] if isinstance(precision, str) else precision,
                      FLAG_CYL_GEOMETRIC_RADIUS if geometric_radius else 0)


def _dvec(params):
    arr = (ctypes.c_double * len(params))(*[float(p) for p in params])
    return arr, len(params)


# ---------------------------------------------------------------------------------------------
# mex-form entry points
# ---------------------------------------------------------------------------------------------
def cudaFluidStep(fluid, geometry, params, num=None):
    """cudaFluidStep([dt, purehydro, gamma, rho_min, method, direction (, c_iso)], fluid, geometry)."""
    f = fluid.c_struct()
    g = geometry.c_struct()
    p, n = _dvec(params)
    nm = ctypes.byref(num) if num is not None else None
    _check("ib_cudaFluidStep", _lib().ib_cudaFluidStep(ctypes.byref(f), ctypes.byref(g), p, n, nm, _stream()))


def fluidstep(fluids, geometry, params, num=None):
    """fluidstep(fluids, [dt, purehydro, +1|-1, iteration, method], geometry)."""
    if isinstance(fluids, Fluid):
        fluids = [fluids]
    fs = (IbFluid * len(fluids))(*[f.c_struct() for f in fluids])
    th = (IbFluidThermo * len(fluids))(*[f.thermo() for f in fluids])
    g = geometry.c_struct()
    p, n = _dvec(params)
    nm = ctypes.byref(num) if num is not None else None
    _check("ib_fluidstep", _lib().ib_fluidstep(fs, th, len(fluids), ctypes.byref(g), p, n, nm, _stream()))


def completeTimestep(fluids, geometry, params, num=None, drag=None):
    """performCompleteTimestep(fluids, [dt, purehydro, iteration, method]): source half step,
    forward fluid step, source step, backward fluid step, source half step.  drag = (thermo_gas,
    thermo_dust, method) makes fluids [gas, dust] exchange momentum by the two-fluid drag; without
    it there is no source and the two same-axis sweeps mid-step run as one launch where they can."""
    if isinstance(fluids, Fluid):
        fluids = [fluids]
    fs = (IbFluid * len(fluids))(*[f.c_struct() for f in fluids])
    th = (IbFluidThermo * len(fluids))(*[f.thermo() for f in fluids])
    g = geometry.c_struct()
    p, n = _dvec(params)
    nm = ctypes.byref(num) if num is not None else None
    ds = None
    if drag is not None:
        tg, td, method = drag
        ds = ctypes.byref(IbDragSource(thermo_struct(tg), thermo_struct(td),
                                       DRAG[method] if isinstance(method, str) else int(method), 0))
    _check("ib_completeTimestep", _lib().ib_completeTimestep(fs, th, len(fluids), ctypes.byref(g), p, n, nm, ds,
                                                             _stream()))


def _drag_struct(drag):
    if drag is None:
        return None
    tg, td, method = drag
    return IbDragSource(thermo_struct(tg), thermo_struct(td), DRAG[method] if isinstance(method, str) else int(method),
                        0)


def completeTimestepDeviceDt(fluids, geometry, dt_device, params, num=None, drag=None):
    """completeTimestep with the timestep read by the kernels from device memory (dt_device: a
    device address, e.g. of an ib_time_state's dt); params = [purehydro, iteration, method]."""
    if isinstance(fluids, Fluid):
        fluids = [fluids]
    fs = (IbFluid * len(fluids))(*[f.c_struct() for f in fluids])
    th = (IbFluidThermo * len(fluids))(*[f.thermo() for f in fluids])
    g = geometry.c_struct()
    p, n = _dvec(params)
    nm = ctypes.byref(num) if num is not None else None
    ds = _drag_struct(drag)
    _check("ib_completeTimestepDeviceDt", _lib().ib_completeTimestepDeviceDt(
        fs, th, len(fluids), ctypes.byref(g), ctypes.c_void_p(int(dt_device)), p, n, nm,
        ctypes.byref(ds) if ds is not None else None, _stream()))


def timeUpdate(ts_device):
    _check("ib_timeUpdate", _lib().ib_timeUpdate(ctypes.c_void_p(int(ts_device)), _stream()))


def timeAdvance(ts_device):
    _check("ib_timeAdvance", _lib().ib_timeAdvance(ctypes.c_void_p(int(ts_device)), _stream()))


def cudaSoundspeed(fluid, gamma):
    cs = torch.empty(fluid.numel, dtype=torch.float64, device=fluid.q.device)
    f = fluid.c_struct()
    _check("ib_cudaSoundspeed", _lib().ib_cudaSoundspeed(ctypes.byref(f), float(gamma), cs.data_ptr(), _stream()))
    return cs


def cflTimestep(fluid, cs, geometry, method):
    """tau = cflTimestep(fluid, soundspeed, geometry, method); already halved for HLL/HLLC."""
    f = fluid.c_struct()
    g = geometry.c_struct()
    tau = ctypes.c_double(0.0)
    _check("ib_cflTimestep", _lib().ib_cflTimestep(ctypes.byref(f), cs.data_ptr(), ctypes.byref(g), int(method),
                                                   ctypes.byref(tau), _stream()))
    return tau.value


def cflTimestepFused(fluid, gamma, geometry, method, tau_device=None):
    """Soundspeed + CFL in one pass.  With tau_device (a 1-element float64 tensor) nothing is
    synchronised and the value is left on the device."""
    f = fluid.c_struct()
    g = geometry.c_struct()
    if tau_device is not None:
        _check("ib_cflTimestepFused", _lib().ib_cflTimestepFused(ctypes.byref(f), float(gamma), ctypes.byref(g),
                                                                 int(method), None, tau_device.data_ptr(), _stream()))
        return tau_device
    tau = ctypes.c_double(0.0)
    _check("ib_cflTimestepFused", _lib().ib_cflTimestepFused(ctypes.byref(f), float(gamma), ctypes.byref(g),
                                                             int(method), ctypes.byref(tau), None, _stream()))
    return tau.value


def freezeAndPtot(fluid, gamma, purehydro, cs_min):
    """[Ptot, Cfreeze] = freezeAndPtot(...); floors E in place where c_s < cs_min."""
    nx, ny, nz = fluid.shape
    ptot = torch.empty(fluid.numel, dtype=torch.float64, device=fluid.q.device)
    freeze = torch.empty(ny * nz, dtype=torch.float64, device=fluid.q.device)
    f = fluid.c_struct()
    _check("ib_freezeAndPtot", _lib().ib_freezeAndPtot(ctypes.byref(f), float(gamma), int(purehydro), float(cs_min),
                                                       ptot.data_ptr(), freeze.data_ptr(), _stream()))
    return ptot, freeze


def cudaStatics(fluid, slab_index, direction, vector_component=None):
    """cudaStatics(ImogenArray, blockdim, geometry, direction) for slab `slab_index` of a fluid
    (0 = mass ... 4 = mom(3)); vector_component defaults to the slab's momentum component."""
    if vector_component is None:
        vector_component = slab_index - 1 if slab_index >= 2 else 0
    nx, ny, nz = fluid.shape
    grid = IbGrid(nx, ny, nz, 0, fluid.slab)
    bc = (ctypes.c_int32 * 6)(*fluid.bc)
    st = fluid.statics[slab_index]
    stc = IbStatics(st.data_ptr(), st.shape[1], st.shape[1]) if st is not None else IbStatics(None, 0, 0)
    ptr = fluid.q.data_ptr() + 8 * slab_index * fluid.slab
    _check("ib_cudaStatics", _lib().ib_cudaStatics(ctypes.c_void_p(ptr), ctypes.byref(grid), bc, fluid.halo,
                                                   int(vector_component), ctypes.byref(stc), int(direction),
                                                   _stream()))


def setFluidBoundary(fluid, direction):
    f = fluid.c_struct()
    _check("ib_setFluidBoundary", _lib().ib_setFluidBoundary(ctypes.byref(f), int(direction), _stream()))


def thermo_struct(t):
    """t: dict or sequence [gamma, mass, mu0, muTindex, sigma0, sigmaTindex, kBolt, Cisothermal]."""
    if isinstance(t, dict):
        t = [t[k] for k in ("gamma", "mass", "dynViscosity", "viscTindex", "sigma", "sigmaTindex",
                            "kBolt", "Cisothermal")]
    return IbThermo(*[float(v) for v in t])


def cudaSource2FluidDrag(gas, dust, thermo_gas, thermo_dust, geometry, params):
    """cudaSource2FluidDrag(FluidManager[gas dust], geometry, [dt, method])."""
    fg, fd = gas.c_struct(), dust.c_struct()
    tg, td = thermo_struct(thermo_gas), thermo_struct(thermo_dust)
    g = geometry.c_struct()
    p, n = _dvec(params)
    _check("ib_cudaSource2FluidDrag", _lib().ib_cudaSource2FluidDrag(ctypes.byref(fg), ctypes.byref(fd),
                                                                     ctypes.byref(tg), ctypes.byref(td),
                                                                     ctypes.byref(g), p, n, _stream()))
