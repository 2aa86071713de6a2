"""CPU-only checks of the C ABI: both builds load, export every entry point that
include/imogen_b200.h declares, and reject malformed calls before touching a device
(the reference's mex functions reject them the same way: cudaFluidStep.cu:167-171,
flux_ML_iface.cu:56-58, cudaSource2FluidDrag.cu:157-163)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "imogen_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"IB_API\s+[\w\s\*]+?\b(ib_\w+)\s*\(", text)))


@pytest.mark.parametrize("variant", ["product", "strict"])
def test_library_exports_every_declared_symbol(variant):
    from gpuimogen_b200 import imogen
    path = imogen.library_path(variant)
    assert os.path.exists(path), "build the library first: python -m gpuimogen_b200.build"
    lib = ctypes.CDLL(path)
    syms = declared_symbols()
    assert len(syms) >= 12
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(imogen.EXPORTS)


def test_status_strings_and_pitch():
    from gpuimogen_b200 import imogen
    L = imogen.load("product")
    assert L.ib_status_string(0) == b"SUCCESSFUL"
    assert L.ib_status_string(-100) == b"ERROR_INVALID_ARGS"
    assert L.ib_status_string(-105) == b"ERROR_NOIMPLEMENT"
    assert L.ib_slab_pitch(256, 256, 256) == 256 ** 3
    assert L.ib_slab_pitch(17, 3, 1) == 64
    assert L.ib_slab_pitch(1, 1, 1) == 32


def _fluid(imogen, shape=(16, 8, 4)):
    f = imogen.IbFluid()
    f.q = 0x10000  # never dereferenced: every call below fails validation first
    nx, ny, nz = shape
    f.grid = imogen.IbGrid(nx, ny, nz, 0, imogen.slab_pitch(nx, ny, nz))
    f.halo = 4
    return f


def test_invalid_calls_rejected_without_device():
    from gpuimogen_b200 import imogen
    L = imogen.load("product")
    geo = imogen.IbGeometry()
    geo.h[0] = geo.h[1] = geo.h[2] = 0.1
    f = _fluid(imogen)
    p = (ctypes.c_double * 6)(1e-3, 1, 1.4, 1e-5, 2, 1)
    # wrong parameter count
    assert L.ib_cudaFluidStep(ctypes.byref(f), ctypes.byref(geo), p, 5, None, None) == -100
    # bad method / direction
    for bad in ((1e-3, 1, 1.4, 1e-5, 4, 1), (1e-3, 1, 1.4, 1e-5, 2, 4)):
        pb = (ctypes.c_double * 6)(*bad)
        assert L.ib_cudaFluidStep(ctypes.byref(f), ctypes.byref(geo), pb, 6, None, None) == -100
    # MHD and shapes other than square and cylindrical are not built
    pm = (ctypes.c_double * 6)(1e-3, 0, 1.4, 1e-5, 2, 1)
    assert L.ib_cudaFluidStep(ctypes.byref(f), ctypes.byref(geo), pm, 6, None, None) == -105
    geo2 = imogen.IbGeometry()
    geo2.shape = 2
    assert L.ib_cudaFluidStep(ctypes.byref(f), ctypes.byref(geo2), p, 6, None, None) == -105
    # cylindrical: the theta layout parameter is 0 or 1; unknown numerics flags are rejected
    geo3 = imogen.IbGeometry()
    geo3.shape = 1
    p8 = (ctypes.c_double * 8)(1e-3, 1, 1.4, 1e-5, 2, 2, -1, 2)
    assert L.ib_cudaFluidStep(ctypes.byref(f), ctypes.byref(geo3), p8, 8, None, None) == -100
    assert L.ib_cudaFluidStep(ctypes.byref(f), ctypes.byref(geo3), p, 9, None, None) == -100
    nmf = imogen.IbNumerics(0, 0, 0, 4)
    assert L.ib_cudaFluidStep(ctypes.byref(f), ctypes.byref(geo3), p, 6, ctypes.byref(nmf), None) == -100
    # null pointers
    assert L.ib_cudaFluidStep(None, ctypes.byref(geo), p, 6, None, None) == -102
    f0 = _fluid(imogen)
    f0.q = None
    assert L.ib_cudaFluidStep(ctypes.byref(f0), ctypes.byref(geo), p, 6, None, None) == -102
    # bad grid: pitch smaller than numel
    fb = _fluid(imogen)
    fb.grid.slab_pitch = 10
    assert L.ib_cudaFluidStep(ctypes.byref(fb), ctypes.byref(geo), p, 6, None, None) == -100
    # bad boundary mode and numerics
    fc = _fluid(imogen)
    fc.bc[0] = 9
    assert L.ib_cudaFluidStep(ctypes.byref(fc), ctypes.byref(geo), p, 6, None, None) == -100
    nm = imogen.IbNumerics(17, 0, 0, 0)
    assert L.ib_cudaFluidStep(ctypes.byref(f), ctypes.byref(geo), p, 6, ctypes.byref(nm), None) == -100
    # fluidstep parameter vector has 5 entries
    th = imogen.IbFluidThermo(1.4, 1e-5, -1)
    p4 = (ctypes.c_double * 4)(1e-3, 1, 1, 0)
    assert L.ib_fluidstep(ctypes.byref(f), ctypes.byref(th), 1, ctypes.byref(geo), p4, 4, None, None) == -100
    # drag parameter vector has 2 entries, methods 0..5
    tg = imogen.IbThermo()
    pd = (ctypes.c_double * 3)(1e-3, 4, 0)
    assert L.ib_cudaSource2FluidDrag(ctypes.byref(f), ctypes.byref(f), ctypes.byref(tg), ctypes.byref(tg),
                                     ctypes.byref(geo), pd, 3, None) == -100
    pd2 = (ctypes.c_double * 2)(1e-3, 6)
    assert L.ib_cudaSource2FluidDrag(ctypes.byref(f), ctypes.byref(f), ctypes.byref(tg), ctypes.byref(tg),
                                     ctypes.byref(geo), pd2, 2, None) == -100
    # ETDRK2 differentiates the pressure: it needs the geometry, and square cells
    pe = (ctypes.c_double * 2)(1e-3, 3)
    assert L.ib_cudaSource2FluidDrag(ctypes.byref(f), ctypes.byref(f), ctypes.byref(tg), ctypes.byref(tg),
                                     None, pe, 2, None) == -102
    assert L.ib_cudaSource2FluidDrag(ctypes.byref(f), ctypes.byref(f), ctypes.byref(tg), ctypes.byref(tg),
                                     ctypes.byref(geo2), pe, 2, None) == -105
    # cudaStatics direction and vector component
    grid = imogen.IbGrid(16, 8, 4, 0, 512)
    bc = (ctypes.c_int32 * 6)(0, 0, 0, 0, 0, 0)
    assert L.ib_cudaStatics(ctypes.c_void_p(0x10000), ctypes.byref(grid), bc, 4, 0, None, 0, None) == -100
    assert L.ib_cudaStatics(ctypes.c_void_p(0x10000), ctypes.byref(grid), bc, 4, 5, None, 1, None) == -100
