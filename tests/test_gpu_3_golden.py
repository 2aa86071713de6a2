"""The library against golden vectors from the reference's own GPU code (tests/golden/).

Strict build vs the reference built with -fmad=false: bit for bit.  Product build vs the reference
as it builds itself: within 1e-12 relative L1 per field after the case's iterations."""
import glob
import json
import os

import numpy as np
import pytest

from helpers import bits_equal, first_diff, host, rel_l1, to_fluid

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FLUID = sorted(p for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
               if os.path.basename(p) not in ("cfl.npz", "drag.npz", "drag_etdrk2.npz", "cylindrical.npz"))


def run_library(ib, meta, q):
    shape = tuple(meta["shape"])
    fl = to_fluid(q, shape, bc=meta["bc"], gamma=meta["gamma"], rho_min=meta["rho_min"], c_iso=meta["c_iso"])
    geo = ib.Geometry(shape)
    tm = ib.TimeManager(cfl=meta["cfl"])
    dts = []
    num = ib.numerics(slope=meta["limiter"])
    for _ in range(meta["niter"]):
        dts.append(ib.run_iteration([fl], geo, tm, meta["method"], num))
    return host(fl), np.array(dts)


@pytest.mark.parametrize("path", FLUID, ids=[os.path.basename(p)[:-4] for p in FLUID])
def test_library_matches_reference_gpu(cuda, ib, path):
    z = np.load(path)
    meta = json.loads(str(z["meta"]))
    shape = tuple(meta["shape"])
    n = shape[0] * shape[1] * shape[2]
    ib.use_variant("strict")
    try:
        out, dts = run_library(ib, meta, np.array(z["input"]))
    finally:
        ib.use_variant("product")
    assert np.array_equal(dts, z["dts_strict"])
    assert bits_equal(out, z["out_strict"], n), first_diff(out, z["out_strict"], n)
    out, dts = run_library(ib, meta, np.array(z["input"]))
    err = rel_l1(out, z["out_fast"], n)
    assert np.all(err <= 1e-12), err


@pytest.mark.parametrize("case", ["", "stiff_"])
@pytest.mark.parametrize("shape", [(16, 8, 1), (8, 6, 5), (12, 1, 6), (32, 1, 1)], ids=lambda s: "%dx%dx%d" % s)
def test_library_etdrk2_matches_reference_gpu(cuda, ib, shape, case):
    """ETDRK2 through the C ABI against the reference's own kernels on the same states.  exp,
    expm1 and pow are CUDA's in both, so the strict build is compared within rounding of the
    transcendental arguments only: relative L1 <= 1e-13 per field (1e-12 for the product build)."""
    z = np.load(os.path.join(GOLDEN, "drag_etdrk2.npz"))
    meta = json.loads(str(z["meta"]))
    key = "%dx%dx%d" % shape
    n = shape[0] * shape[1] * shape[2]
    td = meta["td_stiff"] if case else meta["td"]
    for variant, tag, tol in (("strict", "strict", 1e-13), ("product", "fast", 1e-12)):
        fg = to_fluid(np.array(z["gas_" + key]), shape)
        fd = to_fluid(np.array(z["dust_" + key]), shape)
        ib.use_variant(variant)
        try:
            ib.cudaSource2FluidDrag(fg, fd, meta["tg"], td, ib.Geometry(shape), [meta["dt"], 3])
        finally:
            ib.use_variant("product")
        for mine, ref in ((host(fg), z["gas_out_%s%s_%s" % (case, key, tag)]),
                          (host(fd), z["dust_out_%s%s_%s" % (case, key, tag)])):
            err = rel_l1(mine, ref, n)
            assert np.all(err <= tol), (variant, err)
