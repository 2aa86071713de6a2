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
               if os.path.basename(p) not in ("cfl.npz", "drag.npz"))


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
