"""Failure detection of the TMA-fed sweep kernels, without a GPU fault.

Every wait of these kernels for a tile is bounded; one that runs out makes the kernel wait (with
the full limit) for the copies it has issued, leave, and set the flag ib_device_wait_status reads.
ib_setTileWaitLimit(0) makes every tile wait give up at once while the copies complete normally,
so the drain path runs on valid loads.  For each TMA kernel family (pencil-pair kernel with 2- and
4-pencil boxes, wide-block pipeline, persistent pencil pipeline, chunked pipeline) the test checks
that the call returns, that the status reports the run-out, that the sweep left the state
untouched (no tile was computed or stored), and that after the limit is restored and the flag
cleared the same sweep is correct again.
"""
import numpy as np
import pytest

from gpuimogen_b200 import problems
from helpers import host, product_close, to_fluid

pytestmark = pytest.mark.gpu

CASES = [
    ((64, 64, 64), 2, "fp64"),       # y: pencil-pair kernel (2-pencil boxes)
    ((512, 512, 8), 3, "fp64"),      # z of 2 MB planes: pencil-pair kernel with 4-pencil boxes
    ((512, 512, 8), 3, "fp32flux"),  # the same in FP32 flux: wide-block pipeline (8-column boxes)
    ((8, 300, 6), 2, "fp64"),        # y pencils of 257-511 cells: persistent pencil pipeline
    ((8, 600, 4), 2, "fp64"),        # y pencils above 512 cells: chunked pipeline
]


@pytest.mark.parametrize("shape,direction,precision", CASES, ids=lambda v: str(v))
def test_tile_wait_runs_out_and_recovers(cuda, ib, po, shape, direction, precision):
    L = ib.load("product")
    n = shape[0] * shape[1] * shape[2]
    q0 = problems.random_smooth(shape, gamma=1.4, seed=5, amp=0.3)
    geo = ib.Geometry(shape)
    num = ib.numerics(slope="mc", precision=precision)
    params = [2e-4, 1, 1.4, 1e-5, 2, direction]
    assert ib.device_wait_status(clear=True) in (0, 1)
    assert ib.device_wait_status() == 0
    fl = to_fluid(q0.copy(), shape, gamma=1.4)
    try:
        assert L.ib_setTileWaitLimit(0) == 0
        ib.cudaFluidStep(fl, geo, params, num)   # returns; the kernel leaves early
        assert ib.device_wait_status() == 1
        out = host(fl)
        assert np.array_equal(out[:, :n], q0[:, :n])   # no tile was computed or stored
    finally:
        L.ib_setTileWaitLimit(-1)
    assert ib.device_wait_status(clear=True) == 1
    assert ib.device_wait_status() == 0
    # the next call is a normal, correct sweep
    ib.cudaFluidStep(fl, geo, params, num)
    out = host(fl)
    assert ib.device_wait_status() == 0
    ref = q0.copy()
    sp = po.step_params(2e-4, geo.h, 1.4, method=2, slope="mc")
    po.fluid_sweep(ref, shape, sp, direction)
    if precision == "fp64":
        ok, info = product_close(out, ref, n)
    else:   # FP32 flux arithmetic: within the form's stated 1e-5 relative L1
        ok, info = product_close(out, ref, n, l1=1e-5, scale=1e-4)
    assert ok, info


def test_xinjin_tile_wait_runs_out_and_recovers(cuda, ib, po):
    """The same for the Xin-Jin pencil-box kernel (y sweep of 64-cell pencils)."""
    L = ib.load("product")
    shape = (64, 64, 16)
    n = shape[0] * shape[1] * shape[2]
    q0 = problems.random_smooth(shape, gamma=1.4, seed=6, amp=0.3)
    geo = ib.Geometry(shape)
    params = [2e-4, 1, 1.4, 1e-5, 3, 2]
    ib.device_wait_status(clear=True)
    fl = to_fluid(q0.copy(), shape, gamma=1.4)
    try:
        assert L.ib_setTileWaitLimit(0) == 0
        ib.cudaFluidStep(fl, geo, params)
        assert ib.device_wait_status() == 1
        assert np.array_equal(host(fl)[:, :n], q0[:, :n])
    finally:
        L.ib_setTileWaitLimit(-1)
    assert ib.device_wait_status(clear=True) == 1
    ib.cudaFluidStep(fl, geo, params)
    assert ib.device_wait_status() == 0
    ref = q0.copy()
    po.fluid_sweep(ref, shape, po.step_params(2e-4, geo.h, 1.4, method=3), 2)
    ok, info = product_close(host(fl), ref, n)
    assert ok, info
