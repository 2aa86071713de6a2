"""GPU parity of the fused directional sweeps against the CPU oracle.

The strict build (-fmad=false) must reproduce the oracle bit for bit; the product build (FMA
contraction) must agree to 1e-12 relative per cell after one sweep.  The oracle restates
cukern_HLLC_2ndorder / cukern_HLL_step / cukern_XinJinHydro_step (gpuclass/cudaFluidStep.cu)
one pencil at a time with periodic wrap, as the reference kernels compute each row."""
import numpy as np
import pytest

from gpuimogen_b200 import problems
from helpers import bits_equal, first_diff, host, product_close, to_fluid

pytestmark = pytest.mark.gpu

SHAPES = [
    (37, 11, 9),     # x: row kernel, 1 cell/thread; y,z: tile kernel (odd nx), single chunk
    (600, 5, 4),     # x: row kernel, 2 cells/thread; y,z: TMA pipeline (pencils below 64 cells)
    (1100, 3, 4),    # x: chunked TMA pipeline (rows > 1024); y: 3-cell pencils
    (8, 300, 6),     # y: TMA pipeline, pencils of 257-512 cells (two box rows, 2 cells/thread)
    (6, 7, 130),     # z: pencil-pair kernel, 130-cell pencils
    (5, 4, 3),       # tiny pencils; y,z: tile kernel
    (8, 140, 3),     # y: pencil-pair kernels (HLL/HLLC, Xin-Jin) of 129-256 cells
    (4, 3, 200),     # z: the same
    (160, 3, 2),     # x: HLLC rows of 129-255 cells, planes of a fixed 256-cell stride
    (96, 100, 90),   # x, y, z: HLLC rows and pencils of 65-127 cells, planes of a 128-cell stride
    (300, 4, 3),     # x: HLLC rows of 257-511 cells, planes of a 512-cell stride
]


def _state(shape, seed):
    return problems.random_jumpy(shape, gamma=1.4, seed=seed) if seed % 2 else \
        problems.random_smooth(shape, gamma=1.4, seed=seed, amp=0.3)


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("method", [2, 1, 3])
@pytest.mark.parametrize("direction", [1, 2, 3])
def test_sweep_strict_bitexact(cuda, ib, po, shape, method, direction):
    if shape[direction - 1] < 3:
        pytest.skip("sweep not performed below 3 cells")
    n = shape[0] * shape[1] * shape[2]
    for seed in (1, 2):
        q = _state(shape, seed + 10 * direction + 100 * method)
        h = (0.05, 0.04, 0.03)
        dt = 4e-3
        ref = q.copy()
        sp = po.step_params(dt, h, 1.4, rho_min=1e-5, method=method, slope="ospre")
        po.fluid_sweep(ref, shape, sp, direction)
        ib.use_variant("strict")
        try:
            fl = to_fluid(q, shape)
            geo = ib.Geometry(shape, h)
            ib.cudaFluidStep(fl, geo, [dt, 1, 1.4, 1e-5, method, direction])
            out = host(fl)
        finally:
            ib.use_variant("product")
        assert bits_equal(out, ref, n), first_diff(out, ref, n)
        fl = to_fluid(q, shape)
        ib.cudaFluidStep(fl, ib.Geometry(shape, h), [dt, 1, 1.4, 1e-5, method, direction])
        ok, info = product_close(host(fl), ref, n)
        assert ok, info


@pytest.mark.parametrize("slope", ["ospre", "mc", "vanleer", "minmod", "superbee", "vanalbada", "zero"])
@pytest.mark.parametrize("method", [2, 1])
def test_all_slope_limiters_strict(cuda, ib, po, slope, method):
    shape = (40, 24, 20)
    n = 40 * 24 * 20
    q = problems.random_jumpy(shape, seed=5)
    h = (0.05, 0.05, 0.05)
    for direction in (1, 2, 3):
        ref = q.copy()
        po.fluid_sweep(ref, shape, po.step_params(3e-3, h, 1.4, method=method, slope=slope), direction)
        ib.use_variant("strict")
        try:
            fl = to_fluid(q, shape)
            ib.cudaFluidStep(fl, ib.Geometry(shape, h), [3e-3, 1, 1.4, 1e-5, method, direction],
                             ib.numerics(slope=slope))
            out = host(fl)
        finally:
            ib.use_variant("product")
        assert bits_equal(out, ref, n), (direction, first_diff(out, ref, n))


@pytest.mark.parametrize("fluxlim", ["ospre", "vanleer", "minmod", "superbee", "zero"])
def test_xinjin_flux_limiters_strict(cuda, ib, po, fluxlim):
    shape = (64, 12, 10)
    n = 64 * 12 * 10
    q = problems.random_smooth(shape, seed=9, amp=0.4)
    h = (0.02, 0.03, 0.04)
    for direction in (1, 2, 3):
        ref = q.copy()
        po.fluid_sweep(ref, shape, po.step_params(2e-3, h, 1.4, method=3, fluxlim=fluxlim), direction)
        ib.use_variant("strict")
        try:
            fl = to_fluid(q, shape)
            ib.cudaFluidStep(fl, ib.Geometry(shape, h), [2e-3, 1, 1.4, 1e-5, 3, direction],
                             ib.numerics(fluxlim=fluxlim))
            out = host(fl)
        finally:
            ib.use_variant("product")
        assert bits_equal(out, ref, n), (direction, first_diff(out, ref, n))


def test_hll_isothermal_and_floors_strict(cuda, ib, po):
    """Isothermal HLL (7-element parameter vector: gamma := 2, cudaFluidStep.cu:184-189) and the
    density/energy floors of cukern_PressureSolverHydro on a state that violates them."""
    shape = (48, 10, 6)
    n = 48 * 10 * 6
    q = problems.random_jumpy(shape, seed=13)
    q[0, :n:7] = 1e-7                    # below rho_min -> rescaled
    q[1, 3:n:11] = 0.5 * (q[2, 3:n:11] ** 2 + q[3, 3:n:11] ** 2 + q[4, 3:n:11] ** 2) / q[0, 3:n:11]
    h = (0.05, 0.05, 0.05)
    for direction in (1, 2, 3):
        for params, sp in (
            ([3e-3, 1, 1.4, 1e-5, 1, direction, 0.3], po.step_params(3e-3, h, 2.0, 1e-5, 0.3, method=1)),
            ([3e-3, 1, 1.4, 1e-5, 1, direction], po.step_params(3e-3, h, 1.4, 1e-5, -1, method=1)),
        ):
            ref = q.copy()
            po.fluid_sweep(ref, shape, sp, direction)
            ib.use_variant("strict")
            try:
                fl = to_fluid(q, shape)
                ib.cudaFluidStep(fl, ib.Geometry(shape, h), params)
                out = host(fl)
            finally:
                ib.use_variant("product")
            assert bits_equal(out, ref, n), (direction, len(params), first_diff(out, ref, n))


@pytest.mark.parametrize("direction", [1, 2])
def test_xinjin_tiny_momenta_stay_finite(cuda, ib, po, direction):
    """Momenta near 1e-154 next to exact zeros (as the outflow boundary's transverse momentum
    leaves them while it decays into the grid) make the Xin-Jin flux limiter's denominators
    subnormal: the product build's shared reciprocal must not turn 0 / d into 0 * inf."""
    n = 64
    shape = (n, 1, 1) if direction == 1 else (4, n, 1)
    N = shape[0] * shape[1]
    q = problems.sod(N)
    q[:, :N] = 0
    q[0, :N] = 1.0
    q[1, :N] = 2.5
    tiny = np.zeros(n)
    tiny[10:20] = 1e-150 * 10.0 ** (-2.0 * np.arange(10))   # 1e-150 ... 1e-168, then zeros
    slab = 3 if direction == 1 else 2                       # a transverse momentum
    q[slab, :N] = np.tile(tiny, N // n) if direction == 1 else np.repeat(tiny, shape[0])
    geo = ib.Geometry(shape)
    sp = po.step_params(1e-4, geo.h, 1.4, method=3)
    ref = q.copy()
    po.fluid_sweep(ref, shape, sp, direction)
    assert np.all(np.isfinite(ref[:, :N]))
    for variant in ("product", "strict"):
        fl = to_fluid(q.copy(), shape, gamma=1.4)
        ib.use_variant(variant)
        try:
            ib.cudaFluidStep(fl, geo, [1e-4, 1, 1.4, 1e-5, 3, direction])
        finally:
            ib.use_variant("product")
        out = host(fl)
        assert np.all(np.isfinite(out[:, :N])), variant
        assert np.allclose(out[:, :N], ref[:, :N], rtol=1e-12, atol=1e-300), variant


@pytest.mark.parametrize("shape,direction", [((4, 256, 5), 2), ((2, 5, 512), 3), ((6, 512, 2), 2), ((10, 4, 256), 3),
                                             ((256, 3, 4), 1), ((200, 3, 2), 1), ((96, 5, 2), 1)])
def test_xinjin_pencil_boxes_fixed_lengths(cuda, ib, po, shape, direction):
    """Xin-Jin y/z sweeps of 256- and 512-cell pencils go through the TMA pencil-box kernel's
    fixed-length forms (a 512-cell pencil as two box rows of 256), x rows of 64-256 cells through
    its one-row boxes (256 cells: fixed length; 129-255: the fixed plane stride; up to 128: the
    row length): bit for bit the oracle's."""
    n = shape[0] * shape[1] * shape[2]
    q = problems.random_jumpy(shape, gamma=1.4, seed=17)
    h = (0.05, 0.04, 0.03)
    ref = q.copy()
    po.fluid_sweep(ref, shape, po.step_params(2e-3, h, 1.4, method=3), direction)
    ib.use_variant("strict")
    try:
        fl = to_fluid(q, shape)
        ib.cudaFluidStep(fl, ib.Geometry(shape, h), [2e-3, 1, 1.4, 1e-5, 3, direction])
        out = host(fl)
    finally:
        ib.use_variant("product")
    assert bits_equal(out, ref, n), first_diff(out, ref, n)
    assert ib.device_wait_status() == 0
