"""GPU tests of ib_completeTimestep (performCompleteTimestep, gpuclass/flux_multi.cu:174-272).

Without a source the forward step's last sweep and the backward step's first are along the same
axis (the backward order is the forward one reversed) and run as one double-sweep launch where
the boundary between them is periodic.  That must give the same bits as the reference's two
fluidstep calls (ib_fluidstep +1 then -1), in both builds, for every kernel family the double
sweep goes through: the row kernel (x), the pencil-pair kernel and the TMA pencil pipeline (y, z),
the kernels of z sweeps of large x-y planes (4-pencil boxes in FP64, the wide-block pipeline in
FP32 flux), the chunked pipeline and the tile kernel (which run the sweep twice), the 1-D shortcut
and the FP32-flux form.  Six iterations put the middle pair on x, y, x, y, z, z.

With the two-fluid drag as the source, the composition drag(dt/2), forward, drag(dt), backward,
drag(dt/2) is checked against the same composition of the CPU oracle.
"""
import numpy as np
import pytest
import torch

from gpuimogen_b200 import dusty, problems
from helpers import bits_equal, first_diff, host, product_close, to_fluid

pytestmark = pytest.mark.gpu

CASES = [
    # shape, method, precision
    ((24, 20, 16), 2, "fp64"),    # x row kernel, y/z pencil pipeline
    ((24, 20, 16), 1, "fp64"),    # HLL: floors in both stages of each sweep
    ((24, 20, 16), 2, "fp32flux"),
    ((37, 11, 9), 2, "fp64"),     # odd nx: y/z through the tile kernel (twice)
    ((1100, 4, 5), 2, "fp64"),    # x rows above 1024 cells: chunked pipeline (twice)
    ((8, 600, 4), 2, "fp64"),     # y pencils above 512 cells: chunked pipeline
    ((300, 1, 1), 2, "fp64"),     # 1-D: forward x, backward x
    ((64, 48, 1), 3, "fp64"),     # Xin-Jin: two launches for the pair
]


def _run_pair(ib, shape, method, precision, variant, iters=6, bc="circular"):
    q = problems.random_smooth(shape, gamma=1.4, seed=11, amp=0.3) if method != 1 else \
        problems.random_jumpy(shape, gamma=1.4, seed=12)
    num = ib.numerics(slope="mc", precision=precision)
    geo = ib.Geometry(shape)
    ib.use_variant(variant)
    try:
        a = to_fluid(q.copy(), shape, bc=bc, gamma=1.4)
        b = to_fluid(q.copy(), shape, bc=bc, gamma=1.4)
        for it in range(iters):
            dt_a = 0.4 * ib.cflTimestepFused(a, 1.4, geo, method)
            dt_b = 0.4 * ib.cflTimestepFused(b, 1.4, geo, method)
            assert dt_a == dt_b, (it, dt_a, dt_b)
            ib.completeTimestep([a], geo, [dt_a, 1, it, method], num)
            ib.fluidstep([b], geo, [dt_b, 1, 1, it, method], num)
            ib.fluidstep([b], geo, [dt_b, 1, -1, it, method], num)
    finally:
        ib.use_variant("product")
    return host(a), host(b), q


@pytest.mark.parametrize("variant", ["product", "strict"])
@pytest.mark.parametrize("shape,method,precision", CASES, ids=lambda v: str(v))
def test_complete_step_equals_two_fluidsteps(cuda, ib, shape, method, precision, variant):
    n = shape[0] * shape[1] * shape[2]
    qa, qb, q0 = _run_pair(ib, shape, method, precision, variant)
    assert bits_equal(qa, qb, n), first_diff(qa, qb, n)
    assert not np.array_equal(qa[:, :n], q0[:, :n])


def test_complete_step_wide_planes(cuda, ib):
    """z sweeps of x-y planes above 1 MB: FP64 through the pencil-pair kernel with 4-pencil boxes,
    FP32 flux through the wide-block pipeline (8-column boxes computed 4 at a time, results stored
    from the input tile); iterations 4 and 5 put the middle pair on z."""
    shape = (512, 512, 8)
    n = shape[0] * shape[1] * shape[2]
    for precision in ("fp32flux", "fp64"):
        qa, qb, _ = _run_pair(ib, shape, 2, precision, "product", iters=6)
        assert bits_equal(qa, qb, n), (precision, first_diff(qa, qb, n))


def test_complete_step_nonperiodic_middle_axis_unfused(cuda, ib):
    """Const boundaries on x: the fill between the two x sweeps does work, so they stay separate
    launches; the result is still the two fluidstep calls'."""
    shape = (24, 20, 16)
    n = shape[0] * shape[1] * shape[2]
    bc = ["const", "const", "circular", "circular", "mirror", "mirror"]
    qa, qb, _ = _run_pair(ib, shape, 2, "fp64", "product", bc=bc)
    assert bits_equal(qa, qb, n), first_diff(qa, qb, n)


def test_complete_step_launch_count(cuda, ib):
    """64^3, periodic (x row kernel, y/z pencil pipeline, no boundary fill): five sweep launches
    per complete timestep, for every position of the middle pair."""
    shape = (64, 64, 64)
    q = problems.kelvin_helmholtz(shape, seed=3)
    fl = to_fluid(q, shape, gamma=5 / 3.0)
    geo = ib.Geometry(shape)
    num = ib.numerics(slope="mc")
    torch.cuda.synchronize()
    for it in range(6):
        l0 = ib.imogen.launch_count()
        ib.completeTimestep([fl], geo, [1e-4, 1, it, 2], num)
        assert ib.imogen.launch_count() - l0 == 5, it


def test_two_fluid_complete_step_matches_oracle(cuda, ib, po):
    """Gas (HLLC, gamma 5/3) and isothermal dust (c_s 0.1, gamma := 2) on a 64 x 64 periodic box,
    exact LogTrap2 drag: five iterations of the Strang composition, each dt from the CFL minimum
    over both fluids, against the oracle's fluid steps and drag in the same order."""
    n = 64
    shape, gas, dust = dusty.initial_state(n, seed=9)
    N = n * n
    tg, td = dusty.ld.THERMO_GAS, dusty.ld.THERMO_DUST
    geo = ib.Geometry(shape)
    h = [1.0 / s for s in shape]
    num = ib.numerics(slope="mc")
    fg = to_fluid(gas.copy(), shape, gamma=5 / 3.0)
    fd = to_fluid(dust.copy(), shape, gamma=2.0, c_iso=dusty.C_DUST)
    g_ref, d_ref = gas.copy(), dust.copy()
    sp_g = po.step_params(0.0, h, 5 / 3.0, method=2, slope="mc")
    sp_d = po.step_params(0.0, h, 2.0, c_iso=dusty.C_DUST, method=2, slope="mc")
    bc = ["circular"] * 6
    for it in range(5):
        tau = min(ib.cflTimestepFused(fg, 5 / 3.0, geo, 2), ib.cflTimestepFused(fd, 2.0, geo, 2))
        dt = 0.4 * tau
        ib.completeTimestep([fg, fd], geo, [dt, 1, it, 2], num, drag=(tg, td, "logtrap2"))

        tau_ref = min(po.cfl_timestep(g_ref, shape, 5 / 3.0, h, 2), po.cfl_timestep(d_ref, shape, 2.0, h, 2))
        assert abs(tau - tau_ref) <= 1e-13 * tau_ref, (it, tau, tau_ref)
        sp_g.dt = sp_d.dt = 0.4 * tau_ref
        po.drag_2fluid(g_ref, d_ref, shape, tg, td, 0.5 * sp_g.dt, 4)
        po.fluid_step_3d(g_ref, shape, sp_g, bc, 1, it)
        po.fluid_step_3d(d_ref, shape, sp_d, bc, 1, it)
        po.drag_2fluid(g_ref, d_ref, shape, tg, td, sp_g.dt, 4)
        po.fluid_step_3d(g_ref, shape, sp_g, bc, -1, it)
        po.fluid_step_3d(d_ref, shape, sp_d, bc, -1, it)
        po.drag_2fluid(g_ref, d_ref, shape, tg, td, 0.5 * sp_g.dt, 4)
    # the drag's pow/exp/expm1 come from CUDA on the GPU and glibc on the CPU (as in the drag tests)
    ok, info = product_close(host(fg), g_ref, N, l1=1e-12, scale=1e-11)
    assert ok, info
    ok, info = product_close(host(fd), d_ref, N, l1=1e-12, scale=1e-11)
    assert ok, info
    assert not np.array_equal(d_ref[2, :N], dust[2, :N])  # the drag moved the dust
