"""GPU parity of the full fluid step (Strang sweep order + boundary fill), the CFL reduction,
freezeAndPtot, the per-array boundary conditions and the drag source against the CPU oracle."""
import math

import numpy as np
import pytest
import torch

import riemann_exact as rx
from gpuimogen_b200 import problems
from helpers import bits_equal, first_diff, host, product_close, rel_l1, to_fluid

pytestmark = pytest.mark.gpu

BCSETS = [
    ["circular"] * 6,
    ["const", "const", "mirror", "mirror", "outflow", "outflow"],
    ["outflow", "outflow", "const", "circular", "mirror", "const"],
    ["mirror", "linear", "circular", "circular", "const", "mirror"],
]


@pytest.mark.parametrize("shape", [(24, 20, 18), (32, 26, 1), (70, 1, 1), (12, 4, 30)])
@pytest.mark.parametrize("bcs", range(len(BCSETS)))
@pytest.mark.parametrize("method", [2, 1, 3])
def test_fluidstep_strict_bitexact(cuda, ib, po, shape, bcs, method):
    bc = BCSETS[bcs]
    for d in range(3):  # mirror/outflow need >= 2*halo+1 cells; degenerate axes stay circular
        if shape[d] < 12:
            bc = list(bc)
            bc[2 * d] = bc[2 * d + 1] = "circular"
    n = shape[0] * shape[1] * shape[2]
    q = problems.random_smooth(shape, gamma=5 / 3.0, seed=31 + bcs, amp=0.3)
    h = [1.0 / s for s in shape]
    sp = po.step_params(0.0, h, 5 / 3.0, rho_min=1e-5, method=method, slope="mc")
    ref = q.copy()
    ib.use_variant("strict")
    try:
        fl = to_fluid(q, shape, bc=bc, gamma=5 / 3.0)
        geo = ib.Geometry(shape, h)
        for it in range(3):
            tau = po.cfl_timestep(ref, shape, 5 / 3.0, h, method)
            dt = 0.4 * tau
            sp.dt = dt
            tau_g = ib.cflTimestepFused(fl, 5 / 3.0, geo, method)
            assert tau_g == tau, (it, tau_g, tau)
            for sd in (1, -1):
                po.fluid_step_3d(ref, shape, sp, bc, sd, it)
                ib.fluidstep([fl], geo, [dt, 1, sd, it, method], ib.numerics(slope="mc"))
            out = host(fl)
            assert bits_equal(out, ref, n), (it, first_diff(out, ref, n))
    finally:
        ib.use_variant("product")


def test_cfl_soundspeed_freeze_strict(cuda, ib, po):
    for shape in [(33, 17, 9), (64, 1, 1), (40, 30, 1)]:
        n = shape[0] * shape[1] * shape[2]
        q = problems.random_jumpy(shape, seed=3)
        h = (0.02, 0.03, 0.05)
        ib.use_variant("strict")
        try:
            fl = to_fluid(q, shape)
            geo = ib.Geometry(shape, h)
            cs = ib.cudaSoundspeed(fl, 1.4)
            cs_ref = po.soundspeed(q, shape, 1.4)
            assert np.array_equal(cs.cpu().numpy(), cs_ref)
            for method in (1, 2, 3):
                t_ref = po.cfl_timestep(q, shape, 1.4, h, method, cs_ref)
                assert ib.cflTimestep(fl, cs, geo, method) == t_ref
                assert ib.cflTimestepFused(fl, 1.4, geo, method) == t_ref
            ref = q.copy()
            ptot_ref, fr_ref = po.freeze_and_ptot(ref, shape, 1.4, 0.9)
            ptot, fr = ib.freezeAndPtot(fl, 1.4, 1, 0.9)
            assert np.array_equal(ptot.cpu().numpy(), ptot_ref)
            assert np.array_equal(fr.cpu().numpy(), fr_ref)
            assert bits_equal(host(fl), ref, n)   # E floored in place where c_s < cs_min
        finally:
            ib.use_variant("product")


def test_cfl_device_result_and_nan_ignored(cuda, ib, po):
    shape = (50, 20, 10)
    n = 50 * 20 * 10
    q = problems.random_smooth(shape, seed=4)
    q[0, 17] = np.nan          # a NaN cell never wins the min, as in the reference's ternaries
    fl = to_fluid(q, shape)
    geo = ib.Geometry(shape)
    tau_dev = torch.zeros(1, dtype=torch.float64, device="cuda")
    ib.cflTimestepFused(fl, 1.4, geo, 2, tau_device=tau_dev)
    ref = po.cfl_timestep(q, shape, 1.4, geo.h, 2)
    assert math.isfinite(ref)
    assert abs(float(tau_dev.item()) - ref) <= 1e-15 * ref
    # repeated calls reuse the reduction scratch correctly
    for _ in range(3):
        assert abs(ib.cflTimestepFused(fl, 1.4, geo, 2) - ref) <= 1e-15 * ref


@pytest.mark.parametrize("mode", ["mirror", "const", "linear"])
@pytest.mark.parametrize("direction", [1, 2, 3])
def test_cudaStatics_per_array_strict(cuda, ib, po, mode, direction):
    shape = (14, 12, 11)
    n = 14 * 12 * 11
    q = problems.random_smooth(shape, seed=8)
    bc = ["circular"] * 6
    bc[2 * (direction - 1)] = bc[2 * (direction - 1) + 1] = mode
    fl = to_fluid(q, shape, bc=bc)
    ref = q.copy()
    ib.use_variant("strict")
    try:
        for slab in range(5):
            vec = slab - 1 if slab >= 2 else 0
            phi = ref[slab, :n].copy()
            rc0 = po.array_boundary(phi, shape, mode, direction, 0, vec)
            rc1 = po.array_boundary(phi, shape, mode, direction, 1, vec)
            if rc0 or rc1:
                with pytest.raises(ib.ImogenError):
                    ib.cudaStatics(fl, slab, direction)
                return
            ref[slab, :n] = phi
            ib.cudaStatics(fl, slab, direction)
        out = host(fl)
    finally:
        ib.use_variant("product")
    assert bits_equal(out, ref, n), first_diff(out, ref, n)


def test_statics_fade(cuda, ib, po):
    shape = (16, 8, 4)
    n = 16 * 8 * 4
    q = problems.random_smooth(shape, seed=2)
    rng = np.random.default_rng(0)
    idx = rng.choice(n, size=40, replace=False).astype(np.float64)
    st = np.stack([idx, rng.uniform(0.5, 2, 40), np.where(np.arange(40) % 3 == 0, 1.0, 0.3)])
    ref = q.copy()
    phi = ref[0, :n].copy()
    for _ in range(3):  # fluid step applies the density statics three times per sweep direction
        po.statics_fade(phi, st)
    ref[0, :n] = phi
    fl = to_fluid(q, shape, bc=["circular"] * 6,
                  statics=[torch.from_numpy(st).cuda()] + [None] * 4)
    ib.use_variant("strict")
    try:
        ib.setFluidBoundary(fl, 1)
        out = host(fl)
    finally:
        ib.use_variant("product")
    assert np.array_equal(out[0, :n], ref[0, :n])


@pytest.mark.parametrize("method", [0, 1, 2, 4, 5])
def test_drag_logtrap_matches_oracle(cuda, ib, po, method):
    shape = (64, 32, 1)
    n = 64 * 32
    rng = np.random.default_rng(1)
    cube = (1, 32, 64)
    rho_g = 1.0 + 0.1 * rng.uniform(-1, 1, n)
    gas = problems.pack(shape, rho_g.reshape(cube), 0, (rho_g * rng.uniform(-1e-2, 1e-2, n)).reshape(cube),
                        (rho_g * rng.uniform(-1e-2, 1e-2, n)).reshape(cube), 0)
    gas[1, :n] = 1.0 / (5 / 3.0 - 1) + 0.5 * (gas[2, :n] ** 2 + gas[3, :n] ** 2) / rho_g
    rho_d = rho_g * 10 ** rng.uniform(-2, 0, n)
    dust = problems.pack(shape, rho_d.reshape(cube), 0, (rho_d * rng.uniform(-2e-2, 2e-2, n)).reshape(cube), 0, 0)
    dust[1, :n] = 0.5 * dust[2, :n] ** 2 / rho_d + 1e-4 * rho_d
    tg = [5 / 3.0, 3.3e-27, 8.4e-6, 0.7, 2.4e-19, 0.2, 1.381e-23, -1]
    td = [1.01, 3e-11, 0, 0, math.pi * 25e-12, 0, 1.381e-23, 0.1]
    g_ref, d_ref = gas.copy(), dust.copy()
    po.drag_2fluid(g_ref, d_ref, shape, tg, td, 0.05, method)
    fg, fd = to_fluid(gas, shape), to_fluid(dust, shape)
    ib.cudaSource2FluidDrag(fg, fd, tg, td, ib.Geometry(shape), [0.05, method])
    # transcendental functions (pow, exp, expm1) come from CUDA's libdevice on the GPU and glibc
    # on the CPU, and the momenta are differences of two larger terms (a dust momentum that
    # starts at zero is all cancellation): per field relative L1 <= 1e-12 and every cell within
    # 1e-11 of its field's largest magnitude
    ok, info = product_close(host(fg), g_ref, n, l1=1e-12, scale=1e-11)
    assert ok, info
    ok, info = product_close(host(fd), d_ref, n, l1=1e-12, scale=1e-11)
    assert ok, info
    assert not np.array_equal(g_ref[2, :n], gas[2, :n])   # the drag did act


def _etdrk2_state(shape, seed):
    n = shape[0] * shape[1] * shape[2]
    rng = np.random.Generator(np.random.Philox(seed))
    S = ib_slab_pitch(shape)
    gas, dust = np.zeros((5, S)), np.zeros((5, S))
    gas[0, :n] = 1.0 + 0.1 * rng.uniform(-1, 1, n)
    dust[0, :n] = gas[0, :n] * 10 ** rng.uniform(-2, 0, n)
    for k in (2, 3, 4):
        gas[k, :n] = gas[0, :n] * rng.uniform(-1e-2, 1e-2, n)
        dust[k, :n] = dust[0, :n] * rng.uniform(-2e-2, 2e-2, n)
    P = 1.0 + 0.2 * rng.uniform(-1, 1, n)
    gas[1, :n] = P / (5 / 3.0 - 1) + 0.5 * (gas[2, :n] ** 2 + gas[3, :n] ** 2 + gas[4, :n] ** 2) / gas[0, :n]
    dust[1, :n] = 0.5 * (dust[2, :n] ** 2 + dust[3, :n] ** 2 + dust[4, :n] ** 2) / dust[0, :n] + 1e-4 * dust[0, :n]
    return gas, dust


def ib_slab_pitch(shape):
    n = shape[0] * shape[1] * shape[2]
    return (n + 31) // 32 * 32


ETD_TG = [5 / 3.0, 3.3e-27, 8.4e-6, 0.7, 2.4e-19, 0.2, 1.381e-23, -1]
ETD_TD = {"weak": [1.01, 3e-11, 0, 0, math.pi * 25e-12, 0, 1.381e-23, 0.1],
          "stiff": [1.01, 3e-15, 0, 0, math.pi * 25e-12, 0, 1.381e-23, 0.1]}


@pytest.mark.parametrize("stiff", ["weak", "stiff"])
@pytest.mark.parametrize("shape", [(16, 8, 1), (8, 6, 5), (12, 1, 6), (32, 1, 1), (300, 5, 3), (40, 1, 70)],
                         ids=lambda s: "%dx%dx%d" % s)
def test_drag_etdrk2_matches_oracle(cuda, ib, po, shape, stiff):
    """ETDRK2: pressure gradient by periodic central differences in every gradient layout (x-y,
    3-D, x-z, 1-D; rows longer than one block), then the exponential midpoint update."""
    n = shape[0] * shape[1] * shape[2]
    gas, dust = _etdrk2_state(shape, 7 + shape[0])
    h = [0.5 / shape[0], 0.25 / shape[1], 2.0 / shape[2]]
    g_ref, d_ref = gas.copy(), dust.copy()
    po.drag_2fluid(g_ref, d_ref, shape, ETD_TG, ETD_TD[stiff], 0.05, 3, h=h)
    for variant in ("strict", "product"):
        fg, fd = to_fluid(gas.copy(), shape), to_fluid(dust.copy(), shape)
        ib.use_variant(variant)
        try:
            ib.cudaSource2FluidDrag(fg, fd, ETD_TG, ETD_TD[stiff], ib.Geometry(shape, h=h), [0.05, 3])
        finally:
            ib.use_variant("product")
        # exp, expm1, pow and sqrt come from CUDA on the GPU and glibc on the CPU (see the LogTrap test)
        ok, info = product_close(host(fg), g_ref, n, l1=1e-12, scale=1e-11)
        assert ok, (variant, info)
        ok, info = product_close(host(fd), d_ref, n, l1=1e-12, scale=1e-11)
        assert ok, (variant, info)
    assert not np.array_equal(g_ref[2, :n], gas[2, :n])


def test_drag_etdrk2_zero_relative_velocity_cell_unchanged(cuda, ib, po):
    """A cell whose gas and dust move together (|dv| < 1e-9, drag rate 0) keeps its state, where
    the reference divides 0 by 0; its neighbours still feel their pressure gradient."""
    shape = (16, 8, 1)
    n = 128
    gas, dust = _etdrk2_state(shape, 3)
    j = 37
    dust[2:5, j] = gas[2:5, j] * dust[0, j] / gas[0, j]
    g_ref, d_ref = gas.copy(), dust.copy()
    po.drag_2fluid(g_ref, d_ref, shape, ETD_TG, ETD_TD["weak"], 0.05, 3)
    fg, fd = to_fluid(gas.copy(), shape), to_fluid(dust.copy(), shape)
    ib.cudaSource2FluidDrag(fg, fd, ETD_TG, ETD_TD["weak"], ib.Geometry(shape), [0.05, 3])
    G, D = host(fg), host(fd)
    assert np.array_equal(G[:, j], gas[:, j]) and np.array_equal(D[:, j], dust[:, j])
    assert np.array_equal(g_ref[:, j], gas[:, j])
    ok, info = product_close(G, g_ref, n, l1=1e-12, scale=1e-11)
    assert ok, info


def test_sod_gpu_matches_oracle_and_exact(cuda, ib, po):
    n = 1024
    q = problems.sod(n)
    shape = (n, 1, 1)
    fl = to_fluid(q, shape, bc="const", gamma=1.4)
    geo = ib.Geometry(shape)
    tm = ib.TimeManager(cfl=0.4, tmax=0.2)
    while tm.running:
        ib.run_iteration([fl], geo, tm, 2)
    out = host(fl)
    x = (np.arange(n) + 0.5) / n
    ex = rx.sample(x, tm.time, 0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1), 1.4)
    l1 = np.mean(np.abs(out[0, :n] - ex[0]))
    assert abs(tm.time - 0.2) < 1e-14
    assert l1 < 1.0e-3, l1
    # oracle replay with the same dt sequence semantics
    ref = problems.sod(n)
    sp = po.step_params(0.0, geo.h, 1.4, method=2)
    t, it, kc = 0.0, 0, 0.0
    while t < 0.2 * (1 - 1e-14):
        dt = 0.4 * po.cfl_timestep(ref, shape, 1.4, geo.h, 2)
        if t + 2 * dt > 0.2:
            dt = .5 * (0.2 - t)
        sp.dt = dt
        po.fluid_step_3d(ref, shape, sp, ["const"] * 6, 1, it)
        po.fluid_step_3d(ref, shape, sp, ["const"] * 6, -1, it)
        y = 2 * dt - kc
        tn = t + y
        kc = (tn - t) - y
        t = tn
        it += 1
    assert it == tm.iteration
    assert np.all(rel_l1(out, ref, n) <= 1e-12), rel_l1(out, ref, n)


def test_kelvin_helmholtz_product_vs_oracle(cuda, ib, po):
    """3-D HLLC with the MC limiter, periodic: relative L1 per field after 10 iterations."""
    shape = (48, 48, 48)
    n = 48 ** 3
    q = problems.kelvin_helmholtz(shape, seed=7)
    fl = to_fluid(q, shape, gamma=5 / 3.0)
    geo = ib.Geometry(shape)
    ref = q.copy()
    sp = po.step_params(0.0, geo.h, 5 / 3.0, method=2, slope="mc")
    num = ib.numerics(slope="mc")
    tm = ib.TimeManager(cfl=0.4)
    for it in range(10):
        dt_ref = 0.4 * po.cfl_timestep(ref, shape, 5 / 3.0, geo.h, 2)
        sp.dt = dt_ref
        po.fluid_step_3d(ref, shape, sp, ["circular"] * 6, 1, it)
        po.fluid_step_3d(ref, shape, sp, ["circular"] * 6, -1, it)
        dt = ib.run_iteration([fl], geo, tm, 2, num)
        assert abs(dt - dt_ref) <= 1e-13 * dt_ref
    err = rel_l1(host(fl), ref, n)
    assert np.all(err <= 1e-12), err


@pytest.mark.parametrize("method", [2, 1])
def test_tma_pipeline_many_blocks_per_cta(cuda, ib, po, method):
    """Grids with more pencil blocks than resident CTAs, so every persistent CTA of the TMA-fed
    sweeps cycles through both prefetch tiles several times: strict build bit-exact against the
    oracle, and no bounded device wait ran out."""
    shape = (64, 48, 40)
    n = shape[0] * shape[1] * shape[2]
    q = problems.random_jumpy(shape, gamma=1.4, seed=53)
    h = [1.0 / s for s in shape]
    sp = po.step_params(0.0, h, 1.4, rho_min=1e-5, method=method, slope="mc")
    ref = q.copy()
    ib.use_variant("strict")
    try:
        ib.device_wait_status(clear=True)
        fl = to_fluid(q, shape, bc="circular", gamma=1.4)
        geo = ib.Geometry(shape, h)
        for it in range(2):
            sp.dt = 0.3 * po.cfl_timestep(ref, shape, 1.4, h, method)
            for sd in (1, -1):
                po.fluid_step_3d(ref, shape, sp, ["circular"] * 6, sd, it)
                ib.fluidstep([fl], geo, [sp.dt, 1, sd, it, method], ib.numerics(slope="mc"))
        out = host(fl)
        assert ib.device_wait_status() == 0
    finally:
        ib.use_variant("product")
    assert bits_equal(out, ref, n), first_diff(out, ref, n)


@pytest.mark.parametrize("shape", [(5, 256, 6), (7, 6, 256), (6, 300, 4)])
def test_tile_path_long_pencils(cuda, ib, po, shape):
    """y/z pencils that the TMA-fed sweeps do not take (odd nx, or longer than 256 cells) run
    through the chunked tile kernel: several chunks per pencil, strict build bit-exact."""
    n = shape[0] * shape[1] * shape[2]
    q = problems.random_smooth(shape, gamma=1.4, seed=61, amp=0.3)
    h = [1.0 / s for s in shape]
    sp = po.step_params(0.0, h, 1.4, rho_min=1e-5, method=2, slope="mc")
    ref = q.copy()
    ib.use_variant("strict")
    try:
        fl = to_fluid(q, shape, bc="circular", gamma=1.4)
        geo = ib.Geometry(shape, h)
        for it in range(2):
            sp.dt = 0.4 * po.cfl_timestep(ref, shape, 1.4, h, 2)
            for sd in (1, -1):
                po.fluid_step_3d(ref, shape, sp, ["circular"] * 6, sd, it)
                ib.fluidstep([fl], geo, [sp.dt, 1, sd, it, 2], ib.numerics(slope="mc"))
        out = host(fl)
    finally:
        ib.use_variant("product")
    assert bits_equal(out, ref, n), first_diff(out, ref, n)


@pytest.mark.parametrize("shape,method,slope", [((1100, 3, 2), 2, "mc"), ((1240, 2, 1), 2, "mc"),
                                                ((4, 700, 3), 2, "mc"), ((8, 4, 1030), 2, "mc"),
                                                ((4, 720, 2), 1, "ospre"), ((1028, 520, 1), 2, "mc"),
                                                ((1028, 520, 1), 1, "vanleer"), ((1101, 2, 2), 2, "mc"),
                                                ((6, 4, 600), 2, "mc")])
def test_chunk_pipeline_long_pencils(cuda, ib, po, shape, method, slope):
    """Pencils above 512 cells (x rows above 1024) through the chunked TMA pipeline: chunks of
    248 (x) or 120 (y/z) cells with 4-cell halos, periodic ends from halo boxes, the first chunk's
    first outputs deferred; pencil lengths with a partial and with a whole last chunk (1240 = 5 x
    248, 720 = 6 x 120), HLLC and HLL.  Odd x rows (1101) and nx not a multiple of 4 (6) fall back
    to the tile kernel.  Strict build bit-exact."""
    n = shape[0] * shape[1] * shape[2]
    q = problems.random_smooth(shape, gamma=1.4, seed=71, amp=0.3)
    h = [1.0 / s for s in shape]
    sp = po.step_params(0.0, h, 1.4, rho_min=1e-5, method=method, slope=slope)
    ref = q.copy()
    ib.use_variant("strict")
    try:
        ib.device_wait_status(clear=True)
        fl = to_fluid(q, shape, bc="circular", gamma=1.4)
        geo = ib.Geometry(shape, h)
        for it in range(2):
            sp.dt = 0.4 * po.cfl_timestep(ref, shape, 1.4, h, method)
            for sd in (1, -1):
                po.fluid_step_3d(ref, shape, sp, ["circular"] * 6, sd, it)
                ib.fluidstep([fl], geo, [sp.dt, 1, sd, it, method], ib.numerics(slope=slope))
        out = host(fl)
        assert ib.device_wait_status() == 0
    finally:
        ib.use_variant("product")
    assert bits_equal(out, ref, n), first_diff(out, ref, n)


@pytest.mark.parametrize("shape", [(6, 300, 4), (8, 512, 3), (388, 340, 12), (392, 336, 6)])
def test_pipeline_long_pencils_and_wide_z_blocks(cuda, ib, po, shape):
    """TMA pipeline shapes beyond the basic one: y pencils of 257-512 cells (two box rows, two
    cells per thread) and z sweeps of large x-y planes (blocks four columns wide; with the FP32
    flux and nx a multiple of 8, eight columns computed in groups and stored in place)."""
    n = shape[0] * shape[1] * shape[2]
    q = problems.random_smooth(shape, gamma=1.4, seed=67, amp=0.3)
    h = [1.0 / s for s in shape]
    sp = po.step_params(0.0, h, 1.4, rho_min=1e-5, method=2, slope="mc")
    ref = q.copy()
    ib.use_variant("strict")
    try:
        ib.device_wait_status(clear=True)
        fl = to_fluid(q, shape, bc="circular", gamma=1.4)
        geo = ib.Geometry(shape, h)
        sp.dt = 0.4 * po.cfl_timestep(ref, shape, 1.4, h, 2)
        for sd in (1, -1):
            po.fluid_step_3d(ref, shape, sp, ["circular"] * 6, sd, 0)
            ib.fluidstep([fl], geo, [sp.dt, 1, sd, 0, 2], ib.numerics(slope="mc"))
        out = host(fl)
        assert ib.device_wait_status() == 0
    finally:
        ib.use_variant("product")
    assert bits_equal(out, ref, n), first_diff(out, ref, n)


@pytest.mark.parametrize("precision", ["fp64", "fp32flux"])
@pytest.mark.parametrize("nz", [256, 200])
def test_wide_z_blocks_match_y_sweep_of_transposed_state(cuda, ib, nz, precision):
    """Full-size z sweeps of a 256 x 520 plane (the 8-column wide-block kernel; nz = 256 with the
    pencil length fixed at compile time) against the y sweep of the same state with y and z (and
    p_y and p_z) exchanged, which runs through the ordinary pipeline kernel."""
    shape = (256, 520, nz)
    N = shape[0] * shape[1] * shape[2]
    q = torch.from_numpy(problems.kelvin_helmholtz(shape, seed=3)).cuda()
    h = [1.0 / 256, 1.0 / 520, 1.0 / nz]
    num = ib.numerics(slope="mc", precision=precision)
    dt = 0.2 / (2.0 * 520)
    fl = ib.Fluid(shape, q=q.clone(), gamma=5 / 3.0)
    ib.cudaFluidStep(fl, ib.Geometry(shape, h), [dt, 1, 5 / 3.0, 1e-5, 2, 3], num)
    tshape = (256, nz, 520)
    qt = torch.zeros_like(q)
    qt[:, :N] = q[:, :N].view(5, nz, 520, 256).transpose(1, 2).reshape(5, N)
    qt[[3, 4]] = qt[[4, 3]].clone()
    ft = ib.Fluid(tshape, q=qt, gamma=5 / 3.0)
    ib.cudaFluidStep(ft, ib.Geometry(tshape, [h[0], h[2], h[1]]), [dt, 1, 5 / 3.0, 1e-5, 2, 2], num)
    back = ft.q[:, :N].view(5, 520, nz, 256).transpose(1, 2).reshape(5, N).clone()
    back[[3, 4]] = back[[4, 3]].clone()
    out = fl.q[:, :N]
    assert ib.device_wait_status() == 0
    assert not torch.equal(out, q[:, :N])  # the sweep did act
    err = ((out - back).abs().sum(dim=1) / back.abs().sum(dim=1).clamp_min(1e-300)).cpu().numpy()
    tol = 1e-13 if precision == "fp64" else 1e-7
    assert np.all(err <= tol), err


def test_cfl_host_read_while_a_download_runs(cuda, ib, po):
    """The CFL timestep reaches the host through mapped memory written by the kernel, not a
    device-to-host copy: it must be correct, and bit-identical to the oracle in the strict build,
    while a large state download is in flight on another stream."""
    shape = (48, 40, 36)
    q = problems.random_jumpy(shape, seed=21)
    h = (0.02, 0.025, 0.03)
    big = torch.empty(64 << 20, dtype=torch.float64, device="cuda")  # 512 MB read out meanwhile
    big.fill_(1.0)
    pinned = torch.empty(big.numel(), dtype=torch.float64).pin_memory()
    side = torch.cuda.Stream()
    ib.use_variant("strict")
    try:
        fl = to_fluid(q, shape)
        geo = ib.Geometry(shape, h)
        for method in (1, 2, 3):
            ref = po.cfl_timestep(q, shape, 1.4, h, method)
            torch.cuda.synchronize()
            with torch.cuda.stream(side):
                pinned.copy_(big, non_blocking=True)
            tau = ib.cflTimestepFused(fl, 1.4, geo, method)
            assert tau == ref, (method, tau, ref)
            torch.cuda.synchronize()
    finally:
        ib.use_variant("product")
    assert pinned[-1].item() == 1.0
