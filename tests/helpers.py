"""Shared helpers for the GPU parity tests."""
import numpy as np
import torch

import gpuimogen_b200 as ib


def to_fluid(q, shape, bc="circular", gamma=1.4, rho_min=1e-5, c_iso=-1.0, statics=None):
    t = torch.from_numpy(np.ascontiguousarray(q)).to("cuda")
    return ib.Fluid(shape, bc=bc, q=t, gamma=gamma, rho_min=rho_min, c_isothermal=c_iso, statics=statics)


def host(fl):
    torch.cuda.synchronize()
    return fl.q.detach().cpu().numpy()


def rel_l1(a, b, n):
    """Relative L1 difference per field over the first n cells of each slab."""
    out = []
    for k in range(5):
        den = np.sum(np.abs(b[k, :n]))
        num = np.sum(np.abs(a[k, :n] - b[k, :n]))
        out.append(num / den if den > 0 else num)
    return np.array(out)


def max_rel(a, b, n, floor=1e-300):
    d = np.abs(a[:, :n] - b[:, :n])
    s = np.maximum(np.abs(b[:, :n]), floor)
    return float(np.max(d / np.maximum(s, 1e-12 * np.max(np.abs(b[:, :n]), axis=1, keepdims=True))))


def _bitdiff(a, b, n):
    # NaNs compare equal whatever their payload (x86 and CUDA produce different NaN bits)
    x, y = a[:, :n], b[:, :n]
    both_nan = np.isnan(x) & np.isnan(y)
    return (x.view(np.int64) != y.view(np.int64)) & ~both_nan


def bits_equal(a, b, n):
    return not np.any(_bitdiff(a, b, n))


def product_close(a, b, n, l1=1e-13, scale=1e-11):
    """FMA-contracted product build vs the oracle: relative L1 per field <= l1 and every cell
    within `scale` of its field's largest magnitude."""
    err = rel_l1(a, b, n)
    big = np.max(np.abs(b[:, :n]), axis=1, keepdims=True)
    absd = np.max(np.abs(a[:, :n] - b[:, :n]) / np.maximum(big, 1e-300))
    return bool(np.all(err <= l1) and absd <= scale), (err, absd)


def first_diff(a, b, n):
    d = np.argwhere(_bitdiff(a, b, n))
    if len(d) == 0:
        return None
    k, i = d[0]
    return (int(k), int(i), float(a[k, i]), float(b[k, i]), len(d))


def oracle_cyl_loop(po, q, shape, h, r_inner, method, gamma, c_iso, bc, cfl, niter, slope="ospre",
                    fluxlim="ospre", geometric_radius=False, drag=None, dust=None):
    """The main loop in cylindrical geometry with the oracle, in place on q (and dust): CFL,
    source dt/2, forward step, source dt, backward step, source dt/2 (performCompleteTimestep,
    flux_multi.cu:174-272).  The source is the cylinder terms of every fluid followed by fluid 0's
    boundary fill in directions 1-3 (srcC___, sourceStep.cu:498-518), or with drag = (thermo_gas,
    thermo_dust, method) and the dust state: cylinder dt/2, drag dt, cylinder dt/2, then the fill
    (srcC__D, sourceStep.cu:521-562; the fill indexes fluid 0 once per fluid).  c_iso applies to
    the single fluid; the dust of a two-fluid run is thermo_dust's.  Returns the dts."""
    fluids = [(q, gamma, c_iso)]
    if drag is not None:
        fluids.append((dust, drag[1][0], drag[1][7]))
    dts = []

    def sp_of(dt, g, ci):
        return po.step_params(dt, h, 2.0 if ci != -1 else g, c_iso=ci, method=method, slope=slope,
                              fluxlim=fluxlim, cylindrical=True, r_inner=r_inner,
                              geometric_radius=geometric_radius)

    def source(t):
        for qq, _, _ in fluids:
            po.cyl_source(qq, shape, t * (0.5 if drag is not None else 1.0), h[0], r_inner)
        if drag is not None:
            po.drag_2fluid(q, dust, shape, drag[0], drag[1], t, drag[2], h=h)
            for qq, _, _ in fluids:
                po.cyl_source(qq, shape, 0.5 * t, h[0], r_inner)
        for _ in fluids:
            for d in (1, 2, 3):
                if shape[d - 1] > 3:
                    po.fluid_boundary(q, shape, bc, d)

    for it in range(niter):
        tau = min(po.cfl_timestep(qq, shape, g, h, method, cylindrical=True, r_inner=r_inner)
                  for qq, g, _ in fluids)
        dt = cfl * tau
        dts.append(dt)
        source(0.5 * dt)
        for qq, g, ci in fluids:
            po.fluid_step_3d(qq, shape, sp_of(dt, g, ci), bc, 1, it)
        source(dt)
        for qq, g, ci in fluids:
            po.fluid_step_3d(qq, shape, sp_of(dt, g, ci), bc, -1, it)
        source(0.5 * dt)
    return np.array(dts)
