"""Exact solution of the 1-D Riemann problem for an ideal gas.

Test helper: the published exact solver (Toro, "Riemann Solvers and Numerical Methods for Fluid
Dynamics", ch. 4: Newton iteration on the star-region pressure, then sampling of the wave
pattern).  The reference checks its Sod runs against the same solution
(experiment/RiemannProblem/analysis/SodShockSolution.m, harness run/test_suite/tsSod.m:40-77).
"""
import numpy as np


def _f(p, rho, P, c, g):
    if p > P:  # shock
        A = 2.0 / ((g + 1) * rho)
        B = (g - 1) / (g + 1) * P
        s = np.sqrt(A / (p + B))
        return (p - P) * s, s * (1 - 0.5 * (p - P) / (p + B))
    pr = p / P  # rarefaction
    return (2 * c / (g - 1)) * (pr ** ((g - 1) / (2 * g)) - 1), (1.0 / (rho * c)) * pr ** (-(g + 1) / (2 * g))


def star_state(rl, ul, pl, rr, ur, pr, g):
    cl = np.sqrt(g * pl / rl)
    cr = np.sqrt(g * pr / rr)
    p = max(1e-12, 0.5 * (pl + pr) - 0.125 * (ur - ul) * (rl + rr) * (cl + cr))
    for _ in range(100):
        fl, dl = _f(p, rl, pl, cl, g)
        fr, dr = _f(p, rr, pr, cr, g)
        dp = (fl + fr + (ur - ul)) / (dl + dr)
        pn = max(1e-14, p - dp)
        if abs(pn - p) < 1e-14 * (pn + p):
            p = pn
            break
        p = pn
    fl, _ = _f(p, rl, pl, cl, g)
    fr, _ = _f(p, rr, pr, cr, g)
    u = 0.5 * (ul + ur) + 0.5 * (fr - fl)
    return p, u


def sample(x, t, x0, left, right, g):
    """Density, velocity, pressure at positions x at time t for the initial jump at x0."""
    rl, ul, pl = left
    rr, ur, pr = right
    ps, us = star_state(rl, ul, pl, rr, ur, pr, g)
    cl = np.sqrt(g * pl / rl)
    cr = np.sqrt(g * pr / rr)
    out = np.zeros((3, len(x)))
    for i, xi in enumerate(x):
        s = (xi - x0) / t if t > 0 else np.sign(xi - x0) * np.inf
        if s <= us:  # left of contact
            if ps > pl:
                SL = ul - cl * np.sqrt((g + 1) / (2 * g) * ps / pl + (g - 1) / (2 * g))
                if s <= SL:
                    st = (rl, ul, pl)
                else:
                    r = rl * ((ps / pl + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pl + 1))
                    st = (r, us, ps)
            else:
                SH = ul - cl
                cs = cl * (ps / pl) ** ((g - 1) / (2 * g))
                ST = us - cs
                if s <= SH:
                    st = (rl, ul, pl)
                elif s >= ST:
                    st = (rl * (ps / pl) ** (1 / g), us, ps)
                else:
                    u = 2 / (g + 1) * (cl + (g - 1) / 2 * ul + s)
                    c = 2 / (g + 1) * (cl + (g - 1) / 2 * (ul - s))
                    r = rl * (c / cl) ** (2 / (g - 1))
                    st = (r, u, pl * (c / cl) ** (2 * g / (g - 1)))
        else:
            if ps > pr:
                SR = ur + cr * np.sqrt((g + 1) / (2 * g) * ps / pr + (g - 1) / (2 * g))
                if s >= SR:
                    st = (rr, ur, pr)
                else:
                    r = rr * ((ps / pr + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pr + 1))
                    st = (r, us, ps)
            else:
                SH = ur + cr
                cs = cr * (ps / pr) ** ((g - 1) / (2 * g))
                ST = us + cs
                if s >= SH:
                    st = (rr, ur, pr)
                elif s <= ST:
                    st = (rr * (ps / pr) ** (1 / g), us, ps)
                else:
                    u = 2 / (g + 1) * (-cr + (g - 1) / 2 * ur + s)
                    c = 2 / (g + 1) * (cr - (g - 1) / 2 * (ur - s))
                    r = rr * (c / cr) ** (2 / (g - 1))
                    st = (r, u, pr * (c / cr) ** (2 * g / (g - 1)))
        out[:, i] = st
    return out
