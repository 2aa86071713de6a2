"""Generate golden vectors with the reference's own GPU code (run on a machine with a GPU).

Loads the reference libraries built by oracle/ref_harness/Makefile (oracle/_ref/), which compile
imogenproject/gpuImogen's gpuclass sources unchanged for sm_100a, runs small seeded cases through
the reference's entry points (performFluidUpdate_3D, computeLocalCFLTimestep +
calculateSoundspeed, sourcefunction_2FluidDrag) and writes one .npz per case:

    input  (5, slab) float64    initial state (seeded generators in gpuimogen_b200/problems.py)
    params                      method, limiter, gamma, rho_min, c_iso, h, bc, cfl, niter
    out_fast / dts_fast         reference built as it builds itself (FMA contraction on)
    out_strict / dts_strict     reference built with -fmad=false (comparable bit for bit)

Boundary conditions are limited to circular, const and mirror: the reference's outflow and linear
extrapolation kernels write outside their rows (cudaStatics.cu / boundaryConds.cu), so they are not
run here.

Usage: python tests/golden/make_golden.py OUTDIR [--etdrk2-only | --cyl-only | --cases=name1,name2]
"""
import ctypes
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from gpuimogen_b200 import problems  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
BC = {"circular": 0, "mirror": 1, "const": 4}

TG = [5 / 3.0, 3.3e-27, 8.4e-6, 0.7, 2.4e-19, 0.2, 1.381e-23, -1.0]
TD = [1.01, 3e-11, 0.0, 0.0, np.pi * 25e-12, 0.0, 1.381e-23, 0.1]
TD_STIFF = [1.01, 3e-15, 0.0, 0.0, np.pi * 25e-12, 0.0, 1.381e-23, 0.1]  # k dt of order 1


def lib(limiter, strict):
    name = "libimogen_ref_%s%s.so" % (limiter, "_strict" if strict else "")
    L = ctypes.CDLL(os.path.join(REF, name))
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    L.ref_run.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int64, ctypes.c_double,
                          ctypes.c_double, ctypes.c_double, ctypes.c_int, dp, ip, ctypes.c_double, ctypes.c_int, dp]
    L.ref_cfl.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int64, ctypes.c_double,
                          ctypes.c_int, dp, dp]
    L.ref_drag.argtypes = [dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int64, dp, dp,
                           ctypes.c_double, ctypes.c_int]
    return L


def P(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


FLUID_CASES = [
    # name, generator, shape, method, limiter, gamma, c_iso, bc, cfl, niter
    ("kh_hllc_mc", "kh", (20, 16, 12), 2, "mc", 5 / 3.0, -1.0, ["circular"] * 6, 0.4, 5),
    ("smooth_hllc_ospre_bc", "smooth", (18, 14, 10), 2, "ospre", 1.4, -1.0,
     ["const", "const", "mirror", "mirror", "const", "mirror"], 0.4, 4),
    ("jumpy_hllc_mc", "jumpy", (16, 12, 10), 2, "mc", 1.4, -1.0, ["circular"] * 6, 0.3, 3),
    ("jumpy_hll_ospre_bc", "jumpy", (16, 12, 10), 1, "ospre", 1.4, -1.0,
     ["mirror", "mirror", "const", "const", "circular", "circular"], 0.3, 3),
    ("iso_hll_ospre", "smooth", (16, 12, 1), 1, "ospre", 1.4, 0.3, ["circular"] * 6, 0.3, 4),
    ("sod_hll_const", "sod", (256, 1, 1), 1, "ospre", 1.4, -1.0, ["const"] * 6, 0.4, 25),
    ("sod_hllc_const", "sod", (256, 1, 1), 2, "mc", 1.4, -1.0, ["const"] * 6, 0.4, 25),
    ("sod_xj_const", "sod", (256, 1, 1), 3, "ospre", 1.4, -1.0, ["const"] * 6, 0.4, 25),
    # 100 iterations: the FP64 drop-in's parity bound is stated after 100 steps
    ("kh_hllc_mc_100", "kh", (20, 16, 12), 2, "mc", 5 / 3.0, -1.0, ["circular"] * 6, 0.4, 100),
    ("jumpy_hll_ospre_100", "jumpy", (16, 12, 10), 1, "ospre", 1.4, -1.0, ["circular"] * 6, 0.3, 100),
]
# Multi-dimensional Xin-Jin: the harness hands each Xin-Jin sweep a NULL temporary (see
# oracle/ref_harness/harness.cu, fluid_update_3d): the reference's Xin-Jin branch initialises its
# scratch pointers only when it allocates the temporary itself (cudaFluidStep.cu:315, 362-371).
# With a reused temporary its second sweep of a step used uninitialised pointers, which is how an
# earlier 32x32x1 run of this harness ended in an illegal memory access.
# The extents are ones the reference's Xin-Jin launch covers: it sizes its grid with
# ROUNDUPTO(n, blocksize.x - 4) (cudaFluidStep.cu:410, 458), and ROUNDUPTO (cudaCommon.h:170) does
# not parenthesise its second argument, so the grid holds (n + 24 - n % 32) / 28 blocks of 28
# cells (n when n % 32 == 4): too few for many n (12 cells: no block at all, a launch error; 200
# cells: 196 updated).  32, 64 and 256 are covered.
FLUID_CASES += [
    ("kh_xj_100", "kh", (32, 32, 32), 3, "ospre", 5 / 3.0, -1.0, ["circular"] * 6, 0.4, 100),
    ("jumpy_xj_3d_bc", "jumpy", (32, 32, 32), 3, "ospre", 1.4, -1.0,
     ["const", "const", "mirror", "mirror", "circular", "circular"], 0.3, 4),
    ("kh_xj_2d", "kh", (32, 32, 1), 3, "ospre", 5 / 3.0, -1.0, ["circular"] * 6, 0.4, 6),
]


def make_input(gen, shape, gamma):
    if gen == "kh":
        return problems.kelvin_helmholtz(shape, gamma=gamma, seed=7)
    if gen == "smooth":
        return problems.random_smooth(shape, gamma=gamma, seed=23, amp=0.3)
    if gen == "jumpy":
        return problems.random_jumpy(shape, gamma=gamma, seed=29)
    if gen == "sod":
        return problems.sod(shape[0], gamma)
    raise ValueError(gen)


# ETDRK2 (exponential midpoint) differentiates the gas internal energy, so its states carry a
# seeded pressure field; one per layout the reference distinguishes: x-y plane, 3-D, x-z plane
# (ny = 1 < nz) and 1-D.  Cell sizes are 1/n per axis as the harness's geometry sets them.
ETDRK2_SHAPES = [(16, 8, 1), (8, 6, 5), (12, 1, 6), (32, 1, 1)]


def etdrk2_state(shape, seed):
    n = shape[0] * shape[1] * shape[2]
    rng = np.random.Generator(np.random.Philox(seed))
    S = (n + 31) // 32 * 32
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


def etdrk2_golden(outdir):
    rec = {}
    for j, shape in enumerate(ETDRK2_SHAPES):
        gas, dust = etdrk2_state(shape, 61 + j)
        key = "%dx%dx%d" % shape
        rec["gas_" + key], rec["dust_" + key] = gas, dust
        for case, tdv in (("", TD), ("stiff_", TD_STIFF)):
            for strict in (False, True):
                g, d = gas.copy(), dust.copy()
                rc = lib("ospre", strict).ref_drag(P(g), P(d), shape[0], shape[1], shape[2], g.shape[1],
                                                   P(np.array(TG)), P(np.array(tdv)), 0.05, 3)
                assert rc == 0, (shape, rc)
                tag = "%s%s_%s" % (case, key, "strict" if strict else "fast")
                rec["gas_out_" + tag], rec["dust_out_" + tag] = g, d
    np.savez_compressed(os.path.join(outdir, "drag_etdrk2.npz"),
                        meta=json.dumps({"shapes": [list(s) for s in ETDRK2_SHAPES], "tg": TG, "td": TD,
                                         "td_stiff": TD_STIFF, "dt": 0.05}), **rec)
    print("wrote drag_etdrk2", flush=True)


def main(outdir, only=None, cases=None):
    """only="etdrk2": the ETDRK2 drag vectors alone; cases: run only these fluid cases (their
    entries are merged into an existing index.json) and nothing else."""
    os.makedirs(outdir, exist_ok=True)
    if only == "etdrk2":
        etdrk2_golden(outdir)
        return
    index = {}
    if cases:
        ipath = os.path.join(outdir, "index.json")
        if os.path.exists(ipath):
            with open(ipath) as f:
                index = json.load(f)
    for name, gen, shape, method, limiter, gamma, c_iso, bc, cfl, niter in FLUID_CASES:
        if cases and name not in cases:
            continue
        q0 = make_input(gen, shape, gamma)
        h = np.array([1.0 / s for s in shape])
        bca = (ctypes.c_int * 6)(*[BC[b] for b in bc])
        rec = {"input": q0}
        for strict in (False, True):
            q = q0.copy()
            dts = np.zeros(niter)
            rc = lib(limiter, strict).ref_run(P(q), shape[0], shape[1], shape[2], q.shape[1], gamma, 1e-5, c_iso,
                                               method, P(h), bca, cfl, niter, P(dts))
            assert rc == 0, (name, rc)
            tag = "strict" if strict else "fast"
            rec["out_" + tag] = q
            rec["dts_" + tag] = dts
        meta = dict(kind="fluid", gen=gen, shape=list(shape), method=method, limiter=limiter, gamma=gamma,
                    rho_min=1e-5, c_iso=c_iso, bc=bc, cfl=cfl, niter=niter)
        np.savez_compressed(os.path.join(outdir, name + ".npz"), meta=json.dumps(meta), **rec)
        index[name] = meta
        print("wrote", name, flush=True)
    if cases:
        with open(os.path.join(outdir, "index.json"), "w") as f:
            json.dump(index, f, indent=1)
        return

    # CFL timesteps
    cfl_rec = {}
    for gen, shape, gamma in (("jumpy", (17, 13, 9), 1.4), ("smooth", (40, 30, 1), 5 / 3.0), ("sod", (300, 1, 1), 1.4)):
        q = make_input(gen, shape, gamma)
        h = np.array([0.02, 0.03, 0.05])
        for method in (1, 2, 3):
            for strict in (False, True):
                t = ctypes.c_double(0)
                rc = lib("ospre", strict).ref_cfl(P(q), shape[0], shape[1], shape[2], q.shape[1], gamma, method, P(h),
                                                  ctypes.byref(t))
                assert rc == 0
                cfl_rec["%s_m%d_%s" % (gen, method, "strict" if strict else "fast")] = t.value
    np.savez_compressed(os.path.join(outdir, "cfl.npz"), values=json.dumps(cfl_rec))
    print("wrote cfl", flush=True)

    # two-fluid drag, LogTrap2 / LogTrap3
    shape = (16, 8, 1)
    n = 128
    rng = np.random.Generator(np.random.Philox(41))
    cube = (1, 8, 16)
    rho_g = 1.0 + 0.1 * rng.uniform(-1, 1, n)
    gas = problems.pack(shape, rho_g.reshape(cube), 0, (rho_g * rng.uniform(-1e-2, 1e-2, n)).reshape(cube),
                        (rho_g * rng.uniform(-1e-2, 1e-2, n)).reshape(cube), 0)
    gas[1, :n] = 1.0 / (5 / 3.0 - 1) + 0.5 * (gas[2, :n] ** 2 + gas[3, :n] ** 2) / rho_g
    rho_d = rho_g * 10 ** rng.uniform(-2, 0, n)
    dust = problems.pack(shape, rho_d.reshape(cube), 0, (rho_d * rng.uniform(-2e-2, 2e-2, n)).reshape(cube), 0, 0)
    dust[1, :n] = 0.5 * dust[2, :n] ** 2 / rho_d + 1e-4 * rho_d
    drag = {"gas": gas, "dust": dust}
    tg = np.array(TG)
    # ETDRK2 (method 3) has its own states with a pressure gradient: etdrk2_golden
    for case, tdv in (("", TD), ("stiff_", TD_STIFF)):
        td = np.array(tdv)
        for method in (0, 1, 2, 4, 5):
            for strict in (False, True):
                g, d = gas.copy(), dust.copy()
                rc = lib("ospre", strict).ref_drag(P(g), P(d), shape[0], shape[1], shape[2], g.shape[1], P(tg),
                                                   P(td), 0.05, method)
                assert rc == 0
                tag = "%sm%d_%s" % (case, method, "strict" if strict else "fast")
                drag["gas_" + tag] = g
                drag["dust_" + tag] = d
    np.savez_compressed(os.path.join(outdir, "drag.npz"), meta=json.dumps({"shape": list(shape), "tg": TG, "td": TD,
                                                                          "td_stiff": TD_STIFF, "dt": 0.05}),
                        **drag)
    print("wrote drag", flush=True)
    etdrk2_golden(outdir)
    with open(os.path.join(outdir, "index.json"), "w") as f:
        json.dump(index, f, indent=1)


# ---- cylindrical geometry (x = r, y = theta, z = z) ----
CYL_H = [0.05, 0.04, 0.1]   # dr, dtheta, dz: dtheta != dr shows which spacing the theta sweeps use
CYL_RIN = 1.0
# single sweeps: name, shape, method, c_iso; each along r (dir 1) and theta in both layouts
CYL_SWEEP_CASES = [
    ("hllc3d", (32, 32, 6), 2, -1.0),
    ("hll3d", (32, 32, 6), 1, -1.0),
    ("xj3d", (32, 32, 6), 3, -1.0),
    ("hllc2d", (32, 24, 1), 2, -1.0),
    ("hll2d", (32, 24, 1), 1, -1.0),
    ("hlliso2d", (32, 24, 1), 1, 0.8),
]
CYL_SWEEPS = [(1, 0), (2, 0), (2, 1)]   # (dir, theta layout 0 = theta,r,z / 1 = theta,z,r)
# the cylindrical fixture keeps the strict build's outputs only (the bit-exact pin of the oracle;
# the library's product build is checked against the oracle within 1e-12), to stay small
CYL_VARIANTS = (True,)
# main loops with the cylinder source: name, shape, method, gamma, c_iso, bc, cfl, niter.  Xin-Jin
# runs at extents its launch covers (32), and never on a 2-D grid, where its theta sweep in the
# theta,z,r layout indexes outside its arrays.
CYL_RUN_CASES = [
    ("cyl_hllc_3d", (24, 20, 6), 2, 1.4, -1.0, ["const", "const"] + ["circular"] * 4, 0.4, 6),
    ("cyl_hll_2d", (24, 32, 1), 1, 1.4, -1.0, ["const", "const"] + ["circular"] * 4, 0.4, 6),
    ("cyl_hllc_2d", (24, 32, 1), 2, 5 / 3.0, -1.0, ["mirror", "const"] + ["circular"] * 4, 0.4, 6),
    ("cyl_hlliso_2d", (24, 32, 1), 1, 1.4, 0.8, ["const", "const"] + ["circular"] * 4, 0.4, 6),
    ("cyl_xj_3d", (32, 32, 32), 3, 1.4, -1.0, ["const", "const"] + ["circular"] * 4, 0.3, 4),
]


def cyl_lib(strict):
    L = lib("ospre", strict)
    dp = ctypes.POINTER(ctypes.c_double)
    i64, dbl, cint = ctypes.c_int64, ctypes.c_double, ctypes.c_int
    L.ref_sweep_cyl.argtypes = [dp, cint, cint, cint, i64, dbl, dbl, dbl, cint, dp, dbl, cint, cint, dbl]
    L.ref_cyl_source.argtypes = [dp, cint, cint, cint, i64, dp, dbl, dbl]
    L.ref_cfl_cyl.argtypes = [dp, cint, cint, cint, i64, dbl, cint, dp, dbl, dp]
    L.ref_run_cyl.argtypes = [dp, cint, cint, cint, i64, dbl, dbl, dbl, cint, dp, dbl,
                              ctypes.POINTER(ctypes.c_int), dbl, cint, dp]
    return L


def cyl_golden(outdir):
    h = np.array(CYL_H)
    rec, meta = {}, {"h": CYL_H, "r_inner": CYL_RIN, "sweeps": [], "runs": [], "dt": 0.004}
    for name, shape, method, c_iso in CYL_SWEEP_CASES:
        q0 = problems.rotating_annulus(shape, r_inner=CYL_RIN, dr=CYL_H[0], seed=37)
        rec["in_" + name] = q0
        for d, form in CYL_SWEEPS:
            for strict in CYL_VARIANTS:
                q = q0.copy()
                rc = cyl_lib(strict).ref_sweep_cyl(P(q), shape[0], shape[1], shape[2], q.shape[1], 1.4, 1e-5, c_iso,
                                                   method, P(h), CYL_RIN, d, form, 0.004)
                assert rc == 0, (name, d, form, rc)
                rec["out_%s_d%d_f%d_%s" % (name, d, form, "strict" if strict else "fast")] = q
        meta["sweeps"].append(dict(name=name, shape=list(shape), method=method, c_iso=c_iso))
        print("wrote cyl sweeps", name, flush=True)
    # CFL and the source term on one state; a cold copy makes the source's pressure reset act
    q0 = problems.rotating_annulus((24, 20, 6), r_inner=CYL_RIN, dr=CYL_H[0], seed=41)
    cold = q0.copy()
    n = 24 * 20 * 6
    cold[1, :n] = 0.5 * (cold[2, :n] ** 2 + cold[3, :n] ** 2 + cold[4, :n] ** 2) / cold[0, :n] + 1e-7
    rec["src_in"], rec["src_cold_in"] = q0, cold
    for strict in CYL_VARIANTS:
        tag = "strict" if strict else "fast"
        for key, src in (("src", q0), ("src_cold", cold)):
            q = src.copy()
            assert cyl_lib(strict).ref_cyl_source(P(q), 24, 20, 6, q.shape[1], P(h), CYL_RIN, 0.05) == 0
            rec["%s_out_%s" % (key, tag)] = q
        for shape in ((24, 20, 6), (24, 20, 1), (24, 1, 1)):
            qs = problems.rotating_annulus(shape, r_inner=CYL_RIN, dr=CYL_H[0], seed=43)
            rec["cfl_in_%dx%dx%d" % shape] = qs
            for method in (1, 2, 3):
                t = ctypes.c_double(0)
                assert cyl_lib(strict).ref_cfl_cyl(P(qs), shape[0], shape[1], shape[2], qs.shape[1], 1.4, method,
                                                   P(h), CYL_RIN, ctypes.byref(t)) == 0
                rec["cfl_%dx%dx%d_m%d_%s" % (shape + (method, tag))] = np.array(t.value)
    print("wrote cyl source and cfl", flush=True)
    for name, shape, method, gamma, c_iso, bc, cfl, niter in CYL_RUN_CASES:
        q0 = problems.rotating_annulus(shape, r_inner=CYL_RIN, dr=CYL_H[0], gamma=gamma, seed=47)
        rec["run_in_" + name] = q0
        bca = (ctypes.c_int * 6)(*[BC[b] for b in bc])
        for strict in CYL_VARIANTS:
            q = q0.copy()
            dts = np.zeros(niter)
            rc = cyl_lib(strict).ref_run_cyl(P(q), shape[0], shape[1], shape[2], q.shape[1], gamma, 1e-5, c_iso,
                                             method, P(h), CYL_RIN, bca, cfl, niter, P(dts))
            assert rc == 0, (name, rc)
            tag = "strict" if strict else "fast"
            rec["run_out_%s_%s" % (name, tag)] = q
            rec["run_dts_%s_%s" % (name, tag)] = dts
        meta["runs"].append(dict(name=name, shape=list(shape), method=method, gamma=gamma, c_iso=c_iso, bc=bc,
                                 cfl=cfl, niter=niter))
        print("wrote cyl run", name, flush=True)
    np.savez_compressed(os.path.join(outdir, "cylindrical.npz"), meta=json.dumps(meta), **rec)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    sel = [a.split("=", 1)[1].split(",") for a in sys.argv[1:] if a.startswith("--cases=")]
    out = args[0] if args else os.path.dirname(os.path.abspath(__file__))
    if "--cyl-only" in sys.argv:
        os.makedirs(out, exist_ok=True)
        cyl_golden(out)
    else:
        main(out, only="etdrk2" if "--etdrk2-only" in sys.argv else None, cases=sel[0] if sel else None)
