"""CPU tests of the GPU-tag decoders (host code: no device is touched).

Tags are built by hand in the layout of the reference (gpuclass/cudaCommon.h:184-196, written by
serializeMGArrayToTag, cudaCommon.cu:172-196): a fluid's mass, ener and mom(1..3) are slabs of one
MGA_allocSlab allocation (cudaCommon.cu:339-370) whose pitch is numel * 8 bytes rounded up to
256.  The decoders must accept what sanityCheckTag (cudaCommonML.cu:109-198) accepts and this
library can run, and refuse the rest with the reference's status codes.
"""
import ctypes

import numpy as np
import pytest

from gpuimogen_b200 import imogen

INVALID_ARGS, NULL_POINTER, NOIMPLEMENT = -100, -102, -105
BASE = 0x7F4047000000


def lib():
    return imogen.load("product")


def make_tag(dims, ptr, vec, circ=63, perm=1, ngpu=1, dev=0, halo=0, slab=0):
    t = [dims[0], dims[1], dims[2], slab, halo, 1, ngpu, 0, perm, circ, vec]
    for g in range(ngpu):
        t += [dev, ptr + g * 4096]
    return np.array(t, dtype=np.int64)


def fluid_tags(dims, circ=63, **kw):
    n = dims[0] * dims[1] * dims[2]
    pitch = (n * 8 + 255) // 256 * 256
    vecs = [0, 0, 1, 2, 3]
    slabs = [5, -1, -2, -3, -4]
    return [make_tag(dims, BASE + k * pitch, vecs[k], circ=circ, slab=slabs[k], **kw) for k in range(5)]


def decode(L, tags, bc=None):
    keep = [np.ascontiguousarray(t) for t in tags]
    ptrs = (ctypes.c_void_p * 5)(*[t.ctypes.data for t in keep])
    lens = (ctypes.c_int32 * 5)(*[len(t) for t in keep])
    f = imogen.IbFluid()
    bcs = (ctypes.c_int32 * 6)(*bc) if bc is not None else None
    rc = L.ib_fluidFromGpuTags(ptrs, lens, bcs, ctypes.byref(f))
    return rc, f


def test_fluid_from_tags_periodic():
    L = lib()
    dims = (20, 16, 12)
    rc, f = decode(L, fluid_tags(dims))
    assert rc == 0
    assert f.q == BASE
    assert (f.grid.nx, f.grid.ny, f.grid.nz) == dims
    # 3840 cells * 8 B = 30720 B, a multiple of 256: the pitch is the cell count
    assert f.grid.slab_pitch == 3840 == imogen.slab_pitch(*dims)
    assert list(f.bc) == [imogen.BC["circular"]] * 6
    assert f.halo == 4


def test_fluid_from_tags_pitch_rounding_and_modes():
    L = lib()
    dims = (37, 11, 9)   # 3663 cells: 29304 B rounded to 29440 B = 3680 doubles
    modes = [ib for ib in (L.ib_bcModeFromString(s) for s in
                           (b"const", b"const", b"mirror", b"outflow", b"circ", b"circ"))]
    assert modes == [4, 4, 1, 6, 0, 0]
    # only the z faces share halos circularly (MGA_BOUNDARY_ZMINUS | ZPLUS = 16 | 32)
    rc, f = decode(L, fluid_tags(dims, circ=48), bc=modes)
    assert rc == 0
    assert f.grid.slab_pitch == 3680
    assert list(f.bc) == modes


def test_bc_strings():
    L = lib()
    names = {b"circ": 0, b"mirror": 1, b"wall": 2, b"bcstatic": 3, b"const": 4, b"linear": 5, b"outflow": 6,
             b"freebalance": 7}
    for s, v in names.items():
        assert L.ib_bcModeFromString(s) == v
    assert L.ib_bcModeFromString(b"periodic") == INVALID_ARGS


@pytest.mark.parametrize("case,expect", [
    ("two_gpus", NOIMPLEMENT),          # the library runs on one GPU
    ("permuted", NOIMPLEMENT),          # arrays must be in XYZ order (permtag 1)
    ("bad_permtag", INVALID_ARGS),      # sanityCheckTag: permtag in 0..6
    ("short", INVALID_ARGS),            # fewer than 11 entries
    ("len_mismatch", INVALID_ARGS),     # length != 11 + 2 nGPUs
    ("neg_dim", INVALID_ARGS),
    ("bad_vector", INVALID_ARGS),       # mom(2) tagged as component 1
    ("bad_device", INVALID_ARGS),       # device id outside 0..3
    ("not_slabs", NOIMPLEMENT),         # ener not one pitch after mass
    ("dims_differ", INVALID_ARGS),
    ("circ_vs_mode", INVALID_ARGS),     # a circular face given a const mode
    ("no_modes_not_circ", INVALID_ARGS),
])
def test_fluid_from_tags_rejects(case, expect):
    L = lib()
    dims = (16, 8, 4)
    tags = fluid_tags(dims)
    bc = None
    if case == "two_gpus":
        tags = [make_tag(dims, BASE, 0, ngpu=2)] + tags[1:]
    elif case == "permuted":
        tags[2] = make_tag(dims, int(tags[2][12]), 1, perm=3)
    elif case == "bad_permtag":
        tags[0][8] = 7
    elif case == "short":
        tags[0] = tags[0][:10]
    elif case == "len_mismatch":
        tags[1] = np.concatenate([tags[1], [0]])
    elif case == "neg_dim":
        tags[0][1] = -8
    elif case == "bad_vector":
        tags[3][10] = 1
    elif case == "bad_device":
        tags[4][11] = 4
    elif case == "not_slabs":
        tags[1][12] += 256
    elif case == "dims_differ":
        tags[4][2] = 5
    elif case == "circ_vs_mode":
        bc = [4, 4, 0, 0, 0, 0]
    elif case == "no_modes_not_circ":
        tags = fluid_tags(dims, circ=15)
    rc, _ = decode(L, tags, bc=bc)
    assert rc == expect, case


def test_array_from_tag():
    L = lib()
    t = make_tag((300, 5, 3), BASE, 2, circ=3)
    ptr = ctypes.c_void_p()
    g = imogen.IbGrid()
    vec, circ = ctypes.c_int32(-1), ctypes.c_int32(-1)
    rc = L.ib_arrayFromGpuTag(t.ctypes.data, len(t), ctypes.byref(ptr), ctypes.byref(g), ctypes.byref(vec),
                              ctypes.byref(circ))
    assert rc == 0
    assert ptr.value == BASE
    assert (g.nx, g.ny, g.nz, g.slab_pitch) == (300, 5, 3, 4512)   # 36000 B -> 36096 B
    assert vec.value == 2 and circ.value == 3
    t0 = make_tag((0, 0, 0), 0, 0)
    assert L.ib_arrayFromGpuTag(t0.ctypes.data, len(t0), ctypes.byref(ptr), ctypes.byref(g), None, None) != 0
