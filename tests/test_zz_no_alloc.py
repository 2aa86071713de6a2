"""GPU test of ib_cflTimestepNoAlloc, the CFL entry point that allocates no device memory.

Callers that cannot let the library call cudaMalloc, such as an application that has reserved
the GPU's memory for its own allocator or a loop that must not pay for the device-wide
synchronisation cudaMalloc and cudaFree can cause, use this variant.  It keeps its reduction
scratch in a fixed array built into the library.  Through the C ABI this test checks that it
returns the same timestep as ib_cflTimestepFused on two calls in a row, and that a grid beyond
the fixed scratch limit is refused with IB_ERROR_INVALID_ARGS.
"""
import ctypes

import numpy as np
import pytest
import torch

from gpuimogen_b200 import imogen, problems

pytestmark = pytest.mark.gpu

INVALID_ARGS = -100
MAX_CELLS = 8192 * 256 * 64


def _fluid_struct(q, shape):
    f = imogen.IbFluid()
    f.q = q.data_ptr()
    nx, ny, nz = shape
    f.grid = imogen.IbGrid(nx, ny, nz, 0, q.shape[1])
    f.halo = 4
    return f


def _geometry(shape):
    g = imogen.IbGeometry()
    for i in range(3):
        g.h[i] = 1.0 / shape[i]
        g.global_rez[i] = shape[i]
    return g


# 256^3 folds the minima of hundreds of reduction blocks (4 per SM); (300, 1, 1) with method 3
# is the 1-D Xin-Jin case, which takes the HLL reduction without the halving
@pytest.mark.parametrize("shape,method", [((64, 48, 40), 2), ((64, 48, 40), 3), ((300, 1, 1), 1),
                                          ((300, 1, 1), 3), ((200, 150, 1), 2), ((256, 256, 256), 2)])
def test_no_alloc_cfl_matches_fused(shape, method):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L = imogen.load("product")
    q = torch.from_numpy(problems.random_jumpy(shape, gamma=1.4, seed=17)).cuda()
    f = _fluid_struct(q, shape)
    g = _geometry(shape)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    ref = ctypes.c_double(0.0)
    rc = L.ib_cflTimestepFused(ctypes.byref(f), 1.4, ctypes.byref(g), method, ctypes.byref(ref), None, stream)
    assert rc == 0
    assert np.isfinite(ref.value) and ref.value > 0

    out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda")
    for call in range(2):  # the shared scratch must be reusable by the next call
        rc = L.ib_cflTimestepNoAlloc(ctypes.byref(f), 1.4, ctypes.byref(g), method,
                                     ctypes.c_void_p(out.data_ptr() + 8 * call), stream)
        assert rc == 0
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    # same tolerance as the other CFL device-result tests; the minimum itself is order-free
    assert np.all(np.abs(got - ref.value) <= 1e-15 * ref.value), (got, ref.value)


def test_no_alloc_rejects_grid_beyond_scratch_limit():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L = imogen.load("product")
    shape = (512, 512, 513)  # 134,479,872 cells > 134,217,728
    n = shape[0] * shape[1] * shape[2]
    assert n > MAX_CELLS
    q = torch.empty((5, imogen.slab_pitch(*shape)), dtype=torch.float64, device="cuda")
    f = _fluid_struct(q, shape)
    g = _geometry(shape)
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    rc = L.ib_cflTimestepNoAlloc(ctypes.byref(f), 1.4, ctypes.byref(g), 2, ctypes.c_void_p(out.data_ptr()),
                                 ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == INVALID_ARGS
    torch.cuda.synchronize()
    assert out.item() == -1.0  # nothing was launched
    del q
    torch.cuda.empty_cache()
