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


def bits_equal(a, b, n):
    return np.array_equal(a[:, :n].view(np.int64), b[:, :n].view(np.int64))


def first_diff(a, b, n):
    d = np.argwhere(a[:, :n].view(np.int64) != b[:, :n].view(np.int64))
    if len(d) == 0:
        return None
    k, i = d[0]
    return (int(k), int(i), float(a[k, i]), float(b[k, i]), len(d))
