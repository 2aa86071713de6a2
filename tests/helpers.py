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
