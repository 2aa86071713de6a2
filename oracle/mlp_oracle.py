"""CPU oracle for the drag-decay MLP (TEST INFRASTRUCTURE ONLY: used by tests/ as the checker).

The network of include/imogen_b200.h (16 inputs, 3 x 64 ReLU, 1 linear output, parameters in
one vector at the IB_MLP_OFF_* offsets) restated in numpy:
  * forward(params, x)           FP64 forward pass
  * loss_grad(params, x, target) mean squared error and its gradient by back-propagation, FP64
  * forward_bf16(params, x)      the tensor-core arithmetic: weights and every layer input rounded
                                 to BF16 (round to nearest even), products summed exactly (FP64),
                                 bias and ReLU in FP32 after the sum
  * forward_tc_emulation(p, x)   the tensor-core kernel's own order of roundings (bias split into
                                 BF16 parts inside the first MMA, FP32 accumulation per K = 16 MMA,
                                 FP32 output sums)
and a restatement of the drag law's LogTrap2 decay exponent (cudaSource2FluidDrag.cu:819-890,
1531-1660) for spot checks of the exact training targets.
"""
import numpy as np

IN, H = 16, 64
OFF_W1, OFF_B1, OFF_W2, OFF_B2, OFF_W3, OFF_B3, OFF_W4, OFF_B4, NPARAM = (0, 1024, 1088, 5184, 5248, 9344, 9408,
                                                                          9472, 9473)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[OFF_W1:OFF_B1].reshape(H, IN), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(H, H), p[OFF_B2:OFF_W3],
            p[OFF_W3:OFF_B3].reshape(H, H), p[OFF_B3:OFF_W4], p[OFF_W4:OFF_B4], p[OFF_B4])


def forward(p, x):
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(p)
    x = np.asarray(x, dtype=np.float64)
    h1 = np.maximum(x @ W1.T + b1, 0)
    h2 = np.maximum(h1 @ W2.T + b2, 0)
    h3 = np.maximum(h2 @ W3.T + b3, 0)
    return h3 @ w4 + b4, (x, h1, h2, h3)


def loss_grad(p, x, target):
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(p)
    y, (x, h1, h2, h3) = forward(p, x)
    n = len(y)
    e = y - np.asarray(target, dtype=np.float64)
    loss = float(np.mean(e * e))
    dy = 2 * e / n
    g = np.zeros(NPARAM)
    g[OFF_W4:OFF_B4] = h3.T @ dy
    g[OFF_B4] = dy.sum()
    d3 = np.outer(dy, w4) * (h3 > 0)
    g[OFF_W3:OFF_B3] = (d3.T @ h2).ravel()
    g[OFF_B3:OFF_W4] = d3.sum(0)
    d2 = (d3 @ W3) * (h2 > 0)
    g[OFF_W2:OFF_B2] = (d2.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = d2.sum(0)
    d1 = (d2 @ W2) * (h1 > 0)
    g[OFF_W1:OFF_B1] = (d1.T @ x).ravel()
    g[OFF_B1:OFF_W2] = d1.sum(0)
    return loss, g


def to_bf16(a):
    """Round FP32 values to BF16 (round to nearest even), returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def forward_bf16(p, x):
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(np.asarray(p, dtype=np.float32))
    a = to_bf16(x)
    for W, b, last in ((W1, b1, False), (W2, b2, False), (W3, b3, True)):
        z = (a @ to_bf16(W).T).astype(np.float32) + b.astype(np.float32)
        h = np.maximum(z, np.float32(0))
        a = h.astype(np.float64) if last else to_bf16(h)
    return a @ w4 + b4


def _f32(a):
    return np.asarray(a, dtype=np.float64).astype(np.float32).astype(np.float64)


def forward_tc_emulation(p, x):
    """The tensor-core kernel's arithmetic step by step (ib_drag_learned.cu, mlp_tc_kernel):
    layer 1 is one K = 16 MMA whose inputs 14 and 15 are 1 and whose weight columns there hold the
    bias as BF16 high part and BF16 remainder; layers 2 and 3 are four K = 16 MMAs accumulated in
    FP32 (each chunk's products summed exactly, then added to the FP32 accumulator); hidden biases
    are added in FP32 before ReLU and the BF16 conversion; the output is b4 + the FP32 fused
    multiply-add sums of the even and of the odd hidden units."""
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(np.asarray(p, dtype=np.float32))
    n = len(x)
    a = to_bf16(np.asarray(x, dtype=np.float32))
    a[:, 14:16] = 1.0
    Wb = to_bf16(W1)
    hi = to_bf16(b1.astype(np.float32))
    lo = to_bf16((b1.astype(np.float32) - hi.astype(np.float32)).astype(np.float32))
    Wb[:, 14], Wb[:, 15] = hi, lo
    z = _f32(a @ Wb.T)
    a = to_bf16(np.maximum(z, 0).astype(np.float32))
    for W, b in ((W2, b2), (W3, b3)):
        Wq = to_bf16(W)
        acc = np.zeros((n, H))
        for c in range(0, H, 16):
            acc = _f32(acc + _f32(a[:, c:c + 16] @ Wq[:, c:c + 16].T))
        z = np.maximum(_f32(acc + _f32(b)), 0)
        a = to_bf16(z.astype(np.float32)) if W is W2 else z
    w4 = _f32(w4)
    ye, yo = np.zeros(n), np.zeros(n)
    for j in range(0, H, 2):
        ye = _f32(w4[j] * a[:, j] + ye)
        yo = _f32(w4[j + 1] * a[:, j + 1] + yo)
    return _f32(_f32(b4) + _f32(ye + yo))


def drag_constants(tg, td):
    """dragparams[0..6] (cudaSource2FluidDrag.cu:196-218) from 8-element thermo vectors
    [gamma, mass, mu0, mu_t_index, sigma0, sigma_t_index, k_bolt, c_isothermal]."""
    gam = tg[0]
    ddust = np.sqrt(td[4] / 3.141592653589793)
    return dict(viscpow=-tg[3], lampow=tg[5], alpha=tg[1] * (gam - 1.0) / (298.15 * tg[6]),
                beta=np.sqrt(2.0) * tg[1] / (tg[4] * ddust), delta=ddust / tg[2], epsilon=td[4] / (1.0 * td[1]))


def _k(d, rg, rd, dv, u):
    with np.errstate(all="ignore"):  # cells below the no-drag cut evaluate to 0 below
        return _k_raw(d, rg, rd, dv, u)


def _k_raw(d, rg, rd, dv, u):
    Tn = d["alpha"] * u
    Re = d["delta"] * rg * dv * Tn ** d["viscpow"]
    Kn = d["beta"] * Tn ** d["lampow"] / rg
    cun = 1 + Kn * (1.142 + 0.558 * np.exp(-0.999 / Kn))
    cd = (3 / Re + .45 * Re ** -.319 + .0509 * Re / (8710 + Re)) / cun
    return np.where(dv < 1e-9, 0.0, cd * dv * (rg + rd) * d["epsilon"])


def decay_logtrap2(d, rg, rd, dv, u, dt):
    """s = dt k_eff of LogTrap2 (cukern_LogTrapSolve<2>)."""
    mu = rd / (rg + rd)
    k0 = _k(d, rg, rd, dv, u)
    dv1 = dv * np.exp(-dt * k0)
    duint = -.5 * dv * dv * mu * np.expm1(-2 * k0 * dt)
    k1 = _k(d, rg, rd, dv1, u + duint)
    return dt * .5 * (k0 + k1)
