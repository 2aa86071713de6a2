"""Learned drag: training kernels against the CPU oracle, tensor-core inference against a BF16
emulation, exact labels against the restated drag law, what training gains, and the learned
drag step (conservation, fallback to the exact integrator)."""
import numpy as np
import pytest
import torch

import gpuimogen_b200 as ib
from gpuimogen_b200 import learned_drag as ld
from helpers import bits_equal
from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu


def random_params(seed):
    p = ld.init_params(seed).cpu()
    g = torch.Generator().manual_seed(seed + 7)
    for a, b in (("B1", "W2"), ("B2", "W3"), ("B3", "W4")):
        p[ib.imogen.MLP_OFF[a]:ib.imogen.MLP_OFF[b]] = 0.1 * torch.randn(64, generator=g)
    p[ib.imogen.MLP_OFF["B4"]] = 0.3
    w1 = 0.5 * torch.randn(64, 16, generator=g)
    w1[:, 14:] = 0  # inputs 14 and 15 are reserved for the bias on the tensor cores
    p[ib.imogen.MLP_OFF["W1"]:ib.imogen.MLP_OFF["B1"]] = w1.reshape(-1)  # inputs 0..13 live
    return p.cuda()


def test_mlp_loss_gradient_matches_oracle(cuda, ib):
    p = random_params(3)
    n = 300  # not a multiple of the 64-sample tile
    g = torch.Generator().manual_seed(5)
    x = torch.randn(n, 16, generator=g).cuda()
    t = torch.randn(n, generator=g).cuda()
    tr = ld.Trainer(p.clone(), batch=n)
    grad, loss = tr.loss_grad(x, t)
    torch.cuda.synchronize()
    loss_ref, grad_ref = mo.loss_grad(p.cpu().numpy(), x.cpu().numpy(), t.cpu().numpy())
    assert abs(float(loss) - loss_ref) <= 1e-5 * loss_ref
    got = grad.cpu().numpy().astype(np.float64)
    for a, b in (("W1", "B1"), ("B1", "W2"), ("W2", "B2"), ("B2", "W3"), ("W3", "B3"), ("B3", "W4"), ("W4", "B4")):
        lo, hi = ib.imogen.MLP_OFF[a], ib.imogen.MLP_OFF[b]
        err = np.abs(got[lo:hi] - grad_ref[lo:hi]).max() / max(np.abs(grad_ref[lo:hi]).max(), 1e-30)
        assert err <= 1e-4, (a, err)
    assert abs(got[mo.OFF_B4] - grad_ref[mo.OFF_B4]) <= 1e-5 * max(1e-6, abs(grad_ref[mo.OFF_B4]))
    y = ld.forward_fp32(p, x)
    y_ref, _ = mo.forward(p.cpu().numpy(), x.cpu().numpy())
    assert np.abs(y.cpu().numpy() - y_ref).max() <= 1e-4 * (1 + np.abs(y_ref).max())


def test_tensor_core_inference_matches_bf16_emulation(cuda, ib):
    """tcgen05 MLP (BF16 operands, FP32 accumulation in tensor memory) against the oracle's
    step-by-step emulation of the kernel's roundings, and against the FP32 network.  The hardware's
    summation order inside one MMA is not the emulation's, so an FP32 sum can differ in its last
    bit and, where that straddles a BF16 rounding boundary, one hidden activation moves by one
    BF16 step (2^-8 relative); most cells agree to FP32 rounding."""
    p = random_params(11)
    n = 1000  # not a multiple of the 128-cell tile
    x = torch.randn(n, 16, generator=torch.Generator().manual_seed(13))
    x[:, 14:] = 0
    x = x.cuda()
    y = ld.forward_tc(p, x).cpu().numpy().astype(np.float64)
    y_tc = mo.forward_tc_emulation(p.cpu().numpy(), x.cpu().numpy())
    y32, _ = mo.forward(p.cpu().numpy(), x.cpu().numpy())
    scale = np.abs(y32).max()
    assert ib.device_wait_status() == 0
    d = np.abs(y - y_tc)
    assert np.median(d) <= 1e-6 * scale, np.median(d)
    assert np.mean(d <= 1e-5 * scale) >= 0.95, np.mean(d <= 1e-5 * scale)
    assert d.max() <= 1e-2 * scale, d.max()
    assert np.abs(y - y32).max() <= 6e-2 * scale  # BF16 rounding of weights and activations


def _exact_params(seed):
    """A network whose every FP32 sum is exact: weights on coarse binary grids (W1 multiples of
    1/32 up to 1/4, W2 and W3 of 1/32 up to 1/8, biases of 1/64), so that the result does not
    depend on the order in which the tensor cores add."""
    g = np.random.Generator(np.random.Philox(seed))
    p = np.zeros(ib.imogen.MLP_NPARAM, dtype=np.float32)
    O = ib.imogen.MLP_OFF
    w1 = g.integers(-8, 9, (64, 16)) / 32.0
    w1[:, 14:] = 0
    p[O["W1"]:O["B1"]] = w1.ravel()
    p[O["B1"]:O["W2"]] = g.integers(-8, 9, 64) / 64.0
    p[O["W2"]:O["B2"]] = g.integers(-4, 5, 64 * 64) / 32.0
    p[O["B2"]:O["W3"]] = g.integers(-8, 9, 64) / 64.0
    p[O["W3"]:O["B3"]] = g.integers(-4, 5, 64 * 64) / 32.0
    p[O["B3"]:O["W4"]] = g.integers(-8, 9, 64) / 64.0
    p[O["W4"]:O["B4"]] = g.integers(-8, 9, 64) / 64.0
    p[O["B4"]] = 0.25
    return p


def _sums_exact(p, x):
    """Per row: True where every partial sum of every layer's MMAs is an exact FP32 value (the sum
    of the terms' magnitudes, in units of the finest grid, below 2^24)."""
    W1, b1, W2, b2, W3, b3, w4, b4 = mo.unpack(p)
    a = mo.to_bf16(x.astype(np.float32))
    a[:, 14:16] = 0
    ok = np.ones(len(x), dtype=bool)
    # units: inputs 1/16, W1 1/32 -> 2^-9; hidden values stay on grids as fine as 2^-9, 2^-14, 2^-19
    for W, unit, last in ((W1, 2.0 ** -9, False), (W2, 2.0 ** -14, False), (W3, 2.0 ** -19, True)):
        mag = np.abs(a) @ np.abs(W).T
        ok &= np.all(mag / unit < 2 ** 24, axis=1)
        z = np.maximum(a @ W.T + (b1 if W is W1 else (b2 if W is W2 else b3)), 0)
        a = z if last else mo.to_bf16(z.astype(np.float32))
    return ok


def test_tensor_core_inference_exact_arithmetic(cuda, ib):
    """With a network and inputs on coarse binary grids every tensor-core sum is exact, so the
    kernel must reproduce the emulation to the rounding of its final FP32 output sums: a wrong
    weight layout, row mapping or bias split shows up here at once."""
    p = _exact_params(5)
    n = 2000
    g = np.random.Generator(np.random.Philox(6))
    x = (g.integers(-16, 17, (n, 16)) / 16.0).astype(np.float32)
    x[:, 14:] = 0
    ok = _sums_exact(p, x)
    assert ok.mean() >= 0.9, ok.mean()
    y = ld.forward_tc(torch.from_numpy(p).cuda(), torch.from_numpy(x).cuda()).cpu().numpy().astype(np.float64)
    y_tc = mo.forward_tc_emulation(p, x)
    scale = max(np.abs(y_tc).max(), 1.0)
    assert ib.device_wait_status() == 0
    d = np.abs(y - y_tc)
    assert d[ok].max() <= 1e-6 * scale, d[ok].max()
    assert d.max() <= 1e-4 * scale, d.max()


def test_exact_decay_matches_oracle_drag_law(cuda, ib):
    f = ld.sample_features(20000, seed=4)
    s = ld.exact_decay(f).cpu().numpy()
    fc = f.cpu().numpy()
    d = mo.drag_constants(ld.THERMO_GAS, ld.THERMO_DUST)
    s_ref = mo.decay_logtrap2(d, fc[:, 0], fc[:, 1], fc[:, 2], fc[:, 3], fc[:, 4])
    assert np.all(np.isfinite(s)) and np.all(s > 0)
    assert np.max(np.abs(s - s_ref) / s_ref) <= 1e-12


@pytest.fixture(scope="module")
def trained(cuda, ib):
    model, hist = ld.train(n_samples=400_000, epochs=6, seed=77, batch=8192, lr=3e-3)
    return model, hist


def test_training_gain_over_untrained_network(trained):
    """What the trained network gains: prediction error of log s and of the decay factor against
    the exact integrator, before and after training on its labels."""
    model, hist = trained
    untrained = ld.DragModel(params=ld.init_params(78), feature_shift=model.feature_shift,
                             feature_scale=model.feature_scale, out_shift=model.out_shift,
                             out_scale=model.out_scale)
    e0 = ld.evaluate(untrained, n=200_000, seed=5)
    e1 = ld.evaluate(model, n=200_000, seed=5)
    assert hist["val_rmse_log_s"][-1] < hist["val_rmse_log_s"][0]
    assert e1["rmse_log_s"] < 0.2 * e0["rmse_log_s"], (e0, e1)
    assert e1["rmse_decay"] < 0.2 * e0["rmse_decay"], (e0, e1)


def _pair(shape, seed, outside=0):
    nx, ny = shape
    n = nx * ny
    rng = np.random.Generator(np.random.Philox(seed))
    rg = 1.0 + 0.2 * rng.uniform(-1, 1, n)
    rd = rg * np.exp(rng.uniform(np.log(0.01), 0, n))
    vg = rng.uniform(-1e-2, 1e-2, (3, n))
    vd = rng.uniform(-1e-2, 1e-2, (3, n))
    P = 1.0 + 0.1 * rng.uniform(-1, 1, n)
    if outside:
        rd[:outside] = 10.0  # above the trained dust-density box: these cells take the exact path
    S = ib.slab_pitch(nx, ny, 1)
    gas = np.zeros((5, S))
    dust = np.zeros((5, S))
    gas[0, :n], dust[0, :n] = rg, rd
    gas[2:5, :n], dust[2:5, :n] = rg * vg, rd * vd
    gas[1, :n] = P / (5 / 3.0 - 1) + 0.5 * rg * (vg ** 2).sum(0)
    dust[1, :n] = 0.5 * rd * (vd ** 2).sum(0) + 1e-4 * rd
    return gas, dust


def test_learned_drag_step_conserves_and_falls_back(trained, ib):
    model, _ = trained
    shape = (96, 80)
    n = shape[0] * shape[1]
    outside = 37
    gas, dust = _pair(shape, seed=21, outside=outside)
    mk = lambda q: ib.Fluid((shape[0], shape[1], 1), q=torch.from_numpy(q.copy()).cuda(), gamma=5 / 3.0)
    g1, d1, g2, d2 = mk(gas), mk(dust), mk(gas), mk(dust)
    dt = 2e-5
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    ld.drag_step(g1, d1, model, dt, fallback_counter=cnt)
    geo = ib.Geometry((shape[0], shape[1], 1))
    ib.cudaSource2FluidDrag(g2, d2, ld.THERMO_GAS, ld.THERMO_DUST, geo, [dt, ib.DRAG["logtrap2"]])
    torch.cuda.synchronize()
    assert int(cnt.item()) == outside
    G1, D1 = g1.q.cpu().numpy(), d1.q.cpu().numpy()
    G2, D2 = g2.q.cpu().numpy(), d2.q.cpu().numpy()
    # cells outside the trained box ran the exact integrator: identical to the exact step
    assert bits_equal(G1[:, :outside], G2[:, :outside], outside) and bits_equal(D1[:, :outside], D2[:, :outside], outside)
    # momentum: per cell, gas + dust momentum unchanged; energy: gas heating = dust KE loss
    p0 = gas[2:5, :n] + dust[2:5, :n]
    assert np.abs(G1[2:5, :n] + D1[2:5, :n] - p0).max() <= 1e-15 * 50
    # relative velocity after the step against the exact integrator
    dv = lambda G, D: G[2:5, :n] / G[0, :n] - D[2:5, :n] / D[0, :n]
    dv0 = dv(gas, dust)
    err = np.abs(dv(G1, D1) - dv(G2, D2)).max() / np.abs(dv0).max()
    assert err <= 2e-2, err
    assert np.all(np.isfinite(G1[:, :n])) and np.all(np.isfinite(D1[:, :n]))
