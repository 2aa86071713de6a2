"""Learned two-fluid drag: data from the exact integrator, training on the GPU, tensor-core inference.

The LogTrap2 drag update of a cell is fixed by one number, the decay exponent s = dt * k_eff
of the gas-dust relative velocity.  This module
  * samples (rho_gas, rho_dust, |dv|, u, dt) states log-uniformly over a training box and labels
    them with the exact integrator (ib_dragDecayExact, FP64 LogTrap2);
  * trains the 16-64-64-64-1 ReLU network of include/imogen_b200.h on log s with the library's
    own FP32 training kernels (ib_mlpLossGrad: forward + back-propagation, ib_mlpAdam);
  * evaluates it on the tensor cores (ib_mlpInferTC) against held-out exact labels;
  * runs the learned drag step (ib_cudaSource2FluidDragLearned), where cells outside the trained
    box or with a non-finite prediction fall back to the exact integrator.
"""
import ctypes
import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import imogen as ib

# Drag microphysics of the 2-D gas-dust workload, in code units (gas: the reference's hydrogen
# values; dust: 5 micron grains with the mass scaled so that the stopping time is of the order
# of the CFL timestep of a 2048^2 unit box): [gamma, mass, mu0, mu_t_index, sigma0,
# sigma_t_index, k_bolt, c_isothermal]
THERMO_GAS = [5 / 3.0, 3.3e-27, 8.4e-6, 0.7, 2.4e-19, 0.2, 1.381e-23, -1.0]
THERMO_DUST = [1.01, 3e-19, 0.0, 0.0, math.pi * 25e-12, 0.0, 1.381e-23, 0.1]

# Training box of the raw features (natural log of rho_gas, rho_dust, |dv|, u, dt)
DOMAIN_LO = [math.log(0.5), math.log(0.005), math.log(1e-9), math.log(0.3), math.log(5e-7)]
DOMAIN_HI = [math.log(2.0), math.log(2.0), math.log(1.0), math.log(10.0), math.log(0.1)]


def thermo(v):
    return ib.IbThermo(*[float(a) for a in v])


@dataclass
class DragModel:
    params: torch.Tensor                      # IB_MLP_NPARAM float32 on the device
    feature_shift: list = field(default_factory=lambda: [0.0] * 5)
    feature_scale: list = field(default_factory=lambda: [1.0] * 5)
    out_shift: float = 0.0
    out_scale: float = 1.0
    domain_lo: list = field(default_factory=lambda: list(DOMAIN_LO))
    domain_hi: list = field(default_factory=lambda: list(DOMAIN_HI))

    def struct(self):
        m = ib.IbDragModel()
        m.params = self.params.data_ptr()
        for k in range(5):
            m.feature_shift[k] = self.feature_shift[k]
            m.feature_scale[k] = self.feature_scale[k]
            m.domain_lo[k] = self.domain_lo[k]
            m.domain_hi[k] = self.domain_hi[k]
        m.out_shift = self.out_shift
        m.out_scale = self.out_scale
        return m

    def state_dict(self):
        return {"params": self.params.cpu().numpy().tolist(), "feature_shift": self.feature_shift,
                "feature_scale": self.feature_scale, "out_shift": self.out_shift, "out_scale": self.out_scale,
                "domain_lo": self.domain_lo, "domain_hi": self.domain_hi}


def sample_features(n, seed, lo=DOMAIN_LO, hi=DOMAIN_HI, device="cuda"):
    """n x 5 raw features, log-uniform over the box (seeded)."""
    g = torch.Generator(device="cpu").manual_seed(seed)
    u = torch.rand(n, 5, generator=g, dtype=torch.float64)
    lo_t, hi_t = torch.tensor(lo, dtype=torch.float64), torch.tensor(hi, dtype=torch.float64)
    return torch.exp(lo_t + (hi_t - lo_t) * u).to(device)


def exact_decay(features, tg=THERMO_GAS, td=THERMO_DUST):
    """FP64 LogTrap2 decay exponent s for raw features (device n x 5)."""
    f = features.contiguous()
    s = torch.empty(f.shape[0], dtype=torch.float64, device=f.device)
    a, b = thermo(tg), thermo(td)
    ib._check("ib_dragDecayExact", ib._lib().ib_dragDecayExact(ctypes.c_void_p(f.data_ptr()), f.shape[0],
                                                               ctypes.byref(a), ctypes.byref(b),
                                                               ctypes.c_void_p(s.data_ptr()), ib._stream()))
    return s


def normalise(model, features):
    """n x 16 float32 network inputs for raw features."""
    lf = torch.log(features)
    shift = torch.tensor(model.feature_shift, dtype=torch.float64, device=features.device)
    scale = torch.tensor(model.feature_scale, dtype=torch.float64, device=features.device)
    x = torch.zeros(features.shape[0], ib.MLP_IN, dtype=torch.float32, device=features.device)
    x[:, :5] = ((lf - shift) * scale).float()
    return x


def init_params(seed, device="cuda"):
    """He-initialised parameters (seeded), zero biases."""
    g = torch.Generator(device="cpu").manual_seed(seed)
    p = torch.zeros(ib.MLP_NPARAM, dtype=torch.float32)
    def he(shape, fan_in):
        return torch.randn(*shape, generator=g) * math.sqrt(2.0 / fan_in)
    p[ib.MLP_OFF["W1"]:ib.MLP_OFF["B1"]] = torch.cat([he((64, 5), 5), torch.zeros(64, 11)], 1).reshape(-1)
    p[ib.MLP_OFF["W2"]:ib.MLP_OFF["B2"]] = he((64, 64), 64).reshape(-1)
    p[ib.MLP_OFF["W3"]:ib.MLP_OFF["B3"]] = he((64, 64), 64).reshape(-1)
    p[ib.MLP_OFF["W4"]:ib.MLP_OFF["B4"]] = he((64,), 64) * 0.5
    return p.to(device)


class Trainer:
    """Adam on the mean squared error of the normalised log s, with the library's kernels."""

    def __init__(self, params, lr=2e-3, beta1=0.9, beta2=0.999, eps=1e-8, batch=65536):
        self.p = params
        self.m = torch.zeros_like(params)
        self.v = torch.zeros_like(params)
        self.g = torch.zeros_like(params)
        self.loss = torch.zeros(1, dtype=torch.float32, device=params.device)
        self.lr, self.b1, self.b2, self.eps = lr, beta1, beta2, eps
        self.batch = batch
        self.work = torch.empty(int(ib._lib().ib_mlpWorkspaceFloats(batch)), dtype=torch.float32,
                                device=params.device)
        self.step_no = 0

    def loss_grad(self, x, t):
        n = x.shape[0]
        if self.work.numel() < ib._lib().ib_mlpWorkspaceFloats(n):
            self.work = torch.empty(int(ib._lib().ib_mlpWorkspaceFloats(n)), dtype=torch.float32, device=x.device)
        ib._check("ib_mlpLossGrad", ib._lib().ib_mlpLossGrad(
            ctypes.c_void_p(self.p.data_ptr()), ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(t.data_ptr()), n,
            ctypes.c_void_p(self.g.data_ptr()), ctypes.c_void_p(self.loss.data_ptr()),
            ctypes.c_void_p(self.work.data_ptr()), ib._stream()))
        return self.g, self.loss

    def step(self, x, t, lr=None):
        self.loss_grad(x, t)
        self.step_no += 1
        ib._check("ib_mlpAdam", ib._lib().ib_mlpAdam(
            ctypes.c_void_p(self.p.data_ptr()), ctypes.c_void_p(self.g.data_ptr()),
            ctypes.c_void_p(self.m.data_ptr()), ctypes.c_void_p(self.v.data_ptr()), self.p.numel(),
            ctypes.c_float(lr if lr is not None else self.lr), ctypes.c_float(self.b1), ctypes.c_float(self.b2),
            ctypes.c_float(self.eps), self.step_no, ib._stream()))


def forward_fp32(params, x):
    y = torch.empty(x.shape[0], dtype=torch.float32, device=x.device)
    ib._check("ib_mlpForward", ib._lib().ib_mlpForward(ctypes.c_void_p(params.data_ptr()),
                                                       ctypes.c_void_p(x.data_ptr()), x.shape[0],
                                                       ctypes.c_void_p(y.data_ptr()), ib._stream()))
    return y


def forward_tc(params, x):
    y = torch.empty(x.shape[0], dtype=torch.float32, device=x.device)
    ib._check("ib_mlpInferTC", ib._lib().ib_mlpInferTC(ctypes.c_void_p(params.data_ptr()),
                                                       ctypes.c_void_p(x.data_ptr()), x.shape[0],
                                                       ctypes.c_void_p(y.data_ptr()), ib._stream()))
    return y


def train(n_samples=10_000_000, epochs=8, seed=2024, batch=65536, lr=2e-3, tg=THERMO_GAS, td=THERMO_DUST,
          val_fraction=0.02, verbose=False):
    """Generates n_samples exact labels and trains the network; returns (model, history)."""
    feats = sample_features(n_samples, seed)
    s = exact_decay(feats, tg, td)
    keep = torch.isfinite(s) & (s > 0)
    feats, s = feats[keep], s[keep]
    logs = torch.log(s)
    lf = torch.log(feats)
    model = DragModel(params=init_params(seed + 1))
    model.feature_shift = lf.mean(0).tolist()
    model.feature_scale = (1.0 / lf.std(0)).tolist()
    model.out_shift = float(logs.mean())
    model.out_scale = float(logs.std())
    x = normalise(model, feats)
    t = ((logs - model.out_shift) / model.out_scale).float()
    n = x.shape[0]
    nval = max(1, int(n * val_fraction))
    xv, tv = x[n - nval:], t[n - nval:]
    xt, tt = x[:n - nval], t[:n - nval]
    ntr = xt.shape[0]
    tr = Trainer(model.params, lr=lr, batch=batch)
    steps_per_epoch = ntr // batch
    total = epochs * steps_per_epoch
    hist = {"samples": int(n), "train_samples": int(ntr), "val_samples": int(nval), "epochs": epochs,
            "batch": batch, "steps": total, "val_rmse_log_s": []}
    g = torch.Generator(device="cuda").manual_seed(seed + 2)
    k = 0
    for ep in range(epochs):
        perm = torch.randperm(ntr, device="cuda", generator=g)
        for b in range(steps_per_epoch):
            idx = perm[b * batch:(b + 1) * batch]
            lr_k = lr * (0.05 + 0.95 * 0.5 * (1 + math.cos(math.pi * k / max(1, total))))
            tr.step(xt.index_select(0, idx), tt.index_select(0, idx), lr=lr_k)
            k += 1
        yv = forward_fp32(model.params, xv)
        rmse = float(torch.sqrt(torch.mean((yv - tv) ** 2)).item()) * model.out_scale
        hist["val_rmse_log_s"].append(rmse)
        if verbose:
            print("epoch %d  val rmse(log s) %.4g" % (ep, rmse), flush=True)
    return model, hist


def evaluate(model, n=1_000_000, seed=99, tg=THERMO_GAS, td=THERMO_DUST):
    """Tensor-core predictions against exact labels on fresh samples of the training box: errors
    in log s and in the decay factor exp(-s) that the update applies."""
    feats = sample_features(n, seed)
    s = exact_decay(feats, tg, td)
    x = normalise(model, feats)
    y = forward_tc(model.params, x).double()
    s_hat = torch.exp(model.out_shift + model.out_scale * y)
    dl = torch.log(s_hat) - torch.log(s)
    df = torch.exp(-s_hat) - torch.exp(-s)
    return {"samples": n, "rmse_log_s": float(torch.sqrt(torch.mean(dl ** 2))),
            "max_abs_log_s": float(dl.abs().max()), "rmse_decay": float(torch.sqrt(torch.mean(df ** 2))),
            "max_abs_decay": float(df.abs().max()),
            "p99_abs_decay": float(torch.quantile(df.abs()[:min(n, 1 << 24)].float(), 0.99))}


def drag_step(gas, dust, model, dt, tg=THERMO_GAS, td=THERMO_DUST, fallback_counter=None):
    """Learned drag over dt on two ib.Fluid objects (in place)."""
    a, b = thermo(tg), thermo(td)
    m = model.struct()
    fg, fd = gas.c_struct(), dust.c_struct()
    fc = ctypes.c_void_p(fallback_counter.data_ptr()) if fallback_counter is not None else None
    ib._check("ib_cudaSource2FluidDragLearned", ib._lib().ib_cudaSource2FluidDragLearned(
        ctypes.byref(fg), ctypes.byref(fd), ctypes.byref(a), ctypes.byref(b), ctypes.byref(m), ctypes.c_double(dt),
        fc, ib._stream()))
