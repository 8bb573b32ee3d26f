"""Learned step proposals for Radau IIA: data capture, training and installation.

The network (64 -> 3 x 128 GELU -> 176) and its kernels live in the C-ABI
library (csrc/mlp.cuh for the solver-side inference, csrc/mlp.cu for the
batched forward / backward / Adam on the tensor cores).  This module drives
them: torch supplies device memory and random permutations only; every
FLOP of training and inference runs in the library's own kernels.

Typical use::

    rec = record_steps(mech, y_train, var_train, 0.0, 1e-6, 1e-6)   # plain Radau runs
    model = train(rec, mech.n_state)                                  # on the GPU
    integ = Integrator(num, mech, lu=LU_FP32_ALL)
    model.install(integ, MLP_USE_H)                                   # proposals on
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np

from ._lib import LU_FP64, Integrator, load_library

MLP_USE_H = 1
MLP_USE_Z = 2
D_IN, D_H, D_OUT = 64, 128, 176
REC = D_IN + D_OUT
LAYERS = [(D_IN, D_H), (D_H, D_H), (D_H, D_H), (D_H, D_OUT)]


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def param_offsets():
    """(weight offset, bias offset, din, dout) of each layer in the FP32 parameter vector."""
    out, o = [], 0
    for din, dout in LAYERS:
        out.append((o, o + din * dout, din, dout))
        o += din * dout + dout
    return out, o


def n_params() -> int:
    return param_offsets()[1]


def init_params(seed: int = 0) -> np.ndarray:
    """Uniform(-1/sqrt(din), 1/sqrt(din)) weights, zero biases; the output layer scaled by 0.1."""
    rng = np.random.default_rng(seed)
    offs, n = param_offsets()
    p = np.zeros(n, dtype=np.float32)
    for li, (wo, bo, din, dout) in enumerate(offs):
        a = 1.0 / math.sqrt(din) * (0.1 if li == len(offs) - 1 else 1.0)
        p[wo:bo] = rng.uniform(-a, a, din * dout).astype(np.float32)
    return p


def record_steps(mech, y, var, t0, t1, dt, capacity: int = 1 << 20, device: int = 0, lu: int = LU_FP64,
                 solver: str = "radau2a", stage_extrapolation: int = 0):
    """Run the plain Radau solver on (y, var) and capture one record per accepted step.
    stage_extrapolation: the solver's starting values (Integrator.set_stage_extrapolation),
    that of the form the model will serve.

    Returns a CUDA float32 tensor [n, 240]: raw features then raw targets."""
    import torch
    num = y.shape[1]
    integ = Integrator(num, mech, solver=solver, device=device, lu=lu, stage_extrapolation=stage_extrapolation)
    try:
        rec = torch.zeros((capacity, REC), dtype=torch.float32, device=f"cuda:{device}")
        cnt = torch.zeros(1, dtype=torch.int32, device=f"cuda:{device}")
        rc = integ.lib.accelerInt_set_step_recording(_p(rec), _p(cnt), capacity)
        assert rc == 0
        yd = torch.from_numpy(np.ascontiguousarray(y)).to(rec.device)
        vd = torch.from_numpy(np.ascontiguousarray(var)).to(rec.device)
        integ.integrate_device(t0, t1, dt, yd, vd)
        torch.cuda.synchronize()
        integ.lib.accelerInt_set_step_recording(None, None, 0)
        n = min(int(cnt.item()), capacity)
    finally:
        integ.close()
    return rec[:n].clone()


@dataclass
class Model:
    n_state: int
    params: object          # CUDA float32 [n_params]
    norm: object            # CUDA float32 [2*64 + 2*176]
    history: list

    def install_cost(self, integ: Integrator):
        """Install as the work queue's cost model and switch to learned-cost order."""
        rc = integ.lib.accelerInt_set_cost_model(_p(self.params), _p(self.norm))
        rc = rc or integ.lib.accelerInt_set_queue_order(3)
        if rc != 0:
            raise RuntimeError(f"installing the cost model failed: {rc}")

    def install(self, integ: Integrator, flags: int = MLP_USE_H):
        rc = integ.lib.accelerInt_set_learned(_p(self.params), _p(self.norm), flags)
        if rc != 0:
            raise RuntimeError(f"accelerInt_set_learned failed: {rc}")

    @staticmethod
    def uninstall(integ: Integrator):
        integ.lib.accelerInt_set_learned(None, None, 0)

    def forward(self, x):
        """Batched inference on raw features x [M, 64] (CUDA float32): raw outputs [M, 176]."""
        import torch
        lib = load_library()
        M = x.shape[0]
        Mp = (M + 15) // 16 * 16
        xp = torch.zeros((Mp, D_IN), dtype=torch.float32, device=x.device)
        xp[:M] = x
        y = torch.empty((Mp, D_OUT), dtype=torch.float32, device=x.device)
        rc = lib.accelerInt_mlp_forward(_p(self.params), _p(self.norm), _p(xp), Mp, _p(y), None)
        assert rc == 0
        return y[:M]


def normalisation(rec, n_state: int):
    """Per-feature mean / spread of the records (unused slots: mean 0, spread 1)."""
    import torch
    x, t = rec[:, :D_IN], rec[:, D_IN:]
    nin, nout = n_state + 2, 3 * n_state + 1
    in_mu = torch.zeros(D_IN, device=rec.device)
    in_sd = torch.ones(D_IN, device=rec.device)
    out_mu = torch.zeros(D_OUT, device=rec.device)
    out_sd = torch.ones(D_OUT, device=rec.device)
    in_mu[:nin] = x[:, :nin].mean(0)
    in_sd[:nin] = x[:, :nin].std(0).clamp_min(1e-3)
    out_mu[:nout] = t[:, :nout].mean(0)
    out_sd[:nout] = t[:, :nout].std(0).clamp_min(1e-3)
    return torch.cat([in_mu, in_sd, out_mu, out_sd]).contiguous()


def loss_weights(n_state: int, device, h_weight: float = 16.0):
    import torch
    w = torch.zeros(D_OUT, dtype=torch.float32, device=device)
    w[:3 * n_state] = 1.0
    w[3 * n_state] = h_weight
    return w


def train(rec, n_state: int, epochs: int = 20, batch: int = 1024, lr: float = 1e-3, seed: int = 0,
          h_weight: float = 16.0, holdout: float = 0.1, weights=None) -> Model:
    """Adam on the weighted squared error of the standardised targets, with the
    library's forward / backward kernels.  Returns the model with the held-out
    loss after every epoch."""
    import torch
    assert batch % 16 == 0
    lib = load_library()
    dev = rec.device
    g = torch.Generator(device="cpu").manual_seed(seed)
    rec = rec[torch.isfinite(rec).all(dim=1)]
    perm = torch.randperm(rec.shape[0], generator=g).to(dev)
    rec = rec[perm]
    n_hold = max(16, int(holdout * rec.shape[0]) // 16 * 16)
    hold, tr = rec[:n_hold], rec[n_hold:]
    norm = normalisation(tr, n_state)
    mu_i, sd_i, mu_o, sd_o = norm[:D_IN], norm[D_IN:2 * D_IN], norm[2 * D_IN:2 * D_IN + D_OUT], norm[2 * D_IN + D_OUT:]

    def standardise(r):
        return ((r[:, :D_IN] - mu_i) / sd_i).contiguous(), ((r[:, D_IN:] - mu_o) / sd_o).contiguous()

    xs, ts = standardise(tr)
    xh, th = standardise(hold)
    w = loss_weights(n_state, dev, h_weight) if weights is None else weights.to(dev)
    params = torch.from_numpy(init_params(seed)).to(dev)
    grad = torch.zeros_like(params)
    m1 = torch.zeros_like(params)
    m2 = torch.zeros_like(params)
    loss = torch.zeros(1, dtype=torch.float32, device=dev)
    history = []
    step = 0
    n = xs.shape[0] // batch * batch
    for ep in range(epochs):
        order = torch.randperm(xs.shape[0], generator=g)[:n].to(dev)
        for b0 in range(0, n, batch):
            idx = order[b0:b0 + batch]
            xb, tb = xs[idx].contiguous(), ts[idx].contiguous()
            rc = lib.accelerInt_mlp_loss_grad(_p(params), _p(xb), _p(tb), _p(w), batch, _p(grad), _p(loss), None)
            assert rc == 0
            step += 1
            rc = lib.accelerInt_mlp_adam_step(_p(params), _p(grad), _p(m1), _p(m2), step, lr, 0.9, 0.999, 1e-8,
                                              None)
            assert rc == 0
        rc = lib.accelerInt_mlp_loss_grad(_p(params), _p(xh), _p(th), _p(w), xh.shape[0], _p(grad), _p(loss), None)
        assert rc == 0
        history.append(float(loss.item()))
    return Model(n_state, params, norm, history)


# ---------------------------------------------------------------- cost model
def state_features(y, var, h):
    """The model's input features of whole states (as the device kernel builds them):
    [num, 64] float32 = (T, log10 max(Y_k, 1e-20), log10 h, log10(P / 1 atm), 0...)."""
    n, num = y.shape
    x = np.zeros((num, D_IN), dtype=np.float32)
    x[:, 0] = y[0]
    x[:, 1:n] = np.log10(np.maximum(y[1:], 1e-20)).T
    x[:, n] = np.log10(h)
    x[:, n + 1] = np.log10(var / 101325.0)
    return x


def cost_records(mech, y, var, t0, t1, dt, device: int = 0, lu: int = LU_FP64, stage_extrapolation: int = 0):
    """One record per system and global step: the state's features at the step start
    and, as output 0, log10(1 + Radau steps the plain solver took in that step)."""
    import torch
    num = y.shape[1]
    integ = Integrator(num, mech, device=device, lu=lu, stage_extrapolation=stage_extrapolation)
    dev = f"cuda:{device}"
    recs = []
    try:
        yd = torch.from_numpy(np.ascontiguousarray(y)).to(dev)
        vd = torch.from_numpy(np.ascontiguousarray(var)).to(dev)
        t = t0
        while t + 1e-300 < t1 - 1e-12 * abs(t1):
            tn = min(t1, t + dt)
            st = torch.zeros((num, 10), dtype=torch.int32, device=dev)
            x = state_features(yd.cpu().numpy(), var, tn - t)
            integ.integrate_device(t, tn, tn - t, yd, vd, None, st)
            torch.cuda.synchronize()
            r = np.zeros((num, REC), dtype=np.float32)
            r[:, :D_IN] = x
            r[:, D_IN] = np.log10(1.0 + st[:, 0].cpu().numpy())
            recs.append(r)
            t = tn
    finally:
        integ.close()
    return torch.from_numpy(np.concatenate(recs)).to(dev)


def train_cost(rec, n_state: int, epochs: int = 60, seed: int = 0) -> Model:
    import torch
    w = torch.zeros(D_OUT, dtype=torch.float32)
    w[0] = 1.0
    return train(rec, n_state, epochs=epochs, batch=256, lr=2e-3, seed=seed, weights=w)
