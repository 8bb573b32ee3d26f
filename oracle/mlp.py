"""ORACLE / TEST INFRASTRUCTURE: the step-proposal MLP in torch on the CPU (FP32).

Restates the library's network (accelerint_b200/csrc/mlp.cuh, mlp.cu) with the
same BF16 rounding: each GEMM operand -- weights, activations and, in the
backward pass, the incoming gradient -- is rounded to BF16 (round to nearest
even), products are accumulated in FP32.  Biases, GELU (erf form) and its
derivative stay FP32.  `loss_grad_autograd` is the same network without the
rounding, through torch autograd, to check the hand-written backward pass."""
import math

import torch

D_IN, D_H, D_OUT = 64, 128, 176
LAYERS = [(D_IN, D_H), (D_H, D_H), (D_H, D_H), (D_H, D_OUT)]


def bf(t):
    return t.to(torch.bfloat16).to(torch.float32)


def unpack(p):
    out, o = [], 0
    for din, dout in LAYERS:
        W = p[o:o + din * dout].view(dout, din)
        o += din * dout
        b = p[o:o + dout]
        o += dout
        out.append((W, b))
    return out


def gelu(z):
    return 0.5 * z * (1.0 + torch.erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + torch.erf(z / math.sqrt(2.0))) + z * torch.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def forward(p, xs, rounding=True):
    r = bf if rounding else (lambda t: t)
    a, zs, ins = xs, [], []
    layers = unpack(p)
    for li, (W, b) in enumerate(layers):
        ins.append(a)
        z = r(a) @ r(W).T + b
        zs.append(z)
        a = gelu(z) if li < len(layers) - 1 else z
    return a, zs, ins


def loss_grad(p, xs, ts, w, rounding=True):
    """Loss sum_m sum_j w_j (y - t)^2 / M and its gradient, backward written out
    as the library's kernels compute it (rounding=False: no BF16 rounding)."""
    bf_ = bf if rounding else (lambda t: t)
    M = xs.shape[0]
    y, zs, ins = forward(p, xs, rounding)
    d = y - ts
    loss = float((w * d * d).sum() / M)
    dz = 2.0 * w * d / M
    layers = unpack(p)
    grads = [None] * len(layers)
    for li in range(len(layers) - 1, -1, -1):
        W, _ = layers[li]
        gW = bf_(dz).T @ bf_(ins[li])
        gb = dz.sum(0)
        grads[li] = (gW, gb)
        if li > 0:
            da = bf_(dz) @ bf_(W)
            dz = da * gelu_grad(zs[li - 1])
    g = torch.cat([torch.cat([gW.reshape(-1), gb]) for gW, gb in grads])
    return loss, g


def loss_grad_autograd(p, xs, ts, w):
    p = p.clone().requires_grad_(True)
    y, _, _ = forward(p, xs, False)
    loss = (w * (y - ts) ** 2).sum() / xs.shape[0]
    loss.backward()
    return float(loss), p.grad.detach()
