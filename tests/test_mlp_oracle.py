"""The torch CPU oracle of the step-proposal MLP (oracle/mlp.py): its written-out
backward pass equals torch autograd when no BF16 rounding is applied, and the
rounding changes the gradients by no more than BF16 precision allows."""
import numpy as np
import torch

from accelerint_b200 import learned as L
from oracle import mlp as OM


def _case(M=48, seed=0):
    g = torch.Generator().manual_seed(seed)
    p = torch.from_numpy(L.init_params(seed + 1))
    xs = torch.randn(M, OM.D_IN, generator=g)
    ts = torch.randn(M, OM.D_OUT, generator=g)
    w = L.loss_weights(54, "cpu")
    return p, xs, ts, w


def test_layout_matches_library_constants():
    offs, n = L.param_offsets()
    assert n == 64048 and len(offs) == 4
    assert sum(din * dout + dout for din, dout in OM.LAYERS) == n


def test_written_out_backward_equals_autograd():
    p, xs, ts, w = _case()
    l1, g1 = OM.loss_grad(p, xs, ts, w, rounding=False)
    l2, g2 = OM.loss_grad_autograd(p, xs, ts, w)
    assert abs(l1 - l2) <= 1e-6 * abs(l2)
    assert float((g1 - g2).norm() / g2.norm()) < 1e-5


def test_bf16_rounding_effect_is_bounded():
    p, xs, ts, w = _case(seed=3)
    _, g1 = OM.loss_grad(p, xs, ts, w, rounding=True)
    _, g2 = OM.loss_grad(p, xs, ts, w, rounding=False)
    # 8 significant bits per operand: relative gradient change of order 1e-2
    assert float((g1 - g2).norm() / g2.norm()) < 5e-2
    assert np.isfinite(g1.numpy()).all()
