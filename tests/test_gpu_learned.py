"""The learned step proposals (MLP, BF16 weights, FP32 accumulation) on the GPU.

* The library's hand-written forward / backward kernels against the torch CPU
  oracle (oracle/mlp.py) with the same BF16 rounding: per-tensor relative
  gradient error below 5e-3 (FP32 accumulation order differs; a BF16 rounding
  flip of one operand changes a product by up to 2^-8 relative).
* Training on step records of plain Radau runs lowers the held-out loss.
* What the trained network gains: on a differently seeded batch of the
  53-species mixed-stiffness workload, Radau with the learned step-size
  proposals rejects fewer steps (the plain method's rejections are almost all
  Newton failures after the controller grows the step), attempts fewer steps
  and factorises less often, while its results stay as accurate as the plain
  method's against a tight FP64 oracle (rtol 1e-12).  The test prints the
  counts of both runs.
"""
import numpy as np
import pytest

import accelerint_b200 as A
from accelerint_b200 import learned as L
from tests.helpers import per_system_error

pytestmark = pytest.mark.gpu


def _grad_case(M=64, seed=0):
    import torch
    g = torch.Generator().manual_seed(seed)
    p = torch.from_numpy(L.init_params(seed + 1))
    xs = torch.randn(M, L.D_IN, generator=g)
    ts = torch.randn(M, L.D_OUT, generator=g)
    w = L.loss_weights(54, "cpu")
    return p, xs, ts, w


def test_mlp_gradients_match_torch_oracle():
    import torch
    from oracle import mlp as OM
    p, xs, ts, w = _grad_case()
    lib = A.load_library()
    pd, xd, td, wd = p.cuda(), xs.cuda(), ts.cuda(), w.cuda()
    gd = torch.zeros_like(pd)
    ld = torch.zeros(1, device="cuda")
    assert lib.accelerInt_mlp_loss_grad(L._p(pd), L._p(xd), L._p(td), L._p(wd), xs.shape[0], L._p(gd), L._p(ld),
                                        None) == 0
    torch.cuda.synchronize()
    lc, gc = OM.loss_grad(p, xs, ts, w)
    assert abs(float(ld.item()) - lc) <= 1e-4 * abs(lc)
    gg = gd.cpu()
    offs, _ = L.param_offsets()
    for wo, bo, din, dout in offs:
        for a, b in ((wo, bo), (bo, bo + dout)):
            rel = float((gg[a:b] - gc[a:b]).norm() / gc[a:b].norm())
            assert rel < 5e-3, (a, b, rel)


def test_mlp_batched_forward_matches_torch_oracle():
    import torch
    from oracle import mlp as OM
    p, xs, _, _ = _grad_case(M=48, seed=5)
    norm = torch.cat([torch.zeros(L.D_IN), torch.ones(L.D_IN), torch.zeros(L.D_OUT), torch.ones(L.D_OUT)])
    model = L.Model(54, p.cuda(), norm.cuda(), [])
    y = model.forward(xs.cuda()).cpu()
    yc, _, _ = OM.forward(p, xs, True)
    assert float((y - yc).norm() / yc.norm()) < 2e-3


@pytest.fixture(scope="module")
def trained():
    mech = A.mechanism_53()
    y, var = A.mixed_stiffness_initial_conditions(mech, 1024, 101)
    rec = L.record_steps(mech, y, var, 0.0, 1e-6, 1e-6, capacity=1 << 20)
    model = L.train(rec, mech.n_state, epochs=12)
    return mech, rec, model


def test_records_and_training(trained):
    mech, rec, model = trained
    assert rec.shape[0] > 10000
    assert all(np.isfinite(model.history))
    assert model.history[-1] < 0.8 * model.history[0]


def _run(mech, y, var, model=None, flags=0):
    import torch
    num = y.shape[1]
    integ = A.Integrator(num, mech, lu=A.LU_FP32_ALL)
    try:
        if model is not None:
            model.install(integ, flags)
        yd = torch.from_numpy(y).cuda()
        vd = torch.from_numpy(var).cuda()
        st = torch.zeros((num, A.NSTATS), dtype=torch.int32, device="cuda")
        cd = torch.zeros(num, dtype=torch.int32, device="cuda")
        integ.integrate_device(0.0, 1e-6, 1e-6, yd, vd, cd, st)
        torch.cuda.synchronize()
        return yd.cpu().numpy(), cd.cpu().numpy(), st.cpu().numpy()
    finally:
        integ.close()


def test_learned_step_size_gain(trained, oracle):
    mech, _, model = trained
    y, var = A.mixed_stiffness_initial_conditions(mech, 512, 202)
    yp, cp, sp = _run(mech, y, var)
    yl, cl, sl = _run(mech, y, var, model, L.MLP_USE_H)
    assert (cp == 0).all() and (cl == 0).all()
    plain, learned = sp.sum(0), sl.sum(0)
    print(f"\nplain  : steps {plain[0]} rejected {plain[2]} decomp {plain[4]} newton {plain[5]}"
          f"\nlearned: steps {learned[0]} rejected {learned[2]} decomp {learned[4]} newton {learned[5]} "
          f"proposals {learned[8]}")
    assert learned[8] > 0
    assert learned[2] < plain[2]          # fewer rejected steps (Newton failures)
    assert learned[0] < plain[0]          # fewer attempted steps
    assert learned[4] < plain[4]          # fewer factorisations
    # accuracy against the tight oracle on a subsample: that of the plain method
    # (a different step sequence, so within a factor 2 of its error)
    sub = np.arange(0, 512, 16)
    yt, _, _ = oracle.run("radau2a", mech, y[:, sub], var[sub], 0.0, 1e-6, 1e-6, rtol=1e-12, atol=1e-20)
    ep, el = per_system_error(yp[:, sub], yt), per_system_error(yl[:, sub], yt)
    print(f"error vs tight oracle (median / max): plain {np.median(ep):.3g} / {ep.max():.3g}, "
          f"learned {np.median(el):.3g} / {el.max():.3g}")
    # slack of 0.1: a weighted error below 0.1 is a tenth of the tolerance
    assert np.median(el) <= 2.0 * np.median(ep) + 0.1
    assert el.max() <= 2.0 * ep.max() + 0.1


def test_learned_stage_guess_falls_back_safely(trained):
    """Stage proposals are verified by Newton; a failed start falls back to the
    extrapolated guess at the same step size, so every system still succeeds."""
    mech, _, model = trained
    y, var = A.mixed_stiffness_initial_conditions(mech, 128, 303)
    yp, cp, _ = _run(mech, y, var)
    yz, cz, sz = _run(mech, y, var, model, L.MLP_USE_H | L.MLP_USE_Z)
    assert (cz == 0).all()
    assert not np.isnan(yz).any()
    assert sz[:, 8].sum() > 0
