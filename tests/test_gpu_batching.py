"""Batching row: the persistent work-queue kernels launched directly, through a
captured CUDA graph, and under an autotuned mapping give the same results.

Systems are independent and each is integrated by one team from start to end,
so the order in which teams pull systems from the queue cannot change any
result: the three launch paths must agree bit for bit."""
import numpy as np
import pytest

import accelerint_b200 as A

pytestmark = pytest.mark.gpu


def _case(kind):
    if kind == "vdp":
        mech = A.VanDerPol()
        y, var = A.vdp_initial_conditions(2048, seed=41)
        return mech, y, var, 0.0, 0.05, 0.01
    mech = A.mechanism_13()
    y, var = A.mass_action_initial_conditions(mech, 512, seed=42)
    return mech, y, var, 0.0, 2e-6, 1e-6


def _device_run(integ, y, var, t0, t1, dt):
    import torch
    yd = torch.from_numpy(y).cuda()
    vd = torch.from_numpy(var).cuda()
    cd = torch.zeros(y.shape[1], dtype=torch.int32, device="cuda")
    integ.integrate_device(t0, t1, dt, yd, vd, cd)
    torch.cuda.synchronize()
    return yd.cpu().numpy(), cd.cpu().numpy()


@pytest.mark.parametrize("kind", ["vdp", "ma14"])
def test_graph_launch_matches_direct_launch(kind):
    mech, y, var, t0, t1, dt = _case(kind)
    integ = A.Integrator(y.shape[1], mech)
    try:
        y_direct, c_direct = _device_run(integ, y, var, t0, t1, dt)
        integ.set_graph_launch(True)
        y_graph, c_graph = _device_run(integ, y, var, t0, t1, dt)
        # a second call with other arguments goes through the in-place graph update
        y_half, _ = _device_run(integ, y, var, t0, 0.5 * (t0 + t1), dt)
        integ.set_graph_launch(False)
        y_half_direct, _ = _device_run(integ, y, var, t0, 0.5 * (t0 + t1), dt)
    finally:
        integ.close()
    assert np.array_equal(c_direct, c_graph)
    assert np.array_equal(y_direct, y_graph)
    assert np.array_equal(y_half, y_half_direct)


@pytest.mark.parametrize("kind", ["ma14"])
def test_plain_grid_matches_persistent_queue(kind):
    mech, y, var, t0, t1, dt = _case(kind)
    integ = A.Integrator(y.shape[1], mech)
    try:
        y_queue, c_queue = _device_run(integ, y, var, t0, t1, dt)
        integ.set_persistent(False)
        y_plain, c_plain = _device_run(integ, y, var, t0, t1, dt)
    finally:
        integ.close()
    assert np.array_equal(c_queue, c_plain)
    assert np.array_equal(y_queue, y_plain)


@pytest.mark.parametrize("mode", [1, 2])
def test_queue_order_gives_identical_results(mode):
    """Longest-first queue orders (by temperature, then by the last call's step
    counts) change which team takes which system, not any result."""
    mech, y, var, t0, t1, dt = _case("ma14")
    integ = A.Integrator(y.shape[1], mech)
    try:
        y_index, _ = _device_run(integ, y, var, t0, t1, dt)
        integ.set_queue_order(mode)
        y_first, _ = _device_run(integ, y, var, t0, t1, dt)
        y_second, _ = _device_run(integ, y, var, t0, t1, dt)    # mode 2: ordered by the first call's steps
    finally:
        integ.close()
    assert np.array_equal(y_index, y_first)
    assert np.array_equal(y_index, y_second)


def test_learned_cost_order_gives_identical_results():
    """Queue order 3 evaluates a cost model for every system before the launch
    (an untrained model here: the order is arbitrary, the results must not move)."""
    import torch
    from accelerint_b200 import learned as L
    mech, y, var, t0, t1, dt = _case("ma14")
    norm = torch.cat([torch.zeros(L.D_IN), torch.ones(L.D_IN), torch.zeros(L.D_OUT), torch.ones(L.D_OUT)]).cuda()
    model = L.Model(mech.n_state, torch.from_numpy(L.init_params(3)).cuda(), norm, [])
    integ = A.Integrator(y.shape[1], mech)
    try:
        y_index, _ = _device_run(integ, y, var, t0, t1, dt)
        model.install_cost(integ)
        y_cost, _ = _device_run(integ, y, var, t0, t1, dt)
        integ.set_graph_launch(True)
        y_graph, _ = _device_run(integ, y, var, t0, t1, dt)
    finally:
        integ.close()
    assert np.array_equal(y_index, y_cost)
    assert np.array_equal(y_index, y_graph)


@pytest.mark.parametrize("kind", ["vdp", "ma14"])
def test_autotuned_mapping_gives_identical_results(kind):
    import torch
    mech, y, var, t0, t1, dt = _case(kind)
    integ = A.Integrator(y.shape[1], mech)
    try:
        y_before, _ = _device_run(integ, y, var, t0, t1, dt)
        yd = torch.from_numpy(y).cuda()
        vd = torch.from_numpy(var).cuda()
        occ, order, blk, ms = integ.autotune(t0, t1, dt, yd, vd, sample=y.shape[1] // 2)
        torch.cuda.synchronize()
        assert np.array_equal(yd.cpu().numpy(), y)          # the sample ran on a copy
        assert ms > 0 and occ >= 0 and order in (0, 1) and blk in (32, 64, 128)
        y_after, _ = _device_run(integ, y, var, t0, t1, dt)
    finally:
        integ.close()
    assert np.array_equal(y_before, y_after)
