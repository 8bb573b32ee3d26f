"""bench.py's reference arm runs on the CPU (the reference's own radau2a.c, or
the oracle port) and prints the one JSON line of the bench contract."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_contract_line():
    from oracle import oracle_available, reference_available
    if not (reference_available("radau2a", 54) or oracle_available()):
        pytest.skip("neither the reference build nor the oracle is built")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1", "--cpu-sample", "4"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] in ("reference", "port")


def test_flop_model_counts_events():
    sys.path.insert(0, ROOT)
    import bench
    st = np.zeros((2, 10))
    st[0, 4] = 1          # one factorisation at N = 54
    lu1, lu2 = (2.0 / 3.0) * 54 ** 3, (8.0 / 3.0) * 54 ** 3
    f64, f32 = bench.flops_per_system(st)
    assert f64[1] == 0.0 and f32[1] == 0.0
    assert abs(f64[0] - (lu1 + lu2 + 54 * 54)) < 1e-6 and f32[0] == 0.0
    # the factorisations of FP32 matrices are FP32 flops: E2 for fp32, both for fp32_all
    f64, f32 = bench.flops_per_system(st, lu="fp32")
    assert abs(f64[0] - (lu1 + 54 * 54)) < 1e-6 and abs(f32[0] - lu2) < 1e-6
    f64, f32 = bench.flops_per_system(st, lu="fp32_all")
    assert abs(f64[0] - 54 * 54) < 1e-6 and abs(f32[0] - (lu1 + lu2)) < 1e-6
    # a Newton iteration: the triangular solves follow the matrices' precision
    st[0, 4], st[0, 5] = 0, 1
    f64, f32 = bench.flops_per_system(st, lu="fp32_all")
    assert abs(f32[0] - 10 * 54 * 54) < 1e-6 and abs(f64[0] - 42 * 54) < 1e-6


def test_accuracy_metrics():
    sys.path.insert(0, ROOT)
    import bench
    ref = np.array([[1000.0, 2000.0], [0.5, 1e-12], [0.5, 1.0]])
    y = ref.copy()
    y[0, 1] *= 1 + 2e-6
    a = bench.accuracy(y, ref)
    assert abs(a["rel_T_max"] - 2e-6) < 1e-12
    assert a["rel_Y_max"] == 0.0 and a["finite"]
    assert abs(a["weighted_max"] - 4e-3 / (1e-10 + 2e-3)) < 1e-6 and a["frac_within_tol"] == 0.5


def test_state_features_layout():
    import accelerint_b200 as A
    from accelerint_b200 import learned as L
    mech = A.mechanism_13()
    y, var = A.mass_action_initial_conditions(mech, 5, seed=2)
    x = L.state_features(y, var, 1e-6)
    assert x.shape == (5, L.D_IN)
    assert np.allclose(x[:, 0], y[0]) and np.allclose(x[:, 14], -6.0) and np.allclose(x[:, 15], 0.0)
    assert (x[:, 16:] == 0).all()


def test_tight_fixture_only_for_its_own_sample():
    """The committed rtol-1e-12 solution of the default accuracy sample is used only when the
    run's first 1,024 initial states hash to the ones it was made from, over 20 steps."""
    sys.path.insert(0, ROOT)
    import bench
    if not os.path.exists(bench.TIGHT_FIXTURE):
        pytest.skip("fixture absent")
    _, y, _ = bench.workload(1 << 20, 2024, 0)
    got = bench.tight_fixture(y[:, :1024], 20)
    assert got is not None and got[0].shape == (54, 1024) and (got[1] == 0).all()
    assert bench.tight_fixture(y[:, :1024], 3) is None
    assert bench.tight_fixture(y[:, :512], 20) is None
    z = y[:, :1024].copy()
    z[0, 5] += 1e-9
    assert bench.tight_fixture(z, 20) is None
