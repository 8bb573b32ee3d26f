"""The reference harness's file formats (accelerint_b200/io.py) and the
command-line driver (accelerint_b200/cli.py)."""
import os

import numpy as np
import pytest

import accelerint_b200 as A
from accelerint_b200 import cli, io


def test_initial_conditions_round_trip(tmp_path):
    mech = A.mechanism_13()
    y, var = A.mass_action_initial_conditions(mech, 37, seed=3)
    p = str(tmp_path / "ign_data.bin")
    io.write_initial_conditions(p, y, var, t=0.0)
    assert os.path.getsize(p) == 37 * (mech.n_state + 2) * 8
    y2, v2 = io.read_initial_conditions(p, 37, mech.n_state)
    assert np.array_equal(y, y2) and np.array_equal(var, v2)
    y3, _ = io.read_initial_conditions(p, 5, mech.n_state)      # a prefix, as the reference reads NUM records
    assert np.array_equal(y3, y[:, :5])
    with pytest.raises(ValueError):
        io.read_initial_conditions(p, 38, mech.n_state)


def test_record_layout_matches_reference_reader(tmp_path):
    """(t, y0, p, y1, ...): read_initial_conditions.c:48-60 puts buffer[1] in y[0],
    buffer[2] in var and buffer[3 + j] in y[1 + j]."""
    y = np.array([[1.0, 2.0], [3.0, 4.0]])
    var = np.array([10.0, 20.0])
    p = str(tmp_path / "ic.bin")
    io.write_initial_conditions(p, y, var, t=0.5)
    raw = np.fromfile(p, dtype="<f8")
    assert raw.tolist() == [0.5, 1.0, 10.0, 3.0, 0.5, 2.0, 20.0, 4.0]


def test_log_layout(tmp_path):
    y = np.arange(6.0).reshape(2, 3)
    p = str(tmp_path / "log" / "radau2a-log.bin")
    with io.LogWriter(p) as w:
        w.write(0.0, y)
        w.write(0.1, y + 1)
    raw = np.fromfile(p, dtype="<f8")
    # t, then state of system 0 (y0, y1), system 1, system 2 (solver_main.c:47-66)
    assert raw[:7].tolist() == [0.0, 0.0, 3.0, 1.0, 4.0, 2.0, 5.0]
    frames = io.read_log(p, 3, 2)
    assert [f[0] for f in frames] == [0.0, 0.1]
    assert np.array_equal(frames[1][1], y + 1)


def test_cli_arguments():
    a = cli.parse(["128", "1", "--mech", "ma54"])
    assert (a.N, a.device, a.end_time, a.step) == (128, 1, 1e-3, 1e-6)
    a = cli.parse([])
    assert (a.N, a.device, a.mech) == (1, 0, "vdp")
    with pytest.raises(SystemExit):
        cli.parse(["0"])


def test_same_initial_conditions():
    y, var = cli.same_initial_conditions(A.mechanism_13(), 4)
    assert np.allclose(y[1:].sum(axis=0), 1.0) and (y[0] == 1600.0).all()
    y, var = cli.same_initial_conditions(A.VanDerPol(), 3)
    assert (y[0] == 2.0).all() and (var == 1000.0).all()


@pytest.mark.gpu
def test_cli_run_writes_reference_log(tmp_path, oracle, monkeypatch):
    y, var = A.vdp_initial_conditions(64, seed=9)
    io.write_initial_conditions(str(tmp_path / "ign_data.bin"), y, var)
    (tmp_path / "log").mkdir()
    monkeypatch.chdir(tmp_path)
    assert cli.main(["64", "0", "--mech", "vdp", "--end-time", "0.05", "--step", "0.01", "--log"]) == 0
    frames = io.read_log(str(tmp_path / "log" / "radau2a-log.bin"), 64, 2)
    assert len(frames) == 6 and abs(frames[-1][0] - 0.05) < 1e-15
    yo, _, _ = oracle.run("radau2a", A.VanDerPol(), y, var, 0.0, 0.05, 0.01)
    err = np.max(np.abs(frames[-1][1] - yo) / (1e-10 + 1e-6 * np.abs(yo)))
    assert err < 1.0
