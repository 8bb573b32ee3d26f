"""On-disk formats of the reference's command-line harness.

Initial conditions (generic/read_initial_conditions.c:30-77, the `ign_data.bin`
file): NUM records of N + 2 little-endian doubles,

    t, y_0, p, y_1, ..., y_{N-1}

where y_0 is the temperature (van der Pol: y1), p the per-system parameter
(pressure in Pa for constant pressure; van der Pol: mu) and y_1.. the rest of
the state (mass fractions; van der Pol: y2).  The reference's pyJac masks
(`apply_mask`) reorder species; the mechanisms here have no mask.

Log (generic/solver_main.c:47-66, `log/<solver>-log.bin`): for every logged
time, one double t followed by NUM records of N doubles, y_0 .. y_{N-1}.
"""
from __future__ import annotations

import os

import numpy as np


def write_initial_conditions(path: str, y: np.ndarray, var: np.ndarray, t: float = 0.0) -> None:
    """y[N, NUM] column-major state, var[NUM] -> records (t, y0, var, y1..)."""
    n, num = y.shape
    rec = np.empty((num, n + 2), dtype="<f8")
    rec[:, 0] = t
    rec[:, 1] = y[0]
    rec[:, 2] = var
    rec[:, 3:] = y[1:].T
    with open(path, "wb") as f:
        f.write(rec.tobytes())


def read_initial_conditions(path: str, num: int, n: int):
    """The first `num` records of an initial-condition file for state length n.

    Returns (y[n, num], var[num]).  Raises ValueError when the file holds fewer
    records (the reference prints the count and exits)."""
    need = num * (n + 2)
    data = np.fromfile(path, dtype="<f8", count=need)
    if data.size != need:
        raise ValueError(f"{path}: {need} doubles expected for {num} states of length {n}, {data.size} read")
    rec = data.reshape(num, n + 2)
    y = np.empty((n, num))
    y[0] = rec[:, 1]
    y[1:] = rec[:, 3:].T
    var = rec[:, 2].copy()
    return y, var


class LogWriter:
    """Appends (t, states) frames in the reference's log layout."""

    def __init__(self, path: str):
        os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
        self.f = open(path, "wb")

    def write(self, t: float, y: np.ndarray) -> None:
        self.f.write(np.asarray([t], dtype="<f8").tobytes())
        self.f.write(np.ascontiguousarray(y.T, dtype="<f8").tobytes())

    def close(self) -> None:
        self.f.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def read_log(path: str, num: int, n: int):
    """Frames of a log file: list of (t, y[n, num])."""
    data = np.fromfile(path, dtype="<f8")
    frame = 1 + num * n
    if data.size % frame:
        raise ValueError(f"{path}: size {data.size} is not a multiple of the frame size {frame}")
    out = []
    for k in range(data.size // frame):
        d = data[k * frame:(k + 1) * frame]
        out.append((float(d[0]), d[1:].reshape(num, n).T.copy()))
    return out
