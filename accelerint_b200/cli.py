"""Command-line harness with the reference GPU driver's interface
(generic/solver_main.cu: `[N] [device]`).

    python -m accelerint_b200.cli [N] [device] [--solver radau2a] [--mech vdp|ma14|ma54]
                                  [--input ign_data.bin] [--end-time T] [--step DT]
                                  [--log] [--same-ic] [--lu fp64|fp32|fp32_all]

Reads N initial conditions from the input file (the reference's `ign_data.bin`
layout, accelerint_b200/io.py), integrates them in global steps of DT to T
through the C-ABI, optionally writes `log/<solver>-log.bin` after every step
(solver_main.c:178-239), and prints the reference's summary lines (# ODEs,
Time, Time per step, TFinal).  --same-ic uses one state for all systems
(set_same_initial_conditions of the reference): T = 1600 K, equal mole
fractions (van der Pol: y = (2, 0), mu = 1000).
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np


def _mechanism(name):
    from . import mechanism as M
    return {"vdp": M.VanDerPol, "ma14": M.mechanism_13, "ma54": M.mechanism_53}[name]()


def same_initial_conditions(mech, num):
    from . import mechanism as M
    if mech.n_state == 2:
        y = np.empty((2, num))
        y[0], y[1] = 2.0, 0.0
        return y, np.full(num, 1000.0)
    x = np.full(mech.n_species, 1.0 / mech.n_species)
    yk = x * mech.mw
    yk /= yk.sum()
    y = np.empty((mech.n_state, num))
    y[0] = 1600.0
    y[1:] = yk[:, None]
    return y, np.full(num, M.P_ATM)


def parse(argv=None):
    p = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    p.add_argument("N", nargs="?", type=int, default=1)
    p.add_argument("device", nargs="?", type=int, default=0)
    p.add_argument("--solver", default="radau2a", choices=["radau2a", "exprb43", "exp4", "rkc"])
    p.add_argument("--mech", default="vdp", choices=["vdp", "ma14", "ma54"])
    p.add_argument("--input", default="ign_data.bin")
    p.add_argument("--end-time", type=float, default=None)
    p.add_argument("--step", type=float, default=None)
    p.add_argument("--lu", default="fp64", choices=["fp64", "fp32", "fp32_all"])
    p.add_argument("--log", action="store_true", help="write log/<solver>-log.bin after every global step")
    p.add_argument("--same-ic", action="store_true")
    a = p.parse_args(argv)
    if a.N <= 0:
        p.error("Problem size not in correct range: provide a number greater than 0")
    if a.end_time is None:
        a.end_time = 1.0 if a.mech == "vdp" else 1e-3
    if a.step is None:
        a.step = 1e-2 if a.mech == "vdp" else 1e-6
    return a


def main(argv=None) -> int:
    from . import Integrator, LU_FP32, LU_FP32_ALL, LU_FP64
    from .io import LogWriter, read_initial_conditions
    a = parse(argv)
    mech = _mechanism(a.mech)
    print(f"# ODEs: {a.N}")
    if a.same_ic:
        y, var = same_initial_conditions(mech, a.N)
    else:
        y, var = read_initial_conditions(a.input, a.N, mech.n_state)
    lu = {"fp64": LU_FP64, "fp32": LU_FP32, "fp32_all": LU_FP32_ALL}[a.lu]
    integ = Integrator(a.N, mech, solver=a.solver, device=a.device, lu=lu)
    log = None
    if a.log:
        if not os.path.isdir("log"):
            print("Expecting 'log' subdirectory in current working directory. Please run"
                  " mkdir log (or the equivalent) and run again.")
            return 1
        log = LogWriter(os.path.join("log", f"{a.solver}-log.bin"))
        log.write(0.0, y)
    rc = 0
    try:
        t0 = time.time()
        t, k = 0.0, 0
        t_next = min(a.end_time, a.step)
        eps = np.finfo(float).eps
        while t + eps < a.end_time:
            k += 1
            y, codes, status = integ.integrate(t, t_next, -1.0, y, var)
            if status != 0:
                bad = int(np.flatnonzero(codes)[0])
                print(f"system {bad} returned code {int(codes[bad])} in [{t:e}, {t_next:e}]")
                rc = int(codes[bad])
            t = t_next
            t_next = min(a.end_time, (k + 1) * a.step)
            if log:
                log.write(t, y)
            if rc:
                break
        runtime = time.time() - t0
    finally:
        integ.close()
        if log:
            log.close()
    print(f"Time: {runtime:.15e} sec")
    print(f"Time per step: {runtime:e} (s)\t{runtime / a.N:.15e} (s/thread)")
    print(f"TFinal: {y[0, 0]:e}")
    return rc


if __name__ == "__main__":
    sys.exit(main())
