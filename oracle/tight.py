"""ORACLE / TEST INFRASTRUCTURE: the tight FP64 oracle run in a separate process.

    python -m oracle.tight IN.npz OUT.npz

IN holds the initial states y[N, num], var[num], the global-step interval
(t0, t_end, dt), the tolerances (atol, rtol), the mechanism name ("ma54",
"ma14" or "vdp") and the thread count.  OUT receives y[N, num] at t_end and the
per-system codes.  The integration is the oracle's plain-C restatement of the
reference's CPU radau2a (oracle/radau2a.c, after radau2a/radau2a.c:520-736)
stepped through the reference's global-step loop (generic/solver_main.c:196-209).

bench.py starts it at the beginning of a run so that the many seconds the
rtol-1e-12 integration takes overlap the GPU work; it is a fresh process (not
a fork of one that has touched the GPU).
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def mechanism(name):
    from accelerint_b200 import mechanism as M
    return {"ma54": M.mechanism_53, "ma14": M.mechanism_13, "vdp": M.VanDerPol}[name]()


# Radau step limit of a tight run: at rtol 1e-12 a few ignition systems take more
# steps than the reference's 200000 (the method keeps one Jacobian over many tiny steps)
TIGHT_MAX_STEPS = 20_000_000


def run(y, var, t0, t_end, dt, atol, rtol, mech_name, nthreads):
    from oracle.api import Oracle, global_steps
    o = Oracle()
    mech = mechanism(mech_name)
    codes = np.zeros(y.shape[1], dtype=np.int32)
    for (a, b) in global_steps(t0, t_end, dt):
        y, c, _ = o.integrate("radau2a", mech, y, var, a, b, atol=atol, rtol=rtol, nthreads=nthreads,
                              max_steps=TIGHT_MAX_STEPS)
        codes = np.maximum(codes, c)
    return y, codes


def main(argv):
    src, dst = argv[1], argv[2]
    d = np.load(src)
    y, codes = run(np.array(d["y"]), np.array(d["var"]), float(d["t0"]), float(d["t_end"]), float(d["dt"]),
                   float(d["atol"]), float(d["rtol"]), str(d["mech"]), int(d["nthreads"]))
    tmp = dst + ".part.npz"
    np.savez(tmp, y=y, codes=codes)
    os.replace(tmp, dst)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
