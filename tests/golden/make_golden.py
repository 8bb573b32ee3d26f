"""Generate the golden fixtures of tests/golden/ from the reference's own CPU
integrators (oracle/_ref, compiled from the reference sources by
oracle/build.py).  Run where the reference checkout exists:

    python tests/golden/make_golden.py

Each fixture holds the inputs (y0, var, time grid), the reference's outputs
(y, EC_* codes) and, for the exponential methods, the poles/residues the
reference's cf() computed.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from accelerint_b200 import mechanism as M  # noqa: E402
from oracle import Reference  # noqa: E402
from oracle.build import build_reference  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

CASES = [
    # name, solver, mechanism, num, t_end, dt
    ("vdp_radau2a", "radau2a", "vdp", 64, 0.05, 1e-2),
    ("vdp_rkc", "rkc", "vdp", 64, 0.05, 1e-2),
    ("vdp_exprb43", "exprb43", "vdp", 32, 0.02, 1e-2),
    ("vdp_exp4", "exp4", "vdp", 32, 0.02, 1e-2),
    ("ma14_radau2a", "radau2a", "ma14", 16, 2e-6, 1e-6),
    ("ma14_exprb43", "exprb43", "ma14", 8, 1e-6, 1e-6),
    ("ma14_exp4", "exp4", "ma14", 8, 1e-6, 1e-6),
    ("ma14_rkc", "rkc", "ma14", 4, 2e-9, 1e-9),
    ("ma54_radau2a", "radau2a", "ma54", 8, 1e-6, 1e-6),
]


def inputs(mech_name, num):
    if mech_name == "vdp":
        mech = M.VanDerPol()
        y, var = M.vdp_initial_conditions(num, seed=101)
    elif mech_name == "ma14":
        mech = M.mechanism_13()
        y, var = M.mass_action_initial_conditions(mech, num, seed=102)
    else:
        mech = M.mechanism_53()
        y, var = M.mixed_stiffness_initial_conditions(mech, num, seed=103)
    return mech, y, var


def main():
    build_reference()
    for name, solver, mech_name, num, t_end, dt in CASES:
        mech, y, var = inputs(mech_name, num)
        ref = Reference(solver, mech.n_state)
        ref.set_mechanism(mech)
        yo, codes = ref.run(y, var, 0.0, t_end, dt, nthreads=1)
        poles = ref.poles()
        d = dict(y0=y, var=var, t_end=t_end, dt=dt, y=yo, codes=codes, solver=solver, mech=mech_name)
        if poles is not None:
            d["poles"], d["res"] = poles
        np.savez_compressed(os.path.join(OUT, name + ".npz"), **d)
        print(name, "codes", int(codes.max()), "y[0,:2]", yo[0, :2])


if __name__ == "__main__":
    main()
