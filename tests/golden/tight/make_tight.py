"""Generate the tight-oracle fixture of tests/golden/tight/: 1,024 mixed-stiffness
53-species systems (seed 2027, both stiffness halves interleaved) integrated over
three global steps of 1e-6 s by the oracle (the plain-C restatement of the
reference's CPU radau2a, oracle/radau2a.c) at rtol 1e-12 / atol 1e-20.  The
integration takes several CPU-minutes, too long to repeat inside the GPU tests,
which compare the library's FP32 and learned forms with this reference solution.

    python tests/golden/tight/make_tight.py

The initial conditions are not stored: the tests regenerate them from the seed
with accelerint_b200.mechanism.mixed_stiffness_initial_conditions.
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
sys.path.insert(0, ROOT)

from accelerint_b200 import mechanism as M  # noqa: E402
from oracle import Oracle, global_steps  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ma54_tight.npz")
NUM, SEED, T_END, DT = 1024, 2027, 3e-6, 1e-6
ATOL, RTOL = 1e-20, 1e-12
# at rtol 1e-12 a few ignition systems take more Radau steps than the reference's
# limit of 200000 allows (the method keeps one Jacobian over many tiny steps)
MAX_STEPS = 20_000_000


def main():
    mech = M.mechanism_53()
    y, var = M.mixed_stiffness_initial_conditions(mech, NUM, SEED)
    o = Oracle()
    t0 = time.time()
    codes = np.zeros(NUM, dtype=np.int32)
    for (a, b) in global_steps(0.0, T_END, DT):
        y, c, _ = o.integrate("radau2a", mech, y, var, a, b, atol=ATOL, rtol=RTOL, nthreads=os.cpu_count() or 1,
                              max_steps=MAX_STEPS)
        codes = np.maximum(codes, c)
    assert (codes == 0).all() and np.isfinite(y).all()
    np.savez_compressed(OUT, y=y, num=NUM, seed=SEED, t_end=T_END, dt=DT, atol=ATOL, rtol=RTOL,
                        max_steps=MAX_STEPS)
    print(f"{OUT}: {NUM} systems to t = {T_END}, {time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
