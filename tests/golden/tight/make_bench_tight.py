"""Generate the tight-oracle fixture of the bench's default accuracy sample: the first
1,024 systems of bench.py's default workload (1,048,576 mixed-stiffness 53-species
systems, seed 2024, rank 0) integrated over 20 global steps of 1e-6 s from t = 0 by
the oracle (the plain-C restatement of the reference's CPU radau2a,
oracle/radau2a.c) at rtol 1e-12 / atol 1e-20.  The integration takes CPU-tens of
minutes; bench.py uses this file when its run matches these settings (and the
SHA-256 of the sample's initial states matches), and integrates live otherwise.

    python tests/golden/tight/make_bench_tight.py
"""
import hashlib
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
sys.path.insert(0, ROOT)

from accelerint_b200 import mechanism as M  # noqa: E402
from oracle import Oracle, global_steps  # noqa: E402
from oracle.tight import TIGHT_MAX_STEPS  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "bench_ma54_1m_seed2024_20steps.npz")
NUM, SEED, SAMPLE, STEPS, DT = 1 << 20, 2024, 1024, 20, 1e-6
ATOL, RTOL = 1e-20, 1e-12


def sample_states():
    """(y[N, SAMPLE], var[SAMPLE], sha256 of y) of the bench's default accuracy sample."""
    mech = M.mechanism_53()
    y, var = M.mixed_stiffness_initial_conditions(mech, NUM, SEED)
    y = np.ascontiguousarray(y[:, :SAMPLE])
    return mech, y, np.ascontiguousarray(var[:SAMPLE]), hashlib.sha256(y.tobytes()).hexdigest()


def main():
    mech, y, var, sha = sample_states()
    o = Oracle()
    t0 = time.time()
    codes = np.zeros(SAMPLE, dtype=np.int32)
    for (a, b) in global_steps(0.0, STEPS * DT, DT):
        y, c, _ = o.integrate("radau2a", mech, y, var, a, b, atol=ATOL, rtol=RTOL, nthreads=os.cpu_count() or 1,
                              max_steps=TIGHT_MAX_STEPS)
        codes = np.maximum(codes, c)
    assert np.isfinite(y).all()
    np.savez_compressed(OUT, y=y, codes=codes, y0_sha256=sha, num=NUM, seed=SEED, sample=SAMPLE, steps=STEPS,
                        dt=DT, atol=ATOL, rtol=RTOL)
    print(f"{OUT}: {SAMPLE} systems to t = {STEPS * DT}, codes {np.bincount(codes).tolist()}, "
          f"{time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
