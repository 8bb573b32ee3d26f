"""ORACLE / TEST INFRASTRUCTURE -- the CPU checker for the batched integrators.

Only tests/, __graft_entry__.smoke() and bench.py (its cpu_baseline leg and
its ``--impl reference`` arm) import this package.  The product library never
links, imports or calls it.

Two CPU implementations live here:
  * the oracle: a plain-C restatement of the reference's radau2a / rkc /
    exprb43 / exp4 (oracle/*.c -> oracle/_build/liboracle.so), runtime state
    length, per-system return codes and event counters;
  * oracle/_ref: the reference's own unmodified CPU sources compiled per
    (solver, state length), used to pin the restatement and as the timed
    reference CPU baseline; and its GPU Radau (radau2a.cu under intDriver)
    compiled for sm_100a, timed beside the library's kernels.
"""
from .api import (SOLVERS, STAT_NAMES, Oracle, Reference, ReferenceGPU, cf_poles, global_steps,  # noqa: F401
                  oracle_available, reference_available, reference_gpu_available)
