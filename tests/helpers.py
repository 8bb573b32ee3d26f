"""Shared comparison helpers for the parity tests.

The mass-action workloads are extremely stiff and their adaptive step
sequences are sensitive to the last bit: the reference CPU solver itself,
given initial conditions perturbed by 1e-15 relative, ends some systems with
different step counts and final states that differ by up to ~1e-3 relative.
GPU-vs-CPU parity is therefore checked as
  (1) the share of systems that agree to the parity tolerance (weighted
      error < 1, i.e. |x - x_ref| < atol + rtol |x_ref| with rtol 1e-6, atol
      1e-10) is at least the share the perturbed reference reaches, less a slack
      of 0.02 by default (one system of a 64-system sample), and
  (2) the worst system differs no more than the reference differs from itself
      under a 1e-15 perturbation of its inputs (times a factor, 3 by default), and
  (3) against a tight FP64 oracle (rtol 1e-12), the GPU result is as accurate
      as the reference CPU solver at the same tolerance.
"""
import numpy as np


def weighted_error(x, ref, atol=1e-10, rtol=1e-6):
    """logger.py:53-55 of the reference: |x - x_ref| / (atol + rtol |x_ref|), max over everything."""
    return float(np.max(np.abs(x - ref) / (atol + rtol * np.abs(ref))))


def per_system_error(x, ref, atol=1e-10, rtol=1e-6):
    return np.max(np.abs(x - ref) / (atol + rtol * np.abs(ref)), axis=0)


def relative_error(x, ref, floor=1e-30):
    return float(np.max(np.abs(x - ref) / np.maximum(np.abs(ref), floor)))


def perturbed(y, rel=1e-15, seed=0):
    return y * (1.0 + rel * np.random.default_rng(seed).standard_normal(y.shape))


def check_parity(y_gpu, y_cpu, y_cpu_perturbed, slack=0.02, factor=3.0):
    """y_cpu_perturbed: one perturbed oracle run, or a list of them (the envelope is then
    the per-system maximum over the runs, the share within tolerance the smallest)."""
    e = per_system_error(y_gpu, y_cpu)
    runs = y_cpu_perturbed if isinstance(y_cpu_perturbed, (list, tuple)) else [y_cpu_perturbed]
    env = np.max([per_system_error(yp, y_cpu) for yp in runs], axis=0)
    frac = float(np.mean(e < 1.0))
    frac_env = float(np.mean(env < 1.0))
    assert not np.isnan(y_gpu).any()
    assert frac >= frac_env - slack, (f"{frac:.3f} of systems agree within rtol 1e-6 / atol 1e-10; "
                                      f"the perturbed reference reaches {frac_env:.3f}")
    assert e.max() <= factor * max(env.max(), 1.0), f"worst system {e.max():.3g} vs envelope {env.max():.3g}"
    return frac, float(e.max()), float(env.max())
