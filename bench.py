#!/usr/bin/env python
"""Throughput benchmark: ODE systems/s per global Delta-t step.

Workload (default): the 53-species / 325-reaction synthetic mechanism, 1,048,576
initial conditions of the mixed-stiffness generator (half near equilibrium at
800-1200 K, half ignition at 1400-2400 K, interleaved), Radau IIA at rtol 1e-6 /
atol 1e-10, global steps of dt = 1e-6 s from t = 0 (the reference's global-step
loop, generic/solver_interface.cu:161-211).  A bench step is one global Delta-t
step of all systems; the timed region runs K consecutive global steps from the
initial conditions.  The W warm-up steps run the same calls on the whole batch
with a global step of dt / 1000 (every buffer, graph and code path of the timed
calls, about one Radau step per system), after which the state is reset.

Timed region, one loop for both numbers: every step copies the state from
pinned host memory to the device, integrates it through the C-ABI
(accelerInt_integrate_device), and copies the state and the codes back; L2 is
flushed (a 256 MiB write) before each step.  `value` is K x NUM over the summed
CUDA-event time of the integrate calls (inputs resident), `e2e` is K x NUM over
the wall time of the whole loop (copies included).

The tuned form is three changes on top of the plain FP64 form:
E1/E2 factorised and solved in FP32 (--lu), the persistent work-queue kernel
under a captured CUDA graph with the autotuned mapping and a longest-first
queue order from a learned per-system cost model (--queue-order 3), and the
stage and step-size proposals: the Newton iteration starts from the collocation
polynomial evaluated at all three new nodes (--stage-extrapolation 1; the plain
form keeps the reference's start, radau2a.c:312, for parity) and the learned
step-size proposals cap the step growth (--learned).  Both networks are trained, untimed,
by the library's kernels on plain Radau runs of batches drawn with other seeds.
The plain FP64 form (one team per system over a plain grid, FP64
factorisations, no proposals) is timed on the same batch and steps and reported
as "plain_fp64" with the tuned / plain ratio.

Accuracy (untimed): the first --acc-sample systems (both stiffness halves) of
the tuned and plain final states, and of the reference CPU radau2a at rtol 1e-6,
against the oracle integrated at rtol 1e-12 / atol 1e-20 over the same global
steps: the committed solution tests/golden/tight/bench_ma54_1m_seed2024_20steps.npz
when the sample and steps are its own (the default sample over 20 steps), else the
oracle in a separate process on the host cores while the GPU works.  The plain
form's Newton iterations per step and rejected share are reported beside the
tuned form's.  Errors use the reference's weighted metric |x - x_ref| / (atol + rtol
|x_ref|) with atol 1e-10, rtol 1e-6 (logger.py:53-55), and the maximum
relative error of T and of the mass fractions above 1e-8.

Side lines (after the headline work, untimed by the headline): van der Pol (mu
= 1000, 131,072 ICs, t = 0 -> 1 in 100 steps) with the reference's GPU kernel and
CPU code beside ours; the 13-species mechanism (262,144 ICs) for radau2a and
exprb43 with the reference CPU code beside; optionally the reference GPU kernel
on the 53-species batch (--ref-gpu-sample).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--lu fp32|fp32_all|fp64] [--num NUM]

For N > 1 (torchrun, one rank per GPU) every rank integrates its own batch of
NUM systems (weak scaling, no collective on the data path); the time is the
max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from accelerint_b200 import mechanism as M  # noqa: E402

T_START = time.time()


def phase(name):
    """Progress of the run on stderr (the JSON line alone goes to stdout)."""
    print(f"[bench {time.time() - T_START:7.1f} s] {name}", file=sys.stderr, flush=True)


DT = 1e-6
METRIC = "ODE systems/s per Δt step, 53-species Radau: tuned vs plain FP64 at rtol 1e-6"
UNIT = "system-steps/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--lu", default="fp32_all", choices=["fp32", "fp32_all", "fp64"])
    p.add_argument("--plain-steps", type=int, default=-1,
                   help="global steps of the plain FP64 comparison (-1: as --steps, 0: skip)")
    p.add_argument("--num", type=int, default=1 << 20)
    p.add_argument("--solver", default="radau2a")
    p.add_argument("--seed", type=int, default=2024)
    p.add_argument("--cpu-sample", type=int, default=16384, help="systems in the CPU baseline sample")
    p.add_argument("--acc-sample", type=int, default=1024,
                   help="systems compared with the rtol-1e-12 oracle after the timed steps (0: none)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--ref-gpu-sample", type=int, default=0,
                   help="systems the reference's own GPU Radau integrates over the first global step from t=0 "
                        "(0: skip).  One thread per system runs its whole integration, so the launch lasts as "
                        "long as its slowest system (minutes at 53 species): size it to one wave, e.g. 65536")
    p.add_argument("--no-config1", action="store_true",
                   help="skip the van der Pol line (131,072 ICs, t = 0 -> 1 in 100 steps)")
    p.add_argument("--no-config2", action="store_true",
                   help="skip the 13-species lines (262,144 ICs; radau2a, exprb43, rkc)")
    p.add_argument("--config2-steps", type=int, default=1,
                   help="global steps of 1e-6 s from t=0 in the 13-species lines (the full workload runs 1000)")
    p.add_argument("--config2-rkc", action="store_true", help="time RKC in the 13-species lines too")
    p.add_argument("--config2-exp-num", type=int, default=32768,
                   help="systems (the first of the batch) of the exponential-method line: EXPRB43 runs at "
                        "~1,100 system-steps/s on 13 species, minutes for the whole batch")
    p.add_argument("--config2-cpu-sample", type=int, default=2048,
                   help="systems of the 13-species batch the reference CPU solvers integrate")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-autotune", action="store_true")
    p.add_argument("--queue-order", type=int, default=3, choices=[-1, 0, 1, 2, 3],
                   help="work-queue order (-1: the autotuner's choice; 0 index, 1 hottest first, 2 most steps "
                        "in the previous call first, its history restarted before the timed region; 3 largest "
                        "learned cost first)")
    p.add_argument("--no-graph", action="store_true")
    p.add_argument("--learned", type=int, default=1, choices=[0, 1, 2, 3],
                   help="learned proposals in the tuned form: 1 step size, 2 stages, 3 both (0: off)")
    p.add_argument("--stage-extrapolation", type=int, default=1, choices=[0, 1],
                   help="Radau starting values in the tuned form: 1 the collocation polynomial at all three "
                        "nodes, 0 the reference's (radau2a.c:312, the plain form's)")
    p.add_argument("--growth-floor", type=float, default=2.0,
                   help="learned step-size proposals never hold the step below this x the last accepted")
    p.add_argument("--train-epochs", type=int, default=8)
    p.add_argument("--train-batch", type=int, default=4096)
    p.add_argument("--train-num", type=int, default=4096,
                   help="systems of the differently seeded batch whose plain Radau steps train the MLP")
    args = p.parse_args()
    if args.plain_steps < 0:
        args.plain_steps = args.steps
    return args


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def workload(num, seed, rank=0):
    mech = M.mechanism_53()
    y, var = M.mixed_stiffness_initial_conditions(mech, num, seed + 7919 * rank)
    return mech, y, var


# ---------------------------------------------------------------- FLOP model
LU_NAMES = {"fp64": 0, "fp32": 1, "fp32_all": 2}


def flops_per_system(stats, n=54, R=325, lu="fp64"):
    """Algorithmic flops from the device event counters (FMA = 2 flops), split by the
    pipe that runs them: returns (fp64 flops, fp32 flops) per system.

    decomp:  (2/3) N^3 real LU (E1) + (8/3) N^3 complex LU (E2) + N^2 assembly (FP64);
    newton:  3 RHS (counted separately) + 2 N^2 real (E1) + 8 N^2 complex (E2)
             triangular solves + 42 N transforms, updates and norms (FP64);
    aux:     one error-estimate solve with E1, 2 N^2, + 8 N (FP64); with E1 in FP32
             (fp32_all) it is two FP32 solves (4 N^2) and the FP64 refinement
             residual J x (2 N^2);
    rhs:     14 R + 10 N mass-action evaluation (exponentials not counted);
    jac:     60 R + 4 N^2.
    The factorisations and solves of a matrix held in FP32 are FP32 flops (E2 for
    lu fp32; E1 and E2 for fp32_all), everything else FP64."""
    d, nw, rhs, aux, jac = (stats[:, 4], stats[:, 5], stats[:, 6], stats[:, 7], stats[:, 3])
    lu1 = (2.0 / 3.0) * n ** 3
    lu2 = (8.0 / 3.0) * n ** 3
    fp64 = d * n * n + nw * 42 * n + rhs * (14 * R + 10 * n) + jac * (60 * R + 4 * n * n)
    fp32 = np.zeros_like(fp64)
    e1_32 = lu == "fp32_all"
    e2_32 = lu in ("fp32", "fp32_all")
    if e1_32:
        fp32 = fp32 + d * lu1 + nw * 2 * n * n + aux * 4 * n * n
        fp64 = fp64 + aux * (2 * n * n + 8 * n)
    else:
        fp64 = fp64 + d * lu1 + nw * 2 * n * n + aux * (2 * n * n + 8 * n)
    if e2_32:
        fp32 = fp32 + d * lu2 + nw * 8 * n * n
    else:
        fp64 = fp64 + d * lu2 + nw * 8 * n * n
    return fp64, fp32


def accuracy(y, y_tight, atol=1e-10, rtol=1e-6):
    """Errors of final states y[N, m] against the tight oracle's: the reference's weighted
    metric |x - x_ref| / (atol + rtol |x_ref|) (logger.py:53-55) per system (max over the
    state), and the maximum relative errors of T (row 0) and of mass fractions above 1e-8."""
    w = np.max(np.abs(y - y_tight) / (atol + rtol * np.abs(y_tight)), axis=0)
    rel_t = np.abs(y[0] - y_tight[0]) / np.abs(y_tight[0])
    big = np.abs(y_tight[1:]) > 1e-8
    rel_y = np.where(big, np.abs(y[1:] - y_tight[1:]) / np.where(big, np.abs(y_tight[1:]), 1.0), 0.0)
    finite = bool(np.isfinite(y).all())
    return {"weighted_max": float(np.max(w)), "weighted_median": float(np.median(w)),
            "frac_within_tol": float(np.mean(w < 1.0)), "rel_T_max": float(np.max(rel_t)),
            "rel_Y_max": float(np.max(rel_y)), "finite": finite}


TIGHT_FIXTURE = os.path.join(ROOT, "tests", "golden", "tight", "bench_ma54_1m_seed2024_20steps.npz")


def tight_fixture(y_sample, steps):
    """The committed rtol-1e-12 solution of the default accuracy sample (made by
    tests/golden/tight/make_bench_tight.py), when this run's sample and steps are those it
    was made for (the SHA-256 of the initial states decides); else None."""
    import hashlib
    if not os.path.exists(TIGHT_FIXTURE):
        return None
    d = np.load(TIGHT_FIXTURE)
    y0 = np.ascontiguousarray(y_sample)
    if int(d["steps"]) != steps or y0.shape[1] != int(d["sample"]):
        return None
    if hashlib.sha256(y0.tobytes()).hexdigest() != str(d["y0_sha256"]):
        return None
    return np.array(d["y"]), np.array(d["codes"])


def start_tight_oracle(y, var, t_end, nthreads, path):
    """The rtol-1e-12 oracle over [0, t_end] in steps of DT, in a fresh process (oracle/tight.py)."""
    import tempfile
    fd, src = tempfile.mkstemp(prefix="accelerint_tight_", suffix=".npz")
    os.close(fd)
    np.savez(src, y=y, var=var, t0=0.0, t_end=t_end, dt=DT, atol=1e-20, rtol=1e-12, mech="ma54",
             nthreads=nthreads)
    proc = subprocess.Popen([sys.executable, "-m", "oracle.tight", src, path], cwd=ROOT,
                            stdout=subprocess.DEVNULL, stderr=subprocess.PIPE)
    return proc, src


def finish_tight_oracle(handle, path, timeout=1800.0):
    proc, src = handle
    try:
        proc.wait(timeout=timeout)
    except subprocess.TimeoutExpired:
        proc.kill()
        proc.wait()
    try:
        os.remove(src)
    except OSError:
        pass
    if proc.returncode != 0 or not os.path.exists(path):
        return None, None
    d = np.load(path)
    y, codes = np.array(d["y"]), np.array(d["codes"])
    os.remove(path)
    return y, codes


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        import tempfile
        fd, self.path = tempfile.mkstemp(prefix="accelerint_clocks_", suffix=".csv")
        os.close(fd)

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        try:
            with open(self.path) as f:
                rows = [r.split(",") for r in f.read().strip().splitlines() if r.strip()]
            os.remove(self.path)
        except Exception:
            rows = []
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(rows[0][2]), "reasons": sorted(reasons),
                "samples": len(rows)}


def measure_peak(kind):
    """FMA throughput of this device (TFLOP/s): kind 1 FP64, 0 FP32 scalar, 2 FP32x2 packed."""
    from accelerint_b200 import load_library
    lib = load_library()
    import ctypes
    out = ctypes.c_double(0.0)
    lib.accelerInt_measure_fma_peak.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    rc = lib.accelerInt_measure_fma_peak(kind, ctypes.byref(out))
    return out.value if rc == 0 else None


# ---------------------------------------------------------------- CPU baseline
def cpu_baseline(args, mech, y, var):
    """Reference CPU radau2a (oracle/_ref, the reference's own C sources, OpenMP) on the
    first --cpu-sample systems over the K global steps; returns (line, final states)."""
    sys.path.insert(0, ROOT)
    from oracle import Reference, reference_available, Oracle, oracle_available
    nthreads = os.cpu_count() or 1
    sample = min(args.num, args.cpu_sample)
    ys, vs = y[:, :sample].copy(), var[:sample].copy()
    if reference_available("radau2a", 54):
        ref = Reference("radau2a", 54)
        ref.set_mechanism(mech)
        kind = "reference"
        t0 = time.time()
        for k in range(args.steps):
            ys, codes = ref.integrate(ys, vs, k * DT, (k + 1) * DT, nthreads)
        el = time.time() - t0
    elif oracle_available():
        o = Oracle()
        kind = "port"
        t0 = time.time()
        for k in range(args.steps):
            ys, codes, _ = o.integrate("radau2a", mech, ys, vs, k * DT, (k + 1) * DT, nthreads=nthreads)
        el = time.time() - t0
    else:
        return None, None
    line = {"value": sample * args.steps / el, "unit": UNIT, "cores": nthreads, "kind": kind,
            "sample": f"rate measured on the first {sample} of the {args.num} systems (both stiffness "
                      f"halves) x {args.steps} global steps from t=0 on {nthreads} OpenMP threads "
                      f"({el:.1f} s); a per-system-step rate, not a timing of the whole batch"}
    return line, ys


def run_reference_arm(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    mech, y, var = workload(args.num, args.seed)
    cb, _ = cpu_baseline(args, mech, y, var)
    if cb is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU build (oracle/_ref) and oracle missing"}))
        return 0
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * args.num / cb["value"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": "mass-action 53 species / 325 reactions, mixed stiffness, "
                                                       f"{args.num} ICs, global steps of dt=1e-6 s from t=0, "
                                                       "radau2a rtol 1e-6 atol 1e-10",
                                            "solver": "radau2a (reference CPU, OpenMP)",
                                            "timing": "sampled rate: ms_per_step = the full batch at the rate "
                                                      "measured on the sample (cpu_baseline.sample)"},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------- reference GPU kernel
def reference_gpu_leg(args, mech, y, var, first_tuned, first_plain):
    """The reference's own GPU Radau (oracle/_ref, radau2a.cu under intDriver, one thread per
    system).  As shipped it fails every system (its error estimate solves with the raw
    Jacobian, radau2a.cu:612): that is recorded on 256 systems.  The throughput is the build
    with that one line fixed (solve with the factored E1), on the first --ref-gpu-sample
    systems over the first global step from t=0, compared with the library's own rates on
    that same global step of the whole batch (first_tuned, first_plain: system-steps/s)."""
    from oracle import ReferenceGPU, reference_gpu_available
    if not (reference_gpu_available(54) and reference_gpu_available(54, q3_fix=True)):
        return None
    r = ReferenceGPU(54)
    r.set_mechanism(mech)
    _, codes0, ms0 = r.run(y[:, :256], var[:256], 0.0, DT, DT)
    s = min(args.num, args.ref_gpu_sample)
    r = ReferenceGPU(54, q3_fix=True)
    r.set_mechanism(mech)
    t0 = time.time()
    _, codes, ms = r.run(y[:, :s], var[:s], 0.0, DT, DT)
    rate = s / (ms / 1000.0)
    return {"value": rate, "unit": UNIT, "kind": "reference_gpu",
            "as_shipped": {"systems": 256, "codes": np.bincount(codes0, minlength=5).tolist(), "kernel_ms": ms0,
                           "note": "every system ends with EC_h_plus_t_equals_h: the error estimate solves "
                                   "with the raw Jacobian (radau2a.cu:612), a zero diagonal entry makes the "
                                   "error infinite and the step size zero"},
            "sample": f"first {s} of the {args.num} systems x the first global step from t=0; the "
                      "reference's radau2a.cu with its error-estimate line fixed (E1 = solver->E1), under "
                      "intDriver (one thread per system, 64-thread blocks, strict IEEE flags), built for "
                      f"sm_100a; summed CUDA-event time of its launches ({ms / 1000.0:.1f} s, "
                      f"{time.time() - t0:.1f} s wall)",
            "failed_systems": int((codes != 0).sum()),
            "first_step_tuned": first_tuned, "first_step_plain_fp64": first_plain,
            "tuned_over_reference_gpu": first_tuned / rate,
            "plain_fp64_over_reference_gpu": first_plain / rate if first_plain else None}


def config1_leg(dev):
    """Van der Pol (mu = 1000), 131,072 ICs, t = 0 -> 1 in 100 global steps of 1e-2, plain FP64
    Radau at rtol 1e-6 / atol 1e-10: the library, the reference's GPU kernel and the reference's
    CPU integrator (all host threads), each over the whole batch."""
    import torch
    import accelerint_b200 as A
    from oracle import Reference, ReferenceGPU, reference_available, reference_gpu_available
    num, steps = 131072, 100
    vdp = A.VanDerPol()
    y, var = A.vdp_initial_conditions(num, seed=1)
    integ = A.Integrator(num, vdp, device=dev.index)
    out = {"workload": "van der Pol mu=1000, 131072 ICs y1~U[-2,2] y2~U[-1,1], t 0->1 in 100 steps of 1e-2, "
                       "radau2a FP64 rtol 1e-6 atol 1e-10"}
    try:
        yd = torch.from_numpy(np.ascontiguousarray(y)).to(dev)
        vd = torch.from_numpy(var).to(dev)
        integ.integrate_device(0.0, 1e-2, 1e-2, yd[:, :1024].contiguous(), vd[:1024].contiguous())
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        a.record()
        integ.integrate_device(0.0, 1.0, 1e-2, yd, vd)
        b.record()
        torch.cuda.synchronize(dev)
        ours = num * steps / (a.elapsed_time(b) / 1000.0)
        out["ours"] = {"value": ours, "unit": UNIT, "kernel": "thread per system, one launch for all 100 steps"}
    finally:
        integ.close()
    if reference_gpu_available(2) and reference_gpu_available(2, q3_fix=True):
        _, codes0, _ = ReferenceGPU(2).run(y[:, :256], var[:256], 0.0, 1e-2, 1e-2)
        _, codes, ms = ReferenceGPU(2, q3_fix=True).run(y, var, 0.0, 1.0, 1e-2)
        rg = num * steps / (ms / 1000.0)
        out["reference_gpu"] = {"value": rg, "unit": UNIT, "failed_systems": int((codes != 0).sum()),
                                "ours_over": ours / rg, "build": "error-estimate line fixed (E1 = solver->E1)",
                                "as_shipped_codes_256": np.bincount(codes0, minlength=5).tolist()}
    if reference_available("radau2a", 2):
        ref = Reference("radau2a", 2)
        nthreads = os.cpu_count() or 1
        ys = y.copy()
        t0 = time.time()
        for k in range(steps):
            ys, _ = ref.integrate(ys, var, k * 1e-2, (k + 1) * 1e-2, nthreads)
        el = time.time() - t0
        rc = num * steps / el
        out["reference_cpu"] = {"value": rc, "unit": UNIT, "cores": nthreads, "ours_over": ours / rc}
    return out


def guarded(leg, *a):
    """A side line of the bench (the other workloads): its failure is reported in the JSON line
    instead of ending the run before the headline is printed."""
    try:
        return leg(*a)
    except Exception as e:  # noqa: BLE001 - any failure of a side line is recorded, not raised
        return {"error": f"{type(e).__name__}: {e}"[:500]}


def config2_leg(dev, args):
    """13-species mechanism (27 reactions), 262,144 ICs (T in [1000, 1600] K, Dirichlet(0.5)
    mole fractions), plain FP64 radau2a / exprb43 / rkc at rtol 1e-6 / atol 1e-10 over the first
    --config2-steps global steps of 1e-6 s from t=0: the library over the whole batch for radau2a
    and rkc and over its first --config2-exp-num systems for exprb43 (one launch for all steps,
    CUDA events), and the reference's CPU solver (oracle/_ref, all host threads) on the first
    --config2-cpu-sample systems of the same batch."""
    import torch
    import accelerint_b200 as A
    from oracle import Reference, reference_available
    num, steps = 262144, args.config2_steps
    mech = A.mechanism_13()
    y, var = A.mass_action_initial_conditions(mech, num, seed=2)
    yd0 = torch.from_numpy(np.ascontiguousarray(y)).to(dev)
    vd = torch.from_numpy(np.ascontiguousarray(var)).to(dev)
    nthreads = os.cpu_count() or 1
    out = {"workload": f"mass-action 13 species / 27 reactions, {num} ICs T~U[1000,1600] K, "
                       f"Dirichlet(0.5) mole fractions, {steps} global steps of 1e-6 s from t=0, FP64, "
                       "rtol 1e-6 atol 1e-10"}
    solvers = ("radau2a", "exprb43", "rkc") if args.config2_rkc else ("radau2a", "exprb43")
    if not args.config2_rkc:
        out["rkc"] = {"skipped": "RKC (an explicit stabilised method) takes tens of thousands of steps of "
                                 "thousands of stages on the stiffest of these systems in their first "
                                 "microseconds, on the reference CPU code and on the GPU alike; --config2-rkc "
                                 "times it"}
    for solver in solvers:
        n = min(num, args.config2_exp_num) if solver == "exprb43" else num
        integ = A.Integrator(n, mech, solver=solver, device=dev.index)
        try:
            yw = yd0[:, :2048].contiguous()
            integ.integrate_device(0.0, 1e-8, 1e-8, yw, vd[:2048].contiguous())   # warm-up
            yd = yd0[:, :n].clone().contiguous()   # a copy: the batch's states stay for the next solver
            vn = vd[:n].contiguous()
            codes = torch.zeros(n, dtype=torch.int32, device=dev)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize(dev)
            a.record()
            integ.integrate_device(0.0, steps * DT, DT, yd, vn, codes)
            b.record()
            torch.cuda.synchronize(dev)
            ms = a.elapsed_time(b)
            c = codes.cpu().numpy()
            line = {"value": n * steps / (ms / 1000.0), "unit": UNIT, "ms": ms, "systems": n,
                    "codes": np.bincount(c, minlength=6).tolist()}
        finally:
            integ.close()
        if reference_available(solver, 14):
            s = min(num, args.config2_cpu_sample)
            ref = Reference(solver, 14)
            ref.set_mechanism(mech)
            ys = y[:, :s].copy()
            rcodes = np.zeros(s, dtype=np.int32)
            t0 = time.time()
            for k in range(steps):
                ys, ck = ref.integrate(ys, var[:s], k * DT, (k + 1) * DT, nthreads)
                rcodes = np.maximum(rcodes, ck)
            el = time.time() - t0
            rc = s * steps / el
            line["reference_cpu"] = {"value": rc, "unit": UNIT, "cores": nthreads, "kind": "reference",
                                     "codes": np.bincount(rcodes, minlength=6).tolist(),
                                     "sample": f"first {s} systems x {steps} global steps ({el:.1f} s)"}
            line["ours_over_reference_cpu"] = line["value"] / rc
        out[solver] = line
    return out


# ---------------------------------------------------------------- GPU arm
def run_ours(args):
    import torch
    import accelerint_b200 as A
    ws, rank, local = dist_env()
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
        torch.cuda.set_device(local)
    dev = torch.device("cuda", local if ws > 1 else 0)
    mech, y, var = workload(args.num, args.seed, rank)
    lu = {"fp32": A.LU_FP32, "fp32_all": A.LU_FP32_ALL, "fp64": A.LU_FP64}[args.lu]

    # CPU work first, on rank 0: the reference CPU baseline alone on the host cores, then
    # the tight oracle for the accuracy sample in a separate process during the GPU work
    cb, y_ref_cpu, tight, tight_fix = None, None, None, None
    tight_path = os.path.join(ROOT, f".bench_tight_{os.getpid()}.npz")
    acc_n = min(args.acc_sample, args.num)
    if rank == 0:
        if not args.no_cpu_baseline:
            cb, y_ref_cpu = cpu_baseline(args, mech, y, var)
            phase("reference CPU baseline done")
        tight_fix = tight_fixture(y[:, :acc_n], args.steps) if acc_n > 0 else None
        if acc_n > 0 and tight_fix is None:
            from oracle import oracle_available
            if oracle_available():
                tight = start_tight_oracle(y[:, :acc_n].copy(), var[:acc_n].copy(), args.steps * DT,
                                           max(1, (os.cpu_count() or 2) - 2), tight_path)

    model, learn_info = None, None
    if args.learned:
        # train on plain-Radau step records of a batch drawn with another seed (untimed)
        from accelerint_b200 import learned as Lm
        t0 = time.time()
        yt, vt = M.mixed_stiffness_initial_conditions(mech, args.train_num, args.seed + 104729 + rank)
        rec = Lm.record_steps(mech, yt, vt, 0.0, args.steps * DT, DT, capacity=1 << 22, device=dev.index,
                              stage_extrapolation=args.stage_extrapolation)
        model = Lm.train(rec, mech.n_state, epochs=args.train_epochs, batch=args.train_batch,
                         lr=2e-3 if args.train_batch >= 4096 else 1e-3)
        learn_info = {"flags": args.learned, "train_systems": args.train_num, "records": int(rec.shape[0]),
                      "holdout_loss": model.history[-1], "train_s": time.time() - t0}
        del rec
    cost_model = None
    if args.queue_order == 3:
        from accelerint_b200 import learned as Lm
        t0 = time.time()
        yt, vt = M.mixed_stiffness_initial_conditions(mech, 4 * args.train_num, args.seed + 130363 + rank)
        crec = Lm.cost_records(mech, yt, vt, 0.0, args.steps * DT, DT, device=dev.index, lu=lu,
                               stage_extrapolation=args.stage_extrapolation)
        cost_model = Lm.train_cost(crec, mech.n_state)
        learn_info = dict(learn_info or {}, cost_records=int(crec.shape[0]), cost_holdout_loss=cost_model.history[-1],
                          cost_train_s=time.time() - t0)
    phase("training done")
    integ = A.Integrator(args.num, mech, solver=args.solver, device=dev.index, lu=lu,
                         stage_extrapolation=args.stage_extrapolation)
    if model is not None:
        model.install(integ, args.learned)
        integ.lib.accelerInt_set_learned_growth_floor(args.growth_floor)
        learn_info["growth_floor"] = args.growth_floor
    if cost_model is not None:
        cost_model.install_cost(integ)
    stream = torch.cuda.Stream(device=dev)
    y0 = torch.from_numpy(np.ascontiguousarray(y)).to(dev)
    vd = torch.from_numpy(np.ascontiguousarray(var)).to(dev)
    yd = y0.clone()
    codes = torch.zeros(args.num, dtype=torch.int32, device=dev)
    stats = torch.zeros((args.num, A.NSTATS), dtype=torch.int32, device=dev)
    # the state between steps lives in pinned host memory (the end-to-end chain)
    y_host = torch.from_numpy(np.ascontiguousarray(y)).pin_memory()
    codes_host = torch.zeros(args.num, dtype=torch.int32).pin_memory()

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(v):
        if ws > 1:
            import torch.distributed as dist
            tt = torch.tensor([v], device=dev, dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            return float(tt.item())
        return v

    # mapping picked by the library's autotuner on a sample (a copy; untimed), then
    # every launch of the tuned form goes through a captured CUDA graph
    mapping = None
    if not args.no_autotune:
        sample = min(args.num, 8 * 740)
        occ, order, blk, tms = integ.autotune(0.0, DT / 4, DT / 4, y0, vd, sample)
        mapping = {"occupancy_cap": occ, "queue_order": order, "tps_block": blk, "sample_systems": sample,
                   "best_ms": tms}
    if args.queue_order >= 0:
        integ.set_queue_order(args.queue_order)
        if mapping is not None:
            mapping["queue_order"] = args.queue_order
    if not args.no_graph:
        integ.set_graph_launch(True)
    # warm-up: W global steps of dt/1000 on the whole batch through the timed calls, then reset
    dtw = DT * 1e-3
    with torch.cuda.stream(stream):
        for k in range(args.warmup):
            yd.copy_(y_host, non_blocking=True)
            integ.integrate_device(k * dtw, (k + 1) * dtw, dtw, yd, vd, codes, None, stream)
            y_host.copy_(yd, non_blocking=True)
    stream.synchronize()
    y_host.copy_(torch.from_numpy(np.ascontiguousarray(y)))
    if args.queue_order >= 0:
        # a fresh history: the first timed step knows nothing of the warm-up's step counts
        integ.set_queue_order(args.queue_order)
    barrier()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches0 = integ.kernel_launches()
    with ClockSampler(dev.index) as clk:
        barrier()
        t0 = time.perf_counter()
        with torch.cuda.stream(stream):
            for k in range(args.steps):
                flush.fill_(k & 0xff)
                yd.copy_(y_host, non_blocking=True)
                evs[k][0].record(stream)
                integ.integrate_device(k * DT, (k + 1) * DT, DT, yd, vd, codes, stats, stream)
                evs[k][1].record(stream)
                y_host.copy_(yd, non_blocking=True)
                codes_host.copy_(codes, non_blocking=True)
        stream.synchronize()
        wall = time.perf_counter() - t0
        barrier()
    launches = integ.kernel_launches() - launches0
    phase("timed steps done")
    step_ms = [a.elapsed_time(b) for a, b in evs]
    ms = sum(step_ms)
    t_max = max_over_ranks(ms)
    wall_max = max_over_ranks(wall)
    y_tuned = y_host.numpy()
    codes_np = codes_host.numpy()
    nfail = int((codes_np != 0).sum())
    # a non-finite state would make a step look cheap: count them
    nonfinite = int((~np.isfinite(y_tuned)).any(axis=0).sum())
    st = stats.cpu().numpy().astype(np.float64)
    f64, f32 = flops_per_system(st, mech.n_state, mech.n_reactions, args.lu)
    flops64, flops32 = float(f64.sum()), float(f32.sum())
    # work of the timed steps: a global step lasts about max(total work / teams, the
    # slowest system), so run-to-run changes of the slowest system move the number
    work = {"radau_steps": int(st[:, 0].sum()), "rejected": int(st[:, 2].sum()), "factorisations": int(st[:, 4].sum()),
            "newton_iterations": int(st[:, 5].sum()), "rhs": int(st[:, 6].sum()),
            "max_steps_one_system": int(st[:, 0].max()), "flops_fp64": flops64, "flops_fp32": flops32}
    value = ws * args.num * args.steps / (t_max / 1000.0)
    e2e = None
    if not args.no_e2e:
        nb = args.num * (mech.n_state * 8)
        e2e = {"value": ws * args.num * args.steps / wall_max, "unit": UNIT,
               "h2d_bytes_per_step": nb, "d2h_bytes_per_step": nb + args.num * 4,
               "path": "pinned host state -> device, accelerInt_integrate_device, state and codes -> pinned "
                       "host, every step; wall time of the loop (the L2 flush writes included)"}
    roofline = None
    if rank == 0:
        p64, p32s, p32x2 = measure_peak(1), measure_peak(0), measure_peak(2)
        p32 = max(p32s or 0.0, p32x2 or 0.0) or None
        a64 = flops64 / (ms / 1000.0) / 1e12
        a32 = flops32 / (ms / 1000.0) / 1e12
        f64r = a64 / p64 if p64 else None
        f32r = a32 / p32 if p32 else None
        roofline = {"bound": "fp64+fp32 (CUDA-core FMA pipes; the kernel is issue- and latency-bound, HBM ~0)",
                    "achieved": a64 + a32, "peak": None, "unit": "TFLOP/s",
                    "frac": (f64r or 0.0) + (f32r or 0.0),
                    "fp64": {"achieved": a64, "peak": p64, "frac": f64r},
                    "fp32": {"achieved": a32, "peak": p32, "peak_scalar_ffma": p32s, "peak_packed_ffma2": p32x2,
                             "frac": f32r},
                    "traffic": None,
                    "algorithmic_bytes": args.num * (2 * mech.n_state + 1) * 8,
                    "note": "algorithmic flops from device event counters per system, split by pipe "
                            "(factorisations and solves of the FP32 matrices on the FP32 pipe, the rest FP64), "
                            "over the summed event time of the timed launches; peaks = FMA microbenchmarks "
                            "measured in this run (FP32: the larger of scalar and packed FP32x2); frac = the sum "
                            "of the two pipes' fractions"}

    # the plain FP64 form on the same batch and steps, for the tuned-vs-plain ratio
    plain, y_plain = None, None
    if args.plain_steps > 0 and args.lu != "fp64":
        # the plain form: FP64 factorisations, one team per system over a plain grid
        # (no work queue, no graph, no tuning)
        pinteg = A.Integrator(args.num, mech, solver=args.solver, device=dev.index, lu=A.LU_FP64)
        pinteg.set_persistent(False)
        nw = min(args.num, 4 * 148)
        yw = y0[:, :nw].contiguous()
        pinteg.integrate_device(0.0, dtw, dtw, yw, vd[:nw].contiguous(), None, None, stream)   # warm-up
        yd.copy_(y0)
        stats.zero_()   # the tuned form's counters were read above; now the plain form's
        pev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.plain_steps)]
        barrier()
        with torch.cuda.stream(stream):
            for k in range(args.plain_steps):
                flush.fill_(k & 0xff)
                pev[k][0].record(stream)
                pinteg.integrate_device(k * DT, (k + 1) * DT, DT, yd, vd, None, stats, stream)
                pev[k][1].record(stream)
        barrier()
        pstep = [a.elapsed_time(b) for a, b in pev]
        pms = max_over_ranks(sum(pstep))
        pinteg.close()
        pval = ws * args.num * args.plain_steps / (pms / 1000.0)
        # tuned over the same global steps
        tms = max_over_ranks(sum(step_ms[:args.plain_steps]))
        tval = ws * args.num * args.plain_steps / (tms / 1000.0)
        pst = stats.cpu().numpy().astype(np.float64)
        pwork = {"radau_steps": int(pst[:, 0].sum()), "rejected": int(pst[:, 2].sum()),
                 "factorisations": int(pst[:, 4].sum()), "newton_iterations": int(pst[:, 5].sum()),
                 "max_steps_one_system": int(pst[:, 0].max())}
        plain = {"value": pval, "unit": UNIT, "ms_per_step": pms / args.plain_steps, "steps": args.plain_steps,
                 "tuned_over_plain": tval / pval, "ms_per_global_step": pstep, "work": pwork,
                 "newton_iterations_per_step": pwork["newton_iterations"] / max(1, pwork["radau_steps"]),
                 "rejected_share": pwork["rejected"] / max(1, pwork["radau_steps"])}
        if args.plain_steps == args.steps:
            # the precision form's Newton iterations per step and rejected share, against these
            work["newton_iterations_per_step"] = work["newton_iterations"] / max(1, work["radau_steps"])
            work["rejected_share"] = work["rejected"] / max(1, work["radau_steps"])
        if args.plain_steps == args.steps:
            y_plain = yd[:, :acc_n].cpu().numpy()
    integ.close()
    phase("plain form done")

    if rank == 0:
        acc = None
        if tight is not None or tight_fix is not None:
            y_tight, tcodes = tight_fix if tight_fix is not None else finish_tight_oracle(tight, tight_path)
            if y_tight is not None:
                # systems the tight run did not finish (a nonzero code) are left out
                ok = tcodes == 0
                acc = {"oracle": "oracle radau2a at rtol 1e-12 / atol 1e-20 (plain-C restatement of "
                                 "radau2a/radau2a.c)"
                                 + (", committed solution tests/golden/tight/bench_ma54_1m_seed2024_20steps.npz "
                                    "(its initial states checked by SHA-256)" if tight_fix is not None else
                                    ", integrated during this run"),
                       "systems": int(ok.sum()),
                       "tight_oracle_failed": int((~ok).sum()),
                       "interval": f"0 .. {args.steps} x 1e-6 s in global steps of 1e-6 s",
                       "tuned": accuracy(y_tuned[:, :acc_n][:, ok], y_tight[:, ok])}
                if y_plain is not None:
                    acc["plain_fp64"] = accuracy(y_plain[:, ok], y_tight[:, ok])
                if y_ref_cpu is not None and y_ref_cpu.shape[1] >= acc_n:
                    acc["reference_cpu_rtol1e-6"] = accuracy(y_ref_cpu[:, :acc_n][:, ok], y_tight[:, ok])
        ref_gpu = None
        if args.ref_gpu_sample > 0:
            # one GPU against one GPU: rank 0's own batch
            f_t = args.num / (step_ms[0] / 1000.0)
            f_p = args.num / (plain["ms_per_global_step"][0] / 1000.0) if plain else None
            ref_gpu = guarded(reference_gpu_leg, args, mech, y, var, f_t, f_p)
        phase("accuracy and reference GPU done")
        conf1 = None if args.no_config1 else guarded(config1_leg, dev)
        phase("van der Pol line done")
        conf2 = None if args.no_config2 else guarded(config2_leg, dev, args)
        mb = args.num * mech.n_state * 8 / 1e6
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if args.lu == "fp64" else "f64 (E1/E2 factorised and solved in f32)",
                "data": "synthetic",
                "config": {"workload": f"mass-action 53 species / 325 reactions, mixed stiffness, {args.num} ICs "
                                       f"per GPU, global steps of dt=1e-6 s from t=0, {args.solver} rtol 1e-6 "
                                       f"atol 1e-10, LU {args.lu}, persistent work-queue team kernel"
                                       + (f", learned proposals {args.learned}" if args.learned else "")
                                       + (", collocation starting values" if args.stage_extrapolation else
                                          ", the reference's starting values"),
                           "l2": f"L2 flushed (256 MiB write) before every timed step; state y is {mb:.0f} MB",
                           "warmup": f"{args.warmup} global steps of dt/1000 on the whole batch, then reset",
                           "failed_systems": nfail, "nonfinite_systems": nonfinite,
                           "mapping": mapping, "launch": "persistent kernel, "
                           + ("captured CUDA graph" if not args.no_graph else "direct launch")},
                "clocks": clk.summary(), "e2e": e2e, "gpu_launches": launches,
                "roofline": roofline, "cpu_baseline": cb, "plain_fp64": plain, "accuracy": acc,
                "learned": learn_info, "work": work, "ms_per_global_step": step_ms,
                "reference_gpu": ref_gpu, "config1_van_der_pol": conf1, "config2_13_species": conf2}
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
