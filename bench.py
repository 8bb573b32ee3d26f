#!/usr/bin/env python
"""Throughput benchmark: ODE systems/s per global Delta-t step.

Workload (default): the 53-species / 325-reaction synthetic mechanism, 65,536
initial conditions of the mixed-stiffness generator (half near equilibrium at
800-1200 K, half ignition at 1400-2400 K, interleaved), Radau IIA at rtol 1e-6 /
atol 1e-10, global steps of dt = 1e-6 s from t = 0.  The 1,048,576-IC batch is
`--num 1048576`; one global step of it takes minutes, so the default run uses a
65,536-IC batch from the same generator.  A bench step is one global Delta-t
step of all systems; the timed region runs K consecutive global steps starting
from the initial conditions (the warm-up runs W steps from the same initial
conditions, then the state is reset), so the transient after t = 0 is always
inside the timed region.  L2 is flushed (a 256 MiB write) between timed steps,
outside the per-step event pairs.

The tuned form is three changes on top of the plain FP64 form:
E1/E2 factorised and solved in FP32 (--lu), the persistent work-queue kernel
under a captured CUDA graph with the autotuned mapping and a longest-first
queue order from a learned per-system cost model (--queue-order 3), and the
learned step-size proposals (--learned).  Both networks are trained, untimed,
by the library's kernels on plain Radau runs of batches drawn with other seeds.  The plain FP64 form (one
team per system over a plain grid, FP64 factorisations, no proposals) is timed
on the same batch for `--plain-steps` global steps and reported as
"plain_fp64" with the tuned / plain ratio.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--lu fp32|fp64] [--num NUM] [--solver radau2a]

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
    p.add_argument("--num", type=int, default=1 << 16)
    p.add_argument("--solver", default="radau2a")
    p.add_argument("--seed", type=int, default=2024)
    p.add_argument("--cpu-sample", type=int, default=0, help="systems in the CPU baseline sample (0: auto)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-autotune", action="store_true")
    p.add_argument("--queue-order", type=int, default=3, choices=[-1, 0, 1, 2, 3],
                   help="work-queue order (-1: the autotuner's choice; 0 index, 1 hottest first, 2 most steps "
                        "in the previous call first, its history restarted before the timed region; 3 largest "
                        "learned cost first)")
    p.add_argument("--no-graph", action="store_true")
    p.add_argument("--learned", type=int, default=1, choices=[0, 1, 2, 3],
                   help="learned proposals in the tuned form: 1 step size, 2 stages, 3 both (0: off)")
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
def flops_per_system(stats, n=54, R=325):
    """Algorithmic FP64 flops from the device event counters (FMA = 2 flops).

    decomp: (2/3) N^3 real LU + (8/3) N^3 complex LU + N^2 (E1/E2 assembly);
    newton: 3 RHS (counted separately) + 2 N^2 real + 8 N^2 complex triangular
            solves + 30 N for transforms/updates + 12 N for the norms;
    aux (error-estimate solves): 2 N^2 + 8 N;
    rhs: 14 R + 10 N mass-action evaluation (2 exp counted as 0 flops);
    jac: 60 R + 4 N^2."""
    d, nw, rhs, aux, jac = (stats[:, 4], stats[:, 5], stats[:, 6], stats[:, 7], stats[:, 3])
    f = (d * ((2.0 / 3.0) * n ** 3 + (8.0 / 3.0) * n ** 3 + n * n) +
         nw * (2 * n * n + 8 * n * n + 42 * n) + aux * (2 * n * n + 8 * n) +
         rhs * (14 * R + 10 * n) + jac * (60 * R + 4 * n * n))
    return f


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


def measure_fp64_peak(torch):
    from accelerint_b200 import load_library
    lib = load_library()
    import ctypes
    out = ctypes.c_double(0.0)
    lib.accelerInt_measure_fma_peak.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    rc = lib.accelerInt_measure_fma_peak(1, ctypes.byref(out))
    return out.value if rc == 0 else None


# ---------------------------------------------------------------- CPU baseline
def cpu_baseline(args, mech, y, var):
    """Reference CPU radau2a (oracle/_ref, the reference's own C sources) on a bounded sample."""
    sys.path.insert(0, ROOT)
    from oracle import Reference, reference_available, Oracle, oracle_available
    nthreads = os.cpu_count() or 1
    # 128 systems per thread: the first three 53-species global steps cost ~0.08 s
    # per system on one core, so the sample takes ~10 s whatever the core count, and
    # holds enough of the few very stiff systems for a stable rate
    sample = args.cpu_sample or min(args.num, 16384, 128 * nthreads)
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
        return None
    return {"value": sample * args.steps / el, "unit": UNIT, "cores": nthreads, "kind": kind,
            "sample": f"first {sample} systems (both stiffness halves) x {args.steps} global steps from t=0, "
                      f"{nthreads} OpenMP threads, {el:.2f} s"}


def run_reference_arm(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    mech, y, var = workload(args.num, args.seed)
    cb = cpu_baseline(args, mech, y, var)
    if cb is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU build (oracle/_ref) and oracle missing"}))
        return 0
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * args.num / cb["value"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": "mass-action 53 species / 325 reactions, mixed stiffness, "
                                                       f"{args.num} ICs, dt=1e-6 s, radau2a rtol 1e-6 atol 1e-10",
                                            "solver": "radau2a (reference CPU, OpenMP)"},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


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
    model, learn_info = None, None
    if args.learned:
        # train on plain-Radau step records of a batch drawn with another seed (untimed)
        from accelerint_b200 import learned as Lm
        t0 = time.time()
        yt, vt = M.mixed_stiffness_initial_conditions(mech, args.train_num, args.seed + 104729 + rank)
        rec = Lm.record_steps(mech, yt, vt, 0.0, args.steps * DT, DT, capacity=1 << 22, device=dev.index)
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
        crec = Lm.cost_records(mech, yt, vt, 0.0, args.steps * DT, DT, device=dev.index, lu=lu)
        cost_model = Lm.train_cost(crec, mech.n_state)
        learn_info = dict(learn_info or {}, cost_records=int(crec.shape[0]), cost_holdout_loss=cost_model.history[-1],
                          cost_train_s=time.time() - t0)
    integ = A.Integrator(args.num, mech, solver=args.solver, device=dev.index, lu=lu)
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

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize(dev)

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
    # warm-up: W global steps from the initial conditions, then reset
    with torch.cuda.stream(stream):
        for k in range(args.warmup):
            integ.integrate_device(k * DT, (k + 1) * DT, DT, yd, vd, codes, None, stream)
        yd.copy_(y0)
    if args.queue_order >= 0:
        # a fresh history: the first timed step knows nothing of the warm-up's step counts
        torch.cuda.synchronize(dev)
        integ.set_queue_order(args.queue_order)
    barrier()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches0 = integ.kernel_launches()
    with ClockSampler(dev.index) as clk:
        barrier()
        with torch.cuda.stream(stream):
            for k in range(args.steps):
                flush.fill_(k & 0xff)
                evs[k][0].record(stream)
                integ.integrate_device(k * DT, (k + 1) * DT, DT, yd, vd, codes, stats, stream)
                evs[k][1].record(stream)
        barrier()
    launches = integ.kernel_launches() - launches0
    ms = sum(a.elapsed_time(b) for a, b in evs)
    t_max = ms
    if ws > 1:
        import torch.distributed as dist
        tt = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_max = float(tt.item())
    nfail = int((codes != 0).sum().item())
    # a non-finite state with code 0 would make a step look cheap: count them
    nonfinite = int((~torch.isfinite(yd)).any(dim=0).sum().item())
    st = stats.cpu().numpy().astype(np.float64)
    flops = float(flops_per_system(st).sum())
    # work of the timed steps: a global step lasts about max(total work / teams, the
    # slowest system), so run-to-run changes of the slowest system move the number
    work = {"radau_steps": int(st[:, 0].sum()), "rejected": int(st[:, 2].sum()), "factorisations": int(st[:, 4].sum()),
            "newton_iterations": int(st[:, 5].sum()), "rhs": int(st[:, 6].sum()),
            "max_steps_one_system": int(st[:, 0].max()), "flops": flops}
    value = ws * args.num * args.steps / (t_max / 1000.0)
    peak = measure_fp64_peak(torch) if rank == 0 else None
    achieved = flops / (ms / 1000.0) / 1e12
    # DRAM bytes per launch from one ncu capture of the tuned kernel (1,480 systems, one
    # global step: 4.72 MB read + written), scaled by the systems of this launch
    traffic = 4.72e6 / 1480 * args.num if args.lu != "fp64" else None
    roofline = {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": (achieved / peak) if peak else None, "traffic": traffic,
                "traffic_unit": "bytes per launch (ncu capture scaled by systems)",
                "algorithmic_bytes": args.num * (2 * mech.n_state + 1) * 8,
                "note": "algorithmic FP64 flops from device event counters per system "
                        "(decomp, Newton, RHS, error solves, Jacobians) over the kernel time; "
                        "peak = FP64 FMA microbenchmark measured in this run"}
    # e2e: the C-ABI host path (accelerInt_integrate_status) with host buffers, copies inside the timing
    e2e = None
    if not args.no_e2e:
        t0 = time.time()
        yh = y.copy()
        for k in range(args.steps):
            yh, c, rc = integ.integrate(k * DT, (k + 1) * DT, DT, yh, var)
        el = time.time() - t0
        nb = args.num * (mech.n_state + 1) * 8
        e2e = {"value": ws * args.num * args.steps / el, "unit": UNIT,
               "h2d_bytes_per_step": nb, "d2h_bytes_per_step": args.num * mech.n_state * 8 + args.num * 4}
    integ.close()

    # the plain FP64 form on the same batch, for the tuned-vs-plain ratio
    plain = None
    if args.plain_steps > 0 and args.lu != "fp64":
        # the plain form: FP64 factorisations, one team per system over a plain grid
        # (no work queue, no graph, no tuning)
        pinteg = A.Integrator(args.num, mech, solver=args.solver, device=dev.index, lu=A.LU_FP64)
        pinteg.set_persistent(False)
        nw = min(args.num, 4 * 148)
        yw = y0[:, :nw].contiguous()
        pinteg.integrate_device(0.0, DT, DT, yw, vd[:nw].contiguous(), None, None, stream)   # warm-up
        yd.copy_(y0)
        pev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.plain_steps)]
        barrier()
        with torch.cuda.stream(stream):
            for k in range(args.plain_steps):
                flush.fill_(k & 0xff)
                pev[k][0].record(stream)
                pinteg.integrate_device(k * DT, (k + 1) * DT, DT, yd, vd, None, None, stream)
                pev[k][1].record(stream)
        barrier()
        pms = sum(a.elapsed_time(b) for a, b in pev)
        if ws > 1:
            import torch.distributed as dist
            tt = torch.tensor([pms], device=dev, dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            pms = float(tt.item())
        pinteg.close()
        pval = ws * args.num * args.plain_steps / (pms / 1000.0)
        plain = {"value": pval, "unit": UNIT, "ms_per_step": pms / args.plain_steps, "steps": args.plain_steps,
                 "tuned_over_plain": value / pval}

    if rank == 0:
        cb = None if args.no_cpu_baseline else cpu_baseline(args, mech, y, var)
        mb = args.num * mech.n_state * 8 / 1e6
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if args.lu == "fp64" else "f64 (E1/E2 factorised and solved in f32)",
                "data": "synthetic",
                "config": {"workload": f"mass-action 53 species / 325 reactions, mixed stiffness, {args.num} ICs "
                                       f"per GPU, global steps of dt=1e-6 s from t=0, {args.solver} rtol 1e-6 "
                                       f"atol 1e-10, LU {args.lu}, persistent work-queue team kernel"
                                       + (f", learned proposals {args.learned}" if args.learned else ""),
                           "l2": f"L2 flushed (256 MiB write) before every timed step; state y is {mb:.0f} MB",
                           "failed_systems": nfail, "nonfinite_systems": nonfinite,
                           "mapping": mapping, "launch": "persistent kernel, "
                           + ("captured CUDA graph" if not args.no_graph else "direct launch")},
                "clocks": clk.summary(), "e2e": e2e, "gpu_launches": launches,
                "roofline": roofline, "cpu_baseline": cb, "plain_fp64": plain, "learned": learn_info,
                "work": work}
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
