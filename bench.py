#!/usr/bin/env python
"""Benchmark of the B200 forward model on the reference's batched channel
ensemble: 256 seeded draws of (a1, beta*) in [0.28,0.34]x[0.084,0.096], draw i
on the Re_tau {182.088, 550, 1000}[i mod 3] periodic channel with {128, 256,
512} tanh-stretched cells, tol 1e-8, each with a per-draw FP64 Gaussian
log-likelihood against a seeded synthetic profile.

One step = one batched evaluation of the whole ensemble (every draw solved
from cold start to its verdict) with inputs already in HBM. Prints ONE JSON
line (rank 0). `--impl reference` times the reference's own CPU solver
(oracle/_ref, compiled from the reference sources) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
T_START = time.perf_counter()  # process start, for the wall-clock budget

METRIC = "converged RANS-SST solves/s & p99 latency, batched vs plain GPU, <=1e-6 rel err"
UNIT = "solves/s"
# reference iteration counts of the (0.31, 0.09) draw per class at alpha_U 0.8, tol 1e-8
# (CPU pilot of the compiled reference); used only by the CPU arm's extrapolation
REF_ITERS = (12460, 58690, 258900)
BYTES_OUTER, BYTES_KRYLOV, BYTES_PRESSURE = 1600, 360, 400  # algorithmic B/cell (FP64)
# From one ncu capture of solveKernel<768> solving one 1536-cell draw for 600 outer
# iterations (profiles/solveKernel768_1536cells_full_ncu.md):
# * DRAM bytes (read + write): the first touch of the mesh class and the workspace;
#   later iterations hit L2, so the figure does not grow with the iteration count;
# * L2 bytes (lts__t_sectors x 32 B) per outer iteration: what the solve moves
#   between its SM and L2 (L1 misses, spills, stores);
# * the L2's peak: 3 sectors per cycle on each of the 184 slices (ncu's
#   lts__t_sectors peak_sustained) x 32 B at the 1965 MHz clock.
DRAM_BYTES_PER_DRAW_1536 = 2_609_408 + 2_304
L2_BYTES_PER_ITER_1536 = 280_240_249 * 32 / 600
L2_PEAK_GBS = 3 * 32 * 184 * 1.965


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--draws", type=int, default=256)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--cpu-sample-iters", type=int, default=1500)
    ap.add_argument("--max-iter", type=int, default=None,
                    help="cap on outer iterations per draw (profiling runs only; the "
                         "workload's own cap is 300000)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="ensemble",
                    choices=["ensemble", "linear", "serve", "bump", "calibrate", "plain"],
                    help="ensemble: the 256-draw channel ensemble (headline); linear: 512 "
                         "variable-coefficient Poisson systems by AMG-PCG; serve: open-loop "
                         "Poisson arrivals of channel requests to the serving loop")
    ap.add_argument("--rate", default="200,500,1000,2000",
                    help="serve: arrivals per second (a comma list runs one stream per rate)")
    ap.add_argument("--requests", type=int, default=96, help="serve: requests in the stream")
    ap.add_argument("--systems", type=int, default=512)
    ap.add_argument("--cpu-sample-systems", type=int, default=12)
    ap.add_argument("--budget-s", type=float, default=1400.0,
                    help="wall-clock budget of the whole GPU run from process start: timed "
                         "steps stop when the next one would not finish inside it (the line "
                         "reports the requested and the timed step counts)")
    ap.add_argument("--reference-budget-s", type=float, default=240.0,
                    help="--impl reference: wall-clock budget of its samples")
    return ap.parse_args()


# ---------------------------------------------------------------- CPU arm (reference)
def _ref_pool(workers: int):
    """Processes (spawned, so no GPU state is inherited) for the reference's CPU
    solver, which is not safe to run from several threads of one process."""
    import multiprocessing
    from concurrent.futures import ProcessPoolExecutor

    return ProcessPoolExecutor(max_workers=workers, mp_context=multiprocessing.get_context("spawn"))


def _ref_ensemble_solve(c: int, a1: float, beta_star: float, max_iter: int):
    """One ensemble draw through the reference's own ForwardModel (oracle/_ref): the
    class's mesh, settings and observation (monitor floors included). Returns
    (wall seconds, outer iterations, status)."""
    sys.path.insert(0, str(ROOT))
    from oracle import checker as ck
    import rans_uq_b200.workloads as wl

    re_tau, ny = wl.CLASSES[c]
    x, y = wl.channel_probes(re_tau)
    observed, sigma = wl.class_observation(c)
    case = ck.Case(ny=ny, re_tau=re_tau, nu=1 / re_tau, yplus=0.5, alpha_u=wl.ALPHA_U,
                   tol=wl.TOL, max_iter=max_iter, obs_x=x, obs_y=y, obs_value=observed,
                   obs_sigma=sigma).with_theta(a1, beta_star)
    t = time.perf_counter()
    o = ck.solve(case, "ref")
    return time.perf_counter() - t, int(o.iterations), o.status


def cpu_ensemble_sample(theta, cls, cores: int, sample_iters: int = 1500):
    """The reference's solver on a seeded subset of the ensemble, one process per
    host core, every core busy (memory and frequency contention included):

    * wave 1: the first `cores` Re_tau 182 draws of the ensemble, each solved to its
      verdict (measured converged solves/s, and the per-iteration time of that class);
    * wave 2: `cores` draws of Re_tau 550 and 1000 (half each), capped at
      `sample_iters` outer iterations (their per-iteration times: one converged draw
      of those classes takes 1-10 CPU minutes).

    Returns a dict: per-class seconds per outer iteration under contention, the
    measured subset, and the draws it ran."""
    theta, cls = np.asarray(theta), np.asarray(cls)
    first = [i for i in range(len(cls)) if cls[i] == 0][:cores]
    half = max(cores // 2, 1)
    mid = [i for i in range(len(cls)) if cls[i] == 1][:half]
    big = [i for i in range(len(cls)) if cls[i] == 2][:max(cores - half, 1)]
    with _ref_pool(cores) as ex:
        t0 = time.perf_counter()
        w1 = list(ex.map(_ref_ensemble_solve, [0] * len(first), theta[first, 0], theta[first, 1],
                         [MAX_ITER_CPU] * len(first)))
        wave1 = time.perf_counter() - t0
        rest = mid + big
        w2 = list(ex.map(_ref_ensemble_solve, cls[rest].tolist(), theta[rest, 0], theta[rest, 1],
                         [sample_iters] * len(rest)))
    per_it = [float(np.median([t / max(it, 1) for t, it, _ in w1]))]
    for c, ids in ((1, mid), (2, big)):
        sel = [w2[k] for k, i in enumerate(rest) if cls[i] == c]
        per_it.append(float(np.median([t / max(it, 1) for t, it, _ in sel])))
    conv = sum(1 for _, _, st in w1 if st == "Converged")
    return {"per_iteration_s": per_it, "cores": cores,
            "subset": {"draws": first, "iterations": [it for _, it, _ in w1],
                       "statuses": [st for _, _, st in w1], "wall_s": wave1,
                       "solves_per_s": conv / wave1},
            "capped": {"draws": rest, "iterations": sample_iters}}


def ensemble_iterations_table():
    """Outer iterations of every draw of the 256-draw ensemble as the FP64 GPU path
    counted them (tests/golden/ensemble_iterations.json); None when absent."""
    path = ROOT / "tests" / "golden" / "ensemble_iterations.json"
    if not path.exists():
        return None
    return np.asarray(json.loads(path.read_text())["iterations"], dtype=np.int64)


def cpu_baseline(theta, cls, iters_per_draw, sample, source):
    """The CPU line from one all-core sample: the measured Re_tau 182 subset, and the
    whole ensemble extrapolated as sum over draws of (that draw's outer iterations x
    its class's contended per-iteration time) / cores."""
    cores, t_it = sample["cores"], sample["per_iteration_s"]
    iters = np.asarray(iters_per_draw, dtype=np.int64).copy()
    for k, i in enumerate(sample["subset"]["draws"]):  # measured counts where we have them
        if i < len(iters):
            iters[i] = sample["subset"]["iterations"][k]
    total = float(sum(iters[i] * t_it[int(cls[i])] for i in range(len(cls))))
    value = len(cls) / (total / cores)
    sub = sample["subset"]
    return dict(value=value, unit=UNIT, cores=cores, kind="reference",
                measured_subset={"solves_per_s": sub["solves_per_s"], "draws": len(sub["draws"]),
                                 "wall_s": sub["wall_s"],
                                 "what": "Re_tau 182 draws of the ensemble solved to their "
                                         "verdicts, one process per core, all cores busy"},
                extrapolated={"solves_per_s": value,
                              "per_iteration_ms": [1e3 * t for t in t_it],
                              "iterations_from": source},
                sample=(f"reference ForwardModel (oracle/_ref, g++ -O2) on {cores} processes: "
                        f"{len(sub['draws'])} Re_tau 182 draws converged ({sub['wall_s']:.1f} s), "
                        f"then {len(sample['capped']['draws'])} Re_tau 550/1000 draws capped at "
                        f"{sample['capped']['iterations']} outer iterations; per-iteration times "
                        f"{['%.3g ms' % (1e3 * t) for t in t_it]} x each draw's outer iterations "
                        f"({source}) / {cores} cores (extrapolated; measured subset reported "
                        f"beside it)"))


MAX_ITER_CPU = 300000  # the ensemble's own cap


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import rans_uq_b200.workloads as wl

    if not (ROOT / "oracle" / "_ref" / "libcfdr_ref.so").exists():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built"}))
        return
    ids = np.arange(args.draws)
    cls = ids % 3
    theta = wl.uniform_design(ids)
    table = ensemble_iterations_table()
    if table is not None and len(table) >= len(ids):
        iters, source = table[: len(ids)], "the FP64 GPU solve of the same draw, " \
                                           "tests/golden/ensemble_iterations.json"
    else:
        iters, source = np.array([REF_ITERS[c] for c in cls]), \
            "the reference's count at (0.31, 0.09) per class"
    cores = os.cpu_count() or 1
    vals, steps, t_start = [], 0, time.perf_counter()
    # each step is one all-core sample (about 15 s); stop early rather than run past
    # the budget (the sample, not the step count, is what the line reports)
    while steps < max(args.steps, 1):
        vals.append(cpu_baseline(theta, cls, iters, cpu_ensemble_sample(theta, cls, cores),
                                 source))
        steps += 1
        per = (time.perf_counter() - t_start) / steps
        if time.perf_counter() - t_start + per > args.reference_budget_s:
            break
    cb = vals[-1]
    v = statistics.median(x["value"] for x in vals)
    cb["value"] = v
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "steps_requested": args.steps, "warmup": 0,
        "warmup_requested": args.warmup, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "256-draw channel ensemble, Re_tau {182,550,1000} x {128,256,512} cells",
                   "draws": args.draws, "tol": wl.TOL, "alpha_u": wl.ALPHA_U},
        "cpu_baseline": cb,
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


# ---------------------------------------------------------------- GPU arm
class Clocks:
    """nvidia-smi samples (every 200 ms) of one GPU's clocks and throttle reasons during
    the timed region, written to a scratch file and summarised into the JSON line."""

    def __init__(self, index: int):
        import tempfile

        self.index, self.proc = index, None
        self.path = Path(tempfile.gettempdir()) / f"rq_clocks_gpu{index}_{os.getpid()}.csv"

    def __enter__(self):
        self.path.parent.mkdir(exist_ok=True)
        self.f = open(self.path, "w")
        self.proc = subprocess.Popen(
            ["nvidia-smi", "-i", str(self.index), "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
             "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"],
            stdout=self.f, stderr=subprocess.DEVNULL)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()
        self.f.close()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = max(mx, float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def plan_timed_steps(requested: int, elapsed_s: float, step_s: float, budget_s: float,
                     reserve_s: float = 30.0) -> int:
    """Timed steps to run: the requested count, cut to those that finish inside the
    wall-clock budget (with a reserve for the summary), and never fewer than one."""
    room = budget_s - elapsed_s - reserve_s
    fit = int(room // step_s) if step_s > 0 else requested
    return max(1, min(int(requested), fit))


def plain_per_iteration(cap: int = 3000):
    """The plain one-solve-at-a-time FP64 GPU path: seconds per outer iteration of
    one solve alone (a grid of one CTA) per Re_tau class, from a capped solve at
    (0.31, 0.09) through the host API."""
    import rans_uq_b200.workloads as wl

    per_it = []
    for re_tau, ny in wl.CLASSES:
        b = wl.channel_batch(re_tau, ny, precision="fp64", max_iter=cap)
        t0 = time.perf_counter()
        r = b.evaluate(np.array([[0.31, 0.09]]))
        per_it.append((time.perf_counter() - t0) / max(r.rows[0].result.simple_iters, 1))
    return per_it


def gpu_arm(args):
    import torch
    import torch.distributed as dist
    import rans_uq_b200 as rq
    import rans_uq_b200.replicas as rp
    import rans_uq_b200.workloads as wl

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)

    # ---- set-up (untimed): the three mesh classes and this rank's draws (weak scaling)
    max_iter = args.max_iter or wl.MAX_ITER
    ids = rp.shard_ids(rank, world, args.draws)
    ens = wl.channel_ensemble(args.draws, precision=args.precision, first_id=int(ids[0]),
                              max_iter=max_iter)
    n = len(ens.theta)
    theta = torch.tensor(ens.theta, dtype=torch.float64, device=dev)
    rows = torch.zeros(n * 40, dtype=torch.uint8, device=dev)     # n x 40-byte rq_row_out
    pred = torch.zeros((n, 30), dtype=torch.float64, device=dev)
    clock = torch.zeros((n, 12), dtype=torch.int64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step(e=ens):
        rq.evaluate_multi_device(e.batches, e.cls, theta.data_ptr(), rows.data_ptr(),
                                 pred.data_ptr(), stream.cuda_stream, clock.data_ptr())

    # ---- untimed legs first, so that a slow step can never cost them: the plain
    # one-solve-at-a-time path (per-iteration cost per class from capped single-solve
    # launches) and, at N = 1, the host CPU baseline's all-core sample
    per_it, cpu_sample = None, None
    if rank == 0:
        per_it = plain_per_iteration()
        if not args.no_cpu_baseline and world == 1 and \
                (ROOT / "oracle" / "_ref" / "libcfdr_ref.so").exists():
            cpu_sample = cpu_ensemble_sample(ens.theta, ens.cls, os.cpu_count() or 1)
    if world > 1:
        dist.barrier()

    # ---- warm-up: W >= 3 steps. All but the last two run the same draws through the
    # same launches with every solve capped at 2000 outer iterations (module load,
    # launch path, first touch); then one full device step (its time sizes the timed
    # loop) and one full step through the host API (theta from host memory in, rows and
    # predictions back to host memory), which is the e2e measurement.
    warm = max(args.warmup, 3)
    capped = wl.channel_ensemble(args.draws, precision=args.precision, first_id=int(ids[0]),
                                 max_iter=min(2000, max_iter))
    for _ in range(warm - 2):
        step(capped)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    step()
    e1.record(stream)
    torch.cuda.synchronize()
    warm_ms = e0.elapsed_time(e1)
    t0 = time.perf_counter()
    res = rq.evaluate_multi(ens.batches, ens.cls, ens.theta)
    e2e_s = time.perf_counter() - t0
    e2e_conv = sum(1 for r in res.rows if r.result.status.name == "Converged")
    e2e_conv_total = rp.reduce_count(e2e_conv, device=dev)
    e2e_s = rp.reduce_max(e2e_s, device=dev)
    # the number of timed steps every rank runs: the requested K, cut to what fits in
    # the budget (the same on every rank: step estimate and elapsed time are maxima)
    est_ms = rp.reduce_max(max(warm_ms, 1e3 * e2e_s), device=dev)
    elapsed = rp.reduce_max(time.perf_counter() - T_START, device=dev)
    k = plan_timed_steps(args.steps, elapsed, est_ms / 1e3, args.budget_s)
    times = []
    with Clocks(local) as clk:
        for _ in range(k):
            flush.fill_(1.0)  # L2 flush between timed steps (outside the events)
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
    ms_rank = float(np.median(times))
    print(f"bench: warm-up step {warm_ms:.1f} ms, timed step(s) {times} ms, e2e {e2e_s:.3f} s",
          file=sys.stderr, flush=True)
    recs = rq.rows_from_device_bytes(rows.cpu().numpy())
    clock_host = clock.cpu().numpy()
    conv = int(np.sum(recs["status"] == 0))
    # step time = max over ranks, converged solves summed over ranks
    ms, total_conv, _ = rp.reduce_step(ms_rank, conv, device=dev)
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    cpu = None  # the host baseline is timed at N = 1 only (rank 0), never beside N > 1 ranks
    if cpu_sample is not None:
        cpu = cpu_baseline(ens.theta, ens.cls, recs["iterations"], cpu_sample,
                           "the FP64 GPU solve of the same draw in this run")
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if \
        (ROOT / "MEASURED_PEAKS.json").exists() else {"hbm_gbs": 6650.0}
    cells = np.array([ens.batches[c]._problem.n_cells for c in ens.cls])
    run = argparse.Namespace(**vars(args))
    run.steps, run.steps_requested, run.warmup, run.warmup_requested = k, args.steps, warm, \
        args.warmup
    out = summarize(recs, clock_host, ens.cls, cells, ms, total_conv, world, run, max_iter,
                    e2e_conv_total / e2e_s, n * 2 * 8 + n * 64, n * 40 + n * 30 * 8, per_it,
                    peaks, clk.summary(), cpu)
    out["timing"] = {"warmup_step_ms": warm_ms, "timed_steps_ms": times,
                     "e2e_step_s": e2e_s, "budget_s": args.budget_s,
                     "wall_s_at_end": time.perf_counter() - T_START,
                     "warmup_note": f"{warm - 2} capped warm-up step(s) (every solve capped at "
                                    "2000 outer iterations), 1 full device step, 1 full "
                                    "host-API step (the e2e figure)"}
    print(json.dumps(out))
    if world > 1:
        dist.destroy_process_group()


def summarize(recs, clock, cls, cells, ms, total_conv, world, args, max_iter, e2e_value, h2d,
              d2h, per_it, peaks, clocks, cpu):
    """The JSON line from the host copies of one timed step: rows (status, iterations),
    the 12-int64 clock record per row, the class and cell count per row."""
    import rans_uq_b200.workloads as wl

    status, iters = recs["status"], recs["iterations"].astype(np.int64)
    n = len(status)
    conv = int(np.sum(status == 0))
    value = total_conv / (ms / 1e3)
    lat = (clock[:, 1] - clock[:, 0].min()) / 1e6
    work = cells * (BYTES_OUTER * iters + BYTES_KRYLOV * clock[:, 2] + BYTES_PRESSURE * clock[:, 3])
    alg_bytes = float(np.sum(work))
    # dominant launch: the longest per-class solve kernel of the step (device
    # globaltimer: first CTA start to last CTA end of that class's rows)
    per_class = []
    for c in sorted(set(int(x) for x in cls)):
        sel = cls == c
        dur = (clock[sel, 1].max() - clock[sel, 0].min()) / 1e9
        per_class.append((dur, float(np.sum(work[sel])), c))
    dom_s, dom_bytes, dom_c = max(per_class)
    dom_sel = cls == dom_c
    is1536 = int(np.max(cells[dom_sel])) == 1536
    dram = DRAM_BYTES_PER_DRAW_1536 * int(np.sum(dom_sel)) if is1536 else None
    l2 = L2_BYTES_PER_ITER_1536 * float(np.sum(iters[dom_sel])) if is1536 else None
    names = ["setup", "closure", "momentum", "p_assembly", "p_solve", "amg_refresh", "turbulence",
             "bookkeeping"]
    stages = {}
    for c in sorted(set(int(x) for x in cls)):
        sel = (cls == c) & (iters > 0)
        if not np.any(sel):
            continue
        cyc = clock[sel, 4:12].astype(np.float64).sum(0)
        stages[str(c)] = {"share": {k: round(float(v / max(cyc.sum(), 1.0)), 4)
                                    for k, v in zip(names, cyc)},
                          "krylov_per_outer": float(clock[sel, 2].sum() / iters[sel].sum()),
                          "pressure_per_outer": float(clock[sel, 3].sum() / iters[sel].sum())}
    achieved = dom_bytes / dom_s / 1e9
    plain = None
    if per_it is not None:
        plain_s = float(sum(iters[i] * per_it[cls[i]] for i in range(n)))
        plain = {"solves_per_s": conv / plain_s if plain_s > 0 else 0.0,
                 "per_iteration_ms": [1e3 * x for x in per_it],
                 "method": "capped 3000-iteration single-solve launches x each draw's iterations"}
    hbm = peaks.get("hbm_gbs", 6650.0)
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "steps_requested": getattr(args, "steps_requested", args.steps),
        "warmup": args.warmup, "warmup_requested": getattr(args, "warmup_requested", args.warmup),
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
        "data": "synthetic",
        "config": {"workload": "256-draw channel ensemble, Re_tau {182,550,1000} x {128,256,512} cells",
                   "draws_per_gpu": n, "tol": wl.TOL, "alpha_u": wl.ALPHA_U,
                   "precision": args.precision, "l2": "flushed between timed steps",
                   "max_iter": max_iter, "parallelism": f"replicas x{world}"},
        "converged": conv,
        "statuses": {s: int(np.sum(status == k)) for k, s in
                     enumerate(["converged", "unconverged", "diverged", "invalid", "unknown"])},
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "max": float(lat.max()),
                       "note": "per-solve completion time from the start of the step (device timer)"},
        "iterations": {"mean": float(iters.mean()),
                       "by_class": [int(np.median(iters[cls == c])) for c in range(3)
                                    if np.any(cls == c)]},
        "stages_by_class": stages,
        "plain_fp64": plain,
        "batched_vs_plain": value / plain["solves_per_s"] if plain and plain["solves_per_s"] else None,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": len(per_class) * args.steps,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "algorithmic_frac": achieved / hbm,
                     "traffic": dram, "dram_frac": (dram / dom_s / 1e9 / hbm) if dram else None,
                     "l2_bytes": l2, "l2_gbs": (l2 / dom_s / 1e9) if l2 else None,
                     "l2_peak_gbs": L2_PEAK_GBS,
                     "l2_frac": (l2 / dom_s / 1e9 / L2_PEAK_GBS) if l2 else None,
                     "traffic_note": "DRAM: ncu read+write of one 1536-cell draw (first touch; "
                                     "constant in the iteration count) x draws in the launch; "
                                     "L2: ncu L2 bytes per outer iteration of a 1536-cell draw x "
                                     "the launch's outer iterations",
                     "peak_source": "measured" if "gpu_name" in peaks else "fallback",
                     "kernel": f"solveKernel, Re_tau class {dom_c} ({int(np.sum(cls == dom_c))} rows)",
                     "kernel_ms": dom_s * 1e3, "step_bytes_per_s": alg_bytes / (ms / 1e3),
                     "note": "frac = algorithmic_frac: algorithmic FP64 bytes (1600 B/cell/outer "
                             "+ 360 B/cell/Krylov it + 400 B/cell/pressure it) / time / HBM peak, "
                             "a rate of on-chip work, not HBM use: the state lives in shared "
                             "memory, L1 and L2 (dram_frac), and the bound in practice is the "
                             "dependent work of each outer iteration on one SM (instruction "
                             "issue and the latency of L1 misses served by L2: l2_frac)"},
        "clocks": clocks,
        "cpu_baseline": cpu,
    }


# ---------------------------------------------------------------- linear-solve workload
LIN_METRIC = "converged AMG-PCG linear solves/s, 512 Poisson systems n^2, n in {64..512}, tol 1e-10"
LIN_TOL, LIN_MAX_ITER = 1e-10, 500


def lin_bytes_per_iteration(n_rows, nnz, precision):
    """Algorithmic bytes of one AMG-PCG iteration on level 0 (coarse levels not counted):
    5 CSR passes (matvec, 4 in the V-cycle) and ~32 vector passes."""
    vb, cb = (8, 12) if precision == "fp64" else (4, 8)
    return 5 * (cb * nnz + 4 * n_rows) + 32 * vb * n_rows


def _ref_linear_seconds(arrays):
    sys.path.insert(0, str(ROOT))
    from oracle import checker as ck

    diag, upper, lower, source, own, nbr = arrays
    t = time.perf_counter()
    _, info = ck.linear_solve(0, diag, upper, lower, source, own, nbr, np.zeros(len(diag)),
                              LIN_MAX_ITER, LIN_TOL, lib_kind="ref")
    return time.perf_counter() - t, info["iterations"]


def linear_cpu_sample(systems, sample):
    """The reference's AMGSolver::solve (oracle/_ref) on a seeded sample of the
    systems, one process per host core; returns (solves/s for the whole batch
    extrapolated by rows, cores, description)."""
    rng = np.random.default_rng(7)
    idx = sorted(rng.choice(len(systems), size=min(sample, len(systems)), replace=False))
    cores = os.cpu_count() or 1
    args = [(systems[k].diag, systems[k].upper, systems[k].lower, systems[k].source,
             systems[k].own, systems[k].nbr) for k in idx]
    t0 = time.perf_counter()
    with _ref_pool(min(cores, len(idx))) as ex:
        out = list(ex.map(_ref_linear_seconds, args))
    wall = time.perf_counter() - t0
    per_row = sum(t for t, _ in out) / sum(systems[k].n_cells for k in idx)
    total_cpu = per_row * sum(s.n_cells for s in systems)
    value = len(systems) / (total_cpu / cores)
    return value, cores, (f"reference AMGSolver::solve (oracle/_ref, g++ -O2) on {len(idx)} of "
                          f"{len(systems)} systems ({wall:.1f} s wall, one process per core); "
                          f"seconds per row x all rows / {cores} cores (extrapolated)")


def linear_arm(args):
    import rans_uq_b200.linear as lin
    import rans_uq_b200.workloads as wl

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    systems = wl.linear_workload(args.systems, seed=wl.LINEAR_SEED + 1000 * rank)
    config = {"workload": f"{args.systems} variable-coefficient 5-point Poisson systems, n x n, "
                          "n uniform in {64,128,256,512}, log-normal faces, Dirichlet edge",
              "systems_per_gpu": args.systems, "tol": LIN_TOL, "solver": "AMG-PCG",
              "precision": args.precision, "parallelism": f"replicas x{world}"}
    if args.impl == "reference":
        if rank != 0:
            return
        v, cores, sample = linear_cpu_sample(systems, args.cpu_sample_systems)
        print(json.dumps({"impl": "reference", "metric": LIN_METRIC, "value": v,
                          "unit": "systems/s", "n_gpus": args.gpus, "steps": args.steps,
                          "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                          "config": config,
                          "cpu_baseline": {"value": v, "unit": "systems/s", "cores": cores,
                                           "kind": "reference", "sample": sample},
                          "e2e": {"value": v, "unit": "systems/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return
    import torch
    import rans_uq_b200.replicas as rp

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream(dev)
    t0 = time.perf_counter()
    batch = lin.LinearBatch(systems, kind="AMG", precision=args.precision)
    setup_s = time.perf_counter() - t0
    info = batch.info()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        batch.solve_device(LIN_MAX_ITER, LIN_TOL, stream.cuda_stream)
    torch.cuda.synchronize()
    times = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        batch.solve_device(LIN_MAX_ITER, LIN_TOL, stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    res, _ = batch.results()
    iters = np.array([r.iterations for r in res])
    conv = int(sum(r.converged for r in res))
    ms, total_conv, _ = rp.reduce_step(float(np.median(times)), conv, device=dev)
    batch.destroy()
    # end to end through the one-shot public call: host arrays in and out, host set-up included
    t0 = time.perf_counter()
    res_e2e, xs = lin.solve_batch(systems, kind="AMG", precision=args.precision,
                                  max_iter=LIN_MAX_ITER, tol=LIN_TOL)
    e2e_s = time.perf_counter() - t0
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    nnz = np.array([s.n_cells + 2 * s.n_if for s in systems])
    rows = np.array([s.n_cells for s in systems])
    alg = float(np.sum(iters * lin_bytes_per_iteration(rows, nnz, args.precision)))
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if \
        (ROOT / "MEASURED_PEAKS.json").exists() else {"hbm_gbs": 6650.0}
    hbm = peaks.get("hbm_gbs", 6650.0)
    achieved = alg / (ms / 1e3) / 1e9
    cpu = None
    if not args.no_cpu_baseline and (ROOT / "oracle" / "_ref" / "libcfdr_ref.so").exists():
        v, cores, sample = linear_cpu_sample(systems, args.cpu_sample_systems)
        cpu = {"value": v, "unit": "systems/s", "cores": cores, "kind": "reference",
               "sample": sample}
    h2d = int(sum(8 * (2 * s.n_cells + 2 * s.n_if) + 8 * s.n_if for s in systems))
    print(json.dumps({
        "metric": LIN_METRIC, "value": total_conv / (ms / 1e3), "unit": "systems/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32+f64", "data": "synthetic",
        "config": dict(config, l2="flushed between timed steps; working set above L2"),
        "converged": conv, "iterations": {"mean": float(iters.mean()), "max": int(iters.max()),
                                          "by_n": {int(n): float(iters[rows == n * n].mean())
                                                   for n in wl.LINEAR_SIZES if np.any(rows == n * n)}},
        "setup_s": setup_s, "rows": info["rows"], "nnz_all_levels": info["nnz"],
        "e2e": {"value": sum(r.converged for r in res_e2e) / e2e_s, "unit": "systems/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": int(8 * rows.sum() + 24 * len(systems)),
                "note": "one-shot rq_linear_solve_batch: host set-up, upload, solve, download"},
        "gpu_launches": args.steps,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": None, "kernel": "linKernel<512>",
                     "note": "algorithmic level-0 bytes per AMG-PCG iteration (5 CSR passes + 32 "
                             "vector passes) x iterations; coarse levels not counted"},
        "cpu_baseline": cpu,
    }))
    if world > 1:
        dist.destroy_process_group()


# ---------------------------------------------------------------- serving workload
SERVE_METRIC = "served converged RANS-SST solves/s with p50/p99 request latency (open-loop arrivals)"


def student_t_theta(ids, seed=20261012, center=(0.324, 0.0968), std=(0.004, 0.0012), rho=0.3,
                    nu=4.0):
    """Seeded bivariate Student-t draws, the construction of the reference's importance
    proposal (docs/figures/calibration_coverage.py:165-180) with the serving stream's
    centre, scales and correlation."""
    import rans_uq_b200.workloads as wl

    cov = np.array([[std[0] ** 2, rho * std[0] * std[1]], [rho * std[0] * std[1], std[1] ** 2]])
    chol = np.linalg.cholesky(cov)
    out = []
    for i in ids:
        rng = wl.sample_rng(seed, int(i), "student-t-proposal")
        z, chi2 = rng.standard_normal(2), rng.chisquare(nu)
        out.append(np.asarray(center) + chol @ z * np.sqrt(nu / chi2))
    return np.array(out)


SERVE_BUMP_SIZES = ((100, 50), (200, 100), (400, 200))
SERVE_BUMP_CAP = 200


def serve_stream(n, seed=20261013):
    """The request mix of one stream: 70 % channel (Re_tau 182 / 550 / 1000 equally) and
    30 % bump-wall (100 x 50, 200 x 100, 400 x 200 equally; capped at 200 outer
    iterations, so they come back flagged Unconverged); theta from the Student-t
    proposal; 5 % poisoned, half out of bounds (a1 = 0.95: InvalidParameters) and half
    in bounds but far from the box ((a1, beta*) = (0.1, 0.2), which does not converge).
    Returns (class index per request: 0-2 channel, 3-5 bump; theta; poisoned mask)."""
    rng = np.random.default_rng(seed)
    bump = rng.random(n) < 0.30
    cls = np.where(bump, 3 + rng.integers(0, 3, n), rng.integers(0, 3, n))
    theta = student_t_theta(range(n))
    poisoned = rng.random(n) < 0.05
    far = poisoned & (rng.random(n) < 0.5)
    theta[poisoned & ~far, 0] = 0.95
    theta[far] = (0.1, 0.2)
    return cls, theta, poisoned


def serve_one_rate(rq, batches, rate, R, seed):
    cls, theta, poisoned = serve_stream(R, seed)
    rng = np.random.default_rng(seed + 1)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, R))
    srv = rq.ForwardServer(batches, capacity=R, idle_timeout=10.0)
    done_at = np.full(R, np.nan)
    results = [None] * R
    tickets = []
    t0 = time.perf_counter()

    def poll_all():
        for k, t in enumerate(tickets):
            if results[k] is None:
                r = srv.poll(t)
                if r is not None:
                    results[k] = r
                    done_at[k] = time.perf_counter() - t0

    for i in range(R):
        while time.perf_counter() - t0 < arrivals[i]:
            poll_all()
            time.sleep(2e-4)
        tickets.append(srv.submit(int(cls[i]), theta[i]))
    while any(r is None for r in results):
        poll_all()
        time.sleep(1e-3)
        if time.perf_counter() - t0 > 3600:
            break
    span = float(np.nanmax(done_at))
    info, mem = srv.info(), srv.memory()
    srv.destroy()
    lat = done_at - arrivals
    status = np.array([int(r.status) for r in results])
    conv = status == 0
    service = np.array([(r.end_ns - r.start_ns) / 1e9 for r in results])
    return {
        "rate_per_s": rate, "requests": R, "converged": int(conv.sum()),
        "converged_per_s": float(conv.sum() / span), "span_s": span,
        "poisoned": int(poisoned.sum()),
        "poisoned_flagged": int(sum(1 for k in range(R) if poisoned[k] and results[k].flagged)),
        "returned_poisoned": int(sum(1 for k in range(R) if poisoned[k] and
                                     results[k].predictions is not None)),
        "statuses": {s: int(np.sum(status == k)) for k, s in
                     enumerate(["converged", "unconverged", "diverged", "invalid", "unknown"])},
        "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                      "max": float(lat.max())},
        "latency_converged_s": ({"p50": float(np.percentile(lat[conv], 50)),
                                 "p99": float(np.percentile(lat[conv], 99))} if conv.any() else None),
        "service_s": {"p50": float(np.percentile(service, 50)),
                      "p99": float(np.percentile(service, 99))},
        "slots": info["slots"], "kernel_launches": info["launches"],
        "pool_bytes": mem["pool_bytes"]}


def serve_arm(args):
    """Open-loop Poisson arrivals of the mixed stream (serve_stream) to the serving
    loop, one stream per rate, each on a fresh server over the same six mesh classes."""
    import torch
    import rans_uq_b200 as rq
    import rans_uq_b200.workloads as wl

    if int(os.environ.get("RANK", "0")) != 0:
        return
    torch.cuda.set_device(0)
    ens = wl.channel_ensemble(3)
    bumps = [wl.bump_batch(nx, ny, max_iter=SERVE_BUMP_CAP) for nx, ny in SERVE_BUMP_SIZES]
    batches = ens.batches + bumps
    rates = [float(r) for r in str(args.rate).split(",")]
    per_rate = []
    with Clocks(0) as clk:
        for k, rate in enumerate(rates):
            per_rate.append(serve_one_rate(rq, batches, rate, args.requests, 20261013 + k))
            print(f"serve: rate {rate}: {json.dumps(per_rate[-1])}", file=sys.stderr, flush=True)
    top = per_rate[-1]
    print(json.dumps({
        "metric": SERVE_METRIC, "value": top["converged_per_s"], "unit": "solves/s", "n_gpus": 1,
        "steps": len(rates), "warmup": 0, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.requests} requests per rate: 70 % channel (Re_tau "
                               "182/550/1000), 30 % bump-wall (100x50, 200x100, 400x200, capped at "
                               f"{SERVE_BUMP_CAP} outer iterations); Student-t theta (nu 4, centre "
                               "0.324/0.0968); 5 % poisoned (half out of bounds, half far off)",
                   "rates_per_s": rates},
        "per_rate": per_rate, "clocks": clk.summary(),
        "note": "value = converged solves/s over the stream's span at the highest rate; "
                "latency = scheduled arrival to result seen by poll (host clock)"}))


# ---------------------------------------------------------------- bump-wall workload
BUMP_METRIC = "bump-wall RANS-SST outer iterations/s, 32 draws on 200x100 cells (capped solves)"


def _ref_bump_seconds_per_iteration(theta, iters: int) -> float:
    sys.path.insert(0, str(ROOT))
    from oracle import checker as ck
    import rans_uq_b200.workloads as wl

    xn, yb = wl.bump_geometry(200)
    case = ck.Case(nx=200, ny=100, curved=True, x_nodes=xn, y_bottom=yb, y_top=3.04,
                   re_mesh=5600.0, yplus=1.0, nu=1 / 5600.0, bc=(1.0, 1e-4, 10.0),
                   init_u=(0.3, 0.0, 0.0), init_k=1e-4, init_w=10.0, alpha_u=0.4,
                   alpha_p=0.25, body_force=(4e-3, 0.0, 0.0), tol=1e-8, max_iter=iters,
                   obs_x=np.full(6, 2.0), obs_y=np.linspace(0.2, 2.8, 6),
                   obs_value=np.zeros(6), obs_sigma=np.full(6, 1e-2)).with_theta(*theta)
    t = time.perf_counter()
    o = ck.solve(case, "ref")
    return (time.perf_counter() - t) / max(o.iterations, 1)


def bump_cpu_sample(iters: int = 10, draws: int = 16):
    """The reference's solver (oracle/_ref) on the same mesh and settings: `draws`
    solves capped at `iters` outer iterations, one process per host core; returns
    the median seconds per outer iteration per solve and the process count."""
    import rans_uq_b200.workloads as wl

    cores = os.cpu_count() or 1
    theta = [tuple(t) for t in wl.uniform_design(range(draws))]
    with _ref_pool(min(cores, draws)) as ex:
        per = list(ex.map(_ref_bump_seconds_per_iteration, theta, [iters] * draws))
    return float(np.median(per)), min(cores, draws)


def bump_arm(args):
    import torch
    import rans_uq_b200 as rq
    import rans_uq_b200.workloads as wl

    if int(os.environ.get("RANK", "0")) != 0:
        return
    torch.cuda.set_device(0)
    cap = args.max_iter or 200
    batch = wl.bump_batch(200, 100, max_iter=cap)
    theta = wl.uniform_design(range(32))
    n = len(theta)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    th = torch.tensor(theta, dtype=torch.float64, device=dev)
    rows = torch.zeros(n * 40, dtype=torch.uint8, device=dev)
    pred = torch.zeros((n, 6), dtype=torch.float64, device=dev)
    clock = torch.zeros((n, 12), dtype=torch.int64, device=dev)
    cls = np.zeros(n, np.int32)

    def step():
        rq.evaluate_multi_device([batch], cls, th.data_ptr(), rows.data_ptr(), pred.data_ptr(),
                                 stream.cuda_stream, clock.data_ptr())

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    times = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = float(np.median(times))
    recs = rq.rows_from_device_bytes(rows.cpu().numpy())
    iters = recs["iterations"].astype(np.int64)
    ck_ = clock.cpu().numpy()
    per_solve_ms = float(np.median((ck_[:, 1] - ck_[:, 0]) / 1e6 / np.maximum(iters, 1)))
    value = float(iters.sum()) / (ms / 1e3)
    cpu = None
    if not args.no_cpu_baseline and (ROOT / "oracle" / "_ref" / "libcfdr_ref.so").exists():
        sec, cores = bump_cpu_sample()
        cpu = {"value": cores / sec, "unit": "outer iterations/s", "cores": cores,
               "kind": "reference",
               "sample": f"16 reference solves capped at 10 outer iterations on {cores} threads: "
                         f"{1e3 * sec:.1f} ms per outer iteration per solve; value = threads / that"}
    print(json.dumps({
        "metric": BUMP_METRIC, "value": value, "unit": "outer iterations/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "bump-wall channel 200 x 100 (h 1, L 9h, W 4h, top 3.04h, Re 5600), "
                               "32 draws of the prior box", "max_iter": cap},
        "per_solve_ms_per_outer_iteration": per_solve_ms,
        "statuses": {s: int(np.sum(recs["status"] == k)) for k, s in
                     enumerate(["converged", "unconverged", "diverged", "invalid", "unknown"])},
        "krylov_per_outer": float(ck_[:, 2].sum() / max(iters.sum(), 1)),
        "pressure_per_outer": float(ck_[:, 3].sum() / max(iters.sum(), 1)),
        "gpu_launches": args.steps, "cpu_baseline": cpu,
    }))


# ---------------------------------------------------------------- plain small case
PLAIN_METRIC = "plain FP64 solve time, Re_tau 182 channel on 3 x 128 cells to tol 1e-10"


def plain_cpu_seconds_per_iteration(cap: int = 20000) -> float:
    """The reference's own ForwardModel (oracle/_ref) on the same case, capped at `cap`
    outer iterations on one host thread (about 20 s): seconds per outer iteration."""
    import dataclasses

    from oracle import checker as ck

    t = time.perf_counter()
    out = ck.solve(dataclasses.replace(ck.config1_case(), max_iter=cap), "ref")
    return (time.perf_counter() - t) / max(out.iterations, 1)


def plain_arm(args):
    """Configuration 1 (one plain solve): one cold FP64 solve at (a1, beta*) = (0.31, 0.09) on
    the 3 x 128 channel (y+ 0.5, alpha_U 0.5, tol 1e-10, cap 150000), timed on the device
    with theta resident, and once more through the host API (e2e)."""
    import torch
    import rans_uq_b200 as rq
    import rans_uq_b200.workloads as wl

    if int(os.environ.get("RANK", "0")) != 0:
        return
    torch.cuda.set_device(0)
    batch = wl.channel_batch(182.088, 128, observed=np.zeros(30), sigma=np.full(30, 1e-3),
                             alpha_u=0.5, tol=1e-10, max_iter=150000)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    th = torch.tensor([[0.31, 0.09]], dtype=torch.float64, device=dev)
    rows = torch.zeros(40, dtype=torch.uint8, device=dev)
    pred = torch.zeros((1, 30), dtype=torch.float64, device=dev)
    clock = torch.zeros((1, 12), dtype=torch.int64, device=dev)

    def step():
        rq.evaluate_multi_device([batch], np.zeros(1, np.int32), th.data_ptr(), rows.data_ptr(),
                                 pred.data_ptr(), stream.cuda_stream, clock.data_ptr())

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    times = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = float(np.median(times))
    rec = rq.rows_from_device_bytes(rows.cpu().numpy())
    t0 = time.perf_counter()
    host = batch.evaluate(np.array([[0.31, 0.09]]))
    e2e_s = time.perf_counter() - t0
    cpu = None
    if not args.no_cpu_baseline and (ROOT / "oracle" / "_ref" / "libcfdr_ref.so").exists():
        per = plain_cpu_seconds_per_iteration()
        iters = int(rec["iterations"][0])
        cpu = {"value": per * iters, "unit": "s", "cores": 1, "kind": "reference",
               "sample": f"the reference's ForwardModel (oracle/_ref, g++ -O2) capped at 20000 "
                         f"outer iterations: {1e3 * per:.3f} ms each x the {iters} iterations "
                         f"of the solve (extrapolated)"}
    print(json.dumps({
        "metric": PLAIN_METRIC, "value": ms / 1e3, "unit": "s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "Re_tau 182.088 channel, 3 x 128 cells, y+ 0.5, alpha_U 0.5, "
                               "tol 1e-10, (a1, beta*) = (0.31, 0.09)", "max_iter": 150000},
        "status": int(rec["status"][0]), "iterations": int(rec["iterations"][0]),
        "ms_per_outer_iteration": ms / max(int(rec["iterations"][0]), 1),
        "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": 16,
                "d2h_bytes_per_step": 40 + 30 * 8},
        "e2e_status": host.rows[0].result.status.name,
        "gpu_launches": args.steps, "cpu_baseline": cpu,
    }))


# ---------------------------------------------------------------- calibration workload
CAL_METRIC = "calibration study wall time: uniform design, pattern search, Laplace grid, 2 x 64 importance draws"


def calibrate_arm(args):
    import torch
    import rans_uq_b200.calibration as cal
    import rans_uq_b200.workloads as wl

    if int(os.environ.get("RANK", "0")) != 0:
        return
    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    batch, truth = wl.calibration_study_batch()
    setup = time.perf_counter() - t0
    t0 = time.perf_counter()
    trace = {}
    try:
        out = cal.calibrate(cal.batch_evaluator(batch), trace=trace)
    except RuntimeError as e:
        print(json.dumps({"metric": CAL_METRIC, "failed": str(e),
                          "seconds": time.perf_counter() - t0, "trace": trace}))
        return
    wall = time.perf_counter() - t0
    main, rep = out.importance
    sd = np.sqrt(np.diag(out.scale))
    print(json.dumps({
        "metric": CAL_METRIC, "value": wall, "unit": "s", "n_gpus": 1, "steps": 1, "warmup": 0,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "Re_tau 182.088, 3 x 128 cells, 30 stations (likelihood third), "
                               "synthetic observed profile at (0.3137, 0.0912) x (1 + 0.0014 eps)",
                   "alpha_u": 0.5, "tol": 1e-8},
        "solves": out.solves, "truth_setup_s": setup,
        "stages": [{"name": s.name, "solves": s.solves, "seconds": s.seconds} for s in out.stages],
        "search_path_steps": len(out.path) - 1,
        "laplace": {"center": out.center.tolist(), "sd": sd.tolist(),
                    "correlation": float(out.scale[0, 1] / (sd[0] * sd[1])),
                    "fit_residual_rms": out.laplace["residual_rms"]},
        "importance": {k: main[k] for k in ("effective_sample_size", "max_weight",
                                             "distinct_draws", "theta_mean", "theta_sd")},
        "replicate": {k: rep[k] for k in ("effective_sample_size", "theta_mean", "theta_sd")},
        "true_theta": list(wl.CAL_TRUE_THETA),
        "reference_published": "241 solves in about 50 minutes on 4 threads "
                               "(docs/figures/README.md of the reference)",
    }))


def main():
    args = parse()
    if args.workload == "calibrate":
        calibrate_arm(args)
        return
    if args.workload == "plain":
        plain_arm(args)
        return
    if args.workload == "bump":
        bump_arm(args)
        return
    if args.workload == "serve":
        serve_arm(args)
        return
    if args.workload == "linear":
        linear_arm(args)
    elif args.impl == "reference":
        reference_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
