"""Benchmark: histories/s of the transport hot path on the synthetic CT head
5-field plan (C3: 256x256x120 HU volume, 5 coplanar fields through jaws and a
120-leaf MLC, 6 MV-like phase space), one JSON line on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gegs|reference]

A step transports the whole C3 plan, ``--hist-per-step`` histories (2e8) over
all five fields, in one persistent launch; each step takes its own histories
(the plan's field ranges moved along the history index), so no step repeats
another's random numbers.  ``value`` is
the device-timed throughput (CUDA events on the engine stream) with every
input resident in HBM; ``e2e`` repeats the same steps through the C ABI from
host memory: H2D of the phase-space records from pinned memory, the run, and
D2H of the int64 dose tally into pinned memory.  Multi-GPU (torchrun): each
rank transports its own history range (weak scaling); the tallies are summed
with one NCCL all-reduce.
``--impl reference`` times the reference's own stage kernels built as host
code (``oracle/_ref``, one process per host core) on the C3 plan, or the CPU
restatement of them (the oracle) where that build is absent.
"""
from __future__ import annotations

import argparse
import json
import os
import pathlib
import re
import subprocess
import sys
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

MEASURED = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0
METRIC = "histories/s (CT head 5-field plan, C3)"


def hbm_peak():
    try:
        d = json.loads(MEASURED.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks + throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.device), "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def traffic_from_profile(kind):
    """DRAM bytes per transport step of the photon or electron kernels, from the
    committed ncu summary ``profiles/transport_kernels_c3.md`` (three bulk waves
    of the bench's step in the timed form, DRAM read + write over their steps)."""
    p = ROOT / "profiles" / "transport_kernels_c3.md"
    if not p.exists():
        return None
    m = re.search(rf"{kind}_dram_bytes_per_step:\s*([0-9.eE+-]+)", p.read_text())
    return float(m.group(1)) if m else None


def algorithmic_bytes(job, sample):
    """Per-history algorithmic bytes by stage, counted by the oracle on `sample` histories:
    16 B per region record read, 16 B per tally update (8 B read + 8 B write),
    8 B per float2 table read, 28 B per phase-space record (photon stage)."""
    from oracle import oracle as O
    sh = job.scene()
    _, st = O.run(job.physics, sh, 0, sample)
    cnt = np.array(st["cnt"], np.float64)
    per_stage = (16 * cnt[:, 0] + 16 * cnt[:, 1] + 8 * cnt[:, 2]) / sample
    per_stage[0] += 28.0
    return per_stage, st


def cpu_histories_per_s(job, seconds=15.0, threads=None):
    """Oracle throughput on the host cores over a bounded sample (~`seconds`):
    a warm-up run (thread pool, first touches), then samples growing 4x until
    one takes a second, then one run sized to `seconds`."""
    from oracle import oracle as O
    threads = threads or os.cpu_count()
    sh = job.scene()
    n = 2000
    O.run(job.physics, sh, 0, n, threads=threads, native=True)
    while True:
        t = time.perf_counter()
        O.run(job.physics, sh, 0, n, threads=threads, native=True)
        dt = time.perf_counter() - t
        if dt >= min(1.0, seconds / 4) or n >= 1_000_000:
            break
        n *= 4
    n2 = int(min(4_000_000, n * seconds / max(dt, 1e-3)))
    if n2 > n:
        t = time.perf_counter()
        O.run(job.physics, sh, 0, n2, threads=threads, native=True)
        dt = time.perf_counter() - t
        n = n2
    return n / dt, n, dt, threads


def c4_gradient(args, eng):
    """C4 (CT head, 5 fields x 20 x 20 beamlets of 5 mm): time of one forward and of
    the replay backward, the cost of finite differences over every beamlet, and a
    common-random-number finite-difference check on 16 random beamlets."""
    import torch

    from gegs_b200 import workloads as W
    from gegs_b200.differentiable import BeamletModel, beamlet_dose, fd_gradient, objective
    job = W.config4(histories=args.c4_histories, nphsp=args.nphsp)
    eng.set_physics(job.physics)
    eng.set_scene(job.scene())
    target, organ = job.meta["target"], job.meta["organ"]
    loss = lambda d: objective(d, target, organ)
    w0 = job.beam["beamlets"]["weights"].astype(np.float64)
    model = BeamletModel(eng, job)
    model.calibrate(w0, target, 50.0)
    fwd, bwd = [], []
    for _ in range(2):
        w = torch.tensor(w0, requires_grad=True)
        L = loss(beamlet_dose(w, model))
        fwd.append(model.forward_ms)
        L.backward()
        bwd.append(model.backward_ms)
    g_full = w.grad.numpy()
    small = BeamletModel(eng, job, 0, args.c4_fd_histories, dose_unit=model.unit)
    w = torch.tensor(w0, requires_grad=True)
    loss(beamlet_dose(w, small)).backward()
    g = w.grad.numpy()
    # 16 random beamlets among those that receive histories (g != 0), as C4 states
    live = np.flatnonzero(g != 0)
    pick = np.sort(np.random.default_rng(16).choice(live, size=min(16, live.size), replace=False))
    # 20 projected gradient-descent iterations (forward + replay backward each) on the small model
    from gegs_b200.differentiable import optimize_weights
    import time as _t
    t0 = _t.perf_counter()
    _, hist = optimize_weights(small, w0, target, organ, iterations=args.c4_iterations)
    descent = {"iterations": args.c4_iterations, "histories_per_iteration": args.c4_fd_histories,
               "objective_first": hist[0], "objective_last": hist[-1], "wall_s": _t.perf_counter() - t0}
    fd = fd_gradient(small, w0, pick, loss, delta=0.05)
    f_ms, b_ms = min(fwd), min(bwd)
    return {"workload": f"C4 CT head 256x256x120, 5 fields x 20x20 beamlets of 5 mm, {job.histories} histories",
            "beamlets": int(model.nb), "forward_ms": f_ms, "backward_ms": b_ms, "backward_over_forward": b_ms / f_ms,
            "gradient_ms": f_ms + b_ms, "fd_all_beamlets_ms": 2 * model.nb * f_ms,
            "fd_over_gradient": 2 * model.nb * f_ms / (f_ms + b_ms),
            "fd_check": {"histories": args.c4_fd_histories, "beamlets": [int(b) for b in pick],
                         "replay": [float(x) for x in g[pick]], "fd": [float(x) for x in fd],
                         "max_rel_err": float(np.max(np.abs(g[pick] - fd) / np.abs(fd).max())),
                         "max_rel_err_each": float(np.max(np.abs(g[pick] - fd) / np.maximum(np.abs(fd), 1e-300)))},
            "grad_norm": float(np.linalg.norm(g_full)),
            "descent": descent}


def c5_batch(args, device):
    """C5 serving-style batch at its stated configuration: 32 independent plans
    (slab and CT head, 64^3 to 256x256x128 voxels, 1-7 fields, histories
    log-uniform in 1e6..1e8), one engine per plan. Timed (host wall clock from
    the first launch to the last wait) with the default run options: all plans
    in one graph launch (a branch per plan), all plans launched one per stream,
    and one plan after another; then in one graph launch with options from the
    autotuner (coordinate descent over in-flight batch, grid, step budgets,
    refill threshold, table staging and wave order, timed on a sample of each
    plan's histories before the timed run)."""
    from gegs_b200 import workloads as W
    from gegs_b200.batch import PlanBatch
    jobs = W.config5(n_plans=args.c5_plans, hist_min=args.c5_hist_min, hist_max=args.c5_hist_max,
                     nphsp=1_000_000)
    total = sum(j.histories for j in jobs)
    from gegs_b200.engine import launch_group
    pb = PlanBatch(jobs, device=device, memory_budget_gb=40.0)
    pb.run([max(1, j.histories // 100) for j in jobs])            # warm-up: graphs and queues
    pb.run([max(1, j.histories // 100) for j in jobs], one_launch=False)
    t = time.perf_counter()
    for e, j, o in zip(pb.engines, pb.jobs, pb.options):          # host cost of one launch per plan
        e.launch(0, 1, **o)
    launch_ms = (time.perf_counter() - t) * 1e3
    for e in pb.engines:
        e.wait()
    t = time.perf_counter()
    launch_group(pb.engines, [(0, 1)] * len(jobs), pb.options)    # host cost of the one group launch
    group_launch_ms = (time.perf_counter() - t) * 1e3
    for e in pb.engines:
        e.wait()
    pb.run()                                                       # all plans in one graph launch
    conc = pb.wall_s
    pb.run(one_launch=False)                                       # one launch per plan, one stream each
    conc_streams = pb.wall_s
    pb.run_sequential()
    seq = pb.wall_s
    pb.close()
    t = time.perf_counter()
    pt = PlanBatch(jobs, device=device, memory_budget_gb=40.0, tune_fraction=args.c5_tune_fraction)
    tune_s = time.perf_counter() - t
    pt.run([max(1, j.histories // 100) for j in jobs])
    pt.run()
    tuned = pt.wall_s
    tuned_opts = pt.options
    pt.close()
    dims = [tuple(len(j.phantom[k]) - 1 for k in ("x_bounds", "y_bounds", "z_bounds")) for j in jobs]
    out = {"workload": f"C5: {len(jobs)} plans (slab and CT head, {min(min(d) for d in dims)}^3.."
                       f"{'x'.join(map(str, max(dims, key=lambda d: d[0] * d[1] * d[2])))} voxels, 1-7 fields), "
                       f"histories log-uniform {args.c5_hist_min:.0e}..{args.c5_hist_max:.0e}",
           "histories": total, "concurrent_s": conc, "sequential_s": seq,
           "concurrent_histories_per_s": total / conc, "sequential_histories_per_s": total / seq,
           "concurrent": "all plans as one CUDA graph (one branch per plan), one launch (gegs_launch_group)",
           "concurrent_streams_s": conc_streams,
           "group_launch_ms": group_launch_ms, "launch_ms_all_plans": launch_ms,
           "autotuned": {"concurrent_s": tuned, "concurrent_histories_per_s": total / tuned, "tuning_s": tune_s,
                         "options": [{k: int(v) for k, v in o.items()} for o in tuned_opts]},
           "timing": "host wall clock from the first launch to the last wait"}
    if args.c5_descent_iterations > 0:
        out["descent"] = c5_descent(args, device)
    return out


def c5_descent(args, device):
    """Gradient descent on the beamlet weights of 4 plans at once (CT heads of
    four sizes, 5 fields x 20 x 20 beamlets): every iteration runs the four
    forward transports concurrently, then each plan's replay backward."""
    from gegs_b200 import workloads as W
    from gegs_b200.differentiable import BeamletModel, optimize_weights_batch
    from gegs_b200.engine import Engine
    dims = [(64, 64, 48), (96, 96, 64), (128, 128, 96), (256, 256, 120)]
    h = args.c5_descent_histories
    models, engines, w0s, targets, organs = [], [], [], [], []
    for k, d in enumerate(dims):
        job = W.config4(histories=h, nphsp=1_000_000, dims=d, seed=W.SEED_BASE + 40 + k)
        e = Engine(device)
        e.set_physics(job.physics)
        e.set_scene(job.scene())
        m = BeamletModel(e, job, batch=1 << 20)
        w0 = job.beam["beamlets"]["weights"].astype(np.float64)
        m.calibrate(w0, job.meta["target"], 50.0)
        models.append(m); engines.append(e); w0s.append(w0)
        targets.append(job.meta["target"]); organs.append(job.meta["organ"])
    t0 = time.perf_counter()
    _, hist = optimize_weights_batch(models, w0s, targets, organs, iterations=args.c5_descent_iterations)
    wall = time.perf_counter() - t0
    for e in engines:
        e.close()
    return {"plans": [f"CT head {d[0]}x{d[1]}x{d[2]}, 5 fields x 20x20 beamlets" for d in dims],
            "iterations": args.c5_descent_iterations, "histories_per_iteration": h, "wall_s": wall,
            "objective_first": [x[0] for x in hist], "objective_last": [x[-1] for x in hist]}


def sigma_series(eng, job, args, ropt, rate):
    """Time to 1 % statistical uncertainty on the plan, from two independent
    series of batches (the first and the second half of every field's
    histories). Each batch holds an equal share of every field's histories;
    the device folds each batch's energy into per-voxel sums (gegs_stat_*) and
    returns the relative standard error of the mean with the reference's batch
    formula (CUDA_EGS.cu:817-876). sigma = the mean relative SE over body voxels
    (density >= 0.1 g/cm3) whose dose exceeds 50 % of a robust maximum, the
    99.9th percentile of body-voxel dose. sigma^2 N is constant, so
    t(1 %) = N (sigma / 0.01)^2 / rate with the measured device throughput."""
    M = args.sigma_batches
    mass = job.voxel_mass()
    body = job.phantom["density"].reshape(-1) >= 0.1
    series = []
    for half in (0, 1):
        eng.reset_tally()
        eng.stat_begin()
        n_hist = 0
        for b in range(M):
            for f in job.fields:
                h0, h1 = int(f["hist_begin"]), int(f["hist_end"])
                mid = h0 + (h1 - h0) // 2
                lo_f, hi_f = (h0, mid) if half == 0 else (mid, h1)
                lo = lo_f + (hi_f - lo_f) * b // M
                hi = lo_f + (hi_f - lo_f) * (b + 1) // M
                if hi > lo:
                    eng.run(lo, hi, **ropt)
                    n_hist += hi - lo
            eng.stat_fold()
        mean, rel, nb = eng.stat_get()
        dose = mean / mass
        dmax = float(np.percentile(dose[body], 99.9))
        sel = body & (dose > 0.5 * dmax)
        sig = float(np.mean(rel[sel]))
        series.append({"histories": n_hist, "batches": nb, "voxels": int(sel.sum()), "mean_rel_se": sig,
                       "time_to_1pct_s": n_hist * (sig / 0.01) ** 2 / rate})
    t = [x["time_to_1pct_s"] for x in series]
    return {"estimator": f"batch method, {M} batches per series, the reference's formula "
                         "sqrt((S2/n - (S1/n)^2)/(n-1)) / (S1/n) (CUDA_EGS.cu:817-876), folded on the device",
            "voxels": "density >= 0.1 g/cm3 and batch-mean dose > 50 % of the 99.9th percentile of body-voxel dose",
            "series": series, "time_to_1pct_s": float(np.mean(t)),
            "series_ratio": max(t) / min(t),
            "mean_rel_se_at_2e8": float(np.mean([x["mean_rel_se"] * np.sqrt(x["histories"] / 2e8) for x in series]))}


def c3_config(job, hist_per_step):
    """The workload both arms report in `config`: the C3 plan and the histories of one step."""
    return {"workload": "C3 synthetic CT head 256x256x120 (1x1x2.5 mm), 5 coplanar fields 0/72/144/216/288 deg, "
                        "jaws +-6 cm, 120-leaf MLC with seeded tips, 6 MV-like phase space "
                        f"({len(job.phsp)} records, recycled)",
            "hist_per_step": hist_per_step,
            "l2": "working set (63 MB region table + 63 MB int64 tally + event queues) exceeds the 126 MB L2; no flush"}


def make_job(args, histories):
    from gegs_b200 import workloads as W
    return W.config3(histories=histories, nphsp=args.nphsp)


_REF_JOB = None
_REF_SCENE = None
_REF_PAIR = None


def _ref_worker(rng):
    """One process of the reference arm: histories [h0, h1) of the plan by the
    reference's own kernels (forked from the parent, which holds the plan)."""
    from oracle import refpin as R
    global _REF_PAIR
    h0, h1, seed = rng
    if _REF_PAIR is None:                         # once per process: the reference's globals from the plan
        _REF_PAIR = R.Pair(_REF_JOB.physics, _REF_SCENE)
    pair = _REF_PAIR
    t = time.perf_counter()
    e = pair.transport(h0, h1, seed=seed)
    return time.perf_counter() - t, float(e.sum())


def run_reference_transport(args, job):
    """The reference arm on the reference's own code: whole transports by its
    ten stage kernels compiled as host code (oracle/_ref, ref_transport), one
    process per host core, each on its own share of the step's histories.
    Forked before anything touches CUDA. Returns the JSON line's fields."""
    import multiprocessing as mp
    global _REF_JOB, _REF_SCENE
    _REF_JOB, _REF_SCENE = job, job.scene()
    procs = os.cpu_count() or 1
    ctx = mp.get_context("fork")
    with ctx.Pool(procs) as pool:
        # calibrate: a short run on every process, then size a step to about ref_seconds
        per = 2000
        dts = pool.map(_ref_worker, [(k * per, (k + 1) * per, 9000 + k) for k in range(procs)])
        rate1 = per / max(np.median([d for d, _ in dts]), 1e-6)
        per = max(2000, int(rate1 * args.ref_seconds))
        step_hist = per * procs
        per_step_ms = []
        for s in range(args.warmup + args.steps):
            base = (1 + s) * step_hist
            t = time.perf_counter()
            pool.map(_ref_worker, [(base + k * per, base + (k + 1) * per, 100 * s + k) for k in range(procs)])
            if s >= args.warmup:
                per_step_ms.append((time.perf_counter() - t) * 1e3)
    value = step_hist * args.steps / (sum(per_step_ms) / 1e3)
    return value, per_step_ms, step_hist, procs


def run_reference(args):
    """The reference arm: the reference's own kernels on all host cores when its
    sources compiled here (oracle/_ref), else the CPU restatement (the oracle)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    from oracle import refpin as R
    O.build()
    R.build()
    job = make_job(args, 200_000_000)
    if R.available():
        value, per_step_ms, steps_hist, cores = run_reference_transport(args, job)
        line = {
            "impl": "reference", "metric": METRIC, "value": value, "unit": "histories/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(per_step_ms)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": c3_config(job, args.hist_per_step), "parallelism": f"{cores} host processes",
            "sample_histories_per_step": steps_hist,
            "cpu_baseline": {"value": value, "unit": "histories/s", "cores": cores, "kind": "reference",
                             "sample": f"{steps_hist} C3 histories per step (a bounded sample of the "
                                       f"{args.hist_per_step}-history step) on {cores} processes: the reference's ten "
                                       "stage kernels and geometry compiled from its sources as host code "
                                       "(oracle/_ref, g++ -O2), draining their stacks, one process per core"},
            "e2e": {"value": value, "unit": "histories/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))
        return
    rate, n, dt, cores = cpu_histories_per_s(job, seconds=args.ref_seconds)
    per_step_ms = []
    sh = job.scene()
    steps_hist = n
    for s in range(args.warmup + args.steps):
        t = time.perf_counter()
        O.run(job.physics, sh, s * steps_hist, (s + 1) * steps_hist, threads=cores, native=True)
        if s >= args.warmup:
            per_step_ms.append((time.perf_counter() - t) * 1e3)
    value = steps_hist * args.steps / (sum(per_step_ms) / 1e3)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "histories/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(per_step_ms)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": c3_config(job, args.hist_per_step), "parallelism": f"{cores} host threads",
        "sample_histories_per_step": steps_hist,
        "cpu_baseline": {"value": value, "unit": "histories/s", "cores": cores, "kind": "port",
                         "sample": f"{steps_hist} C3 histories per step (a bounded sample of the "
                                   f"{args.hist_per_step}-history step) on {cores} threads (CPU restatement of the "
                                   f"reference routines, used where the reference's own kernels were not built)"},
        "e2e": {"value": value, "unit": "histories/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gegs", choices=["gegs", "reference"])
    ap.add_argument("--hist-per-step", type=int, default=200_000_000,
                    help="histories of the plan that one step transports, over all five fields in one launch")
    ap.add_argument("--nphsp", type=int, default=10_000_000)
    ap.add_argument("--batch", type=int, default=0)
    ap.add_argument("--mode", default="persistent", choices=["persistent", "plain", "timed"],
                    help="timed: the persistent form's kernels launched wave by wave from the host "
                         "(per-kernel events; for ncu launch lists, which cannot see into the graph)")
    ap.add_argument("--photon-budget", type=int, default=0)
    ap.add_argument("--electron-budget", type=int, default=0)
    ap.add_argument("--ref-seconds", type=float, default=8.0)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--roofline-histories", type=int, default=10_000_000,
                    help="histories of the timed-form run that times each transport kernel for the roofline")
    ap.add_argument("--plain-histories", type=int, default=10_000_000,
                    help="histories of the plain-form comparison (0: skip)")
    ap.add_argument("--c4-histories", type=int, default=50_000_000,
                    help="forward/backward histories of the C4 gradient measurement (0: skip)")
    ap.add_argument("--c4-fd-histories", type=int, default=5_000_000)
    ap.add_argument("--c4-iterations", type=int, default=20)
    ap.add_argument("--sigma-batches", type=int, default=40,
                    help="batches per series of the time-to-1 %% estimate (0: skip)")
    ap.add_argument("--c5-plans", type=int, default=32, help="plans of the batched sweep (0: skip)")
    ap.add_argument("--c5-hist-min", type=int, default=1_000_000)
    ap.add_argument("--c5-hist-max", type=int, default=100_000_000)
    ap.add_argument("--c5-tune-fraction", type=float, default=0.02)
    ap.add_argument("--c5-descent-iterations", type=int, default=20,
                    help="gradient-descent iterations on 4 plans at once (0: skip)")
    ap.add_argument("--c5-descent-histories", type=int, default=1_000_000)
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    from gegs_b200 import build as B
    B.build()
    from gegs_b200.engine import MODE_PERSISTENT, MODE_PLAIN, MODE_TIMED, Engine

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    H = args.hist_per_step
    job = make_job(args, H)                       # the plan: five fields of H/5 histories
    sh = job.scene()
    mode = {"persistent": MODE_PERSISTENT, "plain": MODE_PLAIN, "timed": MODE_TIMED}[args.mode]
    ropt = dict(mode=mode, batch=args.batch, photon_budget=args.photon_budget, electron_budget=args.electron_budget)
    eng = Engine(local)
    eng.set_physics(job.physics)
    eng.set_scene(sh)

    def hist_range(step):
        """Histories [base, base + H) of a step, with the plan's fields moved
        there (gegs_set_field: history ranges only; the phantom stays)."""
        base = (rank * (args.warmup + args.steps) + step) * H
        for i, f in enumerate(job.fields):
            eng.set_field(i, dict(f, hist_begin=f["hist_begin"] + base, hist_end=f["hist_end"] + base))
        return base, base + H

    for s in range(args.warmup):
        eng.run(*hist_range(s), **ropt)
    eng.reset_tally()

    if dist is not None:
        import torch
        dist.barrier()
        torch.cuda.synchronize()
    dev_ms = []
    stats = []
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        for s in range(args.warmup, args.warmup + args.steps):
            h0, h1 = hist_range(s)
            st = eng.run(h0, h1, **ropt)
            dev_ms.append(st["device_ms"])
            stats.append(st)
        if dist is not None:
            import torch

            from gegs_b200.sharding import allreduce_tally_, tally_tensor
            allreduce_tally_(tally_tensor(eng, f"cuda:{local}"))
            torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    elapsed_s = sum(dev_ms) / 1e3
    if dist is not None:
        import torch
        tt = torch.tensor([elapsed_s, wall], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        elapsed_s, wall = float(tt[0]), float(tt[1])
    value = H * args.steps * world / elapsed_s

    # ---- end to end through the C ABI from host buffers -------------------
    # The same steps as the device-timed ones (same histories, same phase-space
    # records, so the same transport work), each preceded by the upload of the
    # whole phase space from pinned host memory and followed by the read of the
    # tally into pinned host memory, both inside the timed region.
    rec_per_step = len(job.phsp)
    e2e_ms = []
    try:
        import torch
        pinned = torch.empty((rec_per_step * 28,), dtype=torch.uint8).pin_memory().numpy()
    except Exception:
        pinned = np.empty(rec_per_step * 28, np.uint8)
    from gegs_b200.scene import PHSP_DTYPE
    chunk = pinned.view(PHSP_DTYPE)
    try:
        host_tally = torch.empty((eng.nvox,), dtype=torch.int64).pin_memory().numpy()
    except Exception:
        host_tally = np.empty(eng.nvox, np.int64)
    for s in range(args.steps):
        chunk[:] = job.phsp
        t = time.perf_counter()
        eng.set_phsp(chunk)
        h0, h1 = hist_range(args.warmup + s)
        eng.run(h0, h1, **ropt)
        eng.tally(out=host_tally)
        e2e_ms.append((time.perf_counter() - t) * 1e3)
    e2e = H * args.steps * world / (sum(e2e_ms) / 1e3)
    if dist is not None:
        import torch
        tt = torch.tensor([sum(e2e_ms)], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e = H * args.steps * world / (float(tt[0]) / 1e3)

    # Every rank leaves the process group here, so that no rank waits on a
    # collective while rank 0 alone measures the rest (at N > 1 only the
    # roofline; the CPU baseline, sigma, plain form, C4 and C5 at N = 1).
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    extras = world == 1

    # ---- roofline of the dominant kernel (timed mode, outside the timed region)
    eng.set_phsp(job.phsp)
    for i, f in enumerate(job.fields):                  # the plan's own history ranges again
        eng.set_field(i, f)
    RH = args.roofline_histories                       # the timed form over the first histories of the plan
    tst = eng.run(0, RH, **dict(ropt, mode=MODE_TIMED))
    kinds = ["photon", "compton", "photo", "rayleigh", "pair", "electron", "moller", "brems", "bhabha", "annih",
             "source", "planner", "photon_jaws", "electron_jaws", "photon_mlc", "electron_mlc"]
    ms = np.array(tst["stage_ms"][:16])
    # a transport stage runs as three launches per wave (jaws, MLC and phantom kernels)
    groups = {k: [i] for i, k in enumerate(kinds[:10])}
    groups["photon"] = [0, 12, 14]
    groups["electron"] = [5, 13, 15]
    stage_ms = {k: float(ms[idx].sum()) for k, idx in groups.items()}
    dom_name = max(stage_ms, key=stage_ms.get)
    dom = kinds.index(dom_name)
    launches = max(1, tst["stage_launches"][dom])              # waves that ran this stage
    per_stage_bytes, ost = algorithmic_bytes(job, sample=20000)
    alg_bytes_per_launch = per_stage_bytes[dom] * RH / launches
    avg_launch_s = stage_ms[dom_name] / 1e3 / launches
    peak, peak_kind = hbm_peak()
    achieved = alg_bytes_per_launch / avg_launch_s / 1e9
    steps_key = {"photon": "photon_steps", "electron": "electron_steps"}.get(dom_name)
    per_step = traffic_from_profile(dom_name)
    tr = per_step * tst[steps_key] / launches if (per_step is not None and steps_key) else None
    total_ms = float(ms[[i for i in range(16) if i != 11]].sum())
    share = {k: float(ms[i] / total_ms) for i, k in enumerate(kinds) if i != 11}

    # ---- statistical uncertainty -> time to 1 % (outside the timed region) --
    sigma = sigma_series(eng, job, args, ropt, value) if extras and args.sigma_batches >= 2 else None

    # ---- the plain form at the reference's launch shape, same histories ------
    plain = None
    if extras and args.plain_histories > 0:
        hp = args.plain_histories
        pst = eng.run(0, hp, mode=MODE_PLAIN, batch=480_000, blocks_per_sm=5, threads=128)
        qst = eng.run(0, hp, **dict(ropt, mode=MODE_PERSISTENT))
        plain = {"histories": hp, "launch": "5 blocks/SM x 128 threads, 480000 histories per batch, host sync + "
                                            "counter read-back after every kernel (CUDA_EGS.cu:226-365, 498-799)",
                 "value": hp / pst["device_ms"] * 1e3, "persistent_value": hp / qst["device_ms"] * 1e3,
                 "persistent_over_plain": pst["device_ms"] / qst["device_ms"],
                 "plan_over_plain": value / (hp / pst["device_ms"] * 1e3),
                 "note": "both forms give the same tally bit for bit, so equal histories give equal sigma "
                         "and gamma; a ratio of rates is the time-to-1% ratio. persistent_over_plain: the same "
                         "10M histories; plan_over_plain: the bench's steps (the whole plan per launch)"}
        if sigma:
            n1 = sigma["time_to_1pct_s"] * value            # histories to 1 % (sigma^2 N is constant)
            plain["histories_to_1pct"] = n1
            plain["time_to_1pct_s"] = n1 / plain["value"]

    # ---- C4: beamlet gradient by replay vs forward and finite differences ---
    grad = c4_gradient(args, eng) if extras and args.c4_histories > 0 else None
    nvox = eng.nvox
    eng.close()                                    # its event queues (up to ~120 GB) before the C5 engines
    batched = c5_batch(args, local) if extras and args.c5_plans > 0 else None

    cpu = None
    if extras and not args.no_cpu:
        crate, cn, cdt, cores = cpu_histories_per_s(job, seconds=args.cpu_seconds)
        r1, n1, dt1, _ = cpu_histories_per_s(job, seconds=3.0, threads=1)
        cpu = {"value": crate, "unit": "histories/s", "cores": cores, "kind": "port",
               "sample": f"{cn} C3 histories in {cdt:.1f} s on {cores} host threads (CPU oracle, same inputs)",
               "value_1_core": r1, "sample_1_core": f"{n1} C3 histories in {dt1:.1f} s on 1 thread"}
    # per step: the first planner launch, then per wave the kernels of one wave and the planner.
    # Plain form: source + 10 stage kernels + planner. Timed form: source, photon jaws / MLC /
    # phantom, 4 photon interactions, electron jaws + near pass, MLC + near pass, phantom, 4
    # electron interactions, planner. Persistent form: the same plus the long jaws-photon kernel.
    per_wave = {"plain": 12, "timed": 18}.get(args.mode, 19)
    launches_per_step = [1 + per_wave * (st["waves"] - 1) for st in stats]
    line = {
        "metric": METRIC, "value": value, "unit": "histories/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": elapsed_s * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": c3_config(job, H), "mode": args.mode, "parallelism": f"histories sharded over {world} GPU(s)",
        "e2e": {"value": e2e, "unit": "histories/s", "h2d_bytes_per_step": rec_per_step * 28,
                "d2h_bytes_per_step": nvox * 8},
        "roofline": {"bound": "hbm", "kernel": f"{dom_name} transport (k_{dom_name}_jaws + k_{dom_name}_mlc + k_{dom_name}, one wave)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "traffic": tr,
                     "alg_bytes_per_launch": alg_bytes_per_launch, "avg_launch_ms": avg_launch_s * 1e3,
                     "kernel_share": share},
        "cpu_baseline": cpu,
        "gpu_launches": int(sum(launches_per_step)),
        "clocks": clk.summary(),
        "plain_form": plain,
        "gradient": grad,
        "batched_plans": batched,
        "stat_uncertainty": sigma,
        "device_stats": {"processed": stats[-1]["processed"], "photon_steps": stats[-1]["photon_steps"],
                         "electron_steps": stats[-1]["electron_steps"], "waves": stats[-1]["waves"]},
        "wall_s": wall,
    }
    print(json.dumps(line))


if __name__ == "__main__":
    main()
