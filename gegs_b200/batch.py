"""Many plans at once on one GPU (serving-style batches, the C5 sweep).

Each plan gets its own engine: its own phantom, tables, tally, event queues,
stream and persistent CUDA graph. ``PlanBatch.run`` launches every plan's
graph (``gegs_launch``) before waiting for any (``gegs_wait``), so the plans'
waves run concurrently on the device and small plans fill the GPU together;
each plan's tally is the same bit for bit as when it runs alone.

Run options per plan come from ``choose_options`` (in-flight batch sized from
the plan's histories within a shared memory budget; step budgets and refill
threshold of the single-plan defaults) or from ``autotune``, which times a few
candidate settings on a sample of the plan's histories and keeps the fastest.
"""
from __future__ import annotations

import time

import numpy as np

from .engine import Engine, launch_group

QUEUE_BYTES_PER_PARTICLE = 5.2e3      # event queues + electron step state per particle of `batch`


def choose_options(histories, share_bytes):
    """In-flight batch: a power of two near a quarter of the histories, at most
    what `share_bytes` of queue memory holds, between 64K and 4M."""
    want = max(1 << 16, min(1 << 22, 1 << int(np.ceil(np.log2(max(histories, 1) / 4)))))
    cap = 1 << int(np.floor(np.log2(max(share_bytes / QUEUE_BYTES_PER_PARTICLE, 1 << 16))))
    b = int(min(want, cap))
    return dict(batch=b, photon_budget=32, electron_budget=8, refill_below=b // 4)


# The autotuner's search space: each dimension's alternatives to the current
# setting (coordinate descent from the defaults of choose_options).
TUNE_DIMENSIONS = {
    "batch": lambda o: [max(o["batch"] // 2, 1 << 16), min(o["batch"] * 2, 1 << 22)],
    "blocks_per_sm": lambda o: [4, 8],
    "photon_budget": lambda o: [16, 64],
    "electron_budget": lambda o: [4, 16],
    "refill_below": lambda o: [max(o["batch"] // 50, 1), max(o["batch"] // 2, 1)],
    "stage_tables": lambda o: [not o.get("stage_tables", False)],
    "pipelined": lambda o: [not o.get("pipelined", True)],
}


def autotune(engine, job, sample=None, candidates=None, dimensions=None, rounds=1, start=None):
    """The fastest run options for `job`, timed on `sample` histories.

    With `candidates`, each is timed and the fastest kept. Otherwise a
    coordinate descent: starting from choose_options, each dimension of
    TUNE_DIMENSIONS (in-flight batch, grid blocks per SM, photon and electron
    step budgets, refill threshold, whether the photon tables are staged in
    shared memory, GEGS_RUN_STAGE_TABLES, and whether a wave's two transport
    phases run at once, GEGS_RUN_SERIAL_WAVES) tries its alternatives with the
    others fixed and keeps any that is faster; `rounds` passes over the
    dimensions.
    Every trial first runs a quarter sample untimed (graph build, queue
    sizing), then the timed sample; the tally is reset afterwards. `start`
    replaces choose_options' defaults (a batch within a memory share). Returns
    (options, device ms of the sample, trials as a list of (options, ms))."""
    h = job.histories if sample is None else min(sample, job.histories)
    trials = []

    def timed(o):
        engine.run(0, max(h // 4, 1), **o)
        t = engine.run(0, h, **o)["device_ms"]
        trials.append((dict(o), t))
        return t

    if candidates is not None:
        best, best_t = None, float("inf")
        for c in candidates:
            t = timed(c)
            if t < best_t:
                best, best_t = c, t
        engine.reset_tally()
        return best, best_t, trials
    best = dict(start) if start is not None else choose_options(job.histories, 64e9)
    best.setdefault("blocks_per_sm", 0)
    best_t = timed(best)
    for _ in range(rounds):
        for dim, alts in (dimensions or TUNE_DIMENSIONS).items():
            for v in alts(best):
                if v == best.get(dim):
                    continue
                cand = dict(best, **{dim: v})
                if dim == "batch":
                    cand["refill_below"] = max(v // 4, 1)
                t = timed(cand)
                if t < best_t:
                    best, best_t = cand, t
    engine.reset_tally()
    return best, best_t, trials


class PlanBatch:
    def __init__(self, jobs, device=0, memory_budget_gb=40.0, tune_sample=0, tune_fraction=0.0):
        """One engine per plan. With tune_sample (histories) or tune_fraction
        (of each plan's histories, at least 1e5), each plan's run options come
        from the coordinate-descent autotuner, kept within the plan's share of
        the queue-memory budget."""
        self.jobs = list(jobs)
        self.engines, self.options, self.tune_ms = [], [], []
        total = float(sum(j.histories for j in self.jobs)) or 1.0
        for job in self.jobs:
            e = Engine(device)
            e.set_physics(job.physics)
            e.set_scene(job.scene())
            share = memory_budget_gb * 1e9 * job.histories / total
            opts = choose_options(job.histories, share)
            sample = tune_sample or (int(max(1e5, tune_fraction * job.histories)) if tune_fraction > 0 else 0)
            if sample:
                cap = 1 << int(np.floor(np.log2(max(share / QUEUE_BYTES_PER_PARTICLE, 1 << 16))))  # what the share holds
                dims = dict(TUNE_DIMENSIONS)
                dims["batch"] = lambda o: [b for b in (max(o["batch"] // 2, 1 << 16), o["batch"] * 2) if b <= cap]
                opts, t, _ = autotune(e, job, sample=sample, dimensions=dims, start=opts)
                self.tune_ms.append(t)
            self.engines.append(e)
            self.options.append(opts)
        self.wall_s = 0.0

    def run(self, histories=None, one_launch=True):
        """Transport every plan's histories (or the first `histories[i]` of plan i)
        concurrently: with one_launch, as one graph with a branch per plan
        (gegs_launch_group); otherwise one launch per plan, each on its engine's stream."""
        t = time.perf_counter()
        ranges = [(0, j.histories if histories is None else histories[i]) for i, j in enumerate(self.jobs)]
        for e in self.engines:
            e.reset_tally()
        if one_launch:
            launch_group(self.engines, ranges, self.options)
        else:
            for e, r, o in zip(self.engines, ranges, self.options):
                e.launch(r[0], r[1], **o)
        stats = [e.wait() for e in self.engines]
        self.wall_s = time.perf_counter() - t
        return stats

    def run_sequential(self, histories=None):
        t = time.perf_counter()
        stats = []
        for i, (e, j, o) in enumerate(zip(self.engines, self.jobs, self.options)):
            e.reset_tally()
            stats.append(e.run(0, j.histories if histories is None else histories[i], **o))
        self.wall_s = time.perf_counter() - t
        return stats

    def tallies(self):
        return [e.tally() for e in self.engines]

    def close(self):
        for e in self.engines:
            e.close()
        self.engines = []
