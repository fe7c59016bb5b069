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

from .engine import Engine

QUEUE_BYTES_PER_PARTICLE = 5.2e3      # event queues + electron step state per particle of `batch`


def choose_options(histories, share_bytes):
    """In-flight batch: a power of two near a quarter of the histories, at most
    what `share_bytes` of queue memory holds, between 64K and 4M."""
    want = max(1 << 16, min(1 << 22, 1 << int(np.ceil(np.log2(max(histories, 1) / 4)))))
    cap = 1 << int(np.floor(np.log2(max(share_bytes / QUEUE_BYTES_PER_PARTICLE, 1 << 16))))
    b = int(min(want, cap))
    return dict(batch=b, photon_budget=32, electron_budget=8, refill_below=b // 4)


def autotune(engine, job, sample=None, candidates=None):
    """Time candidate settings on `sample` histories of the job; return the fastest."""
    h = job.histories if sample is None else min(sample, job.histories)
    base = choose_options(job.histories, 64e9)
    if candidates is None:
        b = base["batch"]
        candidates = [dict(base), dict(base, batch=max(b // 2, 1 << 16), refill_below=max(b // 8, 1)),
                      dict(base, photon_budget=16), dict(base, refill_below=max(b // 50, 1))]
    best, best_t = None, float("inf")
    for c in candidates:
        engine.run(0, max(h // 4, 1), **c)                  # warm: builds the graph, sizes the queues
        t = engine.run(0, h, **c)["device_ms"]
        if t < best_t:
            best, best_t = c, t
    engine.reset_tally()
    return best, best_t


class PlanBatch:
    def __init__(self, jobs, device=0, memory_budget_gb=40.0, tune_sample=0):
        self.jobs = list(jobs)
        self.engines, self.options = [], []
        total = float(sum(j.histories for j in self.jobs)) or 1.0
        for job in self.jobs:
            e = Engine(device)
            e.set_physics(job.physics)
            e.set_scene(job.scene())
            share = memory_budget_gb * 1e9 * job.histories / total
            opts = choose_options(job.histories, share)
            if tune_sample:
                opts, _ = autotune(e, job, sample=tune_sample,
                                   candidates=[opts, dict(opts, photon_budget=16),
                                               dict(opts, refill_below=max(opts["batch"] // 50, 1))])
            self.engines.append(e)
            self.options.append(opts)
        self.wall_s = 0.0

    def run(self, histories=None):
        """Transport every plan's histories (or the first `histories[i]` of plan i) concurrently."""
        t = time.perf_counter()
        for i, (e, j, o) in enumerate(zip(self.engines, self.jobs, self.options)):
            e.reset_tally()
            e.launch(0, j.histories if histories is None else histories[i], **o)
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
