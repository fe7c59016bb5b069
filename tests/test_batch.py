"""Several plans at once on one GPU: each plan's tally equals its own run,
bit for bit, whether the plans run concurrently or one after another."""
import numpy as np
import pytest

from gegs_b200 import workloads as W
from gegs_b200.batch import choose_options


def test_choose_options_respects_memory_share():
    o = choose_options(100_000_000, 64e9)
    assert o["batch"] == 1 << 22 and o["refill_below"] == o["batch"] // 4
    small = choose_options(10_000, 64e9)
    assert small["batch"] == 1 << 16
    capped = choose_options(100_000_000, 1e9)
    assert capped["batch"] * 4.5e3 <= 1e9 and capped["batch"] >= 1 << 16


@pytest.mark.gpu
def test_concurrent_plans_match_their_own_runs(oracle):
    from gegs_b200.batch import PlanBatch
    jobs = W.config5(n_plans=4, hist_min=2000, hist_max=20000, nphsp=5000, dims_max=(48, 48, 32), dims_min=24)
    pb = PlanBatch(jobs, memory_budget_gb=4.0)
    st = pb.run()
    conc = pb.tallies()
    pb.run_sequential()
    seq = pb.tallies()
    for a, b, s in zip(conc, seq, st):
        np.testing.assert_array_equal(a, b)
        assert s["error_bits"] == 0 and a.sum() > 0
    ref, _ = oracle.run(jobs[1].physics, jobs[1].scene(), 0, jobs[1].histories)
    np.testing.assert_array_equal(conc[1], ref)
    pb.close()


def test_launch_group_checks_its_arguments():
    from gegs_b200.engine import launch_group
    with pytest.raises(ValueError):
        launch_group([], [])
    with pytest.raises(ValueError):
        launch_group([object()], [(0, 1), (1, 2)])


@pytest.mark.gpu
def test_one_launch_equals_launches_per_plan_and_the_oracle(oracle):
    """All plans as one graph launch (a branch per plan, gegs_launch_group):
    each plan's tally equals its launch on its own stream and the oracle; the
    group refuses an engine twice and an engine with a run in flight."""
    from gegs_b200.batch import PlanBatch
    from gegs_b200.engine import GegsError, launch_group
    jobs = W.config5(n_plans=5, hist_min=2000, hist_max=20000, nphsp=5000, dims_max=(48, 48, 32), dims_min=24)
    pb = PlanBatch(jobs, memory_budget_gb=4.0)
    st = pb.run(one_launch=True)
    one = pb.tallies()
    pb.run(one_launch=True)                                          # the cached group graph again
    again = pb.tallies()
    pb.run(one_launch=False)
    per = pb.tallies()
    for a, b in zip(one, again):
        np.testing.assert_array_equal(a, b)
    for a, b, s in zip(one, per, st):
        np.testing.assert_array_equal(a, b)
        assert s["error_bits"] == 0 and a.sum() > 0 and s["waves"] > 0
    for k in (0, 3):
        ref, _ = oracle.run(jobs[k].physics, jobs[k].scene(), 0, jobs[k].histories)
        np.testing.assert_array_equal(one[k], ref)
    e = pb.engines
    with pytest.raises(GegsError):
        launch_group([e[0], e[1], e[0]], [(0, 10)] * 3)
    e[2].launch(0, 10)
    with pytest.raises(GegsError):
        launch_group([e[1], e[2]], [(0, 10)] * 2)
    e[2].wait()
    launch_group(e[:2], [(0, 100), (0, 100)])                       # the engines are usable again
    for x in e[:2]:
        x.wait()
    pb.close()


@pytest.mark.gpu
def test_autotuned_plans_keep_their_tallies(oracle):
    """The autotuner changes only how a plan runs (batch, grid, step budgets,
    refill threshold): every candidate it times gives the same tally, and the
    plan tuned by it still equals the oracle bit for bit."""
    from gegs_b200.batch import PlanBatch, autotune
    from gegs_b200.engine import Engine
    job = W.config3(histories=6000, nphsp=4000, dims=(40, 40, 24))
    e = Engine(0)
    e.set_physics(job.physics)
    e.set_scene(job.scene())
    best, best_ms, trials = autotune(e, job, sample=3000)
    assert len(trials) >= 8 and best_ms == min(t for _, t in trials)
    seen = set()
    for o, _ in trials:
        e.reset_tally()
        e.run(0, 3000, **o)
        seen.add(e.tally().tobytes())
    assert len(seen) == 1
    e.close()
    pb = PlanBatch([job], memory_budget_gb=2.0, tune_sample=2000)
    pb.run()
    ref, _ = oracle.run(job.physics, job.scene(), 0, job.histories)
    np.testing.assert_array_equal(pb.tallies()[0], ref)
    pb.close()
