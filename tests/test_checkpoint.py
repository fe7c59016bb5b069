"""Checkpoint and resume: the tally and the next history index are the whole
state of a run (per-history random streams, integer tally), so resuming a
saved run on a fresh engine gives the uninterrupted run's tally bit for bit."""
import numpy as np
import pytest

from gegs_b200 import workloads as W


@pytest.mark.gpu
def test_resume_from_a_checkpoint_gives_the_whole_run(engine, tmp_path):
    from gegs_b200.engine import Engine
    job = W.config3(histories=6000, nphsp=3000, dims=(24, 24, 12))
    sh = job.scene()
    engine.set_physics(job.physics)
    engine.set_scene(sh)
    engine.reset_tally()
    engine.run(0, job.histories)
    whole = engine.tally()
    assert whole.sum() > 0
    engine.reset_tally()
    engine.run(0, 2500)
    engine.checkpoint(tmp_path / "run.npz", 2500)
    e2 = Engine(0)
    try:
        e2.set_physics(job.physics)
        e2.set_scene(sh)
        h = e2.resume(tmp_path / "run.npz")
        assert h == 2500
        e2.run(h, job.histories)
        np.testing.assert_array_equal(e2.tally(), whole)
        with pytest.raises(ValueError):
            e2.set_tally(np.zeros(7, np.int64))
    finally:
        e2.close()
