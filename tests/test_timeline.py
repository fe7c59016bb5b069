"""The wave timeline (tracing): every kernel of the persistent graph stamps
its first start and last end per wave; recording it leaves the tally as it
is bit for bit."""
import numpy as np
import pytest

from gegs_b200 import workloads as W


@pytest.mark.gpu
def test_wave_timeline_stamps_every_kernel_and_keeps_the_tally(engine):
    job = W.config3(histories=6000, nphsp=3000, dims=(24, 24, 12))
    engine.set_physics(job.physics)
    engine.set_scene(job.scene())
    engine.reset_tally()
    engine.run(0, job.histories, batch=1 << 12)
    plain = engine.tally()
    engine.set_timeline(4096)
    try:
        engine.reset_tally()
        st = engine.run(0, job.histories, batch=1 << 12)
        np.testing.assert_array_equal(engine.tally(), plain)
        tl = engine.timeline()[:st["waves"]]
        ran = tl[:, :, 1] > 0
        w = np.flatnonzero(ran.any(axis=1))                # the planner counts waves from 1
        assert ran[w[0], 0]                                # the source runs in the first wave
        for k in (1, 2, 3, 8, 9, 10):                      # every transport consumer ran
            assert ran[:, k].any()
        assert (tl[:, :, 1][ran] >= tl[:, :, 0][ran]).all()
        assert (tl[:, :, 0][~ran] == np.iinfo(np.uint64).max).all()
        # waves are in order: each wave's first start follows the previous wave's last end
        first = np.where(ran, tl[:, :, 0], np.iinfo(np.uint64).max).min(axis=1)
        last = np.where(ran, tl[:, :, 1], 0).max(axis=1)
        assert (first[w[1:]] >= last[w[:-1]]).all()
    finally:
        engine.set_timeline(0)
