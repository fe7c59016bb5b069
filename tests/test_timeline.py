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


class _FakeEngine:
    """Two waves of known stamps (ns): wave 1 runs the source, the photon jaws and
    phantom kernels and the electron phantom kernel; wave 2 only a 2 ms photon-jaws
    launch. The planner counts waves from 1, so index 0 stays empty."""
    TIMELINE_KERNELS = ["source", "photon_jaws", "photon_mlc", "photon", "compton", "photo", "rayleigh", "pair",
                        "electron_jaws", "electron_mlc", "electron", "moller", "brems", "bhabha", "annih",
                        "electron_near", "photon_jaws_long"]

    def run(self, h0, h1, batch=0):
        return {"waves": 3, "device_ms": 9.0}

    def set_timeline(self, n):
        pass

    def timeline(self):
        tl = np.zeros((8, 32, 2), np.uint64)
        tl[:, :, 0] = np.iinfo(np.uint64).max
        ms = 1_000_000
        for k, (a, b) in {0: (0, 1), 1: (1, 3), 3: (1, 4), 10: (5, 7)}.items():
            tl[1, k] = (a * ms, b * ms)
        tl[2, 1] = (8 * ms, 10 * ms)
        return tl


def test_timeline_summary_sums_phases_and_kernels():
    import types
    from gegs_b200.profile_case import timeline_summary
    args = types.SimpleNamespace(first=0, histories=10, batch=0)
    d = timeline_summary(_FakeEngine(), args, (4, 4, 4))
    assert d["phase_ms"]["source"] == 1.0
    assert d["phase_ms"]["photon transport"] == 5.0           # wave 1: 1..4 ms, wave 2: 8..10 ms
    assert d["phase_ms"]["electron transport"] == 2.0
    assert d["kernel_ms"]["photon_jaws"] == 4.0 and d["kernel_ms"]["photon"] == 3.0
    assert d["lone_photon_jaws_waves"] == 1 and d["lone_photon_jaws_ms"] == 2.0
    assert d["wave_ms"] == [7.0, 2.0] and d["gaps_between_waves_ms"] == 1.0
    assert d["waves_under_1ms"] == 0 and d["wave_phase_ms"]["photon transport"] == [3.0, 2.0]
