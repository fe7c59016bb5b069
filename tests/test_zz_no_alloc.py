"""gegs_run_noalloc, the transport entry point that allocates no device memory.

Some callers cannot allocate GPU memory while they run: a planning system or
dose server that reserved the whole GPU when it started (gegs_run's event
queues take several GB at the default batch), or a latency-bound loop that
cannot absorb cudaFree's device-wide synchronisation. For them the library
keeps all transport scratch in one fixed array of GEGS_NOALLOC_MAX_BATCH
particles. These tests call it through the C ABI and compare its tally with
gegs_run's on the same histories, bit for bit (the tolerance of every other
parity test here), over two calls in a row that share the array.

The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from gegs_b200 import workloads as W
from gegs_b200.engine import MODE_TIMED, GegsError

pytestmark = pytest.mark.gpu

MAX_BATCH = 4096   # GEGS_NOALLOC_MAX_BATCH in include/gegs.h


def _noalloc(engine, h0, h1, batch=0):
    st = engine.L.gegs_run_noalloc(engine.h, h0, h1, batch)
    if st != 0:
        raise GegsError(st, engine.L.gegs_last_error(engine.h).decode())


def test_noalloc_matches_gegs_run_on_two_calls_in_a_row(engine):
    # CT phantom behind jaws and MLC, several fields: every kernel of the wave loop runs
    job = W.config3(histories=8000, nphsp=6000, dims=(48, 48, 24))
    engine.set_physics(job.physics)
    engine.set_scene(job.scene())
    first, second = (0, 3000), (3000, 8000)

    engine.reset_tally()
    engine.run(*first)
    ref_first = engine.tally()
    engine.run(*second)
    ref_both = engine.tally()

    engine.reset_tally()
    _noalloc(engine, *first)                      # default batch (the maximum)
    got_first = engine.tally()
    _noalloc(engine, *second, batch=1024)         # straight after, reusing the array
    got_both = engine.tally()

    assert ref_first.sum() > 0
    np.testing.assert_array_equal(got_first, ref_first)
    np.testing.assert_array_equal(got_both, ref_both)
    st = engine.stats()
    assert st["error_bits"] == 0 and st["processed"][0] > 0


def test_noalloc_rejects_batch_above_the_fixed_limit(engine):
    job = W.config1(histories=100, n=10, voxel=3.0)
    engine.set_physics(job.physics)
    engine.set_scene(job.scene())
    with pytest.raises(GegsError) as err:
        _noalloc(engine, 0, 100, batch=MAX_BATCH + 1)
    assert err.value.status == 1
    assert "GEGS_NOALLOC_MAX_BATCH" in str(err.value)
    _noalloc(engine, 0, 100, batch=MAX_BATCH)    # the limit itself is accepted


def test_noalloc_counts_waves_and_steps_like_the_timed_form(engine):
    # The timed form launches the same kernels wave by wave, one at a time;
    # with the same batch, refill threshold and step budgets it plans the same
    # waves, so the statistics (waves, per-stage counts, steps per geometry
    # class) agree as well as the tally.
    job = W.config3(histories=3000, nphsp=3000, dims=(40, 40, 20))
    engine.set_physics(job.physics)
    engine.set_scene(job.scene())
    engine.reset_tally()
    ref = engine.run(0, job.histories, mode=MODE_TIMED, batch=1024, refill_below=1024 // 50,
                     photon_budget=16, electron_budget=8)
    ref_tally = engine.tally()
    engine.reset_tally()
    _noalloc(engine, 0, job.histories, batch=1024)
    got = engine.stats()
    np.testing.assert_array_equal(engine.tally(), ref_tally)
    for key in ("waves", "processed", "photon_steps", "electron_steps", "photon_steps_class",
                "electron_steps_class"):
        assert got[key] == ref[key], key


def test_noalloc_refuses_while_a_launched_run_is_outstanding(engine):
    # gegs_launch leaves a run queued on the engine's stream; the no-allocation
    # call must not queue behind it and take over its events and statistics.
    job = W.config1(histories=2000, n=16, voxel=2.0)
    engine.set_physics(job.physics)
    engine.set_scene(job.scene())
    engine.reset_tally()
    engine.launch(0, job.histories)
    with pytest.raises(GegsError) as err:
        _noalloc(engine, 0, job.histories)
    assert err.value.status == 1
    assert "gegs_wait" in str(err.value)
    st = engine.wait()
    launched = engine.tally()
    assert st["error_bits"] == 0 and launched.sum() > 0
    engine.reset_tally()
    _noalloc(engine, 0, job.histories)            # usable again once the launched run is waited for
    np.testing.assert_array_equal(engine.tally(), launched)
