"""Batch statistics folded on the device (gegs_stat_*) against the same
arithmetic on the host from the batches' tallies: the reference's
GET_UNCERTAINTY formula sqrt((S2/n - (S1/n)^2)/(n-1)) / (S1/n)
(CUDA_EGS.cu:817-876). The device adds the same doubles in the same order, so
the results agree to the last bit."""
import numpy as np
import pytest

from gegs_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_device_batch_statistics_match_the_host_formula(engine):
    job = W.config2(histories=12000, nphsp=6000, n=30)
    engine.set_physics(job.physics)
    engine.set_scene(job.scene())
    nb = 6
    engine.reset_tally()
    engine.run(0, 500)                           # a tally that exists before the series is not counted
    engine.stat_begin()
    prev = engine.tally()
    s1 = np.zeros(engine.nvox)
    s2 = np.zeros(engine.nvox)
    for b in range(nb):
        engine.run(500 + b * 1500, 500 + (b + 1) * 1500)
        engine.stat_fold()
        t = engine.tally()
        x = (t - prev).astype(np.float64) * 2.0 ** -30
        prev = t
        s1 += x
        s2 += x * x
    mean, rel, n = engine.stat_get()
    assert n == nb
    m = s1 / nb
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.where(m > 0, np.sqrt(np.maximum(s2 / nb - m * m, 0.0) / (nb - 1)) / m, 0.0)
    np.testing.assert_array_equal(mean, m)
    np.testing.assert_allclose(rel, r, rtol=1e-15, atol=0)
    hit = m > 0
    assert hit.sum() > 100 and np.all(rel[hit] >= 0) and np.median(rel[hit]) < 1.5


def test_stat_get_needs_two_batches(engine):
    from gegs_b200.engine import GegsError
    job = W.config1(histories=400, n=10, voxel=3.0)
    engine.set_physics(job.physics)
    engine.set_scene(job.scene())
    engine.stat_begin()
    engine.run(0, 200)
    engine.stat_fold()
    with pytest.raises(GegsError, match="two folded batches"):
        engine.stat_get()
    engine.run(200, 400)
    engine.stat_fold()
    assert engine.stat_get()[2] == 2
