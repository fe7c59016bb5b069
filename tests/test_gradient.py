"""Beamlet fluence weights and the gradient by RNG-counter replay.

* The weighted forward is checked against the oracle bit for bit.
* The replayed gradient is checked against a reference gradient built from
  per-beamlet dose runs (dL/dw_b = sum_v dL/dD_v * D_b[v]) and against central
  finite differences with common random numbers.
"""
import numpy as np
import pytest
import torch

from gegs_b200 import workloads as W


def _job(histories=12000):
    job = W.config4(histories=histories, nphsp=6000, dims=(48, 48, 24), nb=8, bixel=1.25)
    job.meta["organ"] = W.ellipsoid_mask(job, (1.2, 0.6, 0.0), (0.8, 0.8, 1.2))
    return job


def test_unit_weights_leave_the_oracle_tally_unchanged(oracle):
    job = _job(3000)
    with_w = job.scene()
    bl = job.beam["beamlets"]
    job.beam["beamlets"] = dict(bl, weights=np.ones_like(bl["weights"]))
    ones = job.scene()
    del job.beam["beamlets"]
    plain = job.scene()
    a, _ = oracle.run(job.physics, ones, 0, job.histories)
    b, _ = oracle.run(job.physics, plain, 0, job.histories)
    c, _ = oracle.run(job.physics, with_w, 0, job.histories)
    np.testing.assert_array_equal(a, b)
    assert c.sum() > a.sum()          # weights 1..1.2 raise the energy of tagged histories


@pytest.mark.gpu
def test_weighted_forward_bit_exact(engine, oracle):
    job = _job()
    sh = job.scene()
    engine.set_physics(job.physics)
    engine.set_scene(sh)
    engine.run(0, job.histories)
    ref, _ = oracle.run(job.physics, sh, 0, job.histories)
    np.testing.assert_array_equal(engine.tally(), ref)


@pytest.mark.gpu
def test_replay_gradient_matches_beamlet_doses_and_finite_differences(engine):
    from gegs_b200.differentiable import (BeamletModel, beamlet_dose, beamlet_doses, fd_gradient,
                                          objective)
    job = _job()
    engine.set_physics(job.physics)
    engine.set_scene(job.scene())
    model = BeamletModel(engine, job)
    w0 = job.beam["beamlets"]["weights"].astype(np.float64)
    target, organ = job.meta["target"], job.meta["organ"]
    model.calibrate(w0, target, 50.0)
    loss = lambda d: objective(d, target, organ)

    w = torch.tensor(w0, requires_grad=True)
    L = loss(beamlet_dose(w, model))
    L.backward()
    g = w.grad.numpy()
    assert np.isfinite(g).all() and np.abs(g).max() > 0

    rng = np.random.default_rng(7)
    live = np.flatnonzero(np.abs(g) > 1e-3 * np.abs(g).max())
    pick = rng.choice(live, size=min(16, live.size), replace=False)
    # reference gradient from per-beamlet dose runs
    d = torch.from_numpy(model.dose(w0)).requires_grad_(True)
    loss(d).backward()
    gD = d.grad.numpy()
    ref = np.array([gD @ Db for Db in beamlet_doses(model, pick)])
    np.testing.assert_allclose(g[pick], ref, rtol=1e-6, atol=1e-9 * np.abs(g).max())
    # central differences, common random numbers
    fd = fd_gradient(model, w0, pick, loss, delta=0.05)
    np.testing.assert_allclose(g[pick], fd, rtol=2e-3, atol=2e-3 * np.abs(g[pick]).max())


@pytest.mark.gpu
def test_gradient_descent_lowers_the_objective(engine):
    from gegs_b200.differentiable import BeamletModel, optimize_weights
    job = _job(6000)
    engine.set_physics(job.physics)
    engine.set_scene(job.scene())
    model = BeamletModel(engine, job)
    w0 = job.beam["beamlets"]["weights"].astype(np.float64)
    model.calibrate(w0, job.meta["target"], 50.0)
    w, hist = optimize_weights(model, w0, job.meta["target"], job.meta["organ"], iterations=8)
    assert len(hist) == 8 and hist[-1] < hist[0]
    assert (w >= 0).all()


@pytest.mark.gpu
def test_descent_on_several_plans_at_once_matches_one_plan_at_a_time(engine):
    from gegs_b200.differentiable import BeamletModel, optimize_weights, optimize_weights_batch
    from gegs_b200.engine import Engine
    jobs = [_job(4000), W.config4(histories=4000, nphsp=6000, dims=(40, 40, 20), nb=8, bixel=1.25,
                                  seed=W.SEED_BASE + 77)]
    jobs[1].meta["organ"] = W.ellipsoid_mask(jobs[1], (1.0, 0.5, 0.0), (0.8, 0.8, 1.0))
    engines, models, w0s = [], [], []
    try:
        for job in jobs:
            e = Engine(0)
            e.set_physics(job.physics)
            e.set_scene(job.scene())
            m = BeamletModel(e, job, batch=1 << 16)
            w0 = job.beam["beamlets"]["weights"].astype(np.float64)
            m.calibrate(w0, job.meta["target"], 50.0)
            engines.append(e); models.append(m); w0s.append(w0)
        targets = [j.meta["target"] for j in jobs]
        organs = [j.meta["organ"] for j in jobs]
        ws, hist = optimize_weights_batch(models, w0s, targets, organs, iterations=4)
        for k in range(len(jobs)):
            w1, h1 = optimize_weights(models[k], w0s[k], targets[k], organs[k], iterations=4)
            np.testing.assert_allclose(hist[k], h1, rtol=1e-9)
            np.testing.assert_allclose(ws[k], w1, rtol=1e-9, atol=1e-12)
            assert hist[k][-1] < hist[k][0]
    finally:
        for e in engines:
            e.close()
