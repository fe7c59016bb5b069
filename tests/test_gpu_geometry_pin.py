"""The CUDA geometry routines checked directly, without a transport run in
between: howfar (region entered, step, state after the call) and hownear of
the phantom, the DYNVMLC and the secondary jaws, run on the device by
gegs_probe_geometry on given particle states.

* against the reference's own routines: the outputs the reference harness
  recorded for 9 559 states of the full CT head 5-field geometry
  (tests/golden/ref_pin_c3.npz, written by tests/golden/make_ref_fixtures.py);
* against the oracle: every particle state that enters the photon and
  electron stages of oracle runs of the full C1, C2 and C3 geometries, at the
  transport's step and at short steps.

Bit for bit."""
import pathlib

import numpy as np
import pytest

import refpin_cases as RC

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


def _engine(engine, job):
    sh = job.scene()
    engine.set_physics(job.physics)
    engine.set_scene(sh)
    return sh


def _compare(res, region, t, particle, tperp):
    assert np.array_equal(res["region"], region), "howfar region"
    assert res["t"].tobytes() == np.asarray(t, np.float32).tobytes(), "howfar step"
    assert res["tperp"].tobytes() == np.asarray(tperp, np.float32).tobytes(), "hownear distance"
    assert res["particle"].tobytes() == np.ascontiguousarray(particle).tobytes(), "state after howfar"


@pytest.mark.gpu
def test_device_geometry_equals_the_reference_recordings(engine):
    z = np.load(GOLDEN / "ref_pin_c3.npz")
    _engine(engine, RC.job("c3"))
    res = engine.probe_geometry(z["geom_in"], z["geom_t_in"])
    assert len(res["region"]) == len(z["geom_in"]) > 9000
    assert set(np.unique(z["geom_in"]["module"])) >= {1, 2, 3, 6}       # jaws Y, jaws X, MLC, phantom
    _compare(res, z["geom_region"], z["geom_t"], z["geom_out"], z["geom_tperp"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c1", "c2", "c3"])
def test_device_geometry_equals_the_oracle(engine, name):
    from oracle import refpin as R
    job = RC.job(name)
    sh = _engine(engine, job)
    pair = R.OraclePair(job.physics, sh)
    cap = pair.capture(0, job.histories, every=1, cap_n=60000)
    parts = np.concatenate([cap[0], cap[5]])                         # photon and electron stage entries
    assert len(parts) > 5000
    rng = np.random.default_rng(11)
    for t_in in (np.full(len(parts), 1e3, np.float32), rng.exponential(0.3, len(parts)).astype(np.float32)):
        want = pair.geom(parts, t_in)
        res = engine.probe_geometry(parts, t_in)
        _compare(res, want["region"], want["t"], want["particle"], want["tperp"])
