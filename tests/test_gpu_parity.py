"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

Per-particle counter-based RNG streams, IEEE-only transcendentals on both
sides and an int64 fixed-point tally make the comparison exact: every voxel's
energy tally must be bit-identical, in both the persistent and the plain form
and for any batch size (the order in which the GPU processes particles does
not enter the result).
"""
import numpy as np
import pytest

from gegs_b200 import workloads as W
from gegs_b200.engine import MODE_PERSISTENT, MODE_PLAIN

pytestmark = pytest.mark.gpu


def _run(engine, job, h0, h1, **kw):
    sh = job.scene(hownear_region_offset=kw.pop("offset", 5))
    engine.set_physics(job.physics)
    engine.set_scene(sh)
    st = engine.run(h0, h1, **kw)
    return engine.tally(), st, sh


def _assert_same(gpu, ref):
    bad = np.flatnonzero(gpu != ref)
    assert bad.size == 0, (f"{bad.size} voxels differ; first {bad[:5]}: gpu {gpu[bad[:5]]} vs oracle {ref[bad[:5]]}; "
                           f"totals {gpu.sum()} vs {ref.sum()}")


def test_c1_persistent_bit_exact(engine, oracle):
    job = W.config1(histories=20000, n=30, voxel=1.0)
    gpu, st, sh = _run(engine, job, 0, job.histories, mode=MODE_PERSISTENT)
    ref, rst = oracle.run(job.physics, sh, 0, job.histories)
    _assert_same(gpu, ref)
    assert st["processed"][0] >= job.histories
    assert gpu.sum() > 0


def test_c1_plain_bit_exact(engine, oracle):
    job = W.config1(histories=5000, n=30, voxel=1.0)
    gpu, st, sh = _run(engine, job, 0, job.histories, mode=MODE_PLAIN)
    ref, _ = oracle.run(job.physics, sh, 0, job.histories)
    _assert_same(gpu, ref)


def test_batch_size_does_not_change_result(engine):
    job = W.config1(histories=8000, n=20, voxel=1.5)
    a, _, _ = _run(engine, job, 0, job.histories, batch=256)
    b, _, _ = _run(engine, job, 0, job.histories, batch=1 << 16, blocks_per_sm=2)
    _assert_same(a, b)


def test_history_ranges_add_up(engine):
    job = W.config1(histories=6000, n=20, voxel=1.5)
    full, _, sh = _run(engine, job, 0, job.histories)
    engine.reset_tally()
    engine.run(0, 2500)
    engine.run(2500, job.histories)
    _assert_same(engine.tally(), full)


def test_c2_phase_space_slab_bit_exact(engine, oracle):
    job = W.config2(histories=20000, nphsp=5000, n=40)
    gpu, st, sh = _run(engine, job, 0, job.histories)
    ref, _ = oracle.run(job.physics, sh, 0, job.histories)
    _assert_same(gpu, ref)
    assert st["processed"][5] > 0          # electrons from the phase space and from interactions


def test_c3_ct_mlc_jaws_five_fields_bit_exact(engine, oracle):
    job = W.config3(histories=30000, nphsp=20000, dims=(64, 64, 30))
    gpu, st, sh = _run(engine, job, 0, job.histories)
    ref, _ = oracle.run(job.physics, sh, 0, job.histories)
    _assert_same(gpu, ref)
    assert gpu.sum() > 0


def test_corrected_hownear_decode_bit_exact(engine, oracle):
    job = W.config1(histories=5000, n=30, voxel=1.0)
    gpu, _, sh = _run(engine, job, 0, job.histories, offset=6)
    ref, _ = oracle.run(job.physics, sh, 0, job.histories)
    _assert_same(gpu, ref)


def test_run_to_run_identical(engine):
    job = W.config2(histories=5000, nphsp=5000, n=30)
    a, _, _ = _run(engine, job, 0, job.histories)
    b, _, _ = _run(engine, job, 0, job.histories)
    _assert_same(a, b)


def test_step_budget_does_not_change_result(engine, oracle):
    """Tracks split across launches (continuation queues) give the same tally
    as tracks run to the end in one launch, and as the oracle."""
    job = W.config3(histories=6000, nphsp=5000, dims=(48, 48, 24))
    a, sa, sh = _run(engine, job, 0, job.histories, photon_budget=1, electron_budget=1)
    b, sb, _ = _run(engine, job, 0, job.histories, photon_budget=8, electron_budget=3)
    c, sc, _ = _run(engine, job, 0, job.histories, photon_budget=60000, electron_budget=60000)
    ref, rst = oracle.run(job.physics, sh, 0, job.histories)
    _assert_same(a, ref)
    _assert_same(b, ref)
    _assert_same(c, ref)
    assert sa["processed"] == sc["processed"]
    assert sa["electron_steps"] == sc["electron_steps"] and sa["photon_steps"] == sc["photon_steps"]
    assert sa["waves"] > sc["waves"]


def test_timed_mode_bit_exact(engine, oracle):
    from gegs_b200.engine import MODE_TIMED
    job = W.config2(histories=4000, nphsp=4000, n=30)
    gpu, st, sh = _run(engine, job, 0, job.histories, mode=MODE_TIMED)
    ref, _ = oracle.run(job.physics, sh, 0, job.histories)
    _assert_same(gpu, ref)
    assert st["stage_launches"][0] == st["waves"] - 1 or st["stage_launches"][0] >= 1
    assert sum(st["stage_ms"]) > 0


# ---- the configurations at their full geometry --------------------------------
# The sizes above keep the oracle fast; these run the geometry the bench and
# BASELINE configurations use -- C1 60^3 at 0.5 cm, C2 120^3 at 0.25 cm, C3
# 256x256x120 at 1x1x2.5 mm (7.9M voxels, above 2^22) with five gantry angles,
# the full 60-pair MLC and the jaws -- on a few 1e4 histories.
def test_c1_full_geometry_bit_exact(engine, oracle):
    job = W.config1(histories=50000)
    assert job.meta["n"] == 60 and job.meta["voxel"] == 0.5
    gpu, st, sh = _run(engine, job, 0, job.histories)
    ref, _ = oracle.run(job.physics, sh, 0, job.histories)
    _assert_same(gpu, ref)
    assert gpu.sum() > 0


def test_c2_full_geometry_bit_exact(engine, oracle):
    job = W.config2(histories=30000, nphsp=30000)
    assert sh_dims(job) == (120, 120, 120)
    gpu, st, sh = _run(engine, job, 0, job.histories)
    ref, _ = oracle.run(job.physics, sh, 0, job.histories)
    _assert_same(gpu, ref)
    assert st["processed"][5] > 0


def test_c3_full_geometry_bit_exact(engine, oracle):
    job = W.config3(histories=30000, nphsp=30000)
    assert sh_dims(job) == (256, 256, 120) and len(job.fields) == 5
    gpu, st, sh = _run(engine, job, 0, job.histories)
    ref, _ = oracle.run(job.physics, sh, 0, job.histories)
    _assert_same(gpu, ref)
    assert gpu.sum() > 0
    assert min(st["photon_steps_class"]) > 0 and min(st["electron_steps_class"]) > 0   # jaws, MLC, phantom


@pytest.mark.parametrize("case", ["c3_full", "c3_small_budget1", "c2"])
def test_pipelined_waves_bit_exact(engine, oracle, case):
    """The persistent form's default pipelined waves (the photon and electron
    transports at once, then all eight interaction kernels; positrons that
    stop in the electron transport annihilate in the annihilation kernel)
    against GEGS_RUN_SERIAL_WAVES: both tallies are the oracle's, and the
    particles processed per stage and the steps taken are the same."""
    kw = {}
    if case == "c3_full":
        job = W.config3(histories=30000, nphsp=30000)
    elif case == "c3_small_budget1":
        job = W.config3(histories=6000, nphsp=5000, dims=(48, 48, 24))
        kw = dict(photon_budget=1, electron_budget=1)
    else:
        job = W.config2(histories=20000, nphsp=20000, n=40)
    serial, ss, sh = _run(engine, job, 0, job.histories, pipelined=False, **kw)
    engine.reset_tally()
    pipe = engine.run(0, job.histories, **kw)
    gpu = engine.tally()
    ref, _ = oracle.run(job.physics, sh, 0, job.histories)
    _assert_same(gpu, ref)
    _assert_same(serial, ref)
    assert pipe["error_bits"] == 0
    assert pipe["processed"] == ss["processed"]
    assert pipe["photon_steps"] == ss["photon_steps"] and pipe["electron_steps"] == ss["electron_steps"]
    assert pipe["photon_steps_class"] == ss["photon_steps_class"]
    assert pipe["electron_steps_class"] == ss["electron_steps_class"]
    if case == "c3_full":
        assert ss["processed"][4] > 0                      # pair production: positrons that come to rest


def sh_dims(job):
    p = job.phantom
    return len(p["x_bounds"]) - 1, len(p["y_bounds"]) - 1, len(p["z_bounds"]) - 1


def test_tables_staged_in_shared_memory_bit_exact(engine, oracle):
    """GEGS_RUN_STAGE_TABLES: the photon consumers read the mean-free-path and
    Rayleigh tables from shared memory; the tally is the oracle's, as without."""
    job = W.config3(histories=8000, nphsp=6000, dims=(48, 48, 24))
    gpu, st, sh = _run(engine, job, 0, job.histories, stage_tables=True)
    ref, _ = oracle.run(job.physics, sh, 0, job.histories)
    _assert_same(gpu, ref)
    engine.reset_tally()
    engine.run(0, job.histories, mode=2, stage_tables=True)          # the timed form launches them by name
    _assert_same(engine.tally(), ref)


@pytest.mark.gpu
def test_run_on_a_callers_stream(engine, oracle):
    """gegs_set_stream: the engine's work goes on the caller's stream; the
    tally is the same, and the engine returns to its own stream after."""
    import torch
    job = W.config1(histories=3000, n=16, voxel=2.0)
    sh = job.scene()
    engine.set_physics(job.physics)
    engine.set_scene(sh)
    s = torch.cuda.Stream(device=0)
    engine.set_stream(s)
    engine.reset_tally()
    engine.run(0, job.histories)
    got = engine.tally()
    engine.set_stream(None)
    ref, _ = oracle.run(job.physics, sh, 0, job.histories)
    np.testing.assert_array_equal(got, ref)
    engine.reset_tally()
    engine.run(0, job.histories)
    np.testing.assert_array_equal(engine.tally(), ref)


@pytest.mark.gpu
def test_set_field_equals_a_new_scene(engine, oracle):
    """gegs_set_field: new leaf positions and jaws for one field, set without
    uploading the phantom again, give the tally of a scene built with them."""
    from gegs_b200 import geometry as G
    job = W.config3(histories=3000, nphsp=3000, dims=(32, 32, 16))
    engine.set_physics(job.physics)
    engine.set_scene(job.scene())
    f = dict(job.fields[2])
    pos = np.asarray(f["leaf_pos"], np.float32) + np.float32(0.7)          # every leaf pair opened by 1.4 cm
    f["leaf_pos"] = pos
    f["endnode"] = G.leaf_endnodes(job.beam["mlc"]["crossYZ"], pos, job.beam["mlc"]["zmin"],
                                   job.beam["mlc"]["zthick"], job.beam["source_to_isocenter"])
    f.update(G.secjaws_polygons(job.meta["jaws"], -4.0, 5.0, -3.0, 4.0, job.beam["source_to_isocenter"]))
    engine.set_field(2, f)
    engine.reset_tally()
    engine.run(0, job.histories)
    job.fields[2] = f
    ref, _ = oracle.run(job.physics, job.scene(), 0, job.histories)
    np.testing.assert_array_equal(engine.tally(), ref)
