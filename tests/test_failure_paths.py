"""Failure paths: every error ends in a clean status or exception, never a
hang, a fault or a silent loss.

The reference has two failure behaviours on this path. A full particle stack
drops the particle with a message (utility.cu:270-275), and an electron that
keeps taking negative steps aborts the program (electron.cu:1881-1889); a bad
input file or CUDA error ends the process through error()/exit()
(output.c:51-90). Here a queue overflow sets a device status bit and the run
returns GEGS_ERR_QUEUE_FULL, a run out of waves returns GEGS_ERR_STEP_BUDGET,
a particle in a module this path does not model returns GEGS_ERR_MODULE, a
history outside every field returns GEGS_ERR_SOURCE, and bad inputs raise
before anything reaches the GPU.

The CPU tests feed corrupt files and tables. The GPU tests make the device
report each status with in-bounds work only (every push checks the queue's
capacity before it writes), and then check that the next normal run on the
same engine is still bit-identical to the oracle.
"""
import numpy as np
import pytest

from gegs_b200 import geometry as G
from gegs_b200 import io_formats as F
from gegs_b200 import physics_data as PD
from gegs_b200 import workloads as W
from gegs_b200.engine import GegsError, check_physics
from gegs_b200.plan import PlanError, load_plan

from test_plan_io import _job, _write_plan

ERR_ARG, ERR_QUEUE_FULL, ERR_MODULE, ERR_STEP_BUDGET, ERR_SOURCE = 1, 3, 4, 6, 7


# ---------------------------------------------------------------------------
# corrupt inputs (CPU)
# ---------------------------------------------------------------------------
def test_truncated_phase_space_is_rejected(tmp_path):
    job = W.config2(histories=1000, nphsp=1000, n=10)
    path = tmp_path / "beam.egsphsp1"
    F.write_egsphsp1(path, job.phsp, "MODE0")
    assert len(F.read_egsphsp1(path)) == 1000
    raw = path.read_bytes()
    path.write_bytes(raw[:-28 * 10 - 5])              # ten and a bit records missing
    with pytest.raises(ValueError, match="truncated"):
        F.read_egsphsp1(path)


def test_phase_space_with_unknown_mode_is_rejected(tmp_path):
    path = tmp_path / "beam.egsphsp1"
    path.write_bytes(b"MODE7" + bytes(100))
    with pytest.raises(ValueError, match="mode"):
        F.read_egsphsp1(path)


def test_egsphant_with_bad_dimension_line_is_rejected(tmp_path):
    job = W.config1(histories=10, n=6, voxel=5.0)
    p = job.phantom
    path = tmp_path / "w.egsphant"
    F.write_egsphant(path, job.media, p["x_bounds"], p["y_bounds"], p["z_bounds"], p["voxel_med"], p["density"])
    assert F.read_egsphant(path)["nx"] == 6
    lines = path.read_text().split("\n")
    k = 2 + len(job.media)                             # count, names, ESTEPE line, then the dimensions
    assert lines[k].split() == ["6", "6", "6"]
    for bad in ("6 6", "6 x 6", "6 0 6"):
        lines[k] = bad
        path.write_text("\n".join(lines))
        with pytest.raises(ValueError, match="voxel counts|nx ny nz"):
            F.read_egsphant(path)


def test_egsphant_with_short_medium_row_is_rejected(tmp_path):
    job = W.config1(histories=10, n=6, voxel=5.0)
    p = job.phantom
    path = tmp_path / "w.egsphant"
    F.write_egsphant(path, job.media, p["x_bounds"], p["y_bounds"], p["z_bounds"], p["voxel_med"], p["density"])
    text = path.read_text().replace("111111\n", "1111\n", 1)
    path.write_text(text)
    with pytest.raises(ValueError, match="medium row"):
        F.read_egsphant(path)


def test_ini_missing_a_required_key_is_rejected(tmp_path):
    ini = _write_plan(tmp_path, _job())
    assert load_plan(ini).job.histories > 0
    text = ini.read_text()
    for key in ("histories", "egsphant file", "mlcinfo file"):
        bad = ini.parent / f"no_{key.replace(' ', '_')}.ini"     # beside the plan: same relative paths
        bad.write_text("\n".join(l for l in text.split("\n") if not l.strip().startswith(key + " ")))
        with pytest.raises(PlanError, match=key):
            load_plan(bad)


def test_physics_block_with_nan_is_rejected_through_the_c_abi():
    blk = PD.build_block(["H2O700ICRU", "AIR700ICRU"])
    check_physics(blk)                                 # the generated block passes
    for name, idx in (("gmfp", (5, 1)), ("dedx", (17, 0)), ("ums_array", (100,)), ("rm", ())):
        bad = blk.copy()
        bad[name][idx] = np.nan
        with pytest.raises(GegsError, match=f"{name}.*not finite") as err:
            check_physics(bad)
        assert err.value.status == ERR_ARG
    bad = blk.copy()
    bad["sig"][3, 1] = np.inf
    with pytest.raises(GegsError, match="sig"):
        check_physics(bad)


def test_physics_block_with_bad_medium_count_is_rejected():
    blk = PD.build_block(["H2O700ICRU"])
    for nmed in (0, -1, 7):
        bad = blk.copy()
        bad["nmed"] = nmed
        with pytest.raises(GegsError, match="nmed"):
            check_physics(bad)


# ---------------------------------------------------------------------------
# device status codes (GPU)
# ---------------------------------------------------------------------------
def _fresh(engine, job):
    sh = job.scene()
    engine.set_physics(job.physics)
    engine.set_scene(sh)
    return sh


def _assert_normal_run_matches_oracle(engine, oracle, job, sh):
    engine.reset_tally()
    engine.run(0, job.histories)
    ref, _ = oracle.run(job.physics, sh, 0, job.histories)
    np.testing.assert_array_equal(engine.tally(), ref)


@pytest.mark.gpu
def test_wave_budget_exhausted_returns_step_budget(engine, oracle):
    job = W.config3(histories=4000, nphsp=4000, dims=(32, 32, 16))
    sh = _fresh(engine, job)
    with pytest.raises(GegsError) as err:
        engine.run(0, job.histories, max_waves=2)
    assert err.value.status == ERR_STEP_BUDGET
    st = engine.stats()
    assert st["waves"] == 2 and st["error_bits"] & 8
    _assert_normal_run_matches_oracle(engine, oracle, job, sh)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 2])
def test_queue_overflow_returns_queue_full(engine, oracle, mode):
    # 2000 primaries into queues capped at 64 records: the pushes past the
    # capacity write nothing, set the status bit, and the run stops
    job = W.config1(histories=2000, n=16, voxel=2.0)
    sh = _fresh(engine, job)
    with pytest.raises(GegsError) as err:
        engine.run(0, job.histories, mode=mode, batch=2000, queue_cap=64)
    assert err.value.status == ERR_QUEUE_FULL
    assert engine.stats()["error_bits"] & 1
    _assert_normal_run_matches_oracle(engine, oracle, job, sh)


@pytest.mark.gpu
def test_unsupported_module_returns_module_error(engine, oracle):
    # the block module starts the beam line: this transport path does not model it
    job = W.config1(histories=500, n=16, voxel=2.0)
    job.beam = dict(job.beam, module_order=G.module_order(False, False, block_on=True))
    _fresh(engine, job)
    with pytest.raises(GegsError) as err:
        engine.run(0, job.histories)
    assert err.value.status == ERR_MODULE
    good = W.config1(histories=500, n=16, voxel=2.0)
    _assert_normal_run_matches_oracle(engine, oracle, good, _fresh(engine, good))


@pytest.mark.gpu
def test_history_outside_every_field_returns_source_error(engine, oracle):
    job = W.config1(histories=1000, n=16, voxel=2.0)
    sh = _fresh(engine, job)
    with pytest.raises(GegsError) as err:
        engine.run(0, job.histories + 50)
    assert err.value.status == ERR_SOURCE
    _assert_normal_run_matches_oracle(engine, oracle, job, sh)
