"""The drop-in boundary: the reference's input files and INI schema in, the
``_DoseResults_NNNxNNNxNNN.bin`` dose grid out.

A synthetic CT plan (the C3 workload on a small grid) is written to disk in
the reference's formats (egsphant, egsphsp1, egsinp with CM DYNVMLC and CM
JAWS SECJAWS, mlcinfo + mlcinp, INI); reading it back with ``load_plan`` must
give the same transport job, so the oracle's tally for both is the same bit
for bit. The GPU test runs the command line on that plan and checks the dose
file against the oracle's tally converted the same way."""
import numpy as np
import pytest

from gegs_b200 import geometry as G
from gegs_b200 import io_formats as F
from gegs_b200 import workloads as W
from gegs_b200.plan import PlanError, load_plan, read_ini
from gegs_b200.scene import PHSP_DTYPE

DIMS = (24, 24, 12)
PER_FIELD = 400


def _job():
    return W.config3(histories=5 * PER_FIELD, nphsp=3000, dims=DIMS)


def _write_plan(tmp_path, job, extra="", per_field=PER_FIELD):
    d = tmp_path / "data"
    d.mkdir()
    p = job.phantom
    F.write_egsphant(d / "head.egsphant", job.media, p["x_bounds"], p["y_bounds"], p["z_bounds"], p["voxel_med"],
                     p["density"])
    F.write_egsphsp1(d / "beam.egsphsp1", job.phsp, "MODE0")
    (d / "VarianMLC.egsinp").write_text("TITLE\n" + F.dynvmlc_egsinp_text(job.meta["mlc"]) +
                                        F.secjaws_egsinp_text(job.meta["jaws"]))
    fields = []
    for i, f in enumerate(job.fields):
        name = f"field{i + 1}.mlcinp"
        F.write_mlcinp(d / name, f["leaf_pos"])
        x1, x2, y1, y2 = f["jaws"]
        fields.append(dict(angle=f["angle"], x1=x1, x2=x2, y1=y1, y2=y2, mu=1, mlcinp=name))
    F.write_mlcinfo(d / "plan.mlcinfo", fields)
    ini = tmp_path / "plan.ini"
    ini.write_text(f"""[General]
output prefix = "T1"
output directory = "out"
histories = {per_field}

[Data]
data directory = "data"
egsinp file = "VarianMLC.egsinp"
pegs file = "700icru.pegs4dat"
default medium = AIR700ICRU

[Phase space]
phsp file number = 1
phase space file = "beam"
z position = {job.beam['z_phsp']}

[SecJaws]
module SecJaws = On
secjaws file = "VarianMLC.egsinp"

[MLC]
module MLC = On
mlcinfo file = "plan.mlcinfo"

[Block]
module Block = Off

[Wedge]
module Wedge = Off

[CTcreate]
use ctcreate = No

[Phantom]
change coordinate = Yes
egsphant file = "head.egsphant"
isocenter location = 0 0 0
source to isocenter = 100

[Calibration]
dose calibration = No
{extra}""")
    return ini


def test_egsphant_round_trip(tmp_path):
    job = _job()
    p = job.phantom
    F.write_egsphant(tmp_path / "a.egsphant", job.media, p["x_bounds"], p["y_bounds"], p["z_bounds"],
                     p["voxel_med"], p["density"])
    r = F.read_egsphant(tmp_path / "a.egsphant")
    assert r["media"] == job.media and (r["nx"], r["ny"], r["nz"]) == DIMS
    for k in ("x_bounds", "y_bounds", "z_bounds", "density"):
        np.testing.assert_array_equal(r[k], np.asarray(p[k], np.float32))
    np.testing.assert_array_equal(r["voxel_med"], p["voxel_med"])


@pytest.mark.parametrize("mode", ["MODE0", "MODE2"])
def test_egsphsp1_round_trip_and_parts(tmp_path, mode):
    recs = _job().phsp[:1000]
    F.write_egsphsp1(tmp_path / "b_p0.egsphsp1", recs[:600], mode)
    F.write_egsphsp1(tmp_path / "b_p1.egsphsp1", recs[600:], mode)
    h = F.read_egsphsp1_header(tmp_path / "b_p0.egsphsp1")
    assert h["mode"] == mode and h["n"] == 600 and h["reclen"] == (28 if mode == "MODE0" else 32)
    got = F.read_phase_space(str(tmp_path / "b"), 2)
    assert got.dtype == PHSP_DTYPE
    np.testing.assert_array_equal(got, recs)
    np.testing.assert_array_equal(F.read_egsphsp1(tmp_path / "b_p1.egsphsp1", start=100, count=50), recs[700:750])


def _as_read(obj):
    """A geometry record with every real number rounded to float, as the
    reference (and the package) reads it from a file."""
    import dataclasses
    vals = {}
    for f in dataclasses.fields(obj):
        v = getattr(obj, f.name)
        if isinstance(v, float):
            v = float(np.float32(v))
        elif dataclasses.is_dataclass(v):
            v = _as_read(v)
        elif isinstance(v, list):
            v = [tuple(float(np.float32(x)) if isinstance(x, float) else x for x in row) for row in v]
        vals[f.name] = v
    return dataclasses.replace(obj, **vals)


def test_egsinp_modules_round_trip(tmp_path):
    m, j = G.DynVMLC.synthetic(), G.SecJaws()
    (tmp_path / "x.egsinp").write_text("a title\n:start geometry:\n" + F.secjaws_egsinp_text(j) +
                                      F.dynvmlc_egsinp_text(m))
    assert F.read_dynvmlc(tmp_path / "x.egsinp") == _as_read(m)
    assert F.read_secjaws(tmp_path / "x.egsinp") == _as_read(j)
    (tmp_path / "none.egsinp").write_text("no modules here\n")
    with pytest.raises(ValueError):
        F.read_dynvmlc(tmp_path / "none.egsinp")


def test_mlcinfo_and_mlcinp_round_trip(tmp_path):
    pos = np.random.default_rng(1).uniform(-3, 9, 120).astype(np.float32)
    F.write_mlcinp(tmp_path / "f.mlcinp", pos)
    np.testing.assert_array_equal(F.read_mlcinp(tmp_path / "f.mlcinp"), pos)
    fl = [dict(angle=a, x1=-5, x2=5.5, y1=-4, y2=6, mu=mu, mlcinp=f"f{i}.mlcinp")
          for i, (a, mu) in enumerate([(0, 100), (72.5, 50)])]
    F.write_mlcinfo(tmp_path / "p.mlcinfo", fl)
    got = F.read_mlcinfo(tmp_path / "p.mlcinfo")
    assert [(g["angle"], g["x1"], g["x2"], g["y1"], g["y2"], g["mu"], g["mlcinp"]) for g in got] == \
           [(f["angle"], f["x1"], f["x2"], f["y1"], f["y2"], f["mu"], f["mlcinp"]) for f in fl]


def test_ini_reader_rules(tmp_path):
    (tmp_path / "a.ini").write_text('[General]\nOutput Prefix = "V1"\n; comment\n[phantom]\nSource to isocenter = 100\n')
    ini = read_ini(tmp_path / "a.ini")
    assert ini["general"]["output prefix"] == "V1" and ini["phantom"]["source to isocenter"] == "100"


def test_plan_from_files_is_the_same_job(tmp_path, oracle):
    job = _job()
    plan = load_plan(_write_plan(tmp_path, job), seed=job.meta["seed"])
    pj = plan.job
    assert (plan.nx, plan.ny, plan.nz) == DIMS and pj.media == job.media and pj.histories == job.histories
    assert plan.output_base.endswith("out/T1") and plan.dose_unit == pytest.approx(1.6e-8)
    np.testing.assert_array_equal(pj.physics, job.physics)
    for k in ("voxel_med", "voxel_rhof", "density"):
        np.testing.assert_array_equal(pj.phantom[k], job.phantom[k])
    assert pj.phantom["other_med"] == job.phantom["other_med"]
    np.testing.assert_array_equal(pj.phsp, job.phsp)
    for a, b in zip(pj.fields, job.fields):
        for k in ("hist_begin", "hist_end", "nrepeat", "cos_angle", "sin_angle"):
            assert a[k] == b[k], k
        for k in ("endnode", "jawsGeomY", "jawsGeomX", "boundMinY", "boundMinX"):
            np.testing.assert_array_equal(a[k], b[k])
    ref, _ = oracle.run(job.physics, job.scene(), 0, job.histories)
    got, _ = oracle.run(pj.physics, pj.scene(), 0, pj.histories)
    assert ref.sum() > 0
    np.testing.assert_array_equal(got, ref)


def test_plan_rejects_unsupported_modules(tmp_path):
    job = _job()
    ini = _write_plan(tmp_path, job)
    txt = ini.read_text().replace("module Wedge = Off", "module Wedge = On")
    ini.write_text(txt)
    with pytest.raises(PlanError, match="Wedge"):
        load_plan(ini)


def test_plan_reads_the_relative_dose_comparison(tmp_path):
    job = _job()
    ini = _write_plan(tmp_path, job, extra="""
[Dose output]
relative dose = Yes
starting point = -1.0 0.5 -1.5
xyz dimensions = 9 1 7
3d voxel sizes = 0.25 0 0.5
PTW729/PTW1000 = PTW729
norm to Max/Center = Center
gamma index (mm,%) = 3 2
measured data = "meas.txt"
""")
    txt = ini.read_text().replace("isocenter location = 0 0 0", "isocenter location = 0.5 0 -0.25")
    ini.write_text(txt)
    rp = load_plan(ini).post["relative"]
    assert rp["start"] == pytest.approx([-0.5, 0.5, -1.75]) and rp["dims"] == [9, 1, 7]
    assert rp["array_type"] == 1 and rp["norm_type"] == 2
    assert rp["gamma_len_cm"] == pytest.approx(0.3) and rp["gamma_dos"] == pytest.approx(0.02)
    assert rp["measured"].endswith("meas.txt") and "data" in rp["measured"]
    ini.write_text(txt.replace("gamma index (mm,%) = 3 2\n", ""))
    with pytest.raises(PlanError, match="gamma index"):
        load_plan(ini)


def test_dose_file_layout(tmp_path):
    d = np.arange(24 * 24 * 12, dtype=np.float32)
    name = F.write_dose(str(tmp_path / "P"), d, 24, 24, 12)
    assert name.endswith("P_DoseResults_024x024x012.bin")
    np.testing.assert_array_equal(F.read_dose(name).reshape(-1), d)


@pytest.mark.gpu
def test_command_line_writes_the_dose_grid(tmp_path, oracle):
    from gegs_b200.__main__ import run_plan
    job = _job()
    ini = _write_plan(tmp_path, job, extra="""
[Interpolation]
do interpolate = Yes
starting point = -2.3 -2.3 -2.9
xyz dimensions = 60 60 20
3d voxel sizes = 0.08 0.08 0.3

[Dose output]
absolute dose = Yes
dose position = 0.1 0.2 0.3
dose measured = 0
relative dose = No
""")
    name = run_plan(str(ini), uncertainty_batches=4)
    plan = load_plan(ini)
    ref, _ = oracle.run(plan.job.physics, plan.job.scene(), 0, plan.job.histories)
    want = F.dose_from_energy(ref.astype(np.float64) * 2.0 ** -30, plan.job.voxel_mass(), plan.dose_unit)
    np.testing.assert_array_equal(F.read_dose(name).reshape(-1), want)
    log = (tmp_path / "out" / "T1_log.txt").read_text()
    assert "absolute dose at" in log
    sig = np.fromfile(tmp_path / "out" / "T1_uncertianty_024x024x012.bin", np.float32)
    dosed = want > 0
    # relative standard error of a mean of 4 non-negative batches: in (0, 1]
    # (1 when one batch holds all of a voxel's energy); NaN where no batch deposits
    assert np.isfinite(sig[dosed]).all() and (sig[dosed] > 0).all() and (sig[dosed] <= 1.0 + 1e-6).all()
    assert np.isnan(sig[~dosed]).all()
    from oracle.post_oracle import interp_dose as ref_interp
    grid = np.fromfile(tmp_path / "out" / "T1_Interpolate_060x060x020.bin", np.float32)
    assert grid[:3].view(np.int32).tolist() == [60, 60, 20]
    p = plan.job.phantom
    np.testing.assert_array_equal(grid[3:].reshape(20, 60, 60),
                                  ref_interp(want, p["x_bounds"], p["y_bounds"], p["z_bounds"],
                                             (-2.3, -2.3, -2.9), (0.08, 0.08, 0.3), (60, 60, 20)))


class _FakeEngine:
    """Tally of a history range: voxel v gets sum over h of ((3 h + v) mod 5) * 2^20."""
    nvox = 6

    def __init__(self):
        self.t = np.zeros(self.nvox, np.int64)

    def reset_tally(self):
        self.t[:] = 0

    def run(self, lo, hi):
        h = np.arange(lo, hi, dtype=np.int64)[:, None]
        self.t += (((3 * h + np.arange(self.nvox)) % 5) << 20).sum(axis=0)

    def tally(self):
        return self.t.copy()


def test_batch_uncertainty_splits_every_field_and_keeps_the_tally(tmp_path):
    from gegs_b200.__main__ import transport_in_batches
    fields = [dict(hist_begin=0, hist_end=100), dict(hist_begin=100, hist_end=250)]
    of = [1.0, 0.5]
    energy, sigma = transport_in_batches(_FakeEngine(), fields, of, 5)
    e = _FakeEngine()
    whole = np.zeros(6)
    batches = np.zeros((5, 6))
    for k, f in enumerate(fields):
        e.reset_tally(); e.run(f["hist_begin"], f["hist_end"]); whole += e.tally() * of[k]
        n = f["hist_end"] - f["hist_begin"]
        for b in range(5):
            e.reset_tally(); e.run(f["hist_begin"] + n * b // 5, f["hist_begin"] + n * (b + 1) // 5)
            batches[b] += e.tally() * of[k]
    np.testing.assert_array_equal(energy, whole)
    m = batches.mean(axis=0)
    want = np.sqrt(np.maximum((batches ** 2).mean(axis=0) - m * m, 0) / 4) / m
    np.testing.assert_allclose(sigma, want, rtol=1e-12)
    name = F.write_uncertainty(str(tmp_path / "U"), sigma.astype(np.float32), 1, 2, 3)
    assert name.endswith("U_uncertianty_001x002x003.bin")
    np.testing.assert_array_equal(np.fromfile(name, np.float32), sigma.astype(np.float32))


def test_reference_example_plans_parse():
    """The reference's own example plans (Test*.ini beside its sources) read
    with the package's INI rules: every section the reference reads is found,
    numbers come out as the reference's sscanf("%f") gives them, and the
    options this path refuses are recognised (CTcreate from DICOM)."""
    from gegs_b200.plan import _floats, _get, _on
    from oracle.refpin import REF_DIR
    plans = sorted(REF_DIR.glob("Test*.ini")) if REF_DIR.is_dir() else []
    if not plans:
        pytest.skip("the reference's example plans are not present")
    for path in plans:
        ini = read_ini(path)
        for sec in ("general", "data", "phase space", "secjaws", "mlc", "phantom"):
            assert sec in ini, (path.name, sec)
        h = _floats(_get(ini, "General", "histories", required=True), 1, "histories")[0]
        assert h == float(np.float32(h)) and h >= 1
        iso = _floats(_get(ini, "Phantom", "isocenter location", required=True), 3, "iso")
        assert all(v == float(np.float32(v)) for v in iso)
        sid = _floats(_get(ini, "Phantom", "source to isocenter", required=True), 1, "sid")[0]
        assert sid > 0
        z = _floats(_get(ini, "Phase space", "z position", required=True), 1, "z")[0]
        assert z == float(np.float32(z))
        assert "\\" in _get(ini, "Data", "data directory") or _get(ini, "Data", "data directory")
        if _on(_get(ini, "Dose output", "relative dose")):
            gl, gd = _floats(_get(ini, "Dose output", "gamma index (mm,%)", required=True), 2, "gamma")
            assert gl > 0 and gd > 0
        assert isinstance(_on(_get(ini, "CTcreate", "use ctcreate")), bool)
