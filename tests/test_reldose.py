"""The relative-dose comparison (postprocess.relative_dose, the reference's
output_RelDos_II, output.c:596-778) against a second statement of it written
in plain C (tests/c/reldose.c), which gets C's float semantics for free: the
same result file, byte for byte, for seeded dose grids, comparison planes
along every axis pair, all three normalisations and both detector arrays.
The GPU test does the same for the file the command line writes from a
transported plan."""
import pathlib
import subprocess
from decimal import Decimal, localcontext

import numpy as np
import pytest

from gegs_b200 import postprocess as PP

ROOT = pathlib.Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def reldose(tmp_path_factory):
    exe = tmp_path_factory.mktemp("reldose") / "reldose"
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-o", str(exe), str(ROOT / "tests" / "c" / "reldose.c"), "-lm"],
                   check=True)
    return exe


def _hex(v):
    return float(np.float32(v)).hex()


def _run_c(exe, tmp, dose, xb, yb, zb, start, sizes, dims, meas_path, norm, array, len_cm, dos, iso):
    dose_f = tmp / "dose.bin"
    bnd_f = tmp / "bounds.bin"
    out = tmp / "c_out.txt"
    np.asarray(dose, np.float32).tofile(dose_f)
    np.concatenate([np.asarray(b, np.float32) for b in (xb, yb, zb)]).tofile(bnd_f)
    args = [str(exe), str(dose_f), str(bnd_f), str(len(xb) - 1), str(len(yb) - 1), str(len(zb) - 1),
            *map(_hex, start), *map(_hex, sizes), *map(str, dims), str(meas_path) if meas_path else "-",
            str(norm), str(array), _hex(len_cm), _hex(dos), *map(_hex, iso), str(out)]
    subprocess.run(args, check=True)
    return out.read_text()


def _python(dose, xb, yb, zb, start, sizes, dims, meas_path, norm, array, len_cm, dos, iso):
    n = int(np.prod(dims))
    meas = PP.read_measured(meas_path, n) if meas_path else None
    lines, _, _ = PP.relative_dose(dose, xb, yb, zb, start, sizes, dims, meas, norm, array, len_cm, dos, iso)
    return "\n".join(lines) + "\n"


def _grid(rng, n=(20, 18, 16), d=(0.2, 0.25, 0.3)):
    """A smooth dose with noise and a few empty voxels, and its boundaries."""
    nx, ny, nz = n
    xb = (np.arange(nx + 1) - nx / 2) * d[0]
    yb = (np.arange(ny + 1) - ny / 2) * d[1]
    zb = (np.arange(nz + 1) - nz / 2) * d[2]
    c = [(b[:-1] + b[1:]) / 2 for b in (xb, yb, zb)]
    Z, Y, X = np.meshgrid(c[2], c[1], c[0], indexing="ij")
    dose = np.exp(-(X ** 2 + Y ** 2) / 4.0) * (1.2 - 0.1 * Z) * (1 + 0.05 * rng.standard_normal(X.shape))
    dose[rng.random(X.shape) < 0.02] = 0.0
    return dose.astype(np.float32).reshape(-1), xb.astype(np.float32), yb.astype(np.float32), zb.astype(np.float32)


PLANES = [((-1.5, 0.0, -2.0), (0.25, 0.0, 0.3), (12, 1, 13)),     # x-z, the detector arrays' plane
          ((-1.5, -1.2, 0.3), (0.3, 0.2, 0.0), (10, 12, 1)),      # x-y
          ((0.1, -1.6, -1.9), (0.0, 0.35, 0.4), (1, 9, 10))]      # y-z


@pytest.mark.parametrize("norm", [0, 1, 2])
@pytest.mark.parametrize("array", [1, 2])
@pytest.mark.parametrize("plane", range(len(PLANES)))
def test_relative_dose_equals_c_statement(reldose, tmp_path, norm, array, plane):
    rng = np.random.default_rng(100 * norm + 10 * array + plane)
    dose, xb, yb, zb = _grid(rng)
    start, sizes, dims = PLANES[plane]
    n = int(np.prod(dims))
    calc = PP.sample_plane(dose, xb, yb, zb, start, sizes, dims)
    # measured data near the calculated dose (some points fail, some only pass
    # through a neighbour), in the unit each normalisation expects
    scale = 0.01 if norm == 0 else 3.7
    meas = calc * scale * (1 + 0.04 * rng.standard_normal(n))
    meas[rng.random(n) < 0.05] *= 1.3
    lines = [f"{float(v)!r}\t{int(rng.integers(0, 99))}" for v in meas]
    meas_path = tmp_path / "meas.txt"
    meas_path.write_text("\n".join(lines) + "\n")
    iso = (start[0] + sizes[0] * (dims[0] // 2), start[1] + sizes[1] * (dims[1] // 2), start[2] + sizes[2] * (dims[2] // 2))
    args = (dose, xb, yb, zb, start, sizes, dims, meas_path, norm, array, 0.3, 0.03, iso)
    want = _run_c(reldose, tmp_path, *args)
    got = _python(*args)
    assert got == want
    assert "points compared" in got.splitlines()[-1] and int(got.splitlines()[-1].split()[1]) > 0


def test_relative_dose_without_measured_data_equals_c_statement(reldose, tmp_path):
    dose, xb, yb, zb = _grid(np.random.default_rng(5))
    start, sizes, dims = PLANES[0]
    args = (dose, xb, yb, zb, start, sizes, dims, None, 1, 2, 0.3, 0.03, (0.0, 0.0, 0.0))
    assert _python(*args) == _run_c(reldose, tmp_path, *args)


def test_measured_values_round_once_to_float():
    # decimals just above and below the midpoint of two float32 neighbours:
    # rounding to double first lands on the midpoint, and the tie then goes
    # to the even neighbour, while C rounds once, to the nearer one
    for base in (1.0, 3.7, 1234.5, 1e-3):
        lo = np.float32(base)
        hi = np.nextafter(lo, np.float32(np.inf))
        with localcontext(prec=100):                          # exact: dyadic values have short decimals
            mid = Decimal(float(lo)) + (Decimal(float(hi)) - Decimal(float(lo))) / 2
            above, below = f"{mid + Decimal('1e-60')}", f"{mid - Decimal('1e-60')}"
        assert float(above) == float(mid) == float(below)     # the double rounding would land on the tie
        assert PP.strtof(above) == hi and PP.strtof(below) == lo
        even = lo if int(lo.view(np.uint32)) % 2 == 0 else hi
        assert PP.strtof(str(mid)) == even
    for s in ("0.1", "1e-3", "-2.5", "3.4028235e38", "7"):
        assert PP.strtof(s) == np.float32(float(s))
    assert PP.strtof("1e39") == np.float32(np.inf) and PP.strtof("-1e39") == np.float32(-np.inf)


@pytest.mark.gpu
def test_command_line_relative_dose_equals_c_statement(tmp_path, reldose):
    from gegs_b200 import io_formats as F
    from gegs_b200 import workloads as W
    from gegs_b200.__main__ import run_plan
    from gegs_b200.plan import load_plan
    from test_plan_io import _write_plan

    job = W.config3(histories=5 * 200000, nphsp=3000, dims=(24, 24, 12))
    per_field = job.histories // len(job.fields)
    for norm_name, norm, array_name, array in (("Max", 1, "PTW1000", 2), ("Center", 2, "PTW729", 1)):
        d = tmp_path / norm_name
        d.mkdir()
        ini = _write_plan(d, job, extra=f"""
[Dose output]
absolute dose = No
relative dose = Yes
starting point = -1.0 0.0 -1.2
xyz dimensions = 9 1 10
3d voxel sizes = 0.25 0 0.25
PTW729/PTW1000 = {array_name}
norm to Max/Center = {norm_name}
gamma index (mm,%) = 3 3
measured data = "meas.txt"
""", per_field=per_field)
        plan = load_plan(ini)
        p = plan.job.phantom
        rp = plan.post["relative"]
        name = run_plan(str(ini))
        dose = F.read_dose(name).reshape(-1)
        calc = PP.sample_plane(dose, p["x_bounds"], p["y_bounds"], p["z_bounds"], rp["start"], rp["sizes"], rp["dims"])
        assert (calc > 0).sum() > 60                                  # the plane has dose
        rng = np.random.default_rng(norm)
        meas = calc * (1 + 0.05 * rng.standard_normal(calc.size)) + 0.02 * calc.max()
        (d / "data" / "meas.txt").write_text("".join(f"{float(v)!r}\n" for v in meas))
        name = run_plan(str(ini))
        out = d / "out" / "T1_RelativeDose_009x001x010.txt"
        want = _run_c(reldose, d, F.read_dose(name).reshape(-1), p["x_bounds"], p["y_bounds"], p["z_bounds"],
                      rp["start"], rp["sizes"], rp["dims"], d / "data" / "meas.txt", norm, array,
                      rp["gamma_len_cm"], rp["gamma_dos"], rp["iso"])
        assert out.read_text() == want
        summary = want.splitlines()[-1]
        assert int(summary.split()[1]) > 0
        assert summary in (d / "out" / "T1_log.txt").read_text()
