"""The C/C++ host side of the drop-in path (include/gegs_plan.h): a plan in
the reference's input formats read by the library's C++ reader gives the same
scene, bit for bit, as the package's Python reader; the dose conversion and
the dose file match the CLI's; and a C program built here drives a whole plan
through the C ABI with no Python in the loop (GPU)."""
import ctypes as C
import pathlib
import subprocess

import numpy as np
import pytest

from gegs_b200 import io_formats as F
from gegs_b200 import physics_data as PD
from gegs_b200 import workloads as W
from gegs_b200.plan import load_plan
from gegs_b200.scene import PHSP_DTYPE, Field, Scene

from test_plan_io import _job, _write_plan

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _lib():
    from gegs_b200 import build as B
    B.build()
    L = C.CDLL(str(B.LIB))
    vp = C.c_void_p
    L.gegs_plan_load.argtypes = [C.c_char_p, C.c_char_p, C.c_uint64, C.POINTER(vp), C.c_char_p, C.c_size_t]
    L.gegs_plan_free.argtypes = [vp]
    L.gegs_plan_free.restype = None
    L.gegs_plan_scene.argtypes = [vp]
    L.gegs_plan_scene.restype = C.POINTER(Scene)
    L.gegs_plan_physics.argtypes = [vp]
    L.gegs_plan_physics.restype = vp
    for f in ("gegs_plan_histories", "gegs_plan_nvox"):
        getattr(L, f).argtypes = [vp]
        getattr(L, f).restype = C.c_uint64
    L.gegs_plan_dose_unit.argtypes = [vp]
    L.gegs_plan_dose_unit.restype = C.c_double
    L.gegs_plan_voxel_mass.argtypes = [vp, vp, C.c_uint64]
    L.gegs_plan_dose.argtypes = [vp, vp, vp, C.c_uint64]
    L.gegs_plan_write_dose.argtypes = [vp, vp, C.c_uint64, C.c_char_p, C.c_size_t]
    return L


@pytest.fixture(scope="module")
def plan_files(tmp_path_factory):
    d = tmp_path_factory.mktemp("cplan")
    ini = _write_plan(d, _job())
    plan = load_plan(ini)
    phys = d / "plan.physics"
    PD.write_physics_file(phys, plan.job.media, plan.job.physics)
    return ini, phys, plan


def _load(L, ini, phys, cap=0):
    h = C.c_void_p()
    msg = C.create_string_buffer(512)
    st = L.gegs_plan_load(str(ini).encode(), str(phys).encode(), cap, C.byref(h), msg, len(msg))
    return st, h, msg.value.decode()


def _arr(ptr, n, dtype):
    return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(np.ctypeslib.as_ctypes_type(dtype))), shape=(n,)).copy()


def test_cpp_plan_reader_gives_the_python_scene(plan_files):
    ini, phys, plan = plan_files
    L = _lib()
    st, h, msg = _load(L, ini, phys)
    assert st == 0, msg
    s = L.gegs_plan_scene(h).contents
    ref = plan.job.scene().scene
    for k, _ in Scene._fields_:
        if k in ("x_bounds", "y_bounds", "z_bounds", "voxel_med", "voxel_rhof", "fields", "phsp", "bl_weight"):
            continue
        a, b = getattr(s, k), getattr(ref, k)
        if isinstance(a, C.Array):
            assert bytes(a) == bytes(b), k
        else:
            assert a == b, k
    nvox = s.nx * s.ny * s.nz
    assert nvox == plan.nx * plan.ny * plan.nz
    for k, n, dt in (("x_bounds", s.nx + 1, np.float32), ("y_bounds", s.ny + 1, np.float32),
                     ("z_bounds", s.nz + 1, np.float32), ("voxel_med", nvox, np.uint16),
                     ("voxel_rhof", nvox, np.float32)):
        assert _arr(getattr(s, k), n, dt).tobytes() == _arr(getattr(ref, k), n, dt).tobytes(), k
    assert s.nfields == ref.nfields == len(plan.job.fields)
    for i in range(s.nfields):
        assert bytes(s.fields[i]) == bytes(ref.fields[i]), f"field {i}"
    got = np.ctypeslib.as_array(C.cast(s.phsp, C.POINTER(C.c_uint8)), shape=(s.nphsp * 28,))
    assert got.tobytes() == np.ascontiguousarray(plan.job.phsp, PHSP_DTYPE).tobytes()
    blk = np.ascontiguousarray(plan.job.physics)
    got_p = np.ctypeslib.as_array(C.cast(L.gegs_plan_physics(h), C.POINTER(C.c_uint8)), shape=(blk.nbytes,))
    assert got_p.tobytes() == blk.tobytes()
    assert L.gegs_plan_histories(h) == plan.job.histories
    assert L.gegs_plan_dose_unit(h) == plan.dose_unit
    L.gegs_plan_free(h)


def test_cpp_dose_conversion_and_file_match_the_cli(plan_files, tmp_path):
    ini, phys, plan = plan_files
    L = _lib()
    st, h, msg = _load(L, ini, phys)
    assert st == 0, msg
    nvox = int(L.gegs_plan_nvox(h))
    mass = np.zeros(nvox, np.float32)
    assert L.gegs_plan_voxel_mass(h, mass.ctypes.data, nvox) == 0
    assert mass.tobytes() == plan.job.voxel_mass().tobytes()
    tally = np.random.default_rng(3).integers(0, 1 << 40, nvox).astype(np.int64)
    dose = np.zeros(nvox, np.float32)
    assert L.gegs_plan_dose(h, tally.ctypes.data, dose.ctypes.data, nvox) == 0
    ref = F.dose_from_energy(tally.astype(np.float64) * (2.0 ** -30), plan.job.voxel_mass(), plan.dose_unit)
    assert dose.tobytes() == ref.tobytes()
    path = C.create_string_buffer(1024)
    assert L.gegs_plan_write_dose(h, dose.ctypes.data, nvox, path, len(path)) == 0
    name = pathlib.Path(path.value.decode())
    assert name.name == f"T1_DoseResults_{plan.nx:03d}x{plan.ny:03d}x{plan.nz:03d}.bin"
    assert name.read_bytes() == ref.tobytes()
    L.gegs_plan_free(h)


def test_cpp_plan_reader_errors(plan_files, tmp_path):
    ini, phys, plan = plan_files
    L = _lib()
    bad = ini.parent / "no_hist.ini"
    bad.write_text("\n".join(l for l in ini.read_text().split("\n") if not l.strip().startswith("histories ")))
    st, h, msg = _load(L, bad, phys)
    assert st == 1 and "histories" in msg
    other = tmp_path / "other.physics"
    PD.write_physics_file(other, ["H2O700ICRU"], PD.build_block(["H2O700ICRU"]))
    st, h, msg = _load(L, ini, other)
    assert st == 1 and "media" in msg
    st, h, msg = _load(L, ini, tmp_path / "missing.physics")
    assert st == 1 and "cannot open" in msg


def _build_c_program(tmp_path):
    from gegs_b200 import build as B
    B.build()
    exe = tmp_path / "plan_dose"
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I", str(ROOT / "include"), str(ROOT / "tests" / "c" / "plan_dose.c"),
                    "-o", str(exe), "-L", str(B.LIB.parent), "-lgegs_b200", f"-Wl,-rpath,{B.LIB.parent}"], check=True)
    return exe


def test_c_program_builds_against_the_headers(tmp_path):
    exe = _build_c_program(tmp_path)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 2 and "usage" in out.stderr


@pytest.mark.gpu
def test_c_program_reproduces_the_cli_dose_file(plan_files, tmp_path):
    """No Python in the loop: the C program's dose file equals the CLI's, byte for byte."""
    from gegs_b200.__main__ import run_plan
    ini, phys, plan = plan_files
    exe = _build_c_program(tmp_path)
    out = subprocess.run([str(exe), str(ini), str(phys)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    c_file = pathlib.Path(out.stdout.strip())
    c_bytes = c_file.read_bytes()
    c_file.unlink()
    cli_file = pathlib.Path(run_plan(str(ini), out=open("/dev/null", "w")))
    assert cli_file == c_file
    assert cli_file.read_bytes() == c_bytes
    assert np.frombuffer(c_bytes, np.float32).sum() > 0
