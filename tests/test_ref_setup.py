"""The plan readers pinned to the reference's own host set-up.

``oracle/ref`` also compiles the reference's set-up routines from init.cu
(init_phantom_and_MLC with read_egsinp_secjaws, read_egsinp and leaf_end;
read_mlcinp; setup_secjaws and init_leaf_pos per field) and the lines of
runSimulation that turn a field's angle into the uploaded cosine and sine
(CUDA_EGS.cu:420-422). The tests run them on the same plan files the
package's readers get, and require the same numbers, bit for bit, from the
Python reader (gegs_b200.plan) and from the C++ reader (include/gegs_plan.h):

* the phantom: voxel counts, boundaries, medium per voxel, densities, voxel
  masses, the media list and the beam-line media;
* the DYNVMLC: its scalar constants, the leaf cross sections crossXZ (the
  entries the reference sets), the XZ and YZ boundaries and the leaf-end
  outline;
* per field: the mlcinfo numbers, the leaf positions, the output factor, the
  jaw polygons, the leaf-end polygons of all 60 pairs, and the gantry angle in
  radians.

The gantry cosine and sine: the reference takes cos and sin of that float
with its platform's library; the package gives the correctly rounded values,
checked here against a 200-bit evaluation.
"""
import ctypes as C
import pathlib

import numpy as np
import pytest

from gegs_b200 import physics_data as PD
from gegs_b200 import workloads as W
from gegs_b200.plan import load_plan
from gegs_b200.scene import Scene

from test_plan_io import _write_plan

OFAC_TEXT = "Output factors of the machine\n5\n4.0 0.951\n6.5 0.9732\n10.0 1.0\n15.0 1.0213\n20.0 1.0337\n"


def _setup_lib():
    from oracle import oracle as O
    from oracle import refpin as R
    O.build()
    R.build()
    if not R.available():
        pytest.skip("reference harness not built (reference sources absent)")
    return R


def _job(seed, angles, jaws, dims=(24, 24, 12)):
    job = W.config3(histories=5 * 200, nphsp=500, dims=dims)       # five fields
    rng = np.random.default_rng(seed)
    for f, a, jw in zip(job.fields, angles, jaws):
        f["angle"] = a
        f["jaws"] = jw
        pos = np.asarray(f["leaf_pos"], np.float32).copy()
        pos += rng.uniform(-0.8, 0.8, pos.size).astype(np.float32)     # leaf tips off the grid
        pos[rng.integers(0, 120, 6)] = -pos[rng.integers(0, 120, 6)]   # and some closed pairs
        f["leaf_pos"] = pos
    return job


def _write(tmp, job, ofac):
    extra = '[Output factor]\nuse output factor = Yes\noutput factor file = "ofac.txt"\n' if ofac else ""
    ini = _write_plan(tmp, job, extra=extra, per_field=200)
    if ofac:
        (tmp / "data" / "ofac.txt").write_text(OFAC_TEXT)
    return ini


def _cpp_scene(ini, plan, tmp):
    from gegs_b200 import build as B
    B.build()
    L = C.CDLL(str(B.LIB))
    vp = C.c_void_p
    L.gegs_plan_load.argtypes = [C.c_char_p, C.c_char_p, C.c_uint64, C.POINTER(vp), C.c_char_p, C.c_size_t]
    L.gegs_plan_scene.argtypes = [vp]
    L.gegs_plan_scene.restype = C.POINTER(Scene)
    L.gegs_plan_voxel_mass.argtypes = [vp, vp, C.c_uint64]
    L.gegs_plan_output_factor.argtypes = [vp, C.c_int32]
    L.gegs_plan_output_factor.restype = C.c_double
    phys = tmp / "plan.physics"
    PD.write_physics_file(phys, plan.job.media, plan.job.physics)
    h = vp()
    msg = C.create_string_buffer(512)
    assert L.gegs_plan_load(str(ini).encode(), str(phys).encode(), 0, C.byref(h), msg, len(msg)) == 0, msg.value
    nvox = plan.nx * plan.ny * plan.nz
    mass = np.zeros(nvox, np.float32)
    assert L.gegs_plan_voxel_mass(h, mass.ctypes.data, nvox) == 0
    ofac = [L.gegs_plan_output_factor(h, i) for i in range(len(plan.job.fields))]
    return L, h, L.gegs_plan_scene(h).contents, mass, ofac


def _crossxz_set_by_reference():
    """The crossXZ entries read_egsinp writes (init.cu:461-538); the rest of
    its malloc'd array stays unset."""
    m = np.zeros((960, 2), bool)
    for i in range(60):
        m[i * 16:i * 16 + 15] = True
    for k in (15, 31, 47, 79, 95):
        m[k] = True
    m[63, 1] = True
    m[111, 0] = True
    return m


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _check(S, plan, scene, mass, ofac, ofac_on):
    p = plan.job.phantom
    assert S.get("dims", np.int32).tolist() == [plan.nx, plan.ny, plan.nz]
    for k in ("x_bounds", "y_bounds", "z_bounds"):
        assert np.array_equal(_bits(S.get(k, np.float32)), _bits(p[k])), k
    assert np.array_equal(S.get("media_index", np.int32) - 1, np.asarray(p["voxel_med"], np.int32))
    assert np.array_equal(_bits(S.get("density", np.float32)), _bits(p["density"]))
    assert np.array_equal(_bits(S.get("voxel_mass", np.float32)), _bits(mass))
    assert S.get("media", None).decode().split("\n")[:-1] == list(plan.job.media)
    assert S.get("other_med", np.int32).tolist() == list(scene.other_med)

    mlc = S.get("mlc", np.float32)
    ours = [scene.mlc_rmax, scene.mlc_zmin, scene.mlc_zthick, scene.mlc_x_start, scene.mlc_x_end, scene.mlc_x_mid_1,
            scene.mlc_x_mid_2, scene.mlc_air_gap, scene.mlc_wl_full, scene.mlc_wl_target, scene.mlc_wl_isocenter,
            scene.mlc_wt]
    assert np.array_equal(_bits(mlc), _bits(ours))
    mask = _crossxz_set_by_reference()
    ref_x = S.get("crossXZ", np.float32).reshape(960, 2)
    our_x = np.ctypeslib.as_array(scene.crossXZ)
    bad = np.argwhere((_bits(ref_x) != _bits(our_x)) & mask)
    assert bad.size == 0, f"crossXZ differs at {bad[:5].tolist()}: {ref_x[tuple(bad[0])]} vs {our_x[tuple(bad[0])]}"
    for k in ("boundaryXZ", "boundaryYZ"):
        assert np.array_equal(_bits(S.get(k, np.float32)), _bits(np.ctypeslib.as_array(getattr(scene, k))).reshape(-1)), k
    assert np.array_equal(_bits(S.get("crossYZ", np.float32)), _bits(plan.job.beam["mlc"]["crossYZ"]).reshape(-1))

    assert S.nfields == scene.nfields == len(plan.job.fields)
    for i in range(S.nfields):
        F = S.field(i)
        pf, sf = plan.job.fields[i], scene.fields[i]
        assert _bits([F["angle"], F["x1"], F["x2"], F["y1"], F["y2"]]).tolist() == \
            _bits([pf["angle"], *pf["jaws"]]).tolist(), f"field {i} numbers"
        assert np.array_equal(_bits(S.get("pos", np.float32, i)), _bits(pf["leaf_pos"])), f"field {i} leaves"
        if ofac_on:         # otherwise the reference never sets nor uses it (CUDA_EGS.cu:1719-1729)
            assert _bits(F["output_factor"]) == _bits(ofac[i]), f"field {i} output factor"
        jaws = S.get("jaws", np.float32, i)
        ours = np.concatenate([np.ctypeslib.as_array(getattr(sf, k)).reshape(-1) for k in
                               ("boundMinY", "boundMinX", "boundMaxY", "boundMaxX", "jawsGeomY", "jawsGeomX")])
        assert np.array_equal(_bits(jaws), _bits(ours)), f"field {i} jaws"
        ref_e = S.get("endnode", np.float32, i)
        our_e = np.ctypeslib.as_array(sf.endnode).reshape(-1)
        bad = np.flatnonzero(_bits(ref_e) != _bits(our_e))
        assert bad.size == 0, f"field {i} endnode differs at {bad[:5]}"
        _check_gantry(F["angle_rad"], sf.cos_angle, sf.sin_angle)


def _check_gantry(a, c, s):
    mpmath = pytest.importorskip("mpmath")
    with mpmath.workprec(200):
        x = mpmath.mpf(float(a))
        for got, want in ((c, mpmath.cos(x)), (s, mpmath.sin(x))):
            f = np.float32(got)
            lo, hi = np.nextafter(f, np.float32(-np.inf)), np.nextafter(f, np.float32(np.inf))
            # correctly rounded: the true value is nearer to f than to either neighbour
            assert abs(want - mpmath.mpf(float(f))) <= abs(want - mpmath.mpf(float(lo)))
            assert abs(want - mpmath.mpf(float(f))) <= abs(want - mpmath.mpf(float(hi)))


SETUP_NAMES = ("dims", "x_bounds", "y_bounds", "z_bounds", "media_index", "density", "voxel_mass", "other_med",
               "mlc", "crossXZ", "boundaryXZ", "boundaryYZ", "crossYZ")
FIELD_NAMES = ("field", "pos", "jaws", "endnode")


def setup_arrays(S):
    """Every result of a reference set-up run, as arrays (for the fixtures)."""
    out = {n: S.get(n, np.uint8) for n in SETUP_NAMES}
    out["media"] = np.frombuffer(S.get("media", None), np.uint8)
    for i in range(S.nfields):
        for n in FIELD_NAMES:
            out[f"f{i}_{n}"] = S.get(n, np.uint8, i)
    return out


class FixtureSetup:
    """The recorded results of a reference set-up run, read like refpin.Setup."""

    def __init__(self, z, case):
        self.z, self.case = z, case
        self.nfields = sum(1 for k in z.files if k.startswith(case + "/f") and k.endswith("_field"))

    def get(self, name, dtype, field=-1):
        key = f"{self.case}/{name}" if field < 0 else f"{self.case}/f{field}_{name}"
        raw = self.z[key].tobytes()
        return raw if dtype is None else np.frombuffer(raw, dtype).copy()

    def field(self, f):
        from oracle.refpin import Setup
        return dict(zip(Setup.FIELD, self.get("field", np.float32, f)))


def case_plan(tmp, case):
    c = CASES[case]
    job = _job(c["seed"], c["angles"], c["jaws"])
    return _write(tmp, job, c["ofac"]), c


def run_reference(R, tmp, c):
    d = tmp / "data"
    return R.Setup(d / "head.egsphant", d / "VarianMLC.egsinp", d / "VarianMLC.egsinp", d / "plan.mlcinfo", d,
                   100.0, "AIR700ICRU", output_factor_file=(d / "ofac.txt") if c["ofac"] else None)


CASES = {
    "five-field": dict(seed=1, angles=[0.0, 72.0, 144.0, 216.0, 288.0],
                       jaws=[(-6.0, 6.0, -6.0, 6.0)] * 5, ofac=False),
    "odd-angles-and-jaws": dict(seed=2, angles=[13.7, 95.25, 181.1, 266.66, 359.9],
                                # the second field is smaller than the output-factor table's first size
                                jaws=[(-4.37, 5.1, -3.33, 7.05), (-0.8, 0.9, -0.7, 0.95), (-0.8, 8.45, -6.6, 1.25),
                                      (-5.55, 5.55, -7.45, 4.4), (-2.05, 3.3, -8.8, 8.15)], ofac=True),
}


def _check_readers(S, ini, plan, c, tmp_path):
    # the Python reader
    _check(S, plan, plan.job.scene().scene, plan.job.voxel_mass(), plan.field_output_factors, c["ofac"])
    # the C++ reader
    L, h, scene, mass, ofac = _cpp_scene(ini, plan, tmp_path)
    _check(S, plan, scene, mass, ofac, c["ofac"])
    if c["ofac"]:
        assert 0.0 in plan.field_output_factors and any(of not in (0.0, 1.0) for of in plan.field_output_factors)


@pytest.mark.parametrize("case", sorted(CASES))
def test_readers_give_the_reference_set_up(tmp_path, case):
    R = _setup_lib()
    ini, c = case_plan(tmp_path, case)
    _check_readers(run_reference(R, tmp_path, c), ini, load_plan(ini), c, tmp_path)


@pytest.mark.parametrize("case", sorted(CASES))
def test_readers_match_the_recorded_reference_set_up(tmp_path, case):
    """The same check against the reference's results recorded in
    tests/golden/ref_setup.npz (tests/golden/make_ref_fixtures.py), for
    machines without the reference sources."""
    z = np.load(pathlib.Path(__file__).resolve().parent / "golden" / "ref_setup.npz")
    ini, c = case_plan(tmp_path, case)
    _check_readers(FixtureSetup(z, case), ini, load_plan(ini), c, tmp_path)


def test_leaf_end_outline_is_the_reference_table():
    """Whatever the leaf radius in the input, the outline is the reference's
    fixed table (leaf_end, init.cu:256-343), so the shape of a closed leaf pair
    does not change with it."""
    from gegs_b200 import geometry as G
    m = G.DynVMLC.synthetic()
    a = m.cross_yz()
    m.rad_end = 3.0
    assert np.array_equal(_bits(a), _bits(m.cross_yz()))
    assert a[2, 1] == np.float32(m.zmin) and a[9, 0] == 0.0 and a[24, 0] == 0.0     # bottom of bank A, both centres
