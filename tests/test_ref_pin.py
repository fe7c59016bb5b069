"""The oracle pinned to the reference's own code.

``oracle/ref`` compiles the reference's device sources (geom.cu, utility.cu,
relax.cu and the ten stage kernels with their samplers) unmodified, as host
code, into ``oracle/_ref/libgegs_ref.so``; its ``curand_uniform`` replays the
uniforms the oracle drew for the same particle, and its transcendental calls
use the oracle's own log/exp/sincos (see oracle/ref/ref_math.h). The tests
here feed identical particle states to the reference's routines and to the
oracle's and require identical results, bit for bit:

* geometry -- howfar (region entered, step, leaf/bank/module state) and
  hownear of the phantom, the DYNVMLC and both secondary jaws, for every
  particle state that enters the photon and electron stages in runs of the
  full C1 (60^3), C2 (120^3) and C3 (256x256x120, five gantry angles, jaws and
  MLC) geometries, with the step the transport asks for and with short steps;
* one pass of each stage kernel -- photon step, Compton (with binding and
  Doppler), photo (with Sauter angle and relaxation), Rayleigh, pair, the
  PRESTA-I electron step (multiple scattering, energy loss, boundary
  crossing), Moller (with EII), brems, Bhabha, annihilation -- per particle:
  the number of uniforms used, every particle pushed and every escore call;
* the direction rotations uphi21/32/11.

The CUDA kernels equal the oracle bit for bit (tests/test_gpu_parity.py), so
these tests tie the GPU path to the reference's own routines. What they do not
pin: the reference's cuRAND XORWOW stream (replaced by per-particle Philox by
design) and the reference's CUDA math library (held fixed to the oracle's).

When the reference sources are not present and the harness was not built,
the live tests skip; ``test_oracle_matches_reference_fixtures`` then still
checks the oracle against outputs the harness recorded (tests/golden/,
written by tests/golden/make_ref_fixtures.py).
"""
import pathlib

import numpy as np
import pytest

import refpin_cases as RC

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


def _refpin():
    from oracle import oracle as O
    from oracle import refpin as R
    O.build()
    R.build()
    if not R.available():
        pytest.skip("reference harness not built (reference sources absent)")
    return R


@pytest.fixture(scope="module", params=["c1", "c2", "c3"])
def setup(request):
    R = _refpin()
    job = RC.job(request.param)
    sh = job.scene()
    pair = R.Pair(job.physics, sh)
    cap = pair.capture(0, job.histories, every=1, cap_n=60000)
    for s in range(10):
        cap[s]["hist"] = np.arange(len(cap[s]), dtype=np.uint32)
    return request.param, job, sh, pair, cap


def test_geometry_bit_exact(setup):
    name, job, sh, pair, cap = setup
    rng = np.random.default_rng(11)
    parts = np.concatenate([cap[0], cap[5]])
    assert len(parts) > 5000
    if name == "c3":
        assert set(np.unique(parts["module"])) >= {1, 2, 3, 6}       # jaws Y, jaws X, MLC, phantom
        assert len(np.unique(parts["field"])) == 5
    for t_in in (np.full(len(parts), 1e3, np.float32),
                 rng.exponential(0.3, len(parts)).astype(np.float32)):
        g = pair.geom(parts, t_in)
        a, b = g["ora"], g["ref"]
        for k in ("region", "t", "tperp"):
            bad = np.flatnonzero(a[k].view(np.uint32) != b[k].view(np.uint32))
            assert bad.size == 0, f"{name} {k}: {bad.size} of {len(parts)} differ, first {bad[:5]}"
        for k in ("leafIndex", "bank", "module", "region"):
            assert np.array_equal(a["particle"][k], b["particle"][k]), k


@pytest.mark.parametrize("stage", range(10), ids=RC.STAGES)
def test_stage_kernel_bit_exact(setup, stage):
    name, job, sh, pair, cap = setup
    parts = cap[stage][:4000]
    if len(parts) == 0:
        pytest.skip(f"no {RC.STAGES[stage]} events in the {name} capture")
    res = pair.stage(stage, parts)
    assert res["ref"]["err"] == 0, "the reference asked for more uniforms than the oracle drew"
    bad = RC.compare_stage(res)
    assert not bad, f"{name} {RC.STAGES[stage]}: {len(bad)} of {len(parts)} particles differ, first {bad[:5]}"


@pytest.mark.parametrize("stage", range(10), ids=RC.STAGES)
def test_stage_kernel_bit_exact_energy_sweep(setup, stage):
    name, job, sh, pair, cap = setup
    if name != "c3":
        pytest.skip("the sweep runs in the CT phantom (all five media)")
    parts = RC.stress(cap, job.physics)[stage]
    res = pair.stage(stage, parts)
    assert res["ref"]["err"] == 0
    bad = RC.compare_stage(res)
    assert not bad, f"{RC.STAGES[stage]} sweep: {len(bad)} of {len(parts)} differ, first {bad[:5]}"
    assert res["ora"]["on"].sum() + res["ora"]["dn"].sum() > 0


def test_uphi_bit_exact():
    R = _refpin()
    from oracle import oracle as O
    rng = np.random.default_rng(5)
    job = RC.W.config1(histories=10, n=8, voxel=4.0)
    pair = R.Pair(job.physics, job.scene())
    n = 3000
    cz = rng.uniform(-1, 1, n)
    ph = rng.uniform(0, 2 * np.pi, n)
    sz = np.sqrt(1 - cz * cz)
    base = np.zeros(n, R.PARTICLE)
    base["u"], base["v"], base["w"] = sz * np.cos(ph), sz * np.sin(ph), cz
    base["u"][:50] = 0.0
    base["v"][:50] = 0.0                                      # the small-polar-angle branch
    base["w"][:50] = np.where(np.arange(50) % 2, 1.0, -1.0)
    base["hist"] = np.arange(n)
    for i in range(n):
        ct = np.float32(rng.uniform(-1, 1))
        st = np.float32(np.sqrt(1 - ct * ct))
        th = np.float32(rng.uniform(0, np.pi))
        for which, a, b in ((21, ct, st), (32, ct, st), (11, th, 0.0)):
            (po, co), (pr, cr) = pair.uphi(which, a, b, base[i], cs=(0.6, 0.8))
            assert po.tobytes() == pr.tobytes(), (which, i)
            assert co.tobytes() == cr.tobytes(), (which, i)


def test_oracle_matches_reference_fixtures():
    """The oracle against outputs the reference harness recorded (no harness
    needed): a geometry set and every stage on the C3 geometry."""
    from oracle import oracle as O
    from oracle import refpin as R
    O.build()
    path = GOLDEN / "ref_pin_c3.npz"
    z = np.load(path)
    job = RC.job("c3")
    sh = job.scene()
    pair = R.OraclePair(job.physics, sh)
    g = pair.geom(z["geom_in"], z["geom_t_in"])
    assert np.array_equal(g["region"], z["geom_region"])
    assert g["t"].tobytes() == z["geom_t"].tobytes()
    assert g["tperp"].tobytes() == z["geom_tperp"].tobytes()
    assert g["particle"].tobytes() == z["geom_out"].tobytes()
    for s in range(10):
        key = f"s{s}_"
        if key + "in" not in z.files:
            continue
        o = pair.stage(s, z[key + "in"])
        assert np.array_equal(o["used"], z[key + "used"]), RC.STAGES[s]
        assert np.array_equal(o["on"], z[key + "on"]), RC.STAGES[s]
        assert np.array_equal(o["dn"], z[key + "dn"]), RC.STAGES[s]
        outs = np.concatenate([R.sort_by_stack(o["out"][i], o["on"][i]) for i in range(len(o["on"]))])
        assert outs.tobytes() == z[key + "out"].tobytes(), RC.STAGES[s]
        dreg = np.concatenate([o["dreg"][i, :o["dn"][i]] for i in range(len(o["dn"]))])
        de = np.concatenate([o["de"][i, :o["dn"][i]] for i in range(len(o["dn"]))])
        assert np.array_equal(dreg, z[key + "dreg"]), RC.STAGES[s]
        assert de.tobytes() == z[key + "de"].tobytes(), RC.STAGES[s]
