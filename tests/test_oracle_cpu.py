"""CPU checks of the oracle and of the host logic (no GPU needed)."""
import ctypes as C
import math

import numpy as np
import pytest

from gegs_b200 import physics_layout as L
from gegs_b200 import scene as S
from gegs_b200 import workloads as W


def test_header_matches_layout():
    from pathlib import Path
    hdr = Path(__file__).resolve().parents[1] / "include" / "gegs_physics.h"
    assert hdr.read_text() == L.render_header()


def test_struct_sizes(oracle):
    lib = oracle.lib()
    assert lib.ora_sizeof_physics() == L.dtype().itemsize
    assert lib.ora_sizeof_scene() == C.sizeof(S.Scene)
    assert lib.ora_sizeof_field() == C.sizeof(S.Field)


def test_philox_known_answers(oracle):
    """Philox4x32-10 known-answer vectors (Random123 kat_vectors)."""
    lib = oracle.lib()
    cases = [
        ((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
        ((0xffffffff,) * 4, (0xffffffff, 0xffffffff), (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
        ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
         (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
    ]
    for ctr, key, want in cases:
        got = tuple(lib.ora_philox(*ctr, *key, lane) for lane in range(4))
        assert got == want


def test_log_exp_sincos_accuracy(oracle):
    lib = oracle.lib()
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.uniform(1e-7, 1, 2000), rng.uniform(1, 1e4, 2000),
                         [5.96e-8, 1.0, 2.0, 0.5, 1e-30, 3e38]]).astype(np.float32)
    for x in xs:
        got = lib.ora_log(float(x))
        want = math.log(float(x))
        assert abs(got - want) <= 2.5 * np.spacing(np.float32(abs(want))) + 1e-37, (x, got, want)
    for x in np.concatenate([rng.uniform(-80, 80, 3000), [0.0, -1e-8, 1e-8, 88.0, -87.0]]).astype(np.float32):
        got = lib.ora_exp(float(x))
        want = math.exp(float(x))
        assert abs(got - want) <= 2.5 * np.spacing(np.float32(want)), (x, got, want)
    s, c = C.c_float(), C.c_float()
    for t in rng.uniform(0, 1, 3000).astype(np.float32):
        lib.ora_sincos_turns(float(t), C.byref(s), C.byref(c))
        a = 2 * math.pi * float(t)
        assert abs(s.value - math.sin(a)) < 3e-7 and abs(c.value - math.cos(a)) < 3e-7


def test_c1_energy_conservation_and_determinism(oracle):
    job = W.config1(histories=4000, n=30, voxel=1.0)
    sh = job.scene()
    t1, s1 = oracle.run(job.physics, sh, 0, job.histories, threads=4)
    t2, s2 = oracle.run(job.physics, sh, 0, job.histories, threads=1)
    assert np.array_equal(t1, t2), "oracle result depends on the thread count"
    total = t1.sum() / 2 ** 30 + s1["e_escaped"]
    assert abs(total - 1.25 * job.histories) < 1e-3
    assert s1["error"] == 0


def test_c1_depth_dose_shape(oracle):
    job = W.config1(histories=20000, n=30, voxel=1.0)
    sh = job.scene()
    t, _ = oracle.run(job.physics, sh, 0, job.histories)
    d = t.reshape(30, 30, 30).sum(axis=(0, 2)) / 2 ** 30
    peak = int(np.argmax(d))
    assert peak <= 4, "1.25 MeV build-up peak expected within the first few cm"
    assert d[25] < d[peak] * 0.7, "dose must fall with depth"


def test_c3_beamline_runs_and_conserves(oracle):
    job = W.config3(histories=4000, nphsp=4000, dims=(48, 48, 20))
    sh = job.scene()
    t, s = oracle.run(job.physics, sh, 0, job.histories)
    assert s["error"] == 0
    assert t.sum() > 0
    # every primary is either transported through the head or discarded at the jaws
    assert s["counts"][0] >= 0.9 * job.histories


def test_ct_ramp_matches_reference_table():
    media = ["AIR700ICRU", "LUNG700ICRU", "ICRUTISSUE700ICRU", "ICRPBONE700ICRU"]
    med, dens = W.hu_to_material(np.array([-1100, -1024, -1000, -974, -800, -724, 0, 101, 1000, 1976, 3000]), media)
    assert med[0] == S.VACUUM_MED and dens[0] == 0
    assert [int(m) for m in med[1:]] == [0, 0, 0, 1, 1, 2, 2, 3, 3, 3]
    assert dens[1] == pytest.approx(0.001) and dens[3] == pytest.approx(0.044)
    assert dens[5] == pytest.approx(0.302) and dens[7] == pytest.approx(1.101)
    assert dens[9] == pytest.approx(2.088) and dens[10] == pytest.approx(2.088)


def test_thick_target_spectrum_mean():
    rng = np.random.default_rng(3)
    e, a = W.thick_target_spectrum(rng, 200000)
    assert e.min() >= 0.1 and e.max() <= 6.0
    assert abs(e.mean() - 1.8) < 0.02
