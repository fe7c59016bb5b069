"""Inputs shared by the reference-pinning tests and the script that writes
their golden fixtures: particle states captured as they enter each stage in
oracle runs of the three geometries (full size), plus stress states that
sweep each stage's energy range in every medium of the CT phantom.

Test infrastructure only."""
from __future__ import annotations

import numpy as np

from gegs_b200 import workloads as W

STAGES = ["photon", "compton", "photo", "rayleigh", "pair", "electron", "moller", "brems", "bhabha", "annih"]
M_PHANTOM = 6


def job(name):
    """The three configurations at their full geometry (the history counts only
    size the capture runs)."""
    if name == "c1":
        return W.config1(histories=20000)                       # 60^3 water, 0.5 cm
    if name == "c2":
        return W.config2(histories=20000, nphsp=20000)          # 120^3 slab, 0.25 cm
    if name == "c3":
        return W.config3(histories=20000, nphsp=20000)          # 256x256x120 CT, 5 fields, jaws + MLC
    raise ValueError(name)


def stress(captured, physics, seed=7, n=400):
    """Per stage: phantom particles of the capture with energies swept over the
    range that stage sees, log-uniform, and fresh random directions; charge
    and sign as the stage needs (electron-side stages alternate e-/e+ where
    both apply). Positions, regions and media stay those of real particles."""
    rng = np.random.default_rng(seed)
    rm = float(physics["rm"])
    base = np.concatenate([captured[s] for s in range(10)])
    base = base[base["module"] == M_PHANTOM]
    out = {}
    # (low, high) total energy in MeV; charge pattern
    spec = {0: (0.0105, 19.9, 0), 1: (0.0105, 19.9, 0), 2: (0.0105, 1.0, 0), 3: (0.0105, 1.0, 0),
            4: (1.03, 19.9, 0), 5: (0.72, 20.4, "pm"), 6: (1.9, 20.4, -1), 7: (0.72, 20.4, "pm"),
            8: (1.9, 20.4, 1), 9: (0.72, 20.4, 1)}
    for s, (lo, hi, q) in spec.items():
        pick = base[rng.integers(0, len(base), n)].copy()
        pick["e"] = np.exp(rng.uniform(np.log(lo), np.log(hi), n)).astype(np.float32)
        cz = rng.uniform(-1.0, 1.0, n)
        ph = rng.uniform(0.0, 2.0 * np.pi, n)
        sz = np.sqrt(1.0 - cz * cz)
        d = np.stack([sz * np.cos(ph), sz * np.sin(ph), cz], 1).astype(np.float32)
        d /= np.linalg.norm(d, axis=1, keepdims=True).astype(np.float32)
        pick["u"], pick["v"], pick["w"] = d[:, 0], d[:, 1], d[:, 2]
        if q == "pm":
            pick["charge"] = np.where(np.arange(n) % 2 == 0, -1, 1)
        else:
            pick["charge"] = q
        pick["status"] = s
        pick["hist"] = np.arange(n, dtype=np.uint32) + 1000000 * (s + 1)
        pick["dnear"] = 0.0
        out[s] = pick
    return out


def compare_stage(res):
    """Indices of particles whose outputs differ between oracle and reference:
    uniforms used, pushed particles (per stack, in push order) and escore calls."""
    from oracle import refpin as R
    a, b = res["ora"], res["ref"]
    bad = []
    for i in range(len(a["on"])):
        if a["used"][i] != b["used"][i] or a["on"][i] != b["on"][i] or a["dn"][i] != b["dn"][i]:
            bad.append(i)
            continue
        oa = R.sort_by_stack(a["out"][i], a["on"][i])
        ob = R.sort_by_stack(b["out"][i], b["on"][i])
        k = int(a["dn"][i])
        if (oa.tobytes() != ob.tobytes() or a["dreg"][i, :k].tobytes() != b["dreg"][i, :k].tobytes()
                or a["de"][i, :k].tobytes() != b["de"][i, :k].tobytes()):
            bad.append(i)
    return bad
