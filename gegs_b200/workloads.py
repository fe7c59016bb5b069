"""Seeded synthetic inputs for the five benchmark configurations.

The reference's own inputs (BEAMnrc phase spaces, egsphant phantoms, MLC plans,
PEGS4 data) are not available; these generators stand in for them with the
shapes, sizes and value distributions the configurations describe.  Every
generator takes a seed (default ``0x6E65 + config id``).

* C1  1.25 MeV parallel 10x10 cm photon beam on a 30 cm water cube, 60^3 voxels.
* C2  6 MV-like phase space (97 % photons, thick-target shape 0.1-6 MeV, mean
      ~1.8 MeV; 3 % electrons 0.2-4 MeV), point source, 10x10 cm at SSD 100,
      water/lung/water slab 3/10/17 cm, 120^3 voxels of 0.25 cm.
* C3  synthetic CT head (256x256x120 HU, 1x1x2.5 mm) through the reference's
      4-material CT ramp, 5 coplanar fields with jaws +-6 cm and a seeded MLC.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import geometry as G
from . import physics_data as PD
from .scene import (DEFAULT_REGION_FLAGS, PHSP_DTYPE, SceneHolder, VACUUM_MED)

SEED_BASE = 0x6E65
RM = PD.RM
LATCH_ELECTRON = 0x40000000


@dataclass
class Job:
    name: str
    media: list
    physics: np.ndarray
    phantom: dict
    beam: dict
    fields: list
    phsp: np.ndarray
    histories: int
    meta: dict = field(default_factory=dict)

    def scene(self, seed=None, hownear_region_offset=5):
        return SceneHolder(self.phantom, self.beam, self.fields, self.phsp,
                           seed=self.meta.get("seed", 0) if seed is None else seed,
                           hownear_region_offset=hownear_region_offset)

    def voxel_mass(self):
        """Voxel masses in g, float32, as the reference computes them from the
        egsphant (init.cu:1256-1271): (dx * dy) * dz in float, made positive,
        times the density; 0 becomes 1."""
        p = self.phantom
        dx, dy, dz = (np.diff(np.asarray(p[k], np.float32)) for k in ("x_bounds", "y_bounds", "z_bounds"))
        vol = np.abs((dx[None, None, :] * dy[None, :, None]) * dz[:, None, None])
        m = (vol.reshape(-1) * np.asarray(p["density"], np.float32).reshape(-1)).astype(np.float32)
        m[m == 0] = 1.0
        return m


def _uniform_bounds(n, size):
    return (np.arange(n + 1, dtype=np.float64) * size - n * size / 2).astype(np.float32)


def _fields_single(nhist, nrepeat=0, angle=0.0, **poly):
    c, s = G.gantry_cos_sin(angle)
    f = dict(cos_angle=c, sin_angle=s, hist_begin=0, hist_end=nhist, nrepeat=nrepeat)
    f.update(poly)
    return [f]


# ---------------------------------------------------------------------------
# phase-space generators
# ---------------------------------------------------------------------------
def thick_target_spectrum(rng, n, emin=0.1, emax=6.0, mean=1.8):
    """E^-a (Emax - E) on [emin, emax] with a tuned so the mean is `mean` (inverse CDF)."""
    grid = np.linspace(emin, emax, 20001)

    def mean_of(a):
        w = grid ** (-a) * (emax - grid)
        return np.trapezoid(grid * w, grid) / np.trapezoid(w, grid)

    lo, hi = -2.0, 3.0
    for _ in range(80):
        mid = 0.5 * (lo + hi)
        if mean_of(mid) > mean:
            lo = mid
        else:
            hi = mid
    a = 0.5 * (lo + hi)
    w = grid ** (-a) * (emax - grid)
    cdf = np.concatenate([[0.0], np.cumsum(0.5 * (w[1:] + w[:-1]) * np.diff(grid))])
    cdf /= cdf[-1]
    return np.interp(rng.random(n), cdf, grid), a


def point_source_phsp(rng, n, z_phsp, half_x, half_y, ssd=100.0, frac_e=0.03):
    """Records on the plane z=z_phsp from a point source at z=0 aimed uniformly
    into a [-half_x, half_x] x [-half_y, half_y] field at z=ssd."""
    rec = np.zeros(n, PHSP_DTYPE)
    is_e = rng.random(n) < frac_e
    e, _ = thick_target_spectrum(rng, n)
    ke = rng.uniform(0.2, 4.0, n)
    X = rng.uniform(-half_x, half_x, n)
    Y = rng.uniform(-half_y, half_y, n)
    norm = np.sqrt(X * X + Y * Y + ssd * ssd)
    rec["u"] = X / norm
    rec["v"] = Y / norm
    rec["x"] = X * z_phsp / ssd
    rec["y"] = Y * z_phsp / ssd
    rec["e"] = np.where(is_e, ke + RM, e)
    rec["latch"] = np.where(is_e, LATCH_ELECTRON, 0).astype(np.uint32)
    rec["wt"] = 1.0
    return rec


# ---------------------------------------------------------------------------
# configurations
# ---------------------------------------------------------------------------
MEDIA_BASE = ["H2O700ICRU", "AIR700ICRU", "W700ICRU"]


def config1(histories=1_000_000, seed=SEED_BASE + 1, n=60, voxel=0.5, nphsp=None):
    rng = np.random.default_rng(seed)
    media = list(MEDIA_BASE)
    phys = PD.build_block(media, mlc_media=["W700ICRU"])
    b = _uniform_bounds(n, voxel)
    nvox = n ** 3
    phantom = dict(x_bounds=b, y_bounds=b, z_bounds=b, voxel_med=np.zeros(nvox, np.uint16),
                   voxel_rhof=np.ones(nvox, np.float32), density=np.ones(nvox, np.float32),
                   other_med=[1, 2, 2, 1, 1], media=media)
    nphsp = nphsp or min(histories, 1_000_000)
    rec = np.zeros(nphsp, PHSP_DTYPE)
    rec["e"] = 1.25
    rec["x"] = rng.uniform(-5, 5, nphsp)
    rec["y"] = rng.uniform(-5, 5, nphsp)
    rec["wt"] = 1.0
    nrep = max(0, (histories - 1) // nphsp)
    beam = dict(change_xyz=True, source_to_isocenter=100.0, iso=(0.0, -15.0, 0.0), z_phsp=50.0,
                module_order=G.module_order(False, False))
    return Job("C1 water 60^3 1.25 MeV", media, phys, phantom, beam, _fields_single(histories, nrep), rec,
               histories, meta=dict(seed=seed, voxel=voxel, n=n))


def slab_phantom(n=120, voxel=0.25, layers=((3.0, "H2O700ICRU", 1.0), (10.0, "LUNG700ICRU", 0.26),
                                            (17.0, "H2O700ICRU", 1.0)), media=None):
    media = media or ["H2O700ICRU", "AIR700ICRU", "W700ICRU", "LUNG700ICRU"]
    b = _uniform_bounds(n, voxel)
    centers = 0.5 * (b[1:] + b[:-1]).astype(np.float64)
    depth = centers - b[0]                 # depth along patient y from the surface
    med_y = np.zeros(n, np.uint16)
    dens_y = np.zeros(n, np.float32)
    start = 0.0
    for thick, name, dens in layers:
        sel = (depth >= start) & (depth < start + thick)
        med_y[sel] = media.index(name)
        dens_y[sel] = dens
        start += thick
    med = np.broadcast_to(med_y[None, :, None], (n, n, n)).reshape(-1).copy()
    dens = np.broadcast_to(dens_y[None, :, None], (n, n, n)).reshape(-1).copy()
    rho = np.array([PD.MEDIA[m].rho for m in media], np.float32)
    rhof = (dens / rho[med]).astype(np.float32)
    return dict(x_bounds=b, y_bounds=b, z_bounds=b, voxel_med=med, voxel_rhof=rhof, density=dens,
                other_med=[1, 2, 2, 1, 1], media=media)


def config2(histories=100_000_000, seed=SEED_BASE + 2, nphsp=10_000_000, n=120):
    rng = np.random.default_rng(seed)
    media = ["H2O700ICRU", "AIR700ICRU", "W700ICRU", "LUNG700ICRU"]
    phys = PD.build_block(media, mlc_media=["W700ICRU"])
    phantom = slab_phantom(n=n, voxel=30.0 / n, media=media)
    nphsp = min(nphsp, histories)
    rec = point_source_phsp(rng, nphsp, z_phsp=50.0, half_x=5.0, half_y=5.0)
    nrep = max(0, (histories - 1) // nphsp)
    beam = dict(change_xyz=True, source_to_isocenter=100.0, iso=(0.0, -15.0, 0.0), z_phsp=50.0,
                module_order=G.module_order(False, False))
    return Job("C2 6MV-like slab 120^3", media, phys, phantom, beam, _fields_single(histories, nrep), rec,
               histories, meta=dict(seed=seed))


# ---- CT ramp (ctcreate.c:913-970, applied at :1057-1104) --------------------
CT_RAMP = [("AIR700ICRU", -974, 0.001, 0.044), ("LUNG700ICRU", -724, 0.044, 0.302),
           ("ICRUTISSUE700ICRU", 101, 0.302, 1.101), ("ICRPBONE700ICRU", 1976, 1.101, 2.088)]
CT_LOWER = -1024


def hu_to_material(hu, media):
    """HU -> (medium index into `media`, density), the reference's 4-material ramp."""
    hu = np.asarray(hu, np.float64)
    med = np.full(hu.shape, VACUUM_MED, np.uint16)
    dens = np.zeros(hu.shape, np.float64)
    hi = hu > CT_RAMP[-1][1]
    med[hi] = media.index(CT_RAMP[-1][0])
    dens[hi] = CT_RAMP[-1][3]
    lower = CT_LOWER
    done = (hu < CT_LOWER) | hi
    for name, ub, dlo, dhi in CT_RAMP:
        sel = (~done) & (hu <= ub)
        med[sel] = media.index(name)
        dens[sel] = dlo + (hu[sel] - lower) * (dhi - dlo) / (ub - lower)
        done |= sel
        lower = ub
    return med, dens.astype(np.float32)


def ct_head(rng, nx=256, ny=256, nz=120):
    """Seeded ellipsoid head: soft tissue, skull, brain, sinus air, N(0,20) noise."""
    x = (np.arange(nx) - nx / 2 + 0.5) * 0.1
    y = (np.arange(ny) - ny / 2 + 0.5) * 0.1
    z = (np.arange(nz) - nz / 2 + 0.5) * 0.25
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    hu = np.full(X.shape, -1000.0)

    def ell(cx, cy, cz, ax, ay, az):
        return ((X - cx) / ax) ** 2 + ((Y - cy) / ay) ** 2 + ((Z - cz) / az) ** 2 <= 1.0

    j = lambda s: rng.normal(0, s)
    hu[ell(j(0.2), j(0.2), 0, 9.0, 11.0, 13.0)] = 0.0           # soft tissue
    hu[ell(j(0.2), j(0.2), 0, 8.4, 10.4, 12.4)] = 1000.0        # skull
    hu[ell(j(0.2), j(0.2), 0, 7.8, 9.8, 11.8)] = 40.0           # brain
    for _ in range(2):                                           # sinuses
        hu[ell(rng.uniform(-2, 2), rng.uniform(6, 8), rng.uniform(-6, -2), 1.5, 1.0, 2.0)] = -1000.0
    hu += rng.normal(0.0, 20.0, hu.shape)
    return hu.astype(np.int16)


def mlc_tips(rng, half=6.0):
    """120 mlcinp positions: 40 central half-leaf pairs open inside +-half, the
    20 outer full-leaf pairs closed (positions in cm at the isocentre)."""
    pos = np.zeros(120, np.float32)
    for j in range(10, 50):
        a = rng.uniform(0.5, half)
        b = rng.uniform(0.5, half)
        pos[j] = a             # bank A (POS after the swap)
        pos[j + 60] = b        # bank B (NEG = -pos[j+60])
    return pos


def config3(histories=200_000_000, seed=SEED_BASE + 3, nphsp=10_000_000, dims=(256, 256, 120),
            angles=(0.0, 72.0, 144.0, 216.0, 288.0), jaw=6.0):
    rng = np.random.default_rng(seed)
    media = ["AIR700ICRU", "LUNG700ICRU", "ICRUTISSUE700ICRU", "ICRPBONE700ICRU", "W700ICRU"]
    phys = PD.build_block(media, mlc_media=["W700ICRU"])
    nx, ny, nz = dims
    hu = ct_head(rng, nx, ny, nz)
    med, dens = hu_to_material(hu.reshape(-1), media)
    rho = np.array([PD.MEDIA[m].rho for m in media] + [1.0], np.float32)
    mi = np.where(med == VACUUM_MED, len(media), med)
    rhof = np.where(dens == 0, 1.0, dens / rho[mi]).astype(np.float32)
    phantom = dict(x_bounds=_uniform_bounds(nx, 0.1), y_bounds=_uniform_bounds(ny, 0.1),
                   z_bounds=_uniform_bounds(nz, 0.25), voxel_med=med, voxel_rhof=rhof, density=dens,
                   other_med=[0, 4, 4, 0, 0], media=media, hu=hu)
    mlc = G.DynVMLC.synthetic()
    mg = mlc.build()
    jaws = G.SecJaws()
    sid = 100.0
    nphsp = min(nphsp, histories)
    z_phsp = 16.44
    rec = point_source_phsp(rng, nphsp, z_phsp=z_phsp, half_x=7.0, half_y=7.0)
    nf = len(angles)
    per = histories // nf
    fields = []
    for i, a in enumerate(angles):
        c, s = G.gantry_cos_sin(a)
        pos = mlc_tips(rng, half=jaw)
        f = dict(cos_angle=c, sin_angle=s, hist_begin=i * per, hist_end=(i + 1) * per if i < nf - 1 else histories,
                 nrepeat=max(0, (per - 1) // nphsp), leaf_pos=pos, angle=a, jaws=(-jaw, jaw, -jaw, jaw))
        f.update(G.secjaws_polygons(jaws, -jaw, jaw, -jaw, jaw, sid))
        f["endnode"] = G.leaf_endnodes(mg["crossYZ"], pos, mlc.zmin, mlc.zthick, sid)
        fields.append(f)
    beam = dict(change_xyz=True, source_to_isocenter=sid, iso=(0.0, 0.0, 0.0), z_phsp=z_phsp,
                module_order=G.module_order(True, True), mlc=mg)
    return Job("C3 CT head 5 fields", media, phys, phantom, beam, fields, rec, histories,
               meta=dict(seed=seed, mlc=mlc, jaws=jaws))


def ellipsoid_mask(job, center, axes):
    """Voxels of the phantom whose centres lie in the ellipsoid (cm, phantom frame)."""
    p = job.phantom
    cx = [(np.asarray(p[k][:-1], np.float64) + np.asarray(p[k][1:], np.float64)) / 2
          for k in ("x_bounds", "y_bounds", "z_bounds")]
    Z, Y, X = np.meshgrid(cx[2], cx[1], cx[0], indexing="ij")
    r = ((X - center[0]) / axes[0]) ** 2 + ((Y - center[1]) / axes[1]) ** 2 + ((Z - center[2]) / axes[2]) ** 2
    return (r <= 1.0).reshape(-1)


def config4(histories=50_000_000, seed=SEED_BASE + 4, nphsp=10_000_000, dims=(256, 256, 120), nb=20, bixel=0.5):
    """C4: the C3 plan with every field split into nb x nb beamlets of `bixel` cm at
    the isocentre (fluence weights 1 + U(0, 0.2)), a seeded ellipsoidal target
    (prescription 60 units) and organ (one-sided limit 20 units)."""
    job = config3(histories=histories, nphsp=nphsp, dims=dims, seed=seed)
    rng = np.random.default_rng(seed + 1000)
    nf = len(job.fields)
    weights = (1.0 + rng.uniform(0.0, 0.2, nf * nb * nb)).astype(np.float32)
    half = nb * bixel / 2
    job.beam["beamlets"] = dict(nx=nb, ny=nb, x0=-half, y0=-half, dx=bixel, dy=bixel, weights=weights)
    j = lambda s: rng.normal(0.0, s)
    job.meta["target"] = ellipsoid_mask(job, (j(0.3), j(0.3), j(0.5)), (2.5, 2.0, 3.0))
    job.meta["organ"] = ellipsoid_mask(job, (3.5 + j(0.3), 0.5 + j(0.3), j(0.5)), (1.0, 1.5, 2.0))
    job.name = "C4 CT head 5 fields, beamlet weights"
    return job


def config5(n_plans=32, seed=SEED_BASE + 5, hist_min=1_000_000, hist_max=100_000_000, nphsp=1_000_000,
            dims_min=64, dims_max=(256, 256, 128)):
    """C5: independent plans of mixed size for a serving-style batch. Phantom
    sizes from dims_min^3 to dims_max (log-uniform per axis), 1-7 fields,
    log-uniform history counts in [hist_min, hist_max]; even plans are the
    slab phantom, odd plans the synthetic CT head with a seeded MLC."""
    rng = np.random.default_rng(seed)
    jobs = []
    for k in range(n_plans):
        h = int(np.exp(rng.uniform(np.log(hist_min), np.log(hist_max))))
        d = [int(np.exp(rng.uniform(np.log(min(dims_min, m)), np.log(m)))) for m in dims_max]
        if k % 2 == 0:
            n = max(dims_min, min(d))
            job = config2(histories=h, seed=seed * 100 + k, nphsp=min(nphsp, h), n=n)
            desc = f"slab {n}^3, 1 field"
        else:
            nf = int(rng.integers(1, 8))
            angles = tuple(float(a) for a in np.linspace(0.0, 360.0, nf, endpoint=False))
            job = config3(histories=h, seed=seed * 100 + k, nphsp=min(nphsp, h), dims=tuple(d), angles=angles)
            desc = f"CT {d[0]}x{d[1]}x{d[2]}, {nf} fields"
        job.name = f"C5 plan {k}: {desc}, {h} histories"
        jobs.append(job)
    return jobs


CONFIGS = {1: config1, 2: config2, 3: config3, 4: config4, 5: config5}
