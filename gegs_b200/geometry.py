"""Beam-line geometry set-up: DYNVMLC leaf cross sections, leaf-end polygons,
secondary-jaw polygons and patient placement.

Restates the reference's host set-up code:

* leaf vertex construction ``Leaf::VerCal_full/target/isocenter``
  (read_egsinp.h:40-88) and the crossXZ / boundary arrays (init.cu:345-611);
* the leaf-end (YZ) outline ``leaf_end`` (init.cu:256-343);
* per-field jaw polygons ``setup_secjaws`` (init.cu:1504-1592);
* per-field leaf-end polygons ``init_leaf_pos`` (init.cu:1594-1662), with the
  reference's bank swap (``INVERSE_MLC_Bank_AB``, CUDA_EGS.h:27);
* gantry cos/sin as uploaded by the reference (CUDA_EGS.cu:426-434);
* the module order (CUDA_EGS.cu:1277-1305).

The reference's leaf-end outline is a hard-coded table of 15 points; here the
outline is computed from a circular leaf end of radius ``rad_end`` (the
``rad_end`` value the DYNVMLC input carries), sampled at the same 15 depths.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .scene import M_PHANTOM, M_SECJAWX, M_SECJAWY, M_VARMLC, M_WEDGE, M_BLOCK


@dataclass
class LeafType:
    wl: float
    wt: float
    wg: float
    wtip: float
    wts: float
    wbs: float
    ztip: float
    zl: float
    zt: float
    zg: float
    zth: float
    zbh: float
    holepos: float
    zts: float
    zbs: float

    def vertices(self, kind, zmin, zthick):
        """14 (x, z) vertices of one leaf type (read_egsinp.h:40-88)."""
        wl, wt, wg, wtip, wts, wbs = self.wl, self.wt, self.wg, self.wtip, self.wts, self.wbs
        zmax = zmin + zthick
        if kind == "full":
            v = [(0, self.ztip), (wtip, self.ztip), (wtip, self.zl), (wt + wl - wg, self.zl),
                 (wt + wl - wg, self.zg), (wt + wl, self.zg), (wt + wl, zmax), (wt + wts - wbs, zmax),
                 (wt + wts - wbs, self.zbs), (wt + wts, self.zbs), (wt + wts, self.zts), (wt, self.zts),
                 (wt, self.zt), (0, self.zt)]
        elif kind == "target":
            v = [(0, zmin), (wt + wl - wbs + wts, zmin), (wt + wl - wbs + wts, self.zts), (wt + wl - wbs, self.zts),
                 (wt + wl - wbs, self.zbs), (wt + wl, self.zbs), (wt + wl, self.zg), (wt + wl - wg, self.zg),
                 (wt + wl - wg, self.ztip), (wt + wl - wg - wtip, self.ztip), (wt + wl - wg - wtip, self.zl),
                 (wt, self.zl), (wt, self.zt), (0, self.zt)]
        else:  # isocenter
            v = [(0, self.zt), (wt, self.zt), (wt, self.ztip), (wt + wtip, self.ztip), (wt + wtip, self.zl),
                 (wt + wl - wg, self.zl), (wt + wl - wg, self.zg), (wt + wl, self.zg), (wt + wl, zmax),
                 (wts - wbs, zmax), (wts - wbs, self.zbs), (wts, self.zbs), (wts, self.zts), (0, self.zts)]
        return np.array(v, np.float64)


@dataclass
class DynVMLC:
    """Parameters of the CM DYNVMLC block (init.cu:390-451)."""
    rmax: float = 20.0
    zmin: float = 48.5
    zthick: float = 6.75
    full: LeafType = None
    target: LeafType = None
    isocenter: LeafType = None
    n_full: int = 10
    n_half: int = 40
    x_start: float = -9.12
    air_gap: float = 0.004
    rad_end: float = 7.0
    leaf_open: list = field(default_factory=lambda: [(-20.0, 20.0, 60)])   # (NEG, POS, NUM) rows
    media: str = "W700ICRU"

    @staticmethod
    def synthetic():
        """A Millennium-like 120-leaf layout (10 full / 40 half / 10 full pairs)."""
        full = LeafType(wl=0.46, wt=0.04, wg=0.04, wtip=0.02, wts=0.10, wbs=0.06, ztip=48.5, zl=48.55,
                        zt=55.0, zg=48.7, zth=50.0, zbh=50.5, holepos=0.0, zts=54.6, zbs=54.9)
        target = LeafType(wl=0.20, wt=0.04, wg=0.04, wtip=0.02, wts=0.05, wbs=0.03, ztip=55.2, zl=55.25,
                          zt=51.0, zg=54.95, zth=50.0, zbh=50.5, holepos=0.0, zts=48.7, zbs=48.9)
        iso = LeafType(wl=0.24, wt=0.04, wg=0.04, wtip=0.02, wts=0.10, wbs=0.05, ztip=48.5, zl=48.55,
                       zt=51.5, zg=48.7, zth=50.0, zbh=50.5, holepos=0.0, zts=54.8, zbs=55.0)
        return DynVMLC(full=full, target=target, isocenter=iso)

    def build(self):
        """crossXZ[960][2], boundaries and the scalar constants the kernels read."""
        cross = np.zeros((960, 2), np.float64)
        zmin, zthick = self.zmin, self.zthick
        vf = self.full.vertices("full", zmin, zthick)
        vt = self.target.vertices("target", zmin, zthick)
        vi = self.isocenter.vertices("isocenter", zmin, zthick)
        X = self.x_start
        i = 0

        def put(i, X, v):
            cross[i * 16:i * 16 + 14, 0] = (X + v[:, 0]) / zmin * v[:, 1]
            cross[i * 16:i * 16 + 14, 1] = v[:, 1]

        for _ in range(self.n_full):
            put(i, X, vf)
            X += self.full.wl + self.air_gap
            i += 1
        x_mid_1 = X
        for _ in range(self.n_half // 2):
            put(i, X, vt)
            X += self.target.wl + self.air_gap
            i += 1
            put(i, X, vi)
            X += self.isocenter.wl + self.air_gap
            i += 1
        x_mid_2 = X
        for _ in range(self.n_full):
            put(i, X, vf)
            X += self.full.wl + self.air_gap
            i += 1
        x_end = X - self.air_gap + self.full.wg
        k = 0
        for neg, pos, num in self.leaf_open:
            for _ in range(num):
                if k < 60:
                    cross[14 + k * 16] = (neg, pos)
                k += 1
        cross[15] = (zmin, zthick)
        cross[31] = (self.x_start, x_end)
        cross[47] = (x_mid_1, x_mid_2)
        cross[63, 1] = self.air_gap
        cross[79] = (self.full.wl, self.target.wl)
        cross[95] = (self.isocenter.wl, self.full.wt)
        cross[111, 0] = self.rmax
        zmax = zmin + zthick
        bxz = np.array([(self.x_start / zmin * zmax, zmax), (self.x_start, zmin), (x_end, zmin),
                        (x_end / zmin * zmax, zmax)], np.float64)
        byz = np.array([(-self.rmax, zmax), (-self.rmax, zmin), (self.rmax, zmin), (self.rmax, zmax)], np.float64)
        return dict(rmax=self.rmax, zmin=zmin, zthick=zthick, x_start=self.x_start, x_end=x_end,
                    x_mid_1=x_mid_1, x_mid_2=x_mid_2, air_gap=self.air_gap, wl_full=self.full.wl,
                    wl_target=self.target.wl, wl_isocenter=self.isocenter.wl, wt=self.full.wt,
                    crossXZ=cross.astype(np.float32), boundaryXZ=bxz.astype(np.float32),
                    boundaryYZ=byz.astype(np.float32), crossYZ=self.cross_yz())

    def cross_yz(self):
        """34-point closed leaf-end outline in the YZ plane (init.cu:256-343)."""
        zmin, zthick, rmax = self.zmin, self.zthick, self.rmax
        zc = zthick / 2
        ys = np.linspace(-zc, zc, 15)
        R = self.rad_end
        xs = -(R - np.sqrt(np.maximum(R * R - ys * ys, 0.0)))
        n = np.zeros((30, 2))
        n[:15, 0] = xs
        n[:15, 1] = ys
        for i in range(15):               # bank B mirrors bank A, ordered bottom to top
            n[29 - i, 0] = -xs[i]
            n[29 - i, 1] = ys[i]
        c = np.zeros((34, 2))
        c[0] = (-rmax, zthick + zmin)
        c[1] = (-rmax, zmin)
        c[2:17, 0] = n[:15, 0]
        c[2:17, 1] = n[:15, 1] + zc + zmin
        c[17:32, 0] = n[15:, 0]
        c[17:32, 1] = n[15:, 1] + zc + zmin
        c[32] = (rmax, zmin)
        c[33] = (rmax, zthick + zmin)
        return c.astype(np.float32)


@dataclass
class SecJaws:
    """CM JAWS 'SECJAWS' (init.cu:612-689): Y jaws above X jaws."""
    rmax: float = 20.0
    zminy: float = 28.0
    zmaxy: float = 35.8
    zminx: float = 36.7
    zmaxx: float = 44.5
    media: str = "W700ICRU"


def secjaws_polygons(jaws: SecJaws, x1, x2, y1, y2, sid):
    """Per-field jaw polygons (setup_secjaws, init.cu:1504-1592)."""
    j = jaws
    bminy = [(x1 * j.zminy / sid - 0.5, y1 * j.zminy / sid - 0.5), (x2 * j.zminy / sid + 0.5, y1 * j.zminy / sid - 0.5),
             (x2 * j.zminy / sid + 0.5, y2 * j.zminy / sid + 0.5), (x1 * j.zminy / sid - 0.5, y2 * j.zminy / sid + 0.5)]
    bminx = [(x1 * j.zminx / sid - 0.5, y1 * j.zminx / sid - 0.5), (x2 * j.zminx / sid + 0.5, y1 * j.zminx / sid - 0.5),
             (x2 * j.zminx / sid + 0.5, y2 * j.zminx / sid + 0.5), (x1 * j.zminx / sid - 0.5, y2 * j.zminx / sid + 0.5)]
    bmaxy = [(-j.rmax, j.zminy), (j.rmax, j.zminy), (j.rmax, j.zmaxy), (-j.rmax, j.zmaxy)]
    bmaxx = [(-j.rmax, j.zminx), (j.rmax, j.zminx), (j.rmax, j.zmaxx), (-j.rmax, j.zmaxx)]
    gy = [(-j.rmax, j.zmaxy), (-j.rmax, j.zminy), (y1 * j.zminy / sid, j.zminy), (y1 * j.zmaxy / sid, j.zmaxy),
          (y2 * j.zmaxy / sid, j.zmaxy), (y2 * j.zminy / sid, j.zminy), (j.rmax, j.zminy), (j.rmax, j.zmaxy)]
    gx = [(-j.rmax, j.zmaxx), (-j.rmax, j.zminx), (x1 * j.zminx / sid, j.zminx), (x1 * j.zmaxx / sid, j.zmaxx),
          (x2 * j.zmaxx / sid, j.zmaxx), (x2 * j.zminx / sid, j.zminx), (j.rmax, j.zminx), (j.rmax, j.zmaxx)]
    f = lambda a: np.array(a, np.float32)
    return dict(boundMinY=f(bminy), boundMinX=f(bminx), boundMaxY=f(bmaxy), boundMaxX=f(bmaxx),
                jawsGeomY=f(gy), jawsGeomX=f(gx))


def leaf_endnodes(cross_yz, leaf_pos, zmin, zthick, sid):
    """endnode[60][34][2] for one field (init_leaf_pos, init.cu:1594-1662).

    ``leaf_pos``: 120 mlcinp positions; pair j uses pos[j] and pos[j+60] with
    the reference's bank swap (POS = pos[j], NEG = -pos[j+60])."""
    zc = zmin + zthick / 2
    out = np.repeat(np.asarray(cross_yz, np.float32)[None], 60, axis=0).copy()
    pos = np.asarray(leaf_pos, np.float32)
    for j in range(60):
        if pos[j] + pos[j + 60] > 0:
            POS = pos[j]
            NEG = -pos[j + 60]
            out[j, 2:17, 0] = cross_yz[2:17, 0] + NEG * zc / sid
            out[j, 17:32, 0] = cross_yz[17:32, 0] + POS * zc / sid
    return out


def gantry_cos_sin(angle_deg):
    """float32 cos/sin exactly as the reference uploads them (CUDA_EGS.cu:426-434)."""
    a = np.float32(np.float32(angle_deg) * 3.1415926 / 180)
    return np.float32(math.cos(float(a))), np.float32(math.sin(float(a)))


def module_order(secjaws_on, mlc_on, block_on=False, wedge_on=False):
    """Next-module table (CUDA_EGS.cu:1277-1305); entry 0 is the first module."""
    order = [0] * 8
    nxt = M_PHANTOM
    if wedge_on:
        order[M_WEDGE] = nxt
        nxt = M_WEDGE
    if block_on:
        order[M_BLOCK] = nxt
        nxt = M_BLOCK
    if mlc_on:
        order[M_VARMLC] = nxt
        nxt = M_VARMLC
    if secjaws_on:
        order[M_SECJAWX] = nxt
        order[M_SECJAWY] = M_SECJAWX
        nxt = M_SECJAWY
    order[0] = nxt
    return order
