"""Beam-line geometry set-up: DYNVMLC leaf cross sections, leaf-end polygons,
secondary-jaw polygons and patient placement.

Restates the reference's host set-up code:

* leaf vertex construction ``Leaf::VerCal_full/target/isocenter``
  (read_egsinp.h:40-88) and the crossXZ / boundary arrays (init.cu:345-611);
* the leaf-end (YZ) outline ``leaf_end`` (init.cu:256-343);
* per-field jaw polygons ``setup_secjaws`` (init.cu:1504-1592);
* per-field leaf-end polygons ``init_leaf_pos`` (init.cu:1594-1662), with the
  reference's bank swap (``INVERSE_MLC_Bank_AB``, CUDA_EGS.h:27);
* gantry cos/sin as uploaded by the reference (CUDA_EGS.cu:420-422);
* the module order (CUDA_EGS.cu:1277-1305).

The reference reads every input number into a float and computes the set-up
in float arithmetic; so does this module (``F``, numpy float32 scalars), in
the reference's operation order, so that the same input files give the same
polygons bit for bit. The leaf-end outline is the reference's fixed table of
15 points per bank (init.cu:266-298): the DYNVMLC input's leaf radius is read
but does not shape it.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .scene import M_PHANTOM, M_SECJAWX, M_SECJAWY, M_VARMLC, M_WEDGE, M_BLOCK

F = np.float32


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
        """14 (x, z) vertices of one leaf type, in float (read_egsinp.h:37-88)."""
        wl, wt, wg, wtip, wts, wbs = (F(getattr(self, k)) for k in ("wl", "wt", "wg", "wtip", "wts", "wbs"))
        ztip, zl, zt, zg, zts, zbs = (F(getattr(self, k)) for k in ("ztip", "zl", "zt", "zg", "zts", "zbs"))
        zmin, zmax = F(zmin), F(zmin) + F(zthick)
        o = F(0.0)
        if kind == "full":
            v = [(o, ztip), (wtip, ztip), (wtip, zl), (wt + wl - wg, zl), (wt + wl - wg, zg), (wt + wl, zg),
                 (wt + wl, zmax), (wt + wts - wbs, zmax), (wt + wts - wbs, zbs), (wt + wts, zbs), (wt + wts, zts),
                 (wt, zts), (wt, zt), (o, zt)]
        elif kind == "target":
            v = [(o, zmin), (wt + wl - wbs + wts, zmin), (wt + wl - wbs + wts, zts), (wt + wl - wbs, zts),
                 (wt + wl - wbs, zbs), (wt + wl, zbs), (wt + wl, zg), (wt + wl - wg, zg), (wt + wl - wg, ztip),
                 (wt + wl - wg - wtip, ztip), (wt + wl - wg - wtip, zl), (wt, zl), (wt, zt), (o, zt)]
        else:  # isocenter
            v = [(o, zt), (wt, zt), (wt, ztip), (wt + wtip, ztip), (wt + wtip, zl), (wt + wl - wg, zl),
                 (wt + wl - wg, zg), (wt + wl, zg), (wt + wl, zmax), (wts - wbs, zmax), (wts - wbs, zbs), (wts, zbs),
                 (wts, zts), (o, zts)]
        return np.array(v, np.float32)


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
        """crossXZ[960][2], boundaries and the scalar constants the kernels read,
        in float as read_egsinp computes them (init.cu:451-561). Entries the
        reference leaves unset (the 16th vertex of most leaves) are 0 here."""
        cross = np.zeros((960, 2), np.float32)
        zmin, zthick, air_gap = F(self.zmin), F(self.zthick), F(self.air_gap)
        vf = self.full.vertices("full", zmin, zthick)
        vt = self.target.vertices("target", zmin, zthick)
        vi = self.isocenter.vertices("isocenter", zmin, zthick)
        X = F(self.x_start)
        i = 0

        def put(i, X, v):
            for j in range(14):
                cross[i * 16 + j] = ((X + v[j, 0]) / zmin * v[j, 1], v[j, 1])

        for _ in range(self.n_full):
            put(i, X, vf)
            X = X + F(self.full.wl) + air_gap
            i += 1
        x_mid_1 = X
        for _ in range(self.n_half // 2):
            put(i, X, vt)
            X = X + F(self.target.wl) + air_gap
            i += 1
            put(i, X, vi)
            X = X + F(self.isocenter.wl) + air_gap
            i += 1
        x_mid_2 = X
        for _ in range(self.n_full):
            put(i, X, vf)
            X = X + F(self.full.wl) + air_gap
            i += 1
        x_end = X - air_gap + F(self.full.wg)
        k = 0
        for neg, pos, num in self.leaf_open:
            for _ in range(num):
                if k < 60:
                    cross[14 + k * 16] = (neg, pos)
                k += 1
        x_start, rmax = F(self.x_start), F(self.rmax)
        cross[15] = (zmin, zthick)
        cross[31] = (x_start, x_end)
        cross[47] = (x_mid_1, x_mid_2)
        cross[63, 1] = air_gap
        cross[79] = (self.full.wl, self.target.wl)
        cross[95] = (self.isocenter.wl, self.full.wt)
        cross[111, 0] = rmax
        ztop = zthick + zmin
        bxz = np.array([(x_start / zmin * (zmin + zthick), ztop), (x_start, zmin), (x_end, zmin),
                        (x_end / zmin * (zmin + zthick), ztop)], np.float32)
        byz = np.array([(-rmax, ztop), (-rmax, zmin), (rmax, zmin), (rmax, ztop)], np.float32)
        f = lambda v: float(F(v))
        return dict(rmax=f(rmax), zmin=f(zmin), zthick=f(zthick), x_start=f(x_start), x_end=f(x_end),
                    x_mid_1=f(x_mid_1), x_mid_2=f(x_mid_2), air_gap=f(air_gap), wl_full=f(self.full.wl),
                    wl_target=f(self.target.wl), wl_isocenter=f(self.isocenter.wl), wt=f(self.full.wt),
                    crossXZ=cross, boundaryXZ=bxz, boundaryYZ=byz, crossYZ=self.cross_yz())

    def cross_yz(self):
        """34-point closed leaf-end outline in the YZ plane (leaf_end, init.cu:256-343)."""
        zmin, zthick, rmax = F(self.zmin), F(self.zthick), F(self.rmax)
        zc = zthick / F(2)
        n = np.zeros((30, 2), np.float32)
        for i in range(15):
            x = F(LEAF_END_X[i])
            y = -zc if i == 0 else (zc if i == 14 else F(LEAF_END_Y[i]))
            n[i] = (x, y)                 # bank A, bottom to top
            n[29 - i] = (abs(x), y)       # bank B mirrors it (x >= 0, +0 at the centre), stored top to bottom
        c = np.zeros((34, 2), np.float32)
        c[0] = (-rmax, zthick + zmin)
        c[1] = (-rmax, zmin)
        for i in range(30):
            c[2 + i] = (n[i, 0], n[i, 1] + zc + zmin)
        c[32] = (rmax, zmin)
        c[33] = (rmax, zthick + zmin)
        return c


# The reference's leaf-end outline of bank A (leaf_end, init.cu:266-280), as
# (x, y) pairs from the bottom of the leaf to its top; the first and last y
# are -/+ half the leaf thickness, set from the input. Bank B is its mirror.
LEAF_END_X = (-0.86708, -0.64016, -0.44640, -0.28667, -0.16167, -0.07199, -0.01802, 0.0,
              -0.01802, -0.07199, -0.16167, -0.28667, -0.44640, -0.64016, -0.86708)
LEAF_END_Y = (None, -2.92273, -2.45316, -1.97406, -1.48729, -0.99475, -0.49834, 0.0,
              0.49834, 0.99475, 1.48729, 1.97406, 2.45316, 2.92273, None)


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
    """Per-field jaw polygons in float (setup_secjaws, init.cu:1504-1592). The
    double literal 0.5 rounds the exact difference once, as a float
    subtraction does."""
    j = jaws
    rmax, zminy, zmaxy, zminx, zmaxx = (F(v) for v in (j.rmax, j.zminy, j.zmaxy, j.zminx, j.zmaxx))
    x1, x2, y1, y2, sid = (F(v) for v in (x1, x2, y1, y2, sid))
    h = F(0.5)
    bminy = [(x1 * zminy / sid - h, y1 * zminy / sid - h), (x2 * zminy / sid + h, y1 * zminy / sid - h),
             (x2 * zminy / sid + h, y2 * zminy / sid + h), (x1 * zminy / sid - h, y2 * zminy / sid + h)]
    bminx = [(x1 * zminx / sid - h, y1 * zminx / sid - h), (x2 * zminx / sid + h, y1 * zminx / sid - h),
             (x2 * zminx / sid + h, y2 * zminx / sid + h), (x1 * zminx / sid - h, y2 * zminx / sid + h)]
    bmaxy = [(-rmax, zminy), (rmax, zminy), (rmax, zmaxy), (-rmax, zmaxy)]
    bmaxx = [(-rmax, zminx), (rmax, zminx), (rmax, zmaxx), (-rmax, zmaxx)]
    gy = [(-rmax, zmaxy), (-rmax, zminy), (y1 * zminy / sid, zminy), (y1 * zmaxy / sid, zmaxy),
          (y2 * zmaxy / sid, zmaxy), (y2 * zminy / sid, zminy), (rmax, zminy), (rmax, zmaxy)]
    gx = [(-rmax, zmaxx), (-rmax, zminx), (x1 * zminx / sid, zminx), (x1 * zmaxx / sid, zmaxx),
          (x2 * zmaxx / sid, zmaxx), (x2 * zminx / sid, zminx), (rmax, zminx), (rmax, zmaxx)]
    f = lambda a: np.array(a, np.float32)
    return dict(boundMinY=f(bminy), boundMinX=f(bminx), boundMaxY=f(bmaxy), boundMaxX=f(bmaxx),
                jawsGeomY=f(gy), jawsGeomX=f(gx))


def leaf_endnodes(cross_yz, leaf_pos, zmin, zthick, sid):
    """endnode[60][34][2] for one field, in float (init_leaf_pos, init.cu:1594-1662).

    ``leaf_pos``: 120 mlcinp positions; pair j uses pos[j] and pos[j+60] with
    the reference's bank swap (POS = pos[j], NEG = -pos[j+60]). A pair whose
    positions do not add up to more than 0 keeps the unshifted outline."""
    zc = F(zmin) + F(zthick) / F(2)
    sid = F(sid)
    cy = np.asarray(cross_yz, np.float32)
    out = np.repeat(cy[None], 60, axis=0).copy()
    pos = np.asarray(leaf_pos, np.float32)
    for j in range(60):
        if pos[j] + pos[j + 60] > 0:
            POS = pos[j]
            NEG = -pos[j + 60]
            out[j, 2:17, 0] = cy[2:17, 0] + NEG * zc / sid
            out[j, 17:32, 0] = cy[17:32, 0] + POS * zc / sid
    return out


def gantry_cos_sin(angle_deg):
    """The cosine and sine the reference uploads for a field (CUDA_EGS.cu:420-422):
    the angle (a float) times 3.1415926 / 180 in double, stored as a float,
    then cos and sin of that float, correctly rounded to float."""
    a = F(float(F(angle_deg)) * 3.1415926 / 180)
    return F(math.cos(float(a))), F(math.sin(float(a)))


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
