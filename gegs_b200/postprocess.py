"""Dose post-processing and CT conversion through the CUDA library
(include/gegs_post.h), plus the reference's scalar dose read-outs.

* ``interp_dose``      dose on a regular output grid (interp_dose, output.c:221-316),
  ``write_interp``     its file ``<base>_Interpolate_NNNxNNNxNNN.bin`` (3 x int32 dims + float32);
* ``gamma3d``          3-D global gamma index and pass rate;
* ``ct_ramp``          HU -> medium, density (CTToMedium's ramp, ctcreate.c:913-970);
* ``point_dose``       the absolute dose at a point (output_AbsDos, output.c:780-871).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from .engine import load_library
from .io_formats import strtof

_ready = False


class CtRampSegment(C.Structure):
    _fields_ = [("hu_upper", C.c_double), ("density_lower", C.c_double), ("density_upper", C.c_double),
                ("medium", C.c_int32), ("pad_", C.c_int32)]


def _lib():
    global _ready
    L = load_library()
    if not _ready:
        vp, f, i = C.c_void_p, C.c_float, C.c_int
        L.gegs_interp_dose.argtypes = [i, vp, i, i, i, vp, vp, vp, f, f, f, f, f, f, i, i, i, vp]
        L.gegs_gamma3d.argtypes = [i, vp, vp, i, i, i, f, f, f, f, f, f, f, vp, C.POINTER(C.c_uint64),
                                   C.POINTER(C.c_uint64)]
        L.gegs_ct_ramp.argtypes = [i, vp, C.c_uint64, vp, i, C.c_double, vp, vp]
        _ready = True
    return L


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} failed with status {rc}")


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def interp_dose(dose, x_bounds, y_bounds, z_bounds, start, sizes, dims, device=0):
    """dose: (nz, ny, nx) or flat, x fastest. Returns the (mz, my, mx) grid."""
    nx, ny, nz = len(x_bounds) - 1, len(y_bounds) - 1, len(z_bounds) - 1
    d = _f32(dose).reshape(-1)
    xb, yb, zb = _f32(x_bounds), _f32(y_bounds), _f32(z_bounds)
    mx, my, mz = (int(v) for v in dims)
    out = np.empty(mx * my * mz, np.float32)
    _check(_lib().gegs_interp_dose(device, d.ctypes.data, nx, ny, nz, xb.ctypes.data, yb.ctypes.data,
                                   zb.ctypes.data, *(float(v) for v in start), *(float(v) for v in sizes),
                                   mx, my, mz, out.ctypes.data), "gegs_interp_dose")
    return out.reshape(mz, my, mx)


def write_interp(base, grid):
    mz, my, mx = grid.shape
    name = f"{base}_Interpolate_{mx:03d}x{my:03d}x{mz:03d}.bin"
    with open(name, "wb") as f:
        f.write(np.array([mx, my, mz], np.int32).tobytes())
        f.write(_f32(grid).tobytes())
    return name


def gamma3d(ref, ev, spacing, dta=0.1, dd=0.01, cutoff=0.10, search=3.0, device=0):
    """Global gamma: dd and cutoff are fractions of max(ref), dta in cm, search
    radius = search * dta. Returns (gamma array with -1 below the cutoff, pass rate)."""
    r, e = _f32(ref), _f32(ev)
    if r.shape != e.shape or r.ndim != 3:
        raise ValueError("ref and eval must be (nz, ny, nx) arrays of one shape")
    nz, ny, nx = r.shape
    rmax = float(r.max())
    g = np.empty(r.size, np.float32)
    ne, npass = C.c_uint64(), C.c_uint64()
    _check(_lib().gegs_gamma3d(device, r.ctypes.data, e.ctypes.data, nx, ny, nz, *(float(s) for s in spacing),
                               float(dta), float(dd * rmax), float(cutoff * rmax), float(search), g.ctypes.data,
                               C.byref(ne), C.byref(npass)), "gegs_gamma3d")
    return g.reshape(r.shape), (npass.value / ne.value if ne.value else float("nan"))


def ct_ramp(hu, segments, hu_lower, device=0):
    """segments: (medium index, HU upper bound, density at the lower end, density at the upper end)."""
    h = np.ascontiguousarray(hu, np.int16).reshape(-1)
    seg = (CtRampSegment * len(segments))()
    for k, (m, ub, dlo, dhi) in enumerate(segments):
        seg[k] = CtRampSegment(float(ub), float(dlo), float(dhi), int(m), 0)
    med = np.empty(h.size, np.uint16)
    dens = np.empty(h.size, np.float32)
    _check(_lib().gegs_ct_ramp(device, h.ctypes.data, h.size, C.cast(seg, C.c_void_p), len(segments),
                               float(hu_lower), med.ctypes.data, dens.ctypes.data), "gegs_ct_ramp")
    return med, dens


def point_dose(dose, x_bounds, y_bounds, z_bounds, pos):
    """Interpolated dose at `pos` between voxel centres, with the reference's
    index search (output_AbsDos, output.c:780-871)."""
    nx, ny, nz = len(x_bounds) - 1, len(y_bounds) - 1, len(z_bounds) - 1
    d = _f32(dose).reshape(-1)
    c = [((_f32(b)[:-1] + _f32(b)[1:]) / np.float32(2)).astype(np.float32) for b in (x_bounds, y_bounds, z_bounds)]
    f = np.float32

    def find(cb, n, v):
        for i in range(1, n - 2):
            if v > cb[i] and v <= cb[i + 1]:
                return i
        return 0 if v <= cb[1] else n - 2

    px, py, pz = (f(v) for v in pos)
    i, j, k = find(c[0], nx, px), find(c[1], ny, py), find(c[2], nz, pz)
    xy = nx * ny
    at = lambda a, b, cc: d[a + nx * b + xy * cc]
    a0 = at(i, j, k) + (pz - c[2][k]) * (at(i, j, k + 1) - at(i, j, k)) / (c[2][k + 1] - c[2][k])
    a1 = at(i + 1, j, k) + (pz - c[2][k]) * (at(i + 1, j, k + 1) - at(i + 1, j, k)) / (c[2][k + 1] - c[2][k])
    a2 = at(i, j + 1, k) + (pz - c[2][k]) * (at(i, j + 1, k + 1) - at(i, j + 1, k)) / (c[2][k + 1] - c[2][k])
    a3 = at(i + 1, j + 1, k) + (pz - c[2][k]) * (at(i + 1, j + 1, k + 1) - at(i + 1, j + 1, k)) / (c[2][k + 1] - c[2][k])
    a0 = a0 + (py - c[1][j]) * (a2 - a0) / (c[1][j + 1] - c[1][j])
    a1 = a1 + (py - c[1][j]) * (a3 - a1) / (c[1][j + 1] - c[1][j])
    return float(a0 + (px - c[0][i]) * (a1 - a0) / (c[0][i + 1] - c[0][i]))


def sample_plane(dose, x_bounds, y_bounds, z_bounds, start, sizes, dims):
    """The dose of the voxel nearest each point of a comparison grid: the
    reference's index `int((pos - c0) / (c1 - c0) + 0.1)` on voxel centres
    (output_RelDos_II, output.c:606-624), the + 0.1 in double as in C.
    A point outside the phantom is an error (the reference reads past the grid)."""
    f = np.float32
    d = _f32(dose).reshape(-1)
    nx, ny, nz = len(x_bounds) - 1, len(y_bounds) - 1, len(z_bounds) - 1
    c = [((_f32(b)[:-1] + _f32(b)[1:]) / f(2)).astype(np.float32) for b in (x_bounds, y_bounds, z_bounds)]
    mx, my, mz = (int(v) for v in dims)
    sx, sy, sz = (f(v) for v in sizes)
    x0, y0, z0 = (f(v) for v in start)
    calc = np.empty(mx * my * mz, np.float32)
    for k in range(mz):
        for j in range(my):
            for i in range(mx):
                px, py, pz = f(x0 + f(sx * f(i))), f(y0 + f(sy * f(j))), f(z0 + f(sz * f(k)))
                ix = int(float(f((px - c[0][0]) / f(c[0][1] - c[0][0]))) + 0.1)    # + 0.1 in double
                iy = int(float(f((py - c[1][0]) / f(c[1][1] - c[1][0]))) + 0.1)
                iz = int(float(f((pz - c[2][0]) / f(c[2][1] - c[2][0]))) + 0.1)
                if not (0 <= ix < nx and 0 <= iy < ny and 0 <= iz < nz):
                    raise ValueError(f"comparison point ({px}, {py}, {pz}) lies outside the phantom")
                calc[mx * my * k + mx * j + i] = d[nx * ny * iz + nx * iy + ix]
    return calc


def relative_dose(dose, x_bounds, y_bounds, z_bounds, start, sizes, dims, measured=None, norm_type=0,
                  array_type=2, gamma_len_cm=0.3, gamma_dos=0.03, iso=(0.0, 0.0, 0.0)):
    """The reference's comparison of the dose with detector-array data
    (output_RelDos_II, output.c:596-778), in float32 as it computes it.

    Samples the dose at the voxel nearest each point of the plane (start
    already moved by the isocentre), normalises both to their maximum
    (norm_type 1) or to the point at the isocentre (2), and marks each point
    above 10 % of the measured maximum as passing when the dose difference is
    within gamma_dos, or -- for the 1000-chamber array (array_type 2) -- when a
    neighbouring point of the plane within gamma_len_cm agrees.
    Without measured data the file lists the sampled doses alone.
    Returns (lines of the result file, compared, passed)."""
    f = np.float32
    mx, my, mz = (int(v) for v in dims)
    sx, sy, sz = (f(v) for v in sizes)
    x0, y0, z0 = (f(v) for v in start)
    calc = sample_plane(dose, x_bounds, y_bounds, z_bounds, start, sizes, dims)
    if measured is None:
        return [f"{v:f}" for v in calc], 0, 0
    meas = _f32(measured).reshape(-1)[:calc.size].copy()
    top = lambda a: max(f(0.0), a.max())  # the reference's running maxima start at 0
    if norm_type == 1:
        meas = meas / top(meas)
        calc = calc / top(calc)
        meas_max = f(1.0)
    elif norm_type == 2:
        center = 0
        if sx != 0:
            center += int(float(f(f(f(iso[0]) - x0) / sx)) + 0.1)
        if sy != 0:
            center += int(float(f(f(f(iso[1]) - y0) / sy)) + 0.1) * mx
        if sz != 0:
            center += int(float(f(f(f(iso[2]) - z0) / sz)) + 0.1) * mx * my
        mc, cc = meas[center], calc[center]
        meas_max = f(top(meas) / mc)
        meas = meas / mc
        calc = calc / cc
    else:
        meas = meas * f(100.0)
        meas_max = top(meas)
    thr = f(meas_max * f(0.1))
    lines, total, count = [], 0, 0
    dos, ln = f(gamma_dos), f(gamma_len_cm)
    def near(a, m):                       # float ratio, squared in float; the sum and sqrt in double
        v = f(f(f(abs(f(a - m)) / m) / dos))
        v = f(v * v)
        return f(np.sqrt(float(v) + 0.25 * 0.25 / float(ln) / float(ln)))
    for i in range(calc.size):
        pas = 0
        m = meas[i]
        if m > thr:
            total += 1
            if array_type == 1:
                pas = 1 if f(abs(f(calc[i] - m)) / m) <= dos else -1
                count += pas > 0
            else:
                if f(abs(f(calc[i] - m)) / m) <= dos:
                    pas += 1
                iz = i // mx
                ix = i - iz * mx
                if ix > 0 and pas <= 0 and near(calc[i - 1], m) <= 1:
                    pas += 1
                if ix + 1 < mx and pas <= 0 and near(calc[i + 1], m) <= 1:
                    pas += 1
                if iz > 0 and near(calc[i - mx], m) <= 1:
                    pas += 1
                if iz + 1 < mz and pas <= 0 and near(calc[i + mx], m) <= 1:
                    pas += 1
                if pas > 0:
                    count += 1
                else:
                    pas = -1
        lines.append(f"{m:f}\t {calc[i]:f}\t {pas}")
    # (float)count / total, times 100 in float, printed with %.0f
    pct = f"{float(f(f(f(count) / f(total)) * f(100.0))):.0f}" if total else "nan"
    lines.append(f"Totally {total} points compared, {count} passed, percentage = {pct} %")
    return lines, total, count


def write_relative_dose(base, lines, dims):
    mx, my, mz = (int(v) for v in dims)
    name = f"{base}_RelativeDose_{mx:03d}x{my:03d}x{mz:03d}.txt"
    with open(name, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    return name


def read_measured(path, n):
    """The measured data file: the first number of each of the first n lines
    (the reference reads `infile >> v` into a float, output.c:641-676, then
    skips the rest of the line)."""
    vals = []
    for line in Path(path).read_text().splitlines():
        tok = line.split()
        if tok:
            vals.append(strtof(tok[0]))
        if len(vals) == n:
            break
    if len(vals) < n:
        raise ValueError(f"measured data {path}: {len(vals)} values, {n} expected")
    return np.array(vals, np.float32)
