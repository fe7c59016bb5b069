"""Readers and writers of the reference's input and output files.

* ``.egsphant`` voxel phantom (EGSnrc text format), read as the reference
  does in ``init_phantom_and_MLC`` (init.cu:1164-1275), plus a writer;
* ``.egsphsp1`` phase space, MODE0 (28-byte records) and MODE2 (32-byte
  records with ZLAST), single file or ``<name>_p<i>.egsphsp1`` parts
  (read_egsphsp.cpp:44-232), plus a writer;
* the BEAMnrc ``.egsinp`` component modules the reference reads: ``CM DYNVMLC``
  (read_mlcinp.cpp:6-186) and ``CM JAWS with identifier SECJAWS``
  (init.cu:611-689);
* the ``.mlcinfo`` field list and the per-field ``.mlcinp`` leaf positions
  (``read_mlcinp``, init.cu:1377-1500), and the output-factor table;
* the dose output ``<prefix>_DoseResults_NNNxNNNxNNN.bin`` (raw float32, x
  fastest; ``write_dose``, output.c:873-918).

The text parsers follow the reference's C++ stream reads (``infile >> value
>> ch`` consumes a number and the one separator character after it;
``ignore(n, '\\n')`` drops the rest of a line), so files the reference reads
are read here to the same numbers.
"""
from __future__ import annotations

import os
import re
import struct
from fractions import Fraction
from pathlib import Path

import numpy as np

from .geometry import DynVMLC, LeafType, SecJaws
from .scene import PHSP_DTYPE

# ---------------------------------------------------------------------------
# a C++-istream-like reader
# ---------------------------------------------------------------------------
_NUM = re.compile(r"[+-]?(\d+\.?\d*|\.\d+)([eE][+-]?\d+)?")


def strtof(tok):
    """A decimal string rounded once, to the nearest float32 (ties to even),
    as the reference's readers round it (`stream >> float`, `%f` in scanf).
    float() alone rounds to double first, and rounding that double to float32
    goes wrong where it lands exactly halfway between two float32 values."""
    d = float(tok)
    with np.errstate(over="ignore"):                # beyond the float range: infinity, as strtof gives
        x = np.float32(d)
        if not np.isfinite(x) or float(x) == d:
            return x
        lo, hi = (np.nextafter(x, np.float32(-np.inf)), x) if float(x) > d else (x, np.nextafter(x, np.float32(np.inf)))
    mid = (float(lo) + float(hi)) / 2.0            # exact: two float32 values and a halving
    if d != mid:
        return x
    exact, m = Fraction(tok.strip()), Fraction(mid)
    if exact != m:
        return hi if exact > m else lo
    return lo if int(lo.view(np.uint32)) % 2 == 0 else hi


def strtof_array(tokens):
    """strtof over a list of decimal strings, vectorised: parsed as doubles,
    rounded to float32, and only the values that landed on a float32 midpoint
    (a double-rounding case) parsed again exactly."""
    d = np.array(tokens, np.float64)
    with np.errstate(over="ignore"):
        x = d.astype(np.float32)
        up = np.nextafter(x, np.where(x.astype(np.float64) < d, np.float32(np.inf), np.float32(-np.inf)))
    tie = np.isfinite(x) & (x.astype(np.float64) != d) & ((x.astype(np.float64) + up.astype(np.float64)) / 2.0 == d)
    for i in np.flatnonzero(tie):
        x[i] = strtof(tokens[i])
    return x


class StreamReader:
    """The subset of std::istream the reference's parsers use."""

    def __init__(self, text: str):
        self.s = text
        self.i = 0

    def eof(self):
        return self.i >= len(self.s)

    def getline(self):
        j = self.s.find("\n", self.i)
        if j < 0:
            line, self.i = self.s[self.i:], len(self.s)
        else:
            line, self.i = self.s[self.i:j], j + 1
        return line

    def ignore(self, n=100, delim="\n"):
        """Drop up to n characters, stopping after `delim`."""
        end = min(len(self.s), self.i + n)
        j = self.s.find(delim, self.i, end)
        self.i = end if j < 0 else j + 1

    def _skip_ws(self):
        while self.i < len(self.s) and self.s[self.i].isspace():
            self.i += 1

    def num(self, kind=float):
        self._skip_ws()
        m = _NUM.match(self.s, self.i)
        if not m:
            raise ValueError(f"expected a number at offset {self.i}: {self.s[self.i:self.i + 30]!r}")
        self.i = m.end()
        txt = m.group(0)
        if kind is int:
            return int(float(txt)) if any(c in txt for c in ".eE") else int(txt)
        return float(strtof(txt)) if kind is float else kind(txt)

    def char(self):
        self._skip_ws()
        c = self.s[self.i] if self.i < len(self.s) else ""
        self.i += 1
        return c

    def num_sep(self, kind=float):
        """`infile >> value >> ch`: a number and the single separator after it."""
        v = self.num(kind)
        self.char()
        return v

    def find_line_starting(self, title: str):
        """Advance past the first line whose beginning equals `title`."""
        while not self.eof():
            line = self.getline()
            if line.startswith(title):
                return True
        return False


def _read_text(path) -> str:
    with open(path, "r", encoding="latin-1", newline="") as f:
        return f.read().replace("\r\n", "\n")


# ---------------------------------------------------------------------------
# egsphant
# ---------------------------------------------------------------------------
def read_egsphant(path):
    """Media names, voxel boundaries, medium index (0-based) and density per voxel.

    Layout: number of media; one medium name per line; one line of ESTEPE
    values (ignored); ``nx ny nz``; nx+1, ny+1, nz+1 boundaries; nz blocks of
    ny lines of nx single-digit medium numbers (1-based), each block followed
    by an empty line; then the densities in the same order."""
    text = _read_text(path)
    lines = text.split("\n")
    k = 0
    nmed = int(lines[k].split()[0]); k += 1
    media = []
    for i in range(nmed):
        name = lines[k].strip(); k += 1
        if not name:
            raise ValueError(f"{path}: medium name {i} is empty")
        media.append(name)
    k += 1                                   # ESTEPE line
    try:
        nx, ny, nz = (int(t) for t in lines[k].split()[:3])
    except (ValueError, IndexError):
        raise ValueError(f"{path}: line {k + 1} must hold the three voxel counts nx ny nz, "
                         f"got {lines[k] if k < len(lines) else ''!r}") from None
    if min(nx, ny, nz) < 1:
        raise ValueError(f"{path}: voxel counts {nx} {ny} {nz} must be positive")
    k += 1
    rest = StreamReader("\n".join(lines[k:]))
    xb = np.array([rest.num() for _ in range(nx + 1)], np.float32)
    yb = np.array([rest.num() for _ in range(ny + 1)], np.float32)
    zb = np.array([rest.num() for _ in range(nz + 1)], np.float32)
    rest.ignore(1 << 30, "\n")
    med = np.empty(nx * ny * nz, np.uint16)
    for z in range(nz):
        for y in range(ny):
            row = rest.getline().strip()
            while row == "" and not rest.eof():
                row = rest.getline().strip()
            if len(row) < nx:
                raise ValueError(f"{path}: medium row (y={y}, z={z}) has {len(row)} of {nx} entries")
            vals = np.frombuffer(row[:nx].encode("ascii"), np.uint8).astype(np.int32) - ord("0")
            if vals.min() < 1 or vals.max() > nmed:
                raise ValueError(f"{path}: medium number outside 1..{nmed} (y={y}, z={z})")
            base = z * nx * ny + y * nx
            med[base:base + nx] = vals - 1
    toks = rest.s[rest.i:].split()
    if len(toks) < nx * ny * nz:
        raise ValueError(f"{path}: {len(toks)} densities for {nx * ny * nz} voxels")
    return dict(media=media, nx=nx, ny=ny, nz=nz, x_bounds=xb, y_bounds=yb, z_bounds=zb,
                voxel_med=med, density=strtof_array(toks[:nx * ny * nz]))


def write_egsphant(path, media, x_bounds, y_bounds, z_bounds, voxel_med, density, estepe=1.0):
    """Write an egsphant file (voxel_med 0-based, x fastest); at most 9 media.
    Numbers carry 9 significant digits, so float32 values read back exactly."""
    nx, ny, nz = len(x_bounds) - 1, len(y_bounds) - 1, len(z_bounds) - 1
    if len(media) > 9:
        raise ValueError("single-digit medium numbers: at most 9 media")
    med = np.asarray(voxel_med).reshape(nz, ny, nx)
    dens = np.asarray(density, np.float32).reshape(nz, ny, nx)
    out = [f"{len(media)}"] + list(media) + ["  ".join(f"{estepe:.4f}" for _ in media), f"{nx} {ny} {nz}"]

    def bounds(b):
        b = np.asarray(b, np.float32)
        return "\n".join(" ".join(f"{float(v):.9g}" for v in b[i:i + 8]) for i in range(0, len(b), 8))

    out += [bounds(x_bounds), bounds(y_bounds), bounds(z_bounds)]
    for z in range(nz):
        out += ["".join(chr(ord("1") + int(v)) for v in med[z, y]) for y in range(ny)]
        out.append("")
    for z in range(nz):
        for y in range(ny):
            out.append(" ".join(f"{float(v):.9g}" for v in dens[z, y]))
        out.append("")
    Path(path).write_text("\n".join(out) + "\n")


# ---------------------------------------------------------------------------
# egsphsp1
# ---------------------------------------------------------------------------
_PHSP2_DTYPE = np.dtype([("latch", "<u4"), ("e", "<f4"), ("x", "<f4"), ("y", "<f4"), ("u", "<f4"), ("v", "<f4"),
                         ("wt", "<f4"), ("zlast", "<f4")])


def read_egsphsp1_header(path):
    with open(path, "rb") as f:
        head = f.read(32)
    mode = head[:5].decode("ascii", "replace")
    if mode not in ("MODE0", "MODE2"):
        raise ValueError(f"{path}: unknown phase-space mode {mode!r}")
    n, nphot = struct.unpack("<ii", head[5:13])
    ekmax, ekmin = struct.unpack("<ff", head[13:21])
    order = "<"
    held = os.path.getsize(path) // 28
    if n < 0 or n > held:                 # written on a big-endian machine, or truncated
        n_be, nphot_be = struct.unpack(">ii", head[5:13])
        if 0 <= n_be <= held:
            order = ">"
            n, nphot = n_be, nphot_be
            ekmax, ekmin = struct.unpack(">ff", head[13:21])
        elif n < 0:
            raise ValueError(f"{path}: negative particle count {n} in the header")
    return dict(mode=mode, n=n, nphot=nphot, ekmax=ekmax, ekmin=ekmin, order=order,
                reclen=28 if mode == "MODE0" else 32)


def read_egsphsp1(path, start=0, count=None):
    """Records [start, start+count) of one file as PHSP_DTYPE (ZLAST dropped)."""
    h = read_egsphsp1_header(path)
    n = h["n"] if count is None else min(count, h["n"] - start)
    dt = PHSP_DTYPE if h["mode"] == "MODE0" else _PHSP2_DTYPE
    if h["order"] == ">":
        dt = dt.newbyteorder(">")
    held = os.path.getsize(path) // h["reclen"] - 1          # records after the header record
    if h["n"] > held:
        raise ValueError(f"{path}: the header announces {h['n']} particles but the file holds {max(held, 0)} "
                         f"records (truncated)")
    with open(path, "rb") as f:
        f.seek(h["reclen"] * (1 + start))
        raw = np.fromfile(f, dtype=dt, count=max(n, 0))
    out = np.empty(len(raw), PHSP_DTYPE)
    for k in PHSP_DTYPE.names:
        out[k] = raw[k]
    return out


def phsp_part_paths(base, nfiles):
    """File names of a phase space given as in the reference's INI
    (``<base>.egsphsp1``, or ``<base>_p<i>.egsphsp1`` for several parts)."""
    if nfiles <= 1:
        return [f"{base}.egsphsp1"]
    return [f"{base}_p{i}.egsphsp1" for i in range(nfiles)]


def read_phase_space(base, nfiles=1):
    return np.concatenate([read_egsphsp1(p) for p in phsp_part_paths(base, nfiles)])


def write_egsphsp1(path, recs, mode="MODE0"):
    recs = np.asarray(recs)
    reclen = 28 if mode == "MODE0" else 32
    e = np.abs(recs["e"]).astype(np.float64)
    charged = (recs["latch"] & np.uint32(0x60000000)) != 0
    ek = np.where(charged, e - 0.5109989461, e)
    nphot = int((~charged).sum())
    head = mode.encode() + struct.pack("<iiff", len(recs), nphot, float(ek.max() if len(ek) else 0.0),
                                       float(ek[charged].min() if charged.any() else 0.0))
    head += b"\0" * (reclen - len(head))
    with open(path, "wb") as f:
        f.write(head)
        if mode == "MODE0":
            f.write(np.ascontiguousarray(recs, PHSP_DTYPE).tobytes())
        else:
            r2 = np.zeros(len(recs), _PHSP2_DTYPE)
            for k in PHSP_DTYPE.names:
                r2[k] = recs[k]
            f.write(r2.tobytes())


# ---------------------------------------------------------------------------
# egsinp component modules
# ---------------------------------------------------------------------------
DYNVMLC_TITLE = "*********** start of CM DYNVMLC"
SECJAWS_TITLE = "*********** start of CM JAWS with identifier SECJAWS"


def read_dynvmlc(path) -> DynVMLC:
    """The CM DYNVMLC block in the order the reference reads it (init.cu:345-460,
    read_mlcinp.cpp:6-186); the medium is the line four lines after the leaf openings."""
    r = StreamReader(_read_text(path))
    if not r.find_line_starting(DYNVMLC_TITLE):
        raise ValueError(f"{path}: no '{DYNVMLC_TITLE}' block")
    rmax = r.num_sep(); r.ignore()
    r.ignore(); r.ignore()
    zmin = r.num_sep(); r.ignore()
    zthick = r.num_sep(); r.ignore()

    def leaf(order):
        vals = {k: r.num_sep() for k in order}
        return LeafType(**vals)

    full_order = ["wl", "wt", "wg", "wtip", "wts", "wbs", "ztip", "zl", "zt", "zg", "zth", "zbh", "holepos", "zts", "zbs"]
    target_order = ["wl", "wt", "wg", "wtip", "wts", "wbs", "zts", "zbs", "zth", "zbh", "holepos", "zt", "zg", "zl", "ztip"]
    full = leaf(full_order)
    target = leaf(target_order)
    iso = leaf(full_order)
    n_full = r.num_sep(int); r.ignore()
    n_half = r.num_sep(int); r.ignore()
    r.ignore()
    x_start = r.num_sep(); r.ignore()
    air_gap = r.num_sep(); r.ignore()
    r.ignore()
    rad_end = r.num_sep(); r.ignore()
    r.ignore()
    rows, total = [], 0
    while total < 60:
        neg, pos, num = r.num_sep(), r.num_sep(), r.num(int)
        rows.append((neg, pos, num))
        total += num
        if num <= 0:
            raise ValueError(f"{path}: leaf-opening row with NUM <= 0")
    r.ignore()          # end of the last opening row
    for _ in range(3):
        r.ignore()
    media = r.getline().strip()
    return DynVMLC(rmax=rmax, zmin=zmin, zthick=zthick, full=full, target=target, isocenter=iso,
                   n_full=n_full, n_half=n_half, x_start=x_start, air_gap=air_gap, rad_end=rad_end,
                   leaf_open=rows, media=media or "W700ICRU")


def dynvmlc_egsinp_text(m: DynVMLC) -> str:
    """A CM DYNVMLC block laid out line by line as read_dynvmlc (and the reference) read it."""
    f = lambda *v: ", ".join(f"{x:g}" for x in v) + ","
    L = lambda lt, order: [f(*[getattr(lt, k) for k in order[0:6]]), f(*[getattr(lt, k) for k in order[6:-3]]),
                           f(getattr(lt, order[-3])), f(*[getattr(lt, k) for k in order[-2:]])]
    full_order = ["wl", "wt", "wg", "wtip", "wts", "wbs", "ztip", "zl", "zt", "zg", "zth", "zbh", "holepos", "zts", "zbs"]
    tgt = ["wl", "wt", "wg", "wtip", "wts", "wbs", "zts", "zbs", "zth", "zbh", "holepos", "zt", "zg", "zl", "ztip"]
    tl = [f(*[getattr(m.target, k) for k in tgt[0:6]]), f(*[getattr(m.target, k) for k in tgt[6:10]]),
          f(m.target.holepos), f(*[getattr(m.target, k) for k in tgt[11:]])]
    lines = [DYNVMLC_TITLE + " with identifier MLC ***********", f"{m.rmax:g}, RMAX", "DYNVMLC", "0, IDMLFC",
             f"{m.zmin:g}, ZMIN", f"{m.zthick:g}, ZTHICK"]
    lines += L(m.full, full_order) + tl + L(m.isocenter, full_order)
    lines += [f"{m.n_full}, # FULL LEAVES ON LEFT", f"{m.n_half}, # HALF LEAF PAIRS", f"{m.n_full}, # FULL LEAVES ON RIGHT",
              f"{m.x_start:g}, START", f"{m.air_gap:g}, LEAFGAP", "0, ENDTYPE", f"{m.rad_end:g}, LEAFRADIUS",
              "0, ZFOCUS"]
    lines += [f"{neg:g}, {pos:g}, {num}" for neg, pos, num in m.leaf_open]
    lines += ["0.7, 0.01, 0, 0, ECUT, PCUT, DOSE ZONE, IREGION", "AIR700ICRU", "0, 0, 0, 0, ...", m.media]
    return "\n".join(lines) + "\n"


def secjaws_egsinp_text(j: SecJaws) -> str:
    """A CM JAWS block with identifier SECJAWS laid out as read_secjaws reads it."""
    lines = [SECJAWS_TITLE + " ***********", f"{j.rmax:g}, RMAX", "SECJAWS", "2, # PAIRED BARS OR JAWS",
             "Y", f"{j.zminy:g}, {j.zmaxy:g}, 0, 0, 0, 0,", "X", f"{j.zminx:g}, {j.zmaxx:g}, 0, 0, 0, 0,",
             "0.7, 0.01, 0, 0,", "0, 0, 0, 0,", j.media]
    return "\n".join(lines) + "\n"


def write_mlcinfo(path, fields):
    """fields: dicts with angle, x1, x2, y1, y2, mu, mlcinp (file name)."""
    lines = ["MLC fields", f"{len(fields)}"]
    for i, f in enumerate(fields):
        lines.append(f"{i + 1}, {f['angle']:g}, {f['x1']:g}, {f['x2']:g}, {f['y1']:g}, {f['y2']:g}, {int(f['mu'])}, {f['mlcinp']}")
    Path(path).write_text("\n".join(lines) + "\n")


def write_mlcinp(path, pos):
    """14 header lines, then 120 lines 'Leaf  nA = value' (banks A then B)."""
    pos = np.asarray(pos, np.float32)
    lines = ["File Rev = H", "Treatment = Static", "Last Name = synthetic", "First Name = ", "Patient ID = ",
             "Number of Fields = 1", "Number of Leaves = 120", "Tolerance = 0.50", "", "Field = 1", "Index = 0.0000",
             "Carriage Group = 1", "Operator = ", "Collimator = 0.0"]
    for j in range(120):
        bank, n = ("A", j + 1) if j < 60 else ("B", j - 59)
        lines.append(f"Leaf{n:3d}{bank} = {float(pos[j]):.9g}")
    Path(path).write_text("\n".join(lines) + "\n")


def read_secjaws(path) -> SecJaws:
    """The SECJAWS block as read_egsinp_secjaws reads it (init.cu:611-689)."""
    r = StreamReader(_read_text(path))
    if not r.find_line_starting(SECJAWS_TITLE):
        raise ValueError(f"{path}: no '{SECJAWS_TITLE}' block")
    rmax = r.num_sep(); r.ignore()
    for _ in range(3):
        r.ignore()
    zminy = r.num_sep(); zmaxy = r.num_sep(); r.ignore()
    r.ignore()
    zminx = r.num_sep(); zmaxx = r.num_sep(); r.ignore()
    r.ignore()
    r.ignore()
    media = r.getline().strip()
    return SecJaws(rmax=rmax, zminy=zminy, zmaxy=zmaxy, zminx=zminx, zmaxx=zmaxx, media=media)


# ---------------------------------------------------------------------------
# mlcinfo / mlcinp / output factors
# ---------------------------------------------------------------------------
def read_mlcinfo(path, max_fields=64):
    """Fields: index, gantry angle, jaws x1 x2 y1 y2, MU and the mlcinp file name."""
    r = StreamReader(_read_text(path))
    r.ignore()
    n = r.num(int); r.ignore()
    fields = []
    for _ in range(min(n, max_fields)):
        if r.eof():
            break
        idx = r.num_sep(int)
        angle, x1, x2, y1, y2 = (r.num_sep() for _ in range(5))
        mu = r.num_sep(int)
        name = r.getline().strip()
        fields.append(dict(index=idx, angle=angle, x1=x1, x2=x2, y1=y1, y2=y2, mu=mu, mlcinp=name))
    return fields


def read_mlcinp(path):
    """120 leaf positions: 14 header lines, then one position per line after
    up to 10 leading characters (the leaf label)."""
    r = StreamReader(_read_text(path))
    for _ in range(14):
        r.ignore()
    pos = np.empty(120, np.float32)
    for j in range(120):
        r.ignore(10, "\n")
        pos[j] = r.num()
        r.ignore()
    return pos


def read_output_factors(path):
    """(field size, output factor) table: a title line, the count, then pairs."""
    r = StreamReader(_read_text(path))
    r.ignore()
    n = r.num(int); r.ignore()
    tab = []
    for _ in range(n):
        a, b = r.num(), r.num()
        r.ignore()
        tab.append((a, b))
    return np.array(tab, np.float32)


def output_factor(table, x1, x2, y1, y2):
    """Linear interpolation in sqrt(field area), in float (read_mlcinp,
    init.cu:1449-1458). A field size outside the table leaves the reference's
    factor unset, which is 0 in its zero-initialised field array; None here,
    for the caller to report and apply as 0."""
    f = np.float32
    tab = np.asarray(table, np.float32)
    size = np.sqrt((f(x2) - f(x1)) * (f(y2) - f(y1)))
    for j in range(len(tab) - 1):
        if tab[j, 0] < size <= tab[j + 1, 0]:
            return float(tab[j, 1] + (size - tab[j, 0]) * (tab[j + 1, 1] - tab[j, 1]) / (tab[j + 1, 0] - tab[j, 0]))
    return None


# ---------------------------------------------------------------------------
# dose output
# ---------------------------------------------------------------------------
def dose_from_energy(energy, voxel_mass, dose_unit):
    """Dose per voxel in float32 from the energy in MeV (double), as write_dose
    computes it (output.c:887-891): (float)E / mass * dose_unit, in float."""
    e = np.asarray(energy, np.float64).astype(np.float32)
    return (e / np.asarray(voxel_mass, np.float32)) * np.float32(dose_unit)


def dose_file_name(base, nx, ny, nz):
    return f"{base}_DoseResults_{nx:03d}x{ny:03d}x{nz:03d}.bin"


def write_dose(base, dose, nx, ny, nz):
    """Raw float32 dose, x fastest, as write_dose writes it; returns the file name."""
    d = np.ascontiguousarray(dose, np.float32).reshape(-1)
    if d.size != nx * ny * nz:
        raise ValueError("dose size does not match the phantom")
    name = dose_file_name(base, nx, ny, nz)
    d.tofile(name)
    return name


def write_uncertainty(base, sigma, nx, ny, nz):
    """Raw float32 relative uncertainty per voxel, x fastest, under the
    reference's file name `<base>_uncertianty_NNNxNNNxNNN.bin` (its spelling,
    output.c:920-944); returns the file name."""
    d = np.ascontiguousarray(sigma, np.float32).reshape(-1)
    if d.size != nx * ny * nz:
        raise ValueError("uncertainty size does not match the phantom")
    name = f"{base}_uncertianty_{nx:03d}x{ny:03d}x{nz:03d}.bin"
    d.tofile(name)
    return name


def read_dose(path):
    m = re.search(r"_DoseResults_(\d+)x(\d+)x(\d+)\.bin$", str(path))
    if not m:
        raise ValueError(f"{path}: not a dose file name")
    nx, ny, nz = (int(g) for g in m.groups())
    return np.fromfile(path, np.float32).reshape(nz, ny, nx)
