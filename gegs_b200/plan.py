"""A treatment plan from the reference's ``.ini`` input (CUDA_EGS.cu:907-1694).

``read_ini`` reads the file with the rules of the Windows profile API the
reference calls (sections and keys case-insensitive, surrounding quotes
removed); ``load_plan`` turns it into a transport job: the egsphant phantom,
the phase space, the secondary jaws and DYNVMLC from the egsinp file, the
fields of the mlcinfo file with their mlcinp leaf positions, history counts
per field (MU x histories per MU, phase-space recycling as in runSimulation,
CUDA_EGS.cu:377-391) and the dose unit (CUDA_EGS.h:536, CUDA_EGS.cu:1478).

Paths: the reference prefixes every data file with ``<data directory>\\``;
Windows separators are accepted, and a relative data directory is taken
relative to the directory of the INI file.

Supported sections: General, Data, Phase space, SecJaws, MLC, Phantom,
Calibration, Output factor, Interpolation, and [Dose output] (point dose and
the relative-dose comparison with measured detector-array data). The physics tables are built by this package's
table generator for the media the phantom and the beam line name (a PEGS4
file named under [Data] is not read). Not supported, with a clear error when
switched on: Block and Wedge modules, CTcreate from DICOM.
"""
from __future__ import annotations

import os
import re
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import geometry as G
from . import io_formats as F
from . import physics_data as PD
from .workloads import SEED_BASE, Job

DOSE_UNIT = 1.6e-8          # MeV/g -> cGy (CUDA_EGS.h:536)


class PlanError(ValueError):
    pass


def read_ini(path) -> dict:
    sections: dict = {}
    cur = None
    for raw in Path(path).read_text(encoding="latin-1").splitlines():
        line = raw.strip()
        if not line or line.startswith(";") or line.startswith("#"):
            continue
        m = re.match(r"^\[(.+)\]$", line)
        if m:
            cur = sections.setdefault(m.group(1).strip().lower(), {})
            continue
        if "=" not in line or cur is None:
            continue
        k, v = line.split("=", 1)
        v = v.strip()
        if len(v) >= 2 and v[0] == v[-1] and v[0] in "\"'":
            v = v[1:-1]
        cur[k.strip().lower()] = v
    return sections


def _get(ini, sec, key, default=None, required=False):
    v = ini.get(sec.lower(), {}).get(key.lower())
    if v is None:
        if required:
            raise PlanError(f'property "{key}" is not specified in the section "{sec}"')
        return default
    return v


def _on(v, default=False):
    if v is None:
        return default
    return v.strip().lower() in ("on", "yes", "true", "1")


def _floats(v, n, what):
    """The first n numbers of an INI value, each rounded once to float, as the
    reference's sscanf("%f") reads them (CUDA_EGS.cu:1076-1680)."""
    try:
        vals = [float(F.strtof(t)) for t in v.split()]
    except (AttributeError, ValueError):
        raise PlanError(f"could not parse {what} {v!r}")
    if len(vals) < n:
        raise PlanError(f"{what} needs {n} numbers, got {v!r}")
    return vals[:n]


def _path(base_dir, rel):
    p = rel.replace("\\", "/")
    return str((Path(base_dir) / p).resolve()) if not os.path.isabs(p) else p


@dataclass
class Plan:
    job: Job
    prefix: str
    output_dir: str
    histories_per_mu: float
    dose_unit: float
    field_output_factors: list
    log: list = field(default_factory=list)
    post: dict = field(default_factory=dict)      # interpolation grid, point-dose position
    nx: int = 0
    ny: int = 0
    nz: int = 0

    @property
    def output_base(self):
        return str(Path(self.output_dir) / self.prefix)


def load_plan(ini_path, seed=SEED_BASE, max_histories=None) -> Plan:
    ini_path = Path(ini_path).resolve()
    ini = read_ini(ini_path)
    here = ini_path.parent
    log = []
    prefix = _get(ini, "General", "output prefix", required=True)
    outdir = _path(here, _get(ini, "General", "output directory", required=True))
    hpm = _floats(_get(ini, "General", "histories", required=True), 1, "histories")[0]
    data_dir = _path(here, _get(ini, "Data", "data directory", required=True))
    data = lambda name: _path(data_dir, name)
    default_medium = _get(ini, "Data", "default medium", "AIR700ICRU")
    egsinp = data(_get(ini, "Data", "egsinp file", required=True))

    # modules
    secjaws_on = _on(_get(ini, "SecJaws", "module SecJaws"))
    mlc_on = _on(_get(ini, "MLC", "module MLC"))
    for sec, key in (("Block", "module Block"), ("Wedge", "module Wedge")):
        if _on(_get(ini, sec, key)):
            raise PlanError(f"the {sec} module is not supported by this transport path")
    if _on(_get(ini, "CTcreate", "use ctcreate")):
        raise PlanError("building the phantom from DICOM (use ctcreate = Yes) is not supported; "
                        "give an egsphant file and set use ctcreate = No")

    # phantom
    ph = F.read_egsphant(data(_get(ini, "Phantom", "egsphant file", required=True)))
    change_xyz = _get(ini, "Phantom", "change coordinate", "Yes").strip().lower() != "no"
    iso = _floats(_get(ini, "Phantom", "isocenter location", required=True), 3, "isocenter location")
    sid = _floats(_get(ini, "Phantom", "source to isocenter", required=True), 1, "source to isocenter")[0]

    # beam-line geometry
    jaws = F.read_secjaws(data(_get(ini, "SecJaws", "secjaws file", "VarianMLC.egsinp"))) if secjaws_on else None
    mlc = F.read_dynvmlc(egsinp) if mlc_on else None
    # region media: phantom media first, then default / jaws / MLC / block / wedge (init.cu:1322-1352)
    media = list(ph["media"])
    other_names = [default_medium, jaws.media if jaws else default_medium, mlc.media if mlc else default_medium,
                   default_medium, default_medium]
    for n in other_names:
        if n not in media:
            media.append(n)
    unknown = [m for m in media if m not in PD.MEDIA]
    if unknown:
        raise PlanError(f"no physics data for media {unknown}; known: {sorted(PD.MEDIA)}")
    phys = PD.build_block(media, mlc_media=[mlc.media] if mlc else [])
    rho = np.array([PD.MEDIA[m].rho for m in media], np.float32)
    med = ph["voxel_med"].astype(np.uint16)
    dens = ph["density"]
    rhof = (dens / rho[med]).astype(np.float32)
    rhof[dens == 0] = 1.0
    phantom = dict(x_bounds=ph["x_bounds"], y_bounds=ph["y_bounds"], z_bounds=ph["z_bounds"], voxel_med=med,
                   voxel_rhof=rhof, density=dens, other_med=[media.index(n) for n in other_names], media=media)

    # phase space
    nfiles = int(_floats(_get(ini, "Phase space", "phsp file number", "1"), 1, "phsp file number")[0])
    base = data(_get(ini, "Phase space", "phase space file", required=True))
    recs = F.read_phase_space(base, nfiles)
    z_phsp = _floats(_get(ini, "Phase space", "z position", required=True), 1, "z position")[0]
    if len(recs) == 0:
        raise PlanError("the phase space holds no particles")

    # fields
    # the mlcinfo file carries the fields (angle, jaws, MU) even when the MLC module is off
    mlcinfo = _get(ini, "MLC", "mlcinfo file", required=mlc_on)
    if mlcinfo is not None:
        finfo = F.read_mlcinfo(data(mlcinfo))
        for f in finfo:
            f["leaf_pos"] = F.read_mlcinp(data(f["mlcinp"])) if mlc_on else None
    else:
        finfo = [dict(index=1, angle=0.0, x1=-20.0, x2=20.0, y1=-20.0, y2=20.0, mu=1, leaf_pos=None)]
    if not finfo:
        raise PlanError("the mlcinfo file lists no fields")
    ofac = [1.0] * len(finfo)
    if _on(_get(ini, "Output factor", "use output factor")):
        tab = F.read_output_factors(data(_get(ini, "Output factor", "output factor file", required=True)))
        ofac = [F.output_factor(tab, f["x1"], f["x2"], f["y1"], f["y2"]) for f in finfo]
        for k, of in enumerate(ofac):
            if of is None:
                log.append(f"field {k + 1}: field size outside the output-factor table; its output factor is 0, "
                           "as the reference leaves it")
        ofac = [0.0 if of is None else of for of in ofac]
    mg = mlc.build() if mlc else None
    fields, h = [], 0
    for f in finfo:
        n = int(f["mu"] * int(hpm))
        if max_histories is not None:
            n = min(n, max_histories)
        nrep = (n - 1) // len(recs) if n > 0 else 0
        if nrep > 255:
            raise PlanError("more than 256 uses of each phase-space particle; add phase-space particles")
        c, s = G.gantry_cos_sin(f["angle"])
        fd = dict(cos_angle=c, sin_angle=s, hist_begin=h, hist_end=h + n, nrepeat=nrep, angle=f["angle"],
                  jaws=(f["x1"], f["x2"], f["y1"], f["y2"]))
        if jaws:
            fd.update(G.secjaws_polygons(jaws, f["x1"], f["x2"], f["y1"], f["y2"], sid))
        if mlc:
            fd["leaf_pos"] = f["leaf_pos"]
            fd["endnode"] = G.leaf_endnodes(mg["crossYZ"], f["leaf_pos"], mlc.zmin, mlc.zthick, sid)
        fields.append(fd)
        h += n
    beam = dict(change_xyz=change_xyz, source_to_isocenter=sid, iso=tuple(iso), z_phsp=z_phsp,
                module_order=G.module_order(secjaws_on, mlc_on), mlc=mg)
    # dose_unit is a float in the reference (CUDA_EGS.h:536), scaled in float (CUDA_EGS.cu:1478)
    f32 = np.float32
    dose_unit = float(f32(DOSE_UNIT))
    if _on(_get(ini, "Calibration", "dose calibration")):
        hpc = _floats(_get(ini, "Calibration", "histories per cGy", required=True), 1, "histories per cGy")[0]
        dose_unit = float(f32(DOSE_UNIT) * f32(hpc) / f32(hpm))
    post = {}
    if _on(_get(ini, "Interpolation", "do interpolate")):
        post["interp"] = dict(
            start=_floats(_get(ini, "Interpolation", "starting point", required=True), 3, "starting point"),
            dims=[int(v) for v in _floats(_get(ini, "Interpolation", "xyz dimensions", required=True), 3,
                                          "xyz dimensions")],
            sizes=_floats(_get(ini, "Interpolation", "3d voxel sizes", required=True), 3, "3d voxel sizes"))
    if _on(_get(ini, "Dose output", "absolute dose")):
        post["point"] = dict(
            pos=_floats(_get(ini, "Dose output", "dose position", required=True), 3, "dose position"),
            measured=_floats(_get(ini, "Dose output", "dose measured", "0"), 1, "dose measured")[0])
    if _on(_get(ini, "Dose output", "relative dose")):
        start = _floats(_get(ini, "Dose output", "starting point", required=True), 3, "starting point")
        arr = (_get(ini, "Dose output", "PTW729/PTW1000", "") or "").strip()
        norm = (_get(ini, "Dose output", "norm to Max/Center", "") or "").strip()
        gl, gd = _floats(_get(ini, "Dose output", "gamma index (mm,%)", required=True), 2, "gamma index (mm,%)")
        meas = _get(ini, "Dose output", "measured data", required=True)
        post["relative"] = dict(
            start=[float(np.float32(start[k]) + np.float32(iso[k])) for k in range(3)],    # float sum (CUDA_EGS.cu:1617-1619)
            dims=[int(v) for v in _floats(_get(ini, "Dose output", "xyz dimensions", required=True), 3,
                                          "xyz dimensions")],
            sizes=_floats(_get(ini, "Dose output", "3d voxel sizes", required=True), 3, "3d voxel sizes"),
            array_type=1 if arr == "PTW729" else 2, norm_type=1 if norm == "Max" else (2 if norm == "Center" else 0),
            gamma_len_cm=float(np.float32(gl) * np.float32(0.1)), gamma_dos=float(np.float32(gd) * np.float32(0.01)), measured=data(meas), iso=list(iso))
    job = Job(f"plan {prefix}", media, phys, phantom, beam, fields, recs, h,
              meta=dict(seed=seed, mlc=mlc, jaws=jaws, ini=str(ini_path)))
    return Plan(job=job, prefix=prefix, output_dir=outdir, histories_per_mu=hpm, dose_unit=dose_unit,
                field_output_factors=ofac, log=log, nx=ph["nx"], ny=ph["ny"], nz=ph["nz"], post=post)
