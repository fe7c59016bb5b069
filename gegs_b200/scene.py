"""ctypes mirror of ``include/gegs_scene.h`` and a builder that keeps the
numpy buffers alive while C code holds pointers into them."""
from __future__ import annotations

import ctypes as C

import numpy as np

N_LEAF_PAIRS = 60
MAX_FIELDS = 32
VACUUM_MED = 0xFFFF

M_FIRST, M_SECJAWY, M_SECJAWX, M_VARMLC, M_WEDGE, M_BLOCK, M_PHANTOM = range(7)
F_RAYLEIGH, F_BOUND_COMPTON, F_ATOMIC_RELAXATION, F_PHOTO_ANGULAR = 0x1, 0x2, 0x10, 0x20
DEFAULT_REGION_FLAGS = F_RAYLEIGH | F_BOUND_COMPTON | F_ATOMIC_RELAXATION | F_PHOTO_ANGULAR


class PhspRecord(C.Structure):
    _fields_ = [("latch", C.c_uint32), ("e", C.c_float), ("x", C.c_float), ("y", C.c_float),
                ("u", C.c_float), ("v", C.c_float), ("wt", C.c_float)]


PHSP_DTYPE = np.dtype([("latch", "<u4"), ("e", "<f4"), ("x", "<f4"), ("y", "<f4"),
                       ("u", "<f4"), ("v", "<f4"), ("wt", "<f4")])

F2 = C.c_float * 2


class Field(C.Structure):
    _fields_ = [
        ("cos_angle", C.c_float), ("sin_angle", C.c_float),
        ("hist_begin", C.c_uint64), ("hist_end", C.c_uint64),
        ("nrepeat", C.c_int32), ("pad_", C.c_int32),
        ("boundMinY", F2 * 4), ("boundMinX", F2 * 4),
        ("boundMaxY", F2 * 4), ("boundMaxX", F2 * 4),
        ("jawsGeomY", F2 * 8), ("jawsGeomX", F2 * 8),
        ("endnode", (F2 * 34) * N_LEAF_PAIRS),
    ]


class Scene(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("x_bounds", C.POINTER(C.c_float)), ("y_bounds", C.POINTER(C.c_float)),
        ("z_bounds", C.POINTER(C.c_float)),
        ("voxel_med", C.POINTER(C.c_uint16)), ("voxel_rhof", C.POINTER(C.c_float)),
        ("other_med", C.c_int32 * 5), ("region_flags", C.c_uint32),
        ("change_xyz", C.c_int32), ("source_to_isocenter", C.c_float),
        ("iso", C.c_float * 3), ("z_phsp", C.c_float), ("module_order", C.c_int8 * 8),
        ("mlc_rmax", C.c_float), ("mlc_zmin", C.c_float), ("mlc_zthick", C.c_float),
        ("mlc_x_start", C.c_float), ("mlc_x_end", C.c_float), ("mlc_x_mid_1", C.c_float),
        ("mlc_x_mid_2", C.c_float), ("mlc_air_gap", C.c_float), ("mlc_wl_full", C.c_float),
        ("mlc_wl_target", C.c_float), ("mlc_wl_isocenter", C.c_float), ("mlc_wt", C.c_float),
        ("crossXZ", F2 * 960), ("boundaryXZ", F2 * 4), ("boundaryYZ", F2 * 4),
        ("nfields", C.c_int32), ("fields", C.POINTER(Field)),
        ("phsp", C.POINTER(PhspRecord)), ("nphsp", C.c_uint64),
        ("hownear_region_offset", C.c_int32), ("pad2_", C.c_int32), ("seed", C.c_uint64),
        ("bl_nx", C.c_int32), ("bl_ny", C.c_int32), ("bl_x0", C.c_float), ("bl_y0", C.c_float),
        ("bl_dx", C.c_float), ("bl_dy", C.c_float), ("bl_weight", C.POINTER(C.c_float)),
    ]


def _ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def fill_field(F, f):
    """A gegs_field from a field dict (cos_angle, sin_angle, hist_begin,
    hist_end, nrepeat and the polygons the field has)."""
    F.cos_angle, F.sin_angle = f["cos_angle"], f["sin_angle"]
    F.hist_begin, F.hist_end = int(f["hist_begin"]), int(f["hist_end"])
    F.nrepeat = int(f["nrepeat"])
    for k in ("boundMinY", "boundMinX", "boundMaxY", "boundMaxX", "jawsGeomY", "jawsGeomX", "endnode"):
        if k in f:
            a = np.ascontiguousarray(f[k], np.float32)
            C.memmove(C.addressof(getattr(F, k)), a.ctypes.data, a.nbytes)
    return F


class SceneHolder:
    """A filled :class:`Scene` plus the numpy arrays its pointers refer to."""

    def __init__(self, phantom, beam, fields, phsp, seed=0x6E65, hownear_region_offset=5,
                 region_flags=DEFAULT_REGION_FLAGS):
        self.keep = []
        s = Scene()
        xb = np.ascontiguousarray(phantom["x_bounds"], np.float32)
        yb = np.ascontiguousarray(phantom["y_bounds"], np.float32)
        zb = np.ascontiguousarray(phantom["z_bounds"], np.float32)
        med = np.ascontiguousarray(phantom["voxel_med"], np.uint16).reshape(-1)
        rhof = np.ascontiguousarray(phantom["voxel_rhof"], np.float32).reshape(-1)
        self.keep += [xb, yb, zb, med, rhof]
        s.nx, s.ny, s.nz = len(xb) - 1, len(yb) - 1, len(zb) - 1
        assert med.size == s.nx * s.ny * s.nz
        s.x_bounds, s.y_bounds, s.z_bounds = _ptr(xb, C.c_float), _ptr(yb, C.c_float), _ptr(zb, C.c_float)
        s.voxel_med = _ptr(med, C.c_uint16)
        s.voxel_rhof = _ptr(rhof, C.c_float)
        for i in range(5):
            s.other_med[i] = int(phantom["other_med"][i])
        s.region_flags = region_flags
        s.change_xyz = 1 if beam.get("change_xyz", True) else 0
        s.source_to_isocenter = beam.get("source_to_isocenter", 100.0)
        for i in range(3):
            s.iso[i] = beam["iso"][i]
        s.z_phsp = beam["z_phsp"]
        for i, v in enumerate(beam["module_order"]):
            s.module_order[i] = v
        mlc = beam.get("mlc")
        if mlc is not None:
            for k in ("rmax", "zmin", "zthick", "x_start", "x_end", "x_mid_1", "x_mid_2", "air_gap",
                      "wl_full", "wl_target", "wl_isocenter", "wt"):
                setattr(s, "mlc_" + k, float(mlc[k]))
            C.memmove(s.crossXZ, np.ascontiguousarray(mlc["crossXZ"], np.float32).ctypes.data, 960 * 8)
            C.memmove(s.boundaryXZ, np.ascontiguousarray(mlc["boundaryXZ"], np.float32).ctypes.data, 32)
            C.memmove(s.boundaryYZ, np.ascontiguousarray(mlc["boundaryYZ"], np.float32).ctypes.data, 32)
        nf = len(fields)
        if not 1 <= nf <= MAX_FIELDS:
            raise ValueError(f"1..{MAX_FIELDS} fields, got {nf}")
        farr = (Field * nf)()
        for i, f in enumerate(fields):
            fill_field(farr[i], f)
        self.fields_arr = farr
        s.nfields = nf
        s.fields = C.cast(farr, C.POINTER(Field))
        ph = np.ascontiguousarray(phsp, PHSP_DTYPE)
        self.keep.append(ph)
        s.phsp = ph.ctypes.data_as(C.POINTER(PhspRecord))
        s.nphsp = len(ph)
        s.hownear_region_offset = hownear_region_offset
        s.seed = seed
        bl = beam.get("beamlets")
        if bl is not None:
            s.bl_nx, s.bl_ny = int(bl["nx"]), int(bl["ny"])
            s.bl_x0, s.bl_y0, s.bl_dx, s.bl_dy = bl["x0"], bl["y0"], bl["dx"], bl["dy"]
            if nf * s.bl_nx * s.bl_ny >= 0xFFFF:
                raise ValueError("at most 65534 beamlets")
            if bl.get("weights") is not None:
                w = np.ascontiguousarray(bl["weights"], np.float32).reshape(-1)
                if w.size != nf * s.bl_nx * s.bl_ny:
                    raise ValueError(f"{w.size} beamlet weights for {nf * s.bl_nx * s.bl_ny} beamlets")
                self.keep.append(w)
                s.bl_weight = _ptr(w, C.c_float)
        self.nbeamlets = nf * s.bl_nx * s.bl_ny
        self.scene = s
        self.nvox = s.nx * s.ny * s.nz
        self.total_histories = max(int(f["hist_end"]) for f in fields)

    @property
    def ref(self):
        return C.byref(self.scene)
