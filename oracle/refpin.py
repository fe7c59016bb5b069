"""The reference's own routines beside the oracle's, on identical inputs
(test infrastructure only).

``oracle/ref`` compiles the reference's device sources, as they are, into
``oracle/_ref/libgegs_ref.so`` (host code; see oracle/ref/Makefile). This
module loads it and the oracle, and runs the same particles through both:

* geometry: ``howfar`` / ``hownear`` of the phantom, the DYNVMLC and the
  secondary jaws (geom.cu:54-1543);
* direction rotations ``uphi21 / uphi32 / uphi11`` (utility.cu:94-218);
* one pass of each stage kernel -- photon step, Compton, photo, Rayleigh,
  pair, electron step, Moller, brems, Bhabha, annihilation -- per particle.
  The oracle draws its uniforms from its own counter-based stream and records
  them; the reference is fed the same values through its curand_uniform in
  the order it asks for them. Equal outputs mean equal branches, equal
  operation order and equal use of the random numbers.

The library only exists where the reference sources were available when
``build()`` ran (``REF_DIR``); callers skip when :func:`available` is False.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib
import subprocess

import numpy as np

from . import oracle as O

HERE = pathlib.Path(__file__).resolve().parent
REF_LIB = HERE / "_ref" / "libgegs_ref.so"
REF_DIR = pathlib.Path(os.environ.get("GEGS_REFERENCE_DIR", "/root/reference"))

PARTICLE = np.dtype([("region", "<u4"), ("charge", "i1"), ("leafIndex", "i1"), ("bank", "i1"), ("module", "u1"),
                     ("field", "u1"), ("status", "u1"), ("pad0", "u1"), ("pad1", "u1"),
                     ("wt", "<f4"), ("e", "<f4"), ("x", "<f4"), ("y", "<f4"), ("z", "<f4"),
                     ("u", "<f4"), ("v", "<f4"), ("w", "<f4"), ("dnear", "<f4"), ("hist", "<u4"), ("pad2", "<u4")])
assert PARTICLE.itemsize == 56

STAGES = ["photon", "compton", "photo", "rayleigh", "pair", "electron", "moller", "brems", "bhabha", "annih"]


def build(force=False):
    """Build the harness from the reference sources when they are present."""
    if not REF_DIR.is_dir():
        return None
    srcs = [p for p in (HERE / "ref").rglob("*") if p.is_file()] + [HERE / "ora_base.c", HERE / "gegs_oracle.h"]
    if force or not REF_LIB.exists() or any(s.stat().st_mtime > REF_LIB.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-s", "-C", str(HERE / "ref"), f"REF={REF_DIR}"], check=True)
    return REF_LIB


def available() -> bool:
    return REF_LIB.exists()


_lib = None
_loaded = None          # the Pair whose plan the harness's globals hold


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(str(REF_LIB))
        vp = C.c_void_p
        L.ref_load.argtypes = [vp, vp]
        L.ref_select_field.argtypes = [C.c_int]
        L.ref_probe_geom.argtypes = [C.c_uint32, vp, vp, vp, vp, vp, vp]
        L.ref_probe_uphi.argtypes = [C.c_int, C.c_float, C.c_float, vp, vp, C.c_float]
        L.ref_probe_stage.argtypes = [C.c_int, C.c_uint32, vp, vp, vp, C.c_uint32, vp, C.c_uint32, vp, vp, vp,
                                      C.c_uint32, vp, vp]
        L.ref_setup_run.argtypes = [C.c_char_p] * 6 + [C.c_float, C.c_char_p, C.c_char_p, C.c_size_t]
        L.ref_setup_get.argtypes = [C.c_char_p, C.c_int, vp, C.c_size_t]
        L.ref_setup_get.restype = C.c_long
        L.ref_transport.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, vp, C.c_uint64]
        L.ref_transport.restype = C.c_long
        _lib = L
    return _lib


def _ora():
    L = O.lib()
    vp = C.c_void_p
    L.ora_probe_geom.argtypes = [vp, vp, C.c_uint32, vp, vp, vp, vp, vp, vp]
    L.ora_probe_stage.argtypes = [vp, vp, C.c_int, C.c_uint32, vp, vp, C.c_uint32, vp, vp, C.c_uint32, vp, vp, vp,
                                  C.c_uint32, vp]
    L.ora_probe_uphi.argtypes = [C.c_int, C.c_float, C.c_float, vp, vp, vp]
    L.ora_capture.argtypes = [vp, vp, C.c_uint64, C.c_uint64, C.c_uint32, vp, C.c_uint32, vp]
    return L


class OraclePair:
    """The oracle side alone (no reference harness needed): the same probes
    as :class:`Pair`, for checking the oracle against recorded outputs."""

    def __init__(self, physics, scene_holder):
        self.phys = np.ascontiguousarray(physics)
        self.sh = scene_holder
        self.scene_ptr = C.addressof(scene_holder.scene)

    def capture(self, h0, h1, every=1, cap_n=4096):
        """Particles as they enter each stage in an oracle run: {stage: array}."""
        cap = np.zeros(10 * cap_n, PARTICLE)
        n = np.zeros(10, np.uint32)
        _ora().ora_capture(self.phys.ctypes.data, self.scene_ptr, h0, h1, every, cap.ctypes.data, cap_n,
                           n.ctypes.data)
        return {s: cap[s * cap_n: s * cap_n + int(n[s])].copy() for s in range(10)}

    def geom(self, parts, t_in):
        parts = np.ascontiguousarray(parts, PARTICLE)
        t_in = np.ascontiguousarray(t_in, np.float32)
        n = len(parts)
        reg, t, po, tn = np.zeros(n, np.uint32), np.zeros(n, np.float32), np.zeros(n, PARTICLE), np.zeros(n, np.float32)
        _ora().ora_probe_geom(self.phys.ctypes.data, self.scene_ptr, n, parts.ctypes.data, t_in.ctypes.data,
                              reg.ctypes.data, t.ctypes.data, po.ctypes.data, tn.ctypes.data)
        return dict(region=reg, t=t, particle=po, tperp=tn)

    def stage(self, stage, parts, ucap=4096, ocap=64, dcap=4096):
        """One pass of `stage` per particle: the uniforms drawn, pushed
        particles and escore calls (counts may exceed capacities: raises)."""
        parts = np.ascontiguousarray(parts, PARTICLE)
        n = len(parts)
        u, un = np.zeros(n * ucap, np.float32), np.zeros(n, np.uint32)
        out, on = np.zeros(n * ocap, PARTICLE), np.zeros(n, np.uint32)
        dreg, de, dn = np.zeros(n * dcap, np.uint32), np.zeros(n * dcap, np.float32), np.zeros(n, np.uint32)
        err = _ora().ora_probe_stage(self.phys.ctypes.data, self.scene_ptr, stage, n, parts.ctypes.data,
                                     u.ctypes.data, ucap, un.ctypes.data, out.ctypes.data, ocap, on.ctypes.data,
                                     dreg.ctypes.data, de.ctypes.data, dcap, dn.ctypes.data)
        if np.any(un > ucap) or np.any(on > ocap) or np.any(dn > dcap):
            # run again with room for the longest particle (each particle has its own stream)
            return OraclePair.stage(self, stage, parts, max(ucap, int(un.max())), max(ocap, int(on.max())),
                              max(dcap, int(dn.max())))
        return dict(err=err, ucap=ucap, ocap=ocap, dcap=dcap, u=u.reshape(n, ucap), un=un, used=un.copy(), out=out.reshape(n, ocap), on=on,
                    dreg=dreg.reshape(n, dcap), de=de.reshape(n, dcap), dn=dn)

    def uphi(self, which, a, b, part, cs=(0.0, 0.0)):
        p = np.ascontiguousarray(np.array([part], PARTICLE))
        c = np.array([cs[0], cs[1], 0.0, 0.0], np.float32)
        u = C.c_float(0.0)
        _ora().ora_probe_uphi(which, a, b, p.ctypes.data, c.ctypes.data, C.byref(u))
        return p[0], c, u.value


class Pair(OraclePair):
    """The reference harness and the oracle, loaded with one physics block and scene."""

    def __init__(self, physics, scene_holder):
        super().__init__(physics, scene_holder)
        self._load()

    def _load(self):
        """Fill the harness's reference globals from this pair's plan (they are
        per process, and the last pair made or used owns them)."""
        global _loaded
        if _loaded is not self:
            if lib().ref_load(self.phys.ctypes.data, self.scene_ptr) != 0:
                raise RuntimeError("ref_load failed")
            _loaded = self

    def geom(self, parts, t_in):
        """howfar / hownear on both sides: {"ora": ..., "ref": ...}."""
        self._load()
        parts = np.ascontiguousarray(parts, PARTICLE)
        t_in = np.ascontiguousarray(t_in, np.float32)
        n = len(parts)
        reg, t, po, tn = np.zeros(n, np.uint32), np.zeros(n, np.float32), np.zeros(n, PARTICLE), np.zeros(n, np.float32)
        bad = lib().ref_probe_geom(n, parts.ctypes.data, t_in.ctypes.data, reg.ctypes.data, t.ctypes.data,
                                   po.ctypes.data, tn.ctypes.data)
        if bad != 0:
            raise RuntimeError(f"reference geometry: {bad} particles in a module it has no routine for")
        return {"ora": super().geom(parts, t_in), "ref": dict(region=reg, t=t, particle=po, tperp=tn)}

    def stage(self, stage, parts, ucap=4096, ocap=64, dcap=4096):
        """One pass of `stage` per particle on both sides; the reference is fed
        the uniforms the oracle drew for each particle."""
        self._load()
        parts = np.ascontiguousarray(parts, PARTICLE)
        n = len(parts)
        ora = super().stage(stage, parts, ucap, ocap, dcap)
        ucap, ocap, dcap = ora["ucap"], ora["ocap"], ora["dcap"]
        out, on = np.zeros(n * ocap, PARTICLE), np.zeros(n, np.uint32)
        dreg, de, dn = np.zeros(n * dcap, np.uint32), np.zeros(n * dcap, np.float32), np.zeros(n, np.uint32)
        used = np.zeros(n, np.uint32)
        u = np.ascontiguousarray(ora["u"])
        err = lib().ref_probe_stage(stage, n, parts.ctypes.data, u.ctypes.data, ora["un"].ctypes.data, ucap,
                                    out.ctypes.data, ocap, on.ctypes.data, dreg.ctypes.data, de.ctypes.data, dcap,
                                    dn.ctypes.data, used.ctypes.data)
        ref = dict(err=err, used=used, out=out.reshape(n, ocap), on=on, dreg=dreg.reshape(n, dcap),
                   de=de.reshape(n, dcap), dn=dn)
        return {"ora": ora, "ref": ref}

    def uphi(self, which, a, b, part, cs=(0.0, 0.0)):
        """(oracle, reference) results of one rotation: particle and cos/sin pairs."""
        self._load()
        po, co, u = super().uphi(which, a, b, part, cs)
        p = np.ascontiguousarray(np.array([part], PARTICLE))
        c = np.array([cs[0], cs[1], 0.0, 0.0], np.float32)
        lib().ref_probe_uphi(which, a, b, p.ctypes.data, c.ctypes.data, u)
        return (po, co), (p[0], c)

    def transport(self, h0, h1, seed=1):
        """Histories [h0, h1) transported by the reference's own kernels (one
        CPU thread, a seeded generator for the random numbers): energy per
        voxel in MeV."""
        L = lib()
        self._load()
        nvox = self.sh.scene.nx * self.sh.scene.ny * self.sh.scene.nz
        tally = np.zeros(nvox, np.float64)
        over = L.ref_transport(h0, h1, seed, tally.ctypes.data, nvox)
        if over != 0:
            raise RuntimeError(f"reference transport: {over} stack overflows")
        return tally


def sort_by_stack(out, on):
    """Pushed particles of one probe as a list sorted by stack, push order kept."""
    rows = out[:int(on)]
    return rows[np.argsort(rows["status"], kind="stable")]


class Setup:
    """The reference's host set-up run on plan files: init_phantom_and_MLC
    (the egsphant, the SECJAWS and DYNVMLC blocks of the egsinp files),
    read_mlcinp (the mlcinfo field list and the mlcinp leaf positions) and,
    per field, setup_secjaws, init_leaf_pos and the gantry cosine and sine
    (init.cu:256-906, 1164-1662; CUDA_EGS.cu:420-422)."""

    FIELD = ("angle", "x1", "x2", "y1", "y2", "mu", "output_factor", "cos_angle", "sin_angle", "angle_rad")

    def __init__(self, egsphant, mlc_egsinp, jaws_egsinp, mlcinfo, data_dir, sid, default_medium,
                 output_factor_file=None):
        global _loaded
        L = lib()
        _loaded = None                      # the set-up overwrites the reference's globals
        msg = C.create_string_buffer(512)
        d = str(data_dir).rstrip("/") + "/"          # the reference prepends it to each mlcinp name
        st = L.ref_setup_run(str(egsphant).encode(), str(mlc_egsinp).encode(), str(jaws_egsinp).encode(),
                             str(mlcinfo).encode(), d.encode(),
                             None if output_factor_file is None else str(output_factor_file).encode(),
                             float(sid), default_medium.encode(), msg, len(msg))
        if st != 0:
            raise RuntimeError(f"reference set-up: {msg.value.decode()}")
        self.nfields = int(self.get("nfields", np.int32)[0])

    def get(self, name, dtype, field=-1):
        L = lib()
        n = L.ref_setup_get(name.encode(), field, None, 0)
        if n < 0:
            raise KeyError(name)
        buf = np.zeros(n, np.uint8)
        L.ref_setup_get(name.encode(), field, buf.ctypes.data, n)
        return buf.view(dtype) if dtype is not None else buf.tobytes()

    def field(self, f):
        v = self.get("field", np.float32, f)
        return dict(zip(self.FIELD, v))
