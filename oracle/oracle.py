"""ctypes loader for the CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke`` and bench.py's CPU-baseline leg import
this module, as the checker.  ``build()`` compiles ``oracle/*.c`` with the
committed Makefile into ``oracle/_build/libgegs_oracle.so``.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB = HERE / "_build" / "libgegs_oracle.so"
# -O3 -march=native build for the timed CPU baseline, made on the host that times it
NATIVE_LIB = HERE / "_build_native" / "libgegs_oracle.so"


class Stats(C.Structure):
    _fields_ = [("counts", C.c_uint64 * 10), ("steps_photon", C.c_uint64), ("steps_electron", C.c_uint64),
                ("e_escaped", C.c_double), ("error", C.c_int32), ("pad_", C.c_int32),
                ("cnt", (C.c_uint64 * 3) * 10)]


def build(force=False):
    srcs = list(HERE.glob("*.c")) + list(HERE.glob("*.h")) + list((HERE.parent / "include").glob("*.h"))
    if force or not LIB.exists() or any(s.stat().st_mtime > LIB.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def build_native():
    """The host-tuned build of the same sources (same results bit for bit)."""
    srcs = list(HERE.glob("*.c")) + list(HERE.glob("*.h")) + list((HERE.parent / "include").glob("*.h"))
    if not NATIVE_LIB.exists() or any(s.stat().st_mtime > NATIVE_LIB.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-s", "-C", str(HERE), "native"], check=True)
    return NATIVE_LIB


_lib = None
_native = None


def lib(native=False):
    global _lib, _native
    if native:
        if _native is None:
            _native = _setup(C.CDLL(str(build_native())))
        return _native
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = _setup(C.CDLL(str(LIB)))
    return _lib


def _setup(L):
    if True:
        L.ora_log.restype = C.c_float
        L.ora_log.argtypes = [C.c_float]
        L.ora_exp.restype = C.c_float
        L.ora_exp.argtypes = [C.c_float]
        L.ora_sincos_turns.argtypes = [C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.ora_philox.restype = C.c_uint32
        L.ora_philox.argtypes = [C.c_uint32] * 6 + [C.c_int]
        L.ora_sizeof_physics.restype = C.c_size_t
        L.ora_sizeof_scene.restype = C.c_size_t
        L.ora_sizeof_field.restype = C.c_size_t
        L.ora_run.restype = C.c_int
        L.ora_run.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.c_int,
                              C.POINTER(C.c_int64), C.POINTER(Stats)]
        L.ora_set_trace.argtypes = [C.c_void_p, C.c_uint32]
        L.ora_trace_count.restype = C.c_uint32
    return L


TRACE_DTYPE = np.dtype([("kind_stage", "<u4"), ("hist_lo", "<u4"), ("sid_lo", "<u4"), ("sid_hi", "<u4"),
                        ("ctr", "<u4"), ("e", "<f4"), ("x", "<f4"), ("region", "<u4")])


def run_traced(physics, scene_holder, h0, h1, cap=1 << 20):
    """Single-threaded run that also returns the push/consume trace."""
    L = lib()
    buf = np.zeros(cap, TRACE_DTYPE)
    L.ora_set_trace(buf.ctypes.data, cap)
    try:
        tally, st = run(physics, scene_holder, h0, h1, threads=1)
        n = L.ora_trace_count()
    finally:
        L.ora_set_trace(None, 0)
    return tally, st, buf[:min(n, cap)]


def run(physics: np.ndarray, scene_holder, h0: int, h1: int, threads: int = 0, native: bool = False):
    """Run histories [h0, h1) on the CPU; returns (int64 tally, stats dict).
    native: the -O3 -march=native build (same results; for timing)."""
    L = lib(native)
    tally = np.zeros(scene_holder.nvox, np.int64)
    st = Stats()
    phys = np.ascontiguousarray(physics)
    rc = L.ora_run(phys.ctypes.data, C.addressof(scene_holder.scene), h0, h1, threads or os.cpu_count(),
                   tally.ctypes.data_as(C.POINTER(C.c_int64)), C.byref(st))
    stats = dict(counts=list(st.counts), steps_photon=st.steps_photon, steps_electron=st.steps_electron,
                 e_escaped=st.e_escaped, error=st.error, rc=rc,
                 cnt=[list(st.cnt[i]) for i in range(10)])
    return tally, stats


# ---- known-answer probes (ora_probe.c) ------------------------------------
def probe_compton(physics, medium, flags, energy, n, seed=1):
    """Scattered-photon energy and cosine of n Compton events at `energy` (MeV)."""
    L = lib()
    blk = np.ascontiguousarray(physics)
    e = np.zeros(n, np.float32)
    c = np.zeros(n, np.float32)
    L.ora_probe_compton.argtypes = [C.c_void_p, C.c_int, C.c_uint32, C.c_float, C.c_uint32, C.c_uint64,
                                    C.c_void_p, C.c_void_p]
    err = L.ora_probe_compton(blk.ctypes.data, medium, flags, energy, n, seed, e.ctypes.data, c.ctypes.data)
    return e, c, err


def probe_photo(physics, medium, flags, energy, n, seed=1):
    """Photoelectron kinetic energy and direction cosine of n photoelectric events at `energy` (MeV)."""
    L = lib()
    blk = np.ascontiguousarray(physics)
    e = np.zeros(n, np.float32)
    c = np.zeros(n, np.float32)
    L.ora_probe_photo.argtypes = [C.c_void_p, C.c_int, C.c_uint32, C.c_float, C.c_uint32, C.c_uint64,
                                  C.c_void_p, C.c_void_p]
    err = L.ora_probe_photo(blk.ctypes.data, medium, flags, energy, n, seed, e.ctypes.data, c.ctypes.data)
    return e, c, err


def probe_moller(physics, medium, ekin, n, seed=1):
    """Slower electron's kinetic-energy fraction and direction cosine of n Moller events at `ekin` (MeV)."""
    L = lib()
    blk = np.ascontiguousarray(physics)
    f = np.zeros(n, np.float32)
    c = np.zeros(n, np.float32)
    L.ora_probe_moller.argtypes = [C.c_void_p, C.c_int, C.c_float, C.c_uint32, C.c_uint64, C.c_void_p, C.c_void_p]
    err = L.ora_probe_moller(blk.ctypes.data, medium, ekin, n, seed, f.ctypes.data, c.ctypes.data)
    return f, c, err


def probe_rotate(n, seed=1):
    L = lib()
    a = np.zeros(n, np.float32)
    b = np.zeros(n, np.float32)
    L.ora_probe_rotate.argtypes = [C.c_uint32, C.c_uint64, C.c_void_p, C.c_void_p]
    L.ora_probe_rotate(n, seed, a.ctypes.data, b.ctypes.data)
    return a, b


def probe_walk(physics, scene_holder, pos, direction, field=0, region=1, maxn=4096):
    """Regions entered and step lengths of howfar_phantom along one straight ray (beam frame)."""
    L = lib()
    blk = np.ascontiguousarray(physics)
    regs = np.zeros(maxn, np.uint32)
    steps = np.zeros(maxn, np.float32)
    p = np.asarray(pos, np.float32)
    d = np.asarray(direction, np.float32)
    L.ora_probe_walk.restype = C.c_uint32
    L.ora_probe_walk.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32,
                                 C.c_void_p, C.c_void_p]
    k = L.ora_probe_walk(blk.ctypes.data, C.addressof(scene_holder.scene), field, region, p.ctypes.data,
                         d.ctypes.data, maxn, regs.ctypes.data, steps.ctypes.data)
    return regs[:k], steps[:k]
