"""ctypes binding of the C ABI (``include/gegs.h``) of ``libgegs_b200.so``.

The CUDA library is the only compute path: if it cannot be loaded, or no GPU
is visible, these calls raise -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import pathlib

import numpy as np

from .scene import PhspRecord

LIB_PATH = pathlib.Path(__file__).resolve().parent / "libgegs_b200.so"

STATUS = {0: "GEGS_OK", 1: "GEGS_ERR_ARG", 2: "GEGS_ERR_CUDA", 3: "GEGS_ERR_QUEUE_FULL", 4: "GEGS_ERR_MODULE",
          5: "GEGS_ERR_NOMEM", 6: "GEGS_ERR_STEP_BUDGET", 7: "GEGS_ERR_SOURCE"}
MODE_PERSISTENT, MODE_PLAIN, MODE_TIMED = 0, 1, 2

EXPORTS = ["gegs_set_trace", "gegs_get_trace", "gegs_set_timeline", "gegs_get_timeline", "gegs_create", "gegs_destroy", "gegs_last_error", "gegs_set_physics", "gegs_set_scene", "gegs_set_phsp",
           "gegs_run", "gegs_reset_tally", "gegs_get_tally", "gegs_set_tally", "gegs_get_dose", "gegs_get_stats",
           "gegs_tally_device_ptr", "gegs_run_noalloc", "gegs_launch", "gegs_wait", "gegs_launch_group", "gegs_probe_geometry", "gegs_set_stream", "gegs_set_field", "gegs_set_beamlet_weights", "gegs_backward", "gegs_sizeof_physics", "gegs_sizeof_scene", "gegs_sizeof_field", "gegs_version",
           "gegs_check_physics", "gegs_stat_begin", "gegs_stat_fold", "gegs_stat_get"]


TRACE_DTYPE = np.dtype([("kind_stage", "<u4"), ("hist_lo", "<u4"), ("sid_lo", "<u4"), ("sid_hi", "<u4"),
                        ("ctr", "<u4"), ("e", "<f4"), ("x", "<f4"), ("region", "<u4")])


class GegsError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class RunOpts(C.Structure):
    _fields_ = [("mode", C.c_int32), ("batch", C.c_uint32), ("blocks_per_sm", C.c_int32),
                ("threads_per_block", C.c_int32), ("max_waves", C.c_uint32), ("step_budget", C.c_uint32),
                ("refill_below", C.c_uint32), ("queue_cap", C.c_uint32), ("flags", C.c_uint32)]

RUN_STAGE_TABLES = 1
RUN_SERIAL_WAVES = 2


# gegs_probe_state (include/gegs.h)
PROBE_DTYPE = np.dtype([("region", "<u4"), ("charge", "i1"), ("leafIndex", "i1"), ("bank", "i1"), ("module", "u1"),
                        ("field", "u1"), ("status", "u1"), ("pad0", "u1"), ("pad1", "u1"),
                        ("wt", "<f4"), ("e", "<f4"), ("x", "<f4"), ("y", "<f4"), ("z", "<f4"),
                        ("u", "<f4"), ("v", "<f4"), ("w", "<f4"), ("dnear", "<f4"), ("hist", "<u4"), ("pad2", "<u4")])


class RunStats(C.Structure):
    _fields_ = [("processed", C.c_uint64 * 10), ("photon_steps", C.c_uint64), ("electron_steps", C.c_uint64),
                ("waves", C.c_uint32), ("error_bits", C.c_uint32), ("device_ms", C.c_double),
                ("stage_ms", C.c_double * 16), ("stage_launches", C.c_uint64 * 16),
                ("photon_steps_class", C.c_uint64 * 3), ("electron_steps_class", C.c_uint64 * 3),
                ("queue_peak", C.c_uint32 * 25), ("queue_cap", C.c_uint32 * 25)]


_lib = None


def load_library(path=None):
    """Load the CUDA library (raises OSError when it is missing)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    L = C.CDLL(str(path or LIB_PATH))
    vp = C.c_void_p
    L.gegs_create.argtypes = [C.c_int, C.POINTER(vp)]
    L.gegs_destroy.argtypes = [vp]
    L.gegs_destroy.restype = None
    L.gegs_last_error.argtypes = [vp]
    L.gegs_last_error.restype = C.c_char_p
    L.gegs_set_physics.argtypes = [vp, vp]
    L.gegs_set_scene.argtypes = [vp, vp]
    L.gegs_set_phsp.argtypes = [vp, vp, C.c_uint64]
    L.gegs_run.argtypes = [vp, C.c_uint64, C.c_uint64, C.POINTER(RunOpts)]
    L.gegs_run_noalloc.argtypes = [vp, C.c_uint64, C.c_uint64, C.c_uint32]
    L.gegs_launch.argtypes = [vp, C.c_uint64, C.c_uint64, C.POINTER(RunOpts)]
    L.gegs_wait.argtypes = [vp]
    L.gegs_launch_group.argtypes = [vp, C.c_int32, vp, vp, vp]
    L.gegs_probe_geometry.argtypes = [vp, C.c_uint32, vp, vp, vp, vp, vp, vp]
    L.gegs_set_stream.argtypes = [vp, vp]
    L.gegs_set_field.argtypes = [vp, C.c_int32, vp]
    L.gegs_set_beamlet_weights.argtypes = [vp, vp, C.c_uint32]
    L.gegs_backward.argtypes = [vp, C.c_uint64, C.c_uint64, vp, vp, C.c_uint32, C.POINTER(RunOpts)]
    L.gegs_reset_tally.argtypes = [vp]
    L.gegs_get_tally.argtypes = [vp, vp, C.c_uint64]
    L.gegs_set_tally.argtypes = [vp, vp, C.c_uint64]
    L.gegs_get_dose.argtypes = [vp, vp, C.c_double, vp, C.c_uint64]
    L.gegs_get_stats.argtypes = [vp, C.POINTER(RunStats)]
    L.gegs_tally_device_ptr.argtypes = [vp, C.POINTER(vp)]
    L.gegs_set_trace.argtypes = [vp, C.c_uint32]
    L.gegs_set_timeline.argtypes = [vp, C.c_uint32]
    L.gegs_get_timeline.argtypes = [vp, vp, C.c_uint32]
    L.gegs_get_trace.argtypes = [vp, vp, C.c_uint32, C.POINTER(C.c_uint32)]
    for f in ("gegs_sizeof_physics", "gegs_sizeof_scene", "gegs_sizeof_field"):
        getattr(L, f).restype = C.c_size_t
    L.gegs_version.restype = C.c_char_p
    L.gegs_check_physics.argtypes = [vp, C.c_char_p, C.c_size_t]
    L.gegs_stat_begin.argtypes = [vp]
    L.gegs_stat_fold.argtypes = [vp]
    L.gegs_stat_get.argtypes = [vp, vp, vp, C.c_uint64, C.POINTER(C.c_uint32)]
    if path is None:
        _lib = L
    return L


def check_physics(block: np.ndarray):
    """Host-side validation of a physics block through the C ABI (no GPU
    needed); raises GegsError naming the first bad entry."""
    L = load_library()
    blk = np.ascontiguousarray(block)
    msg = C.create_string_buffer(192)
    st = L.gegs_check_physics(blk.ctypes.data, msg, len(msg))
    if st != 0:
        raise GegsError(st, msg.value.decode())


def _flags(stage_tables, pipelined):
    """gegs_run_opts.flags; `pipelined` (the default, persistent form): both
    transport phases of a wave at once, then all interactions."""
    return (RUN_STAGE_TABLES if stage_tables else 0) | (0 if pipelined else RUN_SERIAL_WAVES)


class Engine:
    """One CUDA device + stream with the transport state (see include/gegs.h)."""

    def __init__(self, device: int = 0):
        self.L = load_library()
        self.h = C.c_void_p()
        st = self.L.gegs_create(device, C.byref(self.h))
        if st != 0:
            msg = self.L.gegs_last_error(self.h).decode() if self.h else "create failed"
            if self.h:
                self.L.gegs_destroy(self.h)
                self.h = C.c_void_p()
            raise GegsError(st, msg)
        self.nvox = 0
        self._keep = None

    def _check(self, st):
        if st != 0:
            raise GegsError(st, self.L.gegs_last_error(self.h).decode())

    def close(self):
        if self.h:
            self.L.gegs_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_physics(self, block: np.ndarray):
        blk = np.ascontiguousarray(block)
        assert blk.dtype.itemsize == self.L.gegs_sizeof_physics()
        self._check(self.L.gegs_set_physics(self.h, blk.ctypes.data))

    def set_scene(self, scene_holder):
        self._keep = scene_holder
        self._check(self.L.gegs_set_scene(self.h, C.addressof(scene_holder.scene)))
        self.nvox = scene_holder.nvox
        self.nbeamlets = getattr(scene_holder, "nbeamlets", 0)

    def set_beamlet_weights(self, w):
        w = np.ascontiguousarray(w, np.float32).reshape(-1)
        self._check(self.L.gegs_set_beamlet_weights(self.h, w.ctypes.data, w.size))

    def backward(self, h0: int, h1: int, voxel_grad, batch: int = 0):
        """d(objective)/d(beamlet weight) from d(objective)/d(energy per voxel, MeV)."""
        g = np.ascontiguousarray(voxel_grad, np.float64).reshape(-1)
        if g.size != self.nvox:
            raise ValueError(f"voxel gradient has {g.size} entries for {self.nvox} voxels")
        out = np.zeros(self.nbeamlets, np.float64)
        o = RunOpts(MODE_PERSISTENT, batch, 0, 0, 0, 0, 0, 0, 0)
        self._check(self.L.gegs_backward(self.h, h0, h1, g.ctypes.data, out.ctypes.data, out.size, C.byref(o)))
        return out

    def set_phsp(self, recs: np.ndarray):
        r = np.ascontiguousarray(recs)
        self._check(self.L.gegs_set_phsp(self.h, r.ctypes.data, len(r)))

    def run(self, h0: int, h1: int, mode: int = MODE_PERSISTENT, batch: int = 0, blocks_per_sm: int = 0,
            threads: int = 0, max_waves: int = 0, photon_budget: int = 0, electron_budget: int = 0,
            refill_below: int = 0, queue_cap: int = 0, stage_tables: bool = False, pipelined: bool = True):
        o = RunOpts(mode, batch, blocks_per_sm, threads, max_waves, (photon_budget & 0xFFFF) | (electron_budget << 16),
                    refill_below, queue_cap, _flags(stage_tables, pipelined))
        self._check(self.L.gegs_run(self.h, h0, h1, C.byref(o)))
        return self.stats()

    def launch(self, h0: int, h1: int, batch: int = 0, blocks_per_sm: int = 0, threads: int = 0,
               photon_budget: int = 0, electron_budget: int = 0, refill_below: int = 0, stage_tables: bool = False,
               pipelined: bool = True):
        """Queue a persistent-form run and return at once (see wait())."""
        o = RunOpts(MODE_PERSISTENT, batch, blocks_per_sm, threads, 0, (photon_budget & 0xFFFF) | (electron_budget << 16),
                    refill_below, 0, _flags(stage_tables, pipelined))
        self._check(self.L.gegs_launch(self.h, h0, h1, C.byref(o)))

    def wait(self):
        self._check(self.L.gegs_wait(self.h))
        return self.stats()

    def set_field(self, index: int, field: dict):
        """Replace one field of the scene (gegs_set_field): angle, history range,
        jaw and leaf-end polygons, as a field dict of a job."""
        from .scene import Field, fill_field
        F = fill_field(Field(), field)
        self._check(self.L.gegs_set_field(self.h, index, C.byref(F)))

    def set_stream(self, stream=None):
        """Issue the engine's work on a caller's CUDA stream (a torch.cuda.Stream
        or a raw cudaStream_t handle); None returns to the engine's own."""
        handle = getattr(stream, "cuda_stream", stream)
        self._check(self.L.gegs_set_stream(self.h, handle))

    def probe_geometry(self, states, t_in):
        """howfar (step t_in) and hownear of each state on the device
        (gegs_probe_geometry): region entered, step, state after howfar, and
        the distance to the nearest boundary."""
        s = np.ascontiguousarray(states, PROBE_DTYPE)
        t = np.ascontiguousarray(t_in, np.float32)
        n = len(s)
        reg = np.zeros(n, np.uint32)
        ft = np.zeros(n, np.float32)
        out = np.zeros(n, PROBE_DTYPE)
        near = np.zeros(n, np.float32)
        self._check(self.L.gegs_probe_geometry(self.h, n, s.ctypes.data, t.ctypes.data, reg.ctypes.data,
                                               ft.ctypes.data, out.ctypes.data, near.ctypes.data))
        return dict(region=reg, t=ft, particle=out, tperp=near)

    @staticmethod
    def _opts(o):
        return RunOpts(MODE_PERSISTENT, o.get("batch", 0), o.get("blocks_per_sm", 0), o.get("threads", 0), 0,
                       (o.get("photon_budget", 0) & 0xFFFF) | (o.get("electron_budget", 0) << 16),
                       o.get("refill_below", 0), 0, _flags(o.get("stage_tables"), o.get("pipelined", True)))


    def reset_tally(self):
        self._check(self.L.gegs_reset_tally(self.h))

    def tally(self, out=None) -> np.ndarray:
        """The int64 tally (MeV * 2^30 per voxel); into `out` when given (a
        pinned host buffer makes the copy a direct DMA)."""
        if out is None:
            out = np.empty(self.nvox, np.int64)
        elif out.dtype != np.int64 or out.size != self.nvox or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous int64 array of nvox values")
        self._check(self.L.gegs_get_tally(self.h, out.ctypes.data, self.nvox))
        return out

    TIMELINE_KERNELS = ["source", "photon_jaws", "photon_mlc", "photon", "compton", "photo", "rayleigh", "pair",
                        "electron_jaws", "electron_mlc", "electron", "moller", "brems", "bhabha", "annih",
                        "electron_near", "photon_jaws_long"]
    TIMELINE_SLOTS = 32

    def set_timeline(self, max_waves: int):
        """Record the wave timeline of the following runs (0: off)."""
        self._check(self.L.gegs_set_timeline(self.h, int(max_waves)))
        self._timeline_waves = int(max_waves)

    def timeline(self) -> np.ndarray:
        """[waves, 32, 2] start / end stamps (ns) of the last run; see gegs.h."""
        n = getattr(self, "_timeline_waves", 0)
        out = np.zeros((n, self.TIMELINE_SLOTS, 2), np.uint64)
        if n:
            self._check(self.L.gegs_get_timeline(self.h, out.ctypes.data, n))
        return out

    def set_tally(self, tally: np.ndarray):
        t = np.ascontiguousarray(tally, np.int64)
        if t.size != self.nvox:
            raise ValueError(f"tally of {t.size} voxels, the scene has {self.nvox}")
        self._check(self.L.gegs_set_tally(self.h, t.ctypes.data, self.nvox))

    def checkpoint(self, path, next_history: int):
        """Save the tally and the index of the next history to run (.npz)."""
        np.savez(path, tally=self.tally(), next_history=np.uint64(next_history), nvox=np.uint64(self.nvox))

    def resume(self, path) -> int:
        """Load a checkpoint's tally; returns the next history to run. Running
        the remaining histories then gives the whole run's tally bit for bit."""
        with np.load(path) as z:
            if int(z["nvox"]) != self.nvox:
                raise ValueError("checkpoint of another phantom")
            self.set_tally(z["tally"])
            return int(z["next_history"])

    def dose(self, voxel_mass: np.ndarray, dose_unit: float = 1.6e-8) -> np.ndarray:
        m = np.ascontiguousarray(voxel_mass, np.float32)
        out = np.zeros(self.nvox, np.float64)
        self._check(self.L.gegs_get_dose(self.h, m.ctypes.data, dose_unit, out.ctypes.data, self.nvox))
        return out

    # ---- batch statistics (the reference's batch uncertainty, on the device) ----
    def stat_begin(self):
        """Start a series of batches at the current tally."""
        self._check(self.L.gegs_stat_begin(self.h))

    def stat_fold(self):
        """End a batch: what was deposited since the previous fold is one batch."""
        self._check(self.L.gegs_stat_fold(self.h))

    def stat_get(self):
        """(batch-mean energy per voxel in MeV, relative standard error of the
        mean per voxel, number of batches)."""
        mean = np.zeros(self.nvox, np.float64)
        rel = np.zeros(self.nvox, np.float64)
        n = C.c_uint32()
        self._check(self.L.gegs_stat_get(self.h, mean.ctypes.data, rel.ctypes.data, self.nvox, C.byref(n)))
        return mean, rel, n.value

    def stats(self) -> dict:
        s = RunStats()
        self._check(self.L.gegs_get_stats(self.h, C.byref(s)))
        return dict(processed=list(s.processed), photon_steps=s.photon_steps, electron_steps=s.electron_steps,
                    waves=s.waves, error_bits=s.error_bits, device_ms=s.device_ms,
                    stage_ms=list(s.stage_ms), stage_launches=list(s.stage_launches),
                    photon_steps_class=list(s.photon_steps_class), electron_steps_class=list(s.electron_steps_class),
                    queue_peak=list(s.queue_peak), queue_cap=list(s.queue_cap))

    def set_trace(self, capacity: int):
        self._check(self.L.gegs_set_trace(self.h, capacity))
        self._trace_cap = capacity

    def get_trace(self) -> np.ndarray:
        buf = np.zeros(self._trace_cap, TRACE_DTYPE)
        n = C.c_uint32()
        self._check(self.L.gegs_get_trace(self.h, buf.ctypes.data, self._trace_cap, C.byref(n)))
        return buf[:min(n.value, self._trace_cap)]

    def tally_device_ptr(self) -> int:
        p = C.c_void_p()
        self._check(self.L.gegs_tally_device_ptr(self.h, C.byref(p)))
        return p.value


def launch_group(engines, ranges, options=None):
    """Queue the persistent-form runs of several engines (one device) as one
    graph launch (gegs_launch_group); ranges[i] = (h0, h1) of engine i and
    options[i] its run options as for Engine.launch. Finish each with wait()."""
    n = len(engines)
    if n == 0 or len(ranges) != n or (options is not None and len(options) != n):
        raise ValueError("one range (and one option set) per engine")
    L = engines[0].L
    handles = (C.c_void_p * n)(*[e.h for e in engines])
    h0 = (C.c_uint64 * n)(*[int(r[0]) for r in ranges])
    h1 = (C.c_uint64 * n)(*[int(r[1]) for r in ranges])
    opts = (RunOpts * n)(*[Engine._opts(o) for o in (options or [{}] * n)])
    engines[0]._check(L.gegs_launch_group(handles, n, h0, h1, opts))
