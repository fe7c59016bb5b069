"""The C-ABI library loads on a machine without a GPU and exports every
symbol include/gegs.h declares; struct sizes agree with the Python mirrors."""
import ctypes as C
import re
from pathlib import Path

from gegs_b200 import build as B
from gegs_b200 import engine as E
from gegs_b200 import physics_layout as L
from gegs_b200 import scene as S

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    txt = "".join(p.read_text() for p in sorted((ROOT / "include").glob("*.h")))
    return sorted(set(re.findall(r"\b(gegs_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_all_declared_symbols():
    B.build()
    lib = E.load_library()
    names = declared_functions()
    assert set(E.EXPORTS) <= set(names)
    for n in names:
        assert hasattr(lib, n), n


def test_sizes_match():
    lib = E.load_library()
    assert lib.gegs_sizeof_physics() == L.dtype().itemsize
    assert lib.gegs_sizeof_scene() == C.sizeof(S.Scene)
    assert lib.gegs_sizeof_field() == C.sizeof(S.Field)
    assert lib.gegs_version().startswith(b"gegs_b200")


def test_create_without_gpu_reports_error_not_crash():
    import torch
    if torch.cuda.is_available():
        return
    try:
        E.Engine(0)
    except E.GegsError as err:
        assert err.status == 2
    else:
        raise AssertionError("engine creation must fail loudly without a GPU")


def test_engine_binding_has_every_method():
    """The Python binding exposes each C entry point a caller needs as an
    Engine method (checked without a GPU)."""
    from gegs_b200.engine import Engine, launch_group
    for m in ("set_physics", "set_scene", "run", "launch", "wait", "stats", "tally", "reset_tally", "dose",
              "set_tally", "checkpoint", "resume", "set_timeline", "timeline", "set_trace", "get_trace",
              "stat_begin", "stat_fold", "stat_get", "backward", "set_beamlet_weights", "set_phsp"):
        assert callable(getattr(Engine, m, None)), m
    assert callable(launch_group)
