"""The float forms of the kernels' comparisons with double constants
(gegs_b200/csrc/gx_cmp.h) against the double comparison C makes, on the host:
for every constant the kernels compare with, the 2 * 4096 floats nearest to it
on both sides, both signs, zeros, infinities and NaN, and random floats."""
import ctypes as C
import pathlib
import subprocess

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
CONSTANTS = [13.8, 1.0e-20, 1e5, 1e-3, 2.2299, 0.2, 1.99999, 0.1, 0.999999, 1e-9, 1.e-5, 50.0, -0.15, 0.15, 0.01,
             1e-10, 1e-8, 0.001, 2.1, 4.14, 0.5, 1e-30, 0.0005]

SRC = r'''
#include "gx_cmp.h"
extern "C" void cmp_all(const float *x, int n, double d, unsigned char *out)
{
    for (int i = 0; i < n; i++) {
        out[8 * i + 0] = gx_lt(x[i], d); out[8 * i + 1] = x[i] < d;
        out[8 * i + 2] = gx_le(x[i], d); out[8 * i + 3] = x[i] <= d;
        out[8 * i + 4] = gx_gt(x[i], d); out[8 * i + 5] = x[i] > d;
        out[8 * i + 6] = gx_ge(x[i], d); out[8 * i + 7] = x[i] >= d;
    }
}
'''


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    d = tmp_path_factory.mktemp("gxcmp")
    (d / "t.cpp").write_text(SRC)
    so = d / "t.so"
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-shared", "-fPIC", "-I", str(ROOT / "gegs_b200" / "csrc"),
                    str(d / "t.cpp"), "-o", str(so)], check=True)
    L = C.CDLL(str(so))
    L.cmp_all.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_void_p]
    return L


def _around(d, k=4096):
    f = np.float32(d)
    bits = f.view(np.int32).astype(np.int64)
    near = (bits + np.arange(-k, k + 1)).astype(np.int32).view(np.float32)
    return near[np.isfinite(near)]


@pytest.mark.parametrize("d", CONSTANTS)
def test_float_compare_equals_double_compare(lib, d):
    rng = np.random.default_rng(1)
    x = np.concatenate([_around(d), -_around(d), np.float32([0.0, -0.0, np.inf, -np.inf, np.nan]),
                        rng.standard_normal(20000).astype(np.float32) * np.float32(abs(d) * 4 + 1)])
    x = np.ascontiguousarray(x, np.float32)
    out = np.zeros(8 * len(x), np.uint8)
    lib.cmp_all(x.ctypes.data, len(x), d, out.ctypes.data)
    o = out.reshape(-1, 8)
    for k, name in enumerate(("<", "<=", ">", ">=")):
        bad = np.flatnonzero(o[:, 2 * k] != o[:, 2 * k + 1])
        assert bad.size == 0, f"x {name} {d!r}: differs at {x[bad[:5]]}"
