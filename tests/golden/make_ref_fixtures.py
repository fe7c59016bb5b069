"""Write tests/golden/ref_pin_c3.npz: outputs of the reference's own routines
(geom.cu, the stage kernels; compiled as host code by oracle/ref) on particle
states of the full C3 geometry, for tests/test_ref_pin.py to check the oracle
against where the reference sources are absent.

    python tests/golden/make_ref_fixtures.py

Needs the reference sources (oracle/refpin.REF_DIR) to build the harness.
Stored: the inputs, then the reference's results -- howfar region, step and
particle state, hownear distance; per stage the uniforms used, the particles
pushed (sorted by stack, push order kept) and the escore calls.

Also writes tests/golden/ref_setup.npz: the reference's host set-up (the
egsphant, egsinp, mlcinfo and mlcinp readers and the per-field polygons of
init.cu) on the plan files of tests/test_ref_setup.py."""
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE.parent))

from oracle import oracle as O            # noqa: E402
from oracle import refpin as R            # noqa: E402
import refpin_cases as RC                 # noqa: E402


def main():
    O.build()
    R.build()
    if not R.available():
        raise SystemExit("reference harness not available")
    job = RC.job("c3")
    sh = job.scene()
    pair = R.Pair(job.physics, sh)
    cap = pair.capture(0, job.histories, every=1, cap_n=60000)
    for s in range(10):
        cap[s]["hist"] = np.arange(len(cap[s]), dtype=np.uint32)
    rng = np.random.default_rng(3)
    out = {}
    # geometry: photon and electron states, every 10th, with the transport's step and a short one
    g_in = np.concatenate([cap[0][::10], cap[5][::10]])
    t_in = np.where(np.arange(len(g_in)) % 2 == 0, np.float32(1e3),
                    rng.exponential(0.3, len(g_in)).astype(np.float32)).astype(np.float32)
    g = pair.geom(g_in, t_in)["ref"]
    out.update(geom_in=g_in, geom_t_in=t_in, geom_region=g["region"], geom_t=g["t"], geom_tperp=g["tperp"],
               geom_out=g["particle"])
    sweep = RC.stress(cap, job.physics, n=60)
    for s in range(10):
        parts = np.concatenate([cap[s][:240], sweep[s]])
        ref = pair.stage(s, parts)["ref"]
        n = len(parts)
        key = f"s{s}_"
        out[key + "in"] = parts
        out[key + "used"] = ref["used"]
        out[key + "on"] = ref["on"]
        out[key + "dn"] = ref["dn"]
        out[key + "out"] = np.concatenate([R.sort_by_stack(ref["out"][i], ref["on"][i]) for i in range(n)])
        out[key + "dreg"] = np.concatenate([ref["dreg"][i, :ref["dn"][i]] for i in range(n)])
        out[key + "de"] = np.concatenate([ref["de"][i, :ref["dn"][i]] for i in range(n)])
    path = HERE / "ref_pin_c3.npz"
    np.savez_compressed(path, **out)
    print(path, path.stat().st_size, "bytes")
    setup_fixtures()


def setup_fixtures():
    """tests/golden/ref_setup.npz: the reference's host set-up (init.cu) on the
    plan files of each case of tests/test_ref_setup.py."""
    import tempfile
    import test_ref_setup as TS
    out = {}
    for case in sorted(TS.CASES):
        with tempfile.TemporaryDirectory() as d:
            tmp = pathlib.Path(d)
            _, c = TS.case_plan(tmp, case)
            S = TS.run_reference(R, tmp, c)
            out.update({f"{case}/{k}": v for k, v in TS.setup_arrays(S).items()})
    path = HERE / "ref_setup.npz"
    np.savez_compressed(path, **out)
    print(path, path.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
