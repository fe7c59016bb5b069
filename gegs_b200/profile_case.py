"""One transport run of the CT head 5-field plan in the host-driven timed form
(the persistent form's kernels launched wave by wave, which ncu can profile
one by one), printing one JSON line with the step counts and per-kernel device
time. Used as the profiled command for the kernel summaries:

    python -m gegs_b200.profile_case --histories 1000000 --batch 524288
"""
from __future__ import annotations

import argparse
import json


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--histories", type=int, default=1_000_000)
    ap.add_argument("--batch", type=int, default=524288)
    ap.add_argument("--nphsp", type=int, default=2_000_000)
    ap.add_argument("--dims", default="256,256,120")
    args = ap.parse_args()
    from . import build as B
    B.build()
    from . import workloads as W
    from .engine import MODE_TIMED, Engine
    dims = tuple(int(x) for x in args.dims.split(","))
    job = W.config3(histories=max(args.histories, 1), nphsp=args.nphsp, dims=dims)
    eng = Engine(0)
    eng.set_physics(job.physics)
    eng.set_scene(job.scene())
    st = eng.run(0, args.histories, mode=MODE_TIMED, batch=args.batch)
    kinds = ["photon", "compton", "photo", "rayleigh", "pair", "electron", "moller", "brems", "bhabha", "annih",
             "source", "planner", "photon_jaws", "electron_jaws", "photon_mlc", "electron_mlc"]
    print(json.dumps({
        "workload": f"C3 CT head {dims[0]}x{dims[1]}x{dims[2]}, 5 fields, timed wave form",
        "histories": args.histories, "batch": args.batch, "waves": st["waves"],
        "photon_steps": st["photon_steps"], "electron_steps": st["electron_steps"],
        "photon_steps_jaws_mlc_phantom": st["photon_steps_class"],
        "electron_steps_jaws_mlc_phantom": st["electron_steps_class"],
        "processed": dict(zip(kinds[:10], st["processed"])),
        "stage_ms": dict(zip(kinds, st["stage_ms"])), "stage_launches": dict(zip(kinds, st["stage_launches"])),
        "error_bits": st["error_bits"]}))


if __name__ == "__main__":
    main()
