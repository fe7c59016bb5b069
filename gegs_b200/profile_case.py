"""One transport run of the CT head 5-field plan in the host-driven timed form
(the persistent form's kernels launched wave by wave, which ncu can profile
one by one), printing one JSON line with the step counts and per-kernel device
time. Used as the profiled command for the kernel summaries:

    python -m gegs_b200.profile_case --histories 1000000 --batch 524288

With --timeline it runs the persistent form instead (one CUDA graph) and
prints the wave timeline summary: per phase and per kernel the device time
summed over waves, from the first-block start and last-block end stamps that
every kernel writes per wave (gegs_set_timeline).
"""
from __future__ import annotations

import argparse
import json


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--histories", type=int, default=1_000_000)
    ap.add_argument("--batch", type=int, default=524288, help="in-flight batch (0: sized to the run)")
    ap.add_argument("--nphsp", type=int, default=2_000_000)
    ap.add_argument("--dims", default="256,256,120")
    ap.add_argument("--timeline", action="store_true", help="persistent form with the wave timeline")
    ap.add_argument("--serial", action="store_true",
                    help="with --timeline: the serial wave order (GEGS_RUN_SERIAL_WAVES) instead of both "
                         "transport phases at once")
    ap.add_argument("--plan-histories", type=int, default=0, help="histories of the plan (fields split them; 0: --histories)")
    ap.add_argument("--first", type=int, default=0, help="first history of the run")
    ap.add_argument("--max-waves", type=int, default=0,
                    help="stop after this many waves (a short capture of the bulk waves; the run then reports "
                         "the wave budget and its statistics cover those waves)")
    args = ap.parse_args()
    from . import build as B
    B.build()
    from . import workloads as W
    from .engine import MODE_TIMED, Engine
    dims = tuple(int(x) for x in args.dims.split(","))
    job = W.config3(histories=max(args.plan_histories or args.histories, 1), nphsp=args.nphsp, dims=dims)
    eng = Engine(0)
    eng.set_physics(job.physics)
    eng.set_scene(job.scene())
    if args.timeline:
        print(json.dumps(timeline_summary(eng, args, dims)))
        return
    if args.max_waves:
        from .engine import GegsError
        try:
            eng.run(args.first, args.first + args.histories, mode=MODE_TIMED, batch=args.batch,
                    max_waves=args.max_waves)
        except GegsError as err:
            if err.status != 6:                         # GEGS_ERR_STEP_BUDGET: the waves ran out, as asked
                raise
        st = eng.stats()
    else:
        st = eng.run(args.first, args.first + args.histories, mode=MODE_TIMED, batch=args.batch)
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


def timeline_summary(eng, args, dims):
    import numpy as np
    pipe = dict(pipelined=False) if getattr(args, "serial", False) else {}
    eng.run(args.first, args.first + min(args.histories, 1_000_000), batch=args.batch, **pipe)   # graph and queues
    eng.set_timeline(1 << 14)
    st = eng.run(args.first, args.first + args.histories, batch=args.batch, **pipe)
    tl = eng.timeline()[:st["waves"]].astype(np.float64)
    ran = tl[:, :, 1] > 0
    t0 = np.min(np.where(ran, tl[:, :, 0], np.inf))
    s = np.where(ran, (tl[:, :, 0] - t0) / 1e6, np.nan)
    e = np.where(ran, (tl[:, :, 1] - t0) / 1e6, np.nan)
    names = eng.TIMELINE_KERNELS
    groups = {"source": [0], "photon transport": [1, 2, 3], "photon interactions": [4, 5, 6, 7],
              "electron transport": [8, 9, 10, 15], "long jaws-photon tracks": [16], "electron interactions": [11, 12, 13, 14]}
    import warnings
    with np.errstate(all="ignore"), warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)          # waves in which a group did not run
        span = lambda g: np.nan_to_num(np.nanmax(e[:, g], axis=1) - np.nanmin(s[:, g], axis=1))
        phases = {k: float(span(g).sum()) for k, g in groups.items()}
        dur = np.nan_to_num(e - s)
    kern = {names[k]: float(dur[:, k].sum()) for k in range(len(names))}
    # waves whose photon-jaws launch lasts well past every other kernel of the same wave
    pj = dur[:, 1]
    others = np.max(np.delete(dur, [1], axis=1), axis=1)
    lone = (pj > 0.5) & (pj > 2 * others)
    # per wave: span from its first kernel start to its last kernel end, the
    # phases' spans inside it, and the gap to the next wave (the planner node
    # and the graph's conditional hand-over)
    live = ran.any(axis=1)
    ws, we = np.nanmin(s[live], axis=1), np.nanmax(e[live], axis=1)
    wave_ms = we - ws
    gap_ms = np.maximum(ws[1:] - we[:-1], 0.0)
    with np.errstate(all="ignore"), warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        per_phase = {k: np.round(span(g)[live], 3).tolist() for k, g in groups.items()}
    small = wave_ms < 1.0
    return {"workload": f"C3 CT head {dims[0]}x{dims[1]}x{dims[2]}, 5 fields, persistent form"
                        + (", serial waves" if pipe else ", pipelined waves"),
            "histories": args.histories, "first": args.first, "batch": args.batch or "auto",
            "device_ms": st["device_ms"], "waves": st["waves"],
            "phase_ms": {k: round(v, 1) for k, v in phases.items()},
            "kernel_ms": {k: round(v, 1) for k, v in kern.items()},
            "serial_overlap": "kernel sums exceed phase spans where kernels of a phase overlap",
            "lone_photon_jaws_waves": int(lone.sum()),
            "lone_photon_jaws_ms": round(float(pj[lone].sum()), 1),
            "longest_photon_jaws_ms": [round(float(x), 2) for x in np.sort(pj)[::-1][:5]],
            "waves_under_1ms": int(small.sum()), "waves_under_1ms_ms": round(float(wave_ms[small].sum()), 1),
            "gaps_between_waves_ms": round(float(gap_ms.sum()), 1),
            "wave_ms": np.round(wave_ms, 3).tolist(), "wave_phase_ms": per_phase}


if __name__ == "__main__":
    main()
