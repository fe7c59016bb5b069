"""Command line: run a plan given in the reference's INI format.

    python -m gegs_b200 -i plan.ini [--device N] [--max-histories N]

Writes ``<output directory>/<output prefix>_DoseResults_NNNxNNNxNNN.bin``
(raw float32 dose, x fastest, cGy when the plan is calibrated; the layout of
the reference's write_dose, output.c:873-918), ``<prefix>_log.txt``, the
interpolated grid ``<prefix>_Interpolate_NNNxNNNxNNN.bin`` when [Interpolation]
asks for it, and the point dose of [Dose output] in the log.
All fields run in one transport call on the GPU; with output factors the
fields run one by one and their energies are weighted before the dose
conversion (CUDA_EGS.cu:1715-1735).
"""
from __future__ import annotations

import argparse
import sys
import time
from pathlib import Path

import numpy as np


def transport_in_batches(eng, fields, output_factors, nbatch):
    """Every field's histories split into `nbatch` equal parts; batch b runs
    part b of every field. Returns the energy (the same float64 expression of
    the same int64 tallies as an unbatched run) and the relative standard error
    of its mean per voxel from the batch energies, with the reference's batch
    formula sqrt((S2/n - (S1/n)^2) / (n - 1)) / (S1/n) (CUDA_EGS.cu:817-876;
    its last, partial batch has no counterpart here: the batches are equal)."""
    acc = [np.zeros(eng.nvox, np.int64) for _ in fields]
    s1 = np.zeros(eng.nvox, np.float64)
    s2 = np.zeros(eng.nvox, np.float64)
    for b in range(nbatch):
        eb = np.zeros(eng.nvox, np.float64)
        for k, (f, of) in enumerate(zip(fields, output_factors)):
            h0, h1 = int(f["hist_begin"]), int(f["hist_end"])
            lo = h0 + (h1 - h0) * b // nbatch
            hi = h0 + (h1 - h0) * (b + 1) // nbatch
            if hi <= lo:
                continue
            eng.reset_tally()
            eng.run(lo, hi)
            t = eng.tally()
            acc[k] += t
            eb += t.astype(np.float64) * of
        s1 += eb
        s2 += eb * eb
    n = float(nbatch)
    with np.errstate(divide="ignore", invalid="ignore"):
        sigma = np.sqrt(np.maximum(s2 / n - (s1 / n) ** 2, 0.0) / (n - 1.0)) / (s1 / n)
    if all(abs(of - 1.0) < 1e-12 for of in output_factors):
        energy = np.sum(acc, axis=0).astype(np.float64)
    else:
        energy = np.zeros(eng.nvox, np.float64)
        for a, of in zip(acc, output_factors):
            energy += a.astype(np.float64) * of
    return energy, sigma


def run_plan(ini, device=0, max_histories=None, out=sys.stdout, uncertainty_batches=0):
    from . import build as B
    from . import io_formats as F
    from .plan import load_plan
    plan = load_plan(ini, max_histories=max_histories)
    job = plan.job
    B.build()
    from .engine import Engine
    eng = Engine(device)
    eng.set_physics(job.physics)
    eng.set_scene(job.scene())
    t0 = time.perf_counter()
    sigma = None
    if uncertainty_batches:
        if uncertainty_batches < 2:
            raise ValueError("the batch uncertainty needs at least 2 batches")
        energy, sigma = transport_in_batches(eng, job.fields, plan.field_output_factors, uncertainty_batches)
    elif all(abs(f - 1.0) < 1e-12 for f in plan.field_output_factors):
        eng.run(0, job.histories)
        energy = eng.tally().astype(np.float64)
    else:
        energy = np.zeros(eng.nvox, np.float64)
        for f, of in zip(job.fields, plan.field_output_factors):
            eng.reset_tally()
            eng.run(int(f["hist_begin"]), int(f["hist_end"]))
            energy += eng.tally().astype(np.float64) * of
    wall = time.perf_counter() - t0
    dose = F.dose_from_energy(energy * (2.0 ** -30), job.voxel_mass(), plan.dose_unit)
    Path(plan.output_dir).mkdir(parents=True, exist_ok=True)
    name = F.write_dose(plan.output_base, dose.astype(np.float32), plan.nx, plan.ny, plan.nz)
    st = eng.stats()
    extra = []
    if sigma is not None:
        un = F.write_uncertainty(plan.output_base, sigma.astype(np.float32), plan.nx, plan.ny, plan.nz)
        extra.append(f"uncertainty ({uncertainty_batches} batches) {un}")
    p = job.phantom
    bounds = (p["x_bounds"], p["y_bounds"], p["z_bounds"])
    if "interp" in plan.post:
        from .postprocess import interp_dose, write_interp
        ip = plan.post["interp"]
        grid = interp_dose(dose.astype(np.float32), *bounds, ip["start"], ip["sizes"], ip["dims"], device=device)
        extra.append(f"interpolated dose {write_interp(plan.output_base, grid)}")
    if "point" in plan.post:
        from .postprocess import point_dose
        pt = plan.post["point"]
        v = point_dose(dose.astype(np.float32), *bounds, pt["pos"])
        msg = f"absolute dose at ({pt['pos'][0]:.2f}, {pt['pos'][1]:.2f}, {pt['pos'][2]:.2f}) = {v:.4g}"
        if pt["measured"]:
            msg += f" (measured {pt['measured']:.4g}, ratio {v / pt['measured']:.4f})"
        extra.append(msg)
    if "relative" in plan.post:
        from .postprocess import point_dose, read_measured, relative_dose, write_relative_dose
        rp = plan.post["relative"]
        if list(rp["dims"]) == [1, 1, 1]:          # one point: the reference reports the point dose instead
            v = point_dose(dose.astype(np.float32), *bounds, rp["start"])
            extra.append(f"absolute dose at ({rp['start'][0]:.2f}, {rp['start'][1]:.2f}, {rp['start'][2]:.2f})"
                         f" = {v:.4g}")
        else:
            n = int(np.prod(rp["dims"]))
            meas = read_measured(rp["measured"], n) if Path(rp["measured"]).is_file() else None
            rl, tot, ok = relative_dose(dose.astype(np.float32), *bounds, rp["start"], rp["sizes"], rp["dims"],
                                        meas, rp["norm_type"], rp["array_type"], rp["gamma_len_cm"],
                                        rp["gamma_dos"], rp["iso"])
            extra.append(f"relative dose {write_relative_dose(plan.output_base, rl, rp['dims'])}: "
                         + (rl[-1] if meas is not None else f"measured data {rp['measured']} not readable"))
    lines = [f"plan {ini}", f"fields {len(job.fields)}, histories {job.histories}, phase-space particles {len(job.phsp)}",
             f"media {job.media}", f"dose unit {plan.dose_unit:.4e}",
             f"transport {wall:.3f} s ({job.histories / max(wall, 1e-9):.4g} histories/s), waves {st['waves']}",
             f"dose file {name}"] + extra + plan.log
    Path(plan.output_base + "_log.txt").write_text("\n".join(lines) + "\n")
    for l in lines:
        print(l, file=out)
    eng.close()
    return name


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m gegs_b200")
    ap.add_argument("-i", "--input", required=True, help="plan in the reference's INI format")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--max-histories", type=int, default=None, help="cap the histories of each field")
    ap.add_argument("--uncertainty", type=int, default=0, metavar="BATCHES",
                    help="also write the relative standard error per voxel from this many batches "
                         "(the reference's GET_UNCERTAINTY output)")
    ap.add_argument("--write-physics", metavar="FILE", default=None,
                    help="write the plan's physics tables for C/C++ callers (gegs_plan_load) and exit")
    a = ap.parse_args(argv)
    if a.write_physics:
        from . import physics_data as PD
        from .plan import load_plan
        plan = load_plan(a.input, max_histories=a.max_histories)
        PD.write_physics_file(a.write_physics, plan.job.media, plan.job.physics)
        print(f"physics for media {plan.job.media} written to {a.write_physics}")
        return
    run_plan(a.input, a.device, a.max_histories, uncertainty_batches=a.uncertainty)


if __name__ == "__main__":
    main()
