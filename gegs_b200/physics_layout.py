"""Layout of the physics-table block shared by the CUDA library and the CPU oracle.

The transport kernels read EGSnrc-style interpolation tables (log-linear
``a + b*ln(E)`` pairs, Rayleigh form-factor CDFs, Goudsmit-Saunderson
multiple-scattering surfaces, shell/edge data).  In the reference these are
``__device__`` globals filled by HATCH (``commonBlocks dev.h:11-262``,
``media.cu:96-100``).  Here they travel as ONE flat block
whose field order is fixed by :data:`FIELDS`; ``include/gegs_physics.h`` is
generated from the same list (see :func:`render_header`) so the C struct, the
numpy structured dtype and the blob bytes always agree.

Every field is float32 or int32 and every array starts on a 16-byte boundary
(explicit ``_padN`` members), so the C struct has no compiler padding and the
numpy dtype offsets equal the C ``offsetof`` values.

Index conventions follow the reference exactly (e.g. ``gmfp[med*MXGE+lgle]``,
``zelem[k*MXMED+med]``, ``dl1[med*8+l]``, ``sig[qel*MXEKE*MXMED+med*MXEKE+i]``),
so each kernel statement can be checked against the reference line it restates.
"""
from __future__ import annotations

import numpy as np

# Table dimensions (EGSnrc_Parameters.h:2-75)
MXMED = 6
MXGE = 200
MXEKE = 150
MXEL = 10
MXRAYFF = 100
RAYCDFSIZE = 100
MXELEMENT = 100
MXSHELL = 6
MXTRANS = 39
MXEDGE = 16
MXTOTSH = 1538
MXMDSH = 50
MAX_EII_SHELLS = 40
N_EII_BINS = 250
MAX_EII_BINS = N_EII_BINS * MAX_EII_SHELLS
MAXL_MS = 63
MAXQ_MS = 7
MAXU_MS = 31
MS_SIZE = (MAXL_MS + 1) * (MAXQ_MS + 1) * (MAXU_MS + 1)

CONSTANTS = dict(
    MXMED=MXMED, MXGE=MXGE, MXEKE=MXEKE, MXEL=MXEL, MXRAYFF=MXRAYFF,
    RAYCDFSIZE=RAYCDFSIZE, MXELEMENT=MXELEMENT, MXSHELL=MXSHELL,
    MXTRANS=MXTRANS, MXEDGE=MXEDGE, MXTOTSH=MXTOTSH, MXMDSH=MXMDSH,
    MAX_EII_SHELLS=MAX_EII_SHELLS, N_EII_BINS=N_EII_BINS,
    MAXL_MS=MAXL_MS, MAXQ_MS=MAXQ_MS, MAXU_MS=MAXU_MS,
)

F, I = "f", "i"

# (name, kind, shape).  A trailing 2 in the shape is a float2 pair (x, y).
FIELDS = [
    # ---- global scalars -------------------------------------------------
    ("nmed", I, ()),
    ("rm", F, ()), ("prm", F, ()), ("rmt2", F, ()), ("rmsq", F, ()),
    ("estepe", F, ()), ("ximax", F, ()), ("skindepth_for_bca", F, ()),
    ("transport_algorithm", I, ()), ("exact_bca", I, ()), ("spin_effects", I, ()),
    ("ibrdst", I, ()), ("iprdst", I, ()), ("nbr_split", I, ()), ("eii_flag", I, ()),
    # ---- per-medium scalars (thresh, media, brempr, elecin) ----------------
    ("rho", F, (MXMED,)), ("ae", F, (MXMED,)), ("ap", F, (MXMED,)),
    ("ue", F, (MXMED,)), ("up", F, (MXMED,)), ("te", F, (MXMED,)),
    ("thmoll", F, (MXMED,)), ("rlc", F, (MXMED,)), ("delcm", F, (MXMED,)),
    ("zbrang", F, (MXMED,)), ("lzbrang", F, (MXMED,)), ("log_ap", F, (MXMED,)),
    ("blcc", F, (MXMED,)), ("xcc", F, (MXMED,)), ("expeke1", F, (MXMED,)),
    ("smaxir", F, (MXMED,)), ("e_max_rr", F, (MXMED,)), ("i_do_rr", I, (MXMED,)),
    ("nne", I, (MXMED,)),
    ("zelem", F, (MXEL * MXMED,)), ("pz", F, (MXEL * MXMED,)), ("wa", F, (MXEL * MXMED,)),
    ("dl1", F, (8 * MXMED,)), ("dl2", F, (8 * MXMED,)), ("dl3", F, (8 * MXMED,)),
    ("dl4", F, (8 * MXMED,)), ("dl5", F, (8 * MXMED,)), ("dl6", F, (8 * MXMED,)),
    ("bpar", F, (2 * MXMED,)),
    # ---- photon tables (photin) -----------------------------------------
    ("ge", F, (MXMED, 2)),
    ("gmfp", F, (MXMED * MXGE, 2)), ("gbr1", F, (MXMED * MXGE, 2)),
    ("gbr2", F, (MXMED * MXGE, 2)), ("cohe", F, (MXMED * MXGE, 2)),
    ("pmax", F, (MXMED * MXGE, 2)),
    ("rayleigh_data", F, (MXMED * MXRAYFF, 4)),      # xgrid, fcum, b_array, c_array
    ("i_array", I, (MXMED * RAYCDFSIZE,)),
    # ---- electron tables (elecin) ---------------------------------------
    ("eke01", F, (MXMED, 2)),
    ("sig", F, (2 * MXMED * MXEKE, 2)), ("dedx", F, (2 * MXMED * MXEKE, 2)),
    ("ebr1", F, (MXMED * MXEKE, 2)), ("pbr1", F, (MXMED * MXEKE, 2)),
    ("pbr2", F, (MXMED * MXEKE, 2)), ("tmxs", F, (MXMED * MXEKE, 2)),
    ("range_ep", F, (2 * MXEKE * MXMED,)), ("e_array", F, (MXEKE * MXMED,)),
    ("sig_e", F, (2 * MXMED,)), ("sig_ismonotone", I, (2 * MXMED,)),
    # ---- edge / relaxation (edge) ---------------------------------------
    ("binding_energies", F, (MXSHELL * MXELEMENT,)),
    ("interaction_prob", F, (MXSHELL * MXELEMENT,)),
    ("relaxation_prob", F, (MXTRANS * MXELEMENT,)),
    ("edge_energies", F, (MXEDGE * MXELEMENT,)),
    ("edge_a", F, (MXEDGE * MXELEMENT,)), ("edge_b", F, (MXEDGE * MXELEMENT,)),
    ("edge_c", F, (MXEDGE * MXELEMENT,)), ("edge_d", F, (MXEDGE * MXELEMENT,)),
    ("edge_number", I, (MXELEMENT,)),
    # ---- bound Compton (compton_data) -----------------------------------
    ("iz_array", I, (MXTOTSH,)), ("shn_array", I, (MXTOTSH,)), ("ne_array", I, (MXTOTSH,)),
    ("be_array", F, (MXTOTSH,)), ("jo_array", F, (MXTOTSH,)), ("erfjo_array", F, (MXTOTSH,)),
    ("shell_array", I, (MXMDSH * MXMED,)), ("eno_array", F, (MXMDSH * MXMED,)),
    ("eno_atbin_array", I, (MXMDSH * MXMED,)), ("n_shell", I, (MXMED,)),
    # ---- screened-Rutherford multiple scattering (ms_data) --------------
    ("llammin", F, ()), ("llammax", F, ()), ("dllamb", F, ()), ("dllambi", F, ()),
    ("dqms", F, ()), ("dqmsi", F, ()),
    ("ums_array", F, (MS_SIZE,)), ("fms_array", F, (MS_SIZE,)),
    ("wms_array", F, (MS_SIZE,)), ("ims_array", I, (MS_SIZE,)),
    # ---- electron impact ionisation (eii_data) --------------------------
    ("eii_xsection", F, (MAX_EII_BINS, 2)), ("eii_cons", F, (MXMED,)),
    ("eii", F, (MAX_EII_SHELLS, 2)),
    ("eii_z", I, (MAX_EII_SHELLS,)), ("eii_sh", I, (MAX_EII_SHELLS,)),
    ("eii_nshells", I, (MXELEMENT,)), ("eii_nsh", I, (MXMED,)),
    ("eii_first", I, (MXMED * MXEL,)), ("eii_no", I, (MXMED * MXEL,)),
]


def padded_fields():
    """FIELDS with int32 padding so every array field starts on a 16-byte
    boundary (the kernels read float2/float4 table entries with vector loads)."""
    out, off, k = [], 0, 0
    for name, kind, shape in FIELDS:
        if shape and off % 16:
            npad = (16 - off % 16) // 4
            out.append((f"_pad{k}", I, (npad,)))
            off += 4 * npad
            k += 1
        out.append((name, kind, shape))
        off += 4 * int(np.prod(shape)) if shape else 4
    if off % 16:
        out.append((f"_pad{k}", I, ((16 - off % 16) // 4,)))
    return out


def dtype() -> np.dtype:
    """numpy structured dtype equal, byte for byte, to ``struct gegs_physics``."""
    parts = []
    for name, kind, shape in padded_fields():
        base = np.float32 if kind == F else np.int32
        parts.append((name, base, shape) if shape else (name, base))
    dt = np.dtype(parts, align=False)
    return dt


def new_block() -> np.ndarray:
    """Zero-initialised physics block (a 0-d structured array)."""
    return np.zeros((), dtype=dtype())


def render_header() -> str:
    """C header text for the block (kept in ``include/gegs_physics.h``)."""
    out = []
    out.append("/* Generated from gegs_b200/physics_layout.py -- edit the field list there.\n"
               " *\n"
               " * Physics-table block read by the transport kernels.  Same content and\n"
               " * index conventions as the reference's __device__ globals\n"
               " * (commonBlocks dev.h:11-262, media.cu:96-100); float2 pairs are float[2].\n"
               " * Every member is 4 bytes wide; _padN members put every array on a\n"
               " * 16-byte boundary so the kernels can use float2/float4 loads. */\n")
    out.append("#ifndef GEGS_PHYSICS_H\n#define GEGS_PHYSICS_H\n\n#include <stdint.h>\n\n")
    for k, v in CONSTANTS.items():
        out.append(f"#define GEGS_{k} {v}\n")
    out.append(f"#define GEGS_MS_SIZE {MS_SIZE}\n")
    out.append(f"#define GEGS_MAX_EII_BINS {MAX_EII_BINS}\n\n")
    out.append("typedef struct gegs_physics {\n")
    for name, kind, shape in padded_fields():
        ctype = "float" if kind == F else "int32_t"
        dims = "".join(f"[{d}]" for d in shape)
        out.append(f"    {ctype} {name}{dims};\n")
    out.append("} gegs_physics;\n\n")
    out.append("/* X-macro over the float members (every value must be finite; checked by\n"
               " * gegs_check_physics before a block is used). */\n")
    out.append("#define GEGS_PHYSICS_FLOAT_MEMBERS(X) \\\n")
    names = [name for name, kind, _ in FIELDS if kind == F]
    for i, name in enumerate(names):
        out.append(f"    X({name})" + (" \\\n" if i + 1 < len(names) else "\n"))
    out.append("\n#endif /* GEGS_PHYSICS_H */\n")
    return "".join(out)


if __name__ == "__main__":  # regenerate the header
    import pathlib
    p = pathlib.Path(__file__).resolve().parents[1] / "include" / "gegs_physics.h"
    p.write_text(render_header())
    print(p, dtype().itemsize, "bytes")
