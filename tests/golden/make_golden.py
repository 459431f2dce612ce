#!/usr/bin/env python
"""Generate golden vectors by executing the reference's own STEP_7 source.

Run where the reference sources are mounted (they are not needed afterwards),
giving the root of the reference checkout (the directory holding STEP_7/):

    python tests/golden/make_golden.py <reference root>

The STEP_7 routines (setup, initialization, BC_f, BC_g, streaming,
momentsPre, phase_field, forces, collision, moments) are translated by
fsubset.py and stepped in the order of STEP_7/main.f90's time loop, which is
read from main.f90 itself.  The heating-option cases take initialization and
BC_g from STEP_DOCONCURRENT/ with its FROMRIGHT / FROMBOTTOM macros defined.  After initialization, after the first step and
after the last step, all 46 module arrays are stored (float64, reference
layout) in one .npz per case, together with the input parameters.
"""
from __future__ import annotations

import json
import re
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import fsubset  # noqa: E402

FILES = ["setup.f90", "initialization.f90", "BC_f.f90", "BC_g.f90", "streaming.f90",
         "momentsPre.f90", "phase_field.f90", "forces.f90", "collision.f90", "moments.f90"]
FIELDS = ([f"f{k}" for k in range(9)] + [f"g{k}" for k in range(9)]
          + ["rho", "T", "u", "v", "phi", "phi_prec", "rho2", "T2", "u2", "v2"]
          + [f"fp{k}" for k in range(9)] + [f"gp{k}" for k in range(9)])
INPUT_NAMES = ["iter", "noutput", "dump", "Nx", "Ny", "Re", "rho0", "rho1", "tau_f", "tau_g", "T0",
               "T_in_sol", "grav", "eps", "stefan_number", "T_width", "length", "westBC_st",
               "eastBC_st", "northBC_st", "southBC_st"]


def cavity(Nx, Ny, **kw):
    """The benchmark cavity mapping (Ra 1e5, Pr 1, Ste 1) on a small grid."""
    import math
    rho0, rho1 = 1.0, 1.0 / 1.024
    U = 0.1 / math.sqrt(3.0)
    kvisc = U * Ny * math.sqrt(1.0 / 1e5)
    tau = 3.0 * kvisc + 0.5
    d = dict(iter=100, noutput=2, dump=0, Nx=Nx, Ny=Ny, Re=0.0, rho0=rho0, rho1=rho1, tau_f=tau, tau_g=tau,
             T0=283.0, T_in_sol=263.0, grav=U * U / (Ny * (rho0 / rho1 - 1.0)), eps=0.0, stefan_number=1.0,
             T_width=10.0, length=float(Ny), westBC=4, eastBC=4, northBC=4, southBC=4)
    d.update(kw)
    return d


# STEP_DOCONCURRENT's heating options: preprocessor macros of its
# initialization.f90 and BC_g.f90, which replace STEP_7's two routines (the
# rest of the step is STEP_7's); bits as in the oracle's orc_set_heat
HEAT_MACROS = {1: ("FROMRIGHT",), 2: ("FROMBOTTOM",), 3: ("FROMRIGHT", "FROMBOTTOM")}
HEAT_FILES = ("initialization.f90", "BC_g.f90")

# (name, params, steps): small grids the Python execution finishes in seconds
CASES = [
    ("cavity_16x12", cavity(16, 12), 12),
    ("cavity_13x7", cavity(13, 7), 8),
    ("cavity_45x6_strip", cavity(45, 6), 6),
    ("util0_like_10x14", dict(cavity(10, 14), rho0=1.024, rho1=1.0, tau_f=1.0, tau_g=0.51, T0=283.0,
                                  T_in_sol=273.0, grav=0.00025, stefan_number=0.1, length=512.0), 8),
    ("bc_periodic_inflow_9x8", cavity(9, 8, westBC=1, eastBC=3, northBC=6, southBC=6, Re=20.0), 5),
    ("bc_parabolic_sym_9x8", cavity(9, 8, westBC=2, eastBC=0, northBC=5, southBC=0, Re=20.0), 5),
    ("bc_pressure_9x8", cavity(9, 8, westBC=3, eastBC=4, northBC=1, southBC=4, Re=20.0), 5),
    # heating options (params key "heat"): FROMRIGHT on the cavity; FROMRIGHT
    # with a parabolic west inflow, where u(0,j) != 0 exposes the sign of the
    # west g polynomials; FROMBOTTOM with Ny > Nx, where the T buffer loop runs
    # past row 0; both macros; Nx >= 40 so that the liquid strip is wider
    # than the wall column
    ("heat_right_44x10", cavity(44, 10, heat=1), 8),
    ("heat_right_inflow_9x8", cavity(9, 8, westBC=2, eastBC=0, northBC=4, southBC=4, Re=20.0, heat=1), 6),
    ("heat_bottom_10x14", cavity(10, 14, heat=2), 6),
    ("heat_right_bottom_41x9", cavity(41, 9, heat=3), 6),
]


def main_loop_order(ref: Path) -> list[str]:
    stmts = fsubset.preprocess((ref / "STEP_7" / "main.f90").read_text())
    calls, inside = [], False
    for st in stmts:
        low = st.lower().replace(" ", "")
        if low.startswith("doit="):
            inside = True
            continue
        if inside:
            if low.startswith("if("):
                break
            m = re.match(r"call(\w+)", low)
            if m:
                calls.append(m.group(1))
    return calls


def run_case(ref: Path, params: dict, steps: int, order):
    heat = params.get("heat", 0)
    files = [ref / "STEP_DOCONCURRENT" / f if heat and f in HEAT_FILES else f for f in FILES]
    prog = fsubset.Program(ref / "STEP_7", files, defined=HEAT_MACROS.get(heat, ()))
    p = {}
    for nm in INPUT_NAMES:
        key = nm.replace("_st", "") if nm.endswith("_st") else nm
        p[nm] = params[key]
    prog.set_params(p)
    prog.call("setup")
    prog.call("initialization")
    Nx, Ny = params["Nx"], params["Ny"]
    snap = lambda: {f: prog.array(f, Nx, Ny) for f in FIELDS}  # noqa: E731
    out = {"init": snap()}
    for s in range(1, steps + 1):
        for c in order:
            prog.call(c)
        if s == 1:
            out["step1"] = snap()
    out[f"step{steps}"] = snap()
    return out


def main():
    import argparse
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("reference", type=Path, help="root of the reference checkout (the directory holding STEP_7/)")
    ap.add_argument("--only", default="", help="comma list of case names to regenerate (default: all)")
    a = ap.parse_args()
    ref = a.reference
    if not (ref / "STEP_7" / "main.f90").is_file():
        ap.error(f"{ref}/STEP_7/main.f90 not found")
    order = main_loop_order(ref)
    assert order == ["bc_f", "bc_g", "streaming", "momentspre", "phase_field", "forces", "collision",
                     "moments"], order
    only = set(a.only.split(",")) if a.only else None
    for name, params, steps in CASES:
        if only and name not in only:
            continue
        t0 = time.time()
        snaps = run_case(ref, params, steps, order)
        arrays = {f"{tag}/{f}": a for tag, d in snaps.items() for f, a in d.items()}
        np.savez_compressed(HERE / f"{name}.npz", **arrays)
        (HERE / f"{name}.json").write_text(json.dumps({"params": params, "steps": steps,
                                                        "snapshots": list(snaps)}, indent=1) + "\n")
        print(f"{name}: {steps} steps in {time.time() - t0:.1f}s")


if __name__ == "__main__":
    main()
