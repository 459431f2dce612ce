"""Errors of the reduced-precision forms against the FP64 path.

Per field: max-abs and RMS over the interior, normalised as the precision
targets are stated: T by the temperature span dT = T0 - T_in_sol, phi by its
range 2, u and v by max |u| of the FP64 run.  Melt front: per row, the x of
the first crossing phi_i >= 0 > phi_(i+1), linearly interpolated (the
reference detects the same crossing at row Ny/2, STEP_7/forces.f90:31-36,
and prints its integer i); reported at row Ny/2 and as the mean over the
rows where both runs have a front.

The FP64 baseline comes in two kinds: the reference's rounding (collision
temporaries as REAL(4)) and the smooth form (double throughout).  Both are
reported, together with the distance between the two, which is what the
reference's own float roundings move the FP64 result by.

    python -m bgk_pcm_b200.precision --workload cavity4096_ra1e7
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import inputs
from .solver import Solver

FIELDS = ("T", "phi", "u", "v")


def front_x(phi: np.ndarray) -> np.ndarray:
    """x (interior index i, 1-based) of the first crossing phi_i >= 0 >
    phi_(i+1) in each row of an interior field phi[j, i]; NaN where a row
    has none."""
    a, b = phi[:, :-1], phi[:, 1:]
    hit = (a >= 0.0) & (b < 0.0)
    out = np.full(phi.shape[0], np.nan)
    rows = np.nonzero(hit.any(axis=1))[0]
    i = hit[rows].argmax(axis=1)
    pa, pb = a[rows, i], b[rows, i]
    out[rows] = (i + 1) + pa / (pa - pb)
    return out


def run(params: dict, precision: str, steps: int, smooth: bool = False, tanh: str = "device") -> dict:
    s = Solver(params, precision=precision, smooth=smooth, tanh=tanh)
    try:
        s.initialization()
        s.step(steps)
        return {n: s.field(n)[1:-1, 1:-1].copy() for n in FIELDS}
    finally:
        s.close()


def errors(a: dict, b: dict, params: dict) -> dict:
    """Errors of run a against baseline b."""
    dT = params["T0"] - params["T_in_sol"]
    umax = max(np.abs(b["u"]).max(), np.abs(b["v"]).max(), 1e-300)
    scale = {"T": dT, "phi": 2.0, "u": umax, "v": umax}
    e = {}
    for n in FIELDS:
        d = a[n] - b[n]
        e[f"{n}_max"] = float(np.abs(d).max() / scale[n])
        e[f"{n}_rms"] = float(np.sqrt(np.mean(d * d)) / scale[n])
    fa, fb = front_x(a["phi"]), front_x(b["phi"])
    mid = a["phi"].shape[0] // 2
    both = ~np.isnan(fa) & ~np.isnan(fb)
    e["front_x_mid"] = float(fb[mid]) if not np.isnan(fb[mid]) else None
    e["front_dx_mid_cells"] = float(abs(fa[mid] - fb[mid])) if both[mid] else None
    e["front_dx_mean_cells"] = float(np.mean(np.abs(fa[both] - fb[both]))) if both.any() else None
    e["front_dx_max_cells"] = float(np.max(np.abs(fa[both] - fb[both]))) if both.any() else None
    return e


def report(workload: str, steps: int | None = None, forms=("f32", "f32x", "f16")) -> list:
    params = inputs.workload_params(**inputs.WORKLOADS[workload])
    steps = steps or params["iter"]
    smooth = run(params, "f64", steps, smooth=True)
    ref = run(params, "f64", steps)
    rows = [dict(workload=workload, steps=steps, form="f64 reference rounding", vs="f64 smooth",
                 **errors(ref, smooth, params))]
    for f in forms:
        lo = run(params, f, steps)
        rows.append(dict(workload=workload, steps=steps, form=f, vs="f64 smooth", **errors(lo, smooth, params)))
        rows.append(dict(workload=workload, steps=steps, form=f, vs="f64 reference rounding",
                         **errors(lo, ref, params)))
    return rows


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="cavity4096_ra1e7")
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--forms", default="f32,f32x,f16")
    a = ap.parse_args(argv)
    for r in report(a.workload, a.steps, tuple(f for f in a.forms.split(",") if f)):
        print(json.dumps(r), flush=True)


if __name__ == "__main__":
    main()
