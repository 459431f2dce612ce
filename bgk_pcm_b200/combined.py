"""The combined-scale workload: a 16384 x 4096 rectangular cavity (aspect 4),
Ra 1e8, Pr 1, Stefan 0.5.

  1. FP32-deviation forward for `steps` steps, timed (GLUPS, HBM GB/s); the
     state at step steps - adj_steps is kept on the host.
  2. The gradient of a probe loss over the last `adj_steps` steps: an FP64
     smooth-form context is loaded with that state and bgk_adjoint_run
     differentiates L = sum_p phi_p^2 (64 probes on the melting front) with
     respect to the per-row hot-wall temperatures and tau_g.  The checkpoint
     schedule is chosen by the library: sqrt(N) snapshots when they fit in
     free HBM, else the binomial schedule over as many state slots as fit.
  3. FP64 central differences along `ndir` random unit directions in
     (theta, tau_g), theta the dimensionless hot-wall temperature, for step
     sizes h = 1e-6 and 1e-4 (the difference quotient of a long run carries
     rounding noise that grows with the run's length; the larger step shows
     how much of the disagreement at the smaller one is that noise).

    python -m bgk_pcm_b200.combined                      # the full workload
    python -m bgk_pcm_b200.combined --nx 512 --ny 128 --steps 2000 --adjoint-steps 200
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import inputs
from .solver import Solver

STATE_FIELDS = [f"f{k}" for k in range(9)] + [f"g{k}" for k in range(9)] + ["rho", "T", "u", "v", "phi"]


def _sync_time(fn):
    t0 = time.perf_counter()
    fn()
    return time.perf_counter() - t0


def download_state(s: Solver) -> dict:
    return {n: s.field(n) for n in STATE_FIELDS}


def fp64_from_state(p: dict, state: dict, it: int, tin=None, tau_g=None) -> Solver:
    """A smooth FP64 context holding `state` (reference layout), with the
    hot-wall temperatures `tin` per row and relaxation time `tau_g`."""
    q = dict(p)
    if tau_g is not None:
        q["tau_g"] = float(tau_g)
    s = Solver(q, smooth=True)
    s.initialization()
    for n in STATE_FIELDS:
        s.upload(n, state[n])
    s.it = it
    if tin is not None:
        s.set_tin(tin)
    s.sync()
    return s


def front_probes(phi: np.ndarray, nprobes: int, rng) -> tuple[np.ndarray, np.ndarray]:
    """Probe nodes (1-based i, j) one cell behind the first phi >= 0 > phi
    crossing of randomly chosen rows (rows without a front are skipped)."""
    inner = phi[1:-1, 1:-1]
    Ny, Nx = inner.shape
    pi, pj = [], []
    rows = rng.permutation(Ny)
    for j in rows:
        hit = np.nonzero((inner[j, :-1] >= 0.0) & (inner[j, 1:] < 0.0))[0]
        if hit.size:
            pi.append(min(int(hit[0]) + 2, Nx))
            pj.append(int(j) + 1)
        if len(pi) == nprobes:
            break
    if not pi:
        raise RuntimeError("no melting front to place probes on")
    return np.array(pi, dtype=np.int32), np.array(pj, dtype=np.int32)


def loss_fp64(p, state, it, tin, tau_g, steps, pi, pj) -> float:
    s = fp64_from_state(p, state, it, tin, tau_g)
    try:
        s.step(steps)
        phi = s.field("phi")
        return float(np.sum(phi[pj, pi] ** 2))
    finally:
        s.close()


def run(nx=16384, ny=4096, Ra=1e8, Ste=0.5, steps=50000, adj_steps=5000, ndir=8, nprobes=64, seed=0,
        h=(1e-6, 1e-4), checkpoint_every=0, precision="f32"):
    p = inputs.workload_params(Nx=nx, Ny=ny, iter=steps, Ra=Ra, Ste=Ste)
    rng = np.random.default_rng(seed)
    out = {"workload": f"cavity{nx}x{ny}_ra{Ra:.0e}_ste{Ste}", "steps": steps, "adjoint_steps": adj_steps}

    # 1. reduced-precision forward, timed; keep the state at steps - adj_steps
    s = Solver(p, precision=precision)
    s.initialization()
    s.sync()
    n0 = steps - adj_steps
    t1 = _sync_time(lambda: (s.step(n0), s.sync()))
    state = download_state(s)
    t2 = _sync_time(lambda: (s.step(adj_steps), s.sync()))
    s.close()
    nodes = nx * ny
    bpn = {"f32": 152, "f16": 80, "f32x": 160, "f64": 304}[precision]
    glups = nodes * steps / (t1 + t2) / 1e9
    out["forward"] = {"precision": precision, "glups": glups, "hbm_gbs": glups * bpn,
                      "seconds": t1 + t2, "timing": "wall clock around synchronised bgk_step calls"}

    # 2. adjoint over the last adj_steps steps, FP64 smooth form
    dT = p["T0"] - p["T_in_sol"]
    tin = np.full(ny, p["T0"])
    pi, pj = front_probes(state["phi"], nprobes, rng)
    target = np.zeros(pi.size)
    s = fp64_from_state(p, state, n0, tin)
    t0 = time.perf_counter()
    loss, g, gtau = s.adjoint(adj_steps, pi, pj, target, checkpoint_every)
    t_adj = time.perf_counter() - t0
    s.close()
    s = fp64_from_state(p, state, n0, tin)
    t_fwd = _sync_time(lambda: (s.step(adj_steps), s.sync()))
    s.close()
    out["adjoint"] = {"loss": loss, "seconds": t_adj, "forward_seconds": t_fwd, "ratio": t_adj / t_fwd,
                      "nprobes": int(pi.size), "checkpoint_every": checkpoint_every}

    # 3. FP64 central differences in (theta, tau_g), the same directions for
    # every step size h
    hs = (h,) if np.isscalar(h) else tuple(h)
    dirs = []
    for _ in range(ndir):
        v = rng.standard_normal(ny + 1)
        dirs.append(v / np.linalg.norm(v))
    out["fd"] = []
    for hh in hs:
        rows = []
        for v in dirs:
            vt, vtau = v[:-1], v[-1]
            lp = loss_fp64(p, state, n0, tin + hh * dT * vt, p["tau_g"] + hh * vtau, adj_steps, pi, pj)
            lm = loss_fp64(p, state, n0, tin - hh * dT * vt, p["tau_g"] - hh * vtau, adj_steps, pi, pj)
            fd = (lp - lm) / (2 * hh)
            ad = float(dT * (g @ vt) + gtau * vtau)
            rows.append({"fd": fd, "adjoint": ad, "rel_err": abs(fd - ad) / max(abs(ad), 1e-300)})
        out["fd"].append({"h": hh, "directions": rows, "worst_rel_err": max(r["rel_err"] for r in rows)})
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=16384)
    ap.add_argument("--ny", type=int, default=4096)
    ap.add_argument("--ra", type=float, default=1e8)
    ap.add_argument("--ste", type=float, default=0.5)
    ap.add_argument("--steps", type=int, default=50000)
    ap.add_argument("--adjoint-steps", type=int, default=5000)
    ap.add_argument("--ndir", type=int, default=8)
    ap.add_argument("--nprobes", type=int, default=64)
    ap.add_argument("--checkpoint-every", type=int, default=0)
    ap.add_argument("--precision", default="f32")
    ap.add_argument("--h", default="1e-6,1e-4", help="finite-difference steps (comma list)")
    a = ap.parse_args(argv)
    r = run(a.nx, a.ny, a.ra, a.ste, a.steps, a.adjoint_steps, a.ndir, a.nprobes,
            h=tuple(float(x) for x in a.h.split(",")), checkpoint_every=a.checkpoint_every, precision=a.precision)
    print(json.dumps(r), flush=True)


if __name__ == "__main__":
    main()
