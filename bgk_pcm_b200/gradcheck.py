"""The differentiation workload (512x512 cavity, Ra 1e5, 2000 steps): probes,
seeded parameters and the finite-difference check of the adjoint gradient.

Loss L = sum over 64 probe nodes of (phi_final - phi_target)^2, phi_target
from a run with a seeded perturbation of the hot-wall temperatures.
Parameters: Tin_j = T0 + dT * 0.05 * N(0,1) per row (the hot wall at 1 +
0.05 N(0,1) in units of the temperature span dT = T0 - T_in_sol) and tau_g.
Probes sit in the band i in [Nx/40, Nx/40 + 32] that the melting front
reaches within the run.
"""
from __future__ import annotations

import time

import numpy as np

from . import inputs
from .solver import Solver


def setup(Nx=512, Ny=512, steps=2000, Ra=1e5, seed=0, nprobes=64, **overrides):
    p = inputs.workload_params(Nx=Nx, Ny=Ny, iter=steps, Ra=Ra)
    p.update(overrides)
    rng = np.random.default_rng(seed)
    dT = p["T0"] - p["T_in_sol"]
    tin = p["T0"] + dT * 0.05 * rng.standard_normal(Ny)
    tin_target = p["T0"] + dT * 0.05 * rng.standard_normal(Ny)
    i0 = Nx // 40
    pi = i0 + rng.integers(0, min(33, Nx - i0), nprobes) if Nx - i0 > 1 else np.full(nprobes, 1)
    pi = np.clip(pi, 1, Nx)
    pj = rng.integers(1, Ny + 1, nprobes)
    return p, tin, tin_target, pi.astype(np.int32), pj.astype(np.int32)


def forward_phi(p, tin, steps, pi, pj, tau_g=None):
    q = dict(p)
    if tau_g is not None:
        q["tau_g"] = tau_g
    s = Solver(q, smooth=True)
    s.initialization()
    s.set_tin(tin)
    s.step(steps)
    phi = s.field("phi")
    s.close()
    return phi[pj, pi]


def loss_of(p, tin, steps, pi, pj, target, tau_g=None):
    r = forward_phi(p, tin, steps, pi, pj, tau_g) - target
    return float(np.sum(r * r))


def adjoint(p, tin, steps, pi, pj, target, checkpoint_every=45):
    s = Solver(p, smooth=True)
    s.initialization()
    s.set_tin(tin)
    out = s.adjoint(steps, pi, pj, target, checkpoint_every)
    s.close()
    return out


def fd_check(p, tin, steps, pi, pj, target, grad_tin, grad_tau, ndir=16, h=1e-6, seed=1, tin_unit=None):
    """Central differences along random unit directions in (theta, tau_g).

    theta is the dimensionless hot-wall temperature of the workload
    definition (hot wall 1, solid 0): Tin = T_in_sol + tin_unit * theta with
    tin_unit = T0 - T_in_sol, so a step h in theta moves Tin by h * tin_unit
    kelvin.  The derivative along v is tin_unit * <dL/dTin, v_theta> +
    dL/dtau_g * v_tau."""
    if tin_unit is None:
        tin_unit = p["T0"] - p["T_in_sol"]
    rng = np.random.default_rng(seed)
    rows = []
    for _ in range(ndir):
        v = rng.standard_normal(p["Ny"] + 1)
        v /= np.linalg.norm(v)
        vt, vtau = v[:-1], v[-1]
        lp = loss_of(p, tin + h * tin_unit * vt, steps, pi, pj, target, p["tau_g"] + h * vtau)
        lm = loss_of(p, tin - h * tin_unit * vt, steps, pi, pj, target, p["tau_g"] - h * vtau)
        fd = (lp - lm) / (2 * h)
        ad = float(tin_unit * (grad_tin @ vt) + grad_tau * vtau)
        rows.append((fd, ad, abs(fd - ad) / max(abs(ad), 1e-300)))
    return rows


def _autograd_function():
    import torch

    class AdjointLoss(torch.autograd.Function):
        """L(Tin, tau_g) of the workload; the backward pass returns the
        gradient that bgk_adjoint_run computed (ctypes, no torch kernels)."""

        @staticmethod
        def forward(ctx, tin, tau_g, p, steps, pi, pj, target, K):
            q = dict(p)
            q["tau_g"] = float(tau_g.detach().cpu())
            s = Solver(q, smooth=True)
            try:
                s.initialization()
                s.set_tin(tin.detach().cpu().numpy().astype(np.float64))
                loss, g, gtau = s.adjoint(steps, pi, pj, target, K)
            finally:
                s.close()
            ctx.save_for_backward(torch.from_numpy(g), torch.tensor(gtau, dtype=torch.float64))
            return torch.tensor(loss, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gout):
            g, gtau = ctx.saved_tensors
            return gout * g, gout * gtau, None, None, None, None, None, None

    return AdjointLoss


def adjoint_autograd(p, tin, steps, pi, pj, target, checkpoint_every=45):
    """loss, dL/dTin, dL/dtau_g through torch.autograd (the gradient-check
    harness's wrapper of the C ABI)."""
    import torch
    fn = _autograd_function()
    t = torch.tensor(np.asarray(tin, dtype=np.float64), requires_grad=True)
    tau = torch.tensor(float(p["tau_g"]), dtype=torch.float64, requires_grad=True)
    loss = fn.apply(t, tau, p, steps, pi, pj, target, checkpoint_every)
    loss.backward()
    return float(loss.detach()), t.grad.numpy().copy(), float(tau.grad)


def cost_ratio(p, tin, steps, pi, pj, target, checkpoint_every=45, repeats=3):
    """Adjoint cost / forward cost, both timed on an existing context (wall
    clock around synchronised calls, best of `repeats`): the forward solve
    excludes the context's allocation and so does the adjoint, whose
    workspace stays in the context after a first, untimed call."""
    fw, ad = [], []
    s = Solver(p, smooth=True)
    try:
        s.initialization(); s.set_tin(tin)
        s.adjoint(steps, pi, pj, target, checkpoint_every)          # workspace
        for _ in range(repeats):
            s.initialization(); s.set_tin(tin); s.sync()
            t0 = time.perf_counter(); s.step(steps); s.sync(); fw.append(time.perf_counter() - t0)
            s.initialization(); s.set_tin(tin); s.sync()
            t0 = time.perf_counter(); s.adjoint(steps, pi, pj, target, checkpoint_every)
            ad.append(time.perf_counter() - t0)
    finally:
        s.close()
    return min(ad) / min(fw), min(fw), min(ad)


def main(argv=None):
    """python -m bgk_pcm_b200.gradcheck [adjoint|cost|fd]: one adjoint
    gradient, the adjoint/forward cost, or the finite-difference check on
    the differentiation workload."""
    import argparse
    import json
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["adjoint", "cost", "fd"])
    ap.add_argument("--ndir", type=int, default=16)
    a = ap.parse_args(argv)
    p, tin, tin_t, pi, pj = setup()
    steps = p["iter"]
    target = forward_phi(p, tin_t, steps, pi, pj)
    if a.what == "adjoint":
        loss, g, gtau = adjoint(p, tin, steps, pi, pj, target)
        print(json.dumps({"loss": loss, "grad_tau_g": gtau, "grad_tin_norm": float(np.linalg.norm(g))}))
    elif a.what == "cost":
        ratio, tf, ta = cost_ratio(p, tin, steps, pi, pj, target)
        print(json.dumps({"ratio": ratio, "forward_ms": tf * 1e3, "adjoint_ms": ta * 1e3}))
    else:
        loss, g, gtau = adjoint_autograd(p, tin, steps, pi, pj, target)
        rows = fd_check(p, tin, steps, pi, pj, target, g, gtau, ndir=a.ndir)
        print(json.dumps({"loss": loss, "worst_rel_err": max(r[2] for r in rows), "rows": rows}))


if __name__ == "__main__":
    main()
