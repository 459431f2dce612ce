"""The tangent (forward-mode) oracle: its plain-double instantiation equals
the oracle's smooth form bit for bit, and its dual-number derivative agrees
with central differences of itself."""
from __future__ import annotations

import numpy as np

from conftest import small_params


def test_tangent_restatement_matches_oracle(oracle_mod):
    p = small_params(18, 13)
    o = oracle_mod.Oracle(p, smooth=True)
    o.initialization()
    o.step(15)
    phi, T = oracle_mod.tangent_plain(p, np.full(p["Ny"], p["T0"]), 15)
    np.testing.assert_array_equal(phi[1:-1, 1:-1], o.field("phi")[1:-1, 1:-1])
    np.testing.assert_array_equal(T[1:-1, 1:-1], o.field("T")[1:-1, 1:-1])


def test_tangent_matches_central_differences(oracle_mod):
    # solid just below T_crit and probes near the hot wall, so phi responds
    p = small_params(20, 14, T_in_sol=271.0)
    rng = np.random.default_rng(3)
    tin = p["T0"] + rng.standard_normal(p["Ny"])
    pi = rng.integers(1, 6, 8)
    pj = rng.integers(1, 15, 8)
    target = rng.uniform(-1, 1, 8)
    for trial in range(3):
        v = rng.standard_normal(p["Ny"] + 1)
        v /= np.linalg.norm(v)
        L, dL = oracle_mod.tangent_loss(p, tin, v[:-1], v[-1], 40, pi, pj, target)
        assert abs(dL) > 1e-6
        h = 1e-6
        pp = dict(p, tau_g=p["tau_g"] + h * v[-1])
        pm = dict(p, tau_g=p["tau_g"] - h * v[-1])
        Lp, _ = oracle_mod.tangent_loss(pp, tin + h * v[:-1], v[:-1] * 0, 0.0, 40, pi, pj, target)
        Lm, _ = oracle_mod.tangent_loss(pm, tin - h * v[:-1], v[:-1] * 0, 0.0, 40, pi, pj, target)
        fd = (Lp - Lm) / (2 * h)
        assert abs(fd - dL) <= 1e-6 * abs(dL), (fd, dL)
