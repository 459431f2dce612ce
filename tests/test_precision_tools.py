"""Host-side logic of the precision report (no GPU)."""
from __future__ import annotations

import numpy as np

from bgk_pcm_b200.precision import errors, front_x


def test_front_x_linear_interpolation():
    phi = np.array([[1, 1, 0.5, -0.5, -1], [1, -1, -1, -1, -1], [-1, -1, -1, -1, -1.0]])
    x = front_x(phi)
    assert x[0] == 3.5 and x[1] == 1.5 and np.isnan(x[2])


def test_front_x_first_crossing_only():
    phi = np.array([[1.0, -1.0, 1.0, -1.0]])
    assert front_x(phi)[0] == 1.5


def test_errors_normalisation():
    p = {"T0": 283.0, "T_in_sol": 263.0}
    ny, nx = 4, 6
    b = {"T": np.full((ny, nx), 270.0), "phi": np.tile(np.linspace(1, -1, nx), (ny, 1)),
         "u": np.full((ny, nx), 0.01), "v": np.zeros((ny, nx))}
    a = {k: v.copy() for k, v in b.items()}
    a["T"][1, 2] += 0.2          # 0.2 K of a 20 K span
    a["phi"][0, 0] -= 0.02       # of a range of 2
    e = errors(a, b, p)
    assert abs(e["T_max"] - 0.01) < 1e-12 and abs(e["phi_max"] - 0.01) < 1e-12
    assert e["u_max"] == 0.0
    assert e["front_dx_max_cells"] == 0.0


def test_front_probes_sit_behind_the_front():
    from bgk_pcm_b200.combined import front_probes
    ny, nx = 6, 10
    phi = -np.ones((ny + 2, nx + 2))
    fronts = [2, 3, 4, 5, 6, 7]          # last liquid column (1-based) of each interior row
    for j, f in enumerate(fronts, start=1):
        phi[j, 1:f + 1] = 1.0
    pi, pj = front_probes(phi, 4, np.random.default_rng(0))
    assert len(pi) == 4
    for i, j in zip(pi, pj):
        assert i == fronts[j - 1] + 1          # the first solid cell of its row
        assert phi[j, i] < 0 and phi[j, i - 1] >= 0
