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
