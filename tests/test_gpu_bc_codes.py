"""The fused step with walls other than the no-slip code 4.

STEP_7/BC_f.f90 has, besides bounce-back (4), periodic (0), fixed-velocity
(1), parabolic inflow (2), fixed-pressure (3), symmetric (5) and open (6)
branches; no shipped input uses them, but the reference runs them.  With any
of these the f halo cells carry state (periodic copies, inflow equilibria,
values that persist from step to step), so the fused path keeps them in a
ring that a one-block boundary kernel updates before each step exactly as
BC_f does (west, east, north, south), and the step pulls from it.  Both
sides use the portable tanh, so every array must equal the oracle bit for
bit: rho, T, u, v and phi with halos, f with its halo cells, g inside.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import small_params

pytestmark = pytest.mark.gpu

MACRO = ["rho", "T", "u", "v", "phi"]

# every code on every wall it exists for (W 0-4, E 0/3/4, N 0/1/4/5/6, S 0/4/6)
MIXES = [(0, 0, 0, 0), (1, 3, 6, 4), (2, 4, 5, 6), (3, 3, 1, 4), (4, 4, 0, 0), (0, 0, 4, 4),
         (2, 3, 4, 6), (4, 0, 5, 4), (1, 4, 1, 0), (3, 0, 6, 6), (4, 4, 4, 6), (4, 3, 4, 4)]


def _pair(oracle_mod, Nx, Ny, bcs, **kw):
    from bgk_pcm_b200 import Solver
    w, e, n, s_ = bcs
    p = small_params(Nx, Ny, westBC=w, eastBC=e, northBC=n, southBC=s_, Re=5.0)
    o = oracle_mod.Oracle(p, tanh="portable", smooth=kw.get("smooth", False))
    o.initialization()
    s = Solver(p, tanh="portable", **kw)
    s.initialization()
    return o, s


def _assert_equal(o, s, what):
    for name in MACRO:
        np.testing.assert_array_equal(s.field(name), o.field(name), err_msg=f"{name} {what}")
    for k in range(9):
        np.testing.assert_array_equal(s.field(f"f{k}"), o.field(f"f{k}"), err_msg=f"f{k} (with halos) {what}")
        np.testing.assert_array_equal(s.field(f"g{k}")[1:-1, 1:-1], o.field(f"g{k}")[1:-1, 1:-1],
                                      err_msg=f"g{k} {what}")


@pytest.mark.parametrize("bcs", MIXES)
@pytest.mark.parametrize("Nx,Ny", [(12, 9), (131, 37)])
def test_fused_other_wall_codes_bit_exact(oracle_mod, lib, bcs, Nx, Ny):
    o, s = _pair(oracle_mod, Nx, Ny, bcs)
    done = 0
    for n in (1, 2, 5):
        o.step(n)
        s.step(n)
        done += n
        _assert_equal(o, s, f"walls {bcs} after {done} steps")
    s.close()
    o.close()


@pytest.mark.parametrize("bcs", [(0, 0, 0, 0), (3, 3, 1, 4), (2, 4, 5, 6)])
def test_fused_and_staged_interleave_with_other_wall_codes(oracle_mod, lib, bcs):
    """Staged and fused steps switch at step boundaries; the f halo cells
    move between the ring and the staged arrays."""
    o, s = _pair(oracle_mod, 20, 11, bcs)
    s.step(2); o.step(2)
    s.staged_step(); o.step(1)
    s.step(3); o.step(3)
    s.staged_step(); s.staged_step(); o.step(2)
    s.step(1); o.step(1)
    _assert_equal(o, s, f"walls {bcs} after interleaving")
    s.close()
    o.close()


def test_snapshot_keeps_the_halo_ring(oracle_mod, lib, tmp_path):
    from bgk_pcm_b200 import Solver
    o, s = _pair(oracle_mod, 17, 13, (1, 3, 6, 4))
    s.step(4); o.step(4)
    s.save(tmp_path / "ring.bin")
    b = Solver(s.params, tanh="portable")
    b.load(tmp_path / "ring.bin")
    b.step(3); o.step(3)
    _assert_equal(o, b, "after a snapshot round trip")
    b.close()
    s.close()
    o.close()


def test_fma_variant_with_other_wall_codes(oracle_mod, lib):
    """The FMA-contracted variant runs the same ring; in the smooth form it
    stays within max-abs 1e-10 of the oracle."""
    o, s = _pair(oracle_mod, 40, 24, (2, 3, 4, 6), fma=True, smooth=True)
    o.step(50)
    s.step(50)
    for name in MACRO:
        d = np.abs(s.field(name) - o.field(name)).max()
        assert d <= 1e-10, f"{name}: max-abs {d:.3e}"
    s.close()
    o.close()
