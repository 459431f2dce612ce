"""The heating options of the reference's STEP_DOCONCURRENT build
(preprocessor macros FROMRIGHT and FROMBOTTOM; here bgk_options.heat bits)
against the oracle, whose two changed routines are pinned to
STEP_DOCONCURRENT's own source by the heat_* golden fixtures.

* FROMRIGHT (STEP_DOCONCURRENT/BC_g.f90:13-45): the east wall at Tin, the
  west wall zero-gradient in T with the lagged T(1,j); the fused step runs it
  on the halo-ring path, with bc_prep reading T(1,j) from the mirror before
  every step.
* FROMBOTTOM (STEP_DOCONCURRENT/initialization.f90:16-28,123-127): the
  initial liquid layer along the south wall, and the T buffer loop that runs
  past row 0 when Ny > Nx.

Both sides use the portable tanh, so every array equals the oracle bit for
bit: rho, T, u, v, phi with halos, f with its halo cells, g inside (the
staged path also g with halos).
"""
from __future__ import annotations

import subprocess

import numpy as np
import pytest

from conftest import ROOT, small_params

pytestmark = pytest.mark.gpu

MACRO = ["rho", "T", "u", "v", "phi"]
RIGHT, BOTTOM = 1, 2


def _pair(oracle_mod, Nx, Ny, heat, walls=(4, 4, 4, 4), **kw):
    from bgk_pcm_b200 import Solver
    w, e, n, s_ = walls
    p = small_params(Nx, Ny, westBC=w, eastBC=e, northBC=n, southBC=s_, Re=5.0 if walls != (4, 4, 4, 4) else 0.0)
    o = oracle_mod.Oracle(p, tanh="portable", heat=heat)
    o.initialization()
    s = Solver(p, tanh="portable", heat=heat, **kw)
    s.initialization()
    return o, s


def _assert_equal(o, s, what, f_halos=False, g_halos=False):
    """f halo cells are state on the ring path (FROMRIGHT or a wall other
    than code 4) and in the staged arrays; g halo cells only in the latter."""
    for name in MACRO:
        np.testing.assert_array_equal(s.field(name), o.field(name), err_msg=f"{name} {what}")
    for k in range(9):
        for pop, halos in (("f", f_halos), ("g", g_halos)):
            a, b = s.field(f"{pop}{k}"), o.field(f"{pop}{k}")
            if not halos:
                a, b = a[1:-1, 1:-1], b[1:-1, 1:-1]
            np.testing.assert_array_equal(a, b, err_msg=f"{pop}{k} {what}")


CASES = [(RIGHT, 44, 10, (4, 4, 4, 4)), (RIGHT, 131, 37, (4, 4, 4, 4)), (RIGHT, 96, 40, (2, 0, 4, 4)),
         (RIGHT, 83, 29, (1, 3, 6, 4)), (BOTTOM, 30, 45, (4, 4, 4, 4)), (BOTTOM, 131, 37, (4, 4, 4, 4)),
         (BOTTOM, 50, 20, (3, 3, 1, 4)), (RIGHT | BOTTOM, 41, 9, (4, 4, 4, 4)),
         (RIGHT | BOTTOM, 90, 130, (4, 4, 4, 4))]


@pytest.mark.parametrize("heat,Nx,Ny,walls", CASES)
def test_fused_heat_options_bit_exact(oracle_mod, lib, heat, Nx, Ny, walls):
    o, s = _pair(oracle_mod, Nx, Ny, heat, walls)
    ring = bool(heat & RIGHT) or walls != (4, 4, 4, 4)
    _assert_equal(o, s, f"heat {heat} walls {walls} after initialization")
    done = 0
    for n in (1, 2, 5, 40):
        o.step(n)
        s.step(n)
        done += n
        _assert_equal(o, s, f"heat {heat} walls {walls} after {done} steps", f_halos=ring)
    s.close()
    o.close()


@pytest.mark.parametrize("heat", [RIGHT, BOTTOM, RIGHT | BOTTOM])
def test_staged_heat_options_bit_exact(oracle_mod, lib, heat):
    """The stage entry points (bgk_bc_g carries the FROMRIGHT branch), with
    the g halo cells BC_g writes."""
    o, s = _pair(oracle_mod, 45, 50, heat)
    for step in range(3):
        for st in o.STAGES:
            o.stage(st)
        s.staged_step()
        _assert_equal(o, s, f"heat {heat} staged step {step + 1}", f_halos=True, g_halos=True)
    s.close()
    o.close()


def test_heat_right_fused_and_staged_interleave(oracle_mod, lib):
    o, s = _pair(oracle_mod, 60, 21, RIGHT, (2, 4, 5, 6))
    s.step(2); o.step(2)
    s.staged_step(); o.step(1)
    s.step(3); o.step(3)
    s.staged_step(); s.staged_step(); o.step(2)
    s.step(1); o.step(1)
    _assert_equal(o, s, "after interleaving", f_halos=True)
    s.close()
    o.close()


def test_heat_right_upload_of_t_feeds_the_west_wall(oracle_mod, lib):
    """The west wall's T(1,j) is read from the T array each step: an uploaded
    T changes the next step exactly as it does in the reference."""
    o, s = _pair(oracle_mod, 44, 12, RIGHT)
    o.step(3); s.step(3)
    T = o.field("T")
    T[1:-1, 1] += np.linspace(0.0, 2.0, T.shape[0] - 2)
    o.set_field("T", T)
    s.upload("T", T)
    o.step(4); s.step(4)
    _assert_equal(o, s, "after a T upload", f_halos=True)
    s.close()
    o.close()


def test_heat_bottom_reduced_precision_starts_from_the_same_state(oracle_mod, lib):
    """FROMBOTTOM changes only the initial condition, so the FP32 form runs
    it; its initial rho/T/phi equal the oracle's and it stays within the FP32
    form's usual distance of FP64 over 200 steps."""
    from bgk_pcm_b200 import Solver
    p = small_params(64, 80)
    o = oracle_mod.Oracle(p, tanh="portable", heat=BOTTOM)
    o.initialization()
    s = Solver(p, precision="f32", heat="bottom")
    s.initialization()
    for name in ("rho", "T", "phi"):
        np.testing.assert_array_equal(s.field(name), o.field(name), err_msg=name)
    o.step(200)
    s.step(200)
    dT = p["T0"] - p["T_in_sol"]
    err = np.abs(s.field("T")[1:-1, 1:-1] - o.field("T")[1:-1, 1:-1]).max() / dT
    assert err <= 1e-4, err
    s.close()
    o.close()


def test_heat_option_refusals(lib):
    from bgk_pcm_b200 import Solver, capi
    p = small_params(48, 16)
    with pytest.raises(capi.BGKError, match="FP64"):
        Solver(p, precision="f32", heat="right")
    with pytest.raises(capi.BGKError):
        Solver(p, heat=4)
    with pytest.raises(ValueError):
        Solver(p, heat="left")
    s = Solver(p, heat="right")
    s.initialization()
    with pytest.raises(capi.BGKError, match="west"):
        s.set_tin(np.full(16, 290.0))
    with pytest.raises(capi.BGKError):
        s.advance(2)
    s.close()
    import torch
    buf = torch.empty(1 << 20, dtype=torch.uint8, device="cuda")
    b = Solver(p, heat="bottom")
    b.initialization()
    with pytest.raises(capi.BGKError, match="west"):
        b.rows_pack(0, 2, buf.data_ptr())
    b.close()


@pytest.mark.parametrize("flag,bits", [("right", RIGHT), ("bottom", BOTTOM), ("right+bottom", RIGHT | BOTTOM)])
def test_host_program_heat_matches_oracle_program(tmp_path, oracle_mod, lib, flag, bits):
    """bgk_thermal --heat against the oracle's program built with the
    FROMRIGHT / FROMBOTTOM branches: the same output files, bit for bit
    (field_check's means to 1e-7, as for the west-heated program)."""
    from bgk_pcm_b200 import build, inputs
    from test_gpu_host import numbers
    build.build()
    p = small_params(80, 40)
    p.update(iter=2000, noutput=2)
    dirs = {}
    for who in ("oracle", "gpu"):
        d = tmp_path / who
        d.mkdir()
        inputs.write(d / "input.dat", p)
        dirs[who] = d
    oracle_mod.run_main(dirs["oracle"], threads=4, tanh_mode=1, heat=bits)
    r = subprocess.run([str(ROOT / "bgk_pcm_b200" / "bgk_thermal"), str(dirs["gpu"]), "--heat", flag],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert ("Heating from right" if bits & RIGHT else "Heating from left") in r.stdout
    for name in ["fort.666", "fort.667", "fort.668", "non-dim_bulk_numbers.dat", "Output_00002000.vtk"]:
        np.testing.assert_array_equal(numbers(dirs["gpu"] / name), numbers(dirs["oracle"] / name), err_msg=name)
    np.testing.assert_allclose(numbers(dirs["gpu"] / "fort.64"), numbers(dirs["oracle"] / "fort.64"), rtol=1e-7)


def test_heat_snapshot_round_trip_and_mismatch(oracle_mod, lib, tmp_path):
    """A FROMRIGHT snapshot restores bit for bit into a FROMRIGHT context
    and is refused by a west-heated one."""
    from bgk_pcm_b200 import Solver, capi
    o, s = _pair(oracle_mod, 44, 12, RIGHT)
    s.step(3); o.step(3)
    s.save(tmp_path / "right.bin")
    b = Solver(s.params, tanh="portable", heat="right")
    b.load(tmp_path / "right.bin")
    b.step(4); o.step(4)
    _assert_equal(o, b, "after a snapshot round trip", f_halos=True)
    w = Solver(s.params, tanh="portable")
    with pytest.raises(capi.BGKError, match="heat"):
        w.load(tmp_path / "right.bin")
    for x in (w, b, s, o):
        x.close()


def test_heat_right_fma_variant_smooth(oracle_mod, lib):
    """The FMA-contracted FP64 variant runs FROMRIGHT on the same ring path;
    in the smooth form it stays within max-abs 1e-10 of the oracle."""
    from bgk_pcm_b200 import Solver
    p = small_params(80, 30)
    o = oracle_mod.Oracle(p, tanh="portable", smooth=True, heat=RIGHT)
    o.initialization()
    s = Solver(p, tanh="portable", fma=True, smooth=True, heat="right")
    s.initialization()
    o.step(60)
    s.step(60)
    for name in MACRO:
        d = np.abs(s.field(name) - o.field(name)).max()
        assert d <= 1e-10, f"{name}: max-abs {d:.3e}"
    s.close()
    o.close()


@pytest.mark.parametrize("heat,walls", [(RIGHT, (4, 4, 4, 4)), (BOTTOM, (4, 4, 4, 4)), (RIGHT | BOTTOM, (4, 4, 4, 4)),
                                        (RIGHT, (2, 0, 4, 6))])
def test_heat_options_long_run_bit_exact(oracle_mod, lib, heat, walls):
    """2000 steps in calls of 1000 (the plain steps replay captured step
    graphs on this grid, through the halo-ring update for FROMRIGHT): every
    array still equals the oracle bit for bit."""
    o, s = _pair(oracle_mod, 200, 96, heat, walls)
    ring = bool(heat & RIGHT) or walls != (4, 4, 4, 4)
    for _ in range(2):
        o.step(1000)
        s.step(1000)
    _assert_equal(o, s, f"heat {heat} walls {walls} after 2000 steps", f_halos=ring)
    s.close()
    o.close()
