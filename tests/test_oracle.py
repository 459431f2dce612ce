"""CPU checks of the oracle itself: thread determinism (the reference's
RunMe_thread.sh md5 check), conservation identities of the collision, input
parsing, and the portable tanh used for bit-exact GPU parity."""
from __future__ import annotations

import math
import struct

import numpy as np
import pytest

from conftest import ROOT, small_params


def test_threads_bit_identical(oracle_mod):
    p = small_params(48, 40)
    runs = []
    for th in (1, 3, 8):
        o = oracle_mod.Oracle(p, threads=th)
        o.initialization()
        o.step(60)
        runs.append({n: o.field(n) for n in ("rho", "T", "u", "v", "phi", "f5", "g7")})
    for r in runs[1:]:
        for n in r:
            np.testing.assert_array_equal(r[n], runs[0][n], err_msg=n)


def test_collision_conserves_node_moments(oracle_mod):
    """Regularized BGK keeps sum f = rho and sum g = T per node (the
    non-equilibrium part carries no mass): collision.f90:94-111.  The
    reference keeps its regularized populations ft0..ft8 / gt0..gt8 in
    implicit REAL(4) variables, so the identity holds to float precision
    (|1-omega| * sum|ft| * 2**-24), not to double precision."""
    o = oracle_mod.Oracle(small_params(20, 16))
    o.initialization()
    o.step(25)
    for st in ("bc_f", "bc_g", "streaming", "moments_pre", "phase_field", "forces"):
        o.stage(st)
    rho, T = o.field("rho"), o.field("T")
    o.stage("collision")
    sf = sum(o.field(f"f{k}") for k in range(9))
    sg = sum(o.field(f"g{k}") for k in range(9))
    np.testing.assert_allclose(sf[1:-1, 1:-1], rho[1:-1, 1:-1], rtol=2e-7)
    np.testing.assert_allclose(sg[1:-1, 1:-1], T[1:-1, 1:-1], rtol=2e-7)
    # and it is not exact in double: the float rounding is really there
    assert np.abs(sg[1:-1, 1:-1] - T[1:-1, 1:-1]).max() > 0


def test_equilibrium_solid_is_stationary(oracle_mod):
    """A uniform solid far below T_crit with no gravity stays put."""
    p = small_params(24, 24, grav=0.0, T0=200.0, T_in_sol=200.0 - 1e-3)
    o = oracle_mod.Oracle(p)
    o.initialization()
    T0 = o.field("T").copy()
    o.step(50)
    T = o.field("T")
    # the liquid strip at i <= Nx/40 = 0 is only the wall column; interior
    # stays within roundoff of the initial uniform solid state away from it
    assert np.abs(T[1:-1, 3:-1] - T0[1:-1, 3:-1]).max() < 1e-3
    assert np.all(np.abs(o.field("u")[1:-1, 1:-1]) < 1e-6)


def test_initial_condition(oracle_mod):
    p = small_params(80, 10)
    o = oracle_mod.Oracle(p)
    o.initialization()
    T, rho, phi = o.field("T"), o.field("rho"), o.field("phi")
    interf = 80 // 40
    assert np.all(T[:, : interf + 1] == 283.0) and np.all(T[:, interf + 1:] == 263.0)
    assert np.all(rho[:, : interf + 1] == p["rho1"]) and np.all(rho[:, interf + 1:] == 1.0)
    assert np.all(phi[:, : interf + 1] == 1.0) and np.all(phi[:, interf + 1:] == -1.0)
    w = [4 / 9] + [1 / 9] * 4 + [1 / 36] * 4
    for k in range(9):
        np.testing.assert_array_equal(o.field(f"f{k}"), w[k] * rho * 1.0)


UTIL_LIKE = """  iter                50000         ! tempo totale della simulazione
  noutput                2       ! numero di output
  dump                   0           ! restart [0 , 1]
  Nx\t\t       128          ! nodi x-direction
  Ny                   512          ! nodi y-direction
  Re\t\t         0.d0          ! Reynolds number
  rho0                   1.0240d0      ! density of the SOLID phase
  rho1                   1.000d0       ! density of the MELTED phase
  tau_f                  1.000d0       ! relaxation-time
  tau_g                  0.510d0       ! thermal relaxation-time
  T0                   283.d0          ! temperature
  T_in_sol\t       273.0d0         ! Initial Temperature for the SOLID phase
  grav\t\t\t 0.00025d0    ! gravity
  eps\t\t\t 0.00\t       ! volume fraction
  stefan_number\t\t 0.10d0\t       ! Stefan Number
  T_width               10.0d0\t       ! T_width
  length               512.d0        ! lunghezza caratteristica
  westBC_st \t\t 4             ! west bc  - structured   [0 , 1 , 2 , 4]
  eastBC_st \t \t 4             ! east bc  - structured   [0 , 3 , 4    ]
  northBC_st             4             ! north bc - structured   [1 , 4 , 5 , 6]
  southBC_st             4             ! south bc - structured   [4 , 6        ]


 INSTRUCTIONS
"""


def test_input_parsers_agree(oracle_mod, tmp_path):
    from bgk_pcm_b200 import inputs
    f = tmp_path / "input.dat"
    f.write_text(UTIL_LIKE)
    a = oracle_mod.read_input(f)
    b = inputs.read(f)
    assert a == b
    assert a["Nx"] == 128 and a["rho0"] == 1.024 and a["tau_g"] == 0.51 and a["grav"] == 0.00025


def test_input_parser_capi_no_gpu(lib, tmp_path):
    """bgk_read_input is host code: it works without a GPU."""
    from bgk_pcm_b200 import read_input
    f = tmp_path / "input.dat"
    f.write_text(UTIL_LIKE)
    p = read_input(f).as_dict()
    from bgk_pcm_b200 import inputs
    assert p == inputs.read(f)


def test_input_parser_rejects_truncated(lib, tmp_path):
    from bgk_pcm_b200 import BGKError, read_input
    f = tmp_path / "input.dat"
    f.write_text("\n".join(UTIL_LIKE.splitlines()[:7]) + "\n")
    with pytest.raises(BGKError, match="BGK_ERR_IO"):
        read_input(f)


def _ulps(a, b):
    ia = struct.unpack("<q", struct.pack("<d", a))[0]
    ib = struct.unpack("<q", struct.pack("<d", b))[0]
    return abs(ia - ib)


def test_portable_tanh_accuracy(oracle_mod):
    xs = np.concatenate([np.linspace(-25, 25, 20001), np.geomspace(1e-300, 1, 2000),
                         -np.geomspace(1e-20, 3, 500)])
    worst = max(_ulps(oracle_mod.portable_tanh(float(x)), math.tanh(float(x))) for x in xs)
    assert worst <= 4, worst
    assert oracle_mod.portable_tanh(0.0) == 0.0 and math.copysign(1, oracle_mod.portable_tanh(-0.0)) < 0


def test_workload_mapping():
    from bgk_pcm_b200 import inputs
    for name, w in inputs.WORKLOADS.items():
        v = inputs.read(ROOT / "bgk_pcm_b200" / "inputs" / name / "input.dat")
        assert v == inputs.workload_params(**w)
        d = inputs.diag_numbers(v)
        assert abs(d["Ra"] / w["Ra"] - 1) < 1e-12 and abs(d["Pr"] - w["Pr"]) < 1e-12
        assert v["Nx"] == w["Nx"] and v["Ny"] == w["Ny"] and v["stefan_number"] == w["Ste"]


def test_thread_sweep_matches_across_thread_counts(oracle_mod):
    """oracle/thread_sweep.py, the counterpart of UTIL/RunMe_thread.sh: the
    same fields (md5) at every thread count, and a positive rate."""
    from oracle import thread_sweep
    p = small_params(40, 28)
    rows = thread_sweep.threads_sweep(p, 6, 4)
    assert [r["threads"] for r in rows] == [4, 2, 1]
    assert len({r["md5"] for r in rows}) == 1
    assert all(r["mlups"] > 0 for r in rows)
    assert thread_sweep.thread_counts(6) == [6, 4, 2, 1]
