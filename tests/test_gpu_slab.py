"""The y-slab decomposition on one GPU: several contexts, each a slab of rows
with ghost rows, stepped through SlabRun with the LocalTransport (packed rows
copied device to device).  Every owned row must equal the undivided run bit
for bit in every precision form, since the node arithmetic does not depend
on the decomposition; the field sums add in another order and agree to
rounding."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import small_params

pytestmark = pytest.mark.gpu

MACRO = ["rho", "T", "u", "v", "phi"]
POPS = ["f2", "f4", "f5", "f7", "g1", "g4", "g6", "g8"]


def undivided(params, steps, precision, tin=None, chunks=None):
    from bgk_pcm_b200 import Solver
    with Solver(params, precision=precision) as s:
        s.initialization()
        if tin is not None:
            s.set_tin(tin)
        for n in (chunks or [steps]):
            s.step(n)
        return {n: s.field(n) for n in MACRO + POPS}, s.sums()


def check(run, ref, sums):
    for n in MACRO:
        np.testing.assert_array_equal(run.field(n), ref[n], err_msg=n)
    for n in POPS:
        np.testing.assert_array_equal(run.field(n)[1:-1], ref[n][1:-1], err_msg=n)
    s = run.sums()
    np.testing.assert_allclose(s[:3], sums[:3], rtol=1e-12, atol=0)
    assert s[3] == sums[3]


@pytest.mark.parametrize("precision,nslabs,halo,steps", [
    ("f64", 3, 1, 7), ("f64", 3, 4, 13), ("f64", 2, 3, 2), ("f64", 4, 5, 23),
    ("f32", 3, 2, 9), ("f16", 2, 4, 10), ("f32x", 2, 2, 5)])
def test_slabs_match_undivided_run(lib, precision, nslabs, halo, steps):
    from bgk_pcm_b200.slab import SlabRun
    params = small_params(Nx=150, Ny=61, T_in_sol=271.0)
    ref, sums = undivided(params, steps, precision)
    with SlabRun(params, nslabs=nslabs, halo=halo, precision=precision) as run:
        run.initialization()
        run.step(steps)
        check(run, ref, sums)


def test_slabs_with_row_hot_wall_and_repeated_calls(lib):
    """A per-row Tin (the differentiation form's parameter) lands on the
    right rows of each slab, and step(a) then step(b) equals step(a + b)."""
    from bgk_pcm_b200.slab import SlabRun
    params = small_params(Nx=96, Ny=50, T_in_sol=271.0)
    rng = np.random.default_rng(3)
    tin = params["T0"] + 2.0 * rng.standard_normal(params["Ny"])
    ref, sums = undivided(params, 17, "f64", tin=tin, chunks=[6, 11])
    with SlabRun(params, nslabs=3, halo=3) as run:
        run.initialization(tin)
        run.step(6)
        run.step(11)
        check(run, ref, sums)


def test_rows_pack_unpack_round_trip(lib):
    """Rows packed from one context and unpacked into another at other rows
    carry every plane of the step state: packing them again from the second
    context gives the same bytes, and the populations read back equal."""
    import torch
    from bgk_pcm_b200 import Solver
    params = small_params(Nx=70, Ny=40, T_in_sol=271.0)
    with Solver(params) as a, Solver(params) as b:
        a.initialization(); b.initialization()
        a.step(5)
        n = a.rows_bytes(3)
        buf = torch.zeros(n, dtype=torch.uint8, device="cuda")      # section padding stays 0
        again = torch.zeros(n, dtype=torch.uint8, device="cuda")
        a.rows_pack(10, 3, buf.data_ptr())
        a.sync()
        b.rows_unpack(20, 3, buf.data_ptr())
        b.rows_pack(20, 3, again.data_ptr())
        b.sync()
        assert torch.equal(buf, again)
        for name in [f"f{k}" for k in range(9)] + [f"g{k}" for k in range(9)]:
            np.testing.assert_array_equal(b.field(name)[21:24, 1:-1], a.field(name)[11:14, 1:-1], err_msg=name)


def test_rows_arguments_are_checked(lib):
    import torch
    from bgk_pcm_b200 import BGKError, Solver
    params = small_params(Nx=40, Ny=20)
    with Solver(params) as s:
        s.initialization()
        n = s.rows_bytes(2)
        assert n % 16 == 0
        buf = torch.empty(n + 16, dtype=torch.uint8, device="cuda")
        with pytest.raises(BGKError, match="outside"):
            s.rows_pack(19, 2, buf.data_ptr())
        with pytest.raises(BGKError, match="aligned"):
            s.rows_pack(0, 2, buf.data_ptr() + 8)
        host = torch.empty(n, dtype=torch.uint8)
        with pytest.raises(BGKError, match="device memory|CUDA pointer"):
            s.rows_unpack(0, 2, host.data_ptr())
        with pytest.raises(BGKError, match="outside"):
            s.sums_rows(5, 16)
        np.testing.assert_array_equal(s.sums_rows(0, 20), s.sums())
