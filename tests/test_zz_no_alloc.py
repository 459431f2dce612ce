"""bgk_field_sums_static: the allocation-free interior sums over device fields
the caller owns, checked against bgk_field_sums on a context that holds the
same state.  The file name puts it last in collection, so in a full run it
executes after every other test in the same process; it also passes alone.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import has_gpu, small_params

# The static variant adds in another order than bgk_field_sums; both are FP64.
RTOL = 1e-12


def _ptr(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def test_static_sums_rejects_oversize_and_bad_arguments(lib):
    """Argument checks run before any CUDA call, so this needs no GPU."""
    from bgk_pcm_b200 import capi
    fake = ctypes.c_void_p(4096)
    Ny = capi.STATIC_SUMS_MAX_NY + 1
    assert lib.bgk_field_sums_static(fake, fake, fake, 16, Ny, 18, None, fake) == -1
    msg = lib.bgk_last_error().decode()
    assert "exceeds the static scratch" in msg and str(capi.STATIC_SUMS_MAX_NY) in msg
    assert lib.bgk_field_sums_static(fake, fake, fake, 16, 8, 17, None, fake) == -1
    assert "ld" in lib.bgk_last_error().decode()
    assert lib.bgk_field_sums_static(None, fake, fake, 16, 8, 18, None, fake) == -1
    assert lib.bgk_field_sums_static(fake, fake, fake, 0, 8, 18, None, fake) == -1
    assert lib.bgk_field_sums_static(fake, fake, fake, 16, 8, 18, None, ctypes.c_void_p(4100)) == -1
    assert "aligned" in lib.bgk_last_error().decode()


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a GPU")
def test_static_sums_match_context_sums(lib):
    import torch
    from bgk_pcm_b200 import Solver

    p = small_params(Nx=200, Ny=150, T_in_sol=271.0)
    Nx, Ny = p["Nx"], p["Ny"]
    with Solver(p) as s:
        s.initialization()
        s.step(300)
        ref = s.sums()
        host = {n: s.field(n) for n in ("rho", "T", "phi")}
    dev = {n: torch.from_numpy(a).to("cuda:0") for n, a in host.items()}
    stream = torch.cuda.current_stream("cuda:0")

    # Two calls in a row on one stream, into two result buffers.
    outs = [torch.full((4,), float("nan"), dtype=torch.float64, device="cuda:0") for _ in range(2)]
    for out in outs:
        rc = lib.bgk_field_sums_static(_ptr(dev["rho"]), _ptr(dev["T"]), _ptr(dev["phi"]), Nx, Ny, Nx + 2,
                                       ctypes.c_void_p(stream.cuda_stream), _ptr(out))
        assert rc == 0, lib.bgk_last_error()
    torch.cuda.synchronize()
    got = [o.cpu().numpy() for o in outs]
    for g in got:
        np.testing.assert_allclose(g, ref, rtol=RTOL, atol=0)
        assert g[3] == ref[3]
    assert np.array_equal(got[0], got[1])

    interior = {n: a[1:Ny + 1, 1:Nx + 1] for n, a in host.items()}
    expect = [interior["rho"].sum(), interior["T"].sum(), interior["phi"].sum(),
              float((interior["phi"] > 0).sum())]
    np.testing.assert_allclose(got[0], expect, rtol=RTOL, atol=0)

    # A wider leading dimension: the padding (NaN here) is never read.
    ld = Nx + 2 + 30
    wide = {}
    for n, a in host.items():
        w = np.full((Ny + 2, ld), np.nan)
        w[:, :Nx + 2] = a
        wide[n] = torch.from_numpy(w).to("cuda:0")
    out = torch.full((4,), float("nan"), dtype=torch.float64, device="cuda:0")
    rc = lib.bgk_field_sums_static(_ptr(wide["rho"]), _ptr(wide["T"]), _ptr(wide["phi"]), Nx, Ny, ld,
                                   ctypes.c_void_p(stream.cuda_stream), _ptr(out))
    assert rc == 0, lib.bgk_last_error()
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), got[0])

    # Host memory is refused with an error instead of being read by a kernel.
    cpu = torch.zeros(4, dtype=torch.float64)
    assert lib.bgk_field_sums_static(_ptr(dev["rho"]), _ptr(dev["T"]), _ptr(dev["phi"]), Nx, Ny, Nx + 2,
                                     ctypes.c_void_p(stream.cuda_stream), _ptr(cpu)) == -1


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a GPU")
def test_static_sums_at_the_row_limit_and_into_managed_memory(lib):
    """The largest Ny the scratch holds, on a grid one column wide (ld = 3),
    and a result buffer in managed memory (which the call accepts beside
    device memory), both against numpy sums of the same fields."""
    import torch
    from bgk_pcm_b200 import capi
    from cuda.bindings import runtime as rt

    Nx, Ny = 1, capi.STATIC_SUMS_MAX_NY
    rng = np.random.default_rng(7)
    host = {"rho": 1.0 + 0.01 * rng.standard_normal((Ny + 2, Nx + 2)),
            "T": 263.0 + 20.0 * rng.random((Ny + 2, Nx + 2)),
            "phi": rng.uniform(-1.0, 1.0, (Ny + 2, Nx + 2))}
    dev = {n: torch.from_numpy(a).to("cuda:0") for n, a in host.items()}
    interior = {n: a[1:Ny + 1, 1:Nx + 1] for n, a in host.items()}
    expect = np.array([interior["rho"].sum(), interior["T"].sum(), interior["phi"].sum(),
                       float((interior["phi"] > 0).sum())])
    stream = torch.cuda.current_stream("cuda:0")

    err, mptr = rt.cudaMallocManaged(4 * 8, rt.cudaMemAttachGlobal)
    assert err == rt.cudaError_t.cudaSuccess
    try:
        managed = np.ctypeslib.as_array((ctypes.c_double * 4).from_address(int(mptr)))
        for _ in range(2):
            managed[:] = np.nan
            torch.cuda.synchronize()
            rc = lib.bgk_field_sums_static(_ptr(dev["rho"]), _ptr(dev["T"]), _ptr(dev["phi"]), Nx, Ny, Nx + 2,
                                           ctypes.c_void_p(stream.cuda_stream), ctypes.c_void_p(int(mptr)))
            assert rc == 0, lib.bgk_last_error()
            torch.cuda.synchronize()
            got = managed.copy()
            np.testing.assert_allclose(got, expect, rtol=RTOL, atol=1e-9)
            assert got[3] == expect[3]
    finally:
        rt.cudaFree(mptr)
