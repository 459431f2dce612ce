"""The combined workload's pipeline (reduced-precision forward, FP64 adjoint
over the last steps from that state, FP64 finite differences) on a small
rectangular cavity, with the binomial checkpoint schedule forced (three state
slots), so the path the 16384 x 4096 run takes is exercised end to end."""
from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu


def test_combined_pipeline_small_binomial(lib):
    from bgk_pcm_b200 import combined
    r = combined.run(nx=256, ny=64, Ra=1e4, Ste=0.5, steps=1500, adj_steps=300, ndir=3, nprobes=16,
                     checkpoint_every=-3, h=1e-6)
    print(r)
    assert r["forward"]["glups"] > 0
    assert r["adjoint"]["loss"] > 0
    for d in r["fd"][0]["directions"]:
        assert d["rel_err"] <= 1e-5 or abs(d["fd"] - d["adjoint"]) <= 1e-12, r["fd"]


def test_combined_pipeline_at_full_grid_size(lib):
    """The combined workload's grid itself -- 16384 x 4096 (aspect 4), Ra 1e8,
    Stefan 0.5 -- with shortened runs: the FP32 forward for 2000 steps, then
    the FP64 adjoint over the last 100 steps with the binomial schedule over
    four state slots (one FP64 state is 10.2 GB), checked against FP64
    central differences along two random directions (h = 1e-4 of the
    dimensionless hot-wall temperature and of tau_g).  The full run (50,000
    steps, adjoint over 5,000, eight directions) is `python -m
    bgk_pcm_b200.combined`."""
    import psutil
    from bgk_pcm_b200 import combined
    if psutil.virtual_memory().available < 40e9:
        pytest.skip("needs ~40 GB of host memory for the saved state")
    r = combined.run(nx=16384, ny=4096, Ra=1e8, Ste=0.5, steps=2000, adj_steps=100, ndir=2, nprobes=64,
                     checkpoint_every=-4, h=1e-4)
    print({k: r[k] for k in ("forward", "adjoint")}, r["fd"])
    assert r["forward"]["glups"] > 20.0
    assert r["adjoint"]["loss"] > 0
    for d in r["fd"][0]["directions"]:
        assert d["rel_err"] <= 1e-5, r["fd"]
