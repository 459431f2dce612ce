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
