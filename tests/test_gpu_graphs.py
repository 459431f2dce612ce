"""Step graphs: on grids of up to 2^21 nodes the plain steps of a bgk_step
call replay a captured CUDA graph of 32 steps.  The graph holds the same
kernels in the same order as the direct launches, so every array must equal
the run with BGK_GRAPH=0 bit for bit -- across calls that start on either
buffer, in every form, on the halo-ring path, and after the operations that
drop the graphs (bgk_set_tin, bgk_load, bgk_initialize)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import small_params

pytestmark = pytest.mark.gpu

FIELDS = ["rho", "T", "u", "v", "phi"] + [f"f{k}" for k in range(9)] + [f"g{k}" for k in range(9)]


def _run(monkeypatch, graph, params, calls, tmp_path=None, tin=None, **kw):
    from bgk_pcm_b200 import Solver
    monkeypatch.setenv("BGK_GRAPH", "1" if graph else "0")
    s = Solver(params, **kw)
    s.initialization()
    for i, n in enumerate(calls):
        if tin is not None and i == 1:
            s.set_tin(tin)
        if tmp_path is not None and i == 2:
            s.save(tmp_path / f"g{int(graph)}.bin")
            s.load(tmp_path / f"g{int(graph)}.bin")
        s.step(n)
    out = {n: s.field(n) for n in FIELDS}
    s.close()
    return out


@pytest.mark.parametrize("precision", ["f64", "f32", "f16", "f32x"])
def test_graph_replays_equal_direct_launches(monkeypatch, lib, precision):
    p = small_params(96, 64)
    calls = [70, 33, 100, 1, 41]          # both start buffers, short and long calls
    kw = dict(precision=precision, tanh="portable" if precision == "f64" else "device")
    a = _run(monkeypatch, False, p, calls, **kw)
    b = _run(monkeypatch, True, p, calls, **kw)
    for n in FIELDS:
        np.testing.assert_array_equal(b[n], a[n], err_msg=f"{precision} {n}")


def test_graph_replays_on_the_halo_ring_with_tin_and_snapshot(monkeypatch, lib, tmp_path):
    """Walls other than code 4 (three boundary launches per step inside the
    graph), a per-row tin set between calls and a snapshot round trip."""
    p = small_params(80, 40, westBC=2, eastBC=0, northBC=4, southBC=6, Re=5.0)
    tin = np.linspace(p["T0"], p["T0"] + 3.0, 40)
    calls = [50, 60, 45]
    a = _run(monkeypatch, False, p, calls, tmp_path=tmp_path, tin=tin, tanh="portable")
    b = _run(monkeypatch, True, p, calls, tmp_path=tmp_path, tin=tin, tanh="portable")
    for n in FIELDS:
        np.testing.assert_array_equal(b[n], a[n], err_msg=n)
