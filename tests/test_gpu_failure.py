"""Failure detection of the step kernels, without a GPU fault.

Every wait inside the pipeline kernels is bounded (about a second): an
mbarrier wait for a stage, and in the multi-step dataflow launch the wait
for a tile's neighbourhood to finish the previous step.  When one runs out,
the kernel records a code in the context's error flag and every CTA leaves;
bgk_sync reports BGK_ERR_CUDA with the code, and the process and the GPU
carry on.  Here the dataflow launch's dependency waits are made to run out
on purpose: BGK_FLOW_STALL=1 raises every dependency target beyond any count
a tile reaches (a flag that nothing sets), so the first item of the second
step waits until its limit.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import small_params

pytestmark = pytest.mark.gpu


def test_expired_dependency_wait_is_reported_and_the_gpu_carries_on(lib, monkeypatch):
    from bgk_pcm_b200 import BGKError, Solver
    p = small_params(300, 200)
    monkeypatch.setenv("BGK_FLOW", "1")
    monkeypatch.setenv("BGK_FLOW_STALL", "1")
    with Solver(p) as s:
        s.initialization()
        s.step(6)                      # four dataflow steps, then two with moments
        with pytest.raises(BGKError, match="BGK_ERR_CUDA.*bounded wait"):
            s.sync()
        s.sync()                       # the flag was cleared by the report
    monkeypatch.setenv("BGK_FLOW_STALL", "0")
    out = []
    for flow in ("1", "0"):
        monkeypatch.setenv("BGK_FLOW", flow)
        with Solver(p) as s:
            s.initialization()
            s.step(6)
            s.sync()
            out.append(s.field("T"))
    np.testing.assert_array_equal(out[0], out[1])
