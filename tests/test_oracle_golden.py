"""The CPU oracle against golden vectors produced by executing the
reference's own STEP_7 source (tests/golden/make_golden.py): all 46 module
arrays, halos included, bit for bit, after initialization, after the first
step and after the last step of each case.  The heat_* cases run
STEP_DOCONCURRENT's initialization and BC_g with its FROMRIGHT / FROMBOTTOM
macros in place of STEP_7's (params "heat": 1, 2 or both bits)."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem for p in GOLDEN.glob("*.npz"))


def test_fixtures_present():
    assert len(CASES) >= 11


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_reference_source(oracle_mod, case):
    meta = json.loads((GOLDEN / f"{case}.json").read_text())
    data = np.load(GOLDEN / f"{case}.npz")
    o = oracle_mod.Oracle(meta["params"], tanh="libm", heat=meta["params"].get("heat", 0))
    o.initialization()
    done = 0
    for tag in meta["snapshots"]:
        target = 0 if tag == "init" else int(tag[4:])
        o.step(target - done)
        done = target
        for name in oracle_mod.FIELD_NAMES:
            np.testing.assert_array_equal(o.field(name), data[f"{tag}/{name}"], err_msg=f"{case} {tag} {name}")
