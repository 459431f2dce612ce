"""The C-ABI library loads and exports every symbol include/bgk_pcm.h declares
(no compute calls: this runs without a GPU)."""
from __future__ import annotations

import ctypes
import re
import subprocess

import pytest

from conftest import ROOT, has_gpu


def declared_symbols():
    text = (ROOT / "include" / "bgk_pcm.h").read_text()
    return sorted(set(re.findall(r"\b(bgk_[a-z_0-9]+)\s*\(", text)))


def test_header_symbols_exported(lib):
    from bgk_pcm_b200 import capi
    names = declared_symbols()
    assert set(names) == set(capi.EXPORTS)
    nm = subprocess.run(["nm", "-D", "--defined-only", str(capi.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (bgk_\w+)", nm))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    for n in names:
        assert getattr(lib, n) is not None


def test_params_struct_layout(lib):
    from bgk_pcm_b200 import capi
    # 5 ints, padding to 8, 12 doubles, 4 ints
    assert ctypes.sizeof(capi.Params) == 5 * 4 + 4 + 12 * 8 + 4 * 4
    assert capi.Params.Re.offset == 24


@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU failure mode")
def test_create_fails_loudly_without_gpu(lib):
    from bgk_pcm_b200 import BGKError, Solver
    from conftest import small_params
    with pytest.raises(BGKError, match="BGK_ERR_CUDA.*no CPU path"):
        Solver(small_params())


def test_slab_entry_points_reject_null_arguments(lib):
    """The y-slab entry points check their arguments before any CUDA call."""
    size = ctypes.c_size_t()
    out = (ctypes.c_double * 4)()
    fake = ctypes.c_void_p(4096)
    assert lib.bgk_advance(None, 3) == -1
    assert lib.bgk_rows_bytes(None, 2, ctypes.byref(size)) == -1
    assert lib.bgk_rows_pack(None, 0, 2, fake) == -1
    assert lib.bgk_rows_unpack(None, 0, 2, fake) == -1
    assert lib.bgk_field_sums_rows(None, 0, 2, out) == -1
    assert "null" in lib.bgk_last_error().decode()
