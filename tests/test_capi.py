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


def test_options_struct_and_heat_checks_without_gpu(lib):
    """bgk_options carries the heat bits after the five earlier fields, and
    bgk_create checks them before it looks for a device: bits outside
    BGK_HEAT_RIGHT | BGK_HEAT_BOTTOM are BGK_ERR_ARG, FROMRIGHT with a
    reduced-precision form is BGK_ERR_UNSUPPORTED."""
    from bgk_pcm_b200 import capi
    from bgk_pcm_b200.solver import heat_bits
    from conftest import small_params
    assert ctypes.sizeof(capi.Options) == 6 * 4
    assert capi.Options.heat.offset == 20
    hdr = (ROOT / "include" / "bgk_pcm.h").read_text()
    for name, val in (("BGK_HEAT_WEST", 0), ("BGK_HEAT_RIGHT", 1), ("BGK_HEAT_BOTTOM", 2)):
        assert re.search(rf"#define {name}\s+{val}\b", hdr), name
    assert [heat_bits(h) for h in ("west", "right", "bottom", "right+bottom", 3)] == [0, 1, 2, 3, 3]
    with pytest.raises(ValueError):
        heat_bits("left")
    p = capi.Params.from_dict(small_params())
    h = ctypes.c_void_p()
    bad = capi.Options(capi.PREC_F64, capi.TANH_PORTABLE, 0, -1, 0, 4)
    assert lib.bgk_create(ctypes.byref(p), ctypes.byref(bad), ctypes.byref(h)) == -1
    assert "heat" in lib.bgk_last_error().decode()
    f32_right = capi.Options(capi.PREC_F32, capi.TANH_DEVICE, 0, -1, 0, capi.HEAT_RIGHT)
    assert lib.bgk_create(ctypes.byref(p), ctypes.byref(f32_right), ctypes.byref(h)) == -2
    assert "FP64" in lib.bgk_last_error().decode()
    assert not h.value
