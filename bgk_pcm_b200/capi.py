"""ctypes binding of libbgkpcm (include/bgk_pcm.h).

This module only declares the C ABI; `solver.py` builds the reference-shaped
host interface on top of it.  Loading fails loudly when the shared library is
missing: there is no CPU fallback anywhere in the package.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libbgkpcm.so"

BGK_OK = 0
ERRORS = {
    -1: "BGK_ERR_ARG",
    -2: "BGK_ERR_UNSUPPORTED",
    -3: "BGK_ERR_CUDA",
    -4: "BGK_ERR_OOM",
    -5: "BGK_ERR_STATE",
    -6: "BGK_ERR_IO",
    -7: "BGK_ERR_NONFINITE",
}

PREC_F64, PREC_F32, PREC_F16, PREC_F32X = 0, 1, 2, 3
TANH_PORTABLE, TANH_DEVICE = 0, 1
HEAT_WEST, HEAT_RIGHT, HEAT_BOTTOM = 0, 1, 2

FIELD_F0, FIELD_G0 = 0, 9
FIELD_RHO, FIELD_T, FIELD_U, FIELD_V = 18, 19, 20, 21
FIELD_PHI, FIELD_PHI_PREC = 22, 23
FIELD_RHO2, FIELD_T2, FIELD_U2, FIELD_V2 = 24, 25, 26, 27
FIELD_FP0, FIELD_GP0 = 28, 37
NFIELDS = 46

FIELD_NAMES = (
    [f"f{k}" for k in range(9)] + [f"g{k}" for k in range(9)]
    + ["rho", "T", "u", "v", "phi", "phi_prec", "rho2", "T2", "u2", "v2"]
    + [f"fp{k}" for k in range(9)] + [f"gp{k}" for k in range(9)]
)
FIELD_ID = {n: i for i, n in enumerate(FIELD_NAMES)}

# Every symbol include/bgk_pcm.h declares (checked by the CPU test-suite).
EXPORTS = [
    "bgk_last_error", "bgk_read_input", "bgk_create", "bgk_destroy", "bgk_initialize",
    "bgk_step", "bgk_bc_f", "bgk_bc_g", "bgk_streaming", "bgk_moments_pre",
    "bgk_phase_field", "bgk_forces", "bgk_collision", "bgk_moments", "bgk_upload",
    "bgk_download", "bgk_download_region", "bgk_field_sums", "bgk_get_it", "bgk_set_it",
    "bgk_set_tin", "bgk_sync", "bgk_get_stream", "bgk_save", "bgk_load", "bgk_adjoint_run",
    "bgk_field_sums_static", "bgk_advance", "bgk_rows_bytes", "bgk_rows_pack", "bgk_rows_unpack",
    "bgk_field_sums_rows",
]

STATIC_SUMS_MAX_NY = 32768


class Params(ctypes.Structure):
    """bgk_params: the 21 input.dat values in file order."""

    _fields_ = (
        [(n, ctypes.c_int) for n in ("iter", "noutput", "dump", "Nx", "Ny")]
        + [(n, ctypes.c_double) for n in ("Re", "rho0", "rho1", "tau_f", "tau_g", "T0", "T_in_sol",
                                          "grav", "eps", "stefan_number", "T_width", "length")]
        + [(n, ctypes.c_int) for n in ("westBC", "eastBC", "northBC", "southBC")]
    )

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}

    @classmethod
    def from_dict(cls, d: dict) -> "Params":
        p = cls()
        for n, _ in cls._fields_:
            setattr(p, n, d[n])
        return p


class Options(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("tanh_mode", ctypes.c_int), ("fma", ctypes.c_int),
                ("device", ctypes.c_int), ("smooth", ctypes.c_int), ("heat", ctypes.c_int)]


class AdjointSpec(ctypes.Structure):
    _fields_ = [("nsteps", ctypes.c_int), ("checkpoint_every", ctypes.c_int), ("nprobes", ctypes.c_int),
                ("probe_i", ctypes.POINTER(ctypes.c_int)), ("probe_j", ctypes.POINTER(ctypes.c_int)),
                ("phi_target", ctypes.POINTER(ctypes.c_double))]


class BGKError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None


def load() -> ctypes.CDLL:
    """Load libbgkpcm.so from the package directory (built in-tree)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise OSError(f"{LIB_PATH} is missing: build it with `python -m bgk_pcm_b200.build` "
                      "(there is no CPU fallback)")
    lib = ctypes.CDLL(str(LIB_PATH))
    P = ctypes.c_void_p
    dp = ctypes.POINTER(ctypes.c_double)
    sig = {
        "bgk_last_error": (ctypes.c_char_p, []),
        "bgk_read_input": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(Params)]),
        "bgk_create": (ctypes.c_int, [ctypes.POINTER(Params), ctypes.POINTER(Options), ctypes.POINTER(P)]),
        "bgk_destroy": (ctypes.c_int, [P]),
        "bgk_initialize": (ctypes.c_int, [P]),
        "bgk_step": (ctypes.c_int, [P, ctypes.c_int]),
        "bgk_upload": (ctypes.c_int, [P, ctypes.c_int, dp, ctypes.c_int]),
        "bgk_download": (ctypes.c_int, [P, ctypes.c_int, dp, ctypes.c_int]),
        "bgk_download_region": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_int, dp, ctypes.c_int]),
        "bgk_field_sums": (ctypes.c_int, [P, dp]),
        "bgk_get_it": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_int)]),
        "bgk_set_it": (ctypes.c_int, [P, ctypes.c_int]),
        "bgk_set_tin": (ctypes.c_int, [P, dp, ctypes.c_int]),
        "bgk_sync": (ctypes.c_int, [P]),
        "bgk_get_stream": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_void_p)]),
        "bgk_save": (ctypes.c_int, [P, ctypes.c_char_p]),
        "bgk_load": (ctypes.c_int, [P, ctypes.c_char_p]),
        "bgk_adjoint_run": (ctypes.c_int, [P, ctypes.POINTER(AdjointSpec), dp, dp, dp]),
        "bgk_field_sums_static": (ctypes.c_int, [P, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P]),
        "bgk_advance": (ctypes.c_int, [P, ctypes.c_int]),
        "bgk_rows_bytes": (ctypes.c_int, [P, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]),
        "bgk_rows_pack": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_int, P]),
        "bgk_rows_unpack": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_int, P]),
        "bgk_field_sums_rows": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_int, dp]),
    }
    for n in ("bgk_bc_f", "bgk_bc_g", "bgk_streaming", "bgk_moments_pre", "bgk_phase_field",
              "bgk_forces", "bgk_collision", "bgk_moments"):
        sig[n] = (ctypes.c_int, [P])
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != BGK_OK:
        msg = load().bgk_last_error().decode(errors="replace")
        raise BGKError(rc, msg)


def read_input(path: str | os.PathLike) -> Params:
    p = Params()
    check(load().bgk_read_input(str(path).encode(), ctypes.byref(p)))
    return p
