"""Host-side mirror of the reference's interface over the C ABI.

The reference (STEP_7/) is a Fortran program whose step is a sequence of
argument-less subroutines on module state (STEP_7/main.f90:60-69).  `Solver`
holds one device context and exposes the same names -- ``setup`` (the
constructor), ``initialization``, ``BC_f``, ``BC_g``, ``streaming``,
``momentsPre``, ``phase_field``, ``forces``, ``collision``, ``moments`` --
plus ``step(n)``, the fused equivalent of n passes of that sequence.

Fields are numpy arrays of shape (Ny+2, Nx+2) indexed [j, i], i.e. the
reference's (0:Nx+1, 0:Ny+1) column-major arrays seen from C order.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from . import capi

_PREC = {"f64": capi.PREC_F64, "f32": capi.PREC_F32, "f16": capi.PREC_F16, "f32x": capi.PREC_F32X}
_TANH = {"device": capi.TANH_DEVICE, "portable": capi.TANH_PORTABLE}


def heat_bits(heat) -> int:
    """The heated wall: "west" (STEP_7), "right" (STEP_DOCONCURRENT's
    FROMRIGHT), "bottom" (FROMBOTTOM), "right+bottom" (both macros), or the
    BGK_HEAT_* bits as an int."""
    if isinstance(heat, int):
        return heat
    bits = {"west": capi.HEAT_WEST, "right": capi.HEAT_RIGHT, "bottom": capi.HEAT_BOTTOM}
    try:
        return sum(bits[h] for h in str(heat).split("+"))
    except KeyError:
        raise ValueError(f"heat must be west, right, bottom or right+bottom, not {heat!r}") from None


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Solver:
    """One simulation on one B200 (STEP_7/setup.f90 allocates, this creates).

    precision: "f64" (the reference's), "f32", "f16" or "f32x" deviation
    storage; tanh: "portable" (bit-identical to the CPU oracle) or "device";
    fma: multiply-add contraction in FP64; smooth: the REAL(4) collision
    temporaries kept in double (the form the adjoint differentiates); heat:
    the heated wall (see heat_bits)."""

    def __init__(self, params, precision: str = "f64", tanh: str = "portable", fma: bool = False,
                 device: int = -1, smooth: bool = False, heat="west"):
        lib = capi.load()
        if isinstance(params, dict):
            params = capi.Params.from_dict(params)
        self.params = params
        self.Nx, self.Ny = params.Nx, params.Ny
        self.precision = precision
        self.heat = heat_bits(heat)
        opt = capi.Options(_PREC[precision], _TANH[tanh], 1 if fma else 0, device, 1 if smooth else 0, self.heat)
        h = ctypes.c_void_p()
        capi.check(lib.bgk_create(ctypes.byref(params), ctypes.byref(opt), ctypes.byref(h)))
        self._h = h
        self._lib = lib

    # -- life cycle -------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.bgk_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- the reference's subroutines ----------------------------------------
    def initialization(self) -> None:
        capi.check(self._lib.bgk_initialize(self._h))

    def step(self, n: int = 1) -> None:
        capi.check(self._lib.bgk_step(self._h, int(n)))

    def BC_f(self) -> None:
        capi.check(self._lib.bgk_bc_f(self._h))

    def BC_g(self) -> None:
        capi.check(self._lib.bgk_bc_g(self._h))

    def streaming(self) -> None:
        capi.check(self._lib.bgk_streaming(self._h))

    def momentsPre(self) -> None:
        capi.check(self._lib.bgk_moments_pre(self._h))

    def phase_field(self) -> None:
        capi.check(self._lib.bgk_phase_field(self._h))

    def forces(self) -> None:
        capi.check(self._lib.bgk_forces(self._h))

    def collision(self) -> None:
        capi.check(self._lib.bgk_collision(self._h))

    def moments(self) -> None:
        capi.check(self._lib.bgk_moments(self._h))

    STAGES = ("BC_f", "BC_g", "streaming", "momentsPre", "phase_field", "forces", "collision", "moments")

    def staged_step(self) -> None:
        for name in self.STAGES:
            getattr(self, name)()

    # -- data -----------------------------------------------------------------
    @staticmethod
    def field_id(name) -> int:
        return name if isinstance(name, int) else capi.FIELD_ID[name]

    def field(self, name, out: np.ndarray | None = None) -> np.ndarray:
        """Download one field; `out` (C-contiguous float64, shape (Ny+2, Nx+2))
        receives it directly, e.g. a pinned host buffer."""
        if out is None:
            out = np.empty((self.Ny + 2, self.Nx + 2), dtype=np.float64)
        elif out.shape != (self.Ny + 2, self.Nx + 2) or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 array of shape (Ny+2, Nx+2)")
        capi.check(self._lib.bgk_download(self._h, self.field_id(name), _dptr(out), self.Nx + 2))
        return out

    def upload(self, name, arr: np.ndarray) -> None:
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if a.shape != (self.Ny + 2, self.Nx + 2):
            raise ValueError(f"expected shape {(self.Ny + 2, self.Nx + 2)}, got {a.shape}")
        capi.check(self._lib.bgk_upload(self._h, self.field_id(name), _dptr(a), self.Nx + 2))

    def region(self, name, i0: int, j0: int, ni: int, nj: int) -> np.ndarray:
        out = np.empty((nj, ni), dtype=np.float64)
        capi.check(self._lib.bgk_download_region(self._h, self.field_id(name), i0, j0, ni, nj,
                                                 _dptr(out), ni))
        return out

    def sums(self) -> np.ndarray:
        out = np.empty(4, dtype=np.float64)
        capi.check(self._lib.bgk_field_sums(self._h, _dptr(out)))
        return out

    @property
    def it(self) -> int:
        v = ctypes.c_int()
        capi.check(self._lib.bgk_get_it(self._h, ctypes.byref(v)))
        return v.value

    @it.setter
    def it(self, value: int) -> None:
        capi.check(self._lib.bgk_set_it(self._h, int(value)))

    def set_tin(self, tin) -> None:
        if tin is None:
            capi.check(self._lib.bgk_set_tin(self._h, None, 0))
            return
        a = np.ascontiguousarray(tin, dtype=np.float64)
        capi.check(self._lib.bgk_set_tin(self._h, _dptr(a), a.size))

    def sync(self) -> None:
        capi.check(self._lib.bgk_sync(self._h))

    # -- y-slab decomposition (bgk_pcm_b200.slab) ---------------------------
    def advance(self, n: int) -> None:
        """n fused steps without writing the reference-layout fields."""
        capi.check(self._lib.bgk_advance(self._h, int(n)))

    def rows_bytes(self, nrows: int) -> int:
        v = ctypes.c_size_t()
        capi.check(self._lib.bgk_rows_bytes(self._h, int(nrows), ctypes.byref(v)))
        return v.value

    def rows_pack(self, j0: int, nrows: int, dev_ptr: int) -> None:
        """Pack interior rows j0.. (0-based) into device memory at dev_ptr."""
        capi.check(self._lib.bgk_rows_pack(self._h, int(j0), int(nrows), ctypes.c_void_p(dev_ptr)))

    def rows_unpack(self, j0: int, nrows: int, dev_ptr: int) -> None:
        capi.check(self._lib.bgk_rows_unpack(self._h, int(j0), int(nrows), ctypes.c_void_p(dev_ptr)))

    def sums_rows(self, j0: int, nrows: int) -> np.ndarray:
        out = np.empty(4, dtype=np.float64)
        capi.check(self._lib.bgk_field_sums_rows(self._h, int(j0), int(nrows), _dptr(out)))
        return out

    @property
    def stream(self) -> int:
        """The context's cudaStream_t as an integer handle."""
        v = ctypes.c_void_p()
        capi.check(self._lib.bgk_get_stream(self._h, ctypes.byref(v)))
        return v.value or 0

    def adjoint(self, nsteps: int, probe_i, probe_j, phi_target, checkpoint_every: int = 0):
        """Loss sum_p (phi(i_p,j_p) - target_p)^2 after nsteps steps from the
        current state, with dL/dTin (per row, length Ny) and dL/dtau_g.
        Requires a context created with smooth=True."""
        pi = np.ascontiguousarray(probe_i, dtype=np.int32)
        pj = np.ascontiguousarray(probe_j, dtype=np.int32)
        tg = np.ascontiguousarray(phi_target, dtype=np.float64)
        if not (pi.size == pj.size == tg.size):
            raise ValueError("probe_i, probe_j and phi_target must have the same length")
        spec = capi.AdjointSpec(int(nsteps), int(checkpoint_every), int(pi.size),
                                pi.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                pj.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dptr(tg))
        loss = ctypes.c_double()
        gtau = ctypes.c_double()
        gtin = np.zeros(self.Ny, dtype=np.float64)
        capi.check(self._lib.bgk_adjoint_run(self._h, ctypes.byref(spec), ctypes.byref(loss), _dptr(gtin),
                                             ctypes.byref(gtau)))
        return loss.value, gtin, gtau.value

    def save(self, path) -> None:
        capi.check(self._lib.bgk_save(self._h, str(Path(path)).encode()))

    def load(self, path) -> None:
        capi.check(self._lib.bgk_load(self._h, str(Path(path)).encode()))
