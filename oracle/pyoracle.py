"""ctypes binding of the CPU oracle (liborc.so).  TEST INFRASTRUCTURE ONLY:
used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
the checker; the product never imports it."""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liborc.so"
MAIN = HERE / "_build" / "orc_main"

FIELD_NAMES = (
    [f"f{k}" for k in range(9)] + [f"g{k}" for k in range(9)]
    + ["rho", "T", "u", "v", "phi", "phi_prec", "rho2", "T2", "u2", "v2"]
    + [f"fp{k}" for k in range(9)] + [f"gp{k}" for k in range(9)]
)
FIELD_ID = {n: i for i, n in enumerate(FIELD_NAMES)}


class OrcParams(ctypes.Structure):
    _fields_ = (
        [(n, ctypes.c_int) for n in ("iter", "noutput", "dump", "Nx", "Ny")]
        + [(n, ctypes.c_double) for n in ("Re", "rho0", "rho1", "tau_f", "tau_g", "T0", "T_in_sol",
                                          "grav", "eps", "stefan_number", "T_width", "length")]
        + [(n, ctypes.c_int) for n in ("westBC", "eastBC", "northBC", "southBC")]
    )


def build() -> Path:
    """Compile liborc.so / orc_main with the oracle's Makefile (gcc)."""
    r = subprocess.run(["make", "-s", "-C", str(HERE)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return LIB


_lib = None


def load() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        build()
    lib = ctypes.CDLL(str(LIB))
    vp = ctypes.c_void_p
    lib.orc_create.restype = vp
    lib.orc_create.argtypes = [ctypes.POINTER(OrcParams)]
    lib.orc_field.restype = ctypes.POINTER(ctypes.c_double)
    lib.orc_field.argtypes = [vp, ctypes.c_int]
    for n in ("orc_destroy", "orc_initialization", "orc_bc_f", "orc_bc_g", "orc_streaming",
              "orc_moments_pre", "orc_phase_field", "orc_forces", "orc_collision", "orc_moments",
              "orc_diag", "orc_probe", "orc_prof_x", "orc_prof_y", "orc_field_check", "orc_out2d",
              "orc_close_outputs"):
        getattr(lib, n).argtypes = [vp]
        getattr(lib, n).restype = None
    lib.orc_step.argtypes = [vp, ctypes.c_int]
    lib.orc_set_tanh_mode.argtypes = [vp, ctypes.c_int]
    lib.orc_set_smooth.argtypes = [vp, ctypes.c_int]
    lib.orc_set_heat.argtypes = [vp, ctypes.c_int]
    lib.orc_set_threads.argtypes = [ctypes.c_int]
    lib.orc_get_it.argtypes = [vp]
    lib.orc_set_it.argtypes = [vp, ctypes.c_int]
    lib.orc_sums.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
    lib.orc_open_outputs.argtypes = [vp, ctypes.c_char_p]
    lib.orc_read_input.argtypes = [ctypes.c_char_p, ctypes.POINTER(OrcParams)]
    lib.orc_main.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.orc_portable_tanh.restype = ctypes.c_double
    lib.orc_portable_tanh.argtypes = [ctypes.c_double]
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    lib.orc_tangent_loss.argtypes = [ctypes.POINTER(OrcParams), dp, dp, ctypes.c_double, ctypes.c_int,
                                     ctypes.c_int, ip, ip, dp, dp, dp, dp]
    lib.orc_tangent_plain.argtypes = [ctypes.POINTER(OrcParams), dp, ctypes.c_int, dp, dp]
    _lib = lib
    return lib


def read_input(path) -> dict:
    p = OrcParams()
    rc = load().orc_read_input(str(path).encode(), ctypes.byref(p))
    if rc:
        raise ValueError(f"oracle could not parse {path} ({rc})")
    return {n: getattr(p, n) for n, _ in OrcParams._fields_}


class Oracle:
    """The reference's STEP_7 program state, stepped on the CPU."""

    STAGES = ("bc_f", "bc_g", "streaming", "moments_pre", "phase_field", "forces", "collision", "moments")

    def __init__(self, params: dict, tanh: str = "libm", threads: int = 0, smooth: bool = False, heat: int = 0):
        self.lib = load()
        p = OrcParams()
        for n, _ in OrcParams._fields_:
            setattr(p, n, params[n])
        self.Nx, self.Ny = p.Nx, p.Ny
        if threads:
            self.lib.orc_set_threads(threads)
        self.h = self.lib.orc_create(ctypes.byref(p))
        if not self.h:
            raise ValueError("orc_create failed")
        self.lib.orc_set_tanh_mode(self.h, 1 if tanh == "portable" else 0)
        self.lib.orc_set_smooth(self.h, 1 if smooth else 0)
        # STEP_DOCONCURRENT's heating options: 1 FROMRIGHT, 2 FROMBOTTOM, 3 both
        self.lib.orc_set_heat(self.h, int(heat))

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def initialization(self):
        self.lib.orc_initialization(self.h)

    def stage(self, name: str):
        getattr(self.lib, "orc_" + name)(self.h)

    def step(self, n: int = 1):
        self.lib.orc_step(self.h, int(n))

    @property
    def it(self) -> int:
        return self.lib.orc_get_it(self.h)

    def field(self, name) -> np.ndarray:
        k = name if isinstance(name, int) else FIELD_ID[name]
        ptr = self.lib.orc_field(self.h, k)
        a = np.ctypeslib.as_array(ptr, shape=((self.Ny + 2) * (self.Nx + 2),))
        return a.reshape(self.Ny + 2, self.Nx + 2).copy()

    def set_field(self, name, arr: np.ndarray):
        k = name if isinstance(name, int) else FIELD_ID[name]
        ptr = self.lib.orc_field(self.h, k)
        a = np.ctypeslib.as_array(ptr, shape=((self.Ny + 2) * (self.Nx + 2),))
        a[:] = np.ascontiguousarray(arr, dtype=np.float64).ravel()

    def sums(self) -> np.ndarray:
        out = (ctypes.c_double * 4)()
        self.lib.orc_sums(self.h, out)
        return np.array(out[:])


def portable_tanh(x: float) -> float:
    return load().orc_portable_tanh(float(x))


def run_main(workdir, threads: int = 0, tanh_mode: int = 0, heat: int = 0) -> None:
    """Run the STEP_7 program (orc_main) in workdir (must hold input.dat)."""
    if not MAIN.exists():
        build()
    r = subprocess.run([str(MAIN), str(workdir), str(threads), str(tanh_mode), str(heat)], capture_output=True,
                       text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stderr)


def _params(d: dict) -> OrcParams:
    p = OrcParams()
    for n, _ in OrcParams._fields_:
        setattr(p, n, d[n])
    return p


def tangent_loss(params: dict, tin, dtin, dtau_g: float, nsteps: int, pi, pj, target):
    """Loss and its directional derivative along (dtin, dtau_g), by forward
    mode (dual numbers) through the reference's step (smooth form)."""
    dpt = ctypes.POINTER(ctypes.c_double)
    tin = np.ascontiguousarray(tin, dtype=np.float64)
    dtin = np.ascontiguousarray(dtin, dtype=np.float64)
    pi = np.ascontiguousarray(pi, dtype=np.int32)
    pj = np.ascontiguousarray(pj, dtype=np.int32)
    target = np.ascontiguousarray(target, dtype=np.float64)
    loss = ctypes.c_double()
    dloss = ctypes.c_double()
    rc = load().orc_tangent_loss(ctypes.byref(_params(params)), tin.ctypes.data_as(dpt), dtin.ctypes.data_as(dpt),
                                 float(dtau_g), int(nsteps), int(pi.size),
                                 pi.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                 pj.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), target.ctypes.data_as(dpt),
                                 ctypes.byref(loss), ctypes.byref(dloss), None)
    if rc:
        raise ValueError("tangent oracle supports the no-slip cavity with Re = 0 only")
    return loss.value, dloss.value


def tangent_plain(params: dict, tin, nsteps: int):
    """phi and T after nsteps of the templated restatement in plain double."""
    dpt = ctypes.POINTER(ctypes.c_double)
    tin = np.ascontiguousarray(tin, dtype=np.float64)
    shape = (params["Ny"] + 2, params["Nx"] + 2)
    phi = np.empty(shape)
    T = np.empty(shape)
    load().orc_tangent_plain(ctypes.byref(_params(params)), tin.ctypes.data_as(dpt), int(nsteps),
                             phi.ctypes.data_as(dpt), T.ctypes.data_as(dpt))
    return phi, T
