"""input.dat files: reader/writer and the mapping of the benchmark workloads.

The reference reads 21 list-directed "label value" records
(STEP_7/setup.f90:7-31).  The benchmark workloads are described in physical
terms (Rayleigh, Prandtl and Stefan numbers, a Mach-0.1 velocity scale); the
reference takes lattice parameters instead, so each workload is mapped onto
an input.dat as follows (the reference's own semantics are kept):

* T0 = 283 (hot wall, Tin = T0), T_in_sol = 263, so the hard-coded
  T_crit = 273 (STEP_7/phase_field.f90:12) sits at theta_m = 0.5; T_width 10.
* rho0 = 1 (solid), rho1 = 1/1.024 (liquid): rho0/rho1 - 1 = 0.024, the
  density contrast of the reference's UTIL/input.dat.* files.
* Pr = 1 gives tau_f = tau_g = tau.  With U = 0.1*cs = 0.1/sqrt(3):
  grav = U^2 / (Ny (rho0/rho1 - 1)), kvisc = U Ny sqrt(Pr/Ra),
  tau = 3 kvisc + 1/2, so that diag's Ray = grav (rho0/rho1-1) Ny^3 / kvisc^2
  * Pr (STEP_7/diag.f90:31-40) equals Ra.
* Re = 0, eps = 0, length = Ny, no-slip (code 4) on all walls, noutput = 2.
"""
from __future__ import annotations

import math
from pathlib import Path

LABELS = ["iter", "noutput", "dump", "Nx", "Ny", "Re", "rho0", "rho1", "tau_f", "tau_g", "T0",
          "T_in_sol", "grav", "eps", "stefan_number", "T_width", "length", "westBC_st",
          "eastBC_st", "northBC_st", "southBC_st"]
KEYS = ["iter", "noutput", "dump", "Nx", "Ny", "Re", "rho0", "rho1", "tau_f", "tau_g", "T0",
        "T_in_sol", "grav", "eps", "stefan_number", "T_width", "length", "westBC", "eastBC",
        "northBC", "southBC"]
INT_KEYS = {"iter", "noutput", "dump", "Nx", "Ny", "westBC", "eastBC", "northBC", "southBC"}

# The five benchmark workloads: (name, Nx, Ny, iter, Ra, Pr, Stefan, form)
WORKLOADS = {
    "cavity256_ra1e5": dict(Nx=256, Ny=256, iter=20000, Ra=1e5, Pr=1.0, Ste=1.0, form="f64"),
    "cavity2048_ra1e6": dict(Nx=2048, Ny=2048, iter=10000, Ra=1e6, Pr=1.0, Ste=1.0, form="f64"),
    "cavity4096_ra1e7": dict(Nx=4096, Ny=4096, iter=20000, Ra=1e7, Pr=1.0, Ste=1.0, form="f32"),
    "cavity512_ra1e5_adjoint": dict(Nx=512, Ny=512, iter=2000, Ra=1e5, Pr=1.0, Ste=1.0, form="f64"),
    "cavity16384x4096_ra1e8": dict(Nx=16384, Ny=4096, iter=50000, Ra=1e8, Pr=1.0, Ste=0.5, form="f32"),
}


def fortran_real(x: float) -> str:
    """repr() of a double with a Fortran d exponent (read back exactly)."""
    r = repr(float(x))
    if "e" in r:
        m, e = r.split("e")
        return f"{m}d{int(e)}"
    return r + "d0"


def read(path) -> dict:
    vals = {}
    lines = Path(path).read_text().splitlines()
    it = iter(lines)
    for key in KEYS:
        tok = next(it).replace(",", " ").split()
        if len(tok) < 2:
            raise ValueError(f"{path}: record for {key} is malformed")
        v = tok[1]
        vals[key] = int(v) if key in INT_KEYS else float(v.replace("d", "e").replace("D", "e"))
    return vals


def write(path, vals: dict) -> None:
    out = []
    for label, key in zip(LABELS, KEYS):
        v = vals[key]
        s = str(int(v)) if key in INT_KEYS else fortran_real(v)
        out.append(f"  {label:<18s} {s}")
    Path(path).write_text("\n".join(out) + "\n")


def workload_params(Nx: int, Ny: int, iter: int, Ra: float, Pr: float = 1.0, Ste: float = 1.0,
                    noutput: int = 2, **_) -> dict:
    """input.dat values for a cavity of Nx x Ny at the given Ra, Pr, Ste."""
    rho0, rho1 = 1.0, 1.0 / 1.024
    contrast = rho0 / rho1 - 1.0
    U = 0.1 / math.sqrt(3.0)
    grav = U * U / (Ny * contrast)
    kvisc = U * Ny * math.sqrt(Pr / Ra)
    tau_f = 3.0 * kvisc + 0.5
    alpha = kvisc / Pr
    tau_g = 3.0 * alpha + 0.5
    return dict(iter=iter, noutput=noutput, dump=0, Nx=Nx, Ny=Ny, Re=0.0, rho0=rho0, rho1=rho1,
                tau_f=tau_f, tau_g=tau_g, T0=283.0, T_in_sol=263.0, grav=grav, eps=0.0,
                stefan_number=Ste, T_width=10.0, length=float(Ny), westBC=4, eastBC=4, northBC=4,
                southBC=4)


def diag_numbers(vals: dict) -> dict:
    """Gr, Pr, Ra as the reference's diag computes them (STEP_7/diag.f90:31-40),
    with the integer Ny**3 evaluated in 64 bits (no wrap)."""
    cs2 = 1.0 / 3.0
    kvisc = cs2 * (vals["tau_f"] - 0.5)
    dT = vals["T0"] - vals["T_in_sol"]
    beta = (vals["rho0"] / vals["rho1"] - 1.0) / dT
    gras = vals["grav"] * beta * dT * vals["Ny"] ** 3 / kvisc ** 2
    pr = (2.0 * vals["tau_f"] - 1.0) / (2.0 * vals["tau_g"] - 1.0)
    return dict(Gr=gras, Pr=pr, Ra=pr * gras)


def write_all(root=None) -> list:
    root = Path(root) if root else Path(__file__).resolve().parent / "inputs"
    made = []
    for name, w in WORKLOADS.items():
        d = root / name
        d.mkdir(parents=True, exist_ok=True)
        write(d / "input.dat", workload_params(**w))
        made.append(d / "input.dat")
    return made


if __name__ == "__main__":
    for p in write_all():
        print(p)
