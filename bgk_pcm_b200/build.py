"""Build recipe for libbgkpcm.so (sm_100a) and the bgk_thermal host driver.

Everything is compiled in-tree with nvcc for `-gencode arch=compute_100a,
code=sm_100a`.  Translation units that must reproduce the reference's
floating-point roundings are compiled with ``--fmad=false`` (no contracted
multiply-add, like gfortran -O3 on generic x86-64) and their host code with
``-ffp-contract=off``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libbgkpcm.so"
HOST = PKG / "bgk_thermal"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
          "-I", str(ROOT / "include")]
UNITS = {
    "kernels_f64.cu": ["--fmad=false"],
    "kernels_fast.cu": ["--fmad=true"],
    "capi.cu": ["--fmad=false"],
    "adjoint.cu": ["--fmad=true"],
    "static_sums.cu": ["--fmad=false"],
}


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found")
    return cand


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"command failed: {' '.join(cmd[:3])} ...")
    return r.stdout + r.stderr


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    objs = []
    for unit, flags in UNITS.items():
        src = CSRC / unit
        obj = BUILD / (unit + ".o")
        objs.append(obj)
        if force or _stale(obj, [src, *headers, Path(__file__)]):
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            out = _run([nvcc(), *ARCH, *COMMON, *flags, *extra, "-c", str(src), "-o", str(obj)], verbose)
            if ptxas_info:
                print(out)
    if force or _stale(LIB, objs):
        _run([nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs)], verbose)
    host_src = CSRC / "host" / "bgk_thermal.cpp"
    if host_src.exists() and (force or _stale(HOST, [host_src, LIB, *headers])):
        _run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", str(ROOT / "include"), str(host_src),
              "-o", str(HOST), "-L", str(PKG), "-lbgkpcm", f"-Wl,-rpath,$ORIGIN", "-lm"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv)
