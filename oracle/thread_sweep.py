"""CPU baseline sweeps of the oracle, after the reference's UTIL scripts.
TEST INFRASTRUCTURE: times the C restatement of STEP_7 / STEP_OPENMP.

  threads  UTIL/RunMe_thread.sh:2-9 runs bgk_thermal with OMP_NUM_THREADS =
           64, 32, ..., 1, greps Mlups and md5sums the outputs; here the
           oracle runs the same steps from the same initial state at each
           thread count, prints MLUPS, and the md5 of rho/T/u/v/phi must be
           the same at every count (the time loop has no reductions).
  sizes    UTIL/RunMe_size.sh:2-7 runs each input deck in turn; here each
           generated workload deck, a bounded number of steps with all
           threads.

    python -m oracle.thread_sweep threads --workload cavity256_ra1e5 --steps 200
    python -m oracle.thread_sweep sizes --budget 10
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

from oracle import pyoracle  # noqa: E402

FIELDS = ("rho", "T", "u", "v", "phi")


def _run(params: dict, steps: int, threads: int):
    o = pyoracle.Oracle(params, threads=threads)
    o.initialization()
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    h = hashlib.md5()
    for n in FIELDS:
        h.update(o.field(n).tobytes())
    o.close()
    return params["Nx"] * params["Ny"] * steps / dt / 1e6, h.hexdigest()


def thread_counts(max_threads: int):
    t, out = 1, []
    while t < max_threads:
        out.append(t)
        t *= 2
    out.append(max_threads)
    return sorted(set(out), reverse=True)


def threads_sweep(params: dict, steps: int, max_threads: int) -> list:
    rows = []
    for th in thread_counts(max_threads):
        mlups, md5 = _run(params, steps, th)
        rows.append({"threads": th, "steps": steps, "mlups": mlups, "md5": md5})
    return rows


def sizes_sweep(workloads, budget_s: float, threads: int) -> list:
    from bgk_pcm_b200 import inputs
    rows = []
    for wl in workloads:
        params = inputs.workload_params(**inputs.WORKLOADS[wl])
        o = pyoracle.Oracle(params, threads=threads)
        o.initialization()
        t0 = time.perf_counter()
        o.step(1)
        per = time.perf_counter() - t0
        o.close()
        steps = int(max(2, min(params["iter"], budget_s / max(per, 1e-9))))
        mlups, _ = _run(params, steps, threads)
        rows.append({"workload": wl, "Nx": params["Nx"], "Ny": params["Ny"], "threads": threads, "steps": steps,
                     "mlups": mlups})
    return rows


def main(argv=None):
    from bgk_pcm_b200 import inputs
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["threads", "sizes"])
    ap.add_argument("--workload", default="cavity256_ra1e5")
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--threads", type=int, default=0, help="largest thread count (0: all host threads)")
    ap.add_argument("--budget", type=float, default=10.0, help="seconds per workload (sizes)")
    a = ap.parse_args(argv)
    th = a.threads or os.cpu_count() or 1
    if a.what == "threads":
        params = inputs.workload_params(**inputs.WORKLOADS[a.workload])
        rows = threads_sweep(params, a.steps, th)
        for r in rows:
            print(json.dumps(dict(workload=a.workload, **r)), flush=True)
        if len({r["md5"] for r in rows}) != 1:
            print("thread_sweep: results differ between thread counts", file=sys.stderr)
            return 1
    else:
        for r in sizes_sweep(list(inputs.WORKLOADS), a.budget, th):
            print(json.dumps(r), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
