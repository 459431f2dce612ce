#!/usr/bin/env python
"""Benchmark of the fused BGK_PCM time step on B200.

One "step" is one time step of the cavity workload (every node of the grid
advances f, g and phi once, STEP_7/main.f90:60-69).  Default workload: the
2048x2048 cavity at Ra=1e6, FP64 (cavity2048_ra1e6), i.e. the configuration
the headline metric is quoted on; its populations (604 MB) are larger than
L2, so consecutive steps never hit a warm cache.

  value     GLUPS = Nx*Ny*steps / device time / 1e9, summed over ranks
  e2e       the same metric through the public C ABI with host buffers: the
            initial state uploaded from pinned host memory, the steps with the
            reference's diagnostic cadence (sums + probe every 1000 steps), and
            the final fields downloaded, all inside the timed region
  roofline  algorithmic bytes per launch of the fused kernel / its average
            duration, against the measured HBM copy bandwidth
  cpu_baseline  the CPU oracle (C restatement of STEP_7, OpenMP over all host
            threads) on a bounded number of steps of the same workload

`--impl reference` times that CPU implementation alone as the reference arm.
Multi-GPU (torchrun, N ranks): the y-slab decomposition (bgk_pcm_b200.slab).
The cavity grows to N x Ny rows (weak scaling: every rank owns the Ny rows
of the workload plus ghost rows), and the ranks exchange their cut rows
over NCCL every --halo steps.  `--decomp replicas` runs N independent
replicas instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "GLUPS & HBM GB/s: FP32-store vs FP64 at ≤1e-4 err; adjoint/forward cost"
# algorithmic bytes per node and step: 18 populations + phi, read once and
# written once (FP64; FP32 and FP16 deviations with phi in FP32; FP32
# deviations with FP64 arithmetic and phi in FP64)
BYTES_PER_NODE = {"f64": 304, "f32": 152, "f16": 80, "f32x": 160}
FALLBACK_HBM = 6650.0


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    REASONS = {
        0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap",
        0x8: "hw_slowdown", 0x10: "sync_boost", 0x20: "sw_thermal_slowdown",
        0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting",
    }

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 4:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
                bits = int(parts[3], 16) if parts[3].startswith("0x") else int(parts[3])
            except ValueError:
                continue
            for b, n in self.REASONS.items():
                if bits & b:
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def host_cpu() -> dict:
    """The host's CPU model, the logical CPUs this process may run on, and
    the physical cores among them (distinct (package, core) pairs of
    /proc/cpuinfo; SMT siblings share a core)."""
    try:
        allowed = os.sched_getaffinity(0)
    except (AttributeError, OSError):
        allowed = set(range(os.cpu_count() or 1))
    model, cores = None, set()
    try:
        blocks = Path("/proc/cpuinfo").read_text().split("\n\n")
    except OSError:
        blocks = []
    for block in blocks:
        d = {}
        for ln in block.splitlines():
            if ":" in ln:
                k, v = ln.split(":", 1)
                d[k.strip()] = v.strip()
        if "processor" not in d:
            continue
        model = model or d.get("model name")
        p = int(d["processor"])
        if p in allowed:
            cores.add((d.get("physical id", "0"), d.get("core id", str(p))))
    return {"model": model, "logical_cpus": len(allowed), "physical_cores": len(cores) or len(allowed)}


def cpu_oracle_rate(params, budget_s: float = 15.0, max_steps: int = 400, threads: int = 0, warmup: int = 2,
                    tanh: str = "device"):
    """GLUPS of the CPU oracle on whole steps of `params`, with `threads`
    OpenMP threads (0: one per physical core, where the thread sweep of the
    oracle peaks; 1: the serial STEP_7 restatement).  `warmup` untimed steps
    (at least 2) also size the timed sample.  tanh: "portable" (the same
    function as the GPU's portable form) or the host libm's."""
    from oracle import pyoracle
    threads = threads or host_cpu()["physical_cores"]
    o = pyoracle.Oracle(params, threads=threads, tanh="portable" if tanh == "portable" else "libm")
    o.initialization()
    w = max(2, warmup)
    t0 = time.perf_counter()
    o.step(w)
    dt = (time.perf_counter() - t0) / w
    n = int(max(2, min(max_steps, budget_s / max(dt, 1e-9))))
    t0 = time.perf_counter()
    o.step(n)
    t = time.perf_counter() - t0
    o.close()
    glups = params["Nx"] * params["Ny"] * n / t / 1e9
    return glups, n, threads


def load_traffic(kernel_key: str):
    """Per-launch DRAM bytes of a kernel from the committed ncu summary."""
    f = ROOT / "profiles" / "ncu_traffic.json"
    if not f.exists():
        return None
    d = json.loads(f.read_text())
    return d.get(kernel_key, {}).get("traffic_bytes_per_launch")


def max_over_ranks(value: float, dist, device) -> float:
    """The maximum of `value` over all ranks (the job's time is its slowest
    rank's); `dist` is None for a single process."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_glups(nodes: int, steps: int, world: int, ms_max: float) -> float:
    """Node updates of all ranks (each runs its own replica) per second."""
    return nodes * steps * world / (ms_max / 1e3) / 1e9


def time_steps(solver, steps: int, torch):
    stream = torch.cuda.ExternalStream(solver.stream)
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    solver.step(steps)
    end.record(stream)
    end.synchronize()
    return start.elapsed_time(end)


def e2e_run(params, precision, steps, device, torch, tanh="portable"):
    """Public-API run with host buffers: upload, steps + diag cadence, download."""
    import numpy as np

    from bgk_pcm_b200 import Solver
    Nx, Ny = params["Nx"], params["Ny"]
    shape = (Ny + 2, Nx + 2)
    # the fields a step reads: the populations, phi, T (its column Nx is the
    # lagged east wall) and u, v (their halos feed BC_g); rho is recomputed
    # from the populations before anything reads it
    names = [f"f{k}" for k in range(9)] + [f"g{k}" for k in range(9)] + ["T", "u", "v", "phi"]
    src = Solver(params, precision=precision, device=device, tanh=tanh)
    src.initialization()
    host_in = {}
    for n in names:
        t = torch.empty(shape, dtype=torch.float64, pin_memory=True)
        a = t.numpy()
        a[:] = src.field(n)
        host_in[n] = (t, a)
    src.close()
    outs = {n: torch.empty(shape, dtype=torch.float64, pin_memory=True) for n in ("rho", "T", "u", "v", "phi")}
    s = Solver(params, precision=precision, device=device, tanh=tanh)
    stream = torch.cuda.ExternalStream(s.stream)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    h2d = 0
    for n in names:
        s.upload(n, host_in[n][1])
        h2d += host_in[n][1].nbytes
    d2h = 0
    done = 0
    while done < steps:
        chunk = min(1000, steps - done)
        s.step(chunk)
        done += chunk
        sums = s.sums()
        probe = s.region("T", Nx // 2, Ny // 2, 1, 1)
        d2h += sums.nbytes + probe.nbytes
    for n, t in outs.items():
        a = s.field(n, out=t.numpy())
        d2h += a.nbytes
    ev1.record(stream)
    ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    s.close()
    return ms, h2d, d2h


def slab_timed(params, precision, steps, warmup, halo, torch, dist, sampler=None, tanh="portable"):
    """The y-slab run of this rank (DistTransport over NCCL): device time of
    `steps` steps on the rank's context stream, which also orders the halo
    exchanges, with clock samples when a sampler is given."""
    from bgk_pcm_b200.slab import DistTransport, SlabRun
    run = SlabRun(params, halo=halo, precision=precision, transport=DistTransport(), tanh=tanh)
    run.initialization()
    run.sync()
    clocks = None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    # warm-up right before the timed steps (no idle gap between them)
    run.step(warmup)
    run.sync()
    stream = torch.cuda.ExternalStream(run.slabs[0].solver.stream)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    dist.barrier()
    torch.cuda.synchronize()
    ev0.record(stream)
    run.step(steps)
    ev1.record(stream)
    ev1.synchronize()
    if sampler:
        clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1)
    dist.barrier()
    run.close()
    return ms, clocks


def e2e_slab(params, precision, steps, halo, torch, dist, tanh="portable"):
    """The end-to-end run of this rank's slab: the initial fields a step
    reads (as in e2e_run) uploaded from pinned host memory, the steps with the diagnostic cadence (sums
    all-reduced, the probe read back every 1000 steps), and its
    rho/T/u/v/phi downloaded (the slab's whole reference-layout fields)."""
    from bgk_pcm_b200.slab import DistTransport, SlabRun
    names = [f"f{k}" for k in range(9)] + [f"g{k}" for k in range(9)] + ["T", "u", "v", "phi"]
    run = SlabRun(params, halo=halo, precision=precision, transport=DistTransport(), tanh=tanh)
    s = run.slabs[0].solver
    s.initialization()
    host_in = {}
    for n in names:
        t = torch.empty(s.field(n).shape, dtype=torch.float64, pin_memory=True)
        t.numpy()[:] = s.field(n)
        host_in[n] = t
    stream = torch.cuda.ExternalStream(s.stream)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    dist.barrier()
    torch.cuda.synchronize()
    ev0.record(stream)
    h2d = d2h = 0
    for n in names:
        s.upload(n, host_in[n].numpy())
        h2d += host_in[n].numpy().nbytes
    done = 0
    while done < steps:
        chunk = min(1000, steps - done)
        run.step(chunk)
        done += chunk
        sums = run.sums()
        probe = s.region("T", params["Nx"] // 2, 1, 1, 1)
        d2h += sums.nbytes + probe.nbytes
    for n in ("rho", "T", "u", "v", "phi"):
        d2h += run.slabs[0].local_field(n).nbytes      # the slab's whole field crosses
    ev1.record(stream)
    ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    dist.barrier()
    run.close()
    return ms, h2d, d2h


def precision_errors(params, device) -> dict:
    """Errors of the FP32 form against FP64 after the workload's full run
    (params["iter"] steps), per field (max and RMS, normalised as the target
    is stated: T by T0 - T_in_sol, phi by its range 2, u and v by max |u| of
    the FP64 run) and for the melt front (x shift of phi's zero crossing, at
    row Ny/2 and the largest over the rows).
    * `errors`: against FP64 in double throughout (the smooth form), the
      baseline whose own rounding is far below the FP32 form's;
    * `errors_vs_bit_exact`: against the bit-exact FP64 path (the
      reference's REAL(4) collision temporaries, portable tanh);
    * `fp64_spread`: the bit-exact path against the smooth one, i.e. how far
      the reference's own roundings move its FP64 result on this case."""
    from bgk_pcm_b200 import precision as pr
    steps = params["iter"]
    t0 = time.perf_counter()
    smooth = pr.run(params, "f64", steps, smooth=True, tanh="portable")
    ref = pr.run(params, "f64", steps, tanh="portable")
    lo = pr.run(params, "f32", steps)
    e = pr.errors(lo, smooth, params)
    keys = ("T_max", "phi_max", "u_max", "v_max", "front_dx_max_cells")
    ebit = pr.errors(lo, ref, params)
    spread = pr.errors(ref, smooth, params)
    e.update({"steps": steps, "vs": "f64 in double (smooth form)",
              "within_1e-4": bool(e["T_max"] <= 1e-4 and e["phi_max"] <= 1e-4),
              "errors_vs_bit_exact": {k: ebit[k] for k in keys},
              "fp64_spread": {k: spread[k] for k in keys},
              "seconds": time.perf_counter() - t0})
    return e


def fp64_divergence(params, device, tanh_a, tanh_b, fma_b, steps=200) -> float:
    """Largest |difference| over rho, T, u, v, phi (halos included) between
    the headline FP64 form (tanh_a, exact operation order) and a variant
    (tanh_b, fma_b) after the same `steps` steps of the workload.  0 means
    bit-identical; the headline form with the portable tanh is bit-identical
    to the oracle (the parity tests)."""
    import numpy as np

    from bgk_pcm_b200 import Solver
    out = []
    for tanh, fma in ((tanh_a, False), (tanh_b, fma_b)):
        with Solver(params, precision="f64", tanh=tanh, fma=fma, device=device) as s:
            s.initialization()
            s.step(steps)
            out.append({n: s.field(n) for n in ("rho", "T", "u", "v", "phi")})
    return {"steps": steps, "max_abs": max(float(np.abs(out[0][n] - out[1][n]).max()) for n in out[0])}


def adjoint_cost(torch, repeats=3):
    """Cost of one adjoint gradient against one forward solve on the
    differentiation workload (512^2, Ra 1e5, 2000 steps, 64 probes,
    checkpoints every 45 steps).  Both timed on an existing context (wall
    clock around synchronised calls, best of `repeats`); the adjoint's
    workspace stays in the context after a first, untimed call."""
    from bgk_pcm_b200 import gradcheck as gc
    p, tin, tin_t, pi, pj = gc.setup()
    steps, K = p["iter"], 45
    target = gc.forward_phi(p, tin_t, steps, pi, pj)
    ratio, tf, ta = gc.cost_ratio(p, tin, steps, pi, pj, target, K, repeats)
    return {"workload": "cavity512_ra1e5_adjoint", "steps": steps, "checkpoint_every": K,
            "forward_ms": tf * 1e3, "adjoint_ms": ta * 1e3, "ratio": ratio,
            "timing": "wall clock, synchronised, best of %d, on an existing context" % repeats}


def bench_config(args, params, wl) -> dict:
    """The workload, identical in both arms' lines."""
    esz = {"f64": 8, "f32": 4, "f16": 2, "f32x": 4}[args.precision]
    nodes = params["Nx"] * params["Ny"]
    return {"workload": args.workload, "Nx": params["Nx"], "Ny": params["Ny"], "Ra": wl["Ra"], "Pr": wl["Pr"],
            "Ste": wl["Ste"], "precision": args.precision, "tanh": args.tanh,
            "l2": "inputs larger than L2 (A/B populations %.0f MB > 126 MB), no flush" % (2 * 18 * esz * nodes / 1e6)}


def run_reference(args, params, wl):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = max(2, args.warmup)
    cpu = host_cpu()
    glups, n, threads = cpu_oracle_rate(params, budget_s=min(60.0, 5.0 + 0.5 * args.steps), max_steps=args.steps,
                                        warmup=w, tanh=args.tanh)
    line = {
        "impl": "reference", "metric": METRIC, "value": glups, "unit": "GLUPS", "n_gpus": args.gpus,
        "steps": n, "warmup": w, "ms_per_step": params["Nx"] * params["Ny"] / glups / 1e6,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (the reference's initial condition on the generated input.dat)",
        "config": bench_config(args, params, wl),
        "cpu_baseline": {"value": glups, "unit": "GLUPS", "cores": threads, "kind": "port",
                         "threads": threads, "physical_cores": cpu["physical_cores"],
                         "logical_cpus": cpu["logical_cpus"], "cpu_model": cpu["model"],
                         "sample": f"{n} whole steps of the {params['Nx']}x{params['Ny']} grid; C restatement of "
                                   "STEP_7 (OpenMP over the j loops, one thread per physical core, bit-identical "
                                   "to serial); the Fortran reference cannot be compiled in this image"},
        "e2e": {"value": glups, "unit": "GLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10000)
    ap.add_argument("--warmup", type=int, default=100)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cavity2048_ra1e6")
    ap.add_argument("--precision", default="f64", choices=["f64", "f32", "f16", "f32x"])
    ap.add_argument("--tanh", default="portable", choices=["portable", "device"],
                    help="phase-field tanh: the portable one (bit-identical to the oracle) or CUDA's")
    ap.add_argument("--forms", default="headline,f64device,f64fma,f32,f32x",
                    help="forms timed over one common window beside the headline (comma list; "
                         "'headline' is the headline form itself; f16 also exists)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint/forward cost leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg")
    ap.add_argument("--precision-errors", type=int, default=1,
                    help="1: run the precision workload in full (FP64 and FP32) and report the FP32 form's errors")
    ap.add_argument("--sustained", type=int, default=10000,
                    help="steps of one more run of the headline form, timed with its clocks (the power-capped "
                         "sustained rate; 0 skips it)")
    ap.add_argument("--decomp", default="slab", choices=["slab", "replicas"],
                    help="N > 1: y-slab decomposition of one N-times taller cavity, or N replicas")
    ap.add_argument("--halo", type=int, default=8, help="ghost rows per cut (steps between exchanges)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    from bgk_pcm_b200 import inputs
    wl = inputs.WORKLOADS[args.workload]
    params = inputs.workload_params(**wl)

    if args.impl == "reference":
        run_reference(args, params, wl)
        return

    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    from bgk_pcm_b200 import Solver, build
    # one rank brings the in-tree library up to date; the others wait for it
    if rank == 0:
        build.build()
    if dist:
        dist.barrier()

    Nx, Ny = params["Nx"], params["Ny"]
    nodes = Nx * Ny

    def barrier():
        if dist:
            dist.barrier()

    def run_form(precision, fma, steps, warmup, sample_clocks=False, tanh=args.tanh):
        s = Solver(params, precision=precision, fma=fma, device=local, tanh=tanh)
        s.initialization()
        s.sync()
        clocks = None
        sampler = ClockSampler(local) if sample_clocks else None
        if sampler:
            sampler.start()
            time.sleep(0.3)
        # the warm-up runs right before the timed steps, so the GPU does not
        # sit idle (while the clock sampler starts) between the two
        s.step(warmup)
        s.sync()
        barrier()
        torch.cuda.synchronize()
        ms = time_steps(s, steps, torch)
        torch.cuda.synchronize()
        if sampler:
            clocks = sampler.stop()
        barrier()
        s.close()
        return ms, clocks

    slab = world > 1 and args.decomp == "slab"
    gparams = dict(params, Ny=Ny * world) if slab else params
    if slab:
        ms, clocks = slab_timed(gparams, args.precision, args.steps, args.warmup, args.halo, torch, dist,
                                ClockSampler(local), tanh=args.tanh)
    else:
        ms, clocks = run_form(args.precision, False, args.steps, args.warmup, sample_clocks=True)
    ms = max_over_ranks(ms, dist, "cuda")
    value = whole_job_glups(nodes, args.steps, world, ms)
    hbm, hbm_kind = peaks()
    bpn = BYTES_PER_NODE[args.precision]
    achieved = bpn * nodes / (ms / 1e3 / args.steps) / 1e9
    kernel_key = f"fused_{args.precision}_{args.workload}"
    traffic = load_traffic(kernel_key)

    forms = {}
    # extra forms on a single process only: a form that fails on one rank
    # must not leave the ranks at different collective steps
    # name -> (precision, FMA contraction, tanh); the reduced-precision forms
    # are not bit-exact with anything, so they use CUDA's tanh(f)
    form_spec = {"headline": (args.precision, False, args.tanh if args.precision == "f64" else "device"),
                 "f64device": ("f64", False, "device"), "f64fma": ("f64", True, args.tanh),
                 "f32": ("f32", False, "device"), "f16": ("f16", False, "device"),
                 "f32x": ("f32x", False, "device")}
    form_steps = max(args.steps // 4, 100)
    # every form, the headline form included, is timed over the same number
    # of steps, so that the ratios compare like with like (a window of a few
    # steps carries the two moment-writing steps of a call at a larger share)
    form_names = [f for f in args.forms.split(",") if f and f != "none" and world == 1]
    if form_names and "headline" not in form_names:
        form_names.insert(0, "headline")
    for form in form_names:
        if form not in form_spec:
            forms[form] = {"error": "unknown form"}
            continue
        prec, fma, tanh = form_spec[form]
        try:
            fms, _ = run_form(prec, fma, form_steps, args.warmup, tanh=tanh)
        except Exception as exc:  # a form that is not available is reported, not fatal
            forms[form] = {"error": str(exc)}
            continue
        g = nodes * form_steps / (fms / 1e3) / 1e9
        b = BYTES_PER_NODE[prec]
        forms[form] = {"glups": g, "hbm_gbs": g * b, "frac_of_measured_hbm": g * b / hbm, "bytes_per_node": b,
                       "steps": form_steps, "tanh": tanh, "fma": fma}
        if "glups" in forms.get("headline", {}):
            forms[form]["speedup_vs_headline_form"] = g / forms["headline"]["glups"]
        if prec == "f64" and args.precision == "f64" and form != "headline":
            forms[form]["max_abs_vs_headline"] = fp64_divergence(params, local, args.tanh, tanh, fma)

    # the precision-form workload (4096^2, Ra 1e7): FP32 storage against FP64
    # the same form over a long run: a 20-step window runs at the burst
    # clocks, a run of seconds at the clocks the 1000 W power cap leaves
    sustained = None
    if world == 1 and args.sustained and args.sustained > args.steps:
        sms, sclk = run_form(args.precision, False, args.sustained, args.warmup, sample_clocks=True)
        sg = nodes * args.sustained / (sms / 1e3) / 1e9
        sustained = {"steps": args.sustained, "glups": sg, "hbm_gbs": sg * bpn, "frac_of_measured_hbm": sg * bpn / hbm,
                     "clocks": sclk}

    precision_cfg = None
    if world == 1 and "f32" in args.forms.split(",") and args.precision == "f64":
        pwl = "cavity4096_ra1e7"
        pparams = inputs.workload_params(**inputs.WORKLOADS[pwl])
        pn = pparams["Nx"] * pparams["Ny"]
        rates = {}
        for prec in ("f64", "f32"):
            s = Solver(pparams, precision=prec, device=local)
            s.initialization()
            s.step(args.warmup)
            s.sync()
            k = 400
            pms = time_steps(s, k, torch)
            s.close()
            rates[prec] = pn * k / (pms / 1e3) / 1e9
        precision_cfg = {"workload": pwl, "steps": 400, "f64_glups": rates["f64"], "f32_glups": rates["f32"],
                         "f32_over_f64": rates["f32"] / rates["f64"],
                         "f32_hbm_gbs": rates["f32"] * BYTES_PER_NODE["f32"],
                         "f32_frac_of_measured_hbm": rates["f32"] * BYTES_PER_NODE["f32"] / hbm}
        if args.precision_errors:
            precision_cfg["errors"] = precision_errors(pparams, local)

    adjoint = None
    if rank == 0 and world == 1 and not args.no_adjoint:
        adjoint = adjoint_cost(torch)

    e2e = None
    if not args.no_e2e:
        if slab:
            e_ms, h2d, d2h = e2e_slab(gparams, args.precision, args.steps, args.halo, torch, dist, tanh=args.tanh)
        else:
            e_ms, h2d, d2h = e2e_run(params, args.precision, args.steps, local, torch, tanh=args.tanh)
        e_ms = max_over_ranks(e_ms, dist, "cuda")
        e2e = {"value": whole_job_glups(nodes, args.steps, world, e_ms), "unit": "GLUPS",
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
               "what": "initial state (the 22 reference-layout fields a step reads: f, g, T, u, v, phi) uploaded "
                       "from pinned host memory, the steps with field sums + probe read back every 1000 steps, final "
                       "rho/T/u/v/phi downloaded"}

    cpu = cpu1 = None
    if rank == 0 and world == 1 and not args.no_cpu:
        hc = host_cpu()
        glups, n, threads = cpu_oracle_rate(params, tanh=args.tanh)
        cpu = {"value": glups, "unit": "GLUPS", "cores": threads, "kind": "port", "threads": threads,
               "physical_cores": hc["physical_cores"], "logical_cpus": hc["logical_cpus"], "cpu_model": hc["model"],
               "sample": f"{n} whole steps of the {Nx}x{Ny} grid, C restatement of STEP_7 with OpenMP "
                         "(STEP_OPENMP's parallelisation, one thread per physical core; bit-identical to serial)"}
        glups1, n1, _ = cpu_oracle_rate(params, budget_s=8.0, threads=1, tanh=args.tanh)
        cpu1 = {"value": glups1, "unit": "GLUPS", "cores": 1, "kind": "port",
                "sample": f"{n1} whole steps of the {Nx}x{Ny} grid, serial C restatement of STEP_7"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "GLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": args.precision,
            "data": "synthetic (the reference's initial condition on the generated input.dat)",
            "config": bench_config(args, params, wl),
            "layout": {"parallelism": (f"yslab{world}" if slab else
                                       (f"replicas{world}" if world > 1 else "single-gpu")),
                       "global_Ny": Ny * world if slab else Ny,
                       "halo_rows": args.halo if slab else None},
            "hbm_gbs": value / world * bpn,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": traffic, "peak_kind": hbm_kind,
                         "bytes_per_node": bpn},
            "forms": forms,
            "sustained": sustained,
            "precision_config": precision_cfg,
            "adjoint": adjoint,
            "clocks": clocks,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "cpu_baseline_serial": cpu1,
            # the fused steps (in FP64 the step before the last also writes
            # the lagged halo cells; the reduced-precision forms run one
            # halo pass before the last step); with slabs, rank 0 (one cut)
            # also packs and unpacks its rows once per exchange
            "gpu_launches": args.steps + (0 if args.precision == "f64" else 1)
                            + (2 * -(-args.steps // args.halo) if slab else 0),
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
