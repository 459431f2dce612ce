"""y-slab decomposition of the fused step.

The interior rows 0..Ny-1 of one cavity are split into contiguous slabs, one
context per slab.  Slab r owns rows [lo_r, hi_r); its context also holds
``halo`` ghost rows below it (r > 0) and above it (r < nslabs - 1), copies of
the neighbours' rows.  The fused step treats a context's first and last rows
as the N/S walls (STEP_7/BC_f.f90, BC_g.f90), so a ghost row's own update is
wrong, and the error moves one row inward per step (the pull stencil of
STEP_7/streaming.f90:5-27 and the 3x3 phase-field stencil of
STEP_7/phase_field.f90:27-38 reach one row).  A slab therefore takes ``halo``
steps, then replaces its ghost rows by its neighbours' current rows: every
owned row is bit-identical to the undivided run, for every precision form,
because the node arithmetic does not depend on the decomposition.

Per exchange each cut moves ``halo`` rows each way: 18 populations, phi and
the east T column per row: 152 bytes per column and row in FP64, 76 in FP32.

Transports:
  * LocalTransport -- all slabs in this process (one GPU, or several GPUs
    of one process); device-to-device through the packed row buffers.
  * DistTransport  -- one slab per rank of torch.distributed: NCCL
    point-to-point over NVLink between GPUs, gloo between CPU processes.

A slab is any object with the methods of ``SolverSlab`` (the GPU slab over
the C ABI); the transports and ``SlabRun`` only move packed rows between
them.

    run = SlabRun(params, nslabs=4, halo=4)          # one process, one GPU
    run.initialization(); run.step(1000); phi = run.field("phi")
"""
from __future__ import annotations

import contextlib

import numpy as np

from .solver import Solver


class SlabPlan:
    """Rows of each slab: owned [lo, hi), ghost rows below and above."""

    def __init__(self, Ny: int, nslabs: int, halo: int):
        if nslabs < 1:
            raise ValueError("nslabs must be >= 1")
        if halo < 1:
            raise ValueError("halo must be >= 1")
        self.Ny, self.nslabs, self.halo = int(Ny), int(nslabs), int(halo)
        self.bounds = [(self.Ny * r) // self.nslabs for r in range(self.nslabs + 1)]
        for r in range(self.nslabs):
            if self.nslabs > 1 and self.own(r) < self.halo:
                raise ValueError(f"slab {r} owns {self.own(r)} rows, fewer than the {self.halo} ghost rows "
                                 "it must send")

    def lo(self, r: int) -> int:
        return self.bounds[r]

    def hi(self, r: int) -> int:
        return self.bounds[r + 1]

    def own(self, r: int) -> int:
        return self.hi(r) - self.lo(r)

    def below(self, r: int) -> int:
        return self.halo if r > 0 else 0

    def above(self, r: int) -> int:
        return self.halo if r < self.nslabs - 1 else 0

    def local_ny(self, r: int) -> int:
        return self.own(r) + self.below(r) + self.above(r)

    def first_row(self, r: int) -> int:
        """Global row of the context's local row 0."""
        return self.lo(r) - self.below(r)

    def chunks(self, nsteps: int):
        """(steps, final) per chunk between exchanges; `final` chunks run
        through bgk_step so that the last two steps of the call write the
        reference-layout fields (moments and the lagged halos)."""
        done = 0
        while done < nsteps:
            h = min(self.halo, nsteps - done)
            yield h, (nsteps - done - h) < 2
            done += h


class SolverSlab:
    """One slab on a GPU: a context of local_ny rows plus its packed row buffers."""

    def __init__(self, plan: SlabPlan, r: int, params: dict, precision: str = "f64", device: int = -1,
                 **solver_kw):
        import torch
        self.plan, self.r = plan, r
        q = dict(params)
        q["Ny"] = plan.local_ny(r)
        q.setdefault("length", params["Ny"])       # u0 = Re*kvisc/length keeps the global length
        self.solver = Solver(q, precision=precision, device=device, **solver_kw)
        dev = torch.device("cuda", device if device >= 0 else torch.cuda.current_device())
        n = self.solver.rows_bytes(plan.halo)
        self.buf = {k: torch.empty(n, dtype=torch.uint8, device=dev) for k in ("send_lo", "send_hi", "recv_lo", "recv_hi")}
        self.device = dev

    # -- stepping
    def initialization(self, tin=None) -> None:
        self.solver.initialization()
        if tin is not None:
            a = np.asarray(tin, dtype=np.float64)
            f0 = self.plan.first_row(self.r)
            self.solver.set_tin(a[f0:f0 + self.plan.local_ny(self.r)])

    def run(self, nsteps: int, final: bool) -> None:
        if final:
            self.solver.step(nsteps)
        else:
            self.solver.advance(nsteps)

    # -- rows
    def pack(self, side: str):
        """Own rows next to the cut below ('lo') or above ('hi') into the send buffer."""
        p, r = self.plan, self.r
        j0 = p.below(r) if side == "lo" else p.below(r) + p.own(r) - p.halo
        b = self.buf["send_" + side]
        self.solver.rows_pack(j0, p.halo, b.data_ptr())
        return b

    def recv_buffer(self, side: str):
        return self.buf["recv_" + side]

    def unpack(self, side: str) -> None:
        """The receive buffer into the ghost rows below ('lo') or above ('hi')."""
        p, r = self.plan, self.r
        j0 = 0 if side == "lo" else p.below(r) + p.own(r)
        self.solver.rows_unpack(j0, p.halo, self.buf["recv_" + side].data_ptr())

    def stream_context(self):
        import torch
        return torch.cuda.stream(torch.cuda.ExternalStream(self.solver.stream, device=self.device))

    def sync(self) -> None:
        self.solver.sync()

    # -- results
    def own_sums(self) -> np.ndarray:
        return self.solver.sums_rows(self.plan.below(self.r), self.plan.own(self.r))

    def local_field(self, name: str) -> np.ndarray:
        return self.solver.field(name)

    def close(self) -> None:
        self.solver.close()


class LocalTransport:
    """All slabs in this process.  Packs on each slab's stream, waits for the
    packs, copies each send buffer into the neighbour's receive buffer (a
    device-to-device copy, peer-to-peer when the slabs sit on different
    GPUs), waits for the copies, unpacks."""

    def exchange(self, slabs) -> None:
        n = len(slabs)
        sent = [dict() for _ in range(n)]
        for r in range(n):
            if r > 0:
                sent[r]["lo"] = slabs[r].pack("lo")
            if r < n - 1:
                sent[r]["hi"] = slabs[r].pack("hi")
        for s in slabs:
            s.sync()
        moved = []
        for r in range(n - 1):
            slabs[r + 1].recv_buffer("lo").copy_(sent[r]["hi"])
            slabs[r].recv_buffer("hi").copy_(sent[r + 1]["lo"])
            moved += [slabs[r + 1].recv_buffer("lo"), slabs[r].recv_buffer("hi")]
        _wait_copies(moved)
        for r in range(n):
            if r > 0:
                slabs[r].unpack("lo")
            if r < n - 1:
                slabs[r].unpack("hi")


def _wait_copies(tensors) -> None:
    """Tensor copies run on torch's current stream of each device."""
    devs = {t.device for t in tensors if t.device.type == "cuda"}
    if devs:
        import torch
        for d in devs:
            torch.cuda.current_stream(d).synchronize()


class DistTransport:
    """One slab per rank of torch.distributed.  Each cut is one send and one
    receive each way, posted together (batch_isend_irecv) so that NCCL pairs
    them without ordering deadlocks.  With a GPU slab the operations are
    issued on the context's stream, so they follow the packs and precede the
    unpacks on the device without host synchronisation."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def peer(self, r: int) -> int:
        """Global rank of the group's rank r (the slab index)."""
        return r if self.group is None else self.dist.get_global_rank(self.group, r)

    def exchange(self, slabs) -> None:
        (s,) = slabs
        dist, r, n = self.dist, self.rank, self.world
        ctx = s.stream_context() if hasattr(s, "stream_context") else contextlib.nullcontext()
        with ctx:
            ops = []
            if r > 0:
                ops.append(dist.P2POp(dist.isend, s.pack("lo"), self.peer(r - 1), self.group))
                ops.append(dist.P2POp(dist.irecv, s.recv_buffer("lo"), self.peer(r - 1), self.group))
            if r < n - 1:
                ops.append(dist.P2POp(dist.isend, s.pack("hi"), self.peer(r + 1), self.group))
                ops.append(dist.P2POp(dist.irecv, s.recv_buffer("hi"), self.peer(r + 1), self.group))
            if ops:
                for w in dist.batch_isend_irecv(ops):
                    w.wait()
            if r > 0:
                s.unpack("lo")
            if r < n - 1:
                s.unpack("hi")


class SlabRun:
    """A cavity stepped as y-slabs.  With a LocalTransport it owns every
    slab; with a DistTransport it owns the slab of this rank."""

    def __init__(self, params: dict, nslabs: int | None = None, halo: int = 4, precision: str = "f64",
                 transport=None, slab_factory=None, devices=None, **solver_kw):
        self.params = dict(params)
        walls = [self.params.get(k, 4) for k in ("westBC", "eastBC", "northBC", "southBC")]
        if any(int(w) != 4 for w in walls):
            # the fused step (bgk_step, bgk_advance) implements only the
            # no-slip code 4, and a cut is only a wall of code 4 seen from a
            # slab: an inflow or pressure code would be built from the slab's
            # own rows (STEP_7/BC_f.f90:7-60) and be wrong on every slab
            raise ValueError(f"SlabRun needs the no-slip code 4 on every wall, got W/E/N/S = {walls}")
        if solver_kw.get("heat", "west") not in ("west", 0):
            # the heating options place the initial liquid layer and the hot
            # wall by global rows and columns; a slab would place them by its own
            raise ValueError("SlabRun implements the heated west wall only (heat='west')")
        self.transport = transport or LocalTransport()
        dist_mode = isinstance(self.transport, DistTransport)
        if dist_mode:
            nslabs = self.transport.world
        self.plan = SlabPlan(params["Ny"], nslabs or 1, halo)
        make = slab_factory or (lambda plan, r: SolverSlab(plan, r, self.params, precision=precision,
                                                           device=(devices[r] if devices else -1), **solver_kw))
        ranks = [self.transport.rank] if dist_mode else range(self.plan.nslabs)
        self.slabs = [make(self.plan, r) for r in ranks]
        self.it = 0

    def initialization(self, tin=None) -> None:
        """Initial condition on every slab (ghost rows included, so they start
        valid); tin: optional hot-wall temperature per global row."""
        for s in self.slabs:
            s.initialization(tin)
        self.it = 0

    def step(self, nsteps: int) -> None:
        for h, final in self.plan.chunks(int(nsteps)):
            for s in self.slabs:
                s.run(h, final)
            if self.plan.nslabs > 1:
                self.transport.exchange(self.slabs)
            self.it += h

    def sync(self) -> None:
        for s in self.slabs:
            s.sync()

    def sums(self) -> np.ndarray:
        """Interior sums (rho, T, phi, #phi>0) over the owned rows of all slabs."""
        tot = np.zeros(4)
        for s in self.slabs:
            tot += s.own_sums()
        if isinstance(self.transport, DistTransport):
            import torch
            t = torch.tensor(tot, dtype=torch.float64)
            s0 = self.slabs[0]
            if getattr(s0, "device", None) is not None and s0.device.type == "cuda":
                t = t.to(s0.device)
            self.transport.dist.all_reduce(t, group=self.transport.group)
            tot = t.cpu().numpy()
        return tot

    def own_rows(self, s, name: str) -> np.ndarray:
        """Reference-layout rows of slab s: its owned rows, plus the bottom
        halo row (slab 0) and the top halo row (last slab)."""
        p, r = self.plan, s.r
        a = s.local_field(name)
        j0 = p.below(r) + 1 - (1 if r == 0 else 0)
        j1 = p.below(r) + p.own(r) + (2 if r == p.nslabs - 1 else 1)
        return a[j0:j1]

    def field(self, name: str):
        """The global field (Ny+2, Nx+2) in the reference layout; with a
        DistTransport, on rank 0 (None on the other ranks)."""
        parts = [(s.r, self.own_rows(s, name)) for s in self.slabs]
        if isinstance(self.transport, DistTransport):
            d = self.transport.dist
            gathered = [None] * self.transport.world if self.transport.rank == 0 else None
            d.gather_object(parts, gathered, dst=self.transport.peer(0), group=self.transport.group)
            if self.transport.rank != 0:
                return None
            parts = [x for g in gathered for x in g]
        parts.sort(key=lambda t: t[0])
        return np.concatenate([a for _, a in parts], axis=0)

    def close(self) -> None:
        for s in self.slabs:
            s.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
