"""The y-slab decomposition's host logic on CPU.

SlabRun and its transports move packed rows between slabs without knowing
what a slab computes.  Here a slab is the oracle (the CPU restatement of
STEP_7) on its rows plus ghost rows, so the decomposition is checked end to
end without a GPU: slabs in one process (LocalTransport) and one slab per
gloo rank (DistTransport, the code path NCCL takes between GPUs) must give
the undivided oracle run bit for bit.  The oracle's step is unfused, so a
slab exchanges every per-node array of its rows, not only the fused step's
state."""
from __future__ import annotations

import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT, small_params


# --------------------------------------------------------------- the plan
def test_plan_partition_and_ghosts():
    from bgk_pcm_b200.slab import SlabPlan
    p = SlabPlan(100, 3, 4)
    assert [(p.lo(r), p.hi(r)) for r in range(3)] == [(0, 33), (33, 66), (66, 100)]
    assert [(p.below(r), p.above(r)) for r in range(3)] == [(0, 4), (4, 4), (4, 0)]
    assert [p.local_ny(r) for r in range(3)] == [37, 41, 38]
    assert [p.first_row(r) for r in range(3)] == [0, 29, 62]
    one = SlabPlan(7, 1, 5)
    assert (one.below(0), one.above(0), one.local_ny(0)) == (0, 0, 7)


def test_plan_chunks_end_with_two_moment_steps():
    from bgk_pcm_b200.slab import SlabPlan
    assert list(SlabPlan(100, 2, 4).chunks(10)) == [(4, False), (4, False), (2, True)]
    assert list(SlabPlan(100, 2, 4).chunks(9)) == [(4, False), (4, True), (1, True)]
    assert list(SlabPlan(100, 2, 1).chunks(3)) == [(1, False), (1, True), (1, True)]
    assert list(SlabPlan(100, 2, 4).chunks(3)) == [(3, True)]
    assert list(SlabPlan(100, 2, 4).chunks(0)) == []


def test_plan_rejects_thin_slabs():
    from bgk_pcm_b200.slab import SlabPlan
    with pytest.raises(ValueError, match="fewer than"):
        SlabPlan(10, 4, 3)
    with pytest.raises(ValueError):
        SlabPlan(10, 0, 1)
    with pytest.raises(ValueError):
        SlabPlan(10, 2, 0)


# ----------------------------------------------------- an oracle-backed slab
class OracleSlab:
    """A slab whose rows are stepped by the oracle (test infrastructure)."""

    def __init__(self, plan, r, params):
        import torch
        from oracle.pyoracle import FIELD_NAMES, Oracle
        self.plan, self.r = plan, r
        q = dict(params)
        q["Ny"] = plan.local_ny(r)
        self.orc = Oracle(q)
        self.names = FIELD_NAMES
        self.Nx = params["Nx"]
        shape = (len(FIELD_NAMES), plan.halo, self.Nx + 2)
        self.buf = {k: torch.zeros(shape, dtype=torch.float64) for k in ("send_lo", "send_hi", "recv_lo", "recv_hi")}
        self.device = None

    def initialization(self, tin=None):
        assert tin is None
        self.orc.initialization()

    def run(self, nsteps, final):
        self.orc.step(nsteps)

    def _rows(self, side, ghost):
        p, r = self.plan, self.r
        if ghost:
            j0 = 1 if side == "lo" else p.below(r) + p.own(r) + 1
        else:
            j0 = p.below(r) + 1 if side == "lo" else p.below(r) + p.own(r) - p.halo + 1
        return slice(j0, j0 + p.halo)

    def pack(self, side):
        import torch
        rows = self._rows(side, ghost=False)
        b = self.buf["send_" + side]
        b.copy_(torch.from_numpy(np.stack([self.orc.field(n)[rows] for n in self.names])))
        return b

    def recv_buffer(self, side):
        return self.buf["recv_" + side]

    def unpack(self, side):
        rows = self._rows(side, ghost=True)
        b = self.buf["recv_" + side].numpy()
        for k, n in enumerate(self.names):
            a = self.orc.field(n)
            a[rows] = b[k]
            self.orc.set_field(n, a)

    def sync(self):
        pass

    def own_sums(self):
        p, r = self.plan, self.r
        rows = slice(p.below(r) + 1, p.below(r) + p.own(r) + 1)
        rho, T, phi = (self.orc.field(n)[rows, 1:-1] for n in ("rho", "T", "phi"))
        return np.array([rho.sum(), T.sum(), phi.sum(), float((phi > 0).sum())])

    def local_field(self, name):
        return self.orc.field(name)

    def close(self):
        self.orc.close()


def _params():
    return small_params(Nx=23, Ny=31, T_in_sol=271.0)


def _undivided(params, steps):
    from oracle.pyoracle import Oracle
    o = Oracle(params)
    o.initialization()
    o.step(steps)
    out = {n: o.field(n) for n in ("rho", "T", "u", "v", "phi", "f2", "f7", "g4", "g5")}
    o.close()
    return out


@pytest.mark.parametrize("nslabs,halo,steps", [(3, 1, 7), (3, 3, 11), (2, 4, 9)])
def test_local_slabs_match_undivided_oracle(oracle_mod, nslabs, halo, steps):
    from bgk_pcm_b200.slab import LocalTransport, SlabRun
    params = _params()
    ref = _undivided(params, steps)
    run = SlabRun(params, nslabs=nslabs, halo=halo, transport=LocalTransport(),
                  slab_factory=lambda plan, r: OracleSlab(plan, r, params))
    try:
        run.initialization()
        run.step(steps)
        for n, a in ref.items():
            np.testing.assert_array_equal(run.field(n), a, err_msg=n)
        s = run.sums()
        own = ref["rho"][1:-1, 1:-1]
        assert abs(s[0] - own.sum()) <= 1e-12 * abs(own.sum())
        assert s[3] == float((ref["phi"][1:-1, 1:-1] > 0).sum())
    finally:
        run.close()


def test_ghost_rows_are_needed(oracle_mod):
    """Without the exchanges the slabs' cut rows see walls, and the result
    differs from the undivided run: the test above is not vacuous."""
    from bgk_pcm_b200.slab import LocalTransport, SlabRun

    class NoExchange(LocalTransport):
        def exchange(self, slabs):
            pass

    params = _params()
    ref = _undivided(params, 9)
    run = SlabRun(params, nslabs=2, halo=3, transport=NoExchange(),
                  slab_factory=lambda plan, r: OracleSlab(plan, r, params))
    try:
        run.initialization()
        run.step(9)
        assert not np.array_equal(run.field("f2"), ref["f2"])
    finally:
        run.close()


# --------------------------------------------------- one slab per gloo rank
def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, halo, steps, q):
    import datetime
    import sys
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    import torch.distributed as dist
    from bgk_pcm_b200.slab import DistTransport, SlabRun
    from test_slab import OracleSlab, _params
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        params = _params()
        run = SlabRun(params, halo=halo, transport=DistTransport(),
                      slab_factory=lambda plan, r: OracleSlab(plan, r, params))
        run.initialization()
        run.step(steps)
        fields = {n: run.field(n) for n in ("rho", "T", "u", "v", "phi", "f2", "f7", "g4", "g5")}
        sums = run.sums()
        run.close()
        q.put((rank, fields if rank == 0 else None, sums))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,halo,steps", [(2, 2, 9), (3, 1, 5)])
def test_gloo_ranks_match_undivided_oracle(oracle_mod, world, halo, steps):
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, halo, steps, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        rank, fields, sums = q.get(timeout=180)
        res[rank] = (fields, sums)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    ref = _undivided(_params(), steps)
    for n, a in ref.items():
        np.testing.assert_array_equal(res[0][0][n], a, err_msg=n)
    for r in range(world):                       # all_reduce: every rank holds the same sums
        np.testing.assert_array_equal(res[r][1], res[0][1])
    assert res[0][1][3] == float((ref["phi"][1:-1, 1:-1] > 0).sum())


def _subgroup_main(rank, world, port, q):
    import datetime
    import sys
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    import torch.distributed as dist
    from bgk_pcm_b200.slab import DistTransport, SlabRun
    from test_slab import OracleSlab, _params
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        group = dist.new_group([1, 2])              # every rank takes part in new_group
        if rank in (1, 2):
            params = _params()
            run = SlabRun(params, halo=2, transport=DistTransport(group),
                          slab_factory=lambda plan, r: OracleSlab(plan, r, params))
            run.initialization()
            run.step(7)
            phi = run.field("phi")
            run.close()
            q.put((rank, phi))
        else:
            q.put((rank, None))
    finally:
        dist.destroy_process_group()


def test_gloo_subgroup_addresses_peers_by_global_rank(oracle_mod):
    """Slabs on ranks 1 and 2 of a 3-rank world, through a subgroup: the
    group's rank 0 (global rank 1) gathers the field."""
    world, port = 3, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_subgroup_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    ref = _undivided(_params(), 7)
    assert res[0] is None and res[2] is None
    np.testing.assert_array_equal(res[1], ref["phi"])


@pytest.mark.parametrize("wall", ["westBC", "eastBC", "northBC", "southBC"])
def test_slab_run_rejects_walls_other_than_no_slip(wall):
    """A slab builds inflow or pressure walls from its own rows, so only the
    no-slip code 4 decomposes; SlabRun refuses anything else before it
    creates a slab (even a call short enough to run only final chunks)."""
    from bgk_pcm_b200.slab import SlabRun
    params = dict(small_params(12, 16), **{wall: 2})
    made = []
    with pytest.raises(ValueError, match="code 4"):
        SlabRun(params, nslabs=2, halo=2, slab_factory=lambda plan, r: made.append(r))
    assert made == []


@pytest.mark.parametrize("heat", ["right", "bottom", 3])
def test_slab_run_rejects_heating_options(heat):
    """The heating options place the liquid layer and the hot wall by global
    rows and columns, so SlabRun refuses them before it creates a slab."""
    from bgk_pcm_b200.slab import SlabRun
    made = []
    with pytest.raises(ValueError, match="west"):
        SlabRun(small_params(12, 16), nslabs=2, halo=2, slab_factory=lambda plan, r: made.append(r), heat=heat)
    assert made == []
