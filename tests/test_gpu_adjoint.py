"""The differentiation form: the hand-written adjoint of the fused step
against central finite differences of the (smooth) FP64 forward."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


# solid just below T_crit so that the small cavities respond within a few steps
SENSITIVE = dict(T_in_sol=271.0)


@pytest.mark.parametrize("Nx,Ny,steps,K", [(24, 16, 6, 4), (40, 33, 30, 7), (13, 1, 5, 2)])
def test_adjoint_small_fd(lib, Nx, Ny, steps, K):
    from bgk_pcm_b200 import gradcheck as gc
    p, tin, tin_t, pi, pj = gc.setup(Nx=Nx, Ny=Ny, steps=steps, nprobes=12, **SENSITIVE)
    pi = np.clip(pi, 1, Nx)
    target = gc.forward_phi(p, tin_t, steps, pi, pj)
    loss, g, gtau = gc.adjoint(p, tin, steps, pi, pj, target, checkpoint_every=K)
    assert abs(loss - gc.loss_of(p, tin, steps, pi, pj, target)) <= 1e-12 * max(loss, 1e-300)
    rows = gc.fd_check(p, tin, steps, pi, pj, target, g, gtau, ndir=6, h=1e-5)
    for fd, ad, rel in rows:
        assert rel < 1e-5 or abs(fd - ad) < 1e-12, rows


def test_adjoint_matches_tangent_oracle(oracle_mod, lib):
    """<grad L, v> from the adjoint equals the forward-mode derivative of the
    CPU restatement (dual numbers) along random directions v."""
    from bgk_pcm_b200 import gradcheck as gc
    p, tin, tin_t, pi, pj = gc.setup(Nx=20, Ny=14, steps=40, nprobes=8, **SENSITIVE)
    pi = np.clip(pi, 1, 6)
    target = gc.forward_phi(p, tin_t, 40, pi, pj)
    loss, g, gtau = gc.adjoint(p, tin, 40, pi, pj, target, checkpoint_every=7)
    rng = np.random.default_rng(5)
    for _ in range(4):
        v = rng.standard_normal(p["Ny"] + 1)
        Lt, dLt = oracle_mod.tangent_loss(p, tin, v[:-1], v[-1], 40, pi, pj, target)
        assert abs(Lt - loss) <= 1e-10 * abs(loss)
        ad = float(g @ v[:-1] + gtau * v[-1])
        assert abs(ad - dLt) <= 1e-8 * abs(dLt), (ad, dLt)


def test_adjoint_checkpoint_interval_invariant(lib):
    from bgk_pcm_b200 import gradcheck as gc
    p, tin, tin_t, pi, pj = gc.setup(Nx=32, Ny=24, steps=20, nprobes=10, **SENSITIVE)
    target = gc.forward_phi(p, tin_t, 20, pi, pj)
    a = gc.adjoint(p, tin, 20, pi, pj, target, checkpoint_every=20)
    b = gc.adjoint(p, tin, 20, pi, pj, target, checkpoint_every=3)
    assert a[0] == b[0]
    np.testing.assert_allclose(b[1], a[1], rtol=1e-12, atol=1e-300)
    assert abs(a[2] - b[2]) <= 1e-12 * abs(a[2])


def test_adjoint_requires_smooth(lib):
    from bgk_pcm_b200 import BGKError, Solver, inputs
    p = inputs.workload_params(Nx=16, Ny=16, iter=10, Ra=1e5)
    s = Solver(p)
    s.initialization()
    with pytest.raises(BGKError, match="UNSUPPORTED"):
        s.adjoint(3, [2], [2], [0.0])


@pytest.mark.parametrize("slots", [1, 2, 3, 7])
def test_adjoint_binomial_schedule_matches_sqrt_schedule(lib, slots):
    """checkpoint_every < 0 selects the memory-bounded binomial schedule with
    that many state slots (the one a grid too large for sqrt(N) snapshots
    falls back to); every reverse step sees the same forward state, so the
    gradient is identical bit for bit."""
    from bgk_pcm_b200 import gradcheck as gc
    p, tin, tin_t, pi, pj = gc.setup(Nx=40, Ny=33, steps=23, nprobes=10, **SENSITIVE)
    target = gc.forward_phi(p, tin_t, 23, pi, pj)
    a = gc.adjoint(p, tin, 23, pi, pj, target, checkpoint_every=5)
    b = gc.adjoint(p, tin, 23, pi, pj, target, checkpoint_every=-slots)
    assert a[0] == b[0] and a[2] == b[2]
    np.testing.assert_array_equal(a[1], b[1])


@pytest.mark.parametrize("K", [2, 3, 4, 7, 11, 23])
def test_adjoint_last_segment_lengths(lib, K):
    """23 steps with snapshots every K: last segments of 1, 2, 3, 2, 1 and 23
    steps.  From 3 steps on, the forward pass writes the last segment's
    states into the segment buffer instead of the reverse sweep recomputing
    them; every length gives the binomial schedule's gradient bit for bit."""
    from bgk_pcm_b200 import gradcheck as gc
    p, tin, tin_t, pi, pj = gc.setup(Nx=40, Ny=33, steps=23, nprobes=10, **SENSITIVE)
    target = gc.forward_phi(p, tin_t, 23, pi, pj)
    ref = gc.adjoint(p, tin, 23, pi, pj, target, checkpoint_every=-3)
    out = gc.adjoint(p, tin, 23, pi, pj, target, checkpoint_every=K)
    assert out[0] == ref[0] and out[2] == ref[2]
    np.testing.assert_array_equal(out[1], ref[1])


@pytest.mark.parametrize("K", [4, 5, 23])
def test_adjoint_leaves_context_at_step_n(lib, K):
    """After bgk_adjoint_run(N) the context holds S(N) with its moments, as
    after bgk_step(N), whichever way the forward pass ran its last segment."""
    from bgk_pcm_b200 import Solver, gradcheck as gc
    p, tin, tin_t, pi, pj = gc.setup(Nx=40, Ny=33, steps=23, nprobes=10, **SENSITIVE)
    target = gc.forward_phi(p, tin_t, 23, pi, pj)
    names = ["rho", "T", "u", "v", "phi"] + [f"f{k}" for k in range(9)] + [f"g{k}" for k in range(9)]
    with Solver(p, smooth=True) as a, Solver(p, smooth=True) as b:
        for s in (a, b):
            s.initialization()
            s.set_tin(tin)
        a.adjoint(23, pi, pj, target, K)
        b.step(23)
        assert a.it == b.it == 23
        for n in names:
            np.testing.assert_array_equal(a.field(n), b.field(n), err_msg=n)


def test_adjoint_repeated_on_one_context(lib):
    """The workspace kept in the context between calls (and its stale
    contents) does not change the result; a larger second call regrows it."""
    from bgk_pcm_b200 import Solver, gradcheck as gc
    p, tin, tin_t, pi, pj = gc.setup(Nx=40, Ny=33, steps=30, nprobes=10, **SENSITIVE)
    target = gc.forward_phi(p, tin_t, 30, pi, pj)
    ref = gc.adjoint(p, tin, 30, pi, pj, target, checkpoint_every=6)
    with Solver(p, smooth=True) as s:
        for K in (6, 30, 6):
            s.initialization()
            s.set_tin(tin)
            out = s.adjoint(30, pi, pj, target, K)
            assert out[0] == ref[0] and out[2] == ref[2]
            np.testing.assert_array_equal(out[1], ref[1])


@pytest.mark.slow
def test_adjoint_config4_fd_16_directions(lib):
    """512x512, Ra 1e5, 2000 steps, 64 probes, checkpoints every 45 steps:
    relative error <= 1e-5 against central differences with h = 1e-6 on 16
    random unit directions in (theta, tau_g), theta the dimensionless
    hot-wall temperature (Tin = T_in_sol + (T0 - T_in_sol) theta).  The
    gradient is taken through the torch.autograd wrapper of the C ABI."""
    from bgk_pcm_b200 import gradcheck as gc
    p, tin, tin_t, pi, pj = gc.setup()
    target = gc.forward_phi(p, tin_t, 2000, pi, pj)
    loss, g, gtau = gc.adjoint_autograd(p, tin, 2000, pi, pj, target, checkpoint_every=45)
    rows = gc.fd_check(p, tin, 2000, pi, pj, target, g, gtau, ndir=16, h=1e-6)
    worst = max(r[2] for r in rows)
    print("adjoint config4: loss", loss, "worst rel err", worst)
    assert worst <= 1e-5, rows


@pytest.mark.slow
def test_adjoint_config4_cost(lib):
    """Cost of one adjoint gradient in forward solves on the same workload,
    sqrt(N) checkpoints (K = 45).  Measured on B200: 3.62 (forward 36.5 ms,
    adjoint 132 ms); the target is 4.0."""
    from bgk_pcm_b200 import gradcheck as gc
    p, tin, tin_t, pi, pj = gc.setup()
    target = gc.forward_phi(p, tin_t, 2000, pi, pj)
    ratio, tf, ta = gc.cost_ratio(p, tin, 2000, pi, pj, target)
    print(f"adjoint/forward cost {ratio:.2f} (forward {tf*1e3:.1f} ms, adjoint {ta*1e3:.1f} ms)")
    assert ratio <= 4.0


def test_autograd_wrapper_matches_c_abi(lib):
    """The torch.autograd.Function returns exactly what bgk_adjoint_run returns."""
    from bgk_pcm_b200 import gradcheck as gc
    p, tin, tin_t, pi, pj = gc.setup(Nx=32, Ny=24, steps=20, nprobes=10, **SENSITIVE)
    target = gc.forward_phi(p, tin_t, 20, pi, pj)
    a = gc.adjoint(p, tin, 20, pi, pj, target, checkpoint_every=5)
    b = gc.adjoint_autograd(p, tin, 20, pi, pj, target, checkpoint_every=5)
    assert a[0] == b[0] and a[2] == b[2]
    np.testing.assert_array_equal(a[1], b[1])
