"""Learned preconditioner on the GPU: the tensor-core network forward and its
gradients against the FP64 CPU oracle, GCR with and without the network, and
training that lowers the loss and the GCR iteration count."""
import numpy as np
import pytest

import iroiro_b200 as ib
from iroiro_b200 import learned
from oracle import ptc

pytestmark = pytest.mark.gpu

# BF16 operands and weights with FP32 accumulation: a few parts in 1e3 per layer
TOL_NET = 3e-2


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a - b)) / np.linalg.norm(np.ravel(b)))


@pytest.fixture(scope="module")
def small():
    L = [4, 4, 4, 8]
    u = ib.synth_gauge(L, 0.25, 21, gauge_transform=True)
    ctx = ib.Context(L, 0)
    ctx.upload_gauge(u, force=True)
    return L, u, ctx


@pytest.mark.parametrize("widths", [(4, 4), (4, 16, 4), (4, 16, 16, 16, 4), (4, 8, 4)])
def test_forward_vs_oracle(small, widths):
    L, u, ctx = small
    V = int(np.prod(L))
    Ws = learned.init_weights(widths, seed=3, scale=0.5)
    net = learned.PTCNet(ctx, widths, Ws)
    f = ib.synth_gaussian(V, 31)
    got = net.apply(f)
    lat = ptc.Lattice(L, u)
    want = ptc.feat_to_spinor(lat, ptc.forward(lat, Ws, ptc.spinor_to_feat(lat, f))[-1])
    assert rel(got, want) < TOL_NET


def test_loss_and_gradients_vs_oracle(small):
    L, u, ctx = small
    V = int(np.prod(L))
    widths = (4, 16, 16, 16, 4)
    Ws = learned.init_weights(widths, seed=5, scale=0.5)
    net = learned.PTCNet(ctx, widths, Ws)
    b, t = ib.synth_gaussian(V, 41), ib.synth_gaussian(V, 42)
    db = ib.DeviceField(ctx, 2, "double").upload(b)
    dt = ib.DeviceField(ctx, 2, "double").upload(t)
    loss, grads = net.loss_grad(ctx, db, dt)
    lat = ptc.Lattice(L, u)
    loss_o, grads_o, _ = ptc.loss_grad(lat, Ws, ptc.spinor_to_feat(lat, b), ptc.spinor_to_feat(lat, t))
    assert abs(loss - loss_o) < TOL_NET * loss_o
    for g, go in zip(grads, grads_o):
        assert rel(g, go) < 5e-2


def _pair(L, seed):
    u = ib.synth_gauge(L, 0.2, seed)
    ctx = ib.Context(L, 0)
    ctx.upload_gauge(u, force=True)
    D = ib.Dirac_Wilson(0.5 / 0.12 - 4, u, ctx=ctx)
    V = int(np.prod(L))
    b = ib.DeviceField(ctx, 2, "double").upload(ib.synth_gaussian(V, seed + 1))
    return ctx, D, b


@pytest.mark.parametrize("krylov", ["single", "half"])
def test_gcr_converges_with_and_without_network(krylov):
    # FP32 or FP16 directions: the FP64 restarts bring both to the FP64 CG solution
    L = [8, 8, 8, 8]
    ctx, D, b = _pair(L, 61)
    x_cg = ib.DeviceField(ctx, 2, "double")
    outs, rc = ib.Solver_CG(1e-20, 5000, ib.Fopr_DdagD(D)).solve_field(b, x_cg)
    ref = x_cg.download()
    for net in (None, learned.PTCNet(ctx, learned.DEFAULT_WIDTHS)):
        x = ib.DeviceField(ctx, 2, "double")
        o, st = learned.Solver_GCR(D, net, krylov=krylov).solve_field(b, x)
        assert st == ib.OK and o.diff < 1e-10
        assert rel(x.download(), ref) < 1e-8


def test_training_lowers_loss_and_gcr_iterations():
    L = [8, 8, 8, 8]
    pairs = learned.make_pairs(L, 4, seed0=7100)
    net = learned.PTCNet(pairs[0].ctx, learned.DEFAULT_WIDTHS)
    hist = learned.train(net, pairs, epochs=12, lr=3e-3)
    assert hist[-1] < 0.3 * hist[0]
    # an unseen field: fewer GCR iterations with the trained network than with none
    ctx, D, b = _pair(L, 7900)
    its = {}
    for name, n in (("none", None), ("trained", net)):
        x = ib.DeviceField(ctx, 2, "double")
        o, st = learned.Solver_GCR(D, n).solve_field(b, x)
        assert st == ib.OK and o.diff < 1e-10
        its[name] = (o.iterations, o.fallback)
    # the trained network removes the stall (no CG fallback) and most iterations
    assert its["trained"][1] == 0 and its["trained"][0] < 0.6 * its["none"][0], its


def test_solver_scratch_shared_by_gcr_and_md_force():
    """GCR keeps its per-call state (block partials, the cycle's coefficients)
    in the context's solver scratch, which the clover MD force then grows for
    its force and Lambda buffers: on one context a GCR solve, a force and the
    same GCR solve again give the same bits, and the force equals the one of a
    fresh context."""
    L = [8, 8, 8, 8]
    V = int(np.prod(L))
    m, csw = 0.5 / 0.12 - 4, 1.0
    u = ib.synth_gauge(L, 0.2, 131)
    ctx = ib.Context(L, 0)
    ctx.upload_gauge(u, force=True)
    Dw = ib.Dirac_Wilson(m, u, ctx=ctx)
    b = ib.DeviceField(ctx, 2, "double").upload(ib.synth_gaussian(V, 132))
    net = learned.PTCNet(ctx, learned.DEFAULT_WIDTHS)
    x1 = ib.DeviceField(ctx, 2, "double")
    o1, st1 = learned.Solver_GCR(Dw, net).solve_field(b, x1)
    e, z = ib.synth_gaussian(V, 133), ib.synth_gaussian(V, 134)
    F1 = ib.Dirac_Clover(Dw, csw, u, ctx=ctx).md_force(e, z)
    x2 = ib.DeviceField(ctx, 2, "double")
    o2, st2 = learned.Solver_GCR(Dw, net).solve_field(b, x2)
    assert st1 == ib.OK and st2 == ib.OK and o1.iterations == o2.iterations, (o1, o2)
    assert np.array_equal(x1.download(), x2.download())
    ctx2 = ib.Context(L, 0)
    F2 = ib.Dirac_Clover(ib.Dirac_Wilson(m, u, ctx=ctx2), csw, u, ctx=ctx2).md_force(e, z)
    assert np.array_equal(F1, F2)


def test_gcr_zero_source_returns_zero():
    """b = 0: x = 0 is the solution, returned without an iteration."""
    L = [4, 4, 4, 8]
    ctx, D, _ = _pair(L, 141)
    b = ib.DeviceField(ctx, 2, "double").upload(np.zeros(int(np.prod(L)) * 24))
    x = ib.DeviceField(ctx, 2, "double").upload(ib.synth_gaussian(int(np.prod(L)), 142))
    o, st = learned.Solver_GCR(D, learned.PTCNet(ctx, learned.DEFAULT_WIDTHS)).solve_field(b, x)
    assert st == ib.OK and o.iterations == 0 and o.diff == 0.0
    assert not np.any(x.download())
