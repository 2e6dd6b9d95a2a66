"""Learned preconditioner: the gauge-equivariant PTC network, its training,
and flexible GCR with the network as preconditioner.

No counterpart in the reference (its solvers are CG, BiCGStab and
multishift CG).  The network, its forward and backward kernels and the GCR
solver run in libiroiro_b200.so (include/iroiro_b200.h, "learned
preconditioner"); this module holds the host side: weight initialisation,
the Adam optimiser, and the training loop over (source, solution) pairs that
the plain FP64 CG produces.

Layer widths are counted in colour-vector channels: a spinor is 4 channels
(12 spin-colour components).  The default network has 4 layers,
4 -> 16 -> 16 -> 16 -> 4 channels.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass

import numpy as np

from . import (BAD_ARG, NOT_CONVERGED, OK, OP_CLOVER_FULL, OP_WILSON_FULL, Context, DeviceField,
               Fopr_DdagD, IroError, Solver_CG, _VP, _D, lib)

DEFAULT_WIDTHS = (4, 16, 16, 16, 4)


class GCROut(ctypes.Structure):
    _fields_ = [("diff", ctypes.c_double), ("iterations", ctypes.c_int),
                ("timing_ms", ctypes.c_double), ("restarts", ctypes.c_int),
                ("fallback", ctypes.c_int), ("precond_applies", ctypes.c_int)]


class GCRParams(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_double), ("max_iter", ctypes.c_int),
                ("nkrylov", ctypes.c_int), ("delta", ctypes.c_double),
                ("krylov_half", ctypes.c_int)]


def _declare():
    L = lib()
    if getattr(L, "_learned_declared", False):
        return L
    I, D = ctypes.c_int, ctypes.c_double
    F = ctypes.POINTER(ctypes.c_float)
    sig = {
        "iro_ptc_create": (I, [_VP, I, ctypes.POINTER(I), ctypes.POINTER(_VP)]),
        "iro_ptc_destroy": (I, [_VP]),
        "iro_ptc_set_weights": (I, [_VP, I, F]),
        "iro_ptc_apply": (I, [_VP, _VP, _D, _D]),
        "iro_ptc_apply_field": (I, [_VP, _VP, _VP, _VP]),
        "iro_ptc_loss_grad": (I, [_VP, _VP, _VP, _VP, ctypes.POINTER(D), F]),
        "iro_gcr_solve_field": (I, [_VP, I, D, D, _VP, ctypes.POINTER(GCRParams), _VP, _VP,
                                    ctypes.POINTER(GCROut)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    L._learned_declared = True
    return L


def init_weights(widths, seed: int = 0, scale: float = 0.05):
    """Each layer starts as a channel-preserving identity on the site itself
    (so the whole network starts as the identity map) plus small random
    weights on every displacement."""
    rng = np.random.default_rng(seed)
    Ws = []
    for cin, cout in zip(widths[:-1], widths[1:]):
        W = scale * (rng.standard_normal((9, cout, cin)) + 1j * rng.standard_normal((9, cout, cin)))
        W /= np.sqrt(9 * cin)
        for k in range(min(cin, cout)):
            W[0, k, k] += 1.0
        Ws.append(W)
    return Ws


def pack(W: np.ndarray) -> np.ndarray:
    out = np.empty(W.shape + (2,), dtype=np.float32)
    out[..., 0] = W.real
    out[..., 1] = W.imag
    return out.ravel()


class PTCNet:
    """The network on one lattice (any gauge field of that lattice)."""

    def __init__(self, ctx: Context, widths=DEFAULT_WIDTHS, weights=None, seed: int = 0):
        self.L = _declare()
        self.ctx = ctx
        self.widths = tuple(int(w) for w in widths)
        h = _VP()
        arr = (ctypes.c_int * len(self.widths))(*self.widths)
        ctx.check(self.L.iro_ptc_create(ctx.h, len(self.widths) - 1, arr, ctypes.byref(h)),
                  "iro_ptc_create")
        self.h = h
        ctx._owned.add(self)
        self.set_weights(weights if weights is not None else init_weights(self.widths, seed))

    def set_weights(self, Ws):
        self.W = [np.asarray(W, dtype=np.complex128) for W in Ws]
        for l, W in enumerate(self.W):
            p = pack(W)
            rc = self.L.iro_ptc_set_weights(self.h, l, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
            if rc:
                raise IroError(rc, "iro_ptc_set_weights")

    def apply(self, f: np.ndarray, ctx: Context = None) -> np.ndarray:
        ctx = ctx or self.ctx
        f = np.ascontiguousarray(f, dtype=np.float64)
        out = np.empty_like(f)
        ctx.check(self.L.iro_ptc_apply(ctx.h, self.h, f.ctypes.data_as(_D), out.ctypes.data_as(_D)),
                  "iro_ptc_apply")
        return out

    def loss_grad(self, ctx: Context, b: DeviceField, x: DeviceField, want_grad: bool = True):
        loss = ctypes.c_double()
        sizes = [9 * ci * co * 2 for ci, co in zip(self.widths[:-1], self.widths[1:])]
        g = np.empty(sum(sizes), dtype=np.float32) if want_grad else None
        gp = g.ctypes.data_as(ctypes.POINTER(ctypes.c_float)) if want_grad else None
        ctx.check(self.L.iro_ptc_loss_grad(ctx.h, self.h, b.h, x.h, ctypes.byref(loss), gp),
                  "iro_ptc_loss_grad")
        if not want_grad:
            return loss.value, None
        grads, off = [], 0
        for (ci, co), n in zip(zip(self.widths[:-1], self.widths[1:]), sizes):
            a = g[off:off + n].astype(np.float64).reshape(9, co, ci, 2)
            grads.append(a[..., 0] + 1j * a[..., 1])
            off += n
        return loss.value, grads

    def close(self):
        if getattr(self, "h", None):
            self.L.iro_ptc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Adam:
    """Adam (Kingma & Ba, 2015) on complex weights, treating re/im as reals."""

    def __init__(self, Ws, lr=2e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.lr, self.b1, self.b2, self.eps = lr, b1, b2, eps
        self.m = [np.zeros_like(W) for W in Ws]
        self.v = [np.zeros(W.shape + (2,)) for W in Ws]
        self.t = 0

    def step(self, Ws, grads):
        self.t += 1
        out = []
        for k, (W, g) in enumerate(zip(Ws, grads)):
            self.m[k] = self.b1 * self.m[k] + (1 - self.b1) * g
            g2 = np.stack([g.real ** 2, g.imag ** 2], axis=-1)
            self.v[k] = self.b2 * self.v[k] + (1 - self.b2) * g2
            mh = self.m[k] / (1 - self.b1 ** self.t)
            vh = self.v[k] / (1 - self.b2 ** self.t)
            step = mh.real / (np.sqrt(vh[..., 0]) + self.eps) + 1j * mh.imag / (np.sqrt(vh[..., 1]) + self.eps)
            out.append(W - self.lr * step)
        return out


@dataclass
class TrainingPair:
    ctx: Context          # holds the pair's gauge field
    b: DeviceField        # network input
    x: DeviceField        # target, the exact (D^dag D)^-1 b
    cg_iterations: int    # 0 for kind="random" (no solve is needed)


def make_pairs(L, nfields: int, kappa: float = 0.12, eps: float = 0.2, seed0: int = 5000,
               op=OP_WILSON_FULL, csw: float = 0.0, device: int = 0, kind: str = "random"):
    """Training pairs (b, x) with x = (D^dag D)^-1 b, one seeded gauge field each.

    kind="random" (the default): x = v is a Gaussian field and b = D^dag D v,
    the cost |N(D^dag D v) - v|^2 of Lehner & Wettig, which weights every
    eigenmode of the operator alike and needs no solve.  kind="solve": b is
    Gaussian and x comes from the plain FP64 CG to 1e-10; that target is
    dominated by the lowest modes, which a local network cannot represent,
    and trains a much weaker preconditioner."""
    from . import Dirac_Clover, Dirac_Wilson, synth_gauge, synth_gaussian
    if kind not in ("random", "solve"):
        raise ValueError(f"unknown pair kind {kind!r}")
    mass = 0.5 / kappa - 4.0
    V = int(np.prod(L))
    pairs = []
    for k in range(nfields):
        ctx = Context(L, device)
        u = synth_gauge(L, eps, seed0 + k)
        ctx.upload_gauge(u, force=True)
        D = Dirac_Wilson(mass, u, ctx=ctx)
        if op == OP_CLOVER_FULL:
            D = Dirac_Clover(D, csw, u, ctx=ctx)
        g = synth_gaussian(V, seed0 + 100000 + k)
        if kind == "random":
            b = DeviceField(ctx, 2, "double").upload(Fopr_DdagD(D).mult(g))
            pairs.append(TrainingPair(ctx, b, DeviceField(ctx, 2, "double").upload(g), 0))
            continue
        b = DeviceField(ctx, 2, "double").upload(g)
        x = DeviceField(ctx, 2, "double")
        outs, rc = Solver_CG(1e-20, 20000, Fopr_DdagD(D)).solve_field(b, x)
        if rc != OK:
            raise IroError(rc, "training data: CG did not converge")
        pairs.append(TrainingPair(ctx, b, x, outs[0].Iterations))
    return pairs


def train(net: PTCNet, pairs, epochs: int = 20, lr: float = 2e-3, log=None):
    """Adam on the relative error |N(b) - x|^2 / |x|^2 over the pairs; returns
    the mean loss of every epoch."""
    opt = Adam(net.W, lr=lr)
    history = []
    for ep in range(epochs):
        tot = 0.0
        for pr in pairs:
            loss, grads = net.loss_grad(pr.ctx, pr.b, pr.x)
            tot += loss
            net.set_weights(opt.step(net.W, grads))
        history.append(tot / len(pairs))
        if log:
            log(f"epoch {ep}: loss {history[-1]:.4e}")
    return history


class Solver_GCR:
    """Flexible GCR for (D^dag D) x = b on the full lattice with the network
    as right preconditioner (net=None: plain GCR); FP32 inner iterations
    (krylov="half": the directions z_j and w_j = A z_j stored in FP16 and A
    applied in mixed FP16), FP64 restarts and convergence test;
    mixed-precision CG fallback on a stall."""

    def __init__(self, D, net: PTCNet = None, prec: float = 1e-20, max_iter: int = 5000,
                 nkrylov: int = 8, delta: float = 0.1, krylov: str = "single"):
        if D.op not in (OP_WILSON_FULL, OP_CLOVER_FULL):
            raise IroError(BAD_ARG, "GCR needs a full-lattice Wilson or clover operator")
        if krylov not in ("single", "half"):
            raise IroError(BAD_ARG, "krylov must be 'single' or 'half'")
        self.L = _declare()
        self.D, self.net = D, net
        self.params = GCRParams(prec, max_iter, nkrylov, delta, 1 if krylov == "half" else 0)

    def solve_field(self, b: DeviceField, x: DeviceField):
        """Returns (GCROut, status) with status OK or NOT_CONVERGED."""
        D = self.D
        o = GCROut()
        rc = self.L.iro_gcr_solve_field(D.ctx.h, D.op, D.mass, D.csw,
                                        self.net.h if self.net else None, ctypes.byref(self.params),
                                        b.h, x.h, ctypes.byref(o))
        if rc not in (OK, NOT_CONVERGED):
            D.ctx.check(rc, "iro_gcr_solve_field")
        return o, rc
