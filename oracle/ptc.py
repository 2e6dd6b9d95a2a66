"""CPU oracle of the parallel-transport convolution network -- TEST INFRASTRUCTURE ONLY.

FP64 numpy restatement of the gauge-equivariant network the library trains
and applies as a preconditioner (the reference has no learned part):

    out_o(x) = sum_{d=0..8} sum_i W_d[o, i] (T_d in_i)(x)
    T_0 = 1,  T_{+mu} f(x) = U_mu(x) f(x+mu),  T_{-mu} f(x) = U_mu(x-mu)^dag f(x-mu)
    d = 1 + 2*mu (forward), 2 + 2*mu (backward)

Sites are the full lattice in even/odd order, s = p*Vh + hs (hs the index of
the site within its parity in lexicographic order), features are complex
arrays [V, C, 3] (channel, colour).  A spinor in Format_F order is 4
channels, feature[s, spin, colour].

The gradient is the exact adjoint: for y = W x, dL/dW = sum delta conj(x) and
dL/dx = W^dag delta, with delta = dL/dRe(y) + i dL/dIm(y); the transport
adjoints are T_{+mu}^dag g(y) = U_mu(y-mu)^dag g(y-mu) and
T_{-mu}^dag g(y) = U_mu(y) g(y+mu).
"""
from __future__ import annotations

import numpy as np


class Lattice:
    """Neighbour tables and links of the full lattice in e/o order."""

    def __init__(self, L, u_formatG: np.ndarray):
        L = [int(v) for v in L]
        self.L = L
        V = int(np.prod(L))
        Vh = V // 2
        self.V, self.Vh = V, Vh
        # lexicographic site of every e/o site
        hs = np.arange(Vh)
        lex = np.empty(V, dtype=np.int64)
        coords = np.empty((V, 4), dtype=np.int64)
        for p in (0, 1):
            row = hs // (L[0] // 2)
            xh = hs % (L[0] // 2)
            y = row % L[1]
            z = (row // L[1]) % L[2]
            t = row // (L[1] * L[2])
            x = 2 * xh + ((y + z + t + p) & 1)
            s = p * Vh + hs
            lex[s] = x + L[0] * (y + L[1] * (z + L[2] * t))
            coords[s] = np.stack([x, y, z, t], axis=1)
        self.lex = lex
        eo_of_lex = np.empty(V, dtype=np.int64)
        eo_of_lex[lex] = np.arange(V)
        nb = np.empty((V, 8), dtype=np.int64)
        for mu in range(4):
            for k, sg in enumerate((1, -1)):
                c = coords.copy()
                c[:, mu] = (c[:, mu] + sg) % L[mu]
                nl = c[:, 0] + L[0] * (c[:, 1] + L[1] * (c[:, 2] + L[2] * c[:, 3]))
                nb[:, 2 * mu + k] = eo_of_lex[nl]
        self.nb = nb
        Ug = u_formatG.reshape(4, V, 3, 3, 2)
        U = Ug[..., 0] + 1j * Ug[..., 1]            # [mu, lex, 3, 3]
        self.U = U[:, lex]                             # [mu, s, 3, 3] link at e/o site s

    def transport(self, f: np.ndarray, d: int) -> np.ndarray:
        if d == 0:
            return f
        mu, bwd = (d - 1) // 2, (d - 1) % 2
        n = self.nb[:, d - 1]
        if not bwd:
            return np.einsum("sab,scb->sca", self.U[mu], f[n])
        return np.einsum("sba,scb->sca", self.U[mu][n].conj(), f[n])

    def transport_adj(self, g: np.ndarray, d: int) -> np.ndarray:
        if d == 0:
            return g
        mu, bwd = (d - 1) // 2, (d - 1) % 2
        if not bwd:  # T_{+mu}^dag g(y) = U_mu(y-mu)^dag g(y-mu)
            m = self.nb[:, 2 * mu + 1]
            return np.einsum("sba,scb->sca", self.U[mu][m].conj(), g[m])
        m = self.nb[:, 2 * mu]          # T_{-mu}^dag g(y) = U_mu(y) g(y+mu)
        return np.einsum("sab,scb->sca", self.U[mu], g[m])


def spinor_to_feat(lat: Lattice, f_formatF: np.ndarray) -> np.ndarray:
    f = f_formatF.reshape(lat.V, 4, 3, 2)
    c = f[..., 0] + 1j * f[..., 1]
    return c[lat.lex]


def feat_to_spinor(lat: Lattice, feat: np.ndarray) -> np.ndarray:
    out = np.empty((lat.V, 4, 3, 2))
    out[lat.lex, ..., 0] = feat.real
    out[lat.lex, ..., 1] = feat.imag
    return out.ravel()


def layer(lat: Lattice, W: np.ndarray, x: np.ndarray) -> np.ndarray:
    """W: complex [9, cout, cin]; x: [V, cin, 3]."""
    return sum(np.einsum("oi,sia->soa", W[d], lat.transport(x, d)) for d in range(9))


def forward(lat: Lattice, Ws, x: np.ndarray):
    acts = [x]
    for W in Ws:
        acts.append(layer(lat, W, acts[-1]))
    return acts


def loss_grad(lat: Lattice, Ws, x: np.ndarray, t: np.ndarray):
    """loss = |N(x) - t|^2 / |t|^2 and dloss/dW_l (complex, same shapes)."""
    acts = forward(lat, Ws, x)
    tt = np.vdot(t, t).real
    diff = acts[-1] - t
    loss = np.vdot(diff, diff).real / tt
    delta = 2.0 * diff / tt
    grads = [None] * len(Ws)
    for l in range(len(Ws) - 1, -1, -1):
        W, xin = Ws[l], acts[l]
        g = np.zeros_like(W)
        dx = np.zeros_like(xin)
        for d in range(9):
            Tx = lat.transport(xin, d)
            g[d] = np.einsum("soa,sia->oi", delta, Tx.conj())
            dx += lat.transport_adj(np.einsum("oi,soa->sia", W[d].conj(), delta), d)
        grads[l] = g
        delta = dx
    return loss, grads, acts[-1]


def pack(W: np.ndarray) -> np.ndarray:
    """complex [9, cout, cin] -> float32 (re, im) interleaved, the library's layout."""
    out = np.empty(W.shape + (2,), dtype=np.float32)
    out[..., 0] = W.real
    out[..., 1] = W.imag
    return out.ravel()


def unpack(g: np.ndarray, cin: int, cout: int) -> np.ndarray:
    a = np.asarray(g, dtype=np.float64).reshape(9, cout, cin, 2)
    return a[..., 0] + 1j * a[..., 1]
