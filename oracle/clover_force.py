"""Test infrastructure (the oracle, never the product): a numpy restatement of
the molecular-dynamics force of the full Wilson-clover operator,
Dirac_Clover::md_force (lib/Dirac_ops/dirac_clover.cpp:356-367; its clover
block md_force_block, :369-532).

The force of md_force(eta, zeta) is the F with
    Re Tr(X F_mu(x)) = d/de Re(zeta^dag D(U_mu(x) -> (1 + e X) U_mu(x)) eta)
for every complex 3x3 X: the convention of the Wilson force
(Dirac_Wilson::md_force, dirac_wilson.cpp:41-58), which it adds to.  The clover
term of Dirac_Clover::mult (dirac_clover.cpp:334-349) is
    T f(x) = -kappa csw sum_k (i sigma_k (x) F_k(x)) f(x),
    F_k = 0.25 TA(Q_k),  Q_k(x) = L1 - L2 + L3 - L4
(Staples::fieldStrength, lib/Measurements/GaugeM/staples.cpp:587-666), with
the leaves L1..L4 at x of the plane (mu, nu) of k written out in `leaves`
below and TA(A) = (A - A^dag)/2 minus its trace/3 (traceless anti-hermitian
part).  TA is self-adjoint for Re Tr, so
    Re(zeta^dag T eta) = -kappa csw / 4 sum_{x,k} Re Tr(Q_k(x) Lambda_k(x)),
    Lambda_k(x) = TA(sum_{s,t} (i sigma_k)_{st} eta_t(x) zeta_s(x)^dag),
and a link occurring as A U B in a leaf adds U B Lambda A to its force, as
A U^dag B adds U A^dag Lambda^dag B^dag.

Pinned: the reference's own md_force_block returns zero in the build here
(its FieldUtils::field_oprod gives a zero field), so the pin is the
reference's clover OPERATOR: tests/golden holds central finite differences of
Re(zeta^dag D_clover eta) computed by the compiled reference
(tests/golden/make_golden.py), which this restatement and the GPU force meet
to the differences' own accuracy.
"""
import numpy as np

# i sigma_{mu nu} of Dirac_Clover::isigma_{23,31,12,41,42,43}
# (dirac_clover.cpp:221-329), with the planes of Bx,By,Bz,Ex,Ey,Ez
# (set_csw, dirac_clover.cpp:139-162)
PAIRS = [(1, 2), (2, 0), (0, 1), (3, 0), (3, 1), (3, 2)]


def _sigma():
    I = 1j
    S = np.zeros((6, 4, 4), complex)
    S[0][0][1] = I; S[0][1][0] = I; S[0][2][3] = I; S[0][3][2] = I
    S[1][0][1] = 1; S[1][1][0] = -1; S[1][2][3] = 1; S[1][3][2] = -1
    S[2][0][0] = I; S[2][1][1] = -I; S[2][2][2] = I; S[2][3][3] = -I
    S[3][0][3] = -I; S[3][1][2] = -I; S[3][2][1] = -I; S[3][3][0] = -I
    S[4][0][3] = -1; S[4][1][2] = 1; S[4][2][1] = -1; S[4][3][0] = 1
    S[5][0][2] = -I; S[5][1][3] = I; S[5][2][0] = -I; S[5][3][1] = I
    return S


SIG = _sigma()


def _unit(mu, k=1):
    o = [0, 0, 0, 0]
    o[mu] = k
    return o


def _add(a, b):
    return [x + y for x, y in zip(a, b)]


def leaves(mu, nu):
    """The four leaves of Q_{mu nu}(x) as (sign, [(direction, offset, dagger)]):
    L1 = U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag, L2 = U_mu(x) Vdn(x)^dag,
    L3 = Vup(x-mu)^dag U_mu(x-mu), L4 = Vdn(x-mu)^dag U_mu(x-mu) (staples of
    Staples::upper / lower)."""
    O = [0, 0, 0, 0]
    m, n, mm, nn = _unit(mu), _unit(nu), _unit(mu, -1), _unit(nu, -1)
    return [
        (+1, [(mu, O, False), (nu, m, False), (mu, n, True), (nu, O, True)]),
        (-1, [(mu, O, False), (nu, _add(m, nn), True), (mu, nn, True), (nu, nn, False)]),
        (+1, [(nu, O, False), (mu, _add(n, mm), True), (nu, mm, True), (mu, mm, False)]),
        (-1, [(nu, nn, True), (mu, _add(mm, nn), True), (nu, _add(mm, nn), False), (mu, mm, False)]),
    ]


def _dag(A):
    return np.conj(np.swapaxes(A, -1, -2))


def _ta(A):
    ah = 0.5 * (A - _dag(A))
    return ah - (np.trace(ah, axis1=-2, axis2=-1) / 3.0)[..., None, None] * np.eye(3)


def clover_block_force(L, u, mass, csw, eta, zeta):
    """The clover term's part of Dirac_Clover::md_force(eta, zeta), Format_G."""
    Lx, Ly, Lz, Lt = [int(v) for v in L]
    V = Lx * Ly * Lz * Lt
    shape = (Lt, Lz, Ly, Lx)
    ax = {0: 3, 1: 2, 2: 1, 3: 0}
    Ua = np.asarray(u, np.float64).reshape(4, V, 3, 3, 2)
    U = (Ua[..., 0] + 1j * Ua[..., 1]).reshape(4, *shape, 3, 3)

    def spin(f):
        F = np.asarray(f, np.float64).reshape(V, 4, 3, 2)
        return (F[..., 0] + 1j * F[..., 1]).reshape(*shape, 4, 3)

    def shift(A, off):  # A(x + off)
        for mu in range(4):
            if off[mu]:
                A = np.roll(A, -off[mu], axis=ax[mu])
        return A

    def factor(f):
        d, o, dg = f
        A = shift(U[d], o)
        return _dag(A) if dg else A

    e, z = spin(eta), spin(zeta)
    eye = np.broadcast_to(np.eye(3), U[0].shape)
    F = np.zeros_like(U)
    for k, (mu, nu) in enumerate(PAIRS):
        lam = _ta(np.einsum("st,...tb,...sa->...ba", SIG[k], e, np.conj(z)))
        for sign, fs in leaves(mu, nu):
            mats = [factor(f) for f in fs]
            for i, (d, o, dg) in enumerate(fs):
                A = eye.copy()
                for j in range(i):
                    A = A @ mats[j]
                B = eye.copy()
                for j in range(i + 1, 4):
                    B = B @ mats[j]
                Ui = shift(U[d], o)
                C = Ui @ _dag(A) @ _dag(lam) @ _dag(B) if dg else Ui @ B @ lam @ A
                F[d] += sign * shift(C, [-v for v in o])  # link (d, x + o)
    F *= -(0.5 / (4.0 + mass)) * csw / 4.0
    F = F.reshape(4, V, 3, 3)
    return np.stack([F.real, F.imag], -1).ravel()


def clover_md_force(L, u, mass, csw, eta, zeta, port):
    """Dirac_Clover::md_force(eta, zeta): the Wilson force (the port's
    restatement of Dirac_Wilson::md_force) plus the clover block's."""
    return port.md_force(L, u, mass, False, eta, zeta) + clover_block_force(L, u, mass, csw, eta, zeta)


def operator_derivative(apply, u, eta, zeta, x, mu, X, h=1e-5):
    """Central difference of Re(zeta^dag D(U_mu(x) -> (1 + e X) U_mu(x)) eta),
    D given as apply(u, eta) on Format_G / Format_F arrays."""
    V = len(u) // 72
    Ua = np.asarray(u, np.float64).reshape(4, V, 3, 3, 2)
    Uc = Ua[..., 0] + 1j * Ua[..., 1]
    cz = np.asarray(zeta)[0::2] + 1j * np.asarray(zeta)[1::2]

    def s(eps):
        W = Uc.copy()
        W[mu, x] = (np.eye(3) + eps * X) @ W[mu, x]
        De = apply(np.stack([W.real, W.imag], -1).ravel(), eta)
        return float(np.vdot(cz, De[0::2] + 1j * De[1::2]).real)

    return (s(h) - s(-h)) / (2 * h)
