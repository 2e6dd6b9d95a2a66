"""The algebra of the device-side GCR cycle (gcr_coef_kernel, gcr_finish_iteration,
gcr_gamma_kernel in csrc/learned.cu), restated in numpy on a small complex
system with a fixed non-Hermitian right preconditioner:

  * one pass gives <w_q, w_j> (q < j), |w_j|^2 and <r, w_j>; beta_q =
    -<w_q, w_j>/|w_q|^2, |w'_j|^2 = |w_j|^2 - sum_q |<w_q, w_j>|^2/|w_q|^2 and
    <r, w'_j> = <r, w_j> (the w_q are orthogonal, r is orthogonal to them);
  * the directions are kept as produced, z'_j = sum_i T[i][j] z_i, and the
    cycle's correction is e = sum_i gamma_i z_i with gamma = T alpha;
  * the iterated |r|^2 drops by |<r, w'_j>|^2/|w'_j|^2 per iteration.

Checked against GCR with the orthogonalised directions formed explicitly:
the same iterates and residual norms, and the solution of the system."""
import numpy as np
import pytest


def _system(n=48, seed=3):
    rng = np.random.default_rng(seed)
    B = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    A = B.conj().T @ B + n * np.eye(n)             # Hermitian positive definite (like D^dag D)
    G = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(2 * n)
    M = (np.eye(n) + 0.3 * G) @ np.linalg.inv(A)   # M A = 1 + 0.3 G: an inexact, non-Hermitian one
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    return A, M, b


def _cycle_device_form(A, M, r, m, delta, thresh=1e-4, second=None):
    """One cycle as the device forms it (the second pass when |w'_j|^2 falls
    below thresh |w_j|^2; the device's threshold is 1e-4); returns (e,
    iterations, iterated |r|^2)."""
    rr_start = rr = np.vdot(r, r).real
    Z, W, nw = [], [], []
    T = np.zeros((m, m), complex)
    alpha = np.zeros(m, complex)
    jdone = 0
    for j in range(m):
        z = M @ r
        w = A @ z
        g = [np.vdot(Wq, w) for Wq in W] + [np.vdot(w, w), np.vdot(r, w)]
        beta = [-g[q] / nw[q] for q in range(j)]
        nwj = g[j].real - sum(abs(g[q]) ** 2 / nw[q] for q in range(j))
        rw = g[j + 1]
        w = w + sum(beta[q] * W[q] for q in range(j))   # the update kernel's first half
        if not nwj > thresh * g[j].real:
            # w_j nearly in the span of the w_q: the second pass forms both
            # from the orthogonalised vector
            nwj, rw = np.vdot(w, w).real, np.vdot(r, w)
            if second is not None:
                second[0] += 1
        a = np.conj(rw) / nwj
        r = r - a * w                                   # ... and its second
        T[j, j] = 1.0
        for q in range(j):
            for i in range(q + 1):
                T[i, j] += beta[q] * T[i, q]
        alpha[j] = a
        Z.append(z)
        W.append(w)
        nw.append(nwj)
        rr = rr - abs(rw) ** 2 / nwj
        jdone = j + 1
        if rr < delta ** 2 * rr_start:
            break
    gamma = T[:jdone, :jdone] @ alpha[:jdone]
    e = sum(gamma[i] * Z[i] for i in range(jdone))
    return e, jdone, rr


def _cycle_explicit(A, M, r, m, delta):
    """Textbook flexible GCR: z'_j and w'_j orthogonalised explicitly, x and r
    updated every iteration."""
    rr_start = np.vdot(r, r).real
    Zp, Wp = [], []
    e = np.zeros_like(r)
    jdone = 0
    for j in range(m):
        z = M @ r
        w = A @ z
        for zq, wq in zip(Zp, Wp):
            bq = -np.vdot(wq, w) / np.vdot(wq, wq)
            z = z + bq * zq
            w = w + bq * wq
        a = np.vdot(w, r) / np.vdot(w, w)
        e = e + a * z
        r = r - a * w
        Zp.append(z)
        Wp.append(w)
        jdone = j + 1
        if np.vdot(r, r).real < delta ** 2 * rr_start:
            break
    return e, jdone, np.vdot(r, r).real


@pytest.mark.parametrize("thresh", [1e-4, 1.01])
def test_cycle_matches_explicit_gcr(thresh):
    A, M, b = _system()
    second = [0]
    for m, delta in ((8, 0.03), (16, 1e-3), (4, 0.1)):
        e1, j1, rr1 = _cycle_device_form(A, M, b.copy(), m, delta, thresh, second)
        e2, j2, rr2 = _cycle_explicit(A, M, b.copy(), m, delta)
        assert j1 == j2
        assert np.linalg.norm(e1 - e2) < 1e-10 * np.linalg.norm(e2)
        # the iterated |r|^2 equals the true one of the cycle's correction
        rtrue = b - A @ e1
        assert abs(rr1 - np.vdot(rtrue, rtrue).real) < 1e-8 * np.vdot(b, b).real
        assert abs(rr1 - rr2) < 1e-8 * np.vdot(b, b).real
    # above 1 every iteration takes the second pass (|w'_j| <= |w_j|); with
    # this preconditioner the device's threshold never sends one there
    assert (second[0] > 0) == (thresh > 1.0)


def test_restarted_solve_reaches_the_solution():
    A, M, b = _system(seed=5)
    x = np.zeros_like(b)
    r = b.copy()
    for _ in range(50):
        e, _, _ = _cycle_device_form(A, M, r, 8, 0.03)
        x = x + e
        r = b - A @ x                     # the restart's residual (FP64 on the device)
        if np.vdot(r, r).real < 1e-24 * np.vdot(b, b).real:
            break
    assert np.linalg.norm(x - np.linalg.solve(A, b)) < 1e-10 * np.linalg.norm(x)
