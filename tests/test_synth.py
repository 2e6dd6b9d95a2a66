"""Synthetic inputs: SU(3) links, seeded determinism, gauge covariance."""
import numpy as np

import iroiro_b200 as ib


def links(u, V):
    a = u.reshape(4, V, 9, 2)
    return (a[..., 0] + 1j * a[..., 1]).reshape(4, V, 3, 3)


def plaquette(u, L):
    V = int(np.prod(L))
    U = links(u, V)
    idx = np.arange(V).reshape(L[::-1]).transpose(3, 2, 1, 0)  # idx[x,y,z,t]
    tot = 0.0
    for mu in range(4):
        for nu in range(mu + 1, 4):
            xm = np.roll(idx, -1, axis=mu).ravel(order="F")
            xn = np.roll(idx, -1, axis=nu).ravel(order="F")
            s = idx.ravel(order="F")
            P = U[mu][s] @ U[nu][xm] @ np.conj(np.swapaxes(U[mu][xn], 1, 2)) @ np.conj(np.swapaxes(U[nu][s], 1, 2))
            tot += np.trace(P, axis1=1, axis2=2).real.sum()
    return tot / (6 * 3 * V)


def test_links_are_su3():
    L = [4, 4, 4, 4]
    V = 256
    for gt in (False, True):
        U = links(ib.synth_gauge(L, 0.25, 7, gt), V).reshape(-1, 3, 3)
        eye = np.eye(3)
        assert np.abs(U @ np.conj(np.swapaxes(U, 1, 2)) - eye).max() < 1e-14
        assert np.abs(np.linalg.det(U) - 1).max() < 1e-14


def test_seeded_and_deterministic():
    L = [4, 4, 4, 4]
    a = ib.synth_gauge(L, 0.2, 3)
    assert np.array_equal(a, ib.synth_gauge(L, 0.2, 3))
    assert not np.array_equal(a, ib.synth_gauge(L, 0.2, 4))
    g = ib.synth_gaussian(100, 9)
    assert np.array_equal(g, ib.synth_gaussian(100, 9))
    assert abs(g.mean()) < 0.1 and abs(g.std() - 1) < 0.1


def test_gauge_transformation_keeps_plaquette():
    L = [4, 4, 4, 6]
    p0 = plaquette(ib.synth_gauge(L, 0.2, 5, False), L)
    p1 = plaquette(ib.synth_gauge(L, 0.2, 5, True), L)
    assert abs(p0 - p1) < 1e-13
    assert 0.5 < p0 < 1.0


def test_point_sources():
    s = ib.synth_point_sources(16, 5)
    assert s.shape == (12, 384)
    for k in range(12):
        nz = np.flatnonzero(s[k])
        assert list(nz) == [24 * 5 + 2 * k] and s[k, nz[0]] == 1.0


def test_oracle_generator_is_bit_identical():
    """The oracle's C generator (oracle/port/synth.c), which the reference arm
    of the benchmark and the reference-side tests use so as not to load the
    product library, gives the same bits as the product's."""
    import oracle
    P = oracle.port()
    for L, gt in (([4, 4, 4, 8], False), ([6, 2, 4, 4], True), ([8, 8, 8, 16], True)):
        assert np.array_equal(P.synth_gauge(L, 0.2, 123, gt), ib.synth_gauge(L, 0.2, 123, gt))
    assert np.array_equal(P.synth_gaussian(1000, 5), ib.synth_gaussian(1000, 5))
    assert np.array_equal(oracle.synth_point_sources(16, 5), ib.synth_point_sources(16, 5))
