"""MD forces on the GPU: the Wilson ones against the reference's md_force
(golden fixtures, including the 6x2x4x4 lattice whose two y-neighbours
coincide) and the oracle on a larger lattice; the clover one
(Dirac_Clover::md_force) against derivatives of the reference's clover operator
and the oracle's restatement."""
import numpy as np
import pytest

import iroiro_b200 as ib
from conftest import TOL_FP64, load_golden, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["4x4x4x4", "6x2x4x4"])
def test_md_force_vs_reference(name):
    g = load_golden(name)
    L, u, m = [int(v) for v in g["L"]], g["u"], float(g["mass"])
    ctx = ib.Context(L, 0)
    Dw = ib.Dirac_Wilson(m, u, ctx=ctx)
    assert rel(Dw.md_force(g["force_eta"], g["force_zeta"]), g["force_full"]) < TOL_FP64
    De = ib.Dirac_Wilson_EvenOdd(m, u, ctx=ctx)
    assert rel(De.md_force(g["force_eta_half"], g["force_zeta_half"]), g["force_eo"]) < TOL_FP64


def test_md_force_vs_oracle_8x8x8x16(port):
    L = [8, 8, 8, 16]
    V = int(np.prod(L))
    u = ib.synth_gauge(L, 0.2, 77, gauge_transform=True)
    m = 0.5 / 0.124 - 4
    ctx = ib.Context(L, 0)
    e, z = ib.synth_gaussian(V, 78), ib.synth_gaussian(V, 79)
    F = ib.Dirac_Wilson(m, u, ctx=ctx).md_force(e, z)
    assert rel(F, port.md_force(L, u, m, False, e, z)) < TOL_FP64
    eh, zh = ib.synth_gaussian(V // 2, 80), ib.synth_gaussian(V // 2, 81)
    Fe = ib.Dirac_Wilson_EvenOdd(m, u, ctx=ctx).md_force(eh, zh)
    assert rel(Fe, port.md_force(L, u, m, True, eh, zh)) < TOL_FP64


def test_md_force_is_the_derivative_of_the_operator():
    """Re Tr(X F_mu(x)) = d/de Re(zeta^dag D(U_mu(x) -> (1 + e X) U_mu(x)) eta)
    for the full Wilson operator, by central differences on the GPU operator
    itself (the perturbed links are not SU(3): FP64 full-matrix storage)."""
    L = [4, 4, 4, 8]
    V = int(np.prod(L))
    u = ib.synth_gauge(L, 0.2, 91, gauge_transform=True)
    m = 0.5 / 0.12 - 4
    ctx = ib.Context(L, 0)
    e, z = ib.synth_gaussian(V, 92), ib.synth_gaussian(V, 93)
    F = ib.Dirac_Wilson(m, u, ctx=ctx).md_force(e, z).reshape(4, V, 3, 3, 2)
    rng = np.random.default_rng(94)
    cz = z[0::2] + 1j * z[1::2]
    for _ in range(3):
        x, mu = int(rng.integers(V)), int(rng.integers(4))
        X = rng.standard_normal((3, 3)) + 1j * rng.standard_normal((3, 3))

        def f(eps):
            U = u.reshape(4, V, 3, 3, 2)
            Uc = (U[..., 0] + 1j * U[..., 1]).copy()
            Uc[mu, x] = (np.eye(3) + eps * X) @ Uc[mu, x]
            up = np.stack([Uc.real, Uc.imag], -1).ravel()
            ctx.upload_gauge(up, force=True)
            De = ctx.apply(ib.OP_WILSON_FULL, m, 0.0, 0, e)
            return float(np.vdot(cz, De[0::2] + 1j * De[1::2]).real)

        h = 1e-5
        fd = (f(h) - f(-h)) / (2 * h)
        an = float(np.trace(X @ (F[mu, x, ..., 0] + 1j * F[mu, x, ..., 1])).real)
        assert abs(fd - an) < 1e-6 * max(1.0, abs(an)), (fd, an)


@pytest.mark.parametrize("name", ["4x4x4x4", "6x2x4x4"])
def test_clover_md_force_vs_reference_operator(name, port):
    """Dirac_Clover::md_force: the derivative of the reference's own clover
    operator (golden central differences, ~1e-10), and the oracle's
    restatement to FP64 round-off."""
    from oracle.clover_force import clover_md_force
    g = load_golden(name)
    L, u, m, csw = [int(v) for v in g["L"]], g["u"], float(g["mass"]), float(g["csw"])
    V = int(np.prod(L))
    ctx = ib.Context(L, 0)
    Dw = ib.Dirac_Wilson(m, u, ctx=ctx)
    D = ib.Dirac_Clover(Dw, csw, u, ctx=ctx)
    F = D.md_force(g["cforce_eta"], g["cforce_zeta"])
    ref = clover_md_force(L, u, m, csw, g["cforce_eta"], g["cforce_zeta"], port)
    assert rel(F, ref) < TOL_FP64
    Fc = F.reshape(4, V, 3, 3, 2)
    Fc = Fc[..., 0] + 1j * Fc[..., 1]
    X = g["cforce_X"][..., 0] + 1j * g["cforce_X"][..., 1]
    for k, fd in enumerate(g["cforce_fd"]):
        an = float(np.trace(X[k] @ Fc[g["cforce_dirs"][k], g["cforce_sites"][k]]).real)
        assert abs(an - fd) < 1e-8 * max(1.0, abs(fd)), (k, an, fd)


def test_clover_md_force_vs_oracle_8x8x8x16(port):
    from oracle.clover_force import clover_md_force
    L = [8, 8, 8, 16]
    V = int(np.prod(L))
    u = ib.synth_gauge(L, 0.2, 95, gauge_transform=True)
    m, csw = 0.5 / 0.124 - 4, 1.7
    ctx = ib.Context(L, 0)
    D = ib.Dirac_Clover(ib.Dirac_Wilson(m, u, ctx=ctx), csw, u, ctx=ctx)
    e, z = ib.synth_gaussian(V, 96), ib.synth_gaussian(V, 97)
    assert rel(D.md_force(e, z), clover_md_force(L, u, m, csw, e, z, port)) < TOL_FP64
