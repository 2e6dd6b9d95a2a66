"""Wilson MD forces on the GPU against the reference's md_force (golden
fixtures, including the 6x2x4x4 lattice whose two y-neighbours coincide) and
against the oracle on a larger lattice."""
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
