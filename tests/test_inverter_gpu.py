"""The callers of the solvers on the GPU: the even/odd inverter of the full
operator (Inverter_WilsonLike::invert), Qprop_EvenOdd / Qprop with the 12
point sources as one block, and RationalSolver_CG, against the reference's
outputs (golden fixtures) and, for the clover e/o inverter that the reference
lacks, against the full clover operator and the oracle's full-lattice CG."""
import numpy as np
import pytest

import iroiro_b200 as ib
from conftest import TOL_RES, TOL_SOL, load_golden, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g():
    d = load_golden("4x4x4x4")
    ctx = ib.Context(list(d["L"]), 0)
    ctx.upload_gauge(d["u"], force=True)
    d["ctx"] = ctx
    return d


def _full_residual(ctx, op, m, csw, x, b):
    Dx = ctx.apply(op, m, csw, 0, x)
    return float(np.linalg.norm(Dx - b) / np.linalg.norm(b))


@pytest.mark.parametrize("inner", ["double", "single", "half"])
def test_eo_invert_vs_reference(g, inner):
    m = float(g["mass"])
    D = ib.Dirac_Wilson_EvenOdd(m, g["u"], ctx=g["ctx"])
    inv = ib.Inverter_WilsonLike(D, ib.Solver_CG(1e-20, 5000, ib.Fopr_DdagD(D), inner=inner))
    x = np.empty_like(g["f_full"])
    out = inv.invert(x, g["f_full"])
    assert out.diff < TOL_RES
    assert rel(x, g["eoinv_x"]) < TOL_SOL
    assert _full_residual(g["ctx"], ib.OP_WILSON_FULL, m, 0.0, x, g["f_full"]) < 1e-9


@pytest.mark.parametrize("inner", ["double", "half"])
def test_qprop_evenodd_block_vs_reference(g, inner):
    m = float(g["mass"])
    L = [int(v) for v in g["L"]]
    site = int(g["qprop_site"])
    x0 = site % L[0]
    y0 = (site // L[0]) % L[1]
    z0 = (site // (L[0] * L[1])) % L[2]
    t0 = site // (L[0] * L[1] * L[2])
    D = ib.Dirac_Wilson_EvenOdd(m, g["u"], ctx=g["ctx"])
    qp = ib.Qprop_EvenOdd(D, ib.Solver_CG(1e-20, 5000, ib.Fopr_DdagD(D), inner=inner))
    xs = qp.calc(ib.Source_local([x0, y0, z0, t0], L))
    assert len(xs) == 12
    for k in range(12):
        assert qp.last_outputs[k].diff < TOL_RES
        assert rel(xs[k], g["qprop_x"][k]) < TOL_SOL


@pytest.mark.parametrize("op", ["wilson", "clover"])
def test_qprop_point_sources_on_device_match_host_sources(g, op):
    """iro_qprop_point (the Source_local sources built on the device) against
    the same sources built on the host and passed to iro_eo_invert, at an
    even and an odd site; the one-source overload calc(src, s, c); and a
    caller's output buffer reused by two calls."""
    m, csw = float(g["mass"]), float(g["csw"])
    L = [int(v) for v in g["L"]]
    if op == "wilson":
        D = ib.Dirac_Wilson_EvenOdd(m, g["u"], ctx=g["ctx"])
    else:
        D = ib.Dirac_Clover_EvenOdd(m, csw, g["u"], ctx=g["ctx"])
    qp = ib.Qprop_EvenOdd(D, ib.Solver_CG(1e-24, 5000, ib.Fopr_DdagD(D)))
    for sp in ([1, 2, 3, 0], [2, 2, 3, 0]):  # x + y + z + t even, odd
        src = ib.Source_local(sp, L)
        ref = qp.calc([src.mksrc(s, c) for s in range(4) for c in range(3)])
        buf = np.full((12, 24 * g["ctx"].V), np.nan)
        for _ in range(2):
            xs = qp.calc(src, out=buf)
            for k in range(12):
                assert rel(xs[k], ref[k]) < 1e-12, (sp, k)
                assert np.shares_memory(xs[k], buf)
        one = qp.calc(src, 2, 1)
        assert len(one) == 1 and rel(one[0], ref[7]) < 1e-12


def test_qprop_full_matches_evenodd(g):
    """Qprop on the full operator (D^dag D sol = D^dag src) agrees with the
    e/o propagator of the reference."""
    m = float(g["mass"])
    L = [int(v) for v in g["L"]]
    site = int(g["qprop_site"])
    sp = [site % L[0], (site // L[0]) % L[1], (site // (L[0] * L[1])) % L[2], site // (L[0] * L[1] * L[2])]
    D = ib.Dirac_Wilson(m, g["u"], ctx=g["ctx"])
    qp = ib.Qprop(D, ib.Solver_CG(1e-24, 5000, ib.Fopr_DdagD(D)))
    xs = qp.calc(ib.Source_local(sp, L))
    for k in range(12):
        assert rel(xs[k], g["qprop_x"][k]) < TOL_SOL


def test_qprop_multishift(g):
    """Qprop_MultiShift: per source (s-major) and shift (fastest), D x_m with
    (D^dag D + sigma_m) x_m = src.mksrc(s, c)."""
    m = float(g["mass"])
    L = [int(v) for v in g["L"]]
    ctx = g["ctx"]
    D = ib.Dirac_Wilson(m, g["u"], ctx=ctx)
    shifts = [0.01, 0.3]
    src = ib.Source_local([1, 2, 0, 3], L)
    qp = ib.Qprop_MultiShift(D, ib.MultiShiftSolver_CG(ib.Fopr_DdagD(D), 1e-24, 5000))
    props = qp.calc(src, shifts)
    assert len(props) == 12 * len(shifts) and len(qp.last_outputs) == 12
    for k in (0, 7, 11):
        b = src.mksrc(k // 3, k % 3)
        xs = []
        ib.MultiShiftSolver_CG(ib.Fopr_DdagD(D), 1e-24, 5000).solve(xs, b, shifts)
        for i, sig in enumerate(shifts):
            Ax = ctx.apply(ib.OP_WILSON_FULL, m, 0.0, 1, ctx.apply(ib.OP_WILSON_FULL, m, 0.0, 0, xs[i])) + sig * xs[i]
            assert rel(Ax, b) < 1e-10
            assert rel(props[k * len(shifts) + i], D.mult(xs[i])) < 1e-14


def test_clover_eo_invert_solves_full_clover(g):
    """No e/o clover in the reference: the inverter's solution must solve the
    reference-validated full clover operator and equal the oracle's
    full-lattice CG solution of D^dag D x = D^dag b."""
    import oracle
    m, csw = float(g["mass"]), float(g["csw"])
    L = [int(v) for v in g["L"]]
    D = ib.Dirac_Clover_EvenOdd(m, csw, g["u"], ctx=g["ctx"])
    inv = ib.Inverter_WilsonLike(D, ib.Solver_CG(1e-22, 5000, ib.Fopr_DdagD(D)))
    x = np.empty_like(g["f_full"])
    inv.invert(x, g["f_full"])
    assert _full_residual(g["ctx"], ib.OP_CLOVER_FULL, m, csw, x, g["f_full"]) < 1e-10
    port = oracle.port()
    rhs = port.clover_full(L, g["u"], m, csw, 1, g["f_full"])
    xr, _, _ = port.cg(L, g["u"], oracle.CLOVER_FULL, m, csw, rhs, 1e-24, 5000)
    assert rel(x, xr) < TOL_SOL


@pytest.mark.parametrize("name,src", [("wilson_full", "f_full"), ("wilson_eo", "f_half")])
def test_rational_vs_reference(g, name, src):
    m = float(g["mass"])
    D = ib.Dirac_Wilson(m, g["u"], ctx=g["ctx"]) if name == "wilson_full" else \
        ib.Dirac_Wilson_EvenOdd(m, g["u"], ctx=g["ctx"])
    ms = ib.MultiShiftSolver_CG(ib.Fopr_DdagD(D), 1e-20, 5000)
    ra = ib.RationalApprox(float(g["rat_c0"]), g["rat_res"], g["rat_poles"])
    rs = ib.RationalSolver_CG(ms, ra)
    sol = np.empty_like(g[src])
    out = rs.solve(sol, g[src])
    assert out.Nconv == int(g[f"rat_{name}_nconv"])
    assert rel(sol, g[f"rat_{name}_x"]) < TOL_SOL
    with pytest.raises(ib.IroError):
        ib.RationalSolver_CG(ms).solve(sol, g[src])
