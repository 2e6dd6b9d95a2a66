"""CG, mixed-precision CG, block CG and multishift CG on the GPU against the
reference's solutions (golden fixtures) and the FP64 true residual."""
import numpy as np
import pytest

import iroiro_b200 as ib
from conftest import TOL_RES, TOL_SOL, load_golden, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g():
    d = load_golden("4x4x4x4")
    d["ctx"] = ib.context(d["L"])
    d["ctx"].upload_gauge(d["u"], force=True)
    return d


def _dirac(g, name):
    m, u, c = float(g["mass"]), g["u"], g["ctx"]
    if name == "wilson_full":
        return ib.Dirac_Wilson(m, u, ctx=c), g["f_full"]
    if name == "wilson_eo":
        return ib.Dirac_Wilson_EvenOdd(m, u, ctx=c), g["f_half"]
    return ib.Dirac_Clover(ib.Dirac_Wilson(m, u, ctx=c), float(g["csw"]), u, ctx=c), g["f_full"]


@pytest.mark.parametrize("name", ["wilson_full", "wilson_eo", "clover_full"])
@pytest.mark.parametrize("graph", [False, True])
def test_cg_fp64_vs_reference(g, name, graph):
    D, b = _dirac(g, name)
    slv = ib.Solver_CG(1e-20, 5000, ib.Fopr_DdagD(D), use_graph=graph)
    x = np.empty_like(b)
    out = slv.solve(x, b)
    assert abs(out.Iterations - int(g[f"cg_{name}_iters"])) <= 2
    assert out.diff < TOL_RES
    assert rel(x, g[f"cg_{name}_x"]) < TOL_SOL


@pytest.mark.parametrize("name", ["wilson_full", "wilson_eo", "clover_full"])
@pytest.mark.parametrize("inner", ["single", "half"])
def test_cg_mixed_precision(g, name, inner):
    D, b = _dirac(g, name)
    slv = ib.Solver_CG(1e-20, 5000, ib.Fopr_DdagD(D), inner=inner)
    x = np.empty_like(b)
    out = slv.solve(x, b)
    assert out.diff < TOL_RES
    assert out.reliable_updates >= 1
    assert rel(x, g[f"cg_{name}_x"]) < TOL_SOL


def test_cg_not_converged_raises(g):
    D, b = _dirac(g, "wilson_eo")
    with pytest.raises(ib.ConvergenceError):
        ib.Solver_CG(1e-20, 5, ib.Fopr_DdagD(D)).solve(np.empty_like(b), b)


@pytest.mark.parametrize("inner", ["double", "single", "half"])
def test_block_cg_12_rhs(inner):
    """12 point sources at one site solved together, each to 1e-10."""
    L = [8, 8, 8, 8]
    V = int(np.prod(L))
    c = ib.context(L)
    u = ib.synth_gauge(L, 0.2, 71, True)
    c.upload_gauge(u, force=True)
    D = ib.Dirac_Wilson_EvenOdd(0.5 / 0.12 - 4, u, ctx=c)
    src = ib.synth_point_sources(V // 2, 123)
    slv = ib.Solver_CG(1e-20, 5000, ib.Fopr_DdagD(D), inner=inner)
    x, outs, rc = slv.solve_many(src.ravel(), 12)
    assert rc == ib.OK
    x = x.reshape(12, -1)
    ref = ib.Solver_CG(1e-20, 5000, ib.Fopr_DdagD(D))
    for r in (0, 5, 11):
        assert outs[r].diff < TOL_RES
        x1 = np.empty(V * 12)
        ref.solve(x1, src[r])
        assert rel(x[r], x1) < TOL_SOL


def _eo_sites(L):
    V = int(np.prod(L)); Vh = V // 2
    hs = np.arange(Vh); row = hs // (L[0] // 2)
    y = row % L[1]; z = (row // L[1]) % L[2]; t = row // (L[1] * L[2])
    return 2 * hs + ((y + z + t) & 1), 2 * hs + ((y + z + t + 1) & 1)


def test_clover_schur_is_schur_complement_of_reference_operator(g):
    """D [v_e, w_o] = [M v_e, 0] for w_o = kappa A_oo^-1 H_oe v_e, where D is
    the full clover operator (checked against the reference) and M the e/o
    clover Schur operator."""
    m, csw, u, c, L = float(g["mass"]), float(g["csw"]), g["u"], g["ctx"], g["L"]
    V = int(np.prod(L))
    es, os_ = _eo_sites(L)
    v = g["f_half"]
    w = -c.apply(ib.OP_CLOVER_HOP_OE_INV, m, csw, 0, v)
    full = np.zeros((V, 24))
    full[es] = v.reshape(-1, 24)
    full[os_] = w.reshape(-1, 24)
    out = c.apply(ib.OP_CLOVER_FULL, m, csw, 0, full.ravel()).reshape(V, 24)
    Mv = c.apply(ib.OP_CLOVER_SCHUR_EE, m, csw, 0, v)
    assert rel(out[es].ravel(), Mv) < 1e-13
    assert np.linalg.norm(out[os_]) < 1e-13 * np.linalg.norm(v)


@pytest.mark.parametrize("inner", ["double", "single", "half"])
def test_clover_schur_cg(g, inner):
    """CG on the e/o clover Schur operator recovers a known solution."""
    m, csw, u, c = float(g["mass"]), float(g["csw"]), g["u"], g["ctx"]
    Dc = ib.Dirac_Clover_EvenOdd(m, csw, u, ctx=c)
    b = Dc.mult(g["f_half"])
    x = np.empty_like(b)
    out = ib.Solver_CG(1e-20, 5000, ib.Fopr_DdagD(Dc), inner=inner).solve(x, b)
    # (M^dag M) x = b, checked with the operator itself
    assert out.diff < TOL_RES
    assert rel(Dc.mult_dag(Dc.mult(x)), b) < 2 * TOL_RES


@pytest.mark.parametrize("name", ["wilson_full", "wilson_eo"])
def test_multishift_vs_reference(g, name):
    D, b = _dirac(g, name)
    slv = ib.MultiShiftSolver_CG(ib.Fopr_DdagD(D), 1e-20, 5000)
    xs = []
    out = slv.solve(xs, b, g["shifts"])
    assert abs(out.Nconv - int(g[f"ms_{name}_nconv"])) <= 2
    assert out.diff < TOL_RES
    for k in range(len(g["shifts"])):
        assert rel(xs[k], g[f"ms_{name}_x"][k]) < TOL_SOL


@pytest.mark.parametrize("name", ["wilson_full", "wilson_eo"])
@pytest.mark.parametrize("inner", ["single", "half"])
def test_multishift_mixed_vs_reference(g, name, inner):
    """The mixed-precision multishift (FP32 multishift with FP64 recurrences,
    then one block of reliable-update CG refinements, one per shift): every
    shift's solution within 1e-8 of the reference's, every FP64 true
    residual below 1e-10."""
    D, b = _dirac(g, name)
    slv = ib.MultiShiftSolver_CG(ib.Fopr_DdagD(D), 1e-20, 5000, inner=inner)
    xs = []
    out = slv.solve(xs, b, g["shifts"])
    assert out.diff < TOL_RES
    assert out.Nconv > 0
    for k in range(len(g["shifts"])):
        assert rel(xs[k], g[f"ms_{name}_x"][k]) < TOL_SOL


@pytest.mark.parametrize("inner", ["single", "half"])
def test_multishift_mixed_12_shifts_8c8(inner):
    """12 shifts 1e-4..10 at 8^4 on the clover Schur operator: the mixed
    solver's solutions against the FP64 multishift's, and each shifted
    system's residual checked with the operator itself."""
    L = [8, 8, 8, 8]
    V = int(np.prod(L))
    c = ib.context(L)
    u = ib.synth_gauge(L, 0.2, 81, True)
    c.upload_gauge(u, force=True)
    D = ib.Dirac_Clover_EvenOdd(0.5 / 0.12 - 4, 1.0, u, ctx=c)
    b = ib.synth_gaussian(V // 2, 82)
    shifts = [1e-4 * (1e5) ** (k / 11) for k in range(12)]
    x64, xm = [], []
    ib.MultiShiftSolver_CG(ib.Fopr_DdagD(D), 1e-20, 5000).solve(x64, b, shifts)
    out = ib.MultiShiftSolver_CG(ib.Fopr_DdagD(D), 1e-20, 5000, inner=inner).solve(xm, b, shifts)
    assert out.diff < TOL_RES
    for k, s in enumerate(shifts):
        assert rel(xm[k], x64[k]) < TOL_SOL, k
        r = D.mult_dag(D.mult(xm[k])) + s * xm[k] - b
        assert np.linalg.norm(r) < 1.01 * TOL_RES * np.linalg.norm(b), k


def test_multishift_windows_vs_oracle(port):
    """12 shifts 1e-4..10 at 8^3x16 on the e/o Wilson operator, to
    |r|^2/|b|^2 < 1e-22: more than 32 iterations, so the FP64 solver folds
    several windows of residuals into the shifts' x and p.  The iteration
    count equals the oracle's (MultiShiftSolver_CG restated), and every
    shift's solution agrees with the oracle's to 1e-10."""
    import oracle
    L = [8, 8, 8, 16]
    V = int(np.prod(L))
    mass = 0.5 / 0.12 - 4
    u = ib.synth_gauge(L, 0.2, 91, True)
    c = ib.context(L)
    c.upload_gauge(u, force=True)
    D = ib.Dirac_Wilson_EvenOdd(mass, u, ctx=c)
    b = ib.synth_gaussian(V // 2, 92)
    shifts = [1e-4 * (1e5) ** (k / 11) for k in range(12)]
    xs = []
    out = ib.MultiShiftSolver_CG(ib.Fopr_DdagD(D), 1e-22, 5000).solve(xs, b, shifts)
    xo, nco, _ = port.multishift(L, u, oracle.WILSON_EO, mass, 0.0, b, shifts, 1e-22, 5000)
    assert out.Nconv == nco and nco > 64
    for k in range(len(shifts)):
        assert rel(xs[k], xo[k]) < 1e-10, k


def test_multishift_stopped_mid_window_vs_oracle(port):
    """Stopped by the iteration limit (45, inside the second window of
    residuals): the solver reports IRO_NOT_CONVERGED and returns every
    shift's x after 45 iterations, as the oracle does."""
    import ctypes
    import oracle
    L = [8, 8, 8, 16]
    V = int(np.prod(L))
    mass = 0.5 / 0.12 - 4
    u = ib.synth_gauge(L, 0.2, 93, True)
    c = ib.context(L)
    c.upload_gauge(u, force=True)
    b = ib.synth_gaussian(V // 2, 94)
    shifts = np.array([1e-4 * (1e5) ** (k / 11) for k in range(12)])
    x = np.empty(b.size * shifts.size)
    o = ib.SolverOut()
    nconv = ctypes.c_int(0)
    rc = c._lib.iro_multishift_cg_solve_mixed(c.h, ib.OP_WILSON_SCHUR_EE, mass, 0.0, ib._ptr(b),
                                              shifts.size, ib._ptr(shifts), ib._ptr(x), 1e-22, 45,
                                              ib.PREC_DOUBLE, ctypes.byref(o), ctypes.byref(nconv))
    assert rc == ib.NOT_CONVERGED and nconv.value == -1
    xo, nco, _ = port.multishift(L, u, oracle.WILSON_EO, mass, 0.0, b, shifts, 1e-22, 45)
    assert nco == -1
    x = x.reshape(shifts.size, -1)
    for k in range(shifts.size):
        assert rel(x[k], xo[k]) < 1e-10, k
