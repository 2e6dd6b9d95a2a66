"""Parity at the benchmark configurations themselves, against the reference.

Configuration 1 (8^3x16, full-lattice Wilson, eps = 0.2, kappa = 0.12, one
complex-Gaussian source): the mult and mult_dag against the reference's
Dirac_Wilson::mult (dirac_wilson.cpp:28-36) and the CG solution on D^dag D,
FP64 and mixed precision, against the reference's Solver_CG::solve
(solver_CG.cpp:29-80) -- both run by the compiled reference in a child
process (tests/refproc.py).

Configuration 2 (24^3x48, eps = 0.2 field followed by a random SU(3) gauge
transformation, csw = 1.0, kappa = 0.12): the full clover operator
(dirac_clover.cpp:334-353) and the e/o Wilson Schur operator
(dirac_wilson_EvenOdd.hpp:80-92) in FP64 and FP32 against the reference; the
e/o clover Schur operator, which has no reference counterpart, through the
block identity D [v_e, -A_oo^-1 D_oe v_e] = [M v_e, 0] with D the reference's
own full clover operator; and one clover solve at 16^3x32 against the
oracle's CG solution.

Where the compiled reference is absent the C restatement (oracle/port, pinned
to the reference by tests/test_oracle_golden.py) stands in for it.
"""
import numpy as np
import pytest

import iroiro_b200 as ib
import refproc
from conftest import TOL_FP32, TOL_FP64, TOL_RES, TOL_SOL, rel

pytestmark = pytest.mark.gpu

KAPPA = 0.12
MASS = 0.5 / KAPPA - 4.0
CSW = 1.0
WILSON_FULL, WILSON_EO, CLOVER_FULL = 0, 1, 2


def _eo_sites(L):
    V = int(np.prod(L))
    hs = np.arange(V // 2)
    row = hs // (L[0] // 2)
    y = row % L[1]
    z = (row // L[1]) % L[2]
    t = row // (L[1] * L[2])
    return 2 * hs + ((y + z + t) & 1), 2 * hs + ((y + z + t + 1) & 1)


def _reference(L, arrays, jobs, port):
    """The compiled reference when present, else the C restatement."""
    if refproc.available():
        return refproc.run(L, arrays, jobs)
    out = []
    for j in jobs:
        u = arrays[j.get("u", "u")]
        if j["op"] == "wilson_full":
            out.append({"x": port.wilson_full(L, u, j["mass"], j.get("dag", 0), arrays[j["f"]])})
        elif j["op"] == "wilson_eo":
            out.append({"x": port.wilson_eo(L, u, j["mass"], j.get("dag", 0), arrays[j["f"]])})
        elif j["op"] == "clover_full":
            out.append({"x": port.clover_full(L, u, j["mass"], j["csw"], j.get("dag", 0),
                                              arrays[j["f"]])})
        else:
            x, it, diff = port.cg(L, u, j["kind"], j["mass"], j.get("csw", 0.0), arrays[j["b"]],
                                  j["prec"], j["maxiter"])
            out.append({"x": x, "iterations": it, "diff": diff})
    return out


# ---- configuration 1 ------------------------------------------------------------------

L1 = [8, 8, 8, 16]


@pytest.fixture(scope="module")
def c1(port):
    V = int(np.prod(L1))
    u = ib.synth_gauge(L1, 0.2, 1001)
    b = ib.synth_gaussian(V, 1002)
    jobs = [{"op": "wilson_full", "mass": MASS, "dag": 0, "f": "b"},
            {"op": "wilson_full", "mass": MASS, "dag": 1, "f": "b"},
            {"op": "cg", "kind": WILSON_FULL, "mass": MASS, "b": "b", "prec": 1e-20,
             "maxiter": 5000}]
    r = _reference(L1, {"u": u, "b": b}, jobs, port)
    ctx = ib.context(L1)
    ctx.upload_gauge(u, force=True)
    return {"u": u, "b": b, "ctx": ctx, "mult": [r[0]["x"], r[1]["x"]], "cg": r[2]}


@pytest.mark.parametrize("dag", [0, 1])
@pytest.mark.parametrize("prec,tol", [(ib.PREC_DOUBLE, TOL_FP64), (ib.PREC_SINGLE, TOL_FP32)])
def test_c1_wilson_mult_vs_reference(c1, dag, prec, tol):
    got = c1["ctx"].apply(ib.OP_WILSON_FULL, MASS, 0.0, dag, c1["b"], prec=prec)
    assert rel(got, c1["mult"][dag]) < tol


@pytest.mark.parametrize("inner", ["double", "single", "half"])
def test_c1_cg_solution_vs_reference(c1, inner):
    D = ib.Dirac_Wilson(MASS, c1["u"], ctx=c1["ctx"])
    x = np.empty_like(c1["b"])
    out = ib.Solver_CG(1e-20, 5000, ib.Fopr_DdagD(D), inner=inner).solve(x, c1["b"])
    assert out.diff < TOL_RES
    assert rel(x, c1["cg"]["x"]) < TOL_SOL
    if inner == "double":
        assert abs(out.Iterations - int(c1["cg"]["iterations"])) <= 2


# ---- configuration 2 ------------------------------------------------------------------

L2 = [24, 24, 24, 48]


@pytest.fixture(scope="module")
def c2(port):
    V = int(np.prod(L2))
    u = ib.synth_gauge(L2, 0.2, 2001, gauge_transform=True)
    f = ib.synth_gaussian(V, 2002)
    h = ib.synth_gaussian(V // 2, 2003)
    ctx = ib.context(L2)
    ctx.upload_gauge(u, force=True)
    # the e/o clover Schur operator's full-lattice witness [v_e, -A_oo^-1 D_oe v_e]
    es, os_ = _eo_sites(L2)
    w = -ctx.apply(ib.OP_CLOVER_HOP_OE_INV, MASS, CSW, 0, h)
    wit = np.zeros((V, 24))
    wit[es] = h.reshape(-1, 24)
    wit[os_] = w.reshape(-1, 24)
    jobs = [{"op": "clover_full", "mass": MASS, "csw": CSW, "dag": 0, "f": "f"},
            {"op": "clover_full", "mass": MASS, "csw": CSW, "dag": 1, "f": "f"},
            {"op": "wilson_eo", "mass": MASS, "dag": 0, "f": "h"},
            {"op": "wilson_eo", "mass": MASS, "dag": 1, "f": "h"},
            {"op": "clover_full", "mass": MASS, "csw": CSW, "dag": 0, "f": "wit"}]
    r = _reference(L2, {"u": u, "f": f, "h": h, "wit": wit.ravel()}, jobs, port)
    return {"u": u, "f": f, "h": h, "ctx": ctx, "clover": [r[0]["x"], r[1]["x"]],
            "wilson_eo": [r[2]["x"], r[3]["x"]], "witness": r[4]["x"].reshape(V, 24),
            "es": es, "os": os_}


@pytest.mark.parametrize("dag", [0, 1])
@pytest.mark.parametrize("prec,tol", [(ib.PREC_DOUBLE, TOL_FP64), (ib.PREC_SINGLE, TOL_FP32)])
def test_c2_clover_full_vs_reference(c2, dag, prec, tol):
    got = c2["ctx"].apply(ib.OP_CLOVER_FULL, MASS, CSW, dag, c2["f"], prec=prec)
    assert rel(got, c2["clover"][dag]) < tol


@pytest.mark.parametrize("dag", [0, 1])
@pytest.mark.parametrize("prec,tol", [(ib.PREC_DOUBLE, TOL_FP64), (ib.PREC_SINGLE, TOL_FP32)])
def test_c2_wilson_schur_vs_reference(c2, dag, prec, tol):
    got = c2["ctx"].apply(ib.OP_WILSON_SCHUR_EE, MASS, 0.0, dag, c2["h"], prec=prec)
    assert rel(got, c2["wilson_eo"][dag]) < tol


@pytest.mark.parametrize("prec,tol", [(ib.PREC_DOUBLE, TOL_FP64), (ib.PREC_SINGLE, TOL_FP32)])
def test_c2_clover_schur_through_reference_operator(c2, prec, tol):
    """M v_e equals the even half of the reference's clover operator on the
    witness, whose odd half the reference maps to zero."""
    got = c2["ctx"].apply(ib.OP_CLOVER_SCHUR_EE, MASS, CSW, 0, c2["h"], prec=prec)
    want = c2["witness"][c2["es"]].ravel()
    assert rel(got, want) < tol
    assert np.linalg.norm(c2["witness"][c2["os"]]) < TOL_FP64 * np.linalg.norm(c2["h"])


L3 = [16, 16, 16, 32]


@pytest.fixture(scope="module")
def clover_solve(port):
    V = int(np.prod(L3))
    u = ib.synth_gauge(L3, 0.2, 3001, gauge_transform=True)
    b = ib.synth_gaussian(V, 3002)
    x, it, diff = port.cg(L3, u, CLOVER_FULL, MASS, CSW, b, 1e-20, 5000)
    ctx = ib.context(L3)
    ctx.upload_gauge(u, force=True)
    return {"u": u, "b": b, "x": x, "iterations": it, "diff": diff, "ctx": ctx}


@pytest.mark.parametrize("inner", ["double", "half"])
def test_clover_cg_16c32_vs_oracle(clover_solve, inner):
    """Full-lattice clover CG on D^dag D: the solution within 1e-8 of the
    oracle's, at a 1e-10 FP64 true residual."""
    s = clover_solve
    D = ib.Dirac_Clover(ib.Dirac_Wilson(MASS, s["u"], ctx=s["ctx"]), CSW, s["u"], ctx=s["ctx"])
    x = np.empty_like(s["b"])
    out = ib.Solver_CG(1e-20, 5000, ib.Fopr_DdagD(D), inner=inner).solve(x, s["b"])
    assert s["diff"] < TOL_RES
    assert out.diff < TOL_RES
    assert rel(x, s["x"]) < TOL_SOL
    if inner == "double":
        assert abs(out.Iterations - s["iterations"]) <= 2


def test_clover_eo_inverter_16c32_vs_oracle(clover_solve, port):
    """The e/o clover inverter (CG on the Schur complement, odd sites rebuilt,
    Inverter_WilsonLike::invert, eoUtils.cpp:43-81) on the source c = D x,
    where x is the oracle's CG solution and D the oracle's full clover
    operator: its solution is x itself."""
    s = clover_solve
    c = port.clover_full(L3, s["u"], MASS, CSW, 0, s["x"])
    D = ib.Dirac_Clover_EvenOdd(MASS, CSW, s["u"], ctx=s["ctx"])
    inv = ib.Inverter_WilsonLike(D, ib.Solver_CG(1e-20, 5000, ib.Fopr_DdagD(D)))
    y = np.empty_like(c)
    out = inv.invert(y, c)
    assert out.diff < TOL_RES
    assert rel(y, s["x"]) < TOL_SOL
