"""The C restatement of the hot path against the reference's own outputs.

The golden fixtures were produced by the reference's classes compiled from
its sources (tests/golden/make_golden.py); this pins the oracle that the GPU
parity tests use at sizes beyond the fixtures."""
import numpy as np
import pytest

from conftest import TOL_FP64, TOL_SOL, rel

PAIRS = [(1, 2), (2, 0), (0, 1), (3, 0), (3, 1), (3, 2)]


@pytest.mark.parametrize("dag", [0, 1])
def test_wilson_ops(port, golden, dag):
    g = golden
    L, u, m = g["L"], g["u"], float(g["mass"])
    assert rel(port.wilson_full(L, u, m, dag, g["f_full"]), g[f"wilson_full_{dag}"]) < TOL_FP64
    assert rel(port.wilson_hop(L, u, m, 0, dag, g["f_half"]), g[f"hop_eo_{dag}"]) < TOL_FP64
    assert rel(port.wilson_hop(L, u, m, 1, dag, g["f_half"]), g[f"hop_oe_{dag}"]) < TOL_FP64
    assert rel(port.wilson_eo(L, u, m, dag, g["f_half"]), g[f"wilson_eo_{dag}"]) < TOL_FP64


def test_field_strength(port, golden):
    g = golden
    for mu, nu in PAIRS:
        assert rel(port.field_strength(g["L"], g["u"], mu, nu), g[f"F_{mu}{nu}"]) < TOL_FP64


@pytest.mark.parametrize("dag", [0, 1])
def test_clover(port, golden, dag):
    g = golden
    out = port.clover_full(g["L"], g["u"], float(g["mass"]), float(g["csw"]), dag, g["f_full"])
    assert rel(out, g[f"clover_full_{dag}"]) < TOL_FP64


def test_gamma5_involution(port, golden):
    f = golden["f_full"]
    assert np.array_equal(port.gamma5(port.gamma5(f)), f)


@pytest.mark.parametrize("name,op,src", [("wilson_full", 0, "f_full"), ("wilson_eo", 1, "f_half"),
                                         ("clover_full", 2, "f_full")])
def test_cg(port, golden_full, name, op, src):
    g = golden_full
    x, it, diff = port.cg(g["L"], g["u"], op, float(g["mass"]), float(g["csw"]), g[src], 1e-20, 5000)
    assert it == int(g[f"cg_{name}_iters"])
    assert rel(x, g[f"cg_{name}_x"]) < TOL_SOL
    assert abs(diff - float(g[f"cg_{name}_diff"])) < 5e-2 * float(g[f"cg_{name}_diff"])


@pytest.mark.parametrize("name,op,src", [("wilson_full", 0, "f_full"), ("wilson_eo", 1, "f_half")])
def test_multishift(port, golden_full, name, op, src):
    g = golden_full
    x, nc, diff = port.multishift(g["L"], g["u"], op, float(g["mass"]), 0.0, g[src], g["shifts"],
                                  1e-20, 5000)
    assert nc == int(g[f"ms_{name}_nconv"])
    for k in range(len(g["shifts"])):
        assert rel(x[k], g[f"ms_{name}_x"][k]) < TOL_SOL
    assert abs(diff - float(g[f"ms_{name}_diff"])) < 5e-2 * float(g[f"ms_{name}_diff"])


def test_eo_invert(port, golden_full):
    """Inverter_WilsonLike::invert (eoUtils.cpp:43-81) of the Gaussian source
    and of the 12 point sources of Qprop_EvenOdd::calc."""
    g = golden_full
    L, u, m = g["L"], g["u"], float(g["mass"])
    x, it, diff = port.eo_invert(L, u, m, g["f_full"], 1e-20, 5000)
    assert rel(x, g["eoinv_x"]) < TOL_SOL
    site = int(g["qprop_site"])
    V = int(np.prod(L))
    for k in (0, 5, 11):
        s, c = divmod(k, 3)
        src = np.zeros(24 * V)
        src[24 * site + 2 * (c + 3 * s)] = 1.0
        xk, _, _ = port.eo_invert(L, u, m, src, 1e-20, 5000)
        assert rel(xk, g["qprop_x"][k]) < TOL_SOL


@pytest.mark.parametrize("name,op,src", [("wilson_full", 0, "f_full"), ("wilson_eo", 1, "f_half")])
def test_rational(port, golden_full, name, op, src):
    """RationalSolver_CG::solve reconstruction c0 b + sum r_i x_i."""
    g = golden_full
    x, nc, diff = port.rational(g["L"], g["u"], op, float(g["mass"]), float(g["csw"]), g[src],
                                g["rat_poles"], g["rat_res"], float(g["rat_c0"]), 1e-20, 5000)
    assert nc == int(g[f"rat_{name}_nconv"])
    assert rel(x, g[f"rat_{name}_x"]) < TOL_SOL


def test_md_force(port, golden):
    """Dirac_Wilson::md_force and Dirac_Wilson_EvenOdd::md_force."""
    g = golden
    L, u, m = g["L"], g["u"], float(g["mass"])
    assert rel(port.md_force(L, u, m, False, g["force_eta"], g["force_zeta"]), g["force_full"]) < TOL_FP64
    assert rel(port.md_force(L, u, m, True, g["force_eta_half"], g["force_zeta_half"]),
               g["force_eo"]) < TOL_FP64


def test_clover_force_restatement_is_the_operator_derivative(golden, port):
    """The oracle's Dirac_Clover::md_force meets the central differences of the
    reference's own clover operator (the reference's force block returns zero in
    the build here, so its operator is the pin)."""
    from oracle.clover_force import clover_md_force
    g = golden
    L = [int(v) for v in g["L"]]
    V = int(np.prod(L))
    F = clover_md_force(L, g["u"], float(g["mass"]), float(g["csw"]), g["cforce_eta"],
                        g["cforce_zeta"], port).reshape(4, V, 3, 3, 2)
    F = F[..., 0] + 1j * F[..., 1]
    X = g["cforce_X"][..., 0] + 1j * g["cforce_X"][..., 1]
    for k, fd in enumerate(g["cforce_fd"]):
        an = float(np.trace(X[k] @ F[g["cforce_dirs"][k], g["cforce_sites"][k]]).real)
        assert abs(an - fd) < 1e-8 * max(1.0, abs(fd)), (k, an, fd)
