"""Wilson and clover operators on the GPU against the reference.

Against the golden fixtures (the reference's own outputs) at every storage
precision, against the C oracle at 8^3x16, and through size-independent
identities at 24^3x48 (gamma5-hermiticity, the even-odd block structure,
multi-RHS = single-RHS, FP32 vs FP64)."""
import numpy as np
import pytest

import iroiro_b200 as ib
from conftest import TOL_FP16, TOL_FP32, TOL_FP64, load_golden, rel

pytestmark = pytest.mark.gpu

PREC_TOL = [("double", TOL_FP64), ("single", TOL_FP32), ("half", TOL_FP16)]
PAIRS = [(1, 2), (2, 0), (0, 1), (3, 0), (3, 1), (3, 2)]


@pytest.fixture(scope="module", params=["4x4x4x4", "6x2x4x4"])
def g(request):
    d = load_golden(request.param)
    d["ctx"] = ib.context(d["L"])
    d["ctx"].upload_gauge(d["u"], force=True)
    return d


@pytest.mark.parametrize("prec,tol", PREC_TOL)
@pytest.mark.parametrize("dag", [0, 1])
def test_wilson_vs_reference(g, prec, tol, dag):
    c, m = g["ctx"], float(g["mass"])
    c.upload_gauge(g["u"])
    assert rel(c.apply(ib.OP_WILSON_FULL, m, 0, dag, g["f_full"], prec), g[f"wilson_full_{dag}"]) < tol
    assert rel(c.apply(ib.OP_WILSON_HOP_EO, m, 0, dag, g["f_half"], prec), g[f"hop_eo_{dag}"]) < tol
    assert rel(c.apply(ib.OP_WILSON_HOP_OE, m, 0, dag, g["f_half"], prec), g[f"hop_oe_{dag}"]) < tol
    assert rel(c.apply(ib.OP_WILSON_SCHUR_EE, m, 0, dag, g["f_half"], prec), g[f"wilson_eo_{dag}"]) < tol


@pytest.mark.parametrize("prec,tol", PREC_TOL)
@pytest.mark.parametrize("dag", [0, 1])
def test_clover_vs_reference(g, prec, tol, dag):
    c, m, csw = g["ctx"], float(g["mass"]), float(g["csw"])
    c.upload_gauge(g["u"])
    out = c.apply(ib.OP_CLOVER_FULL, m, csw, dag, g["f_full"], prec)
    assert rel(out, g[f"clover_full_{dag}"]) < tol


def test_field_strength_vs_reference(g):
    c = g["ctx"]
    c.upload_gauge(g["u"])
    for mu, nu in PAIRS:
        assert rel(c.field_strength(mu, nu), g[f"F_{mu}{nu}"]) < TOL_FP64


def test_gamma5(g):
    c = g["ctx"]
    f = g["f_full"]
    out = c.gamma5(f).reshape(-1, 4, 6)
    ff = f.reshape(-1, 4, 6)
    assert np.array_equal(out[:, 0], ff[:, 2]) and np.array_equal(out[:, 3], ff[:, 1])


def test_python_mirror_classes(g):
    u, m = g["u"], float(g["mass"])
    ctx = g["ctx"]
    D = ib.Dirac_Wilson(m, u, ctx=ctx)
    assert rel(D.mult(g["f_full"]), g["wilson_full_0"]) < TOL_FP64
    E = ib.Dirac_Wilson_EvenOdd(m, u, ctx=ctx)
    assert rel(E.mult_dag(g["f_half"]), g["wilson_eo_1"]) < TOL_FP64
    assert rel(E.mult_eo(g["f_half"]), g["hop_eo_0"]) < TOL_FP64
    assert rel(E.mult_oe_dag(g["f_half"]), g["hop_eo_1"]) < TOL_FP64
    C = ib.Dirac_Clover(D, float(g["csw"]), u, ctx=ctx)
    assert rel(C.mult(g["f_full"]), g["clover_full_0"]) < TOL_FP64


@pytest.mark.parametrize("L", [[8, 8, 8, 16], [4, 6, 2, 8]])
def test_vs_oracle_port(port, L):
    u = ib.synth_gauge(L, 0.25, 31, True)
    V = int(np.prod(L))
    f = ib.synth_gaussian(V, 32)
    h = ib.synth_gaussian(V // 2, 33)
    c = ib.context(L)
    c.upload_gauge(u, force=True)
    m = 0.5 / 0.124 - 4
    for dag in (0, 1):
        assert rel(c.apply(ib.OP_WILSON_FULL, m, 0, dag, f), port.wilson_full(L, u, m, dag, f)) < TOL_FP64
        assert rel(c.apply(ib.OP_WILSON_SCHUR_EE, m, 0, dag, h), port.wilson_eo(L, u, m, dag, h)) < TOL_FP64
        assert rel(c.apply(ib.OP_CLOVER_FULL, m, 1.0, dag, f), port.clover_full(L, u, m, 1.0, dag, f)) < TOL_FP64


@pytest.fixture(scope="module")
def big():
    L = [24, 24, 24, 48]
    V = int(np.prod(L))
    u = ib.synth_gauge(L, 0.2, 41, True)
    c = ib.context(L)
    c.upload_gauge(u, force=True)
    return dict(L=L, V=V, u=u, c=c, m=0.5 / 0.12 - 4, f=ib.synth_gaussian(V, 42),
                g=ib.synth_gaussian(V, 43), h=ib.synth_gaussian(V // 2, 44), k=ib.synth_gaussian(V // 2, 45))


@pytest.mark.parametrize("op,full,csw", [(ib.OP_WILSON_FULL, True, 0.0), (ib.OP_CLOVER_FULL, True, 1.0),
                                         (ib.OP_WILSON_SCHUR_EE, False, 0.0),
                                         (ib.OP_CLOVER_SCHUR_EE, False, 1.0)])
def test_gamma5_hermiticity_24c48(big, op, full, csw):
    """<g, D f> = <D^dag g, f> with D^dag = gamma5 D gamma5."""
    c, m = big["c"], big["m"]
    f, gg = (big["f"], big["g"]) if full else (big["h"], big["k"])
    a = np.dot(gg, c.apply(op, m, csw, 0, f))
    b = np.dot(c.apply(op, m, csw, 1, gg), f)
    assert abs(a - b) < 1e-12 * abs(a)


def test_even_odd_blocks_24c48(big):
    """The full operators restricted to even-site sources reproduce the e/o
    blocks: D [f_e, 0] = [A_ee f_e, -kappa H_oe f_e]."""
    c, m, L, V = big["c"], big["m"], big["L"], big["V"]
    Vh = V // 2
    h = big["h"]
    # scatter the even half field to lexicographic sites: site = 2*hs + ((y+z+t)&1)
    hs = np.arange(Vh)
    row = hs // (L[0] // 2)
    y = row % L[1]; z = (row // L[1]) % L[2]; t = row // (L[1] * L[2])
    esite = 2 * hs + ((y + z + t) & 1)
    osite = 2 * hs + ((y + z + t + 1) & 1)
    full = np.zeros((V, 24))
    full[esite] = h.reshape(Vh, 24)
    out = c.apply(ib.OP_WILSON_FULL, m, 0, 0, full.ravel()).reshape(V, 24)
    assert rel(out[esite].ravel(), h) < TOL_FP64
    assert rel(out[osite].ravel(), c.apply(ib.OP_WILSON_HOP_OE, m, 0, 0, h)) < TOL_FP64


@pytest.mark.parametrize("prec,tol", [("single", TOL_FP32), ("half", TOL_FP16)])
def test_low_precision_24c48(big, prec, tol):
    c, m = big["c"], big["m"]
    for op, f, csw in ((ib.OP_WILSON_SCHUR_EE, big["h"], 0.0), (ib.OP_CLOVER_SCHUR_EE, big["h"], 1.0),
                       (ib.OP_WILSON_FULL, big["f"], 0.0)):
        ref = c.apply(op, m, csw, 0, f, "double")
        assert rel(c.apply(op, m, csw, 0, f, prec), ref) < tol


@pytest.mark.parametrize("prec", ["double", "single", "half"])
def test_multi_rhs_equals_single(prec):
    L = [8, 8, 8, 8]
    V = int(np.prod(L))
    c = ib.context(L)
    c.upload_gauge(ib.synth_gauge(L, 0.2, 51, True), force=True)
    m = 0.1
    fs = np.stack([ib.synth_gaussian(V // 2, 60 + r) for r in range(12)])
    blk = c.apply(ib.OP_CLOVER_SCHUR_EE, m, 1.0, 0, fs.ravel(), prec, nrhs=12).reshape(12, -1)
    for r in range(12):
        one = c.apply(ib.OP_CLOVER_SCHUR_EE, m, 1.0, 0, fs[r], prec)
        if prec == "double":
            # the autotuner may run one shape on reconstructed third link rows
            # and the other on the stored ones: equal to FP64 rounding
            assert rel(blk[r], one) < 1e-13
        else:
            # FP32/FP16 blocks may run two right-hand sides per thread in
            # packed FP32x2 arithmetic: equal to FP32 rounding, not bitwise
            tol = TOL_FP32 if prec == "single" else TOL_FP16
            assert np.linalg.norm(blk[r] - one) < tol * np.linalg.norm(one)


@pytest.mark.parametrize("prec", ["double", "single", "half"])
@pytest.mark.parametrize("nrhs", [2, 4, 16])
@pytest.mark.parametrize("op", [ib.OP_WILSON_FULL, ib.OP_WILSON_SCHUR_EE])
def test_block_sizes_equal_single(prec, nrhs, op):
    """Blocks of 2, 4 and 16 right-hand sides (every kernel variant the
    autotuner tries for them, the shared-memory staged one included) on the
    full and the Schur operator agree with the single-RHS operator."""
    L = [4, 4, 4, 8]
    V = int(np.prod(L))
    n = V if op == ib.OP_WILSON_FULL else V // 2
    c = ib.context(L)
    c.upload_gauge(ib.synth_gauge(L, 0.2, 52, True), force=True)
    m = 0.5 / 0.12 - 4
    fs = np.stack([ib.synth_gaussian(n, 70 + r) for r in range(nrhs)])
    blk = c.apply(op, m, 0.0, 0, fs.ravel(), prec, nrhs=nrhs).reshape(nrhs, -1)
    tol = {"double": 1e-13, "single": TOL_FP32, "half": TOL_FP16}[prec]
    for r in range(nrhs):
        one = c.apply(op, m, 0.0, 0, fs[r], prec)
        assert np.linalg.norm(blk[r] - one) < tol * np.linalg.norm(one)


@pytest.mark.parametrize("prec", ["double", "single", "half"])
@pytest.mark.parametrize("op,csw", [(ib.OP_WILSON_SCHUR_EE, 0.0), (ib.OP_CLOVER_SCHUR_EE, 1.0)])
def test_schur_pinned_overlapped_equals_plain(big, prec, op, csw):
    """The Schur operator between page-locked arrays (chunked copies in both
    directions overlapped with the stencils, 13 chunks at 24^3x48, single
    t-slices among them) gives the
    plain path's result to the bit.  The first call of a shape may tune the
    stencils on the plain path; the calls after it take the overlapped one."""
    import torch
    c, m, h = big["c"], big["m"], big["h"]
    pin_in = torch.empty(h.size, dtype=torch.float64, pin_memory=True).numpy()
    pin_out = torch.empty(h.size, dtype=torch.float64, pin_memory=True).numpy()
    pin_in[:] = h
    for dag in (0, 1):
        ref = c.apply(op, m, csw, dag, h, prec)  # pageable arrays: the plain path
        for _ in range(2):
            pin_out[:] = np.nan
            c.apply(op, m, csw, dag, pin_in, prec, out=pin_out)
            assert np.array_equal(pin_out, ref)
    # in place on one page-locked array: the plain path (the arrays overlap)
    pin_out[:] = h
    c.apply(op, m, csw, 0, pin_out, prec, out=pin_out)
    assert np.array_equal(pin_out, c.apply(op, m, csw, 0, h, prec))


def test_schur_registered_host_memory_overlapped(big):
    """Ordinary host arrays pinned in place with cudaHostRegister (what an
    adapter does with a Field's storage) take the overlapped path too; the
    result equals the plain path's to the bit."""
    import torch
    c, m, h = big["c"], big["m"], big["h"]
    rt = torch.cuda.cudart()
    a = h.copy()
    out = np.empty_like(h)
    for arr in (a, out):
        err = rt.cudaHostRegister(arr.ctypes.data, arr.nbytes, 0)
        assert int(getattr(err, "value", err)) == 0
    try:
        ref = c.apply(ib.OP_WILSON_SCHUR_EE, m, 0.0, 0, h)
        for _ in range(2):
            out[:] = np.nan
            c.apply(ib.OP_WILSON_SCHUR_EE, m, 0.0, 0, a, out=out)
            assert np.array_equal(out, ref)
    finally:
        for arr in (a, out):
            rt.cudaHostUnregister(arr.ctypes.data)


@pytest.mark.parametrize("prec", ["double", "single", "half"])
@pytest.mark.parametrize("op,csw", [(ib.OP_WILSON_FULL, 0.0), (ib.OP_CLOVER_FULL, 1.0)])
def test_full_pinned_overlapped_equals_plain(big, prec, op, csw):
    """The full-lattice operators between page-locked arrays (chunks of
    t-slices, copies overlapped with the stencil) equal the plain path to the
    bit, both dagger settings."""
    import torch
    c, m, f = big["c"], big["m"], big["f"]
    pin_in = torch.empty(f.size, dtype=torch.float64, pin_memory=True).numpy()
    pin_out = torch.empty(f.size, dtype=torch.float64, pin_memory=True).numpy()
    pin_in[:] = f
    for dag in (0, 1):
        ref = c.apply(op, m, csw, dag, f, prec)
        for _ in range(2):
            pin_out[:] = np.nan
            c.apply(op, m, csw, dag, pin_in, prec, out=pin_out)
            assert np.array_equal(pin_out, ref)


@pytest.mark.parametrize("slices", ["1", "5"])
def test_overlapped_chunk_plans_equal_plain(big, slices, monkeypatch):
    """Other chunk plans (IRO_PIPE_SLICES: 48 single-slice chunks; 5-slice
    middle chunks between single-slice ends) give the plain path's result to
    the bit for the Schur and the full-lattice operator."""
    import torch
    monkeypatch.setenv("IRO_PIPE_SLICES", slices)
    c, m = big["c"], big["m"]
    for op, f in ((ib.OP_WILSON_SCHUR_EE, big["h"]), (ib.OP_WILSON_FULL, big["f"])):
        pin_in = torch.empty(f.size, dtype=torch.float64, pin_memory=True).numpy()
        pin_out = torch.empty(f.size, dtype=torch.float64, pin_memory=True).numpy()
        pin_in[:] = f
        ref = c.apply(op, m, 0.0, 0, f)
        for _ in range(2):
            pin_out[:] = np.nan
            c.apply(op, m, 0.0, 0, pin_in, out=pin_out)
            assert np.array_equal(pin_out, ref)
