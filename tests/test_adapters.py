"""The C++ adapter classes (include/iroiro_b200_adapters.hpp) that a maintainer
adds to the reference: they implement its own interfaces (DiracWilsonLike,
DiracWilsonLike_EvenOdd, Solver, MultiShiftSolver; dirac_WilsonLike.hpp:28-82,
solver.hpp:24-30, multiShiftSolver.hpp:14-23) over the C ABI.

CPU: the header compiles against the reference's headers with the flags of
the reference build (oracle/Makefile), and the check library that links it
with the reference's objects and the product library exports its entry
points.  GPU: through that library, in a child process, the adapters and the
reference's own classes run the same computations -- Dirac_Wilson_EvenOdd
mult and mult_dag, Solver_CG on Fopr_DdagD, and the reference's unchanged
Qprop_MultiShift::calc (qprop_MultiShift.cpp:10-31) over the multishift
solver -- and must agree.
"""
import ctypes
import os
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

import refproc
from conftest import TOL_FP64, TOL_RES, TOL_SOL, rel

ROOT = Path(__file__).resolve().parent.parent
REF = Path(os.environ.get("IROIRO_REFERENCE", str(ROOT.parent / "reference")))
MASS = 0.5 / 0.12 - 4.0

needs_tree = pytest.mark.skipif(not (REF / "lib").is_dir(), reason="reference tree absent")


@needs_tree
def test_adapter_header_compiles_against_reference_headers(tmp_path):
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("no g++")
    src = tmp_path / "tu.cpp"
    src.write_text('#include "iroiro_b200_adapters.hpp"\n'
                   '#include "Measurements/FermionicM/qprop_MultiShift.hpp"\n'
                   'void use(const Field* u) {\n'
                   '  Dirac_Wilson_EvenOdd_B200 D(0.1, u);\n'
                   '  Solver_CG_B200 s(1e-20, 100, &D, IRO_PREC_HALF);\n'
                   '  Dirac_Wilson_B200 W(0.1, u);\n'
                   '  MultiShiftSolver_CG_B200 m(&W, 1e-20, 100);\n'
                   '  Qprop_MultiShift q(&W, &m);\n'
                   '  Dirac_Clover_B200 C(0.1, 1.0, u);\n'
                   '  const DiracWilsonLike_EvenOdd* e = &D; const Solver* sp = &s;\n'
                   '  const MultiShiftSolver* mp = &m; (void)e; (void)sp; (void)mp; (void)C;\n'
                   '}\n')
    cmd = [gxx, "-fsyntax-only", "-std=gnu++11", "-w", "-D_GLIBCXX_USE_CXX11_ABI=0",
           "-DHAVE_CONFIG_H", "-I", str(ROOT / "oracle" / "ref"), "-I", str(REF),
           "-I", str(REF / "include"), "-I", str(REF / "lib"), "-I", str(ROOT / "include"), str(src)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


@needs_tree
def test_adapter_check_library_exports():
    if not refproc.adapter_available():
        pytest.skip("oracle/_ref/libadapter_check.so not built (make -C oracle adapter)")
    out = subprocess.run(["nm", "-D", "--defined-only", str(refproc.ADAPTER_LIB)],
                         capture_output=True, text=True).stdout
    for name in ("adapter_eo_mult", "adapter_cg", "adapter_qprop_multishift", "ref_init"):
        assert f" T {name}" in out, name


def _inputs(L, seed):
    import oracle
    P = oracle.port()
    V = int(np.prod(L))
    return P.synth_gauge(L, 0.2, seed, True), P.synth_gaussian(V // 2, seed + 1), \
        P.synth_gaussian(V, seed + 2)


@pytest.mark.gpu
def test_adapters_agree_with_reference_classes():
    if not refproc.adapter_available():
        pytest.skip("oracle/_ref/libadapter_check.so not built here")
    L = [4, 4, 4, 8]
    u, h, f = _inputs(L, 4401)
    shifts = [1e-4 * (1e5) ** (k / 11) for k in range(12)]
    jobs = [{"op": "adapter_eo_mult", "mass": MASS, "dag": 0, "f": "h"},
            {"op": "adapter_eo_mult", "mass": MASS, "dag": 1, "f": "h"},
            {"op": "adapter_cg", "eo": 1, "mass": MASS, "b": "h", "prec": 1e-20, "maxiter": 5000},
            {"op": "adapter_cg", "eo": 0, "mass": MASS, "b": "f", "prec": 1e-20, "maxiter": 5000},
            {"op": "adapter_qprop_multishift", "mass": MASS, "site": [1, 2, 3, 5],
             "shifts": shifts, "prec": 1e-20, "maxiter": 5000}]
    r = refproc.run(L, {"u": u, "h": h, "f": f}, jobs, lib="adapter")
    for k in (0, 1):
        assert rel(r[k]["x"], r[k]["ref"]) < TOL_FP64
    for k in (2, 3):
        diff_b200, diff_ref = r[k]["diff"]
        it_b200, it_ref = r[k]["iterations"]
        assert diff_b200 < TOL_RES and diff_ref < TOL_RES
        assert abs(it_b200 - it_ref) <= 2
        assert rel(r[k]["x"], r[k]["ref"]) < TOL_SOL
    xb = r[4]["x"].reshape(144, -1)
    xr = r[4]["ref"].reshape(144, -1)
    for k in range(144):
        assert rel(xb[k], xr[k]) < TOL_SOL, k
