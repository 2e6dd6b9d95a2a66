"""Every stencil variant the autotuner may pick, forced one at a time
(IRO_HOP_VARIANT, read once per process, so each variant runs in its own
subprocess): 12-RHS FP32/FP16 operators against the FP64 single-RHS operator,
and a 12-RHS mixed-precision CG whose fused reductions drive the solve.
Variants 4-7 are the two-right-hand-sides-per-thread kernel with four
register caps, 8-9 the same with its neighbours staged through shared memory;
FP64 variants 6-11 are 0-5 on the 18-real links; FP16 10-12 the
mixed-precision kernel (FP16 x FP16 -> FP32 FMAs) on three-row FP16 links,
13-14 the same kernel on the 12-real FP16 links with row 2 rebuilt."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

from conftest import TOL_FP16, TOL_FP32, TOL_RES, TOL_SOL

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent

SCRIPT = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import iroiro_b200 as ib

L = [8, 8, 8, 8]
V = int(np.prod(L))
u = ib.synth_gauge(L, 0.2, 71, gauge_transform=True)
c = ib.Context(L, 0)
c.upload_gauge(u, force=True)
m, csw = 0.5 / 0.12 - 4, 1.0
out = {"ops": {}}
half = [ib.OP_WILSON_SCHUR_EE, ib.OP_CLOVER_SCHUR_EE, ib.OP_CLOVER_HOP_OE_INV, ib.OP_WILSON_HOP_EO]
full = [ib.OP_WILSON_FULL, ib.OP_CLOVER_FULL]
for op in half + full:
    n = V if op in full else V // 2
    fs = np.stack([ib.synth_gaussian(n, 80 + r) for r in range(12)])
    for dag in (0, 1):
        ref = np.stack([c.apply(op, m, csw, dag, fs[r], "double") for r in range(12)])
        for prec in ("single", "half"):
            got = c.apply(op, m, csw, dag, fs.ravel(), prec, nrhs=12).reshape(12, -1)
            err = max(float(np.linalg.norm(got[r] - ref[r]) / np.linalg.norm(ref[r]))
                      for r in range(12))
            out["ops"][f"{op}/{dag}/{prec}"] = err
# 12-RHS mixed-precision CG on the e/o Wilson Schur operator
D = ib.Dirac_Wilson_EvenOdd(m, u, ctx=c)
b = np.stack([ib.synth_gaussian(V // 2, 90 + r) for r in range(12)])
x64, o64, _ = ib.Solver_CG(1e-20, 5000, ib.Fopr_DdagD(D)).solve_many(b.ravel(), 12)
x64 = x64.reshape(12, -1)
for inner in ("single", "half"):
    x, outs, rc = ib.Solver_CG(1e-20, 5000, ib.Fopr_DdagD(D), inner=inner).solve_many(b.ravel(), 12)
    x = x.reshape(12, -1)
    out[f"cg_{inner}"] = {
        "rc": rc, "diff": max(o.diff for o in outs),
        "sol": max(float(np.linalg.norm(x[r] - x64[r]) / np.linalg.norm(x64[r])) for r in range(12)),
        "iters": [o.Iterations for o in outs]}
out["autotune"] = c.autotune_report()
print("RESULT " + json.dumps(out))
"""


@pytest.mark.parametrize("variant", ["0,256", "4,256", "5,128", "6,128", "7,256", "8,128", "9,256", "10,128", "11,256", "12,256",
                                     "13,256", "14,128"])
def test_forced_variant(variant):
    env = dict(os.environ, IRO_HOP_VARIANT=variant)
    r = subprocess.run([sys.executable, "-c", SCRIPT, str(ROOT)], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [l for l in r.stdout.splitlines() if l.startswith("RESULT ")][-1]
    res = json.loads(line[len("RESULT "):])
    v = int(variant.split(",")[0])
    # the forced variant ran: FP64 modulo 6 (12 on an SU(3) field, whose
    # 18-real links are variants 6-11); otherwise modulo 15, a variant the
    # shape lacks (4-9 need an even nrhs, 10-14 FP16) falling back modulo 4
    for t in res["autotune"]:
        if t["prec"] == 0:
            exp = v % (12 if t["recon"] == 12 else 6)
        else:
            w = v % 15
            ok = w < 4 or (w < 10 and t["nrhs"] % 2 == 0) or (w >= 10 and t["prec"] == 2)
            exp = w if ok else w % 4
        assert t["variant"] == exp, t
    for key, err in res["ops"].items():
        tol = TOL_FP32 if key.endswith("single") else TOL_FP16
        assert err < tol, (key, err)
    for inner in ("single", "half"):
        cg = res[f"cg_{inner}"]
        assert cg["rc"] == 0 and cg["diff"] < TOL_RES and cg["sol"] < TOL_SOL, cg
