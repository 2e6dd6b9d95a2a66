"""The ctypes mirrors of the C ABI's structs have the C layout: a small C
program compiled against include/iroiro_b200.h prints every struct's size and
field offsets, which must equal those of the Python structures (a field added
on one side only would shift the others silently)."""
import ctypes
import os
import shutil
import subprocess
import tempfile
from pathlib import Path

import pytest

from iroiro_b200 import CGParams, SolverOut
from iroiro_b200.gaugeconf import GaugeInfo
from iroiro_b200.learned import GCROut, GCRParams

ROOT = Path(__file__).resolve().parent.parent

STRUCTS = [("iro_solver_out", SolverOut), ("iro_cg_params", CGParams),
           ("iro_gcr_params", GCRParams), ("iro_gcr_out", GCROut),
           ("iro_gauge_info", GaugeInfo)]


def _c_layout():
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "iroiro_b200.h"',
             "int main(void) {"]
    for cname, py in STRUCTS:
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "layout.c"), os.path.join(d, "layout")
        Path(src).write_text("\n".join(lines) + "\n")
        subprocess.run([cc, "-std=c99", "-I", str(ROOT / "include"), src, "-o", exe], check=True,
                       capture_output=True, text=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    table = {}
    for line in out.splitlines():
        name, field, value = line.split()
        table[(name, field)] = int(value)
    return table


@pytest.mark.parametrize("cname,py", STRUCTS, ids=[c for c, _ in STRUCTS])
def test_ctypes_struct_matches_c(cname, py):
    table = _c_layout()
    assert ctypes.sizeof(py) == table[(cname, "size")], cname
    for fname, _ in py._fields_:
        assert getattr(py, fname).offset == table[(cname, fname)], (cname, fname)
