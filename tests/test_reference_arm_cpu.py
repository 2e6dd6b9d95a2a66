"""bench.py --impl reference on the host: one JSON line with the GPU arm's
metric, unit and config object, the reference's own CPU implementation timed
(cpu_baseline of kind "reference"), no host<->device bytes, and no use of the
product library (the arm's inputs come from the oracle's generator)."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

import bench
import oracle

ROOT = Path(__file__).resolve().parent.parent


@pytest.mark.skipif(not oracle.ref_available(), reason="the reference library is not built")
def test_reference_arm_line():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    # the arm runs in this child through bench.py's own entry point; then the
    # child reports whether the product library was ever mapped
    code = (
        "import runpy, sys\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '3']\n"
        "rc = 0\n"
        "try:\n"
        "    runpy.run_path('bench.py', run_name='__main__')\n"
        "except SystemExit as e:\n"
        "    rc = e.code or 0\n"
        "print('PRODUCT_MAPPED', 'libiroiro_b200' in open('/proc/self/maps').read())\n"
        "sys.exit(rc)\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1])
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == "GB/s" and line["higher_is_better"]
    assert line["config"] == bench.config_for(1)
    assert line["steps"] == 1 and line["warmup"] == 3 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert "PRODUCT_MAPPED False" in r.stdout
