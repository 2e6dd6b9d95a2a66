"""The device-side bounded wait of the tensor-core kernels: a wait on an
mbarrier that nothing arrives at runs out after its time limit, the host
gets IRO_TIMEOUT, and the context keeps working."""
import ctypes

import numpy as np
import pytest

import iroiro_b200 as ib
from conftest import TOL_FP64, load_golden, rel

pytestmark = pytest.mark.gpu


def test_wait_runs_out_and_context_stays_usable(port):
    g = load_golden("4x4x4x4")
    c = ib.context(g["L"])
    c.upload_gauge(g["u"], force=True)
    waited = ctypes.c_double(0.0)
    for limit in (20.0, 50.0):
        rc = c._lib.iro_selftest_bounded_wait(c.h, limit, ctypes.byref(waited))
        assert rc == ib.TIMEOUT
        assert limit <= waited.value < limit + 200.0
    # the context and the device still work: an operator against the oracle
    m = float(g["mass"])
    f = g["f_half"]
    assert rel(c.apply(ib.OP_WILSON_SCHUR_EE, m, 0.0, 0, f),
               port.wilson_eo(g["L"], g["u"], m, 0, f)) < TOL_FP64


def test_wait_limit_is_checked():
    g = load_golden("4x4x4x4")
    c = ib.context(g["L"])
    waited = ctypes.c_double(0.0)
    for bad in (0.0, -1.0, 1001.0):
        assert c._lib.iro_selftest_bounded_wait(c.h, bad, ctypes.byref(waited)) == ib.BAD_ARG
