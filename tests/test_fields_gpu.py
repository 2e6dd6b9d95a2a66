"""Device-resident fields: boundary round trip and the Field reductions
(Field::norm, include/field.h:74-78; Field::operator*, lib/Fields/field.inl:58-62)."""
import numpy as np
import pytest

import iroiro_b200 as ib
from conftest import TOL_FP16, TOL_FP32, TOL_FP64

pytestmark = pytest.mark.gpu

L = [8, 8, 8, 16]
V = int(np.prod(L))


@pytest.fixture(scope="module")
def ctx():
    return ib.context(L)


@pytest.mark.parametrize("subset", [0, 1, 2])
def test_round_trip_is_bit_exact_in_fp64(ctx, subset):
    n = (24 if subset == 2 else 12) * V
    f = ib.synth_gaussian(n // 24, 81 + subset)
    d = ib.DeviceField(ctx, subset, "double").upload(f)
    assert np.array_equal(d.download(), f)


@pytest.mark.parametrize("prec,tol", [("double", TOL_FP64), ("single", TOL_FP32), ("half", TOL_FP16)])
def test_norm_and_dot(ctx, prec, tol):
    nrhs = 3
    a = ib.synth_gaussian(V * nrhs, 91)
    b = ib.synth_gaussian(V * nrhs, 92)
    da = ib.DeviceField(ctx, 2, prec, nrhs).upload(a)
    db = ib.DeviceField(ctx, 2, prec, nrhs).upload(b)
    A, B = a.reshape(nrhs, -1), b.reshape(nrhs, -1)
    assert np.allclose(da.norm(), np.linalg.norm(A, axis=1), rtol=tol, atol=0)
    ref = np.einsum("ri,ri->r", A, B)
    assert np.all(np.abs(da.dot(db) - ref) <= tol * np.linalg.norm(A, axis=1) * np.linalg.norm(B, axis=1))
