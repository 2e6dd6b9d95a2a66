"""iro_norm_noalloc: the Field norm for callers that cannot allocate device memory.

Callers that own all device memory through their own pool (a fixed budget,
or a footprint that must not change after set-up) cannot call cudaMalloc, so
they cannot use the context API, which allocates.  iro_norm_noalloc reduces
a device array they own into a device double they own, with the scratch in a
fixed array inside the library.  These tests give it caller-owned buffers and
check it against numpy's norm of the same FP64 host array and against the
context API's iro_field_norm (Field::norm), on two calls in a row with
different inputs (the shared scratch must not carry anything from one call
into the next), and on sizes that are not multiples of its 8192-double block
tile, one-block grids included.  The file is collected last, so a run that
stops at the first failure has already run every other test."""
import ctypes

import numpy as np
import pytest

import iroiro_b200 as ib
from conftest import TOL_FP64

pytestmark = pytest.mark.gpu

L = [16, 16, 16, 32]
V = int(np.prod(L))
LIMIT = 67108864  # doubles: the capacity of the fixed scratch


def _noalloc_norm(lib, x, out, stream):
    rc = lib.iro_norm_noalloc(ctypes.c_void_p(x.data_ptr()), x.numel(),
                              ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
    assert rc == ib.OK
    import torch
    torch.cuda.synchronize()
    return float(out.item())


def test_noalloc_norm_matches_numpy_and_field_norm_twice():
    import torch

    lib = ib.lib()
    ctx = ib.context(L, 0)
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream().cuda_stream
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    for call, seed in enumerate((1201, 1202)):
        f = ib.synth_gaussian(V, seed) * (1.0 + call)
        want = float(np.linalg.norm(f))
        field = ib.DeviceField(ctx, 2, "double").upload(f).norm()[0]
        got = _noalloc_norm(lib, torch.from_numpy(f).to("cuda"), out, stream)
        assert abs(got - want) <= TOL_FP64 * want, (call, got, want)
        assert abs(got - field) <= TOL_FP64 * field, (call, got, field)


@pytest.mark.parametrize("n", [1, 8191, 8192, 8193, 3 * 8192 + 17, V * 24 + 5, LIMIT])
def test_noalloc_norm_ragged_sizes(n):
    """Partial tiles (the i < n guard), one-block grids (n <= 8192) and the
    largest size the scratch holds; each size twice in a row."""
    import torch

    lib = ib.lib()
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream().cuda_stream
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    rng = np.random.default_rng(n)
    for call in range(2):
        f = rng.standard_normal(n) * (1.0 + call)
        want = float(np.linalg.norm(f))
        got = _noalloc_norm(lib, torch.from_numpy(f).to("cuda"), out, stream)
        assert abs(got - want) <= TOL_FP64 * want, (n, call, got, want)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = ib.lib()
    dummy = ctypes.c_void_p(8)  # never dereferenced: the size check comes first
    assert lib.iro_norm_noalloc(dummy, LIMIT + 1, dummy, None) == ib.BAD_ARG
    assert lib.iro_norm_noalloc(dummy, 0, dummy, None) == ib.BAD_ARG
    assert lib.iro_norm_noalloc(None, 16, dummy, None) == ib.BAD_ARG
