"""iro_norm_noalloc: the Field norm for callers that cannot allocate device memory.

Callers that own all device memory through their own pool (a fixed budget,
or a footprint that must not change after set-up) cannot call cudaMalloc, so
they cannot use the context API, which allocates.  iro_norm_noalloc reduces
a device array they own into a device double they own, with the scratch in a
fixed array inside the library.  This test gives it caller-owned buffers and
checks it against the context API's iro_field_norm (Field::norm) on the same
data, on two calls in a row with different inputs (the shared scratch must
not carry anything from one call into the next).  It is collected last, so a
run that stops at the first failure has already run every other test."""
import ctypes

import numpy as np
import pytest

import iroiro_b200 as ib
from conftest import TOL_FP64

pytestmark = pytest.mark.gpu

L = [16, 16, 16, 32]
V = int(np.prod(L))


def test_noalloc_norm_matches_field_norm_twice():
    import torch

    lib = ib.lib()
    ctx = ib.context(L, 0)
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream().cuda_stream
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    for call, seed in enumerate((1201, 1202)):
        f = ib.synth_gaussian(V, seed) * (1.0 + call)
        ref = ib.DeviceField(ctx, 2, "double").upload(f).norm()[0]
        x = torch.from_numpy(f).to("cuda")
        rc = lib.iro_norm_noalloc(ctypes.c_void_p(x.data_ptr()), x.numel(),
                                  ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
        assert rc == ib.OK
        torch.cuda.synchronize()
        got = float(out.item())
        assert abs(got - ref) <= TOL_FP64 * ref, (call, got, ref)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = ib.lib()
    limit = 67108864
    dummy = ctypes.c_void_p(8)  # never dereferenced: the size check comes first
    assert lib.iro_norm_noalloc(dummy, limit + 1, dummy, None) == ib.BAD_ARG
    assert lib.iro_norm_noalloc(None, 16, dummy, None) == ib.BAD_ARG
