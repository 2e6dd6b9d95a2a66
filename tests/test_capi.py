"""The C-ABI library loads without a GPU, exports every symbol its headers
declare, and rejects bad arguments before touching the device."""
import ctypes
import re

import numpy as np
import pytest

from conftest import ROOT


def declared_symbols():
    names = set()
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(iro_\w+)\s*\(", text))
    return sorted(names)


def test_headers_declare_entry_points():
    names = declared_symbols()
    assert "iro_ctx_create" in names and "iro_cg_solve" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    import iroiro_b200 as ib
    lib = ib.lib()
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_bad_lattice_rejected_without_device():
    import iroiro_b200 as ib
    lib = ib.lib()
    h = ctypes.c_void_p()
    for L in ([4, 4, 4, 3], [0, 4, 4, 4], [4, 4, 4, 1]):
        assert lib.iro_ctx_create((ctypes.c_int * 4)(*L), 0, ctypes.byref(h)) == ib.BAD_ARG


def test_element_count_bound_rejected_without_device():
    # the device index arithmetic is 32-bit: a context holds fewer than 2^31
    # elements per parity at 16 right-hand sides (Vh * 16 < 2^31)
    import iroiro_b200 as ib
    lib = ib.lib()
    h = ctypes.c_void_p()
    L = [128, 128, 128, 128]  # Vh * 16 = 2^31
    assert lib.iro_ctx_create((ctypes.c_int * 4)(*L), 0, ctypes.byref(h)) == ib.BAD_ARG


def test_chunk_address_formula():
    # chunk 0 of element i of a blocked array with N 16-byte chunks per element
    # (warp blocks of 32 elements) is at unit (i >> 5) * 32 N + (i & 31); the
    # device computes it as (i & ~31) (N - 1) + i from a 32-bit i (at most
    # 2 * Vh * 16 - 1 < 2^32 for a full-lattice field) with a 64-bit product
    edge = [0, 1, 31, 32, 33, 2**31 - 1, 2**31, 2**31 + 31, 2**32 - 33, 2**32 - 1]
    rng = np.random.default_rng(3)
    idx = np.concatenate([np.array(edge, np.uint64), rng.integers(0, 2**32, 4096, dtype=np.uint64)])
    for n in (3, 6, 9, 12, 18, 36):
        blocked = (idx >> np.uint64(5)) * np.uint64(32 * n) + (idx & np.uint64(31))
        device = (idx & np.uint64(0xFFFFFFE0)) * np.uint64(n - 1) + idx
        assert np.array_equal(blocked, device), n


def test_null_arguments_rejected():
    import iroiro_b200 as ib
    lib = ib.lib()
    assert lib.iro_ctx_destroy(None) == ib.BAD_ARG
    assert lib.iro_synth_gauge(None, 0.2, 1, 0, None) == ib.BAD_ARG
    assert lib.iro_synth_point_sources(16, 16, None) == ib.BAD_ARG
    assert lib.iro_last_error(None) == b"null context"


def test_python_mirror_requires_ddagd():
    import iroiro_b200 as ib

    class FakeD:
        op = ib.OP_WILSON_HOP_EO

    with pytest.raises(ib.IroError):
        ib.Solver_CG(1e-20, 100, object())
    with pytest.raises(ib.IroError):
        ib.Solver_CG(1e-20, 100, ib.Fopr_DdagD(FakeD()))
