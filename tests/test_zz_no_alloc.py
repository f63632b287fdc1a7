"""The allocation-free entry point gdl_sort_unique_rows_noalloc.

It serves callers that cannot allocate device memory themselves (code that
runs inside another library's memory arena, or a process that handed all of
HBM to a fixed pool up front): they pass their own input and output
buffers, and all scratch comes from one fixed array inside the library.
Here its output is checked, on two calls in a row (the scratch array keeps
the previous call's contents), against the allocating entry points
gdl_relation_load_device + gdl_relation_export on the same input and
against numpy's sorted unique rows (which share no kernel with it), and a
call above the fixed row limit must be refused with a clear error.
Integer output, so the comparison is exact.

This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from gdlog_b200 import Engine, load_library

pytestmark = pytest.mark.gpu

MAX_ROWS = 1 << 17  # the documented limit of the entry point
GDL_E_CAPACITY = 6


def bind(lib):
    f = lib.gdl_sort_unique_rows_noalloc
    f.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.POINTER(C.c_uint64), C.c_void_p]
    f.restype = C.c_int32
    lib.gdl_last_error.argtypes = [C.c_void_p]
    lib.gdl_last_error.restype = C.c_char_p
    return f


def rows_with_duplicates(n, max_value, seed):
    rng = np.random.default_rng(seed)
    r = rng.integers(0, max_value, size=(n, 2), dtype=np.int64)
    r[n // 3: n // 3 + n // 4] = r[: n // 4]  # exact duplicates
    return r


def reference_rows(torch, d_in, n):
    """Sorted unique rows through the allocating entry points."""
    with Engine("gpu") as eng:
        rel = eng.relation("x")
        torch.cuda.synchronize()
        eng.load_device(rel, d_in.data_ptr(), n)
        return rel.rows()


def test_noalloc_matches_load_and_export():
    torch = pytest.importorskip("torch")
    lib = load_library("gpu")
    f = bind(lib)
    cases = [(100_000, 1 << 20, 11), (MAX_ROWS, 1 << 31, 12)]  # two calls in a row
    for n, max_value, seed in cases:
        rows = rows_with_duplicates(n, max_value, seed)
        d_in = torch.from_numpy(rows).cuda()
        d_out = torch.full_like(d_in, -1)
        got_n = C.c_uint64(0)
        torch.cuda.synchronize()
        status = f(d_in.data_ptr(), n, d_out.data_ptr(), C.byref(got_n), None)
        assert status == 0, lib.gdl_last_error(None)
        got = d_out[: got_n.value].cpu().numpy().astype(np.uint64)
        want = reference_rows(torch, d_in, n)
        assert got_n.value == len(want)
        assert np.array_equal(got, want)
        # and independently of the engine's kernels: numpy's lexicographic
        # sorted unique rows
        exact = np.unique(rows.astype(np.uint64), axis=0)
        assert np.array_equal(got, exact)


def test_noalloc_rejects_rows_above_limit():
    torch = pytest.importorskip("torch")
    lib = load_library("gpu")
    f = bind(lib)
    d = torch.zeros((4, 2), dtype=torch.int64, device="cuda")
    got_n = C.c_uint64(7)
    status = f(d.data_ptr(), MAX_ROWS + 1, d.data_ptr(), C.byref(got_n), None)
    assert status == GDL_E_CAPACITY
    assert got_n.value == 0
    assert b"limit" in lib.gdl_last_error(None)
