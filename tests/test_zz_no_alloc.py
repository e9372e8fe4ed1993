"""gx_sort_noalloc: the radix sort for callers that may not allocate device memory.

Callers such as an application that owns every device buffer through its own pool,
or a real-time loop that must not allocate after start-up, pass their own device
buffers for the input codes and the outputs; the entry point keeps its working
memory in a static device array of the library. This test hands it device buffers
(allocated here by torch, as such a caller's pool would) and checks two calls in a
row -- of different sizes, so stale scratch from the first would show in the
second -- against the existing allocating entry point gx_stage_sort and against the
oracle's restatement of the reference's stable sort, bit for bit (the sort is integer
work). It runs last so that a failure here leaves every other
test already run, and it passes alone in a fresh process as well."""

import ctypes

import numpy as np
import pytest

import galaxy_b200 as gb

pytestmark = pytest.mark.gpu


def _noalloc_sort(codes):
    import torch

    L = gb._lib.lib()
    n = codes.shape[0]
    d_codes = torch.from_numpy(codes.view(np.int32).copy()).to("cuda")
    d_sorted = torch.empty(n, dtype=torch.int32, device="cuda")
    d_order = torch.empty(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = L.gx_sort_noalloc(ctypes.c_void_p(d_codes.data_ptr()), ctypes.c_void_p(d_sorted.data_ptr()),
                           ctypes.c_void_p(d_order.data_ptr()), n, None)
    assert rc == 0, L.gx_last_error(None)
    return d_order.cpu().numpy().view(np.uint32), d_sorted.cpu().numpy().view(np.uint32)


def test_noalloc_sort_matches_allocating_sort_on_two_calls():
    from oracle import oracle

    inputs = [oracle.fixture_random_codes(5, 700_001),
              ((np.arange(1 << 20) % 3) << 28).astype(np.uint32)]  # the maximum size, heavy ties
    for codes in inputs:
        order, sorted_codes = _noalloc_sort(codes)
        ref_order, ref_sorted = gb.stage_sort(codes)
        assert np.array_equal(order, ref_order)
        assert np.array_equal(sorted_codes, ref_sorted)
        # and the reference's own stable sort by (code, index) (solvers/src/lbvh.rs:143-147)
        oracle_order = oracle.reference_sort(codes)
        assert np.array_equal(order, oracle_order)
        assert np.array_equal(sorted_codes, codes[oracle_order])


def test_noalloc_sort_rejects_oversize():
    L = gb._lib.lib()
    n = (1 << 20) + 1
    rc = L.gx_sort_noalloc(ctypes.c_void_p(16), ctypes.c_void_p(16), ctypes.c_void_p(16), n, None)
    assert rc == -8  # GX_ERR_CAPACITY, before touching any memory
    assert b"GX_NOALLOC_MAX_KEYS" in L.gx_last_error(None)
