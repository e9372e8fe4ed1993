"""Host-side checks that need no device: the batch's memory estimate stays linear in
the number of particles and systems (the arena grows only short dimensions)."""

import galaxy_b200 as gb


def test_budget_estimate_is_linear():
    import ctypes

    L = gb._lib.lib()
    # gx_system_bytes needs a batch handle; without a GPU creation fails loudly instead.
    b = ctypes.c_void_p()
    rc = L.gx_batch_create(0, None, ctypes.byref(b))
    if rc != 0:
        assert rc == -3
        return
    out = ctypes.c_size_t()
    assert L.gx_system_bytes(b, 1_000_000, ctypes.byref(out)) == 0
    assert 200e6 < out.value < 1000e6
    L.gx_batch_destroy(b)
