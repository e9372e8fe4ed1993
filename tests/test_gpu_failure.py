"""Failure detection without a GPU fault: a device-side bounded wait that runs out turns
into a status the host reads, the context stays usable, and bad inputs (NaN positions,
out-of-range indices) give statuses or NaN results, never a hang."""

import ctypes as C

import numpy as np
import pytest

import galaxy_b200 as gb
from galaxy_b200 import _lib

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_and_reports():
    word = C.c_uint32(0)
    rc = _lib.lib().gx_selftest_bounded_wait(-1, 2000, C.byref(word))
    assert rc == -6 and word.value & 1  # GX_ERR_DEVICE_CHECK, the wait-ran-out bit
    # the context is still usable: a force evaluation after it is exact
    st = gb.ic.plummer(3000, 8)
    a = gb.GpuLbvh(1.0, 0.01, 0.5, precision="f64").accelerations(st)
    from oracle import oracle

    assert np.array_equal(a, oracle.lbvh_accelerations(st.pos, st.mass, 1.0, 0.01, 0.5))


def test_nan_input_does_not_hang_and_handle_recovers():
    st = gb.ic.plummer(5000, 9)
    bad = st.pos.copy()
    bad[123] = np.nan
    s = gb.GpuLbvh(1.0, 0.01, 0.5)
    try:
        out = s.accelerations(bad, mass=st.mass)
        assert np.isnan(out[123]).any() or np.isfinite(out).all()
    except gb.GxError as e:
        assert e.code == -6  # a device check may trip; either way the call returns
    good = s.accelerations(st)
    ref = gb.GpuLbvh(1.0, 0.01, 0.5).accelerations(st)
    assert np.array_equal(good, ref)


def test_resident_nan_step_returns():
    st = gb.ic.plummer(4000, 10)
    st.vel[7] = np.inf
    r = gb.GpuResidentLeapfrog(1.0, 0.01, 0.5)
    r.upload(st)
    try:
        r.step_many(1e-3, 3)
    except gb.GxError as e:
        assert e.code == -6
    r2 = gb.GpuResidentLeapfrog(1.0, 0.01, 0.5)
    r2.upload(gb.ic.plummer(4000, 10))
    r2.step_many(1e-3, 3)
    assert np.isfinite(r2.snapshot().pos).all()
