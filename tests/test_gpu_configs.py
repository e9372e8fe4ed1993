"""The correctness criteria on the named configurations at test size: RMS force error
of the FP32 walk and of the reference (the FP64 walk, the reference's arithmetic bit
for bit) against the FP64 direct sum, and energy / angular-momentum drift of an FP32
run matching the reference's over the same steps."""

import numpy as np
import pytest

import galaxy_b200 as gb

pytestmark = pytest.mark.gpu


def _rms(a, ref):
    e = np.linalg.norm(a - ref, axis=1) / np.linalg.norm(ref, axis=1)
    return float(np.sqrt(np.mean(e * e)))


def test_plummer_config_force_errors():
    """N = 16,384 Plummer (seed 0), eps 0.01, theta 0.5: monopole FP32 equals the
    reference's error against the direct sum; quadrupole nodes reduce it."""
    st = gb.ic.plummer(16_384, 0)
    exact = gb.GpuLbvh(1.0, 0.01, 0.5).direct_sum_f64(st.pos, st.mass)
    mono = gb.GpuLbvh(1.0, 0.01, 0.5).accelerations(st)
    ref = gb.GpuLbvh(1.0, 0.01, 0.5, precision="f64").accelerations(st)
    quad = gb.GpuLbvh(1.0, 0.01, 0.5, multipole="quad").accelerations(st)
    e_mono, e_ref, e_quad = _rms(mono, exact), _rms(ref, exact), _rms(quad, exact)
    assert abs(e_mono - e_ref) <= 1e-3 * e_ref
    assert e_ref < 0.02  # the reference's own finite-theta bound (solvers/tests/lbvh.rs)
    assert e_quad < 0.5 * e_mono


@pytest.mark.parametrize("workload", ["plummer", "collision"])
def test_drift_matches_reference(workload):
    if workload == "plummer":
        st, eps, dt, steps = gb.ic.plummer(16_384, 0), 0.01, 1e-3, 100
    else:
        st, eps, dt, steps = gb.ic.collision(65_536, 5, mass_ratio=3.0), 0.02, 5e-4, 100
    out = {}
    for prec in ("f32", "f64"):
        r = gb.GpuResidentLeapfrog(1.0, eps, 0.5, precision=prec)
        r.upload(st)
        d0 = r.diagnostics(True)
        r.step_many(dt, steps)
        d1 = r.diagnostics(True)
        out[prec] = ((d1["total"] - d0["total"]) / abs(d0["total"]),
                     np.linalg.norm(d1["angular_momentum"] - d0["angular_momentum"])
                     / np.linalg.norm(d0["angular_momentum"]))
    (e32, l32), (e64, l64) = out["f32"], out["f64"]
    assert abs(e32 - e64) <= 1e-3 * abs(e64) + 1e-10, out
    assert abs(l32 - l64) <= 1e-3 * abs(l64) + 1e-10, out
