"""LeapfrogKdk on host arrays with this library computing the forces
(core/src/integrator.rs:38-78 driving solvers/src/lbvh.rs): in FP64 the trajectory is
bit-identical to the oracle's integrator, including sizes whose accelerations come back
in several ragged copy chunks, and a lone particle only drifts."""

import numpy as np
import pytest

import galaxy_b200 as gb

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [4097, 140_001])  # one chunk; three chunks, the last ragged
def test_kdk_step_host_f64_bit_exact_vs_oracle(oracle, n):
    st = gb.ic.plummer(n, 21)
    pinned = gb.PinnedState.from_state(st)
    h = gb.GpuLbvh(1.0, 0.01, 0.5, precision="f64")
    primed = False
    for _ in range(3):
        primed = h.kdk_step_host(pinned, 1e-3, primed)
    assert primed
    pos, vel = st.pos.copy(), st.vel.copy()
    kdk = oracle.LeapfrogKdkLbvh(1.0, 0.01, 0.5, threads=8)
    kdk.step_many(pos, vel, st.mass, 1e-3, 3)
    assert np.array_equal(np.asarray(pinned.pos), pos)
    assert np.array_equal(np.asarray(pinned.vel), vel)
    assert np.array_equal(np.asarray(pinned.acc), kdk.acc)


def test_kdk_step_host_f32_matches_resident_step():
    # The host-driven step and the resident step compute the same forces.
    st = gb.ic.plummer(70_000, 22)
    pinned = gb.PinnedState.from_state(st)
    h = gb.GpuLbvh(1.0, 0.01, 0.5)
    primed = False
    for _ in range(2):
        primed = h.kdk_step_host(pinned, 5e-4, primed)
    r = gb.GpuResidentLeapfrog(1.0, 0.01, 0.5)
    r.upload(st)
    r.step_many(5e-4, 2)
    snap = r.snapshot()
    assert np.array_equal(np.asarray(pinned.pos), snap.pos)
    assert np.array_equal(np.asarray(pinned.vel), snap.vel)


def test_kdk_step_host_lone_particle_drifts():
    st = gb.State(pos=np.array([[1.0, 2.0, 3.0]]), vel=np.array([[0.5, -0.25, 0.125]]), mass=np.array([2.0]))
    pinned = gb.PinnedState.from_state(st)
    h = gb.GpuLbvh(1.0, 0.01, 0.5)
    primed = h.kdk_step_host(pinned, 0.1, False)
    primed = h.kdk_step_host(pinned, 0.1, primed)
    assert np.array_equal(np.asarray(pinned.vel), st.vel)
    assert np.allclose(np.asarray(pinned.pos), st.pos + 0.2 * st.vel, rtol=0, atol=1e-15)
    assert not np.asarray(pinned.acc).any()
