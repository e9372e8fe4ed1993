"""Parity at the named configurations' full sizes, against the oracle (the C++
restatement of the reference's Lbvh, solvers/src/lbvh.rs:469-524 and :662-676):

* the two-galaxy collision, 2 x 524,288 particles, 30-bit keys (the reference's tree),
  eps 0.02, theta 0.5: the FP32 walk on 8,192 seeded targets, for every warp grouping;
* the precision study's 4,194,304-particle collision (mass ratio 1:3) at theta 0.3,
  0.5 and 0.7 on a 4,096-target subsample;
* energy and angular-momentum drift of an FP32 resident run of the N = 16,384 Plummer
  sphere against the oracle's own LeapfrogKdk + Lbvh trajectory over 100 steps.

Per-particle relative error |a - a_ref| / |a_ref|: median <= 1e-6 and p99 <= 1e-5 (the
FP32 walk makes every opening decision as the reference does; only its summation
differs)."""

import numpy as np
import pytest

import galaxy_b200 as gb
from oracle import oracle

pytestmark = pytest.mark.gpu


def _check(a, ref):
    e = oracle.per_particle_rel_err(a, ref)
    assert np.median(e) <= 1e-6 and np.percentile(e, 99) <= 1e-5, (np.median(e), np.percentile(e, 99), e.max())


@pytest.fixture(scope="module")
def collision():
    return gb.ic.collision(2 * 524_288, 0, mass_ratio=1.0, pericentre=4.0, incl1_deg=30.0, incl2_deg=60.0)


@pytest.mark.parametrize("group", [0, 8, 16, 32])
def test_collision_full_size_against_oracle(collision, group):
    st = collision
    targets = np.sort(np.random.default_rng(8192).choice(len(st), 8192, replace=False)).astype(np.uint32)
    ref = oracle.lbvh_accelerations_subset(st.pos, st.mass, 1.0, 0.02, 0.5, targets, threads=oracle.max_threads())
    a = gb.GpuLbvh(1.0, 0.02, 0.5, walk_group=group).accelerations(st)
    _check(a[targets], ref)


@pytest.fixture(scope="module")
def precision_collision():
    return gb.ic.collision(4_194_304, 0, mass_ratio=3.0, pericentre=4.0, incl1_deg=30.0, incl2_deg=60.0)


@pytest.mark.parametrize("theta", [0.3, 0.5, 0.7])
def test_precision_config_against_oracle(precision_collision, theta):
    st = precision_collision
    targets = np.sort(np.random.default_rng(4096).choice(len(st), 4096, replace=False)).astype(np.uint32)
    ref = oracle.lbvh_accelerations_subset(st.pos, st.mass, 1.0, 0.02, theta, targets, threads=oracle.max_threads())
    a = gb.GpuLbvh(1.0, 0.02, theta).accelerations(st)
    _check(a[targets], ref)


def test_plummer_drift_against_oracle_trajectory():
    """100 KDK steps of the N = 16,384 Plummer sphere (eps 0.01, theta 0.5, dt 1e-3): the
    FP32 resident run's energy and angular-momentum drift equal the oracle's."""
    st = gb.ic.plummer(16_384, 0)
    eps, dt, steps = 0.01, 1e-3, 100
    threads = oracle.max_threads()

    def energy(pos, vel, mass):
        return (oracle.diagnostics(pos, vel, mass)["kinetic"]
                + oracle.potential_parallel(pos, mass, 1.0, eps, threads=threads))

    p, v = st.pos.copy(), st.vel.copy()
    e0, l0 = energy(p, v, st.mass), oracle.diagnostics(p, v, st.mass)["angular_momentum"]
    oracle.LeapfrogKdkLbvh(1.0, eps, 0.5, threads=threads).step_many(p, v, st.mass, dt, steps)
    de_ref = (energy(p, v, st.mass) - e0) / abs(e0)
    dl_ref = np.linalg.norm(oracle.diagnostics(p, v, st.mass)["angular_momentum"] - l0) / np.linalg.norm(l0)
    r = gb.GpuResidentLeapfrog(1.0, eps, 0.5)
    r.upload(st)
    r.step_many(dt, steps)
    s = r.snapshot()
    de = (energy(s.pos, s.vel, st.mass) - e0) / abs(e0)
    dl = np.linalg.norm(oracle.diagnostics(s.pos, s.vel, st.mass)["angular_momentum"] - l0) / np.linalg.norm(l0)
    assert abs(de - de_ref) <= 1e-3 * abs(de_ref) + 1e-10, (de, de_ref)
    assert abs(dl - dl_ref) <= 1e-3 * abs(dl_ref) + 1e-10, (dl, dl_ref)
    # the trajectories themselves stay within the FP32 parity of the forces
    assert np.max(np.abs(s.pos - p)) <= 1e-6 * np.max(np.abs(p))
