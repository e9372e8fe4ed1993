"""Edge cases of the reference path on the GPU: massless particles (the walk skips a
massless node's subtree, solvers/src/lbvh.rs:476-478; the fold falls back to the box
centre for a massless node's centre of mass, :623-636), a system without any mass,
and the smallest systems."""

import numpy as np
import pytest

import galaxy_b200 as gb

pytestmark = pytest.mark.gpu
G, EPS = 1.0, 0.05


def _with_massless(oracle, seed, n, frac):
    """A cluster where a fraction of the particles are massless, plus a clump of 64
    massless particles (a whole massless subtree)."""
    pos, _, mass = oracle.fixture_cluster(seed, n)
    rng = np.random.default_rng(seed)
    mass = mass.copy()
    mass[rng.random(n) < frac] = 0.0
    clump = rng.normal(0.0, 0.01, (64, 3)) + np.array([2.0, -1.0, 0.5])
    return np.vstack([pos, clump]), np.concatenate([mass, np.zeros(64)])


def _parity(approx, exact):
    from oracle import oracle as o

    e = o.per_particle_rel_err(approx, exact)
    return float(np.median(e)), float(np.percentile(e, 99))


@pytest.mark.parametrize("theta", [0.0, 0.5, 0.7])
def test_f64_bit_exact_with_massless(oracle, theta):
    pos, mass = _with_massless(oracle, 11, 3000, 0.3)
    got = gb.GpuLbvh(G, EPS, theta, precision="f64").accelerations(pos, mass=mass)
    assert np.array_equal(got, oracle.lbvh_accelerations(pos, mass, G, EPS, theta))


@pytest.mark.parametrize("theta", [0.3, 0.5, 0.7])
def test_f32_parity_with_massless(oracle, theta):
    pos, mass = _with_massless(oracle, 12, 4000, 0.3)
    ref = oracle.lbvh_accelerations(pos, mass, G, EPS, theta)
    med, p99 = _parity(gb.GpuLbvh(G, EPS, theta).accelerations(pos, mass=mass), ref)
    assert med <= 1e-6 and p99 <= 1e-5, (med, p99)


def test_aggregation_with_massless(oracle):
    pos, mass = _with_massless(oracle, 13, 2000, 0.5)
    codes = oracle.reference_morton(pos)[1]
    order = oracle.reference_sort(codes)
    sc, sp, sm = codes[order], pos[order], mass[order]
    out = gb.stage_build(sc, sp, sm, gb.GpuLbvh(1.0, 0.05, 0.5))
    left, right, _ = oracle.reference_karras(sc)
    agg = oracle.reference_aggregate(left, right, sp, sm)
    for k in ("aabb_min", "aabb_max", "com", "mass"):
        assert np.array_equal(out[k], agg[k]), k


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_massless_system_feels_no_force(oracle, precision):
    pos, _, _ = oracle.fixture_cluster(14, 1000)
    mass = np.zeros(len(pos))
    got = gb.GpuLbvh(G, EPS, 0.5, precision=precision).accelerations(pos, mass=mass)
    assert np.array_equal(got, np.zeros_like(got))
    assert np.array_equal(oracle.lbvh_accelerations(pos, mass, G, EPS, 0.5), np.zeros_like(got))


@pytest.mark.parametrize("n", [2, 3, 5, 33, 4097])
def test_small_and_ragged_systems(oracle, n):
    pos, _, mass = oracle.fixture_cluster(15 + n, n)
    ref = oracle.lbvh_accelerations(pos, mass, G, EPS, 0.5)
    assert np.array_equal(gb.GpuLbvh(G, EPS, 0.5, precision="f64").accelerations(pos, mass=mass), ref)
    med, p99 = _parity(gb.GpuLbvh(G, EPS, 0.5).accelerations(pos, mass=mass), ref)
    assert med <= 1e-6 and p99 <= 1e-5, (n, med, p99)


def test_resident_with_massless_matches_oracle(oracle):
    pos, mass = _with_massless(oracle, 16, 1500, 0.25)
    vel = np.zeros_like(pos)
    r = gb.GpuResidentLeapfrog(G, EPS, 0.5, precision="f64")
    r.upload(gb.State(pos, vel, mass))
    r.step_many(1e-3, 3)
    s = r.snapshot()
    p, v = pos.copy(), vel.copy()
    oracle.LeapfrogKdkLbvh(G, EPS, 0.5).step_many(p, v, mass, 1e-3, 3)
    assert np.array_equal(s.pos, p) and np.array_equal(s.vel, v)
