"""The active-subset force path (ForceSolver::accelerations_active and
gravity_active_cached, core/src/traits.rs:52-54 and :89-91, which Lbvh keeps at the full
fresh pass): the tree is built from every particle and walked for the active targets
only; each active target gets the reference's acceleration (FP64 bit for bit, FP32
within the parity bounds), inactive rows are untouched."""

import numpy as np
import pytest

import galaxy_b200 as gb

pytestmark = pytest.mark.gpu
G, EPS = 1.0, 0.05


def _active(n, frac, seed):
    rng = np.random.default_rng(seed)
    return np.flatnonzero(rng.random(n) < frac)


@pytest.mark.parametrize("frac", [0.01, 0.3, 1.0])
def test_f64_active_bit_exact_vs_oracle(oracle, frac):
    pos, _, mass = oracle.fixture_cluster(31, 5000)
    act = _active(len(pos), frac, 1)
    ref = oracle.lbvh_accelerations(pos, mass, G, EPS, 0.5)
    sentinel = np.full((len(pos), 3), 7.0)
    got = gb.GpuLbvh(G, EPS, 0.5, precision="f64").accelerations_active(pos, act, acc=sentinel, mass=mass)
    assert np.array_equal(got[act], ref[act])
    rest = np.setdiff1d(np.arange(len(pos)), act)
    assert np.all(got[rest] == 7.0)


@pytest.mark.parametrize("frac", [0.01, 0.2])
def test_f32_active_parity(oracle, frac):
    st = gb.ic.collision(65_536, 4)
    act = _active(len(st), frac, 2)
    ref = oracle.lbvh_accelerations(st.pos, st.mass, 1.0, 0.02, 0.5, threads=8)
    got = gb.GpuLbvh(1.0, 0.02, 0.5).accelerations_active(st, act)
    e = oracle.per_particle_rel_err(got[act], ref[act])
    assert np.median(e) <= 1e-6 and np.percentile(e, 99) <= 1e-5
    full = gb.GpuLbvh(1.0, 0.02, 0.5).accelerations(st)
    assert np.max(np.linalg.norm(got[act] - full[act], axis=1) / np.linalg.norm(full[act], axis=1)) < 1e-5


def test_active_repeats_unsorted_and_edges(oracle):
    pos, _, mass = oracle.fixture_cluster(32, 3000)
    ref = oracle.lbvh_accelerations(pos, mass, G, EPS, 0.5)
    s = gb.GpuLbvh(G, EPS, 0.5, precision="f64")
    act = np.array([2999, 5, 5, 1000, 0, 2999, 17])
    got = s.accelerations_active(pos, act, mass=mass)
    assert np.array_equal(got[np.unique(act)], ref[np.unique(act)])
    before = np.ones((3000, 3))
    assert np.array_equal(s.accelerations_active(pos, [], acc=before.copy(), mass=mass), before)
    with pytest.raises(ValueError):
        s.accelerations_active(pos, [3000], mass=mass)
    assert np.array_equal(s.gravity_active_cached(pos, [7, 8], mass=mass)[[7, 8]], ref[[7, 8]])
    one = s.accelerations_active(pos[:1], [0], mass=mass[:1])
    assert np.array_equal(one, np.zeros((1, 3)))


def test_active_walk_follows_full_walk_after_active_call():
    """An active-subset call between full calls leaves the handle fully usable."""
    st = gb.ic.plummer(20_000, 9)
    s = gb.GpuLbvh(1.0, 0.01, 0.5, precision="f64")
    full0 = s.accelerations(st)
    s.accelerations_active(st, np.arange(0, 20_000, 7))
    assert np.array_equal(s.accelerations(st), full0)
