"""The stale-tree active walk (TreeGravity's rebuild_gravity_cache / gravity_active_cached,
solvers/src/barnes_hut.rs:647-711, over the LBVH): the tree frozen at the block-start
state, walked at the current positions -- against the oracle's restatement (the
reference's LbvhFlat walk over a stale flat tree with current positions)."""

import numpy as np
import pytest

import galaxy_b200 as gb

pytestmark = pytest.mark.gpu
G, EPS = 1.0, 0.05


def _moved(pos, h, seed):
    return pos + h * np.random.default_rng(seed).normal(0.0, 1.0, pos.shape)


@pytest.mark.parametrize("theta", [0.3, 0.5, 0.7])
def test_f64_stale_walk_bit_exact(oracle, theta):
    pos0, _, mass = oracle.fixture_cluster(41, 4000)
    pos1 = _moved(pos0, 3e-3, 1)
    act = np.flatnonzero(np.random.default_rng(2).random(4000) < 0.2)
    s = gb.GpuStaleTreeGravity(G, EPS, theta, precision="f64")
    s.rebuild_gravity_cache(pos0, mass=mass)
    got = s.gravity_active_cached(pos1, act, mass=mass)
    ref = oracle.lbvh_accelerations_stale(pos0, mass, pos1, mass, G, EPS, theta, act)
    assert np.array_equal(got[act], ref)


def test_f32_stale_walk_parity_and_fresh_equality(oracle):
    st = gb.ic.collision(65_536, 7)
    pos1 = _moved(st.pos, 1e-3, 3)
    act = np.flatnonzero(np.random.default_rng(4).random(len(st)) < 0.05)
    s = gb.GpuStaleTreeGravity(1.0, 0.02, 0.5)
    s.rebuild_gravity_cache(st)
    got = s.gravity_active_cached(pos1, act, mass=st.mass)
    ref = oracle.lbvh_accelerations_stale(st.pos, st.mass, pos1, st.mass, 1.0, 0.02, 0.5, act, threads=8)
    e = oracle.per_particle_rel_err(got[act], ref)
    assert np.median(e) <= 1e-6 and np.percentile(e, 99) <= 1e-5
    # unchanged positions: the cached walk is the active walk of a fresh tree
    s.rebuild_gravity_cache(st)
    same = s.gravity_active_cached(st, act)
    fresh = gb.GpuLbvh(1.0, 0.02, 0.5).accelerations_active(st, act)
    assert np.max(np.linalg.norm(same[act] - fresh[act], axis=1) / np.linalg.norm(fresh[act], axis=1)) < 1e-5


def test_cache_lifecycle(oracle):
    pos0, _, mass = oracle.fixture_cluster(42, 2000)
    s = gb.GpuStaleTreeGravity(G, EPS, 0.5, precision="f64")
    untouched = np.full((2000, 3), 3.0)
    assert np.array_equal(s.gravity_active_cached(pos0, [1, 2], acc=untouched.copy(), mass=mass), untouched)
    s.rebuild_gravity_cache(pos0, mass=mass)
    a1 = s.gravity_active_cached(_moved(pos0, 1e-3, 5), [1, 2, 3], mass=mass)
    # a fresh full pass runs on its own handle and leaves the cache in place
    full = s.accelerations(pos0, mass=mass)
    assert np.array_equal(full, oracle.lbvh_accelerations(pos0, mass, G, EPS, 0.5))
    a2 = s.gravity_active_cached(_moved(pos0, 1e-3, 5), [1, 2, 3], mass=mass)
    assert np.array_equal(a1, a2)
    # a different particle count needs a rebuild
    with pytest.raises(gb.GxError):
        s.gravity_active_cached(pos0[:1000], [1], mass=mass[:1000])
    # the C handle itself refuses a cache that another force call replaced
    h = gb.GpuLbvh(G, EPS, 0.5, precision="f64")
    lib = gb._lib.lib()
    import ctypes as C
    p, m = np.ascontiguousarray(pos0), np.ascontiguousarray(mass)
    assert lib.gx_rebuild_gravity_cache(h._h, 2000, p.ctypes.data, m.ctypes.data) == 0
    h.accelerations(pos0, mass=mass)
    out = np.zeros((2000, 3))
    idx = np.array([0], np.uint32)
    rc = lib.gx_gravity_active_cached(h._h, 2000, p.ctypes.data, m.ctypes.data, 1, idx.ctypes.data, out.ctypes.data)
    assert rc == -5  # GX_ERR_STATE


def test_stale_walk_with_massless_leaves(oracle):
    pos0, _, mass = oracle.fixture_cluster(43, 3000)
    mass = mass.copy()
    mass[::7] = 0.0
    pos1 = _moved(pos0, 2e-3, 6)
    act = np.arange(0, 3000, 3)
    s = gb.GpuStaleTreeGravity(G, EPS, 0.5, precision="f64")
    s.rebuild_gravity_cache(pos0, mass=mass)
    got = s.gravity_active_cached(pos1, act, mass=mass)
    assert np.array_equal(got[act], oracle.lbvh_accelerations_stale(pos0, mass, pos1, mass, G, EPS, 0.5, act))
