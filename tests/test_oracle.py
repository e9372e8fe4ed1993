"""The oracle pinned against the reference's own known-answer and invariant tests.

Golden vectors: solvers/src/lbvh.rs:691-726 (tests/golden/morton_kat.json).
Invariants restated from solvers/tests/lbvh.rs:88-312 with the reference's bounds.
"""

import json
import os

import numpy as np
import pytest

G = 1.0
EPS = 0.05
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_morton_known_answers(oracle):
    kat = json.load(open(os.path.join(GOLDEN, "morton_kat.json")))
    for v, want in kat["expand10"]:
        assert oracle.expand10(v) == want
    for (x, y, z), want in kat["morton3"]:
        assert oracle.morton3(x, y, z) == want
    prev = -1
    for x in range(kat["monotone_axis_cells"]):
        c = oracle.morton3(x, 0, 0)
        assert c > prev
        prev = c


def test_morton_convention(oracle):
    # reference_morton convention, solvers/src/lbvh.rs:101-104.
    pos = oracle.fixture_cloud(7, 500, 3.0)
    lanes, codes, b = oracle.reference_morton(pos)
    lo, hi = pos.min(0), pos.max(0)
    half = max(0.5 * (hi - lo).max(), 1e-12) * (1.0 + 1e-9)
    center = (lo + hi) * 0.5
    assert np.array_equal(b["bmin"], center - half)
    assert b["size"] == 2.0 * half and b["scale"] == 1024.0 / (2.0 * half)
    assert lanes.max() <= 1023
    want = np.clip(np.floor((pos - b["bmin"]) * b["scale"]), 0, 1023).astype(np.uint32)
    assert np.array_equal(lanes, want)
    for i in range(0, 500, 37):
        assert codes[i] == oracle.morton3(*[int(v) for v in lanes[i]])


def test_sort_is_stable_by_code_then_index(oracle):
    codes = np.array([i % 4 for i in range(5000)], np.uint32)
    order = oracle.reference_sort(codes)
    assert np.array_equal(order, np.lexsort((np.arange(5000), codes)))
    rc = oracle.fixture_random_codes(99, 10000)
    assert np.array_equal(oracle.reference_sort(rc), np.argsort(rc, kind="stable"))


@pytest.mark.parametrize("seed", range(0, 100, 7))
def test_theta_to_zero_reproduces_direct_sum(oracle, seed):
    # solvers/tests/lbvh.rs:88-102
    pos, _, mass = oracle.fixture_cluster(seed, 120)
    exact = oracle.direct_sum(pos, mass, G, EPS)
    got = oracle.lbvh_accelerations(pos, mass, G, EPS, 1e-6)
    assert oracle.worst_rel_err(got, exact) < 1e-9


@pytest.mark.parametrize("seed", range(0, 100, 9))
def test_finite_theta_error_bounded_and_grows(oracle, seed):
    # solvers/tests/lbvh.rs:107-135
    pos, _, mass = oracle.fixture_cluster(seed, 120)
    exact = oracle.direct_sum(pos, mass, G, EPS)
    lo = oracle.lbvh_accelerations(pos, mass, G, EPS, 0.3)
    hi = oracle.lbvh_accelerations(pos, mass, G, EPS, 0.6)
    rl, rh = oracle.rms_rel_err(lo, exact), oracle.rms_rel_err(hi, exact)
    assert rl < 0.02 and rh < 0.10
    assert oracle.worst_rel_err(lo, exact) < 0.15 and oracle.worst_rel_err(hi, exact) < 0.40
    assert rh > rl


def test_momentum_flux_at_theta_zero(oracle):
    # solvers/tests/lbvh.rs:140-157
    for seed in range(32):
        pos, _, mass = oracle.fixture_cluster(seed, 200)
        a = oracle.lbvh_accelerations(pos, mass, G, EPS, 1e-6)
        net = (a * mass[:, None]).sum(0)
        scale = (np.linalg.norm(a, axis=1) * mass).sum()
        assert np.linalg.norm(net) / max(scale, 1e-300) < 1e-9


@pytest.mark.parametrize("n", [1, 2, 3, 5, 17, 128, 257])
def test_karras_structure_is_wellformed(oracle, n):
    # solvers/tests/lbvh.rs:163-245
    for seed in range(8):
        pos, _, mass = oracle.fixture_cluster(seed, n)
        nf, nu, lb = oracle.lbvh_flat(pos, mass)
        assert nf.shape[0] == 2 * n - 1
        leaves = nu[:, 2] > 0
        assert leaves.sum() == n and (nu[leaves, 2] == 1).all()
        assert sorted(lb[nu[leaves, 1]].tolist()) == list(range(n))
        end = 2 * n - 1
        assert all(nu[k, 0] > k and nu[k, 0] <= end for k in range(end))
        assert nu[0, 0] == end
        mn, mx = nf[:, 0:3] - nf[:, 3:6], nf[:, 0:3] + nf[:, 3:6]
        for k in range(end):
            if nu[k, 2] > 0:
                continue
            left, right = k + 1, nu[k + 1, 0]
            assert right < nu[k, 0] and nu[right, 0] == nu[k, 0]
            for c in (left, right):
                assert (mn[c] >= mn[k] - 1e-9).all() and (mx[c] <= mx[k] + 1e-9).all()
        assert (pos >= mn[0] - 1e-9).all() and (pos <= mx[0] + 1e-9).all()


def test_karras_arrays_structural(oracle):
    # gpu/tests/lbvh_tree.rs:159-199 structural invariants on the unified layout.
    for codes in (np.full(4096, 42, np.uint32), np.arange(4096, dtype=np.uint32),
                  (np.arange(5000) // 500).astype(np.uint32)):
        n = codes.shape[0]
        left, right, parent = oracle.reference_karras(codes)
        cc = np.zeros(2 * n - 1, int)
        for i in range(n - 1):
            assert left[i] != right[i]
            assert parent[left[i]] == n + i and parent[right[i]] == n + i
            cc[left[i]] += 1
            cc[right[i]] += 1
        assert parent[n] == 0xFFFFFFFF and cc[n] == 0
        assert (np.delete(cc, n) == 1).all()


def test_coincident_particles_deterministic_and_exact(oracle):
    # solvers/tests/lbvh.rs:267-292
    pos, _, mass = oracle.cluster_with_coincident_knot()
    a1 = oracle.lbvh_accelerations(pos, mass, G, EPS, 0.5)
    a2 = oracle.lbvh_accelerations(pos, mass, G, EPS, 0.5)
    assert np.array_equal(a1, a2)
    exact = oracle.direct_sum(pos, mass, G, EPS)
    got = oracle.lbvh_accelerations(pos, mass, G, EPS, 1e-6)
    assert oracle.worst_rel_err(got, exact) < 1e-9


def test_empty_and_single(oracle):
    # solvers/tests/lbvh.rs:297-312
    a = oracle.lbvh_accelerations(np.zeros((0, 3)), np.zeros(0), G, EPS, 0.5)
    assert a.shape == (0, 3)
    a = oracle.lbvh_accelerations(np.array([[1.0, 2.0, 3.0]]), np.array([1.0]), G, EPS, 0.5)
    assert np.array_equal(a, np.zeros((1, 3)))


def test_threaded_walk_is_identical(oracle):
    pos, _, mass = oracle.fixture_cluster(5, 3000)
    a1 = oracle.lbvh_accelerations(pos, mass, G, EPS, 0.5, threads=1)
    a4 = oracle.lbvh_accelerations(pos, mass, G, EPS, 0.5, threads=4)
    assert np.array_equal(a1, a4)


def test_aggregate_root_matches_totals(oracle):
    pos = oracle.fixture_cloud(3, 4000, 3.0)
    mass = oracle.fixture_masses(3 ^ 0xABCD, 4000)
    _, codes, _ = oracle.reference_morton(pos)
    order = oracle.reference_sort(codes)
    left, right, parent = oracle.reference_karras(codes[order])
    agg = oracle.reference_aggregate(left, right, pos[order], mass[order])
    n = 4000
    assert np.array_equal(agg["aabb_min"][n], pos.min(0))
    assert np.array_equal(agg["aabb_max"][n], pos.max(0))
    assert abs(agg["mass"][n] - mass.sum()) < 1e-9
    com = (pos * mass[:, None]).sum(0) / mass.sum()
    assert np.allclose(agg["com"][n], com, atol=1e-12)


def test_quadrupole_improves_accuracy(oracle):
    pos, _, mass = oracle.fixture_cluster(11, 2000)
    exact = oracle.direct_sum(pos, mass, G, EPS)
    mono = oracle.lbvh_accelerations(pos, mass, G, EPS, 0.5)
    quad = oracle.lbvh_accelerations_quad(pos, mass, G, EPS, 0.5)
    assert oracle.rms_rel_err(quad, exact) < 0.5 * oracle.rms_rel_err(mono, exact)


def test_kdk_matches_hand_loop(oracle):
    # core/src/integrator.rs:38-78 restated with numpy for two steps.
    pos, _, mass = oracle.fixture_cluster(2, 300)
    vel = np.zeros_like(pos)
    p1, v1 = pos.copy(), vel.copy()
    kdk = oracle.LeapfrogKdkLbvh(G, EPS, 0.5)
    kdk.step_many(p1, v1, mass, 1e-3, 2)
    p2, v2 = pos.copy(), vel.copy()
    acc = oracle.lbvh_accelerations(p2, mass, G, EPS, 0.5)
    for _ in range(2):
        v2 = v2 + acc * 0.0005
        p2 = p2 + v2 * 1e-3
        acc = oracle.lbvh_accelerations(p2, mass, G, EPS, 0.5)
        v2 = v2 + acc * 0.0005
    assert np.array_equal(p1, p2) and np.array_equal(v1, v2)


def test_potential_parallel_matches_serial(oracle):
    pos, _, mass = oracle.fixture_cluster(4, 2000)
    s = oracle.potential_serial(pos, mass, G, EPS)
    p = oracle.potential_parallel(pos, mass, G, EPS, threads=4)
    assert abs(p - s) <= 1e-9 * abs(s)


def test_stale_tree_walk_fresh_equals_full_and_converges(oracle):
    """The stale-tree walk (TreeGravity::gravity_active_cached semantics over the LBVH)
    equals the full pass on a fresh tree, and approaches the fresh pass as the drift
    since the tree was built shrinks."""
    pos, _, mass = oracle.fixture_cluster(21, 600)
    full = oracle.lbvh_accelerations(pos, mass, 1.0, 0.05, 0.5)
    t = np.arange(600, dtype=np.uint32)
    assert np.array_equal(oracle.lbvh_accelerations_stale(pos, mass, pos, mass, 1.0, 0.05, 0.5, t), full)
    rng = np.random.default_rng(4)
    step = rng.normal(0.0, 1.0, pos.shape)
    errs = []
    for h in (1e-2, 1e-3, 1e-4):
        moved = pos + h * step
        stale = oracle.lbvh_accelerations_stale(pos, mass, moved, mass, 1.0, 0.05, 0.5, t)
        fresh = oracle.lbvh_accelerations(moved, mass, 1.0, 0.05, 0.5)
        errs.append(float(np.max(np.linalg.norm(stale - fresh, axis=1) / np.linalg.norm(fresh, axis=1))))
    assert errs[0] > errs[1] > errs[2] and errs[2] < 1e-2
