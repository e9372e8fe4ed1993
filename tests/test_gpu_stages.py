"""GPU stage gates against the oracle, restating the reference's stage tests
(gpu/tests/lbvh_morton.rs, lbvh_sort.rs, lbvh_tree.rs). Morton codes, the sort
permutation, the Karras topology and the FP64 aggregation are all bit-exact: the
device computes the bounding cube and lanes in FP64 with the reference's operation
order, and the aggregation folds in FP64 in fixed (left, right) order."""

import numpy as np
import pytest

import galaxy_b200 as gb

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def h():
    return gb.GpuLbvh(1.0, 0.05, 0.5)


@pytest.fixture(scope="module")
def hq():
    return gb.GpuLbvh(1.0, 0.05, 0.5, multipole="quad")


# ---- Morton (gpu/tests/lbvh_morton.rs) ------------------------------------------------
def _check_morton(h, oracle, pos):
    lanes, codes, b = gb.stage_morton(pos, h)
    rl, rc, rb = oracle.reference_morton(pos)
    assert np.array_equal(codes, rc)
    assert np.array_equal(lanes, rl)
    assert np.array_equal(b["bmin"], rb["bmin"]) and b["size"] == rb["size"] and b["scale"] == rb["scale"]


@pytest.mark.parametrize("seed", [1, 7, 42, 1000])
def test_morton_bit_exact_on_clouds(h, oracle, seed):
    _check_morton(h, oracle, oracle.fixture_cloud(seed, 8000, 3.0))


def test_morton_bit_exact_far_from_origin(h, oracle):
    # lbvh_morton.rs:143-170 characterises f32 divergence at |x|~1e6; FP64 here is exact.
    _check_morton(h, oracle, oracle.fixture_cloud(3, 8000, 3.0, (1e6, 1e6, 1e6)))


def test_morton_collinear_degenerate_axes(h, oracle):
    pos = np.array([[i * 0.1, 2.0, -1.0] for i in range(500)])
    _check_morton(h, oracle, pos)


def test_morton_single_and_coincident(h, oracle):
    _check_morton(h, oracle, np.array([[1.0, 2.0, 3.0]]))
    _check_morton(h, oracle, np.tile([1.5, -2.0, 0.25], (512, 1)))


def test_morton_workloads(h, oracle):
    _check_morton(h, oracle, gb.ic.plummer(16384, 0).pos)
    _check_morton(h, oracle, gb.ic.collision(300_000, 1).pos)


# ---- sort (gpu/tests/lbvh_sort.rs) ----------------------------------------------------
def _check_sort(h, oracle, codes):
    codes = np.ascontiguousarray(codes, np.uint32)
    order, sc = gb.stage_sort(codes, h)
    ref = oracle.reference_sort(codes)
    assert np.array_equal(order, ref)
    assert np.array_equal(sc, codes[ref])
    assert np.array_equal(np.sort(order), np.arange(codes.shape[0], dtype=np.uint32))


@pytest.mark.parametrize("seed", [1, 7, 42, 1000])
def test_sort_morton_codes(h, oracle, seed):
    _check_sort(h, oracle, oracle.reference_morton(oracle.fixture_cloud(seed, 8000, 3.0))[1])


@pytest.mark.parametrize("seed", [2, 99, 12345])
def test_sort_random_codes(h, oracle, seed):
    _check_sort(h, oracle, oracle.fixture_random_codes(seed, 10_000))


def test_sort_ties_by_ascending_index(h, oracle):
    _check_sort(h, oracle, np.arange(5000) % 4)


def test_sort_low_byte_pass(h, oracle):
    _check_sort(h, oracle, 0x00ABCD00 | ((np.arange(4096, dtype=np.uint64) * 37) & 0xFF))


def test_sort_high_byte_pass(h, oracle):
    _check_sort(h, oracle, (np.arange(4096) % 64) << 24)


def test_sort_structural_orders(h, oracle):
    _check_sort(h, oracle, np.arange(3000))
    _check_sort(h, oracle, np.arange(3000)[::-1])
    _check_sort(h, oracle, np.full(2048, 42))
    _check_sort(h, oracle, [7])


def test_sort_large_multi_tile(h, oracle):
    _check_sort(h, oracle, oracle.fixture_random_codes(0xBEEF, 65_536))
    _check_sort(h, oracle, oracle.fixture_random_codes(5, 1_000_003))
    # heavy ties across many tiles: look-back chains carry equal digits far
    _check_sort(h, oracle, (np.arange(700_001) % 3) << 28)


def test_sort_deterministic(h, oracle):
    codes = oracle.reference_morton(oracle.fixture_cloud(0x50, 6000, 3.0))[1]
    a, _ = gb.stage_sort(codes, h)
    b, _ = gb.stage_sort(codes, h)
    assert np.array_equal(a, b)


# ---- Karras build + aggregation (gpu/tests/lbvh_tree.rs) -------------------------------
def _sorted_inputs(oracle, pos, mass):
    codes = oracle.reference_morton(pos)[1]
    order = oracle.reference_sort(codes)
    return codes[order], pos[order], mass[order]


def _check_build(h, oracle, sc, sp, sm, quad=False):
    out = gb.stage_build(sc, sp, sm, h, quad=quad)
    left, right, parent = oracle.reference_karras(sc)
    assert np.array_equal(out["left"], left)
    assert np.array_equal(out["right"], right)
    assert np.array_equal(out["parent"], parent)
    agg = oracle.reference_aggregate(left, right, sp, sm)
    for k in ("aabb_min", "aabb_max", "com", "mass"):
        assert np.array_equal(out[k], agg[k]), k
    if quad:
        q = oracle.quadrupole(left, right, agg["com"], agg["mass"])
        assert np.array_equal(out["quad"], q)
    return out


@pytest.mark.parametrize("seed", [1, 7, 42, 1000])
def test_build_topology_morton_codes(h, oracle, seed):
    pos = oracle.fixture_cloud(seed, 6000, 3.0)
    _check_build(h, oracle, *_sorted_inputs(oracle, pos, np.ones(6000)))


def test_build_topology_degenerate_codes(h, oracle):
    for codes in (np.full(4096, 42), (np.arange(5000) // 500), np.arange(4096)):
        n = codes.shape[0]
        pos = np.repeat(np.arange(n, dtype=np.float64)[:, None], 3, axis=1)
        _check_build(h, oracle, codes.astype(np.uint32), pos, np.ones(n))


@pytest.mark.parametrize("n", [255, 256, 257, 511, 513, 4095, 4097])
def test_build_block_and_tile_edges(h, oracle, n):
    # systems ending just inside, at and just past a 256-leaf block (the per-block pass
    # and the cross-block climbs) and a 4096-particle tile
    pos = oracle.fixture_cloud(0x5EED + n, n, 2.0)
    mass = oracle.fixture_masses(0xD00D + n, n)
    _check_build(h, oracle, *_sorted_inputs(oracle, pos, mass))


def test_build_large(h, oracle):
    pos = oracle.fixture_cloud(0xBEEF, 65_536, 5.0)
    _check_build(h, oracle, *_sorted_inputs(oracle, pos, np.ones(65_536)))


@pytest.mark.parametrize("seed", [3, 17, 271])
def test_aggregation_bit_exact(h, oracle, seed):
    pos = oracle.fixture_cloud(seed, 4000, 3.0)
    mass = oracle.fixture_masses(seed ^ 0xABCD, 4000)
    _check_build(h, oracle, *_sorted_inputs(oracle, pos, mass))


def test_aggregation_coincident(h, oracle):
    pos = np.tile([1.5, -2.0, 0.25], (512, 1))
    _check_build(h, oracle, *_sorted_inputs(oracle, pos, oracle.fixture_masses(99, 512)))


def test_aggregation_monotone_chain_payload(h, oracle):
    n = 2048
    _check_build(h, oracle, np.arange(n, dtype=np.uint32), oracle.fixture_cloud(0xC0FFEE, n, 4.0),
                 oracle.fixture_masses(0xBEE, n))


def test_aggregation_single_and_pair(h, oracle):
    _check_build(h, oracle, np.array([5], np.uint32), np.array([[1.0, 2.0, 3.0]]), np.array([2.0]))
    _check_build(h, oracle, np.array([5, 9], np.uint32), np.array([[1.0, 2.0, 3.0], [0.0, 1.0, 0.5]]),
                 np.array([2.0, 0.5]))


def test_quadrupole_bit_exact(hq, oracle):
    pos = oracle.fixture_cloud(11, 5000, 3.0)
    mass = oracle.fixture_masses(12, 5000)
    _check_build(hq, oracle, *_sorted_inputs(oracle, pos, mass), quad=True)


def test_build_deterministic(h, oracle):
    pos = oracle.fixture_cloud(0x50, 5000, 3.0)
    a = gb.stage_build(*_sorted_inputs(oracle, pos, np.ones(5000)), h)
    b = gb.stage_build(*_sorted_inputs(oracle, pos, np.ones(5000)), h)
    for k in a:
        assert np.array_equal(a[k], b[k])
