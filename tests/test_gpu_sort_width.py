"""The radix sort's digit width (8-bit digits in 4 passes, or 10-bit digits in 3 passes,
for 30-bit keys) is a tuning choice: the sort by (code, index) is exact, so the
permutation, the tree and every result are the same with either width, and the FP64
walk still equals the oracle's restatement of the reference (solvers/src/lbvh.rs:143-147,
:469-524) bit for bit."""

import numpy as np
import pytest

import galaxy_b200 as gb
from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [2, 3, 1000, 4096, 4097, 65_553])
def test_wide_digits_equal_narrow_and_oracle(n):
    pos, _, mass = oracle.fixture_cluster(3, n)
    a8 = gb.GpuLbvh(1.0, 0.05, 0.5, radix_bits=8).accelerations(pos, mass=mass)
    a10 = gb.GpuLbvh(1.0, 0.05, 0.5, radix_bits=10).accelerations(pos, mass=mass)
    assert np.array_equal(a8, a10)
    ref = oracle.lbvh_accelerations(pos, mass, 1.0, 0.05, 0.5, threads=oracle.max_threads())
    a64 = gb.GpuLbvh(1.0, 0.05, 0.5, precision="f64", radix_bits=10).accelerations(pos, mass=mass)
    assert np.array_equal(a64, ref)


def test_wide_digits_with_heavy_ties():
    """Particles on a coarse lattice: most Morton codes repeat many times, so the order
    inside each run of equal codes is the index order, across tiles and passes."""
    rng = np.random.default_rng(9)
    n = 50_000
    pos = rng.integers(0, 6, size=(n, 3)).astype(np.float64) * 0.25
    pos += rng.normal(0.0, 1e-9, size=(n, 3))  # no two particles coincide exactly
    mass = rng.uniform(0.5, 1.0, n)
    ref = oracle.lbvh_accelerations(pos, mass, 1.0, 0.01, 0.5, threads=oracle.max_threads())
    for bits in (8, 10):
        a64 = gb.GpuLbvh(1.0, 0.01, 0.5, precision="f64", radix_bits=bits).accelerations(pos, mass=mass)
        assert np.array_equal(a64, ref), bits


def test_wide_digits_full_size_collision_and_resident_steps():
    st = gb.ic.collision(2 * 524_288, 0, mass_ratio=1.0, pericentre=4.0, incl1_deg=30.0, incl2_deg=60.0)
    a8 = gb.GpuLbvh(1.0, 0.02, 0.5, radix_bits=8).accelerations(st)
    a10 = gb.GpuLbvh(1.0, 0.02, 0.5, radix_bits=10).accelerations(st)
    assert np.array_equal(a8, a10)
    small = gb.ic.plummer(20_000, 4)
    runs = []
    for bits in (8, 10):
        r = gb.GpuResidentLeapfrog(1.0, 0.01, 0.5, radix_bits=bits)
        r.upload(small)
        r.step_many(1e-3, 5)
        runs.append(r.snapshot())
    assert np.array_equal(runs[0].pos, runs[1].pos) and np.array_equal(runs[0].vel, runs[1].vel)


def test_batch_with_wide_digits_equals_alone():
    sts = [gb.ic.plummer(5_000 + 3_000 * i, 40 + i) for i in range(3)]
    b = gb.Batch(radix_bits=10)
    ids = [b.add(s, 1.0, 0.01, 0.5, 1e-3) for s in sts]
    b.step(3)
    for sid, st in zip(ids, sts):
        r = gb.GpuResidentLeapfrog(1.0, 0.01, 0.5)
        r.upload(st)
        r.step_many(1e-3, 3)
        assert np.array_equal(b.snapshot(sid).pos, r.snapshot().pos)


def test_autotune_records_a_digit_width():
    st = gb.ic.collision(300_000, 13)  # bucket 18
    r = gb.GpuResidentLeapfrog(1.0, 0.02, 0.5)
    r.upload(st)
    best = r.autotune(repeats=2)
    assert best["radix_bits"] in (8, 10) and best["sort_ms"] > 0
    rec = gb.tuning_lookup(300_000)
    assert rec is not None and rec["radix_bits"] == best["radix_bits"]
    assert gb.tuning_lookup(300_000, morton63=True) is None
