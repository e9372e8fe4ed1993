"""GPU force parity against the oracle, restating the reference's walk gates
(solvers/tests/lbvh.rs, gpu/tests/gpu_lbvh.rs, gpu/tests/gpu_lbvh_fused.rs).

FP64 mode reproduces the reference's Lbvh accelerations bit for bit. FP32 mode (the
fast path) meets the parity tolerance against the reference's FP64 CPU walk on the
same inputs and theta: median per-particle relative error <= 1e-6 and p99 <= 1e-5."""

import os

import numpy as np
import pytest

import galaxy_b200 as gb

pytestmark = pytest.mark.gpu

G, EPS = 1.0, 0.05
MEDIAN_TOL, P99_TOL = 1e-6, 1e-5
THREADS = os.cpu_count() or 1


def _parity(approx, exact):
    from oracle import oracle as o

    e = o.per_particle_rel_err(approx, exact)
    return float(np.median(e)), float(np.percentile(e, 99))


@pytest.mark.parametrize("theta", [1e-6, 0.3, 0.5, 0.7])
def test_f64_bit_exact_cluster(oracle, theta):
    s = gb.GpuLbvh(G, EPS, theta, precision="f64")
    for seed in (0, 5, 17):
        pos, _, mass = oracle.fixture_cluster(seed, 300)
        ref = oracle.lbvh_accelerations(pos, mass, G, EPS, theta)
        assert np.array_equal(s.accelerations(pos, mass=mass), ref)


def test_f64_bit_exact_plummer_config(oracle):
    st = gb.ic.plummer(16384, 0)
    s = gb.GpuLbvh(1.0, 0.01, 0.5, precision="f64")
    ref = oracle.lbvh_accelerations(st.pos, st.mass, 1.0, 0.01, 0.5, threads=THREADS)
    assert np.array_equal(s.accelerations(st), ref)


def test_f64_bit_exact_coincident_knot(oracle):
    pos, _, mass = oracle.cluster_with_coincident_knot()
    for theta in (1e-6, 0.5):
        s = gb.GpuLbvh(G, EPS, theta, precision="f64")
        assert np.array_equal(s.accelerations(pos, mass=mass), oracle.lbvh_accelerations(pos, mass, G, EPS, theta))


@pytest.mark.parametrize("theta", [0.3, 0.5, 0.7])
def test_f32_parity_plummer(oracle, theta):
    st = gb.ic.plummer(16384, 0)
    ref = oracle.lbvh_accelerations(st.pos, st.mass, 1.0, 0.01, theta, threads=THREADS)
    got = gb.GpuLbvh(1.0, 0.01, theta).accelerations(st)
    med, p99 = _parity(got, ref)
    assert med <= MEDIAN_TOL and p99 <= P99_TOL, (med, p99)


def test_f32_parity_collision(oracle):
    st = gb.ic.collision(65_536, 7)
    ref = oracle.lbvh_accelerations(st.pos, st.mass, 1.0, 0.02, 0.5, threads=THREADS)
    got = gb.GpuLbvh(1.0, 0.02, 0.5).accelerations(st)
    med, p99 = _parity(got, ref)
    assert med <= MEDIAN_TOL and p99 <= P99_TOL, (med, p99)


def test_f32_parity_far_from_origin(oracle):
    pos = oracle.fixture_cloud(3, 20000, 3.0, (5e3, -5e3, 1e3))
    mass = oracle.fixture_masses(4, 20000)
    ref = oracle.lbvh_accelerations(pos, mass, G, EPS, 0.5, threads=THREADS)
    med, p99 = _parity(gb.GpuLbvh(G, EPS, 0.5).accelerations(pos, mass=mass), ref)
    assert med <= MEDIAN_TOL and p99 <= P99_TOL, (med, p99)


def test_f32_theta_to_zero_matches_direct_sum(oracle):
    # gpu/tests/gpu_lbvh.rs:100-120: RMS < 3e-4, worst < 5e-2 (ours is far tighter).
    s = gb.GpuLbvh(G, EPS, 1e-6)
    for seed in range(0, 100, 11):
        pos, _, mass = oracle.fixture_cluster(seed, 120)
        exact = oracle.direct_sum(pos, mass, G, EPS)
        got = s.accelerations(pos, mass=mass)
        assert oracle.rms_rel_err(got, exact) < 1e-6
        assert oracle.worst_rel_err(got, exact) < 1e-5


def test_f32_finite_theta_bounded(oracle):
    # gpu/tests/gpu_lbvh.rs:124-150
    for seed in range(0, 100, 13):
        pos, _, mass = oracle.fixture_cluster(seed, 120)
        exact = oracle.direct_sum(pos, mass, G, EPS)
        lo = gb.GpuLbvh(G, EPS, 0.3).accelerations(pos, mass=mass)
        hi = gb.GpuLbvh(G, EPS, 0.6).accelerations(pos, mass=mass)
        rl, rh = oracle.rms_rel_err(lo, exact), oracle.rms_rel_err(hi, exact)
        assert rl < 0.012 and rh < 0.05 and rh > rl


def test_f32_momentum_flux_theta_zero(oracle):
    s = gb.GpuLbvh(G, EPS, 1e-6)
    for seed in range(8):
        pos, _, mass = oracle.fixture_cluster(seed, 200)
        a = s.accelerations(pos, mass=mass)
        net = (a * mass[:, None]).sum(0)
        assert np.linalg.norm(net) / (np.linalg.norm(a, axis=1) * mass).sum() < 1e-6


def test_f32_coincident_knot(oracle):
    pos, _, mass = oracle.cluster_with_coincident_knot()
    s = gb.GpuLbvh(G, EPS, 0.5)
    a1 = s.accelerations(pos, mass=mass)
    a2 = s.accelerations(pos, mass=mass)
    assert np.array_equal(a1, a2)
    med, p99 = _parity(a1, oracle.lbvh_accelerations(pos, mass, G, EPS, 0.5))
    assert p99 <= P99_TOL


def test_deterministic_and_stats(oracle):
    st = gb.ic.plummer(50_000, 3)
    s = gb.GpuLbvh(1.0, 0.01, 0.5, stats=True)
    a = s.accelerations(st)
    sa = s.stats()
    b = s.accelerations(st)
    assert np.array_equal(a, b)
    _, stt = oracle.lbvh_accelerations(st.pos, st.mass, 1.0, 0.01, 0.5, threads=THREADS, stats=True)
    # the lanes make exactly the reference's decisions
    assert sa["leaf_interactions"] == stt["leaf"]
    assert sa["far_interactions"] == stt["far"]
    assert sa["f64_rechecks"] < 1e-3 * (stt["far"] + stt["open"])


def test_empty_and_single():
    s = gb.GpuLbvh(G, EPS, 0.5)
    assert s.accelerations(np.zeros((0, 3)), mass=np.zeros(0)).shape == (0, 3)
    assert np.array_equal(s.accelerations(np.array([[1.0, 2.0, 3.0]]), mass=np.array([1.0])), np.zeros((1, 3)))


def test_length_mismatch_raises():
    s = gb.GpuLbvh(G, EPS, 0.5)
    with pytest.raises(ValueError):
        s.accelerations(np.zeros((4, 3)), acc=np.zeros((3, 3)), mass=np.ones(4))


def test_quadrupole_matches_oracle_and_is_more_accurate(oracle):
    pos, _, mass = oracle.fixture_cluster(11, 4000)
    exact = oracle.direct_sum(pos, mass, G, EPS)
    q_ref = oracle.lbvh_accelerations_quad(pos, mass, G, EPS, 0.5, threads=THREADS)
    q = gb.GpuLbvh(G, EPS, 0.5, multipole="quad").accelerations(pos, mass=mass)
    med, p99 = _parity(q, q_ref)
    assert p99 <= 1e-5, p99
    mono = gb.GpuLbvh(G, EPS, 0.5).accelerations(pos, mass=mass)
    assert oracle.rms_rel_err(q, exact) < 0.5 * oracle.rms_rel_err(mono, exact)


def test_no_kahan_still_close(oracle):
    st = gb.ic.plummer(16384, 0)
    ref = oracle.lbvh_accelerations(st.pos, st.mass, 1.0, 0.01, 0.5, threads=THREADS)
    got = gb.GpuLbvh(1.0, 0.01, 0.5, kahan=False).accelerations(st)
    med, p99 = _parity(got, ref)
    assert p99 < 1e-4


def test_direct_sum_f64_matches_oracle(oracle):
    pos, _, mass = oracle.fixture_cluster(9, 3000)
    s = gb.GpuLbvh(G, EPS, 0.5)
    got = s.direct_sum_f64(pos, mass)
    ref = oracle.direct_sum(pos, mass, G, EPS)
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.abs(ref).max()
    t = np.array([5, 17, 2999], np.uint32)
    sub = s.direct_sum_f64(pos, mass, t)
    assert np.all(np.linalg.norm(sub - ref[t], axis=1) <= 1e-12 * np.linalg.norm(ref[t], axis=1))


def test_potential_energy_matches_oracle(oracle):
    pos, _, mass = oracle.fixture_cluster(4, 5000)
    u = gb.GpuLbvh(G, EPS, 0.5).potential_energy(pos, mass=mass)
    ref = oracle.potential_serial(pos, mass, G, EPS)
    assert abs(u - ref) <= 1e-9 * abs(ref)
