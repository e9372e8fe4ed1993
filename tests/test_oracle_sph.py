"""The SPH oracle (oracle/sph_oracle.cpp) pinned against the reference's frozen output
bits and its invariant gates (solvers/tests/sph_kernel.rs, sph_grid.rs, sph_density.rs,
sph_forces.rs, sph_cfl.rs), plus the host-side SPH API pieces that need no GPU."""

import json
import os
import struct

import numpy as np
import pytest

PINS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "sph_pins.json")))


def f64(h: str) -> float:
    return struct.unpack("<d", struct.pack("<Q", int(h, 16)))[0]


def test_hydro_matches_frozen_reference_bits(oracle):
    # solvers/tests/sph_forces.rs:393-462: byte-identical isothermal accelerations.
    p = PINS["hydro_isothermal_8"]
    n = p["n"]
    pos = oracle.fixture_sph_points(p["pos_seed"], n, p["pos_scale"])
    vel = oracle.fixture_sph_points(p["vel_seed"], n, p["vel_scale"])
    mass = np.array([1.0 + i * 0.1 for i in range(n)])
    rho = np.array([0.8 + i * 0.05 for i in range(n)])
    h = np.array([0.9 + i * 0.03 for i in range(n)])
    acc, _ = oracle.sph_hydro(pos, vel, mass, rho, h, eos=0, eos_param=p["c_s"], threads=1)
    want = np.array([[f64(b) for b in row] for row in p["acc_bits"]])
    assert np.array_equal(acc, want)


def test_cfl_matches_frozen_reference_bits(oracle):
    # solvers/tests/sph_cfl.rs:189-212: the whole cold density solve (bbox, occupancy seeds,
    # bisection) and the signal-velocity bound, bit for bit.
    p = PINS["cfl_isothermal_600"]
    pos = oracle.fixture_sph_points(p["pos_seed"], p["n"], p["pos_scale"])
    vel = oracle.fixture_sph_points(p["vel_seed"], p["n"], p["vel_scale"])
    got = oracle.sph_max_stable_dt(pos, vel, np.ones(p["n"]), np.ones(p["n"], np.uint8), p["c_cfl"])
    assert got == f64(p["min_dt_bits"])


def test_kernel_gates(oracle):
    # solvers/tests/sph_kernel.rs: W(0, h) = 1/(pi h^3), compact support at 2h, continuity
    # at the knots, unit normalisation, grad W against central differences.
    for h in (0.3, 1.0, 2.7):
        assert abs(oracle.sph_w(0.0, h) - 1.0 / (np.pi * h ** 3)) <= 1e-14 * oracle.sph_w(0.0, h)
        assert oracle.sph_w(2.0 * h, h) == 0.0 and oracle.sph_w(2.0001 * h, h) == 0.0
        for q in (1.0, 2.0):
            a, b = oracle.sph_w(q * h * (1 - 1e-9), h), oracle.sph_w(q * h * (1 + 1e-9), h)
            assert abs(a - b) <= 1e-7 * oracle.sph_w(0.0, h)
    r = np.linspace(0.0, 2.0, 20001)
    w = np.array([oracle.sph_w(x, 1.0) for x in r])
    integral = np.trapezoid(4 * np.pi * r * r * w, r)
    assert abs(integral - 1.0) < 1e-6
    h, eps = 0.8, 1e-6
    for d in (np.array([0.3, -0.2, 0.5]), np.array([1.1, 0.4, -0.3])):
        g = oracle.sph_grad_w(d, h)
        num = [(oracle.sph_w(np.linalg.norm(d + eps * e), h) - oracle.sph_w(np.linalg.norm(d - eps * e), h)) / (2 * eps)
               for e in np.eye(3)]
        assert np.allclose(g, num, rtol=1e-6, atol=1e-9)
    assert not oracle.sph_grad_w([0.0, 0.0, 0.0], 1.0).any()
    assert not oracle.sph_grad_w([3.0, 0.0, 0.0], 1.0).any()


@pytest.mark.parametrize("cell", [0.1, 0.37, 1.3])
def test_grid_matches_brute_force(oracle, cell):
    # solvers/tests/sph_grid.rs: the grid query equals the O(N^2) oracle, ascending.
    pos = oracle.fixture_sph_points(5, 600, 2.0)
    pos[:20] = pos[0]  # coincident particles are all returned
    pos[20:40, 0] = np.round(pos[20:40, 0] / cell) * cell  # cell-wall straddlers
    for i in (0, 25, 77, 401):
        for r in (0.05, 0.3, 0.9):
            a = oracle.sph_neighbours(pos, pos[i], r, cell)
            b = oracle.sph_neighbours(pos, pos[i], r, 0.0)
            assert np.array_equal(a, b) and np.all(np.diff(a.astype(np.int64)) > 0)


def test_fixed_h_density_bit_exact_vs_brute_force(oracle):
    # solvers/tests/sph_density.rs:36-48
    pos = oracle.fixture_sph_points(11, 400, 4.0, centered=False)
    mass = np.array([0.5 + (i % 7) * 0.1 for i in range(400)])
    h = np.full(400, 0.35)
    assert np.array_equal(oracle.sph_density_fixed(pos, mass, h), oracle.sph_reference_density(pos, mass, h))


def test_adaptive_density_gates(oracle):
    # solvers/tests/sph_density.rs:91-170: target count within 1, scaling law, warm start
    # bounded by the bisection tolerance, deterministic.
    pos = oracle.fixture_sph_points(21, 2000, 1.0, centered=False)
    mass = np.ones(2000)
    rho, h = oracle.sph_density_adaptive(pos, mass)
    for i in range(0, 2000, 97):
        d = np.linalg.norm(pos[i] - pos, axis=1)
        n = (4 * np.pi / 3) * (2 * h[i]) ** 3 * sum(oracle.sph_w(x, h[i]) for x in d)
        assert abs(n - 48.0) <= 1.0 and rho[i] > 0
    rho2, h2 = oracle.sph_density_adaptive(pos, mass)
    assert np.array_equal(rho, rho2) and np.array_equal(h, h2)
    lam = 4.2
    rb, hb = oracle.sph_density_adaptive(pos * lam, mass)
    assert np.max(np.abs(rb - rho / lam ** 3) / (rho / lam ** 3)) < 1e-2
    assert np.max(np.abs(hb - lam * h) / (lam * h)) < 5e-3
    rw, hw = oracle.sph_density_adaptive(pos, mass, h_init=1.5 * h)
    assert np.max(np.abs(hw - h) / h) <= 2e-3 and np.max(np.abs(rw - rho) / rho) <= 8e-3


def test_underpopulated_and_empty(oracle):
    # solvers/tests/sph_density.rs:172-196
    for n in (1, 2, 3):
        pos = oracle.fixture_sph_points(n + 1, n, 1.0, centered=False)
        rho, h = oracle.sph_density_adaptive(pos, np.ones(n))
        assert np.all(np.isfinite(h)) and np.all(h > 0) and np.all(np.isfinite(rho)) and np.all(rho > 0)
    rho, h = oracle.sph_density_adaptive(np.zeros((0, 3)), np.zeros(0))
    assert rho.size == 0 and h.size == 0


def test_hydro_pair_antisymmetry_and_momentum(oracle):
    # solvers/tests/sph_forces.rs:122-139, 225-254
    pos = np.array([[0.1, -0.2, 0.3], [0.9, 0.4, -0.1]])
    vel = np.array([[0.2, 0.0, -0.1], [-0.3, 0.1, 0.05]])
    acc, _ = oracle.sph_hydro(pos, vel, [0.75, 0.75], [1.7, 2.6], [0.9, 1.25])
    assert np.array_equal(acc[0], -acc[1])
    pos = oracle.fixture_sph_points(7, 300, 2.0)
    vel = oracle.fixture_sph_points(7 ^ 0xABCD, 300, 2.0)
    mass = np.full(300, 0.9)
    rho, h = oracle.sph_density_adaptive(pos, mass)
    acc, dudt = oracle.sph_hydro(pos, vel, mass, rho, h)
    scale = np.sum(mass[:, None] * np.abs(acc))
    assert np.linalg.norm((mass[:, None] * acc).sum(axis=0)) < 1e-12 * scale


def test_cfl_gas_free_is_infinite(oracle):
    pos = oracle.fixture_sph_points(3, 50, 1.0)
    assert oracle.sph_max_stable_dt(pos, pos * 0, np.ones(50), np.zeros(50, np.uint8), 0.25) == np.inf


def test_gravity_sph_routes_hydro_to_gas_rows_only(oracle):
    # solvers/tests/sph_forces.rs:320-375: star rows equal pure gravity exactly.
    pos, vel, mass, kind = oracle.fixture_gas_star_mix(0xA5F0, 120, 240)
    gs = oracle.GravitySph(1.0, 0.05, 0.5)
    acc = gs.accelerations(pos, vel, mass, kind)
    grav = oracle.lbvh_accelerations(pos, mass, 1.0, 0.05, 0.5)
    stars = kind == 0
    assert np.array_equal(acc[stars], grav[stars])
    assert not np.array_equal(acc[~stars], grav[~stars])


def test_gas_star_mix_interleaves_gas(oracle):
    pos, vel, mass, kind = oracle.fixture_gas_star_mix(0x1111, 80, 160)
    assert kind.sum() == 80 and kind[0] == 1 and kind[1] == 0 and kind[3] == 1


def test_sph_params_defaults_from_the_library():
    # The C ABI's defaults are the reference's (forces.rs:75-86, density.rs:44-51).
    import galaxy_b200 as gb

    p = gb.sph_params()
    assert (p.n_ngb, p.h_tol_rel, p.eos, p.c_s, p.alpha, p.beta, p.visc_eps2) == (48.0, 1e-3, 0, 1.0, 1.0, 2.0, 0.01)
    assert gb.sph_params(eos="adiabatic", gamma=1.4).eos == 1
    with pytest.raises(TypeError):
        gb.sph_params(bogus=1)


def test_state_species_columns():
    import galaxy_b200 as gb

    st = gb.State(np.zeros((4, 3)), np.zeros((4, 3)), np.ones(4), kind=[1, 0, 1, 0])
    assert list(st.gas()) == [0, 2] and st.u.shape == (4,)
    with pytest.raises(ValueError):
        gb.State(np.zeros((4, 3)), np.zeros((4, 3)), np.ones(4), kind=[1, 0])


def test_active_path_semantics(oracle):
    # gravity_sph.rs:101-150, 247-286: the first call refreshes every gas particle (equal to
    # the full pass); later calls leave inactive gas rows at gravity alone.
    pos, vel, mass, kind = oracle.fixture_gas_star_mix(0xA5F0, 300, 600)
    full = oracle.GravitySph(1.0, 0.05, 0.5).accelerations(pos, vel, mass, kind)
    g = oracle.GravitySph(1.0, 0.05, 0.5)
    assert np.array_equal(g.accelerations_active(pos, vel, mass, kind, np.arange(len(pos))), full)
    act = np.arange(0, len(pos), 5)
    moved = pos + 1e-4
    a = g.accelerations_active(moved, vel, mass, kind, act)
    grav = oracle.lbvh_accelerations(moved, mass, 1.0, 0.05, 0.5)
    stale = np.setdiff1d(np.flatnonzero(kind == 1), act)
    assert np.array_equal(a[stale], grav[stale])
    fresh = np.intersect1d(np.flatnonzero(kind == 1), act)
    assert not np.array_equal(a[fresh], grav[fresh])


def test_coupled_pairs_against_brute_force(oracle):
    # cfl.rs:195-228: every pair with 0 < r < 2 max(h_a, h_b), once, ascending
    pos, vel, mass, kind = oracle.fixture_gas_star_mix(0x1111, 150, 300)
    pairs = oracle.sph_coupled_pairs(pos, mass, kind)
    gas = np.flatnonzero(kind == 1)
    _, h = oracle.sph_density_adaptive(pos[gas], mass[gas])
    want = []
    for a in range(gas.size):
        for b in range(a + 1, gas.size):
            r = np.sqrt(np.sum((pos[gas[a]] - pos[gas[b]]) ** 2))
            if 0.0 < r < 2.0 * max(h[a], h[b]):
                want.append((gas[a], gas[b]))
    assert np.array_equal(pairs, np.array(want, dtype=np.uint64).reshape(-1, 2))


def test_velocity_divergence_sign(oracle):
    # divergence.rs docs: a converging linear flow gives div v < 0, a diverging one > 0
    pos = oracle.fixture_sph_points(3, 800, 2.0)
    mass = np.ones(800)
    rho, h = oracle.sph_density_adaptive(pos, mass)
    assert np.all(oracle.sph_velocity_divergence(pos, -0.5 * pos, mass, rho, h) < 0)
    assert np.all(oracle.sph_velocity_divergence(pos, 0.5 * pos, mass, rho, h) > 0)
    kind = np.ones(800, np.uint8)
    kind[::2] = 0
    r, d = oracle.sph_sf_fields(pos, -0.5 * pos, mass, kind)
    assert not r[kind == 0].any() and not d[kind == 0].any() and np.all(r[kind == 1] > 0)


def test_cfl_vector_min_and_static_closed_form(oracle):
    # solvers/tests/sph_cfl_vector.rs:56-80, 153-180: the per-particle vector's min is the
    # scalar bound bit for bit; a static isothermal cloud has dt_i = c_cfl h_i / (2 c_s).
    pos = oracle.fixture_sph_points(21, 600, 2.5)
    vel = oracle.fixture_sph_points(22, 600, 1.5)
    kind = np.ones(600, np.uint8)
    m, vec = oracle.sph_max_stable_dt(pos, vel, np.ones(600), kind, 0.25, per_particle=True)
    assert vec.min() == m
    c_s = 2.0
    pos = oracle.fixture_sph_points(11, 800, 3.0)
    _, h = oracle.sph_density_adaptive(pos, np.ones(800))
    _, vec = oracle.sph_max_stable_dt(pos, np.zeros((800, 3)), np.ones(800), np.ones(800, np.uint8), 0.25,
                                      per_particle=True, eos=0, eos_param=c_s)
    assert np.max(np.abs(vec - 0.25 * h / (2.0 * c_s)) / (0.25 * h / (2.0 * c_s))) < 1e-9
