"""ctypes wrapper of the oracle library -- TEST INFRASTRUCTURE ONLY.

The oracle is a CPU f64 restatement of the galaxy reference's LBVH Barnes-Hut
path (solvers/src/lbvh.rs, solvers/src/direct_sum.rs, solvers/src/potential.rs,
core/src/integrator.rs, core/src/diagnostics.rs) in ``lbvh_oracle.cpp``, and of its
SPH toolkit and gravity + SPH composite (solvers/src/sph/*.rs) in ``sph_oracle.cpp``.  Only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use
it, always as the checker or the timed CPU baseline; the product library
``libgalaxy_b200.so`` never calls it.

Parity pinning: the Morton bit-spreading is pinned by the reference's
known-answer tests (solvers/src/lbvh.rs:691-726, in tests/golden/); the rest by
the reference's invariant tests (solvers/tests/lbvh.rs:88-312). The SPH restatement
is pinned by the reference's frozen output bits of hydro_accelerations
(solvers/tests/sph_forces.rs:393-462) and max_stable_dt (solvers/tests/sph_cfl.rs:189-212). Bitwise identity
with the Rust binary is unpinned beyond those (no Rust toolchain here).
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liblbvh_oracle.so")
_lib = None

_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


def build() -> None:
    """Compile the oracle with its Makefile (g++, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        sz, d, u64, i = C.c_size_t, C.c_double, C.c_uint64, C.c_int
        sig = {
            "or_expand10": (C.c_uint32, [C.c_uint32]),
            "or_morton3": (C.c_uint32, [C.c_uint32, C.c_uint32, C.c_uint32]),
            "or_reference_morton": (i, [sz, _f64p, C.c_void_p, _u32p, C.c_void_p]),
            "or_reference_sort": (None, [sz, _u32p, _u32p]),
            "or_reference_karras": (i, [sz, _u32p, _u32p, _u32p, _u32p]),
            "or_reference_aggregate": (i, [sz, _u32p, _u32p, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p]),
            "or_quadrupole": (i, [sz, _u32p, _u32p, _f64p, _f64p, _f64p]),
            "or_lbvh_flat": (i, [sz, _f64p, _f64p, _f64p, _u32p, _u32p]),
            "or_lbvh_accelerations": (i, [sz, _f64p, _f64p, d, d, d, _f64p, i, C.c_void_p]),
            "or_lbvh_accelerations_subset": (i, [sz, _f64p, _f64p, d, d, d, sz, _u32p, _f64p, i]),
            "or_lbvh_accelerations_stale": (i, [sz, _f64p, _f64p, _f64p, _f64p, d, d, d, sz, _u32p, _f64p, i]),
            "or_lbvh_accelerations_k63": (i, [sz, _f64p, _f64p, d, d, d, _f64p, i, C.c_void_p]),
            "or_lbvh_accelerations_quad": (i, [sz, _f64p, _f64p, d, d, d, _f64p, i]),
            "or_direct_sum": (None, [sz, _f64p, _f64p, d, d, _f64p]),
            "or_direct_sum_targets": (None, [sz, _f64p, _f64p, d, d, sz, _u32p, _f64p, i]),
            "or_potential_serial": (d, [sz, _f64p, _f64p, d, d]),
            "or_potential_parallel": (d, [sz, _f64p, _f64p, d, d, i]),
            "or_diagnostics": (None, [sz, _f64p, _f64p, _f64p, _f64p]),
            "or_kdk_lbvh": (i, [sz, _f64p, _f64p, _f64p, _f64p, C.POINTER(C.c_int), d, d, d, d, u64, i]),
            "or_fixture_cluster": (None, [u64, sz, _f64p, _f64p, _f64p]),
            "or_fixture_cloud": (None, [u64, sz, d, d, d, d, _f64p]),
            "or_fixture_masses": (None, [u64, sz, _f64p]),
            "or_fixture_random_codes": (None, [u64, sz, _u32p]),
            "or_openmp_max_threads": (i, []),
            # SPH (sph_oracle.cpp)
            "or_sph_w": (d, [d, d]),
            "or_sph_grad_w": (None, [d, d, d, d, _f64p]),
            "or_sph_neighbours": (sz, [sz, _f64p, d, _f64p, d, _u32p, sz]),
            "or_sph_reference_density": (None, [sz, _f64p, _f64p, _f64p, _f64p]),
            "or_sph_density_fixed": (None, [sz, _f64p, _f64p, _f64p, _f64p]),
            "or_sph_density_adaptive": (None, [sz, _f64p, _f64p, d, d, C.c_void_p, _f64p, _f64p, i]),
            "or_sph_density_seeds": (None, [sz, _f64p, d, _f64p, _f64p]),
            "or_sph_hydro": (None, [sz, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p, i, d, d, d, d, _f64p,
                                    C.c_void_p, i]),
            "or_sph_cfl_given_h": (None, [sz, _f64p, _f64p, _f64p, _f64p, i, d, d, _f64p, i]),
            "or_sph_max_stable_dt": (d, [sz, _f64p, _f64p, _f64p, _u8p, _f64p, i, d, d, d, d, C.c_void_p, i]),
            "or_gravity_sph_accelerations": (i, [sz, _f64p, _f64p, _f64p, _u8p, _f64p, d, d, d, i, d, d, d, d, d,
                                                 d, C.c_void_p, C.c_void_p, C.c_void_p, _f64p, i]),
            "or_kdk_gravity_sph": (i, [sz, _f64p, _f64p, _f64p, _u8p, _f64p, d, d, d, i, d, d, d, d, d, d,
                                       C.c_void_p, C.c_void_p, C.c_void_p, _f64p, C.POINTER(C.c_int), d, u64, i]),
            "or_gravity_sph_accelerations_active": (i, [sz, _f64p, _f64p, _f64p, _u8p, _f64p, d, d, d, i, d, d, d,
                                                        d, d, d, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                        sz, _u32p, _f64p, C.c_void_p, i]),
            "or_sph_velocity_divergence": (None, [sz, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p, i]),
            "or_sph_sf_fields": (None, [sz, _f64p, _f64p, _f64p, _u8p, d, d, _f64p, _f64p, i]),
            "or_sph_coupled_pairs": (sz, [sz, _f64p, _f64p, _u8p, d, d, _u64p, sz, i]),
            "or_fixture_gas_star_mix": (None, [u64, sz, sz, _f64p, _f64p, _f64p, _u8p]),
            "or_fixture_sph_points": (None, [u64, sz, d, d, _f64p]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _pos(a) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a.reshape(-1, 3)


def max_threads() -> int:
    return int(lib().or_openmp_max_threads())


# ---- Morton / sort / Karras / aggregate (solvers/src/lbvh.rs) -------------------------
def expand10(v: int) -> int:
    return int(lib().or_expand10(v))


def morton3(x: int, y: int, z: int) -> int:
    return int(lib().or_morton3(x, y, z))


def reference_morton(pos):
    """Returns (lanes [n,3] u32, codes [n] u32, bounds dict)."""
    pos = _pos(pos)
    n = pos.shape[0]
    lanes = np.zeros((n, 3), np.uint32)
    codes = np.zeros(n, np.uint32)
    b = np.zeros(5, np.float64)
    rc = lib().or_reference_morton(n, pos.reshape(-1), lanes.ctypes.data, codes, b.ctypes.data)
    if rc != 0:
        raise ValueError("reference_morton requires a non-empty system")
    return lanes, codes, {"bmin": b[:3].copy(), "size": float(b[3]), "scale": float(b[4])}


def reference_sort(codes) -> np.ndarray:
    codes = np.ascontiguousarray(codes, dtype=np.uint32)
    order = np.zeros(codes.shape[0], np.uint32)
    lib().or_reference_sort(codes.shape[0], codes, order)
    return order


def reference_karras(sorted_codes):
    """Returns (left [n-1], right [n-1], parent [2n-1]) in the unified index space."""
    sc = np.ascontiguousarray(sorted_codes, dtype=np.uint32)
    n = sc.shape[0]
    if n == 0:
        raise ValueError("reference_karras requires a non-empty system")
    left = np.zeros(max(n - 1, 1), np.uint32)
    right = np.zeros(max(n - 1, 1), np.uint32)
    parent = np.zeros(2 * n - 1, np.uint32)
    lib().or_reference_karras(n, sc, left, right, parent)
    return left[: n - 1], right[: n - 1], parent


def reference_aggregate(left, right, sorted_pos, sorted_mass):
    """Returns dict of aabb_min, aabb_max, com ([2n-1,3]) and mass ([2n-1])."""
    sp = _pos(sorted_pos)
    n = sp.shape[0]
    sm = np.ascontiguousarray(sorted_mass, dtype=np.float64)
    l = np.ascontiguousarray(left if n > 1 else [0], dtype=np.uint32)
    r = np.ascontiguousarray(right if n > 1 else [0], dtype=np.uint32)
    t = 2 * n - 1
    mn, mx, com = (np.zeros((t, 3)) for _ in range(3))
    mass = np.zeros(t)
    lib().or_reference_aggregate(n, l, r, sp.reshape(-1), sm, mn.reshape(-1), mx.reshape(-1), com.reshape(-1), mass)
    return {"aabb_min": mn, "aabb_max": mx, "com": com, "mass": mass}


def quadrupole(left, right, com, mass):
    n = (np.asarray(mass).shape[0] + 1) // 2
    l = np.ascontiguousarray(left if n > 1 else [0], dtype=np.uint32)
    r = np.ascontiguousarray(right if n > 1 else [0], dtype=np.uint32)
    q = np.zeros((2 * n - 1, 6))
    lib().or_quadrupole(n, l, r, np.ascontiguousarray(com, np.float64).reshape(-1),
                        np.ascontiguousarray(mass, np.float64), q.reshape(-1))
    return q


def lbvh_flat(pos, mass):
    """The DFS skip-pointer flat form (reference_flatten): (node_f64 [2n-1,11], node_u32 [2n-1,3], leaf_bodies)."""
    pos = _pos(pos)
    n = pos.shape[0]
    nf = np.zeros((2 * n - 1, 11))
    nu = np.zeros((2 * n - 1, 3), np.uint32)
    lb = np.zeros(n, np.uint32)
    lib().or_lbvh_flat(n, pos.reshape(-1), np.ascontiguousarray(mass, np.float64), nf.reshape(-1), nu.reshape(-1), lb)
    return nf, nu, lb


# ---- solvers ------------------------------------------------------------------------
def lbvh_accelerations(pos, mass, g, softening, theta, threads: int = 1, stats: bool = False):
    """Lbvh::accelerations (solvers/src/lbvh.rs:662-676). Returns acc [n,3] (and stats)."""
    pos = _pos(pos)
    n = pos.shape[0]
    acc = np.zeros((n, 3))
    st = np.zeros(3, np.uint64)
    lib().or_lbvh_accelerations(n, pos.reshape(-1), np.ascontiguousarray(mass, np.float64), g, softening, theta,
                                acc.reshape(-1), threads, st.ctypes.data if stats else None)
    if stats:
        return acc, {"leaf": int(st[0]), "far": int(st[1]), "open": int(st[2])}
    return acc


def lbvh_accelerations_k63(pos, mass, g, softening, theta, threads: int = 1, stats: bool = False):
    """The same solver over 63-bit Morton keys (extension; no reference counterpart)."""
    pos = _pos(pos)
    n = pos.shape[0]
    acc = np.zeros((n, 3))
    st = np.zeros(3, np.uint64)
    lib().or_lbvh_accelerations_k63(n, pos.reshape(-1), np.ascontiguousarray(mass, np.float64), g, softening, theta,
                                    acc.reshape(-1), threads, st.ctypes.data if stats else None)
    if stats:
        return acc, {"leaf": int(st[0]), "far": int(st[1]), "open": int(st[2])}
    return acc


def lbvh_accelerations_subset(pos, mass, g, softening, theta, targets, threads: int = 1):
    pos = _pos(pos)
    t = np.ascontiguousarray(targets, dtype=np.uint32)
    acc = np.zeros((t.shape[0], 3))
    lib().or_lbvh_accelerations_subset(pos.shape[0], pos.reshape(-1), np.ascontiguousarray(mass, np.float64), g,
                                       softening, theta, t.shape[0], t, acc.reshape(-1), threads)
    return acc


def lbvh_accelerations_stale(pos_build, mass_build, pos_now, mass_now, g, softening, theta, targets,
                             threads: int = 1):
    """Stale-tree walk (TreeGravity::gravity_active_cached semantics over the LBVH):
    the tree of (pos_build, mass_build), targets and leaf sources at (pos_now, mass_now)."""
    pb, pn = _pos(pos_build), _pos(pos_now)
    t = np.ascontiguousarray(targets, dtype=np.uint32)
    acc = np.zeros((t.shape[0], 3))
    lib().or_lbvh_accelerations_stale(pb.shape[0], pb.reshape(-1), np.ascontiguousarray(mass_build, np.float64),
                                      pn.reshape(-1), np.ascontiguousarray(mass_now, np.float64), g, softening,
                                      theta, t.shape[0], t, acc.reshape(-1), threads)
    return acc


def lbvh_accelerations_quad(pos, mass, g, softening, theta, threads: int = 1):
    pos = _pos(pos)
    n = pos.shape[0]
    acc = np.zeros((n, 3))
    lib().or_lbvh_accelerations_quad(n, pos.reshape(-1), np.ascontiguousarray(mass, np.float64), g, softening, theta,
                                     acc.reshape(-1), threads)
    return acc


def direct_sum(pos, mass, g, softening):
    """DirectSum::accelerations (solvers/src/direct_sum.rs:25-45), Newton-3 pairing."""
    pos = _pos(pos)
    n = pos.shape[0]
    acc = np.zeros((n, 3))
    lib().or_direct_sum(n, pos.reshape(-1), np.ascontiguousarray(mass, np.float64), g, softening, acc.reshape(-1))
    return acc


def direct_sum_targets(pos, mass, g, softening, targets, threads: int = 0):
    pos = _pos(pos)
    t = np.ascontiguousarray(targets, dtype=np.uint32)
    acc = np.zeros((t.shape[0], 3))
    lib().or_direct_sum_targets(pos.shape[0], pos.reshape(-1), np.ascontiguousarray(mass, np.float64), g, softening,
                                t.shape[0], t, acc.reshape(-1), threads or max_threads())
    return acc


def potential_serial(pos, mass, g, softening) -> float:
    pos = _pos(pos)
    return float(lib().or_potential_serial(pos.shape[0], pos.reshape(-1), np.ascontiguousarray(mass, np.float64), g,
                                           softening))


def potential_parallel(pos, mass, g, softening, threads: int = 0) -> float:
    pos = _pos(pos)
    return float(lib().or_potential_parallel(pos.shape[0], pos.reshape(-1), np.ascontiguousarray(mass, np.float64),
                                             g, softening, threads or max_threads()))


def diagnostics(pos, vel, mass):
    """core/src/diagnostics.rs: kinetic energy, momentum, angular momentum."""
    pos, vel = _pos(pos), _pos(vel)
    out = np.zeros(7)
    lib().or_diagnostics(pos.shape[0], pos.reshape(-1), vel.reshape(-1), np.ascontiguousarray(mass, np.float64), out)
    return {"kinetic": float(out[0]), "momentum": out[1:4].copy(), "angular_momentum": out[4:7].copy()}


class LeapfrogKdkLbvh:
    """LeapfrogKdk (core/src/integrator.rs:38-78) driving the Lbvh solver, in place on f64 arrays."""

    def __init__(self, g, softening, theta, threads: int = 1):
        self.g, self.softening, self.theta, self.threads = g, softening, theta, threads
        self.acc = None
        self.primed = C.c_int(0)

    def step_many(self, pos, vel, mass, dt, steps):
        n = pos.shape[0]
        if self.acc is None or self.acc.shape[0] != n:
            self.acc = np.zeros((n, 3))
            self.primed = C.c_int(0)
        if steps == 0:
            return
        lib().or_kdk_lbvh(n, pos.reshape(-1), vel.reshape(-1), np.ascontiguousarray(mass, np.float64),
                          self.acc.reshape(-1), C.byref(self.primed), self.g, self.softening, self.theta, dt, steps,
                          self.threads)

    def prime(self, pos, mass):
        """The integrator's first force evaluation (what its first step does before kicking)."""
        n = pos.shape[0]
        if self.acc is None or self.acc.shape[0] != n:
            self.acc = np.zeros((n, 3))
        if not self.primed.value:
            self.acc[:] = lbvh_accelerations(pos, mass, self.g, self.softening, self.theta, threads=self.threads)
            self.primed = C.c_int(1)


# ---- workloads -----------------------------------------------------------------------
# The seeded workload generator (galaxy_b200/csrc/gx_ic.cpp) is compiled into this
# library too, so the CPU baseline builds the benchmark's inputs without loading the
# product library. The two copies are the same source: identical inputs.
def _ic(name, n, *args):
    pos, vel, mass = np.empty((n, 3)), np.empty((n, 3)), np.empty(n)
    fn = getattr(lib(), name)
    fn.restype = C.c_int
    rc = fn(C.c_size_t(n), *args, pos.ctypes.data_as(C.c_void_p), vel.ctypes.data_as(C.c_void_p),
            mass.ctypes.data_as(C.c_void_p))
    if rc != 0:
        raise ValueError(f"{name} failed ({rc})")
    return pos, vel, mass


def ic_plummer(n: int, seed: int = 0, g: float = 1.0, total_mass: float = 1.0, scale_radius: float = 1.0):
    """(pos, vel, mass) of Plummer::sample (ic/src/plummer.rs:94-175)."""
    return _ic("gx_ic_plummer", n, C.c_uint64(seed), C.c_double(g), C.c_double(total_mass), C.c_double(scale_radius))


def ic_collision(n_total: int, seed: int = 0, mass_ratio: float = 1.0, pericentre: float = 4.0,
                 incl1_deg: float = 30.0, incl2_deg: float = 60.0):
    """(pos, vel, mass) of the two-galaxy collision workload."""
    return _ic("gx_ic_collision", n_total, C.c_uint64(seed), C.c_double(mass_ratio), C.c_double(pericentre),
               C.c_double(incl1_deg), C.c_double(incl2_deg))


# ---- reference test fixtures ---------------------------------------------------------
def fixture_cluster(seed: int, n: int):
    """solvers/tests/lbvh.rs:27-44: (pos, vel, mass)."""
    pos, vel, mass = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n)
    lib().or_fixture_cluster(seed, n, pos.reshape(-1), vel.reshape(-1), mass)
    return pos, vel, mass


def fixture_cloud(seed: int, n: int, r: float, center=(0.0, 0.0, 0.0)):
    """gpu/tests/lbvh_sort.rs:25-37."""
    pos = np.zeros((n, 3))
    lib().or_fixture_cloud(seed, n, r, float(center[0]), float(center[1]), float(center[2]), pos.reshape(-1))
    return pos


def fixture_masses(seed: int, n: int):
    """gpu/tests/lbvh_tree.rs:47-58."""
    m = np.zeros(n)
    lib().or_fixture_masses(seed, n, m)
    return m


def fixture_random_codes(seed: int, n: int):
    """gpu/tests/lbvh_sort.rs:41-51."""
    c = np.zeros(n, np.uint32)
    lib().or_fixture_random_codes(seed, n, c)
    return c


def cluster_with_coincident_knot():
    """solvers/tests/lbvh.rs:249-261: cluster(3, 60) plus 8 coincident particles."""
    pos, _, mass = fixture_cluster(3, 60)
    knot = np.tile([0.25, -0.1, 0.4], (8, 1))
    kmass = np.array([0.5 + 0.05 * k for k in range(8)])
    pos = np.vstack([pos, knot])
    mass = np.concatenate([mass, kmass])
    return pos, np.zeros_like(pos), mass


# ---- error metrics (solvers/tests/lbvh.rs:54-82) ---------------------------------------
def rms_accel(a) -> float:
    a = np.asarray(a)
    return max(float(np.sqrt(np.sum(a * a) / a.shape[0])), 1e-300)


def rms_rel_err(approx, exact) -> float:
    d = np.asarray(approx) - np.asarray(exact)
    return float(np.sqrt(np.sum(d * d) / d.shape[0])) / rms_accel(exact)


def worst_rel_err(approx, exact) -> float:
    d = np.asarray(approx) - np.asarray(exact)
    return float(np.max(np.sqrt(np.sum(d * d, axis=1)))) / rms_accel(exact)


def per_particle_rel_err(approx, exact) -> np.ndarray:
    """|a - a_ref| / |a_ref| per particle (the parity metric for median/p99)."""
    approx, exact = np.asarray(approx), np.asarray(exact)
    num = np.sqrt(np.sum((approx - exact) ** 2, axis=1))
    den = np.maximum(np.sqrt(np.sum(exact * exact, axis=1)), 1e-300)
    return num / den


# ---- SPH (solvers/src/sph) -------------------------------------------------------------
SPH_DEFAULTS = dict(n_ngb=48.0, h_tol_rel=1e-3, eos=0, eos_param=1.0, alpha=1.0, beta=2.0, visc_eps2=0.01)


def _sph(kw):
    p = dict(SPH_DEFAULTS)
    p.update(kw)
    return p


def sph_w(r: float, h: float) -> float:
    """kernel.rs:27-38."""
    return lib().or_sph_w(float(r), float(h))


def sph_grad_w(r_ij, h: float) -> np.ndarray:
    """kernel.rs:40-53."""
    out = np.zeros(3)
    lib().or_sph_grad_w(float(r_ij[0]), float(r_ij[1]), float(r_ij[2]), float(h), out)
    return out


def sph_neighbours(pos, center, r: float, cell: float = 0.0) -> np.ndarray:
    """HashGrid::neighbours_within (grid.rs:57-82) with cells of edge `cell`, or the
    brute-force reference_neighbours (reference.rs:10-18) when cell <= 0."""
    pos = _pos(pos)
    c = np.ascontiguousarray(center, dtype=np.float64)
    cap = pos.shape[0]
    out = np.zeros(max(cap, 1), dtype=np.uint32)
    k = lib().or_sph_neighbours(pos.shape[0], pos.reshape(-1), float(cell), c, float(r), out, cap)
    return out[:k].copy()


def sph_reference_density(pos, mass, h) -> np.ndarray:
    pos = _pos(pos)
    out = np.zeros(pos.shape[0])
    lib().or_sph_reference_density(pos.shape[0], pos.reshape(-1), np.ascontiguousarray(mass, np.float64),
                                   np.ascontiguousarray(h, np.float64), out)
    return out


def sph_density_fixed(pos, mass, h) -> np.ndarray:
    pos = _pos(pos)
    out = np.zeros(pos.shape[0])
    lib().or_sph_density_fixed(pos.shape[0], pos.reshape(-1), np.ascontiguousarray(mass, np.float64),
                               np.ascontiguousarray(h, np.float64), out)
    return out


def sph_density_adaptive(pos, mass, n_ngb=48.0, h_tol_rel=1e-3, h_init=None, threads: int = 0):
    """density_adaptive (density.rs:86-96): (rho, h)."""
    pos = _pos(pos)
    n = pos.shape[0]
    rho, h = np.zeros(n), np.zeros(n)
    hi = None if h_init is None else np.ascontiguousarray(h_init, dtype=np.float64)
    lib().or_sph_density_adaptive(n, pos.reshape(-1), np.ascontiguousarray(mass, np.float64), float(n_ngb),
                                  float(h_tol_rel), None if hi is None else hi.ctypes.data, rho, h,
                                  threads or max_threads())
    return rho, h


def sph_density_seeds(pos, n_ngb=48.0):
    """The per-particle bracket seeds and the cap of DensitySetup::new (density.rs:166-220)."""
    pos = _pos(pos)
    n = pos.shape[0]
    seeds, sc = np.zeros(n), np.zeros(4)
    lib().or_sph_density_seeds(n, pos.reshape(-1), float(n_ngb), seeds, sc)
    return seeds, float(sc[0])


def sph_hydro(pos, vel, mass, rho, h, u=None, threads: int = 0, **kw):
    """hydro_accel_and_dudt (forces.rs:160-172): (acc [n,3], dudt [n])."""
    p = _sph(kw)
    pos, vel = _pos(pos), _pos(vel)
    n = pos.shape[0]
    acc, dudt = np.zeros((n, 3)), np.zeros(n)
    uu = np.zeros(n) if u is None else np.ascontiguousarray(u, dtype=np.float64)
    lib().or_sph_hydro(n, pos.reshape(-1), vel.reshape(-1), np.ascontiguousarray(mass, np.float64),
                       np.ascontiguousarray(rho, np.float64), np.ascontiguousarray(h, np.float64), uu,
                       int(p["eos"]), float(p["eos_param"]), float(p["alpha"]), float(p["beta"]),
                       float(p["visc_eps2"]), acc.reshape(-1), dudt.ctypes.data, threads or max_threads())
    return acc, dudt


def sph_cfl_given_h(gpos, gvel, h, c_cfl, u=None, threads: int = 0, **kw) -> np.ndarray:
    """The per-particle CFL bound of cfl.rs:67-121 over a gas subset with given h."""
    p = _sph(kw)
    gpos, gvel = _pos(gpos), _pos(gvel)
    n = gpos.shape[0]
    out = np.zeros(n)
    uu = np.zeros(n) if u is None else np.ascontiguousarray(u, dtype=np.float64)
    lib().or_sph_cfl_given_h(n, gpos.reshape(-1), gvel.reshape(-1), np.ascontiguousarray(h, np.float64), uu,
                             int(p["eos"]), float(p["eos_param"]), float(c_cfl), out, threads or max_threads())
    return out


def sph_max_stable_dt(pos, vel, mass, kind, c_cfl, u=None, per_particle: bool = False, threads: int = 0, **kw):
    """max_stable_dt (cfl.rs:49-125); with per_particle, also the state-indexed vector of
    max_stable_dt_per_particle (cfl.rs:134-185)."""
    p = _sph(kw)
    pos, vel = _pos(pos), _pos(vel)
    n = pos.shape[0]
    uu = np.zeros(n) if u is None else np.ascontiguousarray(u, dtype=np.float64)
    vec = np.zeros(n) if per_particle else None
    m = lib().or_sph_max_stable_dt(n, pos.reshape(-1), vel.reshape(-1), np.ascontiguousarray(mass, np.float64),
                                   np.ascontiguousarray(kind, np.uint8), uu, int(p["eos"]), float(p["eos_param"]),
                                   float(p["n_ngb"]), float(p["h_tol_rel"]), float(c_cfl),
                                   None if vec is None else vec.ctypes.data, threads or max_threads())
    return (m, vec) if per_particle else m


def sph_velocity_divergence(pos, vel, mass, rho, h, threads: int = 0) -> np.ndarray:
    """divergence.rs:34-72 over a gas subset with given rho / h."""
    pos, vel = _pos(pos), _pos(vel)
    out = np.zeros(pos.shape[0])
    lib().or_sph_velocity_divergence(pos.shape[0], pos.reshape(-1), vel.reshape(-1),
                                     np.ascontiguousarray(mass, np.float64), np.ascontiguousarray(rho, np.float64),
                                     np.ascontiguousarray(h, np.float64), out, threads or max_threads())
    return out


def sph_sf_fields(pos, vel, mass, kind, n_ngb=48.0, h_tol_rel=1e-3, threads: int = 0):
    """GravitySph::sf_fields (gravity_sph.rs:353-382): state-indexed (rho, div_v)."""
    pos, vel = _pos(pos), _pos(vel)
    n = pos.shape[0]
    rho, dv = np.zeros(n), np.zeros(n)
    lib().or_sph_sf_fields(n, pos.reshape(-1), vel.reshape(-1), np.ascontiguousarray(mass, np.float64),
                           np.ascontiguousarray(kind, np.uint8), float(n_ngb), float(h_tol_rel), rho, dv,
                           threads or max_threads())
    return rho, dv


def sph_coupled_pairs(pos, mass, kind, n_ngb=48.0, h_tol_rel=1e-3, threads: int = 0) -> np.ndarray:
    """cfl.rs:195-228 coupled_pairs: [P, 2] global index pairs, ascending."""
    pos = _pos(pos)
    n = pos.shape[0]
    args = (n, pos.reshape(-1), np.ascontiguousarray(mass, np.float64), np.ascontiguousarray(kind, np.uint8),
            float(n_ngb), float(h_tol_rel))
    cap = 64 * max(n, 1)
    out = np.zeros(2 * cap, dtype=np.uint64)
    k = lib().or_sph_coupled_pairs(*args, out, cap, threads or max_threads())
    if k > cap:
        out = np.zeros(2 * k, dtype=np.uint64)
        k = lib().or_sph_coupled_pairs(*args, out, k, threads or max_threads())
    return out[:2 * k].reshape(-1, 2).copy()


class GravitySph:
    """GravitySph (gravity_sph.rs:24-207) over the Lbvh gravity solver: gravity on every
    particle, hydro on the gas rows (kind == 1), h warm-started across calls. g <= 0
    turns gravity off (the reference's hydro_only)."""

    def __init__(self, g, softening, theta, threads: int = 0, **kw):
        self.g, self.softening, self.theta = g, softening, theta
        self.p = _sph(kw)
        self.threads = threads or max_threads()
        self.h_hint = None
        self.h_valid = C.c_int(0)
        self.rho = None
        self.acc = None
        self.primed = C.c_int(0)

    def _hint(self, n_gas):
        if self.h_hint is None or self.h_hint.shape[0] != n_gas:
            self.h_hint = np.zeros(max(n_gas, 1))
            self.rho = np.zeros(max(n_gas, 1))
            self.h_valid = C.c_int(0)

    def _args(self):
        p = self.p
        return (float(self.g), float(self.softening), float(self.theta), int(p["eos"]), float(p["eos_param"]),
                float(p["alpha"]), float(p["beta"]), float(p["visc_eps2"]), float(p["n_ngb"]), float(p["h_tol_rel"]))

    def accelerations(self, pos, vel, mass, kind, u=None) -> np.ndarray:
        pos, vel = _pos(pos), _pos(vel)
        n = pos.shape[0]
        kind = np.ascontiguousarray(kind, np.uint8)
        self._hint(int((kind == 1).sum()))
        acc = np.zeros((n, 3))
        uu = np.zeros(n) if u is None else np.ascontiguousarray(u, dtype=np.float64)
        lib().or_gravity_sph_accelerations(n, pos.reshape(-1), vel.reshape(-1), np.ascontiguousarray(mass, np.float64),
                                           kind, uu, *self._args(), self.h_hint.ctypes.data,
                                           C.addressof(self.h_valid), self.rho.ctypes.data, acc.reshape(-1),
                                           self.threads)
        return acc

    def accelerations_active(self, pos, vel, mass, kind, active, u=None) -> np.ndarray:
        """GravitySph::accelerations_active (gravity_sph.rs:247-286): fresh gravity on all,
        hydro on the active gas targets from the persistent (rho, h) scratch."""
        return self.accel_and_dudt_active(pos, vel, mass, kind, active, u)[0]

    def accel_and_dudt_active(self, pos, vel, mass, kind, active, u=None):
        """GravitySph::accel_and_dudt_active (gravity_sph.rs:288-319): (acc, dudt), du/dt
        set on the active gas rows (all gas when the scratch was refreshed), zero elsewhere."""
        pos, vel = _pos(pos), _pos(vel)
        n = pos.shape[0]
        kind = np.ascontiguousarray(kind, np.uint8)
        ng = int((kind == 1).sum())
        self._hint(ng)
        if getattr(self, "rho_scratch", None) is None or self.rho_scratch.shape[0] != max(ng, 1):
            self.rho_scratch = np.zeros(max(ng, 1))
            self.rho_valid = C.c_int(0)
        acc = np.zeros((n, 3))
        dudt = np.zeros(n)
        uu = np.zeros(n) if u is None else np.ascontiguousarray(u, dtype=np.float64)
        act = np.ascontiguousarray(active, dtype=np.uint32)
        lib().or_gravity_sph_accelerations_active(n, pos.reshape(-1), vel.reshape(-1),
                                                  np.ascontiguousarray(mass, np.float64), kind, uu, *self._args(),
                                                  self.h_hint.ctypes.data, C.addressof(self.h_valid),
                                                  self.rho_scratch.ctypes.data, C.addressof(self.rho_valid),
                                                  act.shape[0], act, acc.reshape(-1), dudt.ctypes.data, self.threads)
        return acc, dudt

    def step_many(self, pos, vel, mass, kind, dt, steps, u=None):
        """LeapfrogKdk (integrator.rs:38-78) driving this composite, in place."""
        n = pos.shape[0]
        kind = np.ascontiguousarray(kind, np.uint8)
        self._hint(int((kind == 1).sum()))
        if self.acc is None or self.acc.shape[0] != n:
            self.acc = np.zeros((n, 3))
            self.primed = C.c_int(0)
        uu = np.zeros(n) if u is None else np.ascontiguousarray(u, dtype=np.float64)
        lib().or_kdk_gravity_sph(n, pos.reshape(-1), vel.reshape(-1), np.ascontiguousarray(mass, np.float64), kind, uu,
                                 *self._args(), self.h_hint.ctypes.data, C.addressof(self.h_valid),
                                 self.rho.ctypes.data, self.acc.reshape(-1), C.byref(self.primed), float(dt),
                                 int(steps), self.threads)


def fixture_gas_star_mix(seed: int, n_gas: int, n_star: int):
    """gpu/tests/gpu_resident_sph.rs:38-96: (pos, vel, mass, kind), gas interleaved."""
    n = n_gas + n_star
    pos, vel, mass, kind = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n), np.zeros(n, dtype=np.uint8)
    lib().or_fixture_gas_star_mix(seed, n_gas, n_star, pos.reshape(-1), vel.reshape(-1), mass, kind)
    return pos, vel, mass, kind


def fixture_sph_points(seed: int, n: int, scale: float, centered: bool = True) -> np.ndarray:
    """The SPH tests' random_points: (u - 0.5) * scale when centered (sph_forces.rs:18-29,
    sph_cfl.rs:10-21), u * scale otherwise (sph_density.rs:15-27)."""
    pos = np.zeros((n, 3))
    lib().or_fixture_sph_points(seed, n, float(scale), 0.5 if centered else 0.0, pos.reshape(-1))
    return pos
