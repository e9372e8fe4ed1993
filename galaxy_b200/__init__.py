"""galaxy_b200 -- B200 (sm_100a) LBVH Barnes-Hut gravity step behind galaxy's solver API.

Host-side mirror of the reference interfaces (paths relative to the reference
project root), each a thin layer over the C ABI of ``libgalaxy_b200.so``:

* :class:`State` -- ``core/src/state.rs:29`` (SoA f64 pos/vel/mass, time).
* :class:`ForceSolver` -- ``core/src/traits.rs:24-157``: ``accelerations(state, acc)``
  and ``potential_energy(state)``.
* :class:`GpuLbvh` -- the drop-in GPU backend, ``gpu/src/gpu_lbvh_fused.rs:44-146``
  (``Lbvh::new(g, softening, theta)`` semantics, ``solvers/src/lbvh.rs:643-683``).
* :class:`LeapfrogKdk` -- ``core/src/integrator.rs:6-78``.
* :class:`GpuResidentLeapfrog` -- ``gpu/src/gpu_resident.rs:1685-1960``
  (upload / step / step_many / snapshot / time / len / submits).
* :class:`Batch` -- many independent systems stepped by one launch per stage.
* :class:`GpuGravitySph` -- ``solvers/src/sph/gravity_sph.rs`` (gravity + SPH on the gas
  rows), and the resident gas mode of :class:`GpuResidentLeapfrog`
  (``gpu_resident.rs:1393-1660``: ``new_with_sph``, ``snapshot_gas_density``,
  ``snapshot_gas_accel``, ``min_stable_dt``, ``snapshot_gas_dt``, ``snapshot_accel``).
* stage functions ``stage_morton`` / ``stage_sort`` / ``stage_build`` -- the
  ``reference_*`` oracles' GPU counterparts (``solvers/src/lbvh.rs:105-348``).

Errors follow the reference's conventions: constructors raise on a missing device
(``GpuError``), a length mismatch raises like the reference's ``assert_eq!``.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import (GX_FLAG_MORTON63, GX_FLAG_NO_KAHAN, GX_FLAG_STAGE_TIMES, GX_FLAG_STATS, GX_MULTIPOLE_MONO,
                   GX_MULTIPOLE_QUAD, GX_PREC_F32, GX_PREC_F64, GxError, check, lib)

__all__ = [
    "State", "ForceSolver", "GpuLbvh", "GpuStaleTreeGravity", "GpuGravitySph", "LeapfrogKdk", "GpuResidentLeapfrog",
    "Batch", "sph_params", "GasDensity", "GasCfl", "GAS", "COLLISIONLESS",
    "Server", "GxError",
    "PinnedState",
    "stage_morton",
    "stage_sort", "stage_build", "device_info", "device_synchronize", "ic", "tuning_lookup",
]


def _f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        a = a.reshape(shape)
    return a


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


GAS, COLLISIONLESS = 1, 0  # core/src/state.rs:17-22 Species


@dataclass
class State:
    """core/src/state.rs:29 -- positions/velocities [n,3] f64, masses [n] f64, time; the
    species column ``kind`` [n] u8 (1 = gas) and internal energy ``u`` [n] f64."""

    pos: np.ndarray
    vel: np.ndarray
    mass: np.ndarray
    time: float = 0.0
    kind: np.ndarray = None
    u: np.ndarray = None

    def __post_init__(self):
        self.pos = _f64(self.pos).reshape(-1, 3)
        self.vel = _f64(self.vel).reshape(-1, 3)
        self.mass = _f64(self.mass).reshape(-1)
        n = self.pos.shape[0]
        if self.vel.shape[0] != n or self.mass.shape[0] != n:
            raise ValueError("vel/mass length must match pos")
        self.kind = (np.zeros(n, dtype=np.uint8) if self.kind is None
                     else np.ascontiguousarray(self.kind, dtype=np.uint8).reshape(-1))
        self.u = np.zeros(n) if self.u is None else _f64(self.u).reshape(-1)
        if self.kind.shape[0] != n or self.u.shape[0] != n:
            raise ValueError("kind/u length must match pos")

    def __len__(self):
        return self.pos.shape[0]

    def copy(self) -> "State":
        return State(self.pos.copy(), self.vel.copy(), self.mass.copy(), self.time, self.kind.copy(), self.u.copy())

    def gas(self) -> np.ndarray:
        """Indices of the gas rows, ascending."""
        return np.flatnonzero(self.kind == GAS).astype(np.uint32)


class ForceSolver:
    """core/src/traits.rs:24-157 (the gravity part of the trait, with its defaults)."""

    def accelerations(self, state: State, acc: np.ndarray) -> None:
        raise NotImplementedError

    def accelerations_active(self, state: State, active, acc: np.ndarray):
        """traits.rs:52-54 default: the full pass (rows outside ``active`` unspecified)."""
        return self.accelerations(state, acc)

    def rebuild_gravity_cache(self, state: State) -> None:
        """traits.rs:78 default: nothing to cache."""

    def gravity_active_cached(self, state: State, active, acc: np.ndarray):
        """traits.rs:89-91 default: a fresh full pass."""
        return self.accelerations(state, acc)

    def max_stable_dt(self, state: State) -> float:
        """traits.rs:106-108 default: pure gravity imposes no step limit."""
        return float("inf")

    def potential_energy(self, state: State) -> float:
        raise NotImplementedError


def _options(precision: str, multipole: str, kahan: bool, stats: bool, device: int, walk_block: int,
             stage_times: bool = False, walk_ctas_per_sm: int = 0, morton63: bool = False, walk_group: int = 0,
             radix_bits: int = 0):
    o = _lib.Options()
    o.struct_size = C.sizeof(_lib.Options)
    o.precision = {"f32": GX_PREC_F32, "f64": GX_PREC_F64}[precision]
    o.multipole = {"mono": GX_MULTIPOLE_MONO, "quad": GX_MULTIPOLE_QUAD}[multipole]
    o.flags = ((0 if kahan else GX_FLAG_NO_KAHAN) | (GX_FLAG_STATS if stats else 0) |
               (GX_FLAG_STAGE_TIMES if stage_times else 0) | (GX_FLAG_MORTON63 if morton63 else 0))
    o.device = device
    o.walk_block = walk_block
    o.walk_ctas_per_sm = walk_ctas_per_sm
    o.walk_group = walk_group
    o.radix_bits = radix_bits
    return o


class _Handle:
    def __init__(self, g, softening, theta, precision="f32", multipole="mono", kahan=True, stats=False, device=-1,
                 walk_block=0, stage_times=False, walk_ctas_per_sm=0, morton63=False, walk_group=0, radix_bits=0):
        self.g, self.softening, self.theta = float(g), float(softening), float(theta)
        self._h = C.c_void_p()
        o = _options(precision, multipole, kahan, stats, device, walk_block, stage_times, walk_ctas_per_sm, morton63,
                     walk_group, radix_bits)
        rc = lib().gx_create(self.g, self.softening, self.theta, C.byref(o), C.byref(self._h))
        if rc != 0:
            check(rc, None)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().gx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        check(rc, self._h)

    def stats(self) -> dict:
        s = _lib.Stats()
        self._ck(lib().gx_get_stats(self._h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in s._fields_}


class GpuLbvh(_Handle, ForceSolver):
    """Drop-in GPU ForceSolver (gpu/src/gpu_lbvh_fused.rs:44-146) over libgalaxy_b200.

    precision: "f32" (FP32 walk, Kahan-compensated, opening decisions guarded in
    FP64) or "f64" (the reference's arithmetic, bit-identical to Lbvh on the CPU).
    multipole: "mono" (the reference) or "quad" (adds node quadrupoles).
    """

    def accelerations(self, state, acc=None, mass=None):
        """Fill acc[n,3] (or return a new array) with the acceleration of each particle.

        Accepts a State, or positions [n,3] plus ``mass``.
        """
        if isinstance(state, State):
            pos, m = state.pos, state.mass
        else:
            pos, m = _f64(state).reshape(-1, 3), _f64(mass).reshape(-1)
        n = pos.shape[0]
        out = acc if acc is not None else np.empty((n, 3))
        if out.shape != (n, 3) or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("acc length must match particle count (C-contiguous f64 [n,3])")
        self._ck(lib().gx_accelerations(self._h, n, _ptr(pos), _ptr(m), _ptr(out)))
        return out

    def accelerations_active(self, state, active, acc=None, mass=None):
        """ForceSolver::accelerations_active (core/src/traits.rs:52-54): fill acc[i] for
        i in ``active`` with what ``accelerations`` gives particle i, walking the tree for
        those targets only; other rows of ``acc`` are left as they are."""
        if isinstance(state, State):
            pos, m = state.pos, state.mass
        else:
            pos, m = _f64(state).reshape(-1, 3), _f64(mass).reshape(-1)
        n = pos.shape[0]
        out = acc if acc is not None else np.zeros((n, 3))
        if out.shape != (n, 3) or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("acc length must match particle count (C-contiguous f64 [n,3])")
        idx = np.ascontiguousarray(active, dtype=np.int64).reshape(-1)
        if idx.size and (idx.min() < 0 or idx.max() >= n):
            raise ValueError("active index out of range")
        idx = idx.astype(np.uint32)
        self._ck(lib().gx_accelerations_active(self._h, n, _ptr(pos), _ptr(m), idx.size, _ptr(idx), _ptr(out)))
        return out

    def rebuild_gravity_cache(self, state) -> None:
        """ForceSolver::rebuild_gravity_cache (core/src/traits.rs:78): Lbvh caches nothing."""

    def gravity_active_cached(self, state, active, acc=None, mass=None):
        """ForceSolver::gravity_active_cached (core/src/traits.rs:89-91), which Lbvh keeps
        at its default: the accelerations of a fresh pass, here for the active targets."""
        return self.accelerations_active(state, active, acc, mass)

    def potential_energy(self, state, mass=None) -> float:
        pos, m = (state.pos, state.mass) if isinstance(state, State) else (_f64(state).reshape(-1, 3), _f64(mass))
        out = C.c_double()
        self._ck(lib().gx_potential_energy(self._h, pos.shape[0], _ptr(pos), _ptr(m), C.byref(out)))
        return out.value

    def kdk_step_host(self, st: "PinnedState", dt: float, primed: bool) -> bool:
        """One LeapfrogKdk step (core/src/integrator.rs:38-78) on host arrays, this solver
        computing the accelerations. Returns the integrator's primed flag."""
        p = C.c_int(1 if primed else 0)
        self._ck(lib().gx_kdk_step_host(self._h, len(st), _ptr(st.pos), _ptr(st.vel), _ptr(st.mass), _ptr(st.acc),
                                        C.byref(p), float(dt)))
        st.time += dt
        return bool(p.value)

    def direct_sum_f64(self, pos, mass, targets=None):
        """FP64 direct summation on the GPU (the large-N force oracle)."""
        pos, mass = _f64(pos).reshape(-1, 3), _f64(mass)
        t = None if targets is None else np.ascontiguousarray(targets, dtype=np.uint32)
        nt = pos.shape[0] if t is None else t.shape[0]
        out = np.empty((nt, 3))
        self._ck(lib().gx_direct_sum_f64(self._h, pos.shape[0], _ptr(pos), _ptr(mass), nt, _ptr(t), _ptr(out)))
        return out


class GpuStaleTreeGravity(GpuLbvh):
    """TreeGravity's stale-tree active walk (solvers/src/barnes_hut.rs:647-711) over the
    LBVH: ``rebuild_gravity_cache`` freezes the tree at the block-start state;
    ``gravity_active_cached`` walks it for the active targets at the current positions
    (leaf sources current, internal aggregates frozen); ``accelerations`` is a fresh
    full pass, on a second handle so that it leaves the cache alone."""

    def __init__(self, g, softening, theta, **kw):
        super().__init__(g, softening, theta, **kw)
        self._kw = dict(kw)
        self._fresh = None
        self._cached = False

    def accelerations(self, state, acc=None, mass=None):
        if self._fresh is None:
            self._fresh = GpuLbvh(self.g, self.softening, self.theta, **self._kw)
        return self._fresh.accelerations(state, acc, mass)

    def rebuild_gravity_cache(self, state, mass=None) -> None:
        pos, m = (state.pos, state.mass) if isinstance(state, State) else (_f64(state).reshape(-1, 3), _f64(mass))
        self._ck(lib().gx_rebuild_gravity_cache(self._h, pos.shape[0], _ptr(pos), _ptr(m)))
        self._cached = pos.shape[0] > 0  # an empty system has no tree (the reference's None)

    def gravity_active_cached(self, state, active, acc=None, mass=None):
        if isinstance(state, State):
            pos, m = state.pos, state.mass
        else:
            pos, m = _f64(state).reshape(-1, 3), _f64(mass).reshape(-1)
        n = pos.shape[0]
        out = acc if acc is not None else np.zeros((n, 3))
        if out.shape != (n, 3) or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("acc length must match particle count (C-contiguous f64 [n,3])")
        if not self._cached:
            return out  # never rebuilt (or empty): nothing to walk, as the reference
        idx = np.ascontiguousarray(active, dtype=np.int64).reshape(-1)
        if idx.size and (idx.min() < 0 or idx.max() >= n):
            raise ValueError("active index out of range")
        idx = idx.astype(np.uint32)
        self._ck(lib().gx_gravity_active_cached(self._h, n, _ptr(pos), _ptr(m), idx.size, _ptr(idx), _ptr(out)))
        return out


class GpuGravitySph(GpuLbvh):
    """GravitySph (solvers/src/sph/gravity_sph.rs:24-402) over this library's LBVH gravity:
    gravity on every particle, density, smoothing lengths and the hydro force on the gas
    rows (``state.kind == 1``), h warm-started across calls while the gas count holds.
    SPH parameters as :func:`sph_params` keywords (``sph=dict(...)``)."""

    def __init__(self, g, softening, theta, sph=None, **kw):
        super().__init__(g, softening, theta, **kw)
        self.params = sph_params(**(sph or {}))
        self._ck(lib().gx_sph_enable(self._h, C.byref(self.params)))

    def accelerations(self, state, acc=None):
        n = len(state)
        if acc is None:
            acc = np.empty((n, 3))
        elif acc.shape != (n, 3) or not acc.flags.c_contiguous or acc.dtype != np.float64:
            raise ValueError("acc length must match particle count (C-contiguous f64 [n,3])")
        self._ck(lib().gx_sph_accelerations(self._h, n, _ptr(state.pos), _ptr(state.vel), _ptr(state.mass),
                                            _ptr(state.kind), _ptr(state.u), _ptr(acc)))
        return acc

    def accelerations_active(self, state, active, acc=None):
        """GravitySph::accelerations_active (gravity_sph.rs:247-286): gravity of every
        particle, then density and hydro for the active gas particles only, from the
        persistent (rho, h) scratch (inactive neighbours read stale, as the reference)."""
        n = len(state)
        acc = np.empty((n, 3)) if acc is None else acc
        act = np.ascontiguousarray(active, dtype=np.uint32)
        self._ck(lib().gx_sph_accelerations_active(self._h, n, _ptr(state.pos), _ptr(state.vel), _ptr(state.mass),
                                                   _ptr(state.kind), _ptr(state.u), act.shape[0], _ptr(act),
                                                   _ptr(acc)))
        return acc

    def accel_and_dudt_active(self, state, active, acc=None, dudt=None):
        """GravitySph::accel_and_dudt_active (gravity_sph.rs:288-319): (acc, dudt) of the
        active path; dudt zero except on the refreshed gas rows."""
        n = len(state)
        acc = np.empty((n, 3)) if acc is None else acc
        dudt = np.empty(n) if dudt is None else dudt
        act = np.ascontiguousarray(active, dtype=np.uint32)
        self._ck(lib().gx_sph_accel_and_dudt_active(self._h, n, _ptr(state.pos), _ptr(state.vel), _ptr(state.mass),
                                                    _ptr(state.kind), _ptr(state.u), act.shape[0], _ptr(act),
                                                    _ptr(acc), _ptr(dudt)))
        return acc, dudt

    def rebuild_gravity_cache(self, state) -> None:
        """GravitySph::rebuild_gravity_cache (gravity_sph.rs:321-327) delegates to its
        gravity solver, Lbvh, which caches nothing."""

    def gravity_active_cached(self, state, active, acc=None, mass=None):
        """GravitySph::gravity_active_cached (gravity_sph.rs:329-341): the gravity-ONLY walk
        (no hydro), Lbvh's default -- a fresh pass, here for the active targets."""
        return GpuLbvh.accelerations_active(self, state, active, acc, mass)

    def sf_fields(self, state):
        """GravitySph::sf_fields (gravity_sph.rs:353-382): state-indexed (rho, div_v) from a
        cold-start density solve; zero on collisionless rows."""
        n = len(state)
        rho, dv = np.zeros(n), np.zeros(n)
        self._ck(lib().gx_sph_sf_fields(self._h, n, _ptr(state.pos), _ptr(state.vel), _ptr(state.mass),
                                        _ptr(state.kind), _ptr(rho), _ptr(dv)))
        return rho, dv

    def coupled_pairs(self, state) -> np.ndarray:
        """GravitySph::coupled_pairs (cfl.rs:195-228): [P, 2] global index pairs, ascending."""
        n = len(state)
        cap = 64 * max(n, 1)
        out = np.zeros(2 * cap, dtype=np.uint64)
        k = C.c_size_t()
        args = (self._h, n, _ptr(state.pos), _ptr(state.mass), _ptr(state.kind))
        self._ck(lib().gx_sph_coupled_pairs(*args, _ptr(out), cap, C.byref(k)))
        if k.value > cap:
            out = np.zeros(2 * k.value, dtype=np.uint64)
            self._ck(lib().gx_sph_coupled_pairs(*args, _ptr(out), k.value, C.byref(k)))
        return out[:2 * k.value].reshape(-1, 2).copy()

    def accel_and_dudt(self, state, acc=None, dudt=None):
        """ForceSolver::accel_and_dudt of GravitySph (gravity_sph.rs:209-245): (acc [n,3],
        dudt [n], zero on collisionless rows)."""
        n = len(state)
        acc = np.empty((n, 3)) if acc is None else acc
        dudt = np.empty(n) if dudt is None else dudt
        self._ck(lib().gx_sph_accel_and_dudt(self._h, n, _ptr(state.pos), _ptr(state.vel), _ptr(state.mass),
                                             _ptr(state.kind), _ptr(state.u), _ptr(acc), _ptr(dudt)))
        return acc, dudt

    def density(self, pos, mass, h_init=None):
        """density_adaptive (density.rs:86-96) over gas positions: (rho, h)."""
        pos, mass = _f64(pos).reshape(-1, 3), _f64(mass).reshape(-1)
        n = pos.shape[0]
        rho, h = np.zeros(n), np.zeros(n)
        hi = None if h_init is None else _f64(h_init).reshape(-1)
        self._ck(lib().gx_sph_density(self._h, n, _ptr(pos), _ptr(mass), _ptr(hi), _ptr(rho), _ptr(h)))
        return rho, h

    def hydro(self, pos, vel, mass, rho, h, u=None):
        """hydro_accel_and_dudt (forces.rs:160-172): (acc [n,3], dudt [n])."""
        pos, vel = _f64(pos).reshape(-1, 3), _f64(vel).reshape(-1, 3)
        n = pos.shape[0]
        acc, dudt = np.zeros((n, 3)), np.zeros(n)
        uu = None if u is None else _f64(u).reshape(-1)
        self._ck(lib().gx_sph_hydro(self._h, n, _ptr(pos), _ptr(vel), _ptr(_f64(mass)), _ptr(_f64(rho)),
                                    _ptr(_f64(h)), _ptr(uu), _ptr(acc), _ptr(dudt)))
        return acc, dudt

    def cfl(self, pos, vel, h, c_cfl, u=None):
        """The per-particle CFL bound (cfl.rs:134-185 body) with given h: (dt [n], min)."""
        pos, vel = _f64(pos).reshape(-1, 3), _f64(vel).reshape(-1, 3)
        n = pos.shape[0]
        dt, m = np.zeros(n), C.c_double()
        uu = None if u is None else _f64(u).reshape(-1)
        self._ck(lib().gx_sph_cfl(self._h, n, _ptr(pos), _ptr(vel), _ptr(_f64(h)), _ptr(uu), float(c_cfl),
                                  _ptr(dt), C.byref(m)))
        return dt, m.value

    def max_stable_dt_per_particle(self, state, c_cfl: float = 1.0) -> np.ndarray:
        """cfl.rs:134-185 (gravity_sph.rs:380-386 at Courant number 1): state-indexed,
        +inf on collisionless rows; h from a cold-start density solve."""
        out = np.empty(len(state))
        m = C.c_double()
        self._ck(lib().gx_sph_max_stable_dt(self._h, len(state), _ptr(state.pos), _ptr(state.vel),
                                            _ptr(state.mass), _ptr(state.kind), _ptr(state.u), float(c_cfl),
                                            _ptr(out), C.byref(m)))
        return out

    def max_stable_dt(self, state, c_cfl: float = 1.0) -> float:
        """ForceSolver::max_stable_dt of GravitySph (gravity_sph.rs:371-378; cfl.rs:49-125),
        reduced on the device."""
        m = C.c_double()
        self._ck(lib().gx_sph_max_stable_dt(self._h, len(state), _ptr(state.pos), _ptr(state.vel),
                                            _ptr(state.mass), _ptr(state.kind), _ptr(state.u), float(c_cfl),
                                            None, C.byref(m)))
        return m.value


class LeapfrogKdk:
    """core/src/integrator.rs:6-78 -- kick-drift-kick with cached accelerations (host arrays)."""

    def __init__(self):
        self.acc = np.zeros((0, 3))
        self.primed = False

    def reset(self):
        self.acc = np.zeros((0, 3))
        self.primed = False

    def prime(self, state: State, solver: ForceSolver):
        self.acc = np.zeros((len(state), 3))
        solver.accelerations(state, self.acc)
        self.primed = True

    def step(self, state: State, solver: ForceSolver, dt: float):
        n = len(state)
        if self.acc.shape[0] != n:
            self.acc = np.zeros((n, 3))
            self.primed = False
        if not self.primed:
            solver.accelerations(state, self.acc)
            self.primed = True
        half = 0.5 * dt
        state.vel += self.acc * half
        state.pos += state.vel * dt
        solver.accelerations(state, self.acc)
        state.vel += self.acc * half
        state.time += dt


def sph_params(**kw) -> "_lib.SphParams":
    """HydroParams (solvers/src/sph/forces.rs:64-87) + DensityConfig (density.rs:33-51) as
    the C struct: the reference defaults, overridden by keyword (n_ngb, h_tol_rel, eos
    "isothermal" / "adiabatic", c_s, gamma, alpha, beta, visc_eps2, warm_start)."""
    p = _lib.SphParams()
    lib().gx_sph_default_params(C.byref(p))
    for k, v in kw.items():
        if k == "eos":
            v = {"isothermal": _lib.GX_EOS_ISOTHERMAL, "adiabatic": _lib.GX_EOS_ADIABATIC}.get(v, v)
        if not hasattr(p, k):
            raise TypeError(f"unknown SPH parameter {k}")
        setattr(p, k, int(v) if k in ("eos", "warm_start") else float(v))
    return p


@dataclass
class GasDensity:
    """gpu_resident.rs GasDensity: the gas map and its (rho, h), ascending gas index."""

    gas_idx: np.ndarray
    rho: np.ndarray
    h: np.ndarray


@dataclass
class GasCfl:
    gas_idx: np.ndarray
    dt: np.ndarray


class GpuResidentLeapfrog(_Handle):
    """gpu/src/gpu_resident.rs:1685-1960 -- state kept on the device across KDK steps.

    ``sph`` (a dict of :func:`sph_params` keywords, or True for the defaults) is
    ``new_with_sph`` (gpu_resident.rs:1393): gas mode, SPH on the ``kind == 1`` rows."""

    MAX_BATCH = 64  # the reference's submit cap; steps here are graph launches, not submits

    def __init__(self, g, softening, theta, sph=None, **kw):
        super().__init__(g, softening, theta, **kw)
        self._mass = np.zeros(0)
        self._kind = np.zeros(0, dtype=np.uint8)
        self._u = np.zeros(0)
        self.gas_mode = sph is not None and sph is not False
        if self.gas_mode:
            p = sph_params(**(sph if isinstance(sph, dict) else {}))
            self._ck(lib().gx_sph_enable(self._h, C.byref(p)))

    @classmethod
    def new_with_sph(cls, g, softening, theta, sph=None, **kw):
        """GpuResidentLeapfrog::new_with_sph (gpu_resident.rs:1393-1404): ``sph`` holds the
        :func:`sph_params` keywords (HydroParams + DensityConfig), ``kw`` the handle's."""
        return cls(g, softening, theta, sph=dict(sph or {}), **kw)

    def upload(self, state: State):
        self._mass = state.mass.copy()
        self._kind = state.kind.copy()
        self._u = state.u.copy()
        if self.gas_mode:
            self._ck(lib().gx_upload_species(self._h, len(state), _ptr(state.pos), _ptr(state.vel),
                                             _ptr(state.mass), _ptr(state.kind), _ptr(state.u)))
        else:
            self._ck(lib().gx_upload(self._h, len(state), _ptr(state.pos), _ptr(state.vel), _ptr(state.mass)))

    def gas_count(self) -> int:
        n = C.c_size_t()
        self._ck(lib().gx_gas_count(self._h, C.byref(n)))
        return n.value

    def snapshot_gas_density(self) -> GasDensity:
        """gpu_resident.rs:1566-1587."""
        ng = self.gas_count()
        idx, rho, h = np.zeros(ng, dtype=np.uint32), np.zeros(ng), np.zeros(ng)
        self._ck(lib().gx_snapshot_gas_density(self._h, _ptr(idx), _ptr(rho), _ptr(h)))
        return GasDensity(idx, rho, h)

    def snapshot_gas_accel(self, with_dudt: bool = False):
        """gpu_resident.rs:1593-1607: the hydro acceleration of the gas rows alone."""
        ng = self.gas_count()
        acc, dudt = np.zeros((ng, 3)), np.zeros(ng)
        self._ck(lib().gx_snapshot_gas_accel(self._h, _ptr(acc), _ptr(dudt)))
        return (acc, dudt) if with_dudt else acc

    def snapshot_accel(self) -> np.ndarray:
        """gpu_resident.rs:1655: the full acceleration of every particle."""
        out = np.empty((len(self), 3))
        self._ck(lib().gx_snapshot_accel(self._h, _ptr(out)))
        return out

    def min_stable_dt(self, c_cfl: float) -> float:
        """gpu_resident.rs:1614-1626: min_i c_cfl h_i / v_sig,i, reduced on the device."""
        out = C.c_double()
        self._ck(lib().gx_min_stable_dt(self._h, float(c_cfl), C.byref(out)))
        return out.value

    def snapshot_gas_dt(self, c_cfl: float) -> GasCfl:
        """gpu_resident.rs:1632-1650."""
        ng = self.gas_count()
        dt = np.zeros(ng)
        if ng:
            self._ck(lib().gx_snapshot_gas_dt(self._h, float(c_cfl), _ptr(dt)))
        return GasCfl(self.snapshot_gas_density().gas_idx, dt)

    def step(self, dt: float):
        self._ck(lib().gx_step(self._h, float(dt)))

    def step_many(self, dt: float, steps: int):
        self._ck(lib().gx_step_many(self._h, float(dt), int(steps)))

    def step_many_timed(self, dt: float, steps: int) -> float:
        """Run steps and return their device time in ms (CUDA events on the handle's stream)."""
        ms = C.c_float()
        self._ck(lib().gx_step_many_timed(self._h, float(dt), int(steps), C.byref(ms)))
        return ms.value

    def step_many_async(self, dt: float, steps: int):
        self._ck(lib().gx_step_many_async(self._h, float(dt), int(steps)))

    def autotune(self, repeats: int = 3) -> dict:
        """Pick the walk launch for this N bucket by timing force evaluations on the
        resident state (which stays bit-identical); see gx_autotune."""
        return _tune(lambda b, t, n: lib().gx_autotune(self._h, int(repeats), b, t, n), self._ck)

    def synchronize(self):
        self._ck(lib().gx_synchronize(self._h))

    def snapshot(self) -> State:
        n = len(self)
        pos, vel = np.empty((n, 3)), np.empty((n, 3))
        self._ck(lib().gx_snapshot(self._h, _ptr(pos), _ptr(vel)))
        return State(pos, vel, self._mass.copy(), self.time(), self._kind.copy(), self._u.copy())

    def accelerations(self) -> np.ndarray:
        out = np.empty((len(self), 3))
        self._ck(lib().gx_resident_accelerations(self._h, _ptr(out)))
        return out

    def diagnostics(self, with_potential: bool = True) -> dict:
        out = np.zeros(8)
        self._ck(lib().gx_diagnostics(self._h, int(with_potential), _ptr(out)))
        return {"kinetic": out[0], "potential": out[1], "total": out[0] + out[1], "momentum": out[2:5].copy(),
                "angular_momentum": out[5:8].copy()}

    def time(self) -> float:
        t = C.c_double()
        self._ck(lib().gx_time(self._h, C.byref(t)))
        return t.value

    def __len__(self):
        n = C.c_size_t()
        self._ck(lib().gx_len(self._h, C.byref(n)))
        return n.value

    def submits(self) -> int:
        v = C.c_uint64()
        self._ck(lib().gx_launches(self._h, C.byref(v)))
        return v.value


class PinnedState:
    """A State whose arrays live in page-locked host memory (gx_host_alloc), plus the
    integrator's cached acceleration."""

    def __init__(self, n: int):
        self.n = n
        self._bufs = []
        self.pos = self._alloc((n, 3))
        self.vel = self._alloc((n, 3))
        self.mass = self._alloc((n,))
        self.acc = self._alloc((n, 3))
        self.time = 0.0

    def _alloc(self, shape):
        nbytes = int(np.prod(shape)) * 8
        p = C.c_void_p()
        check(lib().gx_host_alloc(max(nbytes, 8), C.byref(p)))
        self._bufs.append(p)
        buf = (C.c_double * max(int(np.prod(shape)), 1)).from_address(p.value)
        return np.frombuffer(buf, dtype=np.float64, count=int(np.prod(shape))).reshape(shape)

    @classmethod
    def from_state(cls, st: State) -> "PinnedState":
        p = cls(len(st))
        p.pos[:] = st.pos
        p.vel[:] = st.vel
        p.mass[:] = st.mass
        p.acc[:] = 0.0
        p.time = st.time
        return p

    def __len__(self):
        return self.n

    def __del__(self):
        try:
            for b in self._bufs:
                lib().gx_host_free(b)
            self._bufs = []
        except Exception:
            pass


class Batch:
    """Many independent systems, one launch per stage (see include/galaxy_b200.h)."""

    def __init__(self, budget_bytes: int = 0, precision="f32", multipole="mono", kahan=True, stats=False, device=-1,
                 walk_block=0, walk_ctas_per_sm=0, morton63=False, walk_group=0, radix_bits=0):
        self._b = C.c_void_p()
        o = _options(precision, multipole, kahan, stats, device, walk_block, False, walk_ctas_per_sm, morton63,
                     walk_group, radix_bits)
        rc = lib().gx_batch_create(int(budget_bytes), C.byref(o), C.byref(self._b))
        if rc != 0:
            check(rc, None)
        self._mass = {}

    def _ck(self, rc):
        check(rc, self._b, "gx_batch_last_error")

    def close(self):
        if getattr(self, "_b", None) and self._b.value:
            lib().gx_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, state: State, g: float, softening: float, theta: float, dt: float) -> int:
        sid = C.c_uint64()
        self._ck(lib().gx_system_add(self._b, len(state), _ptr(state.pos), _ptr(state.vel), _ptr(state.mass), g,
                                     softening, theta, dt, C.byref(sid)))
        self._mass[sid.value] = state.mass.copy()
        return sid.value

    def remove(self, sid: int):
        self._ck(lib().gx_system_remove(self._b, sid))
        self._mass.pop(sid, None)

    def system_bytes(self, n: int) -> int:
        out = C.c_size_t()
        self._ck(lib().gx_system_bytes(self._b, n, C.byref(out)))
        return out.value

    def step(self, steps: int = 1):
        self._ck(lib().gx_batch_step(self._b, int(steps)))

    def set_graph(self, enable: bool):
        self._ck(lib().gx_batch_set_graph(self._b, int(enable)))

    def autotune(self, repeats: int = 3) -> dict:
        """gx_batch_autotune: the persistent walk launch for this batch's N bucket."""
        return _tune(lambda b, t, n: lib().gx_batch_autotune(self._b, int(repeats), b, t, n), self._ck)

    def snapshot(self, sid: int) -> State:
        n = C.c_size_t()
        self._ck(lib().gx_system_len(self._b, sid, C.byref(n)))
        pos, vel, t = np.empty((n.value, 3)), np.empty((n.value, 3)), C.c_double()
        self._ck(lib().gx_system_snapshot(self._b, sid, _ptr(pos), _ptr(vel), C.byref(t)))
        return State(pos, vel, self._mass[sid].copy(), t.value)

    def stats(self) -> dict:
        s = _lib.BatchStats()
        self._ck(lib().gx_batch_stats_get(self._b, C.byref(s)))
        return {f: getattr(s, f) for f, _ in s._fields_}


class Server:
    """Continuous-batching server (include/galaxy_b200.h, gx_server_*): submit systems
    from any thread; a native stepping thread admits them against the device budget,
    steps all live systems together and retires each after its steps."""

    QUEUED, RUNNING, DONE, REJECTED, CANCELLED = 0, 1, 2, 3, 4

    def __init__(self, budget_bytes: int = 0, precision="f32", multipole="mono", kahan=True, device=-1,
                 morton63=False):
        self._s = C.c_void_p()
        o = _options(precision, multipole, kahan, False, device, 0, morton63=morton63)
        rc = lib().gx_server_create(int(budget_bytes), C.byref(o), C.byref(self._s))
        if rc != 0:
            check(rc, None)
        self._n = {}

    def _ck(self, rc):
        check(rc, self._s, "gx_server_last_error")

    def close(self):
        if getattr(self, "_s", None) and self._s.value:
            lib().gx_server_destroy(self._s)
            self._s = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, state: State, g: float, softening: float, theta: float, dt: float, steps: int,
               snapshot_every: int = 0, snapshot_prefix: str | None = None, rng_seed: int = 0, config_hash: int = 0,
               units: str | None = None) -> int:
        """Queue a scenario. With snapshot_every > 0 a GLXYSNAP v4 file
        "<snapshot_prefix>.<step:08d>.glxysnap" is emitted every that many steps and
        after the last (see gx_server_submit_snapshots)."""
        rid = C.c_uint64()
        if snapshot_every:
            if not snapshot_prefix:
                raise ValueError("snapshot_prefix is required with snapshot_every")
            o = _lib.SnapOpts(C.sizeof(_lib.SnapOpts), int(snapshot_every), snapshot_prefix.encode(), int(rng_seed),
                              int(config_hash), units.encode() if units else None)
            self._ck(lib().gx_server_submit_snapshots(self._s, len(state), _ptr(state.pos), _ptr(state.vel),
                                                      _ptr(state.mass), g, softening, theta, dt, int(steps),
                                                      C.byref(o), C.byref(rid)))
        else:
            self._ck(lib().gx_server_submit(self._s, len(state), _ptr(state.pos), _ptr(state.vel),
                                            _ptr(state.mass), g, softening, theta, dt, int(steps), C.byref(rid)))
        self._n[rid.value] = (len(state), state.mass.copy())
        return rid.value

    def cancel(self, rid: int) -> None:
        """gx_server_cancel: a queued request leaves the queue, a running one the batch."""
        self._ck(lib().gx_server_cancel(self._s, rid))

    def set_metrics_log(self, path: str | None) -> None:
        """Append one JSON line per batched step to ``path`` (None stops)."""
        self._ck(lib().gx_server_set_metrics_log(self._s, path.encode() if path else None))

    def snapshots_written(self, rid: int) -> int:
        v = C.c_uint64()
        self._ck(lib().gx_server_snapshots_written(self._s, rid, C.byref(v)))
        return v.value

    def status(self, rid: int):
        st, done = C.c_int(), C.c_uint64()
        self._ck(lib().gx_server_status(self._s, rid, C.byref(st), C.byref(done)))
        return st.value, done.value

    def wait(self, rid: int, timeout: float = 600.0) -> None:
        self._ck(lib().gx_server_wait(self._s, rid, float(timeout)))

    def result(self, rid: int) -> State:
        n, mass = self._n[rid]
        pos, vel, t = np.empty((n, 3)), np.empty((n, 3)), C.c_double()
        self._ck(lib().gx_server_result(self._s, rid, _ptr(pos), _ptr(vel), C.byref(t)))
        return State(pos, vel, mass.copy(), t.value)

    def release(self, rid: int) -> None:
        self._ck(lib().gx_server_release(self._s, rid))
        self._n.pop(rid, None)

    def stats(self) -> dict:
        s = _lib.ServerStats()
        self._ck(lib().gx_server_stats_get(self._s, C.byref(s)))
        return {f: getattr(s, f) for f, _ in s._fields_}


# ---- stage entry points (parity tests) ------------------------------------------------
def _stage_handle(h=None, **kw):
    return h if h is not None else GpuLbvh(1.0, 0.0, 0.5, **kw)


def stage_morton(pos, handle=None):
    """reference_morton on the GPU: (lanes [n,3] u32, codes [n] u32, bounds dict)."""
    h = _stage_handle(handle)
    pos = _f64(pos).reshape(-1, 3)
    n = pos.shape[0]
    lanes = np.empty((n, 3), np.uint32)
    codes = np.empty(n, np.uint32)
    b = np.empty(5)
    h._ck(lib().gx_stage_morton(h._h, n, _ptr(pos), _ptr(lanes), _ptr(codes), _ptr(b)))
    return lanes, codes, {"bmin": b[:3].copy(), "size": float(b[3]), "scale": float(b[4])}


def stage_sort(codes, handle=None):
    """reference_sort on the GPU: (order [n] u32, sorted_codes [n] u32)."""
    h = _stage_handle(handle)
    codes = np.ascontiguousarray(codes, dtype=np.uint32)
    n = codes.shape[0]
    order = np.empty(n, np.uint32)
    sc = np.empty(n, np.uint32)
    h._ck(lib().gx_stage_sort(h._h, n, _ptr(codes), _ptr(order), _ptr(sc)))
    return order, sc


def stage_build(sorted_codes, sorted_pos, sorted_mass, handle=None, quad=False):
    """reference_karras + reference_aggregate on the GPU."""
    h = _stage_handle(handle, multipole="quad" if quad else "mono")
    sc = np.ascontiguousarray(sorted_codes, dtype=np.uint32)
    sp = _f64(sorted_pos).reshape(-1, 3)
    sm = _f64(sorted_mass)
    n = sc.shape[0]
    t = 2 * n - 1
    left = np.empty(max(n - 1, 1), np.uint32)
    right = np.empty(max(n - 1, 1), np.uint32)
    parent = np.empty(t, np.uint32)
    mn, mx, com = np.empty((t, 3)), np.empty((t, 3)), np.empty((t, 3))
    mass = np.empty(t)
    q = np.empty((t, 6)) if quad else None
    h._ck(lib().gx_stage_build(h._h, n, _ptr(sc), _ptr(sp), _ptr(sm), _ptr(left), _ptr(right), _ptr(parent), _ptr(mn),
                               _ptr(mx), _ptr(com), _ptr(mass), _ptr(q)))
    out = {"left": left[: n - 1], "right": right[: n - 1], "parent": parent, "aabb_min": mn, "aabb_max": mx,
           "com": com, "mass": mass}
    if quad:
        out["quad"] = q
    return out


def _tune(call, ck) -> dict:
    best = _lib.Tuning()
    tried = (_lib.Tuning * _lib.GX_TUNE_MAX_CANDIDATES)()
    n = C.c_uint32()
    ck(call(C.byref(best), tried, C.byref(n)))
    row = lambda t: {"walk_block": t.walk_block, "walk_ctas_per_sm": t.walk_ctas_per_sm,  # noqa: E731
                     "walk_group": t.walk_group, "radix_bits": t.radix_bits, "ms": t.ms, "sort_ms": t.sort_ms}
    return {**row(best), "tried": [row(tried[i]) for i in range(n.value)]}


def tuning_lookup(n: int, batched: bool = False, precision: str = "f32", multipole: str = "mono",
                  morton63: bool = False, device: int = -1):
    """The tuned walk launch recorded for n particles under these options, or None."""
    o = _options(precision, multipole, True, False, device, 0, False, 0, morton63)
    t = _lib.Tuning()
    rc = lib().gx_tuning_lookup(int(device), int(n), C.byref(o), int(batched), C.byref(t))
    if rc == _lib.ERRORS_BY_NAME["GX_ERR_STATE"]:
        return None
    check(rc, None)
    return {"walk_block": t.walk_block, "walk_ctas_per_sm": t.walk_ctas_per_sm, "walk_group": t.walk_group,
            "radix_bits": t.radix_bits, "ms": t.ms, "sort_ms": t.sort_ms}


def device_synchronize(device: int = -1) -> None:
    """Wait for all device work (cudaDeviceSynchronize), e.g. around a timed region."""
    check(lib().gx_device_synchronize(int(device)), None)


def device_info(device: int = 0) -> dict:
    name = C.create_string_buffer(256)
    sm, ma, mi, mem = C.c_int(), C.c_int(), C.c_int(), C.c_size_t()
    rc = lib().gx_device_info(device, name, 256, C.byref(sm), C.byref(ma), C.byref(mi), C.byref(mem))
    check(rc, None)
    return {"name": name.value.decode(), "sm_count": sm.value, "cc": (ma.value, mi.value), "total_mem": mem.value}


from . import ic  # noqa: E402  (uses the helpers above)
