"""Seeded synthetic workloads of the benchmarks (shapes and distributions of the
named configurations; no dataset is involved).

* ``collision``  -- two composite disk galaxies, 2 x 524,288 particles, 1:1, parabolic,
  pericentre 4 Rd, disks inclined 30 and 60 degrees; eps 0.02, theta 0.5, dt 5e-4.
* ``plummer``    -- the N=16,384 Plummer sphere of seed 0 (G = M = a = 1); eps 0.01,
  theta 0.5, dt 1e-3.
* ``batched_mix`` -- independent systems with N log-uniform in [4,096, 262,144], half
  Plummer spheres and half disk + halo galaxies, eps 0.01, theta 0.5, dt 1e-3 or 5e-4.
* ``request_stream`` -- a Poisson stream of collision scenarios (rate, N log-uniform,
  mass ratio uniform in [1, 10], pericentre uniform in [2, 8] Rd, 100-1,000 steps).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import State, ic


@dataclass
class SystemSpec:
    state: State
    g: float
    eps: float
    theta: float
    dt: float
    name: str = ""


def collision(seed: int = 0, n_per_galaxy: int = 524_288) -> SystemSpec:
    st = ic.collision(2 * n_per_galaxy, seed, mass_ratio=1.0, pericentre=4.0, incl1_deg=30.0, incl2_deg=60.0)
    return SystemSpec(st, 1.0, 0.02, 0.5, 5e-4, f"collision-2x{n_per_galaxy}")


def plummer(seed: int = 0, n: int = 16_384) -> SystemSpec:
    return SystemSpec(ic.plummer(n, seed), 1.0, 0.01, 0.5, 1e-3, f"plummer-{n}")


def batched_sizes(count: int, seed: int, n_min: int = 4096, n_max: int = 262_144) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(n_min), np.log(n_max), count)).astype(np.int64)


def batched_mix(count: int = 256, seed: int = 0, n_min: int = 4096, n_max: int = 262_144,
                indices=None) -> list[SystemSpec]:
    """The mix's systems (all of them, or those listed in `indices`)."""
    sizes = batched_sizes(count, seed, n_min, n_max)
    out = []
    for i in (range(count) if indices is None else indices):
        n = int(sizes[i])
        if i % 2 == 0:
            st = ic.plummer(n, seed * 100_003 + i)
            kind = "plummer"
        else:
            st = ic.disk_galaxy(n, seed * 100_003 + i)
            kind = "disk"
        dt = 1e-3 if (i // 2) % 2 == 0 else 5e-4
        out.append(SystemSpec(st, 1.0, 0.01, 0.5, dt, f"{kind}-{n}"))
    return out


@dataclass
class Request:
    rid: int
    arrival: float  # seconds after the stream starts
    n: int
    mass_ratio: float
    pericentre: float
    steps: int
    seed: int

    def spec(self) -> SystemSpec:
        st = ic.collision(self.n, self.seed, mass_ratio=self.mass_ratio, pericentre=self.pericentre,
                          incl1_deg=30.0, incl2_deg=60.0)
        return SystemSpec(st, 1.0, 0.02, 0.5, 5e-4, f"request-{self.rid}")


def request_stream(count: int, rate: float = 50.0, seed: int = 0, n_min: int = 16_384, n_max: int = 2_097_152,
                   steps_min: int = 100, steps_max: int = 1000) -> list[Request]:
    """Poisson arrivals (exponential gaps of mean 1/rate) of collision scenarios."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, count))
    n = np.exp(rng.uniform(np.log(n_min), np.log(n_max), count)).astype(np.int64)
    q = rng.uniform(1.0, 10.0, count)
    rp = rng.uniform(2.0, 8.0, count)
    steps = rng.integers(steps_min, steps_max + 1, count)
    return [Request(i, float(t[i]), int(n[i]), float(q[i]), float(rp[i]), int(steps[i]), seed * 1_000_003 + i)
            for i in range(count)]


def gas_star_mix(n_gas: int, n_star: int, seed: int = 0) -> State:
    """A gas blob inside a wider star field, the resident SPH gates' setup scaled up
    (gpu/tests/gpu_resident_sph.rs:38-96: gas in a cube of side 2 at every
    (1 + n_star/n_gas)-th index, stars in a cube of side 6, velocities of 0.1 scale).
    Seeded numpy draws; total mass 1 (gas masses U[0.5, 1), star masses U[0.1, 1), scaled)."""
    rng = np.random.default_rng(seed)
    n = n_gas + n_star
    gpos = (rng.random((n_gas, 3)) - 0.5) * 2.0
    gvel = (rng.random((n_gas, 3)) - 0.5) * 0.1
    gm = 0.5 + 0.5 * rng.random(n_gas)
    spos = (rng.random((n_star, 3)) - 0.5) * 6.0
    svel = (rng.random((n_star, 3)) - 0.5) * 0.1
    sm = 0.1 + 0.9 * rng.random(n_star)
    take = max(n_star // max(n_gas, 1), 1)
    gas_rows = np.arange(n_gas) * (1 + take)
    gas_rows = gas_rows[gas_rows < n]
    kind = np.zeros(n, np.uint8)
    kind[gas_rows[:n_gas]] = 1
    gi = np.flatnonzero(kind == 1)
    si = np.flatnonzero(kind == 0)
    pos, vel, mass = np.empty((n, 3)), np.empty((n, 3)), np.empty(n)
    pos[gi], vel[gi], mass[gi] = gpos[:gi.size], gvel[:gi.size], gm[:gi.size]
    pos[si], vel[si], mass[si] = spos[:si.size], svel[:si.size], sm[:si.size]
    mass /= mass.sum()
    return State(pos, vel, mass, kind=kind)
