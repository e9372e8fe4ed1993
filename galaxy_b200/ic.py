"""Seeded initial conditions (host code in libgalaxy_b200: see csrc/gx_ic.cpp).

plummer: Plummer::sample of the reference (ic/src/plummer.rs:94-140), same realisation.
collision / disk_galaxy: synthetic halo + exponential disk + Hernquist bulge galaxies
standing in for the reference's collision scenarios (ic/src/disk_collision.rs).
"""

from __future__ import annotations

import numpy as np

from . import State
from ._lib import check, lib


def _arrays(n):
    return np.empty((n, 3)), np.empty((n, 3)), np.empty(n)


def plummer(n: int, seed: int = 0, g: float = 1.0, total_mass: float = 1.0, scale_radius: float = 1.0) -> State:
    pos, vel, mass = _arrays(n)
    check(lib().gx_ic_plummer(n, seed, g, total_mass, scale_radius, pos.ctypes.data, vel.ctypes.data,
                              mass.ctypes.data))
    return State(pos, vel, mass)


def collision(n_total: int, seed: int = 0, mass_ratio: float = 1.0, pericentre: float = 4.0, incl1_deg: float = 30.0,
              incl2_deg: float = 60.0) -> State:
    pos, vel, mass = _arrays(n_total)
    check(lib().gx_ic_collision(n_total, seed, mass_ratio, pericentre, incl1_deg, incl2_deg, pos.ctypes.data,
                                vel.ctypes.data, mass.ctypes.data))
    return State(pos, vel, mass)


def disk_galaxy(n: int, seed: int = 0) -> State:
    pos, vel, mass = _arrays(n)
    check(lib().gx_ic_disk_galaxy(n, seed, pos.ctypes.data, vel.ctypes.data, mass.ctypes.data))
    return State(pos, vel, mass)
