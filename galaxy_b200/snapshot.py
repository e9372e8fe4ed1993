"""GLXYSNAP v4 snapshot files (io/src/snapshot.rs): ``write`` through the library's C
writer, ``read`` restating the reference's reader (``from_reader``, :200-305, including
its defaults for the v1-v3 streams)."""

from __future__ import annotations

import struct

import numpy as np

from . import State, _lib, check, lib

MAGIC = b"GLXYSNAP"
FORMAT_VERSION = 4
MIN_READ_VERSION = 1
MAX_STR_LEN = 1 << 16


class SnapshotError(ValueError):
    pass


def write(path: str, state: State, step: int = 0, softening: float = 0.0, rng_seed: int = 0, config_hash: int = 0,
          units: str = "nbody-G1") -> None:
    n = len(state)
    pos = np.ascontiguousarray(state.pos, np.float64)
    vel = np.ascontiguousarray(state.vel, np.float64)
    mass = np.ascontiguousarray(state.mass, np.float64)
    check(lib().gx_glxysnap_write(str(path).encode(), float(state.time), int(step), float(softening), int(rng_seed),
                                  int(config_hash), units.encode(), n, pos.ctypes.data, vel.ctypes.data,
                                  mass.ctypes.data), None)


def read(path: str) -> tuple[dict, dict]:
    """(header, columns) of a snapshot; columns: pos, vel [n,3] f64, mass [n] (the
    f32-rounded values as f64), id u64, progenitor u16, kind u8, u f64, formation_time f64."""
    with open(path, "rb") as f:
        data = f.read()
    off = 0

    def take(k: int) -> bytes:
        nonlocal off
        if off + k > len(data):
            raise SnapshotError("truncated snapshot")
        b = data[off:off + k]
        off += k
        return b

    if take(8) != MAGIC:
        raise SnapshotError("not a galaxy snapshot (bad magic)")
    (version,) = struct.unpack("<I", take(4))
    if not MIN_READ_VERSION <= version <= FORMAT_VERSION:
        raise SnapshotError(f"unsupported snapshot format version {version}")
    time, step, scale, soft, n, seed, chash = struct.unpack("<dQddQQQ", take(56))

    def string() -> str:
        (k,) = struct.unpack("<I", take(4))
        if k > MAX_STR_LEN:
            raise SnapshotError("header string too long")
        return take(k).decode("utf-8")

    units, code_version = string(), string()

    def column(dtype, count):
        a = np.frombuffer(take(np.dtype(dtype).itemsize * count), dtype=dtype)
        return a.copy()

    cols = {"pos": column("<f8", 3 * n).reshape(n, 3), "vel": column("<f8", 3 * n).reshape(n, 3),
            "mass": column("<f4", n).astype(np.float64), "id": column("<u8", n), "progenitor": column("<u2", n)}
    cols["kind"] = column("u1", n) if version >= 2 else np.zeros(n, np.uint8)
    if version >= 2 and np.any(cols["kind"] > 1):
        raise SnapshotError("unknown species byte")
    cols["u"] = column("<f8", n) if version >= 3 else np.zeros(n)
    cols["formation_time"] = column("<f8", n) if version >= 4 else np.full(n, -np.inf)
    header = {"version": version, "time": time, "step": step, "scale_factor": scale, "softening": soft,
              "n_particles": n, "rng_seed": seed, "config_hash": chash, "units": units,
              "code_version": code_version}
    return header, cols


__all__ = ["write", "read", "SnapshotError", "MAGIC", "FORMAT_VERSION", "_lib"]
