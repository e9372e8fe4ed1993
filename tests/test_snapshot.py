"""GLXYSNAP v4 files (io/src/snapshot.rs): the library's writer against an independent
restatement of the reference's ``to_writer`` (:130-199) byte for byte, and the reader
(``from_reader``, :200-305) on round trips, older versions and corrupt streams
(io/tests/roundtrip.rs)."""

import struct

import numpy as np
import pytest

import galaxy_b200 as gb
from galaxy_b200 import snapshot as snap


def _reference_bytes(state, step, softening, seed, chash, units, code_version):
    """to_writer's byte sequence, field by field."""
    n = len(state)
    out = bytearray(b"GLXYSNAP")
    out += struct.pack("<I", 4)
    out += struct.pack("<dQddQQQ", state.time, step, 1.0, softening, n, seed, chash)
    for s in (units, code_version):
        b = s.encode()
        out += struct.pack("<I", len(b)) + b
    for p in state.pos:
        out += struct.pack("<ddd", *p)
    for v in state.vel:
        out += struct.pack("<ddd", *v)
    for m in state.mass:
        out += struct.pack("<f", m)  # `m as f32`: round to nearest
    for i in range(n):
        out += struct.pack("<Q", i)
    out += b"\x00\x00" * n  # progenitor
    out += b"\x00" * n  # kind: collisionless
    out += struct.pack("<d", 0.0) * n  # u
    out += struct.pack("<d", float("-inf")) * n  # formation time: primordial
    return bytes(out)


@pytest.mark.parametrize("n", [0, 1, 5, 33])
def test_writer_matches_reference_layout(tmp_path, n):
    st = gb.ic.plummer(max(n, 1), 3)
    st = gb.State(st.pos[:n].copy(), st.vel[:n].copy(), st.mass[:n].copy() * 1.37, 0.625)
    path = tmp_path / "s.glxysnap"
    snap.write(path, st, step=12, softening=0.02, rng_seed=99, config_hash=0xABCDEF, units="nbody-G1")
    assert path.read_bytes() == _reference_bytes(st, 12, 0.02, 99, 0xABCDEF, "nbody-G1", "galaxy_b200 0.1")


def test_round_trip(tmp_path):
    st = gb.ic.plummer(1000, 4)
    st.time = 1.5
    path = tmp_path / "r.glxysnap"
    snap.write(path, st, step=3, softening=0.01, rng_seed=7, config_hash=11, units="kpc")
    h, c = snap.read(path)
    assert (h["version"], h["time"], h["step"], h["scale_factor"], h["softening"]) == (4, 1.5, 3, 1.0, 0.01)
    assert (h["n_particles"], h["rng_seed"], h["config_hash"], h["units"]) == (1000, 7, 11, "kpc")
    assert np.array_equal(c["pos"], st.pos) and np.array_equal(c["vel"], st.vel)
    assert np.array_equal(c["mass"], st.mass.astype(np.float32).astype(np.float64))
    assert np.array_equal(c["id"], np.arange(1000)) and not c["progenitor"].any() and not c["kind"].any()
    assert not c["u"].any() and np.all(c["formation_time"] == -np.inf)


def test_reader_rejects_corrupt_streams(tmp_path):
    st = gb.ic.plummer(10, 5)
    good = tmp_path / "g.glxysnap"
    snap.write(good, st)
    data = good.read_bytes()
    for name, blob in (("magic", b"NOTASNAP" + data[8:]), ("version", data[:8] + struct.pack("<I", 5) + data[12:]),
                       ("short", data[:-3]), ("empty", b"")):
        p = tmp_path / name
        p.write_bytes(blob)
        with pytest.raises(snap.SnapshotError):
            snap.read(p)


def test_v1_stream_reads_with_defaults(tmp_path):
    """A v1 stream (no kind, u, formation-time columns) reads as collisionless, u = 0 and
    primordial, as the reference reader defaults them."""
    st = gb.ic.plummer(4, 6)
    full = _reference_bytes(st, 1, 0.0, 0, 0, "x", "y")
    head = 8 + 4 + 56 + (4 + 1) * 2
    cols = full[head:head + 4 * (24 + 24 + 4 + 8 + 2)]
    v1 = full[:8] + struct.pack("<I", 1) + full[12:head] + cols
    p = tmp_path / "v1.glxysnap"
    p.write_bytes(v1)
    h, c = snap.read(p)
    assert h["version"] == 1 and np.array_equal(c["pos"], st.pos)
    assert not c["kind"].any() and not c["u"].any() and np.all(c["formation_time"] == -np.inf)
