"""CPU-side checks of the C-ABI library: it loads, exports every symbol the public
header declares, fails loudly without a device, and its host-only input generators
(seeded initial conditions) behave."""

import ctypes

import numpy as np
import pytest


@pytest.fixture(scope="module")
def gb():
    import galaxy_b200

    galaxy_b200._lib.lib()
    return galaxy_b200


def test_exports_every_header_symbol(gb):
    L = gb._lib.lib()
    syms = gb._lib.header_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(L, s)]
    assert missing == []


def test_create_reports_missing_device_or_succeeds(gb):
    L = gb._lib.lib()
    h = ctypes.c_void_p()
    rc = L.gx_create(1.0, 0.01, 0.5, None, ctypes.byref(h))
    if rc == 0:
        L.gx_destroy(h)
    else:
        assert rc == -3  # GX_ERR_NO_DEVICE: no CPU fallback
        assert L.gx_last_error(None)


def test_invalid_options_rejected(gb):
    o = gb._lib.Options()
    o.struct_size = ctypes.sizeof(o)
    o.precision = 7
    h = ctypes.c_void_p()
    assert gb._lib.lib().gx_create(1.0, 0.01, 0.5, ctypes.byref(o), ctypes.byref(h)) in (-1, -3)


def test_plummer_sample_properties(gb):
    # ic/src/plummer.rs:94-140: equal masses summing to M, zero COM and momentum.
    s = gb.ic.plummer(16384, seed=0)
    assert s.pos.shape == (16384, 3)
    assert np.all(s.mass == 1.0 / 16384)
    assert np.abs(s.pos.mean(0)).max() < 1e-12 and np.abs(s.vel.mean(0)).max() < 1e-12
    r = np.linalg.norm(s.pos, axis=1)
    # half-mass radius of a Plummer sphere: 1.30477 a
    assert abs(np.median(r) - 1.30477) < 0.05
    again = gb.ic.plummer(16384, seed=0)
    assert np.array_equal(s.pos, again.pos) and np.array_equal(s.vel, again.vel)
    assert not np.array_equal(s.pos, gb.ic.plummer(16384, seed=1).pos)


def test_collision_ic_properties(gb):
    s = gb.ic.collision(20000, seed=3, mass_ratio=3.0, pericentre=4.0)
    m = s.mass
    assert abs(m.sum() - 4.0) < 1e-9
    com = (s.pos * m[:, None]).sum(0) / m.sum()
    mom = (s.vel * m[:, None]).sum(0)
    assert np.abs(com).max() < 1e-9 and np.abs(mom).max() < 1e-9
    n1 = 5000
    c1 = (s.pos[:n1] * m[:n1, None]).sum(0) / m[:n1].sum()
    c2 = (s.pos[n1:] * m[n1:, None]).sum(0) / m[n1:].sum()
    assert np.linalg.norm(c2 - c1) > 15.0  # the two galaxies start well separated


def test_disk_galaxy_properties(gb):
    s = gb.ic.disk_galaxy(10000, seed=2)
    assert abs(s.mass.sum() - 1.0) < 1e-12
    # disk particles (the 35% after the halo) are thin
    disk = s.pos[6000:9500]
    assert np.abs(disk[:, 2]).mean() < 0.2


def test_stage_inputs_validated_without_device(gb):
    with pytest.raises(gb.GxError):
        gb.GpuLbvh(1.0, 0.01, 0.5) if not _has_gpu() else (_ for _ in ()).throw(gb.GxError(-1, "skip"))


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
