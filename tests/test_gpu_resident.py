"""Resident KDK stepping (gpu/tests/gpu_resident.rs gates, restated): the FP64 mode's
trajectory is bit-identical to the reference integrator (core/src/integrator.rs)
driving the reference solver; batching steps does not change the arithmetic;
snapshot/upload round trips; conservation over the Plummer workload."""

import numpy as np
import pytest

import galaxy_b200 as gb

pytestmark = pytest.mark.gpu


def test_f64_trajectory_bit_exact_vs_oracle(oracle):
    st = gb.ic.plummer(4096, 0)
    r = gb.GpuResidentLeapfrog(1.0, 0.01, 0.5, precision="f64")
    r.upload(st)
    r.step_many(1e-3, 10)
    snap = r.snapshot()
    pos, vel = st.pos.copy(), st.vel.copy()
    kdk = oracle.LeapfrogKdkLbvh(1.0, 0.01, 0.5, threads=8)
    kdk.step_many(pos, vel, st.mass, 1e-3, 10)
    assert np.array_equal(snap.pos, pos) and np.array_equal(snap.vel, vel)
    assert abs(snap.time - 10e-3) < 1e-15


def test_step_many_equals_repeated_step():
    st = gb.ic.plummer(5000, 2)
    a = gb.GpuResidentLeapfrog(1.0, 0.01, 0.5)
    b = gb.GpuResidentLeapfrog(1.0, 0.01, 0.5)
    a.upload(st)
    b.upload(st)
    a.step_many(1e-3, 12)
    for _ in range(12):
        b.step(1e-3)
    sa, sb = a.snapshot(), b.snapshot()
    assert np.array_equal(sa.pos, sb.pos) and np.array_equal(sa.vel, sb.vel)


def test_resident_matches_host_driven_solver():
    # gpu/tests/gpu_resident.rs:113-152: resident == host round trip (here bit-exact).
    st = gb.ic.plummer(3000, 5)
    r = gb.GpuResidentLeapfrog(1.0, 0.01, 0.5)
    r.upload(st)
    r.step_many(5e-4, 7)
    host = st.copy()
    kdk = gb.LeapfrogKdk()
    solver = gb.GpuLbvh(1.0, 0.01, 0.5)
    for _ in range(7):
        kdk.step(host, solver, 5e-4)
    snap = r.snapshot()
    assert np.array_equal(snap.pos, host.pos) and np.array_equal(snap.vel, host.vel)


def test_snapshot_upload_round_trip_continues_identically():
    st = gb.ic.plummer(2000, 9)
    a = gb.GpuResidentLeapfrog(1.0, 0.01, 0.5)
    a.upload(st)
    a.step_many(1e-3, 5)
    mid = a.snapshot()
    a.step_many(1e-3, 5)
    b = gb.GpuResidentLeapfrog(1.0, 0.01, 0.5)
    b.upload(mid)
    b.step_many(1e-3, 5)
    sa, sb = a.snapshot(), b.snapshot()
    assert np.array_equal(sa.pos, sb.pos) and np.array_equal(sa.vel, sb.vel)


def test_resident_accelerations_are_current():
    st = gb.ic.plummer(3000, 1)
    r = gb.GpuResidentLeapfrog(1.0, 0.01, 0.5)
    r.upload(st)
    r.step_many(1e-3, 3)
    snap = r.snapshot()
    acc = gb.GpuLbvh(1.0, 0.01, 0.5).accelerations(snap)
    assert np.array_equal(r.accelerations(), acc)


def test_diagnostics_match_oracle(oracle):
    st = gb.ic.plummer(8192, 4)
    r = gb.GpuResidentLeapfrog(1.0, 0.01, 0.5)
    r.upload(st)
    r.step_many(1e-3, 4)
    d = r.diagnostics(True)
    snap = r.snapshot()
    ref = oracle.diagnostics(snap.pos, snap.vel, snap.mass)
    assert abs(d["kinetic"] - ref["kinetic"]) <= 1e-12 * ref["kinetic"]
    assert np.allclose(d["angular_momentum"], ref["angular_momentum"], rtol=0, atol=1e-15)
    u = oracle.potential_serial(snap.pos, snap.mass, 1.0, 0.01)
    assert abs(d["potential"] - u) <= 1e-9 * abs(u)


def test_energy_conservation_plummer_config():
    # The N=16,384 Plummer workload: theta=0.5, eps=0.01, dt=1e-3, 100 KDK steps.
    st = gb.ic.plummer(16384, 0)
    r = gb.GpuResidentLeapfrog(1.0, 0.01, 0.5)
    r.upload(st)
    e0 = r.diagnostics(True)
    r.step_many(1e-3, 100)
    e1 = r.diagnostics(True)
    assert abs(e1["total"] - e0["total"]) < 1e-3 * abs(e0["total"])
    # Barnes-Hut forces are not pairwise antisymmetric: momentum drifts at the force-error level.
    snap = r.snapshot()
    scale = float((np.linalg.norm(snap.vel, axis=1) * snap.mass).sum())
    assert np.linalg.norm(e1["momentum"]) < 1e-4 * scale
    assert abs(r.time() - 0.1) < 1e-12


def test_empty_and_lone_particle():
    r = gb.GpuResidentLeapfrog(1.0, 0.01, 0.5)
    r.upload(gb.State(np.zeros((0, 3)), np.zeros((0, 3)), np.zeros(0)))
    r.step_many(0.5, 4)
    assert r.time() == 2.0 and len(r) == 0
    r.upload(gb.State([[1.0, 2.0, 3.0]], [[0.5, 0.0, -1.0]], [1.0]))
    r.step_many(0.25, 4)
    s = r.snapshot()
    assert np.allclose(s.pos, [[1.5, 2.0, 2.0]]) and np.array_equal(s.vel, [[0.5, 0.0, -1.0]])


def test_step_before_upload_is_an_error():
    r = gb.GpuResidentLeapfrog(1.0, 0.01, 0.5)
    with pytest.raises(gb.GxError):
        r.step(1e-3)


def test_stage_times_follow_each_step():
    """With GX_FLAG_STAGE_TIMES the stage times are those of the latest step, not of
    the priming force evaluation at upload."""
    st = gb.ic.collision(65_536, 2)
    r = gb.GpuResidentLeapfrog(1.0, 0.02, 0.5, stage_times=True)
    r.upload(st)
    seen = {r.stats()["ms_total"]}
    for _ in range(3):
        r.step(5e-4)
        s = r.stats()
        assert s["ms_walk"] > 0 and s["ms_build"] > 0 and s["ms_sort"] > 0
        parts = s["ms_bbox_morton"] + s["ms_sort"] + s["ms_build"] + s["ms_walk"]
        assert abs(parts - s["ms_total"]) <= 1e-3 * s["ms_total"] + 1e-3
        seen.add(s["ms_total"])
    # event times have a resolution of about half a microsecond: two steps may coincide
    assert len(seen) >= 3
