"""Batched systems: one launch per stage over many systems, persistent work-stealing
walk, CUDA-graph replay. Every system's trajectory must be bit-identical to stepping
it alone, whatever else is in the batch and whenever it joined."""

import numpy as np
import pytest

import galaxy_b200 as gb

pytestmark = pytest.mark.gpu


def _alone(st, theta, eps, dt, steps, precision="f32"):
    r = gb.GpuResidentLeapfrog(1.0, eps, theta, precision=precision)
    r.upload(st)
    r.step_many(dt, steps)
    return r.snapshot()


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_batch_equals_alone(precision):
    systems = [(gb.ic.plummer(5000, 1), 0.5, 0.01, 1e-3), (gb.ic.disk_galaxy(9000, 2), 0.5, 0.02, 5e-4),
               (gb.ic.plummer(37, 3), 0.7, 0.01, 1e-3), (gb.ic.plummer(1, 4), 0.5, 0.01, 1e-3),
               (gb.ic.plummer(2, 5), 0.3, 0.01, 1e-3), (gb.ic.plummer(4097, 6), 0.5, 0.01, 5e-4)]
    b = gb.Batch(precision=precision)
    ids = [b.add(st, 1.0, eps, th, dt) for st, th, eps, dt in systems]
    b.step(6)
    for sid, (st, th, eps, dt) in zip(ids, systems):
        got = b.snapshot(sid)
        ref = _alone(st, th, eps, dt, 6, precision)
        assert np.array_equal(got.pos, ref.pos) and np.array_equal(got.vel, ref.vel)
        assert abs(got.time - 6 * dt) < 1e-15


def test_join_and_leave_mid_run():
    a, c = gb.ic.plummer(3000, 11), gb.ic.plummer(6000, 12)
    b = gb.Batch()
    ia = b.add(a, 1.0, 0.01, 0.5, 1e-3)
    b.step(3)
    ic_ = b.add(c, 1.0, 0.01, 0.5, 1e-3)
    b.step(4)
    b.remove(ia)
    b.step(2)
    ref_c = _alone(c, 0.5, 0.01, 1e-3, 6)
    got = b.snapshot(ic_)
    assert np.array_equal(got.pos, ref_c.pos) and np.array_equal(got.vel, ref_c.vel)
    with pytest.raises(gb.GxError):
        b.snapshot(ia)


def test_graph_and_eager_identical():
    sts = [gb.ic.plummer(4000 + 100 * i, 20 + i) for i in range(5)]
    outs = []
    for graph in (True, False):
        b = gb.Batch()
        b.set_graph(graph)
        ids = [b.add(s, 1.0, 0.01, 0.5, 1e-3) for s in sts]
        b.step(5)
        outs.append([b.snapshot(i) for i in ids])
    for x, y in zip(*outs):
        assert np.array_equal(x.pos, y.pos) and np.array_equal(x.vel, y.vel)


def test_budget_rejects():
    b = gb.Batch(budget_bytes=50 << 20)
    b.add(gb.ic.plummer(10000, 1), 1.0, 0.01, 0.5, 1e-3)
    with pytest.raises(gb.GxError) as e:
        b.add(gb.ic.plummer(400_000, 2), 1.0, 0.01, 0.5, 1e-3)
    assert e.value.code == -4
    assert b.stats()["systems"] == 1


def test_many_systems_memory_stays_linear():
    b = gb.Batch()
    sts = [gb.ic.plummer(500 + (i % 7) * 50, 300 + i) for i in range(150)]
    for st in sts:
        b.add(st, 1.0, 0.01, 0.5, 1e-3)
    s = b.stats()
    assert s["systems"] == 150
    per_particle = s["bytes_in_use"] / s["particles"]
    assert per_particle < 3000, per_particle  # ~400 B/particle plus headroom and per-system tables
    b.step(2)
    ref = gb.GpuResidentLeapfrog(1.0, 0.01, 0.5)
    ref.upload(sts[77])
    ref.step_many(1e-3, 2)
    got = b.snapshot(78)  # ids start at 1
    assert np.array_equal(got.pos, ref.snapshot().pos)
