"""Autotuning of the walk launch (gx_autotune / gx_batch_autotune): the sweep leaves
the state bit-identical, records its winner for the N bucket, and the launch
configuration never changes a result."""

import numpy as np
import pytest

import galaxy_b200 as gb

pytestmark = pytest.mark.gpu


def test_launch_configuration_never_changes_results():
    st = gb.ic.collision(65_536, 11)
    ref = gb.GpuLbvh(1.0, 0.02, 0.5, walk_block=128).accelerations(st)
    for block, ctas in ((64, 0), (128, 7), (64, 3), (96, 1)):
        got = gb.GpuLbvh(1.0, 0.02, 0.5, walk_block=block, walk_ctas_per_sm=ctas).accelerations(st)
        assert np.array_equal(got, ref), (block, ctas)


def test_autotune_keeps_state_and_records_bucket():
    st = gb.ic.collision(98_304, 12)  # bucket floor(log2 98304) = 16
    r = gb.GpuResidentLeapfrog(1.0, 0.02, 0.5)
    r.upload(st)
    r.step_many(5e-4, 3)
    before = r.snapshot()
    acc_before = r.accelerations()
    best = r.autotune(repeats=2)
    assert best["tried"] and best["ms"] == min(t["ms"] for t in best["tried"])
    assert best["walk_block"] in (64, 128)
    after = r.snapshot()
    assert np.array_equal(before.pos, after.pos) and np.array_equal(before.vel, after.vel)
    assert np.array_equal(acc_before, r.accelerations())
    for n in (65_536, 100_000, 131_071):
        rec = gb.tuning_lookup(n)
        assert rec is not None and (rec["walk_block"], rec["walk_ctas_per_sm"]) == (best["walk_block"],
                                                                                 best["walk_ctas_per_sm"])
    assert gb.tuning_lookup(98_304, precision="f64") is None
    # the trajectory continues exactly as an untuned twin's
    twin = gb.GpuResidentLeapfrog(1.0, 0.02, 0.5, walk_block=128)
    twin.upload(st)
    twin.step_many(5e-4, 3)
    r.step_many(5e-4, 4)
    twin.step_many(5e-4, 4)
    assert np.array_equal(r.snapshot().pos, twin.snapshot().pos)


def test_batch_autotune_keeps_state():
    sts = [gb.ic.plummer(20_000 + 5_000 * i, 90 + i) for i in range(3)]
    b = gb.Batch()
    ids = [b.add(s, 1.0, 0.01, 0.5, 1e-3) for s in sts]
    b.step(2)
    before = [b.snapshot(i) for i in ids]
    best = b.autotune(repeats=2)
    assert all(t["walk_ctas_per_sm"] > 0 for t in best["tried"])  # the batch walk is persistent
    for i, s0 in zip(ids, before):
        s1 = b.snapshot(i)
        assert np.array_equal(s0.pos, s1.pos) and np.array_equal(s0.vel, s1.vel)
    n_total = sum(len(s) for s in sts)
    rec = gb.tuning_lookup(n_total, batched=True)
    assert rec is not None and rec["walk_block"] == best["walk_block"]
    b.step(2)
    # stepping after tuning matches single-system handles exactly
    for sid, st in zip(ids, sts):
        r = gb.GpuResidentLeapfrog(1.0, 0.01, 0.5)
        r.upload(st)
        r.step_many(1e-3, 4)
        assert np.array_equal(b.snapshot(sid).pos, r.snapshot().pos)
