"""Autotuning of the walk launch (gx_autotune / gx_batch_autotune): the sweep leaves
the state bit-identical, records its winner for the N bucket, block size and scheduling
never change a result, and the warp grouping changes only the FP32 summation order."""

import numpy as np
import pytest

import galaxy_b200 as gb
from oracle import oracle

pytestmark = pytest.mark.gpu


def test_launch_configuration_never_changes_results():
    st = gb.ic.collision(65_536, 11)
    for group in (8, 16, 32):
        ref = gb.GpuLbvh(1.0, 0.02, 0.5, walk_block=128, walk_group=group).accelerations(st)
        for block, ctas in ((64, 0), (128, 4), (64, 3), (96, 1)):
            got = gb.GpuLbvh(1.0, 0.02, 0.5, walk_block=block, walk_ctas_per_sm=ctas,
                             walk_group=group).accelerations(st)
            assert np.array_equal(got, ref), (group, block, ctas)


def test_walk_groups_take_the_same_terms():
    """8, 16 or 32 targets a warp: the same interaction counts (every lane's exact
    decisions) and accelerations within the FP32 parity bounds of the reference walk."""
    st = gb.ic.plummer(20_000, 5)
    ref = oracle.lbvh_accelerations(st.pos, st.mass, 1.0, 0.01, 0.5, threads=oracle.max_threads())
    counts = set()
    for group in (8, 16, 32):
        h = gb.GpuLbvh(1.0, 0.01, 0.5, walk_group=group, stats=True)
        a = h.accelerations(st)
        s = h.stats()
        counts.add((s["leaf_interactions"], s["far_interactions"], s["nodes_opened"]))
        err = oracle.per_particle_rel_err(a, ref)
        assert np.median(err) <= 1e-6 and np.percentile(err, 99) <= 1e-5, group
    assert len(counts) == 1


def test_autotune_keeps_state_and_records_bucket():
    st = gb.ic.collision(98_304, 12)  # bucket floor(log2 98304) = 16
    r = gb.GpuResidentLeapfrog(1.0, 0.02, 0.5)
    r.upload(st)
    r.step_many(5e-4, 3)
    before = r.snapshot()
    acc_before = r.accelerations()
    best = r.autotune(repeats=2)
    assert best["tried"] and best["ms"] == min(t["ms"] for t in best["tried"])
    assert best["walk_block"] in (64, 128) and best["walk_group"] in (8, 16, 32)
    assert {t["walk_group"] for t in best["tried"]} == {8, 16, 32}
    after = r.snapshot()
    assert np.array_equal(before.pos, after.pos) and np.array_equal(before.vel, after.vel)
    # the handle now walks with the tuned grouping: a handle given it explicitly agrees
    acc_after = r.accelerations()
    fixed = gb.GpuLbvh(1.0, 0.02, 0.5, walk_group=best["walk_group"]).accelerations(after)
    assert np.array_equal(acc_after, fixed)
    err = oracle.per_particle_rel_err(acc_after, acc_before)
    assert np.percentile(err, 99) <= 1e-5
    key = ("walk_block", "walk_ctas_per_sm", "walk_group")
    for n in (65_536, 100_000, 131_071):
        rec = gb.tuning_lookup(n)
        assert rec is not None and tuple(rec[k] for k in key) == tuple(best[k] for k in key)
    assert gb.tuning_lookup(98_304, precision="f64") is None
    # new handles of this bucket take the table's entry: one with the tuned options given
    # explicitly follows the same trajectory
    twin = gb.GpuResidentLeapfrog(1.0, 0.02, 0.5)
    explicit = gb.GpuResidentLeapfrog(1.0, 0.02, 0.5, **{k: best[k] for k in key})
    for h in (twin, explicit):
        h.upload(st)
        h.step_many(5e-4, 4)
    assert np.array_equal(twin.snapshot().pos, explicit.snapshot().pos)


def test_autotune_keeps_a_fixed_grouping():
    st = gb.ic.collision(40_000, 13)
    r = gb.GpuResidentLeapfrog(1.0, 0.02, 0.5, walk_group=16)
    r.upload(st)
    r.step_many(5e-4, 2)
    best = r.autotune(repeats=1)
    assert best["walk_group"] == 16
    assert {t["walk_group"] for t in best["tried"]} == {16}
    # the table's entry leaves the grouping open for handles that do not fix it
    rec = gb.tuning_lookup(40_000)
    assert rec is not None and rec["walk_group"] == 0


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
