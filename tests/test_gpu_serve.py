"""Continuous-batching server: requests submitted while others run are admitted
between batched steps; every result equals the same system stepped alone, bit for
bit; a request larger than the device budget is rejected, not queued forever."""

import threading
import time

import numpy as np
import pytest

import galaxy_b200 as gb

pytestmark = pytest.mark.gpu


def _alone(st, eps, theta, dt, steps):
    r = gb.GpuResidentLeapfrog(1.0, eps, theta)
    r.upload(st)
    r.step_many(dt, steps)
    return r.snapshot()


def test_results_equal_alone_with_staggered_arrivals():
    reqs = [(gb.ic.collision(6000 + 1000 * i, 10 + i, mass_ratio=1.0 + i, pericentre=3.0), 0.02, 0.5, 5e-4, 20 + 7 * i)
            for i in range(5)] + [(gb.ic.plummer(3000, 77), 0.01, 0.7, 1e-3, 15)]
    srv = gb.Server()
    rids = []
    for k, (st, eps, th, dt, steps) in enumerate(reqs):
        rids.append(srv.submit(st, 1.0, eps, th, dt, steps))
        time.sleep(0.02 * (k % 3))  # later requests join a batch already in flight
    for rid in rids:
        srv.wait(rid, 300)
    s = srv.stats()
    assert s["completed"] == len(reqs) and s["max_live"] >= 2
    for rid, (st, eps, th, dt, steps) in zip(rids, reqs):
        got = srv.result(rid)
        ref = _alone(st, eps, th, dt, steps)
        assert np.array_equal(got.pos, ref.pos) and np.array_equal(got.vel, ref.vel)
        assert abs(got.time - steps * dt) < 1e-12
    assert s["step_ms_p99"] >= s["step_ms_p50"] > 0


def test_submit_from_threads():
    srv = gb.Server()
    out = {}

    def client(i):
        st = gb.ic.plummer(2000 + 100 * i, 200 + i)
        out[i] = (srv.submit(st, 1.0, 0.01, 0.5, 1e-3, 10), st)

    th = [threading.Thread(target=client, args=(i,)) for i in range(4)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for i, (rid, st) in out.items():
        srv.wait(rid, 300)
        ref = _alone(st, 0.01, 0.5, 1e-3, 10)
        got = srv.result(rid)
        assert np.array_equal(got.pos, ref.pos)


def test_oversize_request_rejected():
    srv = gb.Server(budget_bytes=20 << 20)
    rid = srv.submit(gb.ic.plummer(300_000, 1), 1.0, 0.01, 0.5, 1e-3, 5)
    with pytest.raises(gb.GxError):
        srv.wait(rid, 60)
    assert srv.status(rid)[0] == gb.Server.REJECTED
    small = srv.submit(gb.ic.plummer(2000, 2), 1.0, 0.01, 0.5, 1e-3, 5)
    srv.wait(small, 60)
    assert srv.status(small)[0] == gb.Server.DONE


def test_budget_admits_as_room_frees():
    """A budget that holds two systems at a time: four requests all finish, at most two
    are resident at once, the later ones wait in the queue, and every result still
    equals the system stepped alone."""
    one = gb.Batch().system_bytes(20_000)
    srv = gb.Server(budget_bytes=int(2.4 * one))
    reqs = [(gb.ic.plummer(20_000, 300 + i), 12 + 4 * i) for i in range(4)]
    rids = [srv.submit(st, 1.0, 0.01, 0.5, 1e-3, steps) for st, steps in reqs]
    for rid in rids:
        srv.wait(rid, 300)
    s = srv.stats()
    assert s["completed"] == 4 and s["max_live"] == 2
    assert s["queue_s_p99"] > 0.0
    for rid, (st, steps) in zip(rids, reqs):
        got = srv.result(rid)
        ref = _alone(st, 0.01, 0.5, 1e-3, steps)
        assert np.array_equal(got.pos, ref.pos) and np.array_equal(got.vel, ref.vel)


def test_snapshot_emission_matches_alone(tmp_path):
    """Served scenarios emit GLXYSNAP v4 files every K steps and after the last; each file
    holds the state the same system has at that step when stepped alone."""
    from galaxy_b200 import snapshot as snap

    reqs = [(gb.ic.plummer(5000 + 1000 * i, 400 + i), 12 + i) for i in range(3)]
    srv = gb.Server()
    rids = [srv.submit(st, 1.0, 0.01, 0.5, 1e-3, steps, snapshot_every=5, snapshot_prefix=str(tmp_path / f"r{k}"),
                       rng_seed=k, config_hash=77)
            for k, (st, steps) in enumerate(reqs)]
    for rid in rids:
        srv.wait(rid, 300)
    for k, (rid, (st, steps)) in enumerate(zip(rids, reqs)):
        marks = sorted({5, 10, steps})
        assert srv.snapshots_written(rid) == len(marks)
        r = gb.GpuResidentLeapfrog(1.0, 0.01, 0.5)
        r.upload(st)
        done = 0
        for m in marks:
            r.step_many(1e-3, m - done)
            done = m
            ref = r.snapshot()
            h, c = snap.read(tmp_path / f"r{k}.{m:08d}.glxysnap")
            assert (h["step"], h["n_particles"], h["softening"], h["rng_seed"], h["config_hash"]) == (
                m, len(st), 0.01, k, 77)
            assert abs(h["time"] - m * 1e-3) < 1e-15
            assert np.array_equal(c["pos"], ref.pos) and np.array_equal(c["vel"], ref.vel)
            assert np.array_equal(c["mass"], st.mass.astype(np.float32).astype(np.float64))
        final = srv.result(rid)
        assert np.array_equal(final.pos, ref.pos) and np.array_equal(final.vel, ref.vel)


def test_cancel_queued_and_running_leaves_others_exact(tmp_path):
    """Fault injection on the host: a request cancelled while queued and one cancelled
    mid-stream; the rest finish bit-identical to running alone, and every step appears
    in the JSON-lines metrics stream."""
    import json

    one = gb.Batch().system_bytes(8_000)
    srv = gb.Server(budget_bytes=int(2.4 * one))  # two resident at a time
    log = tmp_path / "metrics.jsonl"
    srv.set_metrics_log(str(log))
    sts = [gb.ic.plummer(8_000, 500 + i) for i in range(4)]
    rids = [srv.submit(st, 1.0, 0.01, 0.5, 1e-3, 400 if i == 0 else 30) for i, st in enumerate(sts)]
    srv.cancel(rids[3])  # still queued behind the two resident ones
    t0 = time.time()
    while srv.status(rids[0])[1] < 5 and time.time() - t0 < 60:
        time.sleep(0.005)
    srv.cancel(rids[0])  # running: leaves at the next step boundary
    for rid in (rids[0], rids[3]):
        with pytest.raises(gb.GxError) as e:
            srv.wait(rid, 60)
        assert e.value.code == -9
        assert srv.status(rid)[0] == gb.Server.CANCELLED
    for rid, st in zip(rids[1:3], sts[1:3]):
        srv.wait(rid, 300)
        ref = _alone(st, 0.01, 0.5, 1e-3, 30)
        assert np.array_equal(srv.result(rid).pos, ref.pos)
    with pytest.raises(gb.GxError):
        srv.cancel(rids[1])  # already finished
    s = srv.stats()
    srv.set_metrics_log(None)
    lines = [json.loads(x) for x in log.read_text().splitlines()]
    assert len(lines) == s["steps"] and lines[-1]["completed"] == s["completed"]
    assert all(x["ms"] > 0 and x["live"] >= 1 for x in lines)
