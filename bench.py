"""Benchmark of the LBVH Barnes-Hut gravity step on B200.

Default workload (one line of JSON on rank 0): the two-galaxy collision, 2 x 524,288
particles (halo 60% / exponential disk 35% / Hernquist bulge 5% per galaxy, mass
ratio 1:1, parabolic orbit, pericentre 4 Rd, disks inclined 30 and 60 degrees),
eps = 0.02, theta = 0.5, dt = 5e-4, FP32 walk with FP64 positions/velocities. A step
is one resident KDK step (kick + drift + bbox, Morton, 4 sort passes, build +
aggregation, tree walk). The state plus tree (~330 MB) is larger than the 126 MB
L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config collision|plummer|batched|serving|precision|sph]

Under torchrun each rank steps its own replica (a single system does not shard:
replicas only) and value = all ranks' particle-steps / max-over-ranks device time.
--impl reference times the reference algorithm's CPU implementation (the oracle's
C++ restatement of Lbvh + LeapfrogKdk; the Rust reference cannot be built here) on
the host cores with all threads, rank 0 only.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from galaxy_b200 import ranks, roofline  # noqa: E402  (rank discovery, reductions, roofline arithmetic)

METRIC = "particle-steps/s at theta=0.5 (resident KDK step, plain single-system path)"
N_PER_GALAXY = 524_288


def _peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device, self.lines, self.proc = device, [], None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


WORKLOADS = {
    "collision": dict(eps=0.02, theta=0.5, dt=5e-4, name="collision-2x524288", multipole="mono",
                      n=2 * N_PER_GALAXY),
    "plummer": dict(eps=0.01, theta=0.5, dt=1e-3, name="plummer-16384", multipole="quad", n=16_384),
}


def workload(config: str, seed: int):
    """The seeded workload state (product library's generator) and its parameters."""
    import galaxy_b200 as gb

    p = WORKLOADS["plummer" if config == "plummer" else "collision"]
    if config == "plummer":
        return gb.ic.plummer(p["n"], seed), p
    return gb.ic.collision(p["n"], seed, mass_ratio=1.0, pericentre=4.0, incl1_deg=30.0, incl2_deg=60.0), p


def workload_oracle(config: str, seed: int):
    """The same inputs from the oracle library's copy of the generator, so the CPU
    reference arm never loads the product library."""
    from oracle import oracle

    p = WORKLOADS["plummer" if config == "plummer" else "collision"]
    if config == "plummer":
        return oracle.ic_plummer(p["n"], seed), p
    return oracle.ic_collision(p["n"], seed, 1.0, 4.0, 30.0, 60.0), p


def native_libraries() -> list:
    """Shared libraries of this repository mapped into this process (from /proc/self/maps)."""
    try:
        with open("/proc/self/maps") as f:
            paths = {ln.split()[-1] for ln in f if ln.rstrip().endswith(".so")}
    except OSError:
        return []
    return sorted(os.path.relpath(q, ROOT) for q in paths if q.startswith(ROOT + os.sep))


def shared_config(p: dict, n: int) -> dict:
    """The workload as both arms print it (the same dict in the GPU and the CPU line)."""
    return {"workload": p["name"], "particles": n, "theta": p["theta"], "eps": p["eps"], "dt": p["dt"], "g": 1.0,
            "multipole": p["multipole"], "seed": 0,
            "l2": (f"working set ~{352 * n / 1e6:.0f} MB > 126 MB L2 (no flush needed)" if 352 * n > 126e6 else
                   f"working set ~{352 * n / 1e6:.0f} MB fits in L2: steps replay back to back with the state "
                   f"resident, as a resident integrator runs (not a flushed-cache number)")}


# ---- algorithmic work per launch (bytes / flops) ----------------------------------------
def profiled_walk(workload_name: str, key: str):
    """A per-launch figure of the walk (`traffic_bytes_per_launch`, `instructions_per_launch`)
    from the committed ncu summary of this workload, or None."""
    import re

    path = os.path.join(ROOT, "profiles", f"k_walk_f32_{workload_name.replace('collision-', 'collision_')}.md")
    try:
        m = re.search(key + r":\s*(\d+)", open(path).read())
        return int(m.group(1)) if m else None
    except OSError:
        return None


def cpu_sample_step(pos, mass, params, threads: int, n_targets: int, rng) -> float:
    """Seconds for one CPU force evaluation estimated from a bounded sample: the oracle's
    full tree build plus the walk of n_targets random targets, scaled to all N targets."""
    from oracle import oracle

    n = len(mass)
    t0 = time.perf_counter()
    oracle.lbvh_accelerations_subset(pos, mass, 1.0, params["eps"], params["theta"], np.zeros(1, np.uint32),
                                     threads=threads)
    t_build = time.perf_counter() - t0
    tg = rng.choice(n, n_targets, replace=False).astype(np.uint32)
    t0 = time.perf_counter()
    oracle.lbvh_accelerations_subset(pos, mass, 1.0, params["eps"], params["theta"], tg, threads=threads)
    t_walk = time.perf_counter() - t0 - t_build
    return t_build + max(t_walk, 0.0) * n / n_targets


def walk_roofline(p: dict, n: int, stage: dict, counts: dict, peaks: dict, radix_bits: int = 8,
                  walk_group: int = 32) -> dict:
    """Roofline of the dominant kernel (the FP32 walk) and the HBM fractions of the other
    stages: algorithmic flops (or bytes) per launch over the launch's CUDA-event time."""
    quad = p["multipole"] == "quad"
    sb = roofline.stage_bytes(n, key64=False, quad=quad, radix_bits=radix_bits)
    passes = roofline.sort_passes(False, radix_bits)
    flops = roofline.walk_flops(counts["leaf"], counts["far"], counts["open"], quad=quad)
    walk_s = stage["ms_walk"] / 1e3
    mhz = peaks.get("sm_max_mhz", 1965.0)
    fp32_peak = 148 * 128 * 2 * mhz * 1e6 / 1e12
    achieved = flops / walk_s / 1e12
    hbm = peaks.get("hbm_gbs", 6650.0)
    sort_gbs = roofline.hbm_fraction(sb["sort"], stage["ms_sort"], hbm)[0]
    build_gbs = roofline.hbm_fraction(sb["build"], stage["ms_build"], hbm)[0]
    mort_gbs = roofline.hbm_fraction(sb["kick_drift_bbox"] + sb["morton"], stage["ms_bbox_morton"], hbm)[0]
    prof = f"profiles/k_walk_f32_{p['name'].replace('collision-', 'collision_')}.md"
    # the capture of the same warp grouping as this run's walk
    traffic = profiled_walk(p["name"], f"traffic_bytes_per_launch_g{walk_group}")
    inst = profiled_walk(p["name"], f"instructions_per_launch_g{walk_group}")
    issue = None
    if inst:
        rate, frac = roofline.issue_fraction(inst, stage["ms_walk"], 148, mhz)
        issue = {"achieved_ginst_s": rate, "peak_ginst_s": 148 * 4 * mhz / 1e3, "frac": frac,
                 "source": f"warp instructions per launch from {prof} over this run's walk time; peak = one warp "
                           f"instruction per scheduler per clock"}
    return {"kernel": "k_walk_f32 (tree walk)", "bound": "fp32", "achieved": achieved, "peak": fp32_peak,
            "unit": "TFLOP/s", "frac": achieved / fp32_peak, "traffic": traffic,
            "traffic_source": f"ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch with {walk_group} "
                              f"targets a warp, {prof}" if traffic else None, "walk_group": walk_group,
            "algorithmic_bytes_per_launch": sb["walk"],
            "peak_source": "nominal FP32 CUDA-core rate 148 SM x 128 lanes x 2 x clocks.max.sm (MEASURED_PEAKS.json "
                           "has no FP32 figure); no tensor-core work in this path",
            "flops_per_launch": flops, "ms_per_launch": stage["ms_walk"], "issue": issue,
            "interactions_per_particle": (counts["leaf"] + counts["far"]) / n,
            "hbm_stages": {
                f"sort ({passes} onesweep passes, {radix_bits}-bit digits)": {
                    "achieved_gbs": sort_gbs, "frac": sort_gbs / hbm, "ms": stage["ms_sort"], "bytes": sb["sort"]},
                "build + aggregation": {"achieved_gbs": build_gbs, "frac": build_gbs / hbm, "ms": stage["ms_build"],
                                        "bytes": sb["build"]},
                "kick/drift/bbox + Morton": {"achieved_gbs": mort_gbs, "frac": mort_gbs / hbm,
                                             "ms": stage["ms_bbox_morton"],
                                             "bytes": sb["kick_drift_bbox"] + sb["morton"]},
                "peak_gbs": hbm, "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"}}


def run_reference_sph(args, threads: int):
    """The gas-mode reference arm: the oracle's GravitySph (Lbvh gravity + adaptive-h density
    + hydro, h warm-started across steps) driving LeapfrogKdk on a bounded sample of the
    same gas/star mix (--gas / 16 gas particles and as many stars), per particle."""
    from galaxy_b200 import workloads
    from oracle import oracle

    ng = max(args.gas // 16, 4096)
    st = workloads.gas_star_mix(ng, ng, seed=0)
    n = len(st)
    gs = oracle.GravitySph(1.0, 0.01, 0.5, threads=threads)
    pos, vel = st.pos.copy(), st.vel.copy()
    gs.step_many(pos, vel, st.mass, st.kind, 1e-4, max(args.warmup, 1))  # prime + warm-up steps
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        gs.step_many(pos, vel, st.mass, st.kind, 1e-4, 1)
        times.append(time.perf_counter() - t0)
    t_step = statistics.mean(times)
    value = n / t_step
    sample = (f"per step: one KDK step of a {n}-particle gas/star mix ({ng} gas) through the oracle's "
              f"GravitySph with {threads} threads (C++ restatement of the reference; the Rust crate cannot "
              f"be built here), per particle")
    line = {"impl": "reference", "metric": "particle-steps/s (resident KDK step with SPH on the gas subset)",
            "value": value, "unit": "particle-steps/s", "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"gas-star-mix-{args.gas}+{args.gas}", "sample_particles": n, "gas": ng,
                       "eps": 0.01, "theta": 0.5, "dt": 1e-4,
                       "sampled": f"the rate is per particle-step of a {ng}+{ng} sample of the workload "
                                  f"(the full size does not fit the run's time on the host)"},
            "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_reference(args):
    dist, rank, ws, local = ranks.init()
    if rank != 0:
        # rank 0 alone times the CPU reference; the other ranks have no work
        if dist is not None:
            dist.destroy_process_group()
        return
    from oracle import oracle

    threads = os.cpu_count() or 1
    if args.config == "sph":
        run_reference_sph(args, threads)
        if dist is not None:
            dist.destroy_process_group()
        return
    (pos, vel, mass), p = workload_oracle(args.config, 0)
    n = len(mass)
    # Whole KDK steps of the full system (LeapfrogKdk + Lbvh: a serial tree build and the
    # walk over every target on all host threads, then the kicks and the drift), the
    # oracle's C++ restatement of the reference (the Rust crate cannot be built here).
    # The priming force evaluation runs before the warm-up steps.
    kdk = oracle.LeapfrogKdkLbvh(1.0, p["eps"], p["theta"], threads=threads)
    kdk.step_many(pos, vel, mass, p["dt"], 0)
    kdk.prime(pos, mass)
    for _ in range(args.warmup):
        kdk.step_many(pos, vel, mass, p["dt"], 1)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        kdk.step_many(pos, vel, mass, p["dt"], 1)
        times.append(time.perf_counter() - t0)
    t_step = statistics.mean(times)
    value = n / t_step
    ref_config = shared_config(p, n)
    if p["multipole"] != "mono":
        ref_config["multipole"] = "mono (the reference has no quadrupole nodes)"
    sample = (f"whole KDK steps of the full {n}-particle system: tree build, walk of every target with "
              f"{threads} threads, kicks and drift (the oracle's C++ restatement of LeapfrogKdk + Lbvh; monopole, "
              f"as the reference)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": ref_config,
            "step_ms_p50": float(np.percentile(times, 50)) * 1e3, "step_ms_p99": float(np.percentile(times, 99)) * 1e3,
            "native_libraries": native_libraries(),
            "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def measure_mix(args, dist, rank, ws, local, steps: int, warmup: int) -> dict:
    """The batched uneven-systems mix (N log-uniform in [4096, 262144], half Plummer
    spheres, half disk + halo galaxies, eps 0.01, theta 0.5, dt 1e-3 / 5e-4): the batch
    (one launch per stage, persistent work-stealing walk, CUDA-graph replay) against the
    plain single-system path stepping the same systems one after another. Per-step device
    times (CUDA events) of both; the max over ranks; each rank builds only its shard."""
    import galaxy_b200 as gb
    from galaxy_b200 import workloads

    sizes = workloads.batched_sizes(args.systems * ws, seed=0)
    mine = ranks.shard(sizes, ws)[rank]
    mix = workloads.batched_mix(args.systems * ws, seed=0, indices=mine)
    n_tot = sum(len(m.state) for m in mix)
    k63 = args.morton63
    b = gb.Batch(device=local, morton63=k63)
    for m in mix:
        b.add(m.state, m.g, m.eps, m.theta, m.dt)
    b.step(max(warmup, 1))
    tune = b.autotune(repeats=2)  # persistent walk launch for this batch (untimed)
    b.step(1)  # re-capture the step graph outside the timed region
    gb.device_synchronize(local)
    ranks.barrier(dist, local)
    ms = []
    for _ in range(steps):
        b.step(1)
        ms.append(b.stats()["ms_last_step"])
    gb.device_synchronize(local)
    ranks.barrier(dist, local)
    t = ranks.max_over_ranks(dist, sum(ms) / 1e3, local)
    n_all = ranks.sum_over_ranks(dist, n_tot, local)  # particles on all ranks
    value = n_all * steps / t
    del b
    # plain path: the same systems, each stepped alone by the single-system handle
    hs = []
    for m in mix:
        r = gb.GpuResidentLeapfrog(m.g, m.eps, m.theta, device=local, morton63=k63)
        r.upload(m.state)
        r.step_many(m.dt, 1)
        if gb.tuning_lookup(len(m.state), morton63=k63, device=local) is None:
            r.autotune(repeats=2)  # the plain path is tuned per N bucket too
        r.step_many(m.dt, 2)  # capture the handle's step graph before timing (as the batch's)
        hs.append((r, m))
    k_plain = max(1, min(steps, 3))
    t_plain = 0.0
    plain_ms = []
    by_bucket = {}  # floor(log2 N): [systems, particles, device ms per pass]
    for rep in range(k_plain):
        t_pass = 0.0
        for r, m in hs:
            t_sys = r.step_many_timed(m.dt, 1)
            t_pass += t_sys
            if rep == k_plain - 1:
                e = by_bucket.setdefault(int(np.log2(len(m.state))), [0, 0, 0.0])
                e[0] += 1
                e[1] += len(m.state)
                e[2] += t_sys
        plain_ms.append(t_pass)
        t_plain += t_pass / 1e3
    t_plain = ranks.max_over_ranks(dist, t_plain, local)
    plain = n_all * k_plain / t_plain
    del hs
    return {"workload": f"batched-{args.systems}-systems", "systems": args.systems * ws, "particles": n_all,
            "morton_bits": 63 if k63 else 30, "n_range": [4096, 262144], "theta": 0.5, "eps": 0.01,
            "dt": [1e-3, 5e-4], "value": value, "unit": "particle-steps/s", "steps": steps,
            "step_ms_p50": float(np.percentile(ms, 50)), "step_ms_p99": float(np.percentile(ms, 99)),
            "plain_value": plain, "plain_steps": k_plain,
            "plain_pass_ms_p50": float(np.percentile(plain_ms, 50)),
            "plain_how": "same systems, one single-system handle each, stepped one after another (device time of "
                         "each step summed)",
            "batched_over_plain": value / plain, "gpu_launches_per_step": 13 if k63 else 9,
            "batch_ns_per_particle_step": float(np.percentile(ms, 50)) * 1e6 / max(n_tot, 1),
            "plain_by_log2_n": {str(k): {"systems": v[0], "particles": v[1], "ms": v[2],
                                         "ns_per_particle_step": v[2] * 1e6 / v[1]}
                                for k, v in sorted(by_bucket.items())},
            "walk_launch": {k: tune[k] for k in ("walk_block", "walk_ctas_per_sm")}}


def run_ours(args):
    dist, rank, ws, local = ranks.init()
    import galaxy_b200 as gb

    st, p = workload(args.config, rank)
    n = len(st)
    dt = p["dt"]
    peaks = _peaks()

    # --- headline: resident steps, CUDA-graph replay, device time (CUDA events) ---
    mp = p["multipole"]
    r = gb.GpuResidentLeapfrog(1.0, p["eps"], p["theta"], multipole=mp, device=local, walk_group=args.walk_group)
    r.upload(st)
    r.step_many(dt, args.warmup)
    tune = r.autotune(repeats=3)  # walk launch for this N bucket (outside the timed region)
    if args.walk_group:
        tune["walk_group"] = args.walk_group  # fixed by the option (the handle keeps it)
    r.step_many(dt, 1)  # re-capture the step graph outside the timed region
    clocks = ClockSampler(local)
    clocks.start()
    gb.device_synchronize(local)
    ranks.barrier(dist, local)
    ms = r.step_many_timed(dt, args.steps)
    gb.device_synchronize(local)
    ranks.barrier(dist, local)
    clk = clocks.stop()
    ms_max = ranks.max_over_ranks(dist, ms, local)
    value = n * ws * args.steps / (ms_max / 1e3)
    # per-step latency of the same path: single graph replays, each timed on the device
    lat = [r.step_many_timed(dt, 1) for _ in range(max(args.steps, 10))]

    # --- e2e: the reference-facing ForceSolver path (LeapfrogKdk on host arrays) ---
    pinned = gb.PinnedState.from_state(st)
    h = gb.GpuLbvh(1.0, p["eps"], p["theta"], multipole=mp, device=local, walk_group=args.walk_group)
    primed = h.kdk_step_host(pinned, dt, primed=False)  # prime + one step (warm-up)
    k_e2e = max(1, min(args.steps, 10))
    reps = []
    for _ in range(3):  # host-memory-bound kicks vary between runs: the median of three
        gb.device_synchronize(local)
        ranks.barrier(dist, local)
        t0 = time.perf_counter()
        for _ in range(k_e2e):
            primed = h.kdk_step_host(pinned, dt, primed=primed)
        gb.device_synchronize(local)
        t_rep = time.perf_counter() - t0
        ranks.barrier(dist, local)
        reps.append(ranks.max_over_ranks(dist, t_rep, local))
    t_e2e = statistics.median(reps)
    e2e = {"value": n * ws * k_e2e / t_e2e, "unit": "particle-steps/s", "h2d_bytes_per_step": 32 * n,
           "d2h_bytes_per_step": 24 * n, "steps": k_e2e, "repetitions": 3,
           "path": "LeapfrogKdk on pinned host f64 arrays, gx_accelerations per step (upload pos+mass, download acc)"}
    del pinned, h

    # --- per-stage device times (eager launches with CUDA events on the handle's stream) ---
    rs = gb.GpuResidentLeapfrog(1.0, p["eps"], p["theta"], multipole=mp, device=local, stage_times=True,
                                walk_group=args.walk_group)
    rs.upload(st)
    stage = {"ms_bbox_morton": 0.0, "ms_sort": 0.0, "ms_build": 0.0, "ms_walk": 0.0}
    k_st = max(1, min(args.steps, 10))
    rs.step(dt)
    for _ in range(k_st):
        rs.step(dt)
        s = rs.stats()
        for k in stage:
            stage[k] += s[k] / k_st
    del rs
    counts_h = gb.GpuLbvh(1.0, p["eps"], p["theta"], multipole=mp, device=local, stats=True)
    counts_h.accelerations(st)
    c = counts_h.stats()
    del counts_h
    counts = {"leaf": c["leaf_interactions"], "far": c["far_interactions"], "open": c["nodes_opened"],
              "pair_records": c["warp_node_visits"], "f64_rechecks": c["f64_rechecks"]}
    roof = walk_roofline(p, n, stage, counts, peaks, tune["radix_bits"], tune["walk_group"])

    # --- the batched mix (BASELINE metric: batched vs plain, p50/p99), default workload ---
    mix = None
    if args.config == "collision" and not args.no_batched:
        mix = measure_mix(args, dist, rank, ws, local, steps=max(3, min(args.steps, 5)), warmup=args.warmup)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        from oracle import oracle

        # the serial reference (one thread: Lbvh's per-target loop, solvers/src/lbvh.rs:673-675)
        rng = np.random.default_rng(1)
        t = statistics.mean(cpu_sample_step(st.pos, st.mass, p, 1, 8192, rng) for _ in range(2))
        cpu = {"value": n / t, "unit": "particle-steps/s", "cores": 1, "kind": "port",
               "sample": f"2 samples of: the full {n}-particle tree build + the walk of 8192 random targets on one "
                         f"thread, scaled to all targets (the oracle's serial C++ restatement of Lbvh, as the "
                         f"reference's serial per-target loop); whole all-core KDK steps are the reference arm"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": shared_config(p, n),
                "implementation": {"precision": "FP32 walk (Kahan), FP64 pos/vel and opening re-checks",
                                   "parallelism": "replicas" if ws > 1 else "single system", "cuda_graph": True,
                                   "walk_launch": {k: tune[k] for k in ("walk_block", "walk_ctas_per_sm",
                                                                        "walk_group")},
                                   "sort": {"radix_bits": tune["radix_bits"], "sort_ms": tune["sort_ms"]}},
                "step_ms_p50": float(np.percentile(lat, 50)), "step_ms_p99": float(np.percentile(lat, 99)),
                "e2e": e2e, "gpu_launches": (5 + roofline.sort_passes(False, tune["radix_bits"])) * args.steps,
                "roofline": roof, "cpu_baseline": cpu,
                "clocks": clk, "stage_ms": stage, "walk_counts": counts}
        if mix is not None:
            line["batched_over_plain"] = mix["batched_over_plain"]
            line["batched"] = mix
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def run_batched(args):
    """256 independent systems in one batch vs the plain single-system path stepping
    the same systems one at a time (see measure_mix)."""
    import galaxy_b200 as gb

    dist, rank, ws, local = ranks.init()
    clocks = ClockSampler(local)
    clocks.start()
    mix = measure_mix(args, dist, rank, ws, local, steps=args.steps, warmup=args.warmup)
    clk = clocks.stop()
    del gb
    if rank == 0:
        line = {"metric": "particle-steps/s at theta=0.5, batched uneven systems", "value": mix["value"],
                "unit": "particle-steps/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": mix["step_ms_p50"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {k: mix[k] for k in ("workload", "systems", "particles", "morton_bits", "n_range", "theta",
                                               "eps", "dt")},
                "step_ms_p50": mix["step_ms_p50"], "step_ms_p99": mix["step_ms_p99"],
                "plain_path": {"value": mix["plain_value"], "unit": "particle-steps/s", "steps": mix["plain_steps"],
                               "how": mix["plain_how"]},
                "batched_over_plain": mix["batched_over_plain"],
                "gpu_launches": mix["gpu_launches_per_step"] * args.steps, "clocks": clk,
                "walk_launch": mix["walk_launch"], "batch_ns_per_particle_step": mix["batch_ns_per_particle_step"],
                "plain_by_log2_n": mix["plain_by_log2_n"]}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def run_serving(args):
    """A Poisson stream (50 req/s) of collision scenarios, N log-uniform in [16384,
    2097152], mass ratio U[1,10], pericentre U[2,8] Rd, 100-1000 steps each, served
    with continuous batching against a 150 GB budget for a fixed horizon."""
    import galaxy_b200 as gb
    from galaxy_b200 import workloads

    dist, rank, ws, local = ranks.init()
    reqs = workloads.request_stream(args.requests, rate=50.0, seed=rank)
    specs = [r.spec() for r in reqs]  # generated before the clock starts
    srv = gb.Server(budget_bytes=150 << 30, device=local, morton63=args.morton63)
    snap_dir = None
    if args.snapshot_every:
        import tempfile

        snap_dir = tempfile.mkdtemp(prefix="glxysnap_")
    clocks = ClockSampler(local)
    clocks.start()
    t0 = time.perf_counter()
    rids = []
    for r, sp in zip(reqs, specs):
        delay = r.arrival - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        if args.snapshot_every:
            rids.append(srv.submit(sp.state, sp.g, sp.eps, sp.theta, sp.dt, r.steps,
                                   snapshot_every=args.snapshot_every,
                                   snapshot_prefix=os.path.join(snap_dir, f"req{r.rid}"), rng_seed=r.seed))
        else:
            rids.append(srv.submit(sp.state, sp.g, sp.eps, sp.theta, sp.dt, r.steps))
    deadline = t0 + args.horizon
    for rid in rids:
        left = deadline - time.perf_counter()
        if left <= 0:
            break
        try:
            srv.wait(rid, left)
        except gb.GxError:
            break
    wall = time.perf_counter() - t0
    st = srv.stats()
    clk = clocks.stop()
    states = [srv.status(rid)[0] for rid in rids]
    counts = {name: sum(1 for x in states if x == code) for name, code in
              (("queued", srv.QUEUED), ("running", srv.RUNNING), ("completed", srv.DONE), ("rejected", srv.REJECTED),
               ("cancelled", srv.CANCELLED))}
    snaps = sum(srv.snapshots_written(rid) for rid in rids) if args.snapshot_every else 0
    srv.close()
    if snap_dir:
        import shutil

        shutil.rmtree(snap_dir, ignore_errors=True)
    if rank == 0:
        line = {"metric": "particle-steps/s at theta=0.5, served (continuous batching)",
                "value": st["particle_steps_per_s_device"], "unit": "particle-steps/s", "n_gpus": ws,
                "steps": st["steps"], "warmup": 0, "ms_per_step": st["step_ms_mean"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": f"serving-{args.requests}-requests", "rate_per_s": 50.0,
                           "n_range": [16384, 2097152], "steps_range": [100, 1000], "budget_gb": 150,
                           "horizon_s": args.horizon, "snapshot_every": args.snapshot_every},
                "snapshots_written": snaps,
                "step_ms_p50": st["step_ms_p50"], "step_ms_p99": st["step_ms_p99"],
                "wall_particle_steps_per_s": st["particle_steps"] / wall, "completed": st["completed"],
                "submitted": len(rids), "admitted": counts["running"] + counts["completed"],
                "rejected": counts["rejected"], "still_queued": counts["queued"], "request_states": counts,
                "demand_particle_steps": int(sum(r.n * r.steps for r in reqs)), "wall_s": wall,
                "max_live": st["max_live"], "queue_s_p50": st["queue_s_p50"],
                "queue_s_p99": st["queue_s_p99"], "clocks": clk}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def run_precision(args):
    """Precision study: the collision setup at N = 4,194,304 (mass ratio 1:3), for
    theta in {0.3, 0.5, 0.7}. Force error of the FP32 walk and of the FP64 walk (the
    reference's own arithmetic, bit-identical to its CPU Lbvh) against an FP64 direct
    sum on a seeded 65,536-particle subsample; per-particle error of FP32 against the
    FP64 walk; energy and angular-momentum drift of the FP32 run over --steps steps,
    and of both runs over the first --fp64-steps steps. Energies use the FP64 O(N^2)
    potential, evaluated only at the start and at the ends of the runs."""
    import galaxy_b200 as gb

    dist, rank, ws, local = ranks.init()
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    n = 4_194_304
    eps, dt = 0.02, 5e-4
    st = gb.ic.collision(n, 0, mass_ratio=3.0, pericentre=4.0, incl1_deg=30.0, incl2_deg=60.0)
    sub = np.sort(np.random.default_rng(65_536).choice(n, 65_536, replace=False)).astype(np.uint32)
    ds = gb.GpuLbvh(1.0, eps, 0.5, device=local).direct_sum_f64(st.pos, st.mass, sub)
    dsn = np.linalg.norm(ds, axis=1)

    def err_vs(a, ref, refn):
        e = np.linalg.norm(a - ref, axis=1) / refn
        return {"rms": float(np.sqrt(np.mean(e * e))), "median": float(np.median(e)),
                "p99": float(np.percentile(e, 99)), "max": float(e.max())}

    def rel(d, d0):
        return {"dE_rel": float((d["total"] - d0["total"]) / abs(d0["total"])),
                "dL_rel": float(np.linalg.norm(d["angular_momentum"] - d0["angular_momentum"])
                                / np.linalg.norm(d0["angular_momentum"]))}

    d0 = None  # the initial state's diagnostics (the same for every theta)
    results = []
    for theta in (0.3, 0.5, 0.7):
        a32 = gb.GpuLbvh(1.0, eps, theta, device=local).accelerations(st)[sub]
        a64 = gb.GpuLbvh(1.0, eps, theta, precision="f64", device=local).accelerations(st)[sub]
        k = args.steps
        k64 = min(args.fp64_steps, k)
        r = gb.GpuResidentLeapfrog(1.0, eps, theta, device=local)
        r.upload(st)
        if d0 is None:
            d0 = r.diagnostics(True)
        ms32 = r.step_many_timed(dt, k64)
        d32_short = r.diagnostics(True)
        if k > k64:
            ms32 += r.step_many_timed(dt, k - k64)
        d32 = r.diagnostics(True)
        del r
        r = gb.GpuResidentLeapfrog(1.0, eps, theta, precision="f64", device=local)
        r.upload(st)
        ms64 = r.step_many_timed(dt, k64)
        d64 = r.diagnostics(True)
        del r
        results.append({"theta": theta,
                        "force_err_vs_direct_sum": {"f32_walk": err_vs(a32, ds, dsn),
                                                    "f64_walk_reference": err_vs(a64, ds, dsn)},
                        "f32_vs_f64_walk": err_vs(a32, a64, np.linalg.norm(a64, axis=1)),
                        "drift_f32": {"steps": k, **rel(d32, d0)}, "ms_per_step_f32": ms32 / k,
                        "drift_at_fp64_horizon": {"steps": k64, "f32": rel(d32_short, d0),
                                                  "f64_reference": rel(d64, d0)},
                        "ms_per_step_f64": ms64 / k64})
    line = {"metric": "force error vs FP64 direct sum and energy drift (precision study)", "value": None,
            "unit": None, "n_gpus": 1, "steps": args.steps, "warmup": 0, "higher_is_better": False,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": "collision-4194304-q3", "particles": n, "mass_ratio": 3.0, "eps": eps, "dt": dt,
                       "subsample": 65_536, "subsample_seed": 65_536, "thetas": [0.3, 0.5, 0.7],
                       "fp64_steps": args.fp64_steps},
            "results": results}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


# Kernels a gas-mode step adds to the 9 of the gravity step: gather, scalars, 3 grids
# (keys, histogram, 4 sort passes, fill, mixed flags), seeds, density cell, density, h_max,
# hydro cell, pack, hydro, scatter.
SPH_LAUNCHES_PER_STEP = 2 + 3 * 8 + 8


def sph_roofline(n_gas: int, stage: dict, peaks: dict) -> dict:
    """Issue-rate roofline of the SPH root-find and hydro kernels: warp instructions per gas
    particle (ncu summary in profiles/, scaled to this n_gas) over this run's stage times;
    the peak is one warp instruction per scheduler per clock. FP64 work with L2-resident
    data: neither HBM nor tensor cores bound it."""
    import re

    path = os.path.join(ROOT, "profiles", "k_sph_kernels_gas_star_mix_262144.md")
    try:
        text = open(path).read()
        per = {k: float(re.search(k + r":\s*([0-9.]+)", text).group(1))
               for k in ("density_instructions_per_gas", "hydro_instructions_per_gas")}
    except (OSError, AttributeError):
        return {"kernel": "k_sph_density + k_sph_hydro", "bound": "issue", "achieved": None}
    mhz = peaks.get("sm_max_mhz", 1965.0)
    peak = 148 * 4 * mhz / 1e3  # G warp instructions / s
    ms_d = stage["ms_sph_density"]
    ms_h = stage["ms_sph"] - stage["ms_sph_density"]
    inst = (per["density_instructions_per_gas"] + per["hydro_instructions_per_gas"]) * n_gas
    ach = inst / ((ms_d + ms_h) * 1e-3) / 1e9
    return {"kernel": "k_sph_density + k_sph_hydro (FP64, one warp per gas particle)", "bound": "issue",
            "achieved": ach, "peak": peak, "unit": "G warp instructions/s", "frac": ach / peak,
            "traffic": None, "instructions_per_gas": per,
            "source": "instructions per gas particle from profiles/k_sph_kernels_gas_star_mix_262144.md; "
                      "time = this run's SPH stage events (grids, pack and scatter included)",
            "peak_source": "148 SMs x 4 schedulers x clocks.max.sm"}


def run_sph(args):
    """Resident gas mode (GpuResidentLeapfrog::new_with_sph, gpu_resident.rs:1393-1565):
    a gas blob of --gas particles inside a field of as many stars. Each step: KDK with
    gravity on every particle, then FP64 adaptive-h density, hydro force and the
    scatter-add on the gas rows. Device time over CUDA-graph replays; stage times of
    eager steps; e2e through GravitySph on host arrays (LeapfrogKdk in numpy); the CPU
    baseline is the oracle's GravitySph on a bounded 131,072-particle mix."""
    import galaxy_b200 as gb
    from galaxy_b200 import workloads

    dist, rank, ws, local = ranks.init()
    ng = args.gas
    st = workloads.gas_star_mix(ng, ng, seed=rank)
    n = len(st)
    eps, theta, dt = 0.01, 0.5, 1e-4
    peaks = _peaks()
    r = gb.GpuResidentLeapfrog.new_with_sph(1.0, eps, theta, device=local)
    r.upload(st)
    r.step_many(dt, args.warmup)
    tune = r.autotune(repeats=3)
    r.step_many(dt, 1)
    clocks = ClockSampler(local)
    clocks.start()
    gb.device_synchronize(local)
    ranks.barrier(dist, local)
    ms = r.step_many_timed(dt, args.steps)
    gb.device_synchronize(local)
    ranks.barrier(dist, local)
    clk = clocks.stop()
    ms_max = ranks.max_over_ranks(dist, ms, local)
    value = n * ws * args.steps / (ms_max / 1e3)
    cfl = r.min_stable_dt(0.25)

    rs = gb.GpuResidentLeapfrog.new_with_sph(1.0, eps, theta, device=local, stage_times=True)
    rs.upload(st)
    keys = ("ms_bbox_morton", "ms_sort", "ms_build", "ms_walk", "ms_sph", "ms_sph_density")
    stage = dict.fromkeys(keys, 0.0)
    k_st = max(1, min(args.steps, 5))
    rs.step(dt)
    for _ in range(k_st):
        rs.step(dt)
        sd = rs.stats()
        for k in keys:
            stage[k] += sd[k] / k_st
    del rs

    # e2e: GravitySph on host arrays driven by LeapfrogKdk (copies each step)
    host = st.copy()
    solver = gb.GpuGravitySph(1.0, eps, theta, device=local)
    kdk = gb.LeapfrogKdk()
    kdk.step(host, solver, dt)
    k_e2e = max(1, min(args.steps, 5))
    gb.device_synchronize(local)
    ranks.barrier(dist, local)
    t0 = time.perf_counter()
    for _ in range(k_e2e):
        kdk.step(host, solver, dt)
    t_e2e = ranks.max_over_ranks(dist, time.perf_counter() - t0, local)
    e2e = {"value": n * ws * k_e2e / t_e2e, "unit": "particle-steps/s", "h2d_bytes_per_step": 57 * n,
           "d2h_bytes_per_step": 24 * n, "steps": k_e2e,
           "path": "LeapfrogKdk (numpy kicks) + GpuGravitySph.accelerations on host arrays "
                   "(upload pos, vel, mass, kind, u; download acc)"}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        from oracle import oracle

        threads = os.cpu_count() or 1
        sample = workloads.gas_star_mix(65_536, 65_536, seed=7)
        gs = oracle.GravitySph(1.0, eps, theta, threads=threads)
        t0 = time.perf_counter()
        gs.accelerations(sample.pos, sample.vel, sample.mass, sample.kind)
        t = time.perf_counter() - t0
        cpu = {"value": len(sample) / t, "unit": "particle-steps/s", "cores": threads, "kind": "port",
               "sample": f"one GravitySph force evaluation (Lbvh gravity + adaptive-h density + hydro) of a "
                         f"131072-particle mix (65536 gas), {threads} threads, per particle (oracle C++ "
                         f"restatement)"}
    if rank == 0:
        gas_frac = stage["ms_sph"] / max(ms_max / args.steps, 1e-9)
        line = {"metric": "particle-steps/s (resident KDK step with SPH on the gas subset)", "value": value,
                "unit": "particle-steps/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64 (SPH), f32 (gravity walk)", "data": "synthetic",
                "config": {"workload": f"gas-star-mix-{ng}+{ng}", "particles_per_gpu": n, "gas": ng, "eps": eps,
                           "theta": theta, "dt": dt, "sph": "isothermal c_s 1, n_ngb 48, h_tol 1e-3, alpha 1, "
                                                        "beta 2, warm-started h",
                           "parallelism": "replicas" if ws > 1 else "single system", "cuda_graph": True,
                           "l2": f"working set ~{900 * n / 1e6:.0f} MB > 126 MB L2 (no flush needed)",
                           "walk_launch": {k: tune[k] for k in ("walk_block", "walk_ctas_per_sm", "walk_group")}},
                "gas_particle_steps_per_s": ng * ws * args.steps / (ms_max / 1e3),
                "e2e": e2e, "gpu_launches": (9 + SPH_LAUNCHES_PER_STEP) * args.steps, "cpu_baseline": cpu,
                "clocks": clk, "stage_ms": stage, "sph_share_of_step": gas_frac, "min_stable_dt_c0.25": cfl,
                "roofline": sph_roofline(ng, stage, peaks)}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="collision",
                    choices=["collision", "plummer", "batched", "serving", "precision", "sph"])
    ap.add_argument("--gas", type=int, default=1 << 20, help="sph: gas particles (and as many stars)")
    ap.add_argument("--systems", type=int, default=256, help="batched: number of systems")
    ap.add_argument("--requests", type=int, default=24, help="serving: requests in the stream")
    ap.add_argument("--horizon", type=float, default=60.0, help="serving: seconds to serve")
    ap.add_argument("--morton30", dest="morton63", action="store_false",
                    help="batched mix / serving: the reference's 30-bit Morton keys (default 63-bit)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.set_defaults(morton63=True)
    ap.add_argument("--no-batched", action="store_true", help="default workload: skip the batched-mix measurement")
    ap.add_argument("--walk-group", type=int, default=0, choices=[0, 8, 16, 32],
                    help="targets per warp of the walk (0: tuned)")
    ap.add_argument("--fp64-steps", type=int, default=100, help="precision: horizon of the FP64 run")
    ap.add_argument("--snapshot-every", type=int, default=0, help="serving: emit GLXYSNAP v4 files every K steps")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.config == "batched":
        run_batched(args)
    elif args.config == "serving":
        run_serving(args)
    elif args.config == "precision":
        run_precision(args)
    elif args.config == "sph":
        run_sph(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
