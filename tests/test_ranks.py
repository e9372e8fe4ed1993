"""Host side of the multi-GPU path (one process per GPU, no data-path collective):
sharding of independent systems and the timing reductions, run as world_size-2 gloo
process groups on the CPU, plus the reference arm of bench.py under torchrun."""

import json
import os
import socket
import subprocess
import sys

import numpy as np

from galaxy_b200 import ranks, workloads

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _torchrun(nproc: int, *argv: str, timeout: float = 240.0) -> subprocess.CompletedProcess:
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="2")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={nproc}",
           "--master-addr=127.0.0.1", f"--master-port={_free_port()}", *argv]
    return subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=timeout)


def test_shard_partitions_and_balances():
    sizes = workloads.batched_sizes(256, seed=0)
    for world in (1, 2, 3, 8):
        parts = ranks.shard(sizes, world)
        assert sorted(i for p in parts for i in p) == list(range(len(sizes)))
        loads = [int(sum(sizes[i] for i in p)) for p in parts]
        # greedy largest-first: no rank exceeds the mean by more than the largest system
        assert max(loads) - sum(loads) / world <= int(sizes.max())
    assert ranks.shard([5, 5, 5], 5) == [[0], [1], [2], [], []]
    assert ranks.shard([], 2) == [[], []]


def test_shard_is_deterministic():
    sizes = workloads.batched_sizes(100, seed=3)
    assert ranks.shard(sizes, 4) == ranks.shard(list(sizes), 4)


def test_single_process_reductions_are_identity():
    assert ranks.init() == (None, 0, 1, 0) or int(os.environ.get("WORLD_SIZE", "1")) > 1
    assert ranks.max_over_ranks(None, 2.5) == 2.5
    assert ranks.sum_over_ranks(None, 7) == 7.0


def test_two_gloo_ranks_partition_and_reduce():
    res = _torchrun(2, os.path.join("tests", "gloo_ranks_worker.py"))
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, res.stdout
    d = json.loads(lines[0])
    assert d["world"] == 2 and d["covered"]
    assert d["t_max"] == 2.0  # max of 1 + rank over ranks 0 and 1
    assert d["n_all"] == d["n_mix"] == sum(d["loads"])
    assert abs(d["loads"][0] - d["loads"][1]) <= 262_144


def test_bench_reference_arm_two_ranks():
    """Under torchrun rank 0 alone times the CPU reference (whole KDK steps of the
    oracle, inputs from the oracle's copy of the generator) and prints one line; the
    other rank exits 0 without work. The product library is never loaded."""
    res = _torchrun(2, "bench.py", "--impl", "reference", "--gpus", "2", "--steps", "2", "--warmup", "1",
                    "--config", "plummer")
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, res.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["e2e"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] == "port" and np.isfinite(d["ms_per_step"])
    assert d["steps"] == 2 and d["warmup"] == 1 and d["config"]["particles"] == 16_384
    assert d["native_libraries"] == ["oracle/liblbvh_oracle.so"]
