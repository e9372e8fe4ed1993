"""Worker of tests/test_ranks.py, launched under torchrun on CPU (gloo): every rank
takes its shard of a batched mix, and rank 0 checks that the shards partition the
mix and that the timing reductions see every rank."""

import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from galaxy_b200 import ranks, workloads  # noqa: E402


def main():
    dist, rank, world, local = ranks.init(timeout_s=60)
    assert dist is not None and world == int(os.environ["WORLD_SIZE"])
    sizes = workloads.batched_sizes(64 * world, seed=0)
    mine = ranks.shard(sizes, world)[rank]
    parts = [None] * world
    dist.all_gather_object(parts, mine)
    load = sum(int(sizes[i]) for i in mine)
    t_max = ranks.max_over_ranks(dist, 1.0 + rank, local)
    n_all = ranks.sum_over_ranks(dist, load, local)
    ranks.barrier(dist, local)
    if rank == 0:
        flat = sorted(i for p in parts for i in p)
        print(json.dumps({"world": world, "covered": flat == list(range(len(sizes))),
                          "loads": [sum(int(sizes[i]) for i in p) for p in parts], "t_max": t_max,
                          "n_all": n_all, "n_mix": int(sum(int(x) for x in sizes))}), flush=True)
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
