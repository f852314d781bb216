"""One rank of bench.py's multi-rank layout on CPU (gloo), started by bench.launch_ranks.

Each rank reads its rank and world size from the launcher's environment, takes its slice of
a BFS-like source order, and the ranks agree on the slowest rank's time; rank 0 prints one
JSON line with the world size, as bench.py's rank 0 does. Used by tests/test_multirank_cpu.py.
"""
import datetime
import json
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import bench  # noqa: E402


def main():
    import torch.distributed as dist

    rank, world, local = bench.rank_env()
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        order = np.random.default_rng(0).permutation(int(sys.argv[1]))
        share = bench.shard_sources(order, world, rank)
        sizes = [None] * world
        dist.all_gather_object(sizes, int(share.size))
        slowest = bench.max_over_ranks(1.0 + rank, dist, "cpu")
        dist.barrier()
        if rank == 0:
            print(json.dumps({"n_gpus": world, "ranks_sources": sizes, "slowest": slowest,
                              "local_rank": local, "parallelism": f"replicas{world}"}), flush=True)
    finally:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
