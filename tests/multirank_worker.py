"""One rank of the two-rank CPU test of bench.py's multi-GPU host logic
(tests/test_multirank_host.py), launched by torch.distributed.run with the
gloo backend: the units each rank takes, the reductions of the timings and
counts, and the rank-0-only reference arm.  Writes rank<r>.json into argv[1]."""
from __future__ import annotations

import datetime
import json
import os
import sys

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, ROOT)

import torch.distributed as dist  # noqa: E402

import bench  # noqa: E402


class _RefArgs:
    impl, steps, warmup, gpus = "reference", 1, 3, 2


def main() -> None:
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    rank, world = dist.get_rank(), dist.get_world_size()
    res = {
        "rank": rank,
        "world": world,
        "batch_seeds": list(bench.shard(4096, rank, world)),
        "cftp_seeds": list(bench.shard(32, rank, world)),
        "replica_seed": bench.replica_seed(rank),
        "max": bench.all_max(dist, 1.5 + rank),
        "sum": bench.all_sum(dist, [rank + 1.0, 10.0 * (rank + 1)]),
    }
    if rank != 0:
        bench.run_reference(_RefArgs())  # a non-zero rank returns at once, without work
        res["reference_arm_returned"] = True
    dist.barrier()
    with open(os.path.join(sys.argv[1], f"rank{rank}.json"), "w") as f:
        json.dump(res, f)
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
