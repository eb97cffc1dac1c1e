"""One rank of the two-rank CPU test of bench.py's multi-GPU host logic
(tests/test_multirank_host.py) with the gloo backend: the units each rank
takes, the reductions of the timings and counts, and the rank-0-only
reference arm; or (argv[2] == "lost") a rank that leaves.  Writes
rank<r>.json into argv[1]."""
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


def lost_rank() -> None:
    """argv[2] == "lost": rank 1 leaves after joining the group (between
    steps, nothing in flight); rank 0's next reduction must end with an error
    within the group's short timeout instead of waiting for good."""
    import time

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=10))
    rank = dist.get_rank()
    if rank == 1:
        os._exit(3)
    t0 = time.monotonic()
    try:
        bench.all_max(dist, 1.0)
        res = {"rank": 0, "error": None}
    except Exception as e:  # the collective's failure, reported to the caller
        res = {"rank": 0, "error": type(e).__name__}
    res["seconds"] = time.monotonic() - t0
    with open(os.path.join(sys.argv[1], "rank0.json"), "w") as f:
        json.dump(res, f)
    os._exit(0)


def main() -> None:
    if len(sys.argv) > 2 and sys.argv[2] == "lost":
        lost_rank()
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
