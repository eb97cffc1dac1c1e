"""bench.py's multi-GPU host logic with two gloo ranks on the CPU: every
batch chain and CFTP seed goes to exactly one rank, replica seeds differ,
device times reduce to their maximum over the ranks and counts to their sum,
and the reference arm runs on rank 0 only.  The GPU work itself is
single-GPU by design (one walk is one lattice; ranks are independent
replicas)."""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys

from conftest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_shard_and_reduce(tmp_path):
    worker = os.path.join(ROOT, "tests", "multirank_worker.py")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), worker, str(tmp_path)]
    subprocess.run(cmd, check=True, timeout=300, cwd=ROOT, capture_output=True)
    r = [json.load(open(tmp_path / f"rank{k}.json")) for k in range(2)]
    assert [x["world"] for x in r] == [2, 2]
    for key, count in (("batch_seeds", 4096), ("cftp_seeds", 32)):
        a, b = set(r[0][key]), set(r[1][key])
        assert not a & b and a | b == set(range(count)), key
        assert abs(len(a) - len(b)) <= 1
    assert r[0]["replica_seed"] != r[1]["replica_seed"]
    assert r[0]["max"] == r[1]["max"] == 2.5
    assert r[0]["sum"] == r[1]["sum"] == [3.0, 30.0]
    assert r[1].get("reference_arm_returned") and "reference_arm_returned" not in r[0]


def test_a_lost_rank_ends_the_next_reduction_with_an_error(tmp_path):
    """Rank 1 leaves between steps; rank 0's reduction of the timings fails
    with an exception (no hang), well inside the group's 10 s timeout bound."""
    worker = os.path.join(ROOT, "tests", "multirank_worker.py")
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, worker, str(tmp_path), "lost"], cwd=ROOT, env=env,
                                      stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL))
    codes = [p.wait(timeout=120) for p in procs]
    assert codes == [0, 3]
    r = json.load(open(tmp_path / "rank0.json"))
    assert r["error"] is not None and r["seconds"] < 60
