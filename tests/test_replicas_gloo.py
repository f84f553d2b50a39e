"""The multi-GPU path on CPU: two ranks over gloo.

bench.py runs N independent replicas (or shards ensemble members) with no
data-path collective; the ranks meet only for the barrier and the maximum of
their device times.  Two gloo ranks exercise that logic without a GPU."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

WORKER = Path(__file__).resolve().parent / "replica_worker.py"


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_shard_and_time():
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(rank),
                   LOCAL_RANK=str(rank))
        procs.append(subprocess.Popen([sys.executable, str(WORKER)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=180)
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    outs.sort(key=lambda d: d["rank"])
    # members: disjoint, complete, round robin
    assert outs[0]["members"] == [0, 2, 4, 6, 8, 10] and outs[1]["members"] == [1, 3, 5, 7, 9]
    # every rank sees the slowest rank's time, and the job throughput counts both ranks' work
    assert all(d["ms_max"] == 15.0 for d in outs)
    assert all(abs(d["value"] - 1.0e9 * 3 * 2 / 0.015 / 1e9) < 1e-9 for d in outs)


def test_single_rank_without_torchrun():
    from openswpc_b200 import replicas
    env_keys = ("WORLD_SIZE", "RANK", "LOCAL_RANK")
    saved = {k: os.environ.pop(k, None) for k in env_keys}
    try:
        r = replicas.init("gloo")
        assert (r.world, r.rank, r.dist) == (1, 0, None)
        assert r.max(3.5) == 3.5
        assert replicas.shard(list(range(5)), 1, 0) == [0, 1, 2, 3, 4]
    finally:
        for k, v in saved.items():
            if v is not None:
                os.environ[k] = v
