"""One rank of the two-rank gloo test (tests/test_replicas_gloo.py): joins the
group from the torchrun-style environment, shards 11 members, takes the
maximum of a per-rank time and prints what it saw as one JSON line."""
import json
import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

from openswpc_b200 import replicas  # noqa: E402


def main():
    ranks = replicas.init("gloo", timeout_s=60)
    members = replicas.shard(list(range(11)), ranks.world, ranks.rank)
    ms = 10.0 + 5.0 * ranks.rank          # rank 1 is the slower one
    ranks.barrier()
    ms_max = ranks.max(ms)
    ranks.barrier()
    value = replicas.throughput(1.0e9, 3, ranks.world, ms_max)
    print(json.dumps({"rank": ranks.rank, "world": ranks.world, "members": members, "ms_max": ms_max,
                      "value": value}), flush=True)
    ranks.close()


if __name__ == "__main__":
    main()
