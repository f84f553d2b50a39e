"""The decomposed grid's sleeve exchange on CPU: 2 x 2 and 3 x 1 gloo ranks.

Each rank holds one block of a seeded global wavefield (global__setup2's
block extents) with a zero sleeve and trades the planes of global__comm_stress
and global__comm_vel (src/swpc_3d/m_global.f90:393-609) with its neighbours
through openswpc_b200.decomp.HaloTransport (torch.distributed point-to-point,
gloo here, NCCL between GPUs).  After both exchanges every sleeve plane the
reference fills holds the neighbour's values and nothing else changed."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

from openswpc_b200.decomp import block_range, neighbours
from tests.test_replicas_gloo import free_port

WORKER = Path(__file__).resolve().parent / "decomp_worker.py"


@pytest.mark.parametrize("nproc_x,nproc_y", [(2, 2), (3, 1), (1, 3)])
def test_sleeve_exchange_over_gloo(nproc_x, nproc_y):
    port = free_port()
    world = nproc_x * nproc_y
    procs = []
    for rank in range(world):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                   RANK=str(rank), LOCAL_RANK=str(rank))
        procs.append(subprocess.Popen([sys.executable, str(WORKER), str(nproc_x), str(nproc_y)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=180)
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    assert all(d["ok"] for d in outs), outs
    # interior blocks receive on every side they have a neighbour
    assert any(d["filled"] > 0 for d in outs)


def test_block_extents_follow_global_setup2():
    """m_global.f90:236-249, 276-288: the first nproc - n mod nproc blocks
    hold n div nproc cells, the others one more; blocks tile 1..n."""
    for n in range(4, 80):
        for nproc in range(1, 7):
            r = [block_range(n, nproc, q) for q in range(nproc)]
            sizes = [e - b + 1 for b, e in r]
            m = n % nproc
            assert r[0][0] == 1 and r[-1][1] == n
            assert all(r[q][1] + 1 == r[q + 1][0] for q in range(nproc - 1))
            assert sizes == [n // nproc] * (nproc - m) + [n // nproc + 1] * m


def test_neighbour_table():
    # rank = px + py * nproc_x (m_global.f90:239-240); faces have no neighbour
    assert neighbours(0, 0, 2, 2) == [None, 1, None, 2]
    assert neighbours(1, 1, 2, 2) == [2, None, 1, None]
    assert neighbours(1, 0, 3, 1) == [0, 2, None, None]
