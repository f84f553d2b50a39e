"""One rank of the gloo test of the sleeve exchange (tests/test_decomp_gloo.py):
joins the group from the torchrun-style environment, takes block
(rank mod nproc_x, rank div nproc_x) of a seeded global wavefield, trades its
sleeve planes with its neighbours through HaloTransport (the messages packed
and unpacked by the oracle's restatement of global__comm_*), and prints, as
one JSON line, whether every sleeve plane now holds the global field's
values and every other sleeve cell is still zero."""
import json
import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

import numpy as np  # noqa: E402
import torch  # noqa: E402

from openswpc_b200 import replicas  # noqa: E402
from openswpc_b200.decomp import OPPOSITE, HaloTransport, block_range, neighbours  # noqa: E402
from oracle import decomp as od  # noqa: E402


def main():
    nproc_x, nproc_y = int(sys.argv[1]), int(sys.argv[2])
    NX, NY, NZ = 13, 11, 5
    ranks = replicas.init("gloo", timeout_s=60)
    px, py = ranks.rank % nproc_x, ranks.rank // nproc_x
    ib, ie = block_range(NX, nproc_x, px)
    jb, je = block_range(NY, nproc_y, py)
    nx, ny = ie - ib + 1, je - jb + 1
    rng = np.random.default_rng(5)
    glob = {f: rng.standard_normal((NY + 6, NX + 6, NZ + 6)).astype(np.float32) for f in range(9)}
    # the block's own cells; its sleeve starts at zero
    own = {}
    for f, a in glob.items():
        b = np.zeros((ny + 6, nx + 6, NZ + 6), np.float32)
        b[3:3 + ny, 3:3 + nx, 3:-3] = a[jb + 2:je + 3, ib + 2:ie + 3, 3:-3]
        own[f] = b
    nbr = neighbours(px, py, nproc_x, nproc_y)
    tr = HaloTransport(nbr)
    ok = True
    expect = {f: b.copy() for f, b in own.items()}
    for half in (0, 1):
        send, recv = {}, {}
        for s in range(4):
            if nbr[s] is None:
                continue
            send[s] = torch.from_numpy(od.pack(own, "3d", half, s, nx, ny))
            ok &= send[s].numel() == od.count("3d", half, s, nx, ny, NZ)
            recv[s] = torch.empty(od.count("3d", half, OPPOSITE[s], nx, ny, NZ), dtype=torch.float32)
        tr.exchange(send, recv)
        for s, t in recv.items():
            od.unpack(own, t.numpy(), "3d", half, s, nx, ny)
            # the planes this side fills, from the global field
            ax, up = s // 2, s % 2 == 1
            for f, to_plus, to_minus in od.halo_fields("3d", half, ax):
                for o in (to_minus if up else to_plus):
                    if ax == 0:
                        q = nx + o if up else o
                        expect[f][3:3 + ny, q + 2, 3:-3] = glob[f][jb + 2:je + 3, ib - 1 + q + 2, 3:-3]
                    else:
                        q = ny + o if up else o
                        expect[f][q + 2, 3:3 + nx, 3:-3] = glob[f][jb - 1 + q + 2, ib + 2:ie + 3, 3:-3]
    ok &= all(np.array_equal(own[f], expect[f]) for f in range(9))
    filled = sum(int(np.count_nonzero(own[f])) - nx * ny * NZ for f in range(9))
    ranks.barrier()
    print(json.dumps({"rank": ranks.rank, "ok": bool(ok), "filled": filled, "neighbours": nbr}), flush=True)
    ranks.close()


if __name__ == "__main__":
    main()
