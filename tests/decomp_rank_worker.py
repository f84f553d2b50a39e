"""One rank of the BlockRank3D tests (tests/test_gpu_decomp.py): joins a
gloo group (every rank on cuda:0, the halo messages staged through host
memory) or an NCCL group (rank r on cuda:r, the messages device to device)
from the torchrun-style environment, runs its block of the decomposed test
case (3D, or P-SV with kind psv), and saves its traces, station indices,
block extents, fields and report values to <outdir>/rank<r>.npz.

usage: decomp_rank_worker.py nproc_x nproc_y outdir [kind [backend]]"""
import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

import numpy as np  # noqa: E402

from openswpc_b200 import _lib, replicas  # noqa: E402
from openswpc_b200.decomp import BlockRank3D  # noqa: E402
from tests.test_gpu_decomp import FIELDS, FIELDS_PSV, decomp_case, decomp_case_2d  # noqa: E402


def main():
    nproc_x, nproc_y, outdir = int(sys.argv[1]), int(sys.argv[2]), Path(sys.argv[3])
    kind = sys.argv[4] if len(sys.argv) > 4 else "3d"
    backend = sys.argv[5] if len(sys.argv) > 5 else "gloo"
    ranks = replicas.init(backend, timeout_s=120)
    device = ranks.local if backend == "nccl" else 0
    if kind == "3d":
        p, xi = decomp_case()
        r = BlockRank3D(p, nproc_x, nproc_y, xi, device=device)
        fields = FIELDS
    else:
        p = decomp_case_2d(kind)
        r = BlockRank3D(p, nproc_x, nproc_y, device=device, kind=kind)
        fields = FIELDS_PSV
    rep = r.run(1, p.nt)
    b = r.block
    ext = [b.ib, b.ie, getattr(b, "jb", 1), getattr(b, "je", 1)]
    out = {"wav": r.waveforms(_lib.WAV_V), "stations": b.stations, "ext": np.array(ext),
           "reports": np.array([v for _, v in rep])}
    for f in fields:
        out[f"f{f}"] = b.download(f)
    np.savez(outdir / f"rank{ranks.rank}.npz", **out)
    ranks.barrier()
    r.close()
    ranks.close()


if __name__ == "__main__":
    main()
