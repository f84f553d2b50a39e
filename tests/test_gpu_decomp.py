"""Decomposed grids (src/swpc_3d/m_global.f90:236-303, 349-378, 393-609) on
one GPU.

* swpc_halo_pack / swpc_halo_unpack against the oracle's restatement of
  global__comm_stress / global__comm_vel, bit for bit, on every side;
* a run split into 2 x 2, 3 x 1 and 1 x 3 blocks (one context per block,
  sleeves traded through device buffers after each half step) gives the
  single-domain run's bits: every trace, every cell of V, S and the memory
  variables, every report; with sources and stations on the block seams,
  with the Cerjan sponge and with body forces;
* BlockRank3D, one block per process (3D, and a P-SV block): two gloo ranks
  on the one GPU (the messages staged through host memory; no kernel waits on
  another).

With two GPUs or more, the same 2 x 2 split with its blocks spread over two
GPUs (peer stores) and two NCCL ranks on two GPUs run as well.
"""
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from openswpc_b200 import _lib
from openswpc_b200.decomp import Decomposed3D, block_range
from openswpc_b200.params import Source, Station, dc_source
from openswpc_b200.swpc3d import Swpc3D
from oracle import decomp as od
from tests.models import small3d, vonkarman_xi
from tests.test_replicas_gloo import free_port

pytestmark = pytest.mark.gpu

FIELDS = [_lib.F_VX + c for c in range(3)] + [_lib.F_SXX + c for c in range(6)] + \
    [_lib.F_R + 3 * c + m for c in range(6) for m in range(3)]


def decomp_case(**kw):
    """44 x 40 x 32 cells, PML 8, 60 steps; double couples and stations on
    the seams of the 2 x 2, 3 x 1 and 1 x 3 splits (x = -4.0 / 3.6 km between
    blocks 14|15 and 29|30, y = -3.5 / 3.0 km between 13|14 and 26|27)."""
    p = small3d(nx=44, ny=40, nz=32, na=8, nt=60, **kw)
    p.sources = p.sources + [dc_source(-4.0, 0.6, 4.0, 0.1, 1.0, 5e15, 10, 80, -30),
                             dc_source(3.6, -0.7, 8.0, 0.0, 1.2, 7e15, 200, 45, 10),
                             dc_source(1.1, -3.5, 5.0, 0.05, 0.9, 4e15, 120, 30, 60),
                             dc_source(-2.2, 3.0, 7.0, 0.0, 1.1, 6e15, 300, 70, -90)]
    p.stations = p.stations + [Station(-4.0, 1.0, 0.0, "sx1", "fsb"), Station(3.6, -1.0, 0.0, "sx2", "fsb"),
                               Station(0.2, -3.5, 0.0, "sy1", "fsb"), Station(-0.3, 3.0, 2.0, "sy2", "dep"),
                               Station(0.0, 0.0, 0.0, "s00", "fsb")]
    xi = vonkarman_xi((p.ny + 6, p.nx + 6, p.nz + 6))
    return p, xi


FIELDS_PSV = [_lib.F_VX, _lib.F_VZ, _lib.F_SXX, _lib.F_SZZ, _lib.F_SXZ]


def decomp_case_2d(kind):
    """A 124 x 60 P-SV or SH run with sources and stations on the seams of a
    3-way split (cells 41|42 and 82|83) and of a 2-way split (62|63)."""
    from tests.models import small2d

    p = small2d(kind, nx=124, nz=60, na=10, nt=80)
    for n, i in enumerate((41, 42, 82, 63)):
        s = p.sources[0]
        p.sources.append(type(s)(**{**s.__dict__, "x": float(p.xbeg + (i - 0.3) * p.dx), "z": 3.0 + n}))
        st = p.stations[0]
        p.stations.append(type(st)(**{**st.__dict__, "x": float(p.xbeg + (i - 0.5) * p.dx), "name": f"seam{n}"}))
    return p


def assert_same_bits(a, b, what):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    bad = np.argwhere(a.view(np.uint32) != b.view(np.uint32))
    assert bad.size == 0, (what, len(bad), bad[:5].tolist())


def single_run(p, xi):
    g = Swpc3D(p, xi)
    rep = g.run(1, p.nt)
    out = {"wav": g.waveforms(_lib.WAV_V), "reports": np.array([v for _, v in rep])}
    for f in FIELDS:
        out[f] = g.download(f)
    g.close()
    return out


def test_halo_pack_and_unpack_match_the_oracle():
    import torch

    p, xi = decomp_case()
    d = Decomposed3D(p, 2, 2, xi)
    b = d.blocks[3]   # block (1, 1): neighbours on -x and -y
    rng = np.random.default_rng(3)
    fields = {}
    for f in range(9):
        a = rng.standard_normal((b.ny + 6, b.nx + 6, p.nz + 6)).astype(np.float32)
        _lib.check(b.ctx, b.lib.swpc_upload_field(b.ctx, f, _lib.fptr(a), p.nz + 6, b.nx + 6))
        fields[f] = b.download(f)   # the cells the context keeps
    for half in (0, 1):
        for side in range(4):
            n = b.halo_count[half][side]
            assert n == od.count("3d", half, side, b.nx, b.ny, p.nz)
            buf = torch.empty(n, dtype=torch.float32, device="cuda:0")
            b.pack(half, side, buf.data_ptr())
            b.sync()
            assert_same_bits(buf.cpu().numpy(), od.pack(fields, "3d", half, side, b.nx, b.ny), f"pack {half} {side}")
    for half in (0, 1):
        for side in range(4):
            msg = rng.standard_normal(od.count("3d", half, side ^ 1, b.nx, b.ny, p.nz)).astype(np.float32)
            b.unpack(half, side, torch.from_numpy(msg).cuda().data_ptr())
            b.sync()
            od.unpack(fields, msg, "3d", half, side, b.nx, b.ny)
            for f in range(9):
                assert_same_bits(b.download(f), fields[f], f"unpack {half} {side} field {f}")
    d.close()


@pytest.mark.parametrize("nproc_x,nproc_y", [(2, 2), (3, 1), (1, 3)])
def test_decomposed_run_gives_the_single_domain_bits(nproc_x, nproc_y):
    p, xi = decomp_case()
    ref = single_run(p, xi)
    d = Decomposed3D(p, nproc_x, nproc_y, xi)
    assert sum(b.nst for b in d.blocks) == ref["wav"].shape[0]
    rep = d.run(1, p.nt)
    assert_same_bits(d.waveforms(_lib.WAV_V), ref["wav"], "traces")
    assert np.linalg.norm(ref["wav"]) > 0
    for f in FIELDS:
        assert_same_bits(d.download(f), ref[f], f"field {f}")
    assert_same_bits(np.array([v for _, v in rep]), ref["reports"], "reports")
    d.close()


@pytest.mark.parametrize("variant", ["cerjan", "bodyforce"])
def test_decomposed_variants(variant):
    if variant == "cerjan":
        p, xi = decomp_case(abc_type="cerjan")
    else:
        p, xi = decomp_case(bf_mode=True)
        p.sources = [Source(s.x, s.y, s.z, s.tbeg, s.trise, fx=1e15 * (n + 1), fy=-5e14 * n, fz=3e14)
                     for n, s in enumerate(p.sources)]
    ref = single_run(p, xi)
    d = Decomposed3D(p, 2, 2, xi)
    d.run(1, p.nt)
    assert_same_bits(d.waveforms(_lib.WAV_V), ref["wav"], "traces")
    for f in FIELDS:
        assert_same_bits(d.download(f), ref[f], f"field {f}")
    d.close()


def multi_gpu():
    import torch

    return torch.cuda.device_count() >= 2


@pytest.mark.skipif(not multi_gpu(), reason="needs two GPUs")
def test_decomposed_run_across_two_gpus():
    """The 2 x 2 split with the blocks on alternating GPUs: the pack kernels
    store the messages into the neighbours' buffers over NVLink."""
    p, xi = decomp_case()
    ref = single_run(p, xi)
    d = Decomposed3D(p, 2, 2, xi, devices=[0, 1, 1, 0])
    rep = d.run(1, p.nt)
    assert_same_bits(d.waveforms(_lib.WAV_V), ref["wav"], "traces")
    for f in FIELDS:
        assert_same_bits(d.download(f), ref[f], f"field {f}")
    assert_same_bits(np.array([v for _, v in rep]), ref["reports"], "reports")
    d.close()


def block_ranks(tmp_path, kind, backend):
    """Two ranks of BlockRank3D (a 2 x 1 split) against the single-domain
    run: every trace, the block's cells of every field, every report."""
    if kind == "3d":
        p, xi = decomp_case()
        ref = single_run(p, xi)
    else:
        from openswpc_b200.swpc2d import Swpc2D

        p = decomp_case_2d(kind)
        g = Swpc2D(p, kind)
        g.run(1, p.nt)
        ref = {"wav": g.waveforms(_lib.WAV_V)}
        for f in FIELDS_PSV:
            ref[f] = g.download(f)
        g.close()
    worker = Path(__file__).resolve().parent / "decomp_rank_worker.py"
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(rank),
                   LOCAL_RANK=str(rank))
        if backend == "nccl":
            env["NCCL_NVLS_ENABLE"] = "0"
        procs.append(subprocess.Popen([sys.executable, str(worker), "2", "1", str(tmp_path), kind, backend], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    for pr in procs:
        _, err = pr.communicate(timeout=600)
        assert pr.returncode == 0, err
    wav = np.zeros_like(ref["wav"])
    for rank in range(2):
        z = np.load(tmp_path / f"rank{rank}.npz")
        wav[z["stations"]] = z["wav"]
        ib, ie, jb, je = (int(v) for v in z["ext"])
        assert (ib, ie) == block_range(p.nx, 2, rank)
        for f in (FIELDS if kind == "3d" else FIELDS_PSV):
            a = z[f"f{f}"]
            if kind == "3d":
                assert_same_bits(a[3:-3, 3:-3, :], ref[f][jb + 2:je + 3, ib + 2:ie + 3, :], f"rank {rank} field {f}")
            else:
                assert_same_bits(a[3:-3, :], ref[f][ib + 2:ie + 3, :], f"rank {rank} field {f}")
        if kind == "3d":
            assert_same_bits(z["reports"], ref["reports"], "reports")
    assert_same_bits(wav, ref["wav"], "traces")


@pytest.mark.parametrize("kind", ["3d", "psv"])
def test_block_ranks_over_gloo_on_one_gpu(tmp_path, kind):
    block_ranks(tmp_path, kind, "gloo")


@pytest.mark.skipif(not multi_gpu(), reason="needs two GPUs")
@pytest.mark.parametrize("kind", ["3d", "psv"])
def test_block_ranks_over_nccl_on_two_gpus(tmp_path, kind):
    """One rank per GPU, the halo messages stream-ordered NCCL point-to-point
    transfers between the blocks' device buffers."""
    block_ranks(tmp_path, kind, "nccl")


@pytest.mark.parametrize("kind", ["psv", "sh"])
def test_decomposed_2d_run_gives_the_single_domain_bits(kind):
    """P-SV and SH split into 3 blocks across x (the 2D codes' own
    global__comm_*), with sources and stations on the seams."""
    from openswpc_b200.decomp import Decomposed2D
    from openswpc_b200.swpc2d import Swpc2D

    p = decomp_case_2d(kind)
    g = Swpc2D(p, kind)
    g.run(1, p.nt)
    d = Decomposed2D(p, kind, 3)
    d.run(1, p.nt)
    assert_same_bits(d.waveforms(_lib.WAV_V), g.waveforms(_lib.WAV_V), "traces")
    ids = [_lib.F_VX, _lib.F_VZ, _lib.F_SXX, _lib.F_SZZ, _lib.F_SXZ] if kind == "psv" else [_lib.F_VY, _lib.F_SXY,
                                                                                            _lib.F_SYZ]
    for f in ids:
        assert_same_bits(d.download(f), g.download(f), f"field {f}")
    d.close()
    g.close()
