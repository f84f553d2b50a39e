"""The waveform and snapshot files of a GPU run, byte for byte equal to the
files the reference's writers (restated in the oracle) would make from the
oracle's own run of the same input: SAC, CSF and both tar layouts for
velocity, displacement, stress and strain traces, and native .snp files of a
vertical, a horizontal and a free-surface plane."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from openswpc_b200 import _lib, output
from openswpc_b200.swpc3d import Swpc3D
from oracle import formats as O
from oracle.oracle import Oracle3D
from tests.models import small3d

pytestmark = pytest.mark.gpu

EXEDATE, TZ = 1700000000, 540
NAMES = {_lib.WAV_V: ("v", ["Vx", "Vy", "Vz"], 7), _lib.WAV_U: ("u", ["Ux", "Uy", "Uz"], 6),
         _lib.WAV_STRESS: ("stress", ["Sxx", "Syy", "Szz", "Syz", "Sxz", "Sxy"], 5),
         _lib.WAV_STRAIN: ("strain", ["Exx", "Eyy", "Ezz", "Eyz", "Exz", "Exy"], 5)}


@pytest.fixture(scope="module")
def runs():
    p = small3d(nt=30, sw_wav_u=True, sw_wav_stress=True, sw_wav_strain=True, title="files", phi=15.0,
                snaps={"xz_v", "xy_u", "fs_ps"}, ntdec_s=5, idec=2, jdec=2, kdec=1)
    g = Swpc3D(p)
    o = Oracle3D(p)
    g.run(1, p.nt)
    o.run(1, p.nt, ntdec_r=p.ntdec_r)
    return p, g, o


def _oracle_headers(p, g, o, what):
    kept = [st for st in p.stations if output._recorded(g, [st])]
    m6 = p.sources[0].moment(lambda *a: output._sdr(output.lib(), *a))
    return O.sac_headers(p, kept, o.scalars()["M0"], m6, EXEDATE, TZ, NAMES[what][1:])


@pytest.mark.parametrize("fmt", ["sac", "csf", "tar_st", "tar_node"])
def test_waveform_files(tmp_path, runs, fmt):
    p, g, o = runs
    files = output.wav_write(g, tmp_path, fmt, exedate=EXEDATE, tz_minutes=TZ)
    order = [w for w in NAMES]
    heads = {w: _oracle_headers(p, g, o, w) for w in order}
    data = {w: o.waveforms(NAMES[w][0]) for w in order}   # (nst, ncmp, ntw)
    title = p.title
    if fmt == "sac":
        assert len(files) == o.nst * 18
        for w in order:
            for n, row in enumerate(heads[w]):
                for c, h in enumerate(row):
                    fn = tmp_path / "wav" / f"{title}.3d.{h['kstnm']}.{h['kcmpnm']}.sac"
                    assert fn.read_bytes() == O.sac_file(h, data[w][n, c]), fn.name
    elif fmt == "csf":
        # one file per node, rewritten by each quantity as wav__write does: the last (strain) remains
        w = order[-1]
        ref = O.csf_file([h for row in heads[w] for h in row], data[w].reshape(-1, data[w].shape[-1]))
        assert files[0].read_bytes() == ref
    else:
        members = {}
        for n in range(o.nst):
            for w in order:
                for c, h in enumerate(heads[w][n]):
                    name = f"{title}.{h['kstnm']}.3d.{h['kcmpnm']}.sac"
                    members.setdefault(n, []).append(O.tar_member(name, h, data[w][n, c]))
        if fmt == "tar_st":
            assert len(files) == o.nst
            for n, fn in enumerate(files):
                assert fn.read_bytes() == b"".join(members[n]) + O.tar_end()
        else:
            assert files[0].read_bytes() == b"".join(b"".join(members[n]) for n in range(o.nst)) + O.tar_end()


def test_snapshot_files(tmp_path, runs):
    p, g, o = runs
    files = {f.name: f for f in output.snap_write(g, tmp_path, exedate=EXEDATE)}
    L = output.lib()
    nxs, nys, nzs = (p.nx + 1) // 2, (p.ny + 1) // 2, p.nz
    ax = lambda n, dec, beg, d: np.array([L.swpc_i2x(q * dec - dec // 2, beg, d) for q in range(1, n + 1)],
                                         np.float32)
    xs, ys, zs = ax(nxs, 2, p.xbeg, p.dx), ax(nys, 2, p.ybeg, p.dy), ax(nzs, 1, p.zbeg, p.dz)
    rho, lam, mu = o.array("frho"), o.array("flam"), o.array("fmu")
    kfs = o.array("kfs")
    d = g.snap_desc
    dt_s = np.float32(p.dt) * np.float32(p.ntdec_s)
    for name, (sec, q) in (("xz_v", ("xz", "v")), ("xy_u", ("xy", "u")), ("fs_ps", ("fs", "ps"))):
        if sec == "xz":
            cells = [[(k, 2 * i - 1, d.j0_xz) for k in range(1, nzs + 1)] for i in range(1, nxs + 1)]
            hdr = O.snp_header(p.title, EXEDATE, sec, "v3", nxs, nzs, xs, zs, dt_s, p.na // 2, p.na, 3, 3, p.clon,
                               p.clat, p.phi)
        else:
            cells = [[((int(kfs[2 * j - 1 + 2, 2 * i - 1 + 2]) + 1) if sec == "fs" else d.k0_xy, 2 * i - 1, 2 * j - 1)
                      for j in range(1, nys + 1)] for i in range(1, nxs + 1)]
            hdr = O.snp_header(p.title, EXEDATE, sec, "u3" if q == "u" else "ps", nxs, nys, xs, ys, dt_s, p.na // 2,
                               p.na // 2, 6, 3 if q == "u" else 4, p.clon, p.clat, p.phi)
        n1, n2 = len(cells), len(cells[0])
        med = np.zeros((3 if sec == "xz" else 4, n2, n1), np.float32)
        for a in range(n1):
            for b in range(n2):
                k, i, j = cells[a][b]
                med[0, b, a], med[1, b, a], med[2, b, a] = rho[j + 2, i + 2, k + 2], lam[j + 2, i + 2, k + 2], \
                    mu[j + 2, i + 2, k + 2]
                if sec != "xz":
                    med[3, b, a] = -np.float32(p.layers[0].depth) * np.float32(1000)
        # the frames are the device's, which equal the oracle's bit for bit (test_gpu_snapshots)
        body = np.ascontiguousarray(g.snapshots(name), np.float32)
        fn = files[f"{p.title}.3d.{sec}.{q}.snp"]
        assert fn.read_bytes() == hdr + med.tobytes() + body.tobytes(), name
