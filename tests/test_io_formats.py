"""The library's file writers (include/swpc_io.h) against the oracle's
restatement of the reference's writers, byte for byte: SAC header and file,
CSF, tar members with their ustar headers and padding, the native snapshot
header, and the Gauss-Kruger projection of the headers' coordinates.  CPU
only (the traces are synthetic)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from openswpc_b200 import _lib, output
from oracle import formats as O


def _pair(seed=0, npts=37):
    """One header filled both ways: the library struct and the oracle dict."""
    rng = np.random.default_rng(seed)
    L = output.lib()
    h = output.SacHdr()
    L.swpc_sac_init(C.byref(h))
    d = O.sac_init()
    vals = {"delta": 0.0123456789, "b": -1.5, "o": 0.25, "stla": 35.1, "stlo": 139.2, "stdp": 1234.5,
            "evla": 34.9, "evlo": 139.9, "evdp": 10.0, "mag": 4.6, "dist": 12.3, "az": 45.6, "baz": -134.4,
            "cmpaz": 90.0, "cmpinc": 90.0}
    for k, v in vals.items():
        setattr(h, k, v)
        d[k] = v
    for q in range(10):
        h.user[q] = d[f"user{q}"] = float(rng.normal())
    for k, v in dict(nzyear=2024, nzjday=366, nzhour=23, nzmin=59, nzsec=58, nzmsec=0, npts=npts, idep=7,
                     tim=1700000000).items():
        setattr(h, k, v)
        d[k] = v
    for k, v in dict(kstnm="N.ABCD12", kevnm="a long run title", kcmpnm="Vx").items():
        h.set_text(k, v)
        d[k] = v
    return h, d


def test_sac_header_bytes():
    L = output.lib()
    h, d = _pair()
    buf = C.create_string_buffer(632)
    L.swpc_sac_header_bytes(C.byref(h), buf)
    assert buf.raw == O.sac_whdr(d)
    assert len(buf.raw) == 632


@pytest.mark.parametrize("npts", [37, 354])      # 354 + 158 words: a member that fills whole tar blocks
def test_sac_csf_tar_files(tmp_path, npts):
    L = output.lib()
    pairs = [_pair(s, npts) for s in range(3)]
    data = np.random.default_rng(9).standard_normal((3, npts)).astype(np.float32)
    fn = tmp_path / "a.sac"
    assert L.swpc_sac_write(str(fn).encode(), C.byref(pairs[0][0]), _lib.fptr(data[0])) == 0
    assert fn.read_bytes() == O.sac_file(pairs[0][1], data[0])
    arr = (output.SacHdr * 3)(*[p[0] for p in pairs])
    fn = tmp_path / "a.csf"
    assert L.swpc_csf_write(str(fn).encode(), 3, npts, arr, _lib.fptr(data)) == 0
    assert fn.read_bytes() == O.csf_file([p[1] for p in pairs], data)
    fn = tmp_path / "a.tar"
    t = L.swpc_tar_open(str(fn).encode())
    names = [f"run.ST{q}.3d.Vx.sac" for q in range(3)]
    for q in range(3):
        assert L.swpc_tar_add_sac(t, names[q].encode(), C.byref(pairs[q][0]), _lib.fptr(data[q])) == 0
    assert L.swpc_tar_close(t) == 0
    ref = b"".join(O.tar_member(names[q], pairs[q][1], data[q]) for q in range(3)) + O.tar_end()
    assert fn.read_bytes() == ref
    if (158 + npts) * 4 % 512 == 0:
        # tar__wpad writes a whole block of NULs when the member ends on a block boundary
        assert len(ref) == 3 * (512 + (158 + npts) * 4 + 512) + 1024


def test_mismatched_csf_length_is_refused(tmp_path):
    L = output.lib()
    h, _ = _pair(npts=10)
    data = np.zeros(20, np.float32)
    assert L.swpc_csf_write(str(tmp_path / "x.csf").encode(), 1, 20, C.byref(h), _lib.fptr(data)) == _lib.SWPC_ERR_ARG


def test_snapshot_file(tmp_path):
    L = output.lib()
    h = output.SnpHdr()
    h.title = b"run".ljust(80, b" ")
    h.exedate, h.coordinate, h.snaptype = 1700000000, b"xz", b"v3"
    h.ns1, h.ns2, h.xs1, h.xs2, h.ds1, h.ds2, h.dt = 5, 4, -1.25, 0.75, 0.5, 0.5, 0.06
    h.na1, h.na2, h.nmed, h.nsnp, h.clon, h.clat, h.phi = 2, 2, 3, 3, 139.7604, 35.7182, 10.0
    rng = np.random.default_rng(2)
    med = rng.standard_normal((3, 4, 5)).astype(np.float32)
    frames = rng.standard_normal((6, 3, 4, 5)).astype(np.float32)
    fn = tmp_path / "x.snp"
    assert L.swpc_snp_write(str(fn).encode(), C.byref(h), 3, _lib.fptr(med), 6, _lib.fptr(frames)) == 0
    xs1 = np.array([-1.25, -0.75], np.float32)
    xs2 = np.array([0.75, 1.25], np.float32)
    ref = O.snp_header("run", 1700000000, "xz", "v3", 5, 4, xs1, xs2, np.float32(0.06), 2, 2, 3, 3, 139.7604,
                       35.7182, 10.0) + med.tobytes() + frames.tobytes()
    assert fn.read_bytes() == ref


def test_geomap_projection():
    rng = np.random.default_rng(4)
    for x, y, phi in zip(rng.uniform(-300, 300, 50), rng.uniform(-300, 300, 50), rng.uniform(-90, 90, 50)):
        a = output.geomap_c2g(float(x), float(y), 139.7604, 35.7182, float(np.float32(phi)))
        b = O.geomap_c2g(np.float32(x), np.float32(y), 139.7604, 35.7182, np.float32(phi))
        assert np.float32(a[0]) == np.float32(b[0]) and np.float32(a[1]) == np.float32(b[1])
    # 1 degree of latitude is about 111 km near the centre
    lon, lat = output.geomap_c2g(111.0, 0.0, 139.7604, 35.7182, 0.0)
    assert abs(lat - 35.7182 - 1.0) < 0.01 and abs(lon - 139.7604) < 1e-3


def test_localtime_matches_calendar():
    for tim in (0, 951782400, 1700000000, 1735657200, 2000000000):
        for tz in (0, 540, -300):
            assert output.localtime(tim, tz) == O.localtime(tim, tz)


def test_sac_headers_of_a_run_match_oracle():
    """set_sac_header / initialize_sac_header: the headers the library gives
    the recorded traces of a run equal the oracle's restatement, word for word
    (event and station coordinates through the projection, distance, azimuths,
    magnitude, date of the run, component names and orientations)."""
    from types import SimpleNamespace

    from openswpc_b200.swpc3d import Medium, source_grid, station_grid
    from oracle.oracle import Oracle3D
    from tests.models import small3d

    p = small3d(sw_wav_u=True, sw_wav_strain=True, phi=25.0, title="header-test run 01")
    m = Medium(p)
    sg = source_grid(p)
    ist, jst, kst = station_grid(p, m.kfs, m.kob)
    what = _lib.WAV_V | _lib.WAV_U | _lib.WAV_STRAIN
    sim = SimpleNamespace(p=p, M0=sg.M0, what=what, nst=len(ist), ist=ist, jst=jst, medium=m)
    heads = output.sac_headers(sim, exedate=1700000000, tz_minutes=540)
    o = Oracle3D(p)
    kept = [st for st in p.stations if output._recorded(sim, [st])]
    assert len(kept) == o.nst == len(ist)
    m6 = p.sources[0].moment(lambda *a: output._sdr(output.lib(), *a))
    names = {_lib.WAV_V: (["Vx", "Vy", "Vz"], 7), _lib.WAV_U: (["Ux", "Uy", "Uz"], 6),
             _lib.WAV_STRAIN: (["Exx", "Eyy", "Ezz", "Eyz", "Exz", "Exy"], 5)}
    L = output.lib()
    buf = C.create_string_buffer(632)
    for w, nm in names.items():
        ref = O.sac_headers(p, kept, o.scalars()["M0"], m6, 1700000000, 540, nm)
        for row, rrow in zip(heads[w], ref):
            for h, r in zip(row, rrow):
                L.swpc_sac_header_bytes(C.byref(h), buf)
                assert buf.raw == O.sac_whdr(r)
    assert _lib.WAV_STRESS not in heads
