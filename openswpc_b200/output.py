"""Waveform and snapshot files of a run, in the reference's formats.

wav__write (src/swpc_3d/m_wav.f90:661-811) with the SAC headers of
set_sac_header / initialize_sac_header (:276-398), and the native snapshot
files of snap__setup / newfile_* / snap__write (src/swpc_3d/m_snap.f90:
95-473, 838-939).  The traces and frames come from the device
(``Swpc3D.waveforms``, ``Swpc3D.snapshots``); the bytes are written by the
library's writers (include/swpc_io.h).

The header values that depend on when and where the reference ran --
``exedate`` (POSIX time of the run) and the machine's UTC offset that
daytim__localtime applies -- are arguments, so that a file is reproducible.
"""
from __future__ import annotations

import ctypes as C
import time
from pathlib import Path

import numpy as np

from . import _lib
from .params import Params

f32 = np.float32

# single-precision libm functions, as the Fortran intrinsics of real(4) arguments call them
_libm = C.CDLL("libm.so.6")
for _fn in ("log10f", "atan2f"):
    getattr(_libm, _fn).restype = C.c_float
_libm.log10f.argtypes = [C.c_float]
_libm.atan2f.argtypes = [C.c_float, C.c_float]


class SacHdr(C.Structure):
    """swpc_sac_hdr of include/swpc_io.h (sac__hdr, m_sac.f90:21-156)."""
    _fields_ = ([(n, C.c_double) for n in ("delta", "depmin", "depmax", "scale", "odelta", "b", "e", "o", "a")] +
                [("t", C.c_double * 10), ("f", C.c_double), ("resp", C.c_double * 10)] +
                [(n, C.c_double) for n in ("stla", "stlo", "stel", "stdp", "evla", "evlo", "evel", "evdp", "mag")] +
                [("user", C.c_double * 10)] +
                [(n, C.c_double) for n in ("dist", "az", "baz", "gcarc", "depmen", "cmpaz", "cmpinc", "xminimum",
                                            "xmaximum", "yminimum", "ymaximum")] +
                [("user_x", C.c_double * 7)] +
                [(n, C.c_int) for n in ("nzyear", "nzjday", "nzhour", "nzmin", "nzsec", "nzmsec", "nvhdr", "norid",
                                         "nevid", "npts", "nwfid", "nxsize", "nysize", "iftype", "idep", "iztype",
                                         "iinst", "istreg", "ievreg", "ievtyp", "iqual", "isynth", "imagtyp",
                                         "imagsrc")] +
                [("iuser", C.c_int * 8)] +
                [(n, C.c_int) for n in ("leven", "lpspol", "lovrok", "lcalda", "luser0")] +
                [("kstnm", C.c_char * 8), ("kevnm", C.c_char * 16), ("khole", C.c_char * 8), ("ko", C.c_char * 8),
                 ("ka", C.c_char * 8), ("kt", (C.c_char * 8) * 10), ("kf", C.c_char * 8),
                 ("kuser", (C.c_char * 8) * 3), ("kcmpnm", C.c_char * 8), ("knetwk", C.c_char * 8),
                 ("kdatrd", C.c_char * 8), ("kinst", C.c_char * 8)] +
                [(n, C.c_int) for n in ("nzmonth", "nzday", "tim")])

    def set_text(self, field: str, text: str) -> None:
        """A Fortran character assignment: truncated or blank padded."""
        desc = getattr(type(self), field)
        raw = text.encode()[:desc.size].ljust(desc.size, b" ")
        C.memmove(C.addressof(self) + desc.offset, raw, desc.size)

    def copy(self) -> "SacHdr":
        h = SacHdr()
        C.pointer(h)[0] = self
        return h


class SnpHdr(C.Structure):
    """swpc_snp_hdr of include/swpc_io.h (write_snp_header, m_snap.f90:838-884)."""
    _fields_ = [("title", C.c_char * 80), ("exedate", C.c_int), ("coordinate", C.c_char * 2),
                ("snaptype", C.c_char * 2), ("ns1", C.c_int), ("ns2", C.c_int), ("xs1", C.c_float),
                ("xs2", C.c_float), ("ds1", C.c_float), ("ds2", C.c_float), ("dt", C.c_float), ("na1", C.c_int),
                ("na2", C.c_int), ("nmed", C.c_int), ("nsnp", C.c_int), ("clon", C.c_float), ("clat", C.c_float),
                ("phi", C.c_float)]


_SIGS = {
    "swpc_sac_init": (None, [C.POINTER(SacHdr)]),
    "swpc_sac_header_bytes": (None, [C.POINTER(SacHdr), C.c_char_p]),
    "swpc_sac_write": (C.c_int, [C.c_char_p, C.POINTER(SacHdr), _lib._FP]),
    "swpc_csf_write": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.POINTER(SacHdr), _lib._FP]),
    "swpc_tar_open": (C.c_void_p, [C.c_char_p]),
    "swpc_tar_add_sac": (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(SacHdr), _lib._FP]),
    "swpc_tar_close": (C.c_int, [C.c_void_p]),
    "swpc_snp_write": (C.c_int, [C.c_char_p, C.POINTER(SnpHdr), C.c_int, _lib._FP, C.c_int, _lib._FP]),
    "swpc_geomap_c2g": (None, [C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.POINTER(C.c_float),
                               C.POINTER(C.c_float)]),
}


def lib():
    L = _lib.load()
    for name, (res, args) in _SIGS.items():
        fn = getattr(L, name)
        fn.restype, fn.argtypes = res, args
    return L


def _check(rc, what):
    if rc:
        raise _lib.SwpcError(rc, f"{what} failed")


def geomap_c2g(x: float, y: float, clon: float, clat: float, phi: float) -> tuple[float, float]:
    """Longitude and latitude of grid coordinates (geomap__c2g)."""
    lon, lat = C.c_float(), C.c_float()
    lib().swpc_geomap_c2g(x, y, clon, clat, phi, C.byref(lon), C.byref(lat))
    return lon.value, lat.value


def _is_leap(y: int) -> bool:
    return y % 4 == 0 and (y % 100 != 0 or y % 400 == 0)


def localtime(tim: int, tz_minutes: int) -> tuple[int, int, int, int, int, int, int]:
    """daytim__localtime (src/shared/m_daytim.f90:246-314) shifted by the UTC
    offset: (year, month, day, hour, min, sec, day of year)."""
    t = tim + tz_minutes * 60
    year = 1970
    while t < 0:
        year -= 1
        t += (366 if _is_leap(year) else 365) * 86400
    while t >= (366 if _is_leap(year) else 365) * 86400:
        t -= (366 if _is_leap(year) else 365) * 86400
        year += 1
    jday = t // 86400 + 1
    dom = [31, 29 if _is_leap(year) else 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31]
    month, day = 1, jday
    while day > dom[month - 1]:
        day -= dom[month - 1]
        month += 1
    t -= (jday - 1) * 86400
    hour = t // 3600
    t -= hour * 3600
    return year, month, day, hour, t // 60, t - (t // 60) * 60, jday


def moment_magnitude(m0: float) -> float:
    """moment_magnitude (src/shared/m_fdtool.f90:281-293) in single precision."""
    m0 = f32(m0)
    if m0 < np.finfo(np.float32).eps:
        return -12345.0
    return float((f32(_libm.log10f(float(m0))) - f32(9.1)) * f32(2.0) / f32(3.0))


def local_offset_minutes() -> int:
    """The machine's UTC offset, as date_and_time reports it to daytim__localtime."""
    return int(time.localtime().tm_gmtoff // 60)


def sac_headers(sim, exedate: int | None = None, tz_minutes: int | None = None) -> dict[int, list[list[SacHdr]]]:
    """SAC headers of every recorded trace of a 3D run: {WAV_*: [station][component]}
    as set_sac_header / initialize_sac_header fill them (m_wav.f90:276-398)."""
    p: Params = sim.p
    exedate = int(time.time()) if exedate is None else int(exedate)
    tz = local_offset_minutes() if tz_minutes is None else int(tz_minutes)
    L = lib()
    h0 = SacHdr()
    L.swpc_sac_init(C.byref(h0))
    # the first source record is the hypocentre (m_source.f90:673-686)
    s0 = p.sources[0] if p.sources else None
    sx0 = f32(s0.x) if s0 else f32(0.0)
    sy0 = f32(s0.y) if s0 else f32(0.0)
    if s0 is not None:
        h0.evlo, h0.evla = geomap_c2g(float(sx0), float(sy0), p.clon, p.clat, p.phi)
        h0.evdp = float(f32(s0.z))
        h0.o = float(f32(s0.tbeg))
    h0.tim = exedate
    h0.b = float(f32(p.tbeg))
    h0.delta = float(f32(p.ntdec_w) * f32(p.dt))
    h0.npts = (p.nt - 1) // p.ntdec_w + 1
    h0.mag = moment_magnitude(sim.M0)
    if s0 is not None:
        if p.bf_mode:
            for q, v in enumerate((s0.fx, s0.fy, s0.fz)):
                h0.user[q] = float(f32(v))
        else:
            m6 = s0.moment(lambda *a: _sdr(L, *a))
            for q, v in enumerate(m6):
                h0.user[q] = float(f32(v))
    h0.user[6], h0.user[7], h0.user[8] = float(f32(p.clon)), float(f32(p.clat)), float(f32(p.phi))
    y, mo, d, hh, mi, ss, jd = localtime(exedate, tz)
    h0.nzyear, h0.nzmonth, h0.nzday, h0.nzhour, h0.nzmin, h0.nzsec, h0.nzjday, h0.nzmsec = y, mo, d, hh, mi, ss, jd, 0
    title16 = p.title[:16].strip()
    comps = {_lib.WAV_V: (["Vx", "Vy", "Vz"], 7), _lib.WAV_U: (["Ux", "Uy", "Uz"], 6),
             _lib.WAV_STRESS: (["Sxx", "Syy", "Szz", "Syz", "Sxz", "Sxy"], 5),
             _lib.WAV_STRAIN: (["Exx", "Eyy", "Ezz", "Eyz", "Exz", "Exy"], 5)}
    stations = [st for st in p.stations]
    out = {}
    for what, (names, idep) in comps.items():
        if not (sim.what & what):
            continue
        rows = []
        for st in _recorded(sim, stations):
            lon, lat = geomap_c2g(st.x, st.y, p.clon, p.clat, p.phi)
            xs, ys = f32(st.x), f32(st.y)
            base = h0.copy()
            base.set_text("kevnm", title16)
            base.set_text("kstnm", st.name.strip())
            base.stlo, base.stla = lon, lat
            base.stdp = float(f32(st.z) * f32(1000))
            base.lcalda = 0
            base.dist = float(np.sqrt((sx0 - xs) ** 2 + (sy0 - ys) ** 2, dtype=np.float32))
            # std__rad2deg of single precision: real(180 / PI * rad) in double (m_std.f90:152-159)
            base.az = float(f32(180.0 / np.pi * float(f32(_libm.atan2f(float(ys - sy0), float(xs - sx0))))))
            base.baz = float(f32(180.0 / np.pi * float(f32(_libm.atan2f(float(sy0 - ys), float(sx0 - xs))))))
            row = []
            for c, name in enumerate(names):
                h = base.copy()
                h.set_text("kcmpnm", name)
                h.idep = idep
                if what in (_lib.WAV_V, _lib.WAV_U):
                    # x and y along the rotated grid axes, z vertical (m_wav.f90:289-291)
                    h.cmpinc = 90.0
                    h.cmpaz = float(f32(0.0) + f32(p.phi)) if c == 0 else float(f32(90.0) + f32(p.phi)) \
                        if c == 1 else 0.0
                row.append(h)
            rows.append(row)
        out[what] = rows
    return out


def _sdr(L, strike, dip, rake):
    m6 = (C.c_float * 6)()
    L.swpc_sdr2moment(strike, dip, rake, m6)
    return tuple(m6)


def _recorded(sim, stations):
    """The stations set_stinfo kept, in file order (the same selection the
    trace buffer follows)."""
    from .swpc3d import station_grid

    kept = []
    for st in stations:
        q = Params(**{**sim.p.__dict__, "stations": [st]})
        i, _, _ = station_grid(q, sim.medium.kfs, sim.medium.kob)
        if len(i):
            kept.append(st)
    return kept


def wav_write(sim, odir: str | Path, wav_format: str = "sac", exedate: int | None = None,
              tz_minutes: int | None = None) -> list[Path]:
    """wav__write (m_wav.f90:661-811): every recorded trace to
    ``odir/wav`` as SAC files, one CSF file per quantity, or SAC members of
    tar archives per station ('tar_st') or for the node ('tar_node')."""
    p: Params = sim.p
    L = lib()
    wdir = Path(odir) / "wav"
    wdir.mkdir(parents=True, exist_ok=True)
    heads = sac_headers(sim, exedate, tz_minutes)
    title = p.title.strip()
    traces = {what: sim.waveforms(what) for what in heads}   # (nst, ncmp, ntw)
    written = []
    order = [w for w in (_lib.WAV_V, _lib.WAV_U, _lib.WAV_STRESS, _lib.WAV_STRAIN) if w in heads]
    if wav_format == "sac":
        for n in range(sim.nst):
            for what in order:
                for c, h in enumerate(heads[what][n]):
                    fn = wdir / f"{title}.3d.{_txt(h.kstnm)}.{_txt(h.kcmpnm)}.sac"
                    data = np.ascontiguousarray(traces[what][n, c], np.float32)
                    _check(L.swpc_sac_write(str(fn).encode(), C.byref(h), _lib.fptr(data)), "swpc_sac_write")
                    written.append(fn)
    elif wav_format == "csf":
        fn = wdir / f"{title}__{0:05d}__.csf"
        for what in order:
            hs = [h for row in heads[what] for h in row]
            arr = (SacHdr * len(hs))(*hs)
            data = np.ascontiguousarray(traces[what].reshape(-1, traces[what].shape[-1]), np.float32)
            _check(L.swpc_csf_write(str(fn).encode(), len(hs), data.shape[1], arr, _lib.fptr(data)),
                   "swpc_csf_write")
        written.append(fn)
    elif wav_format in ("tar_st", "tar_node"):
        t = None
        if wav_format == "tar_node":
            fn = wdir / f"{title}.3d.{0:06d}.sac.tar"
            t = L.swpc_tar_open(str(fn).encode())
            written.append(fn)
        for n in range(sim.nst):
            if wav_format == "tar_st":
                fn = wdir / f"{title}.3d.{_txt(heads[order[0]][n][0].kstnm)}.sac.tar"
                t = L.swpc_tar_open(str(fn).encode())
                written.append(fn)
            if not t:
                raise OSError(f"cannot open {fn}")
            for what in order:
                for c, h in enumerate(heads[what][n]):
                    name = f"{title}.{_txt(h.kstnm)}.3d.{_txt(h.kcmpnm)}.sac"
                    data = np.ascontiguousarray(traces[what][n, c], np.float32)
                    _check(L.swpc_tar_add_sac(t, name.encode(), C.byref(h), _lib.fptr(data)), "swpc_tar_add_sac")
            if wav_format == "tar_st":
                _check(L.swpc_tar_close(t), "swpc_tar_close")
        if wav_format == "tar_node":
            _check(L.swpc_tar_close(t), "swpc_tar_close")
    else:
        raise ValueError(f"unknown wav_format {wav_format!r}")
    return written


def _txt(field) -> str:
    return bytes(field).decode().rstrip()


_COORD = {0: "yz", 1: "xz", 2: "xy", 3: "fs", 4: "ob"}
_QUANT = {0: ("ps", 4), 1: ("v3", 3), 2: ("u3", 3)}


def snap_write(sim, odir: str | Path, exedate: int | None = None) -> list[Path]:
    """The native snapshot files of every plane the run recorded (snp_format
    'native'): odir/<title>.3d.<section>.<quantity>.snp with the header of
    write_snp_header, the medium planes of newfile_yz / newfile_xz /
    newfile_xy and the frames (m_snap.f90:240-256, 324-473, 838-884)."""
    from .params import SNAP_QUANTITIES, SNAP_SECTIONS, snap_plane

    p: Params = sim.p
    L = lib()
    exedate = int(time.time()) if exedate is None else int(exedate)
    Path(odir).mkdir(parents=True, exist_ok=True)
    m = sim.medium
    ix = lambda k, i, j: (j + 2, i + 2, k + 2)   # memory-box indexing of the host medium
    nxs = (p.nx + p.idec // 2) // p.idec
    nys = (p.ny + p.jdec // 2) // p.jdec
    nzs = (p.nz + p.kdec // 2) // p.kdec
    ax = lambda n, dec, beg, d: np.array([L.swpc_i2x(q * dec - dec // 2, beg, d) for q in range(1, n + 1)],
                                         np.float32)
    xsnp, ysnp, zsnp = ax(nxs, p.idec, p.xbeg, p.dx), ax(nys, p.jdec, p.ybeg, p.dy), ax(nzs, p.kdec, p.zbeg, p.dz)
    d = sim.snap_desc                            # the section positions of snap__setup (m_snap.f90:157-159)
    i0, j0, k0 = d.i0_yz, d.j0_xz, d.k0_xy
    written = []
    for name in sorted(p.snaps, key=snap_plane):
        sec, q = name.split("_")
        s = SNAP_SECTIONS.index(sec)
        snaptype, nsnp = _QUANT[SNAP_QUANTITIES.index(q)]
        h = SnpHdr()
        h.title = p.title.encode()[:80].ljust(80, b" ")
        h.exedate = exedate
        h.coordinate = sec.encode()
        h.snaptype = snaptype.encode()
        if sec == "yz":
            axes, (n1, n2), (na1, na2) = (ysnp, zsnp), (nys, nzs), (p.na // p.jdec, p.na // p.kdec)
            cells = [[(k * p.kdec - p.kdec // 2, i0, j * p.jdec - p.jdec // 2) for k in range(1, n2 + 1)]
                     for j in range(1, n1 + 1)]
            nmed = 3
        elif sec == "xz":
            axes, (n1, n2), (na1, na2) = (xsnp, zsnp), (nxs, nzs), (p.na // p.idec, p.na // p.kdec)
            cells = [[(k * p.kdec - p.kdec // 2, i * p.idec - p.idec // 2, j0) for k in range(1, n2 + 1)]
                     for i in range(1, n1 + 1)]
            nmed = 3
        else:
            axes, (n1, n2), (na1, na2) = (xsnp, ysnp), (nxs, nys), (p.na // p.idec, p.na // p.jdec)
            cells = []
            for i in range(1, n1 + 1):
                row = []
                for j in range(1, n2 + 1):
                    ii, jj = i * p.idec - p.idec // 2, j * p.jdec - p.jdec // 2
                    kk = (int(m.kfs[jj + 2, ii + 2]) + 1 if sec == "fs" else
                          int(m.kob[jj + 2, ii + 2]) + 1 if sec == "ob" else k0)
                    row.append((kk, ii, jj))
                cells.append(row)
            nmed = 6
        h.ns1, h.ns2 = n1, n2
        h.xs1, h.xs2 = axes[0][0], axes[1][0]
        h.ds1, h.ds2 = axes[0][1] - axes[0][0], axes[1][1] - axes[1][0]
        h.dt = f32(p.dt) * f32(p.ntdec_s)
        h.na1, h.na2 = na1, na2
        h.nmed, h.nsnp = nmed, nsnp
        h.clon, h.clat, h.phi = p.clon, p.clat, p.phi
        # medium planes buf(n1, n2) in Fortran order: rho, lam, mu (+ topography of the horizontal planes)
        med = [np.zeros((n2, n1), np.float32) for _ in range(3)]
        for a in range(n1):
            for b in range(n2):
                e = ix(*cells[a][b])
                med[0][b, a], med[1][b, a], med[2][b, a] = m.rho[e], m.lam[e], m.mu[e]
        if sec in ("xy", "fs", "ob"):
            from .params import bddep_of
            bd = bddep_of(p)
            topo = np.zeros((n2, n1), np.float32)
            for a in range(n1):
                for b in range(n2):
                    ii, jj = (a + 1) * p.idec - p.idec // 2, (b + 1) * p.jdec - p.jdec // 2
                    topo[b, a] = -bd[jj + 2, ii + 2, 0] * f32(1000)
            med.append(topo)
        medarr = np.ascontiguousarray(np.stack(med), np.float32)
        frames = np.ascontiguousarray(sim.snapshots(name), np.float32)
        nframes = frames.shape[0]
        fn = Path(odir) / f"{p.title.strip()}.3d.{sec}.{q}.snp"
        _check(L.swpc_snp_write(str(fn).encode(), C.byref(h), len(med), _lib.fptr(medarr), nframes,
                                _lib.fptr(frames)), "swpc_snp_write")
        written.append(fn)
    return written
