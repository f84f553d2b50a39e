"""The reference's output formats restated in Python (TEST INFRASTRUCTURE ONLY).

Byte layouts of sac__whdr / wsac_s / wcsf_s (src/shared/m_sac.f90:267-449,
585-648), tar__whdr / tar__wpad / tar__wend (src/shared/m_tar.f90) as
sac__wtar uses them, write_snp_header and the medium planes of the native
snapshot files (src/swpc_3d/m_snap.f90:324-473, 838-884), the SAC header
values of set_sac_header / initialize_sac_header (src/swpc_3d/m_wav.f90:
276-398) and the Gauss-Kruger inverse projection of geomap__c2g
(src/shared/m_geomap.f90:44-65, src/shared/m_gk.f90).  Only tests/ use it,
to check the library's writers byte for byte.
"""
from __future__ import annotations

import ctypes as C
import math
import struct

import numpy as np

f32 = np.float32
_libm = C.CDLL("libm.so.6")
for _n, _a in (("sinf", 1), ("cosf", 1), ("log10f", 1), ("atan2f", 2)):
    getattr(_libm, _n).restype = C.c_float
    getattr(_libm, _n).argtypes = [C.c_float] * _a

FERR, IERR = -12345.0, -12345


def sac_init() -> dict:
    """sac__init (m_sac.f90:452-562)."""
    h = {k: FERR for k in ("delta", "depmin", "depmax", "b", "e", "o", "a", "stla", "stlo", "stel", "stdp", "evla",
                           "evlo", "evel", "evdp", "mag", "dist", "az", "baz", "gcarc", "depmen", "cmpaz", "cmpinc")}
    h.update({f"t{q}": FERR for q in range(10)})
    h.update({f"user{q}": FERR for q in range(17)})
    h.update({k: IERR for k in ("nzyear", "nzjday", "nzhour", "nzmin", "nzsec", "nzmsec", "npts", "ievtyp", "idep")})
    h.update({f"iuser{q}": IERR for q in range(8)})
    h.update(nvhdr=6, iftype=1, leven=True, lpspol=False, lovrok=True, lcalda=False, luser0=False, tim=0)
    for k in ("kstnm", "khole", "ko", "ka", "kf", "kcmpnm", "knetwk", "kdatrd", "kinst"):
        h[k] = "-12345"
    h["kevnm"] = "-12345"
    h.update({f"kt{q}": "-12345" for q in range(10)})
    h.update({f"kuser{q}": "-12345" for q in range(3)})
    return h


def _ch(s: str, n: int) -> bytes:
    return s.encode()[:n].ljust(n, b" ")


def sac_whdr(h: dict) -> bytes:
    """sac__whdr (m_sac.f90:314-449): 70 reals, 35 integers, 5 logicals, 48 4-byte characters."""
    fh = [FERR] * 70
    fh[0] = float(f32(f32(int(h["delta"] * 1e7)) / f32(1e7)))
    for w, k in ((2, "depmin"), (3, "depmax"), (6, "b"), (7, "e"), (8, "o"), (9, "a"), (32, "stla"), (33, "stlo"),
                 (34, "stel"), (35, "stdp"), (36, "evla"), (37, "evlo"), (38, "evel"), (39, "evdp"), (40, "mag"),
                 (51, "dist"), (52, "az"), (53, "baz"), (54, "gcarc"), (57, "depmen"), (58, "cmpaz"),
                 (59, "cmpinc")):
        fh[w - 1] = h[k]
    for q in range(10):
        fh[10 + q] = h[f"t{q}"]
        fh[40 + q] = h[f"user{q}"]
    for q in range(7):
        fh[63 + q] = h[f"user{10 + q}"]
    ih = [IERR] * 35
    for w, k in ((71, "nzyear"), (72, "nzjday"), (73, "nzhour"), (74, "nzmin"), (75, "nzsec"), (76, "nzmsec"),
                 (77, "nvhdr"), (80, "npts"), (86, "iftype"), (87, "idep"), (93, "ievtyp")):
        ih[w - 71] = h[k]
    for q in range(8):
        ih[27 + q] = h[f"iuser{q}"]
    lh = [int(bool(h[k])) for k in ("leven", "lpspol", "lovrok", "lcalda", "luser0")]
    chars = _ch(h["kstnm"], 8) + _ch(h["kevnm"], 16)
    for k in ["khole", "ko", "ka"] + [f"kt{q}" for q in range(10)] + ["kf", "kuser0", "kuser1", "kuser2", "kcmpnm",
                                                                       "knetwk", "kdatrd", "kinst"]:
        chars += _ch(h[k], 8)
    return struct.pack("<70f", *fh) + struct.pack("<35i", *ih) + struct.pack("<5i", *lh) + chars


def sac_file(h: dict, data) -> bytes:
    return sac_whdr(h) + np.asarray(data, "<f4").tobytes()


def csf_file(hs: list[dict], data) -> bytes:
    """wcsf_s: 'CSFD', ntrace, npts, then header + data per trace."""
    data = np.asarray(data, "<f4")
    out = b"CSFD" + struct.pack("<2i", len(hs), data.shape[1])
    for h, d in zip(hs, data):
        out += sac_whdr(h) + d.tobytes()
    return out


def _oct(v: int, w: int) -> bytes:
    return format(v, "o").rjust(w, "0")[-w:].encode()


def tar_member(name: str, h: dict, data) -> bytes:
    """tarwrite_s (m_sac.f90:812-829) with tar__whdr and tar__wpad (m_tar.f90)."""
    fsize = (158 + h["npts"]) * 4
    b = bytearray(b"\0" + b" " * 511)                   # character(512) assigned one NUL: blank padded
    nm = name.encode()
    b[0:len(nm) + 1] = nm + b"\0"
    b[100:108] = _oct(420, 8)
    b[108:116] = _oct(0, 8)
    b[116:124] = _oct(0, 8)
    b[124:136] = _oct(fsize, 12)
    b[136:148] = _oct(h["tim"], 12)
    b[148:156] = b" " * 8
    b[156:157] = b"0"
    b[157:159] = b"\0\0"                                 # linkname: NUL, then the terminating NUL
    b[257:263] = b"ustar\0"
    b[265:270] = b"root\0"
    b[297:302] = b"root\0"
    b[329:331] = b"\0\0"
    b[337:339] = b"\0\0"
    b[345:347] = b"\0\0"
    b[148:156] = _oct(sum(b), 8)
    return bytes(b) + sac_file(h, data) + b"\0" * (512 - fsize % 512)


def tar_end() -> bytes:
    return b"\0" * 1024


def snp_header(title, exedate, coordinate, snaptype, ns1, ns2, xs1, xs2, dt_s, na1, na2, nmed, nsnp, clon, clat,
               phi) -> bytes:
    """write_snp_header (m_snap.f90:838-884)."""
    return (b"STREAMIO" + b"SWPC_3D " + struct.pack("<i", 6) + _ch(title, 80) + struct.pack("<i", exedate) +
            coordinate.encode() + snaptype.encode() + struct.pack("<2i", ns1, ns2) +
            struct.pack("<2f", xs1[0], xs2[0]) +
            struct.pack("<2f", float(f32(xs1[1]) - f32(xs1[0])), float(f32(xs2[1]) - f32(xs2[0]))) +
            struct.pack("<f", dt_s) + struct.pack("<4i", na1, na2, nmed, nsnp) +
            struct.pack("<3f", clon, clat, phi) + struct.pack("<3f", 1.0, 1.0, 1.0))


# ---------------------------------------------------------------- geography
def geomap_c2g(x, y, clon, clat, phi):
    """geomap__c2g: single-precision rotation, then xytoll_d (m_gk.f90) in double."""
    phr = float(f32(math.pi / 180.0 * float(f32(phi))))
    c, s = f32(_libm.cosf(phr)), f32(_libm.sinf(phr))
    xx = float(c * f32(x) - s * f32(y))
    yy = float(s * f32(x) + c * f32(y))
    a, F, m0 = 6378137.0, 298.257222101, 0.9999
    n = 1.0 / (2.0 * F - 1.0)
    beta = [(1 / 2 + (-2 / 3 + (37 / 96 + (-1 / 360 - 81 / 512 * n) * n) * n) * n) * n,
            ((1 / 48 + (1 / 15 + (-437 / 1440 + 46 / 105 * n) * n) * n) * n) * n,
            (((17 / 480 + (-37 / 840 - 209 / 4480 * n) * n) * n) * n) * n,
            ((((4397 / 161280 - 11 / 504 * n) * n) * n) * n) * n,
            ((((4583 / 161280 * n) * n) * n) * n) * n]
    delta = [(2 + (-2 / 3 + (-2 + (116 / 45 + (26 / 45 + (-2854 / 675) * n) * n) * n) * n) * n) * n,
             ((7 / 3 + (-8 / 5 + (-227 / 45 + (2704 / 315 + (2323 / 945) * n) * n) * n) * n) * n) * n,
             (((56 / 15 + (-136 / 35 + (-1262 / 105 + (73814 / 2835) * n) * n) * n) * n) * n) * n,
             ((((4279 / 630 + (-332 / 35 + (-399572 / 14175) * n) * n) * n) * n) * n) * n,
             (((((4174 / 315 + (-144838 / 6237) * n) * n) * n) * n) * n) * n,
             ((((((601676 / 22275) * n) * n) * n) * n) * n) * n]
    n2 = n * n
    n3, n4 = n2 * n, n2 * n2
    AA = [1 + (1 / 4 + 1 / 64 * n2) * n2, -3 / 2 * (1 - 1 / 8 * n2 - 1 / 64 * n4) * n, 15 / 16 * (1 - 1 / 4 * n2) * n2,
          -35 / 48 * (1 - 5 / 16 * n2) * n3, 315 / 512 * n4, -693 / 1280 * (n4 * n)]
    lam0, phi0 = math.pi / 180.0 * float(f32(clon)), math.pi / 180.0 * float(f32(clat))   # clon, clat are real(SP)
    Abar = m0 * a / (1 + n) * AA[0]
    S = AA[0] * phi0
    for j in range(1, 6):
        S = S + AA[j] * math.sin(2 * j * phi0)
    S = S * (m0 * a / (1 + n))
    xi, eta = (xx * 1000 + S) / Abar, yy * 1000 / Abar
    xi2, eta2 = xi, eta
    for j in range(1, 6):
        xi2 = xi2 - beta[j - 1] * math.sin(2 * j * xi) * math.cosh(2 * j * eta)
        eta2 = eta2 - beta[j - 1] * math.cos(2 * j * xi) * math.sinh(2 * j * eta)
    chi = math.asin(math.sin(xi2) / math.cosh(eta2))
    lam = lam0 + math.atan(math.sinh(eta2) / math.cos(xi2))
    ph = chi
    for j in range(1, 7):
        ph = ph + delta[j - 1] * math.sin(2 * j * chi)
    return float(f32(180.0 / math.pi * lam)), float(f32(180.0 / math.pi * ph))


def localtime(tim, tz_minutes):
    """daytim__localtime with the UTC offset (m_daytim.f90:246-314), via the
    calendar: (year, month, day, hour, min, sec, day of year)."""
    import datetime as dt

    t = dt.datetime(1970, 1, 1) + dt.timedelta(seconds=tim + tz_minutes * 60)
    return t.year, t.month, t.day, t.hour, t.minute, t.second, t.timetuple().tm_yday


def sac_headers(p, stations, M0, m6_first, exedate, tz_minutes, what_names):
    """set_sac_header / initialize_sac_header (m_wav.f90:276-398) for the
    recorded stations: [station][component] dicts of one quantity."""
    names, idep = what_names
    h0 = sac_init()
    s0 = p.sources[0] if p.sources else None
    sx0 = f32(s0.x) if s0 else f32(0)
    sy0 = f32(s0.y) if s0 else f32(0)
    if s0 is not None:
        h0["evlo"], h0["evla"] = geomap_c2g(sx0, sy0, p.clon, p.clat, p.phi)
        h0["evdp"] = float(f32(s0.z))
        h0["o"] = float(f32(s0.tbeg))
    h0["tim"] = exedate
    h0["b"] = float(f32(p.tbeg))
    h0["delta"] = float(f32(p.ntdec_w) * f32(p.dt))
    h0["npts"] = (p.nt - 1) // p.ntdec_w + 1
    m0 = f32(M0)
    h0["mag"] = -12345.0 if m0 < np.finfo(np.float32).eps else \
        float((f32(_libm.log10f(float(m0))) - f32(9.1)) * f32(2.0) / f32(3.0))
    if s0 is not None:
        vals = (s0.fx, s0.fy, s0.fz) if p.bf_mode else m6_first
        for q, v in enumerate(vals):
            h0[f"user{q}"] = float(f32(v))
    h0["user6"], h0["user7"], h0["user8"] = float(f32(p.clon)), float(f32(p.clat)), float(f32(p.phi))
    y, mo, d, hh, mi, ss, jd = localtime(exedate, tz_minutes)
    h0.update(nzyear=y, nzjday=jd, nzhour=hh, nzmin=mi, nzsec=ss, nzmsec=0)
    rows = []
    for st in stations:
        xs, ys = f32(st.x), f32(st.y)
        base = dict(h0)
        base["kevnm"] = p.title[:16].strip()
        base["kstnm"] = st.name.strip()
        base["stlo"], base["stla"] = geomap_c2g(xs, ys, p.clon, p.clat, p.phi)
        base["stdp"] = float(f32(st.z) * f32(1000))
        base["lcalda"] = False
        base["dist"] = float(f32(np.sqrt(f32((sx0 - xs) ** 2 + (sy0 - ys) ** 2))))
        base["az"] = float(f32(180.0 / math.pi * float(f32(_libm.atan2f(float(ys - sy0), float(xs - sx0))))))
        base["baz"] = float(f32(180.0 / math.pi * float(f32(_libm.atan2f(float(sy0 - ys), float(sx0 - xs))))))
        row = []
        for c, nm in enumerate(names):
            h = dict(base)
            h["kcmpnm"] = nm
            h["idep"] = idep
            if idep in (6, 7):
                h["cmpinc"] = 90.0
                h["cmpaz"] = (float(f32(0) + f32(p.phi)), float(f32(90) + f32(p.phi)), 0.0)[c]
            row.append(h)
        rows.append(row)
    return rows
