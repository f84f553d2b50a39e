"""Run parameters of OpenSWPC and a reader for its ``input.inf`` files.

The reference reads ``key = value`` lines with ``!!`` comments, falls back to
a default for every missing key and expands ``${VAR}`` from the environment
(src/shared/m_readini.f90:29-100, src/shared/m_system.f90:75-102).  The
defaults below are the ones global__readprm, medium__setup, source__setup,
wav__setup and m_report use (src/swpc_3d/m_global.f90:126-179,
m_medium.f90:79-84, m_source.f90:93-99, m_wav.f90:76-84,
m_report.f90 ntdec_r).
"""
from __future__ import annotations

import os
import re
import warnings
from dataclasses import dataclass, field, fields
from pathlib import Path

import numpy as np


@dataclass
class Layer:
    """One row of an ``lhm`` velocity file: depth(top) rho vp vs qp qs."""

    depth: float
    rho: float
    vp: float
    vs: float
    qp: float
    qs: float


@dataclass
class Source:
    """One source grid point after parsing (xym0ij layout: x y z tbeg trise mo mij)."""

    x: float
    y: float
    z: float
    tbeg: float
    trise: float
    mo: float = 0.0
    mxx: float = 0.0
    myy: float = 0.0
    mzz: float = 0.0
    myz: float = 0.0
    mxz: float = 0.0
    mxy: float = 0.0
    fx: float = 0.0
    fy: float = 0.0
    fz: float = 0.0
    # double couple (xym0dc / xymwdc): strike (from the map azimuth), dip and
    # rake in degrees; the moment tensor is then formed by sdr2moment
    # (m_fdtool.f90:307-336) by whoever consumes the source, in place of mij
    strike: float | None = None
    dip: float | None = None
    rake: float | None = None

    def moment(self, sdr2moment) -> tuple:
        """(mxx, myy, mzz, myz, mxz, mxy): the given components, or for a
        double couple the result of ``sdr2moment(strike, dip, rake)``."""
        if self.strike is None:
            return (self.mxx, self.myy, self.mzz, self.myz, self.mxz, self.mxy)
        return tuple(sdr2moment(self.strike, self.dip, self.rake))


@dataclass
class Station:
    """One station (m_wav.f90 set_stinfo): x y z name zsw."""

    x: float
    y: float
    z: float
    name: str = "st"
    zsw: str = "dep"


@dataclass
class Params:
    title: str = "swpc3d"
    # map projection of the grid (m_global.f90:171-173): centre longitude, latitude, azimuth of the x axis
    clon: float = 139.7604
    clat: float = 35.7182
    phi: float = 0.0
    nx: int = 256
    ny: int = 256
    nz: int = 256
    nt: int = 1000
    dx: float = 0.5
    dy: float = 0.5
    dz: float = 0.5
    dt: float = 0.01
    na: int = 20
    nm: int = 3
    xbeg: float | None = None
    ybeg: float | None = None
    zbeg: float | None = None
    tbeg: float = 0.0
    fq_min: float = 0.05
    fq_max: float = 5.0
    fq_ref: float = 1.0
    vcut: float = 0.0
    rhomin: float = 1.0
    stftype: str = "kupper"
    bf_mode: bool = False
    green_mode: bool = False
    green_cmp: str = "z"
    green_trise: float = 1.0
    green_station: int = 0
    ntdec_r: int = 50
    ntdec_w: int = 10
    sw_wav_v: bool = True
    sw_wav_u: bool = False
    sw_wav_stress: bool = False
    sw_wav_strain: bool = False
    abc_type: str = "pml"
    stabilize_pml: bool = False   # m_medium.f90:219-222 (3D)
    munk_profile: bool = False    # Munk's seawater profile above depth(1) (m_vmodel_lhm.f90:53-54)
    # plane-wave mode (m_source.f90:67-79, pw_setup :315-465): a plane P or S wave in place of a source grid
    pw_mode: bool = False
    pw_ztop: float = 1e30
    pw_zlen: float = -1.0
    pw_ps: str = ""
    pw_strike: float = 0.0
    pw_dip: float = 0.0
    pw_rake: float = 0.0
    # source depth fitted to a boundary depth: 'asis' or 'bd0'..'bd9' (m_source.f90:99, 262-270)
    sdep_fit: str = "asis"
    # boundary depths bddep(i, j, 0:9) of the memory box, shape (ny+6, nx+6, 10) in 3D and (nx+6, 10) in 2D, for
    # a velocity model that carries its own (vmodel_grd / vmodel_user); None takes vmodel_lhm's: depth(1) of
    # the layer table at index 0 and -9999 at 1..9 (m_vmodel_lhm.f90:104, 161)
    bddep: np.ndarray | None = None
    # snapshots (m_snap.f90:105-127): enabled planes as "<section>_<quantity>"
    # names (sections yz xz xy fs ob, quantities ps v u), e.g. {"xz_v", "fs_u"}
    snaps: set = field(default_factory=set)
    z0_xy: float | None = None
    x0_yz: float | None = None
    y0_xz: float | None = None
    idec: int = 1
    jdec: int = 1
    kdec: int = 1
    ntdec_s: int = 10
    layers: list[Layer] = field(default_factory=list)
    sources: list[Source] = field(default_factory=list)
    stations: list[Station] = field(default_factory=list)

    def __post_init__(self):
        # m_global.f90:167-169 (integer division nx/2 in the defaults)
        if self.xbeg is None:
            self.xbeg = float(np.float32(-(self.nx // 2)) * np.float32(self.dx))
        if self.ybeg is None:
            self.ybeg = float(np.float32(-(self.ny // 2)) * np.float32(self.dy))
        if self.zbeg is None:
            self.zbeg = float(np.float32(-30) * np.float32(self.dz))

    def check(self) -> None:
        if self.sdep_fit != "asis" and self.sdep_fit not in BD_NAMES:
            raise ValueError("sdep_fit must be 'asis' or 'bd0'..'bd9'")
        if self.abc_type not in ("pml", "cerjan"):
            raise ValueError("abc_type must be 'pml' or 'cerjan'")
        if self.nm not in (0, 1, 2, 3):
            raise ValueError("nm must be 0..3")
        if self.stftype not in ("kupper", "boxcar", "triangle", "herrmann", "cosine", "scosine", "texp"):
            raise ValueError(f"unknown stftype {self.stftype!r}")


NBD = 9   # boundary depths kept per column (m_global.f90:32)
BD_NAMES = tuple(f"bd{n}" for n in range(NBD + 1))
# station depth modes of set_stinfo (m_wav.f90:209-225): the code is 10 + n for 'bd<n>'
ZSW_CODES = {"dep": 0, "fsb": 1, "obb": 2, "oba": 3, **{f"bd{n}": 10 + n for n in range(NBD + 1)}}


def zsw_code(zsw: str, name: str = "") -> int:
    """The depth-mode code of a station; an unknown mode is taken as 'dep'
    with a message, as set_stinfo does (m_wav.f90:224-226)."""
    code = ZSW_CODES.get(zsw)
    if code is None:
        warnings.warn(f"unknown zsw type {zsw!r} in station file (station {name}). Assume 'dep'", stacklevel=2)
        return 0
    return code


def sdep_index(p) -> int:
    """The bddep index that sdep_fit selects, or -1 for 'asis'."""
    s = getattr(p, "sdep_fit", "asis")
    return BD_NAMES.index(s) if s in BD_NAMES else -1


def bddep_of(p, two_d: bool = False) -> np.ndarray:
    """bddep over the memory box: the caller's array, else vmodel_lhm's rule
    (depth(1) of the layer table, then -9999; m_vmodel_lhm.f90:104, 161)."""
    shape = (p.nx + 6, NBD + 1) if two_d else (p.ny + 6, p.nx + 6, NBD + 1)
    if getattr(p, "bddep", None) is not None:
        bd = np.ascontiguousarray(p.bddep, np.float32)
        if bd.shape != shape:
            raise ValueError(f"bddep must have shape {shape}, got {bd.shape}")
        return bd
    bd = np.full(shape, np.float32(-9999.0), np.float32)
    bd[..., 0] = np.float32(p.layers[0].depth) if p.layers else np.float32(0.0)
    return bd


SNAP_SECTIONS = ("yz", "xz", "xy", "fs", "ob")
SNAP_QUANTITIES = ("ps", "v", "u")


def snap_plane(name: str) -> int:
    """Plane id 3*section + quantity of a "<section>_<quantity>" name."""
    sec, q = name.split("_")
    return 3 * SNAP_SECTIONS.index(sec) + SNAP_QUANTITIES.index(q)


_COMMENT = re.compile(r"!!.*$")


def _expand_env(s: str) -> str:
    return re.sub(r"\$\{(\w+)\}", lambda m: os.environ.get(m.group(1), ""), s)


def read_ini(path: str | Path) -> dict[str, str]:
    """Parse an OpenSWPC ``input.inf`` into a key -> raw value mapping."""
    out: dict[str, str] = {}
    for line in Path(path).read_text().splitlines():
        line = _COMMENT.sub("", line).strip()
        if not line or line.startswith("#") or "=" not in line:
            continue
        key, val = line.split("=", 1)
        key = key.strip()
        val = _expand_env(val.strip())
        if len(val) >= 2 and val[0] == val[-1] and val[0] in "'\"":
            val = val[1:-1]
        out[key] = val
    return out


def _conv(val: str, typ):
    if typ is bool:
        v = val.strip().lower()
        if v in (".true.", "true", "t", ".t."):
            return True
        if v in (".false.", "false", "f", ".f."):
            return False
        raise ValueError(f"not a logical: {val!r}")
    if typ is int:
        return int(float(val))
    if typ is float:
        return float(val.replace("d", "e").replace("D", "e"))
    return val


def params_from_ini(path: str | Path, strict: bool = False) -> Params:
    """Build :class:`Params` from an input file; missing keys take defaults
    (or raise with ``strict``, as readini__strict_mode does)."""
    kv = read_ini(path)
    types = {"title": str, "nx": int, "ny": int, "nz": int, "nt": int, "dx": float, "dy": float, "dz": float,
             "dt": float, "na": int, "xbeg": float, "ybeg": float, "zbeg": float, "tbeg": float, "fq_min": float,
             "fq_max": float, "fq_ref": float, "vcut": float, "rhomin": float, "stftype": str, "bf_mode": bool,
             "green_mode": bool, "green_cmp": str, "green_trise": float, "ntdec_r": int, "ntdec_w": int,
             "sw_wav_v": bool, "sw_wav_u": bool, "sw_wav_stress": bool, "sw_wav_strain": bool, "abc_type": str,
             "stabilize_pml": bool, "sdep_fit": str, "munk_profile": bool, "pw_mode": bool, "pw_ztop": float,
             "pw_zlen": float, "pw_ps": str, "pw_strike": float, "pw_dip": float, "pw_rake": float,
             "clon": float, "clat": float, "phi": float}
    args = {}
    for key, typ in types.items():
        if key in kv:
            args[key] = _conv(kv[key], typ)
        elif strict and key not in ("xbeg", "ybeg", "zbeg", "sdep_fit", "munk_profile", "clon", "clat", "phi") \
                and not key.startswith("pw_"):
            raise KeyError(f"parameter {key} missing in strict mode")
    for key in ("z0_xy", "x0_yz", "y0_xz"):
        if key in kv:
            args[key] = _conv(kv[key], float)
    for key in ("idec", "jdec", "kdec", "ntdec_s"):
        if key in kv:
            args[key] = _conv(kv[key], int)
    args["snaps"] = {f"{sec}_{q}" for sec in SNAP_SECTIONS for q in SNAP_QUANTITIES
                     if _conv(kv.get(f"{sec}_{q}%sw", ".false."), bool)}
    p = Params(**args)
    base = Path(path).parent
    if kv.get("vmodel_type", "lhm") == "lhm" and "fn_lhm" in kv:
        p.layers = read_lhm(_resolve(base, kv["fn_lhm"]))
    if "fn_stf" in kv and not p.green_mode and not p.pw_mode:
        p.sources = read_sources(_resolve(base, kv["fn_stf"]), kv.get("stf_format", "xym0ij"), p.bf_mode)
    if "fn_stloc" in kv:
        p.stations = read_stations(_resolve(base, kv["fn_stloc"]))
    return p


def _resolve(base: Path, fn: str) -> Path:
    p = Path(fn)
    if p.exists():
        return p
    return base / fn if (base / fn).exists() else base.parent / fn


def _data_lines(path: Path):
    for line in Path(path).read_text().splitlines():
        s = line.strip()
        if not s or s.startswith("#"):
            continue
        yield s.split()


def read_lhm(path: str | Path) -> list[Layer]:
    """``lhm`` file: depth rho vp vs qp qs per line (m_vmodel_lhm.f90:80-90)."""
    return [Layer(*map(float, t[:6])) for t in _data_lines(Path(path))]


def read_sources(path: str | Path, stf_format: str = "xym0ij", bf_mode: bool = False) -> list[Source]:
    """Source list in the xy-based formats of source__grid_moment /
    source__grid_bodyforce (m_source.f90:511-559, 740-744)."""
    out = []
    for t in _data_lines(Path(path)):
        v = [float(x) for x in t[:12] if _isnum(x)]
        if bf_mode:
            out.append(Source(x=v[0], y=v[1], z=v[2], tbeg=v[3], trise=v[4], fx=v[5], fy=v[6], fz=v[7]))
        elif stf_format == "xym0ij":
            out.append(Source(*v[:5], mo=v[5], mxx=v[6], myy=v[7], mzz=v[8], myz=v[9], mxz=v[10], mxy=v[11]))
        elif stf_format == "xym0dc":
            out.append(dc_source(*v[:6], strike=v[6], dip=v[7], rake=v[8]))
        elif stf_format in ("xymwij", "xymwdc"):
            mo = float(np.float32(10.0) ** np.float32(1.5 * v[5] + 9.05))
            if stf_format == "xymwij":
                out.append(Source(*v[:5], mo=mo, mxx=v[6], myy=v[7], mzz=v[8], myz=v[9], mxz=v[10], mxy=v[11]))
            else:
                out.append(dc_source(*v[:5], mo, strike=v[6], dip=v[7], rake=v[8]))
        else:
            raise ValueError(f"source format {stf_format!r} is not supported (geographic formats need m_geomap)")
    return out


def dc_source(x, y, z, tbeg, trise, mo, strike, dip, rake, phi: float = 0.0) -> Source:
    """Double-couple source (xym0dc): strike is measured from the map azimuth
    phi (m_source.f90:525).  The moment tensor is not formed here: the solver
    forms it with its own sdr2moment (m_fdtool.f90:307-336) at source setup,
    see :meth:`Source.moment`."""
    return Source(x, y, z, tbeg, trise, mo=mo, strike=float(np.float32(strike) - np.float32(phi)),
                  dip=float(dip), rake=float(rake))


def _isnum(s: str) -> bool:
    try:
        float(s)
        return True
    except ValueError:
        return False


def read_stations(path: str | Path) -> list[Station]:
    """``stloc.xy``: x y z name zsw (m_wav.f90:178-181)."""
    out = []
    for t in _data_lines(Path(path)):
        out.append(Station(float(t[0]), float(t[1]), float(t[2]), t[3] if len(t) > 3 else "st",
                           t[4] if len(t) > 4 else "dep"))
    return out
