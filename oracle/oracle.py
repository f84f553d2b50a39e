"""ctypes driver of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads ``oracle/lib/liboracle3d_<variant>.so`` (built by build_oracle.py) and
runs the reference's setup and time loop as restated in swpc3d_oracle.c.
Only tests/, the package smoke check and bench.py's cpu_baseline leg use it,
as the checker or as the timed CPU baseline.

The oracle's own setup follows the reference modules; every input it shares
with the GPU driver (layer table, perturbation xi, source and station lists)
is the raw input a user would give OpenSWPC.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "lib"

_FP = C.POINTER(C.c_float)
_IP = C.POINTER(C.c_int)
_cache: dict[str, C.CDLL] = {}

# station depth modes of set_stinfo (m_wav.f90:209-225); 'bd<n>' is 10 + n, anything else is 'dep'
ZSW = {"dep": 0, "fsb": 1, "obb": 2, "oba": 3, **{f"bd{n}": 10 + n for n in range(10)}}
NBD = 9


def _sdep(p) -> int:
    """sdep_fit of the run (m_source.f90:99): -1 for 'asis', n for 'bd<n>'."""
    s = getattr(p, "sdep_fit", "asis")
    return int(s[2:]) if len(s) == 3 and s[:2] == "bd" and s[2].isdigit() else -1


def _moment6(lib, s):
    """The moment tensor of a source: its components, or for a double couple
    (strike/dip/rake given) the oracle's own sdr2moment (m_fdtool.f90:307-336)."""
    if getattr(s, "strike", None) is None:
        return [s.mxx, s.myy, s.mzz, s.myz, s.mxz, s.mxy]
    m6 = (C.c_float * 6)()
    lib.o3d_sdr2moment(s.strike, s.dip, s.rake, m6)
    return list(m6)
STF = {"kupper": 0, "boxcar": 1, "triangle": 2, "herrmann": 3, "cosine": 4, "scosine": 4, "texp": 5}

# field ids of o3d_ptr
FIELD_IDS = {"Vx": 0, "Vy": 1, "Vz": 2, "Sxx": 3, "Syy": 4, "Szz": 5, "Syz": 6, "Sxz": 7, "Sxy": 8,
             "Rxx": 10, "Ryy": 11, "Rzz": 12, "Ryz": 13, "Rxz": 14, "Rxy": 15,
             "lam": 20, "mu": 21, "taup": 22, "taus": 23, "bx": 24, "by": 25, "bz": 26, "muyz": 27,
             "muxz": 28, "muxy": 29, "frho": 30, "flam": 31, "fmu": 32, "ftaup": 33, "ftaus": 34, "fbx": 35,
             "fby": 36, "fbz": 37, "fmuyz": 38, "fmuxz": 39, "fmuxy": 40, "kfs": 50, "kob": 51, "kfs_top": 52,
             "kfs_bot": 53, "kob_top": 54, "kob_bot": 55, "kbeg_a": 56, "bddep": 57}
AUX_NAMES = ["axVx", "ayVx", "azVx", "axVy", "ayVy", "azVy", "axVz", "ayVz", "azVz",
             "axSxx", "aySxy", "azSxz", "axSxy", "aySyy", "azSyz", "axSxz", "aySyz", "azSzz"]
for _n, _a in enumerate(AUX_NAMES):
    FIELD_IDS[_a] = 60 + _n
# Cerjan sponge factors (n values per axis)
CERJAN_NAMES = ["gx_c", "gx_b", "gy_c", "gy_b", "gz_c", "gz_b"]
for _n, _a in enumerate(CERJAN_NAMES):
    FIELD_IDS[_a] = 110 + _n


def load(variant: str = "f32", kind: str = "3d") -> C.CDLL:
    key = f"{kind}_{variant}"
    if key in _cache:
        return _cache[key]
    path = LIB / f"liboracle{kind}_{variant}.so"
    if not path.exists():
        import importlib.util
        spec = importlib.util.spec_from_file_location("build_oracle", HERE / "build_oracle.py")
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    lib = C.CDLL(str(path))
    vp, i, f, d = C.c_void_p, C.c_int, C.c_float, C.c_double
    sig = {
        "o3d_create": (vp, [i, i, i, i, i, i, d, d, d, f, f, f, f, f, i]),
        "o3d_destroy": (None, [vp]),
        "o3d_vmodel_lhm": (None, [vp, i, _FP, _FP, _FP, _FP, _FP, _FP, f, _FP, f, _FP, _FP]),
        "o3d_medium_setup": (None, [vp, _FP, _FP, f, f, f]),
        "o3d_set_medium": (None, [vp, _FP, _FP, _FP, _FP, _FP, _FP, _FP, _FP, _FP, _FP, _FP]),
        "o3d_set_maps": (None, [vp, _IP, _IP, _IP, _IP, _IP, _IP]),
        "o3d_kernel_setup": (None, [vp]),
        "o3d_absorb_setup": (None, [vp, f]),
        "o3d_cerjan_setup": (None, [vp]),
        "o3d_set_stabilize": (None, [vp, i]),
        "o3d_green_store_setup": (None, [vp, i, _IP, _IP, _IP, i, i]),
        "o3d_set_profiles": (None, [vp, _FP, _FP, _FP, _FP, _FP, _FP]),
        "o3d_set_sdep_fit": (None, [vp, i]),
        "o3d_set_munk": (None, [vp, i]),
        "o3d_pw_setup": (None, [vp, f, f, i, f, f, f, i]),
        "o3d_seawater_vel": (f, [f, i]),
        "o3d_set_bddep": (None, [vp, _FP]),
        "o3d_source_setup": (i, [vp, i, i, _FP, _FP, _FP, _FP, _FP, _FP, _FP, i]),
        "o3d_green_setup": (None, [vp, i, i, i, C.c_char, f, f, i]),
        "o3d_wav_setup": (i, [vp, i, _FP, _FP, _FP, _IP, i, i, i, i, i, _IP, _IP, _IP]),
        "o3d_step": (None, [vp, i]),
        "o3d_vmax": (None, [vp, _FP]),
        "o3d_dims": (None, [vp, C.POINTER(C.c_long)]),
        "o3d_scalars": (None, [vp, _FP]),
        "o3d_ptr": (vp, [vp, i]),
        "o3d_mpr_size": (i, []),
        "o3d_spr_size": (i, []),
        "o3d_x2i": (i, [f, f, f]),
        "o3d_i2x": (f, [i, f, f]),
        "o3d_momentrate": (f, [f, i, f, f]),
        "o3d_sdr2moment": (None, [f, f, f, _FP]),
        "o3d_visco_set_relaxtime": (None, [i, _FP, f, f]),
        "o3d_visco_constq_zeta": (f, [i, f, f, _FP]),
        "o3d_snap_setup": (i, [vp, i, i, i, i, i, f, f, f]),
        "o3d_snap_write": (None, [vp, i]),
        "o3d_snap_dims": (None, [vp, _IP]),
        "o3d_snap_frames": (vp, [vp, i]),
        "o3d_snap_max": (vp, [vp, i]),
    }
    for name in ("o3d_update_stress", "o3d_absorb_update_stress", "o3d_update_vel", "o3d_absorb_update_vel",
                 "o3d_comm_stress", "o3d_comm_vel"):
        sig[name] = (None, [vp])
    for name in ("o3d_stressglut", "o3d_bodyforce", "o3d_green_source", "o3d_wav_store"):
        sig[name] = (None, [vp, i])
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _cache[key] = lib
    return lib


def _f(a):
    return None if a is None else np.ascontiguousarray(a, np.float32).ctypes.data_as(_FP)


class Oracle3D:
    """The reference 3D run restated on the CPU.

    ``p`` is an ``openswpc_b200.params.Params``-like object (duck-typed: the
    oracle reads attributes only).  ``variant`` selects f32 / mixed / f64.
    """

    def __init__(self, p, xi=None, variant: str = "f32", threads: int = 1, medium=None, profiles=None):
        self.p = p
        self.lib = lib = load(variant)
        self.variant = variant
        self.mpr = np.float32 if lib.o3d_mpr_size() == 4 else np.float64
        self.spr = np.float32 if lib.o3d_spr_size() == 4 else np.float64
        self.o = lib.o3d_create(p.nx, p.ny, p.nz, p.na, p.nm, p.nt, float(np.float32(p.dx)),
                                float(np.float32(p.dy)), float(np.float32(p.dz)), p.dt, p.xbeg, p.ybeg, p.zbeg,
                                p.tbeg, threads)
        self._hold = []
        shape = (p.ny + 6, p.nx + 6, p.nz + 6)
        if medium is None:
            L = p.layers
            arr = lambda a: np.array([getattr(l, a) for l in L], np.float32)
            qp = np.zeros(shape, np.float32)
            qs = np.zeros(shape, np.float32)
            xi_c = None if xi is None else np.ascontiguousarray(xi, np.float32)
            lib.o3d_set_munk(self.o, int(getattr(p, "munk_profile", False)))
            lib.o3d_vmodel_lhm(self.o, len(L), _f(arr("depth")), _f(arr("rho")), _f(arr("vp")), _f(arr("vs")),
                               _f(arr("qp")), _f(arr("qs")), p.vcut, _f(xi_c), p.rhomin, _f(qp), _f(qs))
            lib.o3d_set_stabilize(self.o, int(getattr(p, "stabilize_pml", False)))
            lib.o3d_medium_setup(self.o, _f(qp), _f(qs), p.fq_min, p.fq_max, p.fq_ref)
        else:
            # externally prepared medium (e.g. to isolate the time step)
            m = medium
            lib.o3d_set_medium(self.o, _f(m.lam), _f(m.mu), _f(m.taup), _f(m.taus), _f(m.bx), _f(m.by),
                               _f(m.bz), _f(m.muyz), _f(m.muxz), _f(m.muxy), _f(m.ts))
            ip = lambda a: np.ascontiguousarray(a, np.int32).ctypes.data_as(_IP)
            lib.o3d_set_maps(self.o, ip(m.kfs), ip(m.kob), ip(m.kfs_top), ip(m.kfs_bot), ip(m.kob_top),
                             ip(m.kob_bot))
        if getattr(p, "bddep", None) is not None:
            bd = np.ascontiguousarray(p.bddep, np.float32)
            assert bd.shape == (p.ny + 6, p.nx + 6, NBD + 1)
            lib.o3d_set_bddep(self.o, _f(bd))
        lib.o3d_kernel_setup(self.o)
        # sources
        stf = STF[p.stftype]
        if getattr(p, "pw_mode", False):
            # pw_setup (m_source.f90:315-465) in place of a source grid
            lib.o3d_pw_setup(self.o, p.pw_ztop, p.pw_zlen, 0 if p.pw_ps.lower() == "p" else 1, p.pw_strike,
                             p.pw_dip, p.pw_rake, stf)
            self.nsrc = 0
        elif p.green_mode:
            self.nsrc = 0
        else:
            S = p.sources
            n = len(S)
            sx = np.array([s.x for s in S], np.float32)
            sy = np.array([s.y for s in S], np.float32)
            sz = np.array([s.z for s in S], np.float32)
            prm = np.array([[s.tbeg, s.trise] for s in S], np.float32).reshape(n, 2)
            mo = np.array([s.mo for s in S], np.float32)
            m6 = np.array([_moment6(lib, s) for s in S], np.float32).reshape(n, 6)
            f3 = np.array([[s.fx, s.fy, s.fz] for s in S], np.float32).reshape(n, 3)
            self._hold += [sx, sy, sz, prm, mo, m6, f3]
            lib.o3d_set_sdep_fit(self.o, _sdep(p))
            self.nsrc = lib.o3d_source_setup(self.o, int(p.bf_mode), n, _f(sx), _f(sy), _f(sz), _f(prm), _f(mo),
                                             _f(m6), _f(f3), stf)
            if self.nsrc < 0:
                raise ValueError("source depth outside the model after sdep_fit")
        sc = self.scalars()
        fcut = sc["fcut"] if not p.green_mode else float(np.float32(1.0) / np.float32(p.green_trise))
        if getattr(p, "abc_type", "pml") == "cerjan":
            # absorb__setup's dispatch (m_absorb.f90:25-41): the sponge, and
            # the kernel region over the whole domain
            lib.o3d_cerjan_setup(self.o)
        else:
            lib.o3d_absorb_setup(self.o, fcut)
        if profiles is not None:
            lib.o3d_set_profiles(self.o, *[_f(profiles[k]) for k in ("gxc", "gxe", "gyc", "gye", "gzc", "gze")])
        if p.green_mode:
            st = p.stations[p.green_station]
            from_ijk = self._station_cells([st])
            i, j, k = from_ijk[0][0], from_ijk[1][0], from_ijk[2][0]
            lib.o3d_green_setup(self.o, i, j, k, p.green_cmp.encode()[0:1], 0.0, p.green_trise, stf)
        self.nst = 0
        if p.stations and not p.green_mode and (p.sw_wav_v or p.sw_wav_u or p.sw_wav_stress or p.sw_wav_strain):
            S = p.stations
            xs = np.array([s.x for s in S], np.float32)
            ys = np.array([s.y for s in S], np.float32)
            zs = np.array([s.z for s in S], np.float32)
            zsw = np.array([ZSW.get(s.zsw, 0) for s in S], np.int32)
            ist = np.zeros(len(S), np.int32)
            jst = np.zeros(len(S), np.int32)
            kst = np.zeros(len(S), np.int32)
            ip = lambda a: a.ctypes.data_as(_IP)
            self.nst = lib.o3d_wav_setup(self.o, len(S), _f(xs), _f(ys), _f(zs), ip(zsw), p.ntdec_w,
                                         int(p.sw_wav_v), int(p.sw_wav_u), int(p.sw_wav_stress),
                                         int(p.sw_wav_strain), ip(ist), ip(jst), ip(kst))
            self.ist, self.jst, self.kst = ist[:self.nst], jst[:self.nst], kst[:self.nst]

    def _station_cells(self, stations):
        """set_stinfo for a station list (used for the green source cell)."""
        lib = self.lib
        p = self.p
        kfs = self.array("kfs")
        kob = self.array("kob")
        out = ([], [], [])
        for st in stations:
            i = lib.o3d_x2i(st.x, p.xbeg, p.dx)
            j = lib.o3d_x2i(st.y, p.ybeg, p.dy)
            k = lib.o3d_x2i(st.z, p.zbeg, p.dz)
            z = ZSW.get(st.zsw, 0)
            if z == 1:
                k = int(kfs[j + 2, i + 2]) + 1
            elif z == 2:
                k = int(kob[j + 2, i + 2]) + 1
            elif z == 3:
                k = int(kob[j + 2, i + 2]) - 1
            elif z >= 10:
                bd = self.bddep()
                k = lib.o3d_x2i(float(bd[j + 2, i + 2, z - 10]), p.zbeg, p.dz)
            out[0].append(i)
            out[1].append(j)
            out[2].append(k)
        return out

    def close(self):
        if self.o:
            self.lib.o3d_destroy(self.o)
            self.o = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- access -------------------------------------------------------------
    def dims(self) -> dict:
        a = (C.c_long * 17)()
        self.lib.o3d_dims(self.o, a)
        keys = ["nk", "ni", "nj", "nkk", "nik", "njk", "nka", "ibeg_k", "iend_k", "jbeg_k", "jend_k", "kbeg_k",
                "kend_k", "kbeg_min", "nst", "ntw", "nsrc"]
        return dict(zip(keys, list(a)))

    def scalars(self) -> dict:
        a = (C.c_float * 13)()
        self.lib.o3d_scalars(self.o, a)
        keys = ["M0", "UC", "fcut", "fmax", "vmin", "vmax", "zeta", "xend", "yend", "zend", "ts1", "ts2", "ts3"]
        return dict(zip(keys, list(a)))

    def array(self, name: str) -> np.ndarray:
        """Copy of an oracle array in the reference layout (numpy view order)."""
        d = self.dims()
        p = self.p
        fid = FIELD_IDS[name]
        ptr = self.lib.o3d_ptr(self.o, fid)
        if fid in range(0, 9):
            dt, shape = self.mpr, (d["nj"], d["ni"], d["nk"])
        elif fid in range(10, 16):
            dt, shape = self.spr, (d["njk"], d["nik"], d["nkk"], p.nm)
        elif fid in range(20, 30):
            dt, shape = self.spr, (d["nj"], d["ni"], d["nk"])
        elif fid in range(30, 41):
            dt, shape = np.float32, (d["nj"], d["ni"], d["nk"])
        elif fid in range(50, 57):
            dt, shape = np.int32, (d["nj"], d["ni"])
        elif fid == 57:
            dt, shape = np.float32, (d["nj"], d["ni"], NBD + 1)
        elif fid in range(60, 78):
            dt, shape = self.spr, (p.ny, p.nx, d["nka"])
        elif fid in range(110, 116):
            dt, shape = self.spr, ((p.nx, p.nx, p.ny, p.ny, p.nz, p.nz)[fid - 110],)
        else:
            raise KeyError(name)
        n = int(np.prod(shape))
        buf = (C.c_char * (n * np.dtype(dt).itemsize)).from_address(ptr)
        return np.frombuffer(buf, dtype=dt).reshape(shape).copy()

    def bddep(self) -> np.ndarray:
        """Boundary depths bddep(i, j, 0:NBD) of the memory box, shape (nj, ni, NBD + 1)."""
        return self.array("bddep")

    def green_store_setup(self, ig, jg, kg, bforce: bool = False, ntdec_w: int = 1):
        """green__store (m_green.f90:389-534) at the given grid cells; o3d_step
        then calls it beside wav__store."""
        ip = lambda a: np.ascontiguousarray(a, np.int32)
        self._green = (ip(ig), ip(jg), ip(kg), 9 if bforce else 6, (self.p.nt - 1) // ntdec_w + 1)
        g = self._green
        self.lib.o3d_green_store_setup(self.o, len(g[0]), *(a.ctypes.data_as(_IP) for a in g[:3]), int(bforce),
                                       ntdec_w)

    def green_functions(self) -> np.ndarray:
        """gf(ntw, ncmp*ng) as the reference holds it, returned as (ncmp*ng, ntw)."""
        ig, _, _, ncmp, ntw = self._green
        n = ncmp * len(ig) * ntw
        buf = (C.c_float * n).from_address(self.lib.o3d_ptr(self.o, 120))
        return np.frombuffer(buf, dtype=np.float32).reshape(ncmp * len(ig), ntw).copy()

    def waveforms(self, comp: str = "v") -> np.ndarray:
        d = self.dims()
        fid = {"v": 90, "u": 91, "stress": 92, "strain": 93}[comp]
        ncmp = 3 if comp in ("v", "u") else 6
        ptr = self.lib.o3d_ptr(self.o, fid)
        n = d["ntw"] * ncmp * d["nst"]
        if n == 0:
            return np.zeros((d["nst"], ncmp, d["ntw"]), np.float32)
        buf = (C.c_float * n).from_address(ptr)
        return np.frombuffer(buf, dtype=np.float32).reshape(d["nst"], ncmp, d["ntw"]).copy()

    def set_array(self, name: str, values: np.ndarray):
        """Overwrite an oracle field (V, S, R or PML auxiliary)."""
        cur = self.array(name)
        fid = FIELD_IDS[name]
        ptr = self.lib.o3d_ptr(self.o, fid)
        v = np.ascontiguousarray(values, cur.dtype).reshape(cur.shape)
        C.memmove(ptr, v.ctypes.data, v.nbytes)

    # -- snapshots (m_snap.f90) --------------------------------------------
    def snap_setup(self, planes: int, idec: int, jdec: int, kdec: int, ntdec_s: int, x0_yz: float, y0_xz: float,
                   z0_xy: float) -> int:
        """snap__setup for the planes whose bit (3*section + quantity) is set;
        sections yz xz xy fs ob, quantities ps v u.  Returns the frame count."""
        return self.lib.o3d_snap_setup(self.o, planes, idec, jdec, kdec, ntdec_s, x0_yz, y0_xz, z0_xy)

    def snap_dims(self) -> dict:
        out = np.zeros(7, np.int32)
        self.lib.o3d_snap_dims(self.o, out.ctypes.data_as(_IP))
        return dict(zip(("nxs", "nys", "nzs", "nframes", "i0_yz", "j0_xz", "k0_xy"), (int(v) for v in out)))

    def snap_frames(self, plane: int) -> np.ndarray:
        """(nframes, nvar, n2, n1) frames of one plane."""
        d = self.snap_dims()
        sec, q = divmod(plane, 3)
        nv = 4 if q == 0 else 3
        n1, n2 = {0: (d["nys"], d["nzs"]), 1: (d["nxs"], d["nzs"])}.get(sec, (d["nxs"], d["nys"]))
        ptr = self.lib.o3d_snap_frames(self.o, plane)
        n = d["nframes"] * nv * n1 * n2
        buf = (C.c_float * n).from_address(ptr)
        return np.frombuffer(buf, dtype=np.float32).reshape(d["nframes"], nv, n2, n1).copy()

    def snap_max(self, which: int) -> np.ndarray:
        """Running maxima (3, nys, nxs): 0 fs v, 1 fs u, 2 ob v, 3 ob u."""
        d = self.snap_dims()
        ptr = self.lib.o3d_snap_max(self.o, which)
        buf = (C.c_float * (3 * d["nxs"] * d["nys"])).from_address(ptr)
        return np.frombuffer(buf, dtype=np.float32).reshape(3, d["nys"], d["nxs"]).copy()

    def snap_write(self, it: int):
        self.lib.o3d_snap_write(self.o, it)

    # -- stepping -----------------------------------------------------------
    def step(self, it: int):
        self.lib.o3d_step(self.o, it)

    def vmax(self) -> np.ndarray:
        out = np.zeros(3, np.float32)
        self.lib.o3d_vmax(self.o, _f(out))
        return out

    def run(self, it0: int, nsteps: int, ntdec_r: int | None = None):
        reports = []
        sc = self.scalars()
        for it in range(it0, it0 + nsteps):
            if ntdec_r and it % ntdec_r == 0:
                reports.append((it, self.vmax() * np.float32(sc["UC"]) * np.float32(sc["M0"])))
            self.lib.o3d_step(self.o, it)
        return reports


def load2d(variant: str = "f32") -> C.CDLL:
    key = f"2d_{variant}"
    if key in _cache:
        return _cache[key]
    path = LIB / f"liboracle2d_{variant}.so"
    if not path.exists():
        import importlib.util
        spec = importlib.util.spec_from_file_location("build_oracle", HERE / "build_oracle.py")
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    lib = C.CDLL(str(path))
    vp, i, f, d = C.c_void_p, C.c_int, C.c_float, C.c_double
    sig = {
        "o2d_create": (vp, [i, i, i, i, i, i, d, d, f, f, f, f, i]),
        "o2d_destroy": (None, [vp]),
        "o2d_vmodel_lhm": (None, [vp, i, _FP, _FP, _FP, _FP, _FP, _FP, f, _FP, f, _FP, _FP]),
        "o2d_medium_setup": (None, [vp, _FP, _FP, f, f, f]),
        "o2d_kernel_setup": (None, [vp]),
        "o2d_absorb_setup": (None, [vp, f]),
        "o2d_cerjan_setup": (None, [vp]),
        "o2d_set_stabilize": (None, [vp, i]),
        "o2d_set_bddep": (None, [vp, _FP]),
        "o2d_set_munk": (None, [vp, i]),
        "o2d_set_sdep_fit": (None, [vp, i]),
        "o2d_source_setup": (i, [vp, i, i, _FP, _FP, _FP, _FP, _FP, _FP, i]),
        "o2d_wav_setup": (i, [vp, i, _FP, _FP, _IP, i, i, i]),
        "o2d_step": (None, [vp, i]),
        "o2d_vmax": (None, [vp, _FP]),
        "o2d_dims": (None, [vp, C.POINTER(C.c_long)]),
        "o2d_scalars": (None, [vp, _FP]),
        "o2d_ptr": (vp, [vp, i]),
        "o2d_mpr_size": (i, []),
        "o2d_spr_size": (i, []),
        "o2d_visco_chi": (f, [i, _FP, f, f]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _cache[key] = lib
    return lib


class Oracle2D:
    """The reference P-SV (kind 'psv') or SH ('sh') run restated on the CPU."""

    KIND = {"psv": 2, "sh": 1}

    def __init__(self, p, kind: str = "psv", variant: str = "f32", threads: int = 1):
        self.p, self.kind = p, kind
        self.lib = lib = load2d(variant)
        self.mpr = np.float32 if lib.o2d_mpr_size() == 4 else np.float64
        self.spr = np.float32 if lib.o2d_spr_size() == 4 else np.float64
        self.o = lib.o2d_create(self.KIND[kind], p.nx, p.nz, p.na, p.nm, p.nt, float(np.float32(p.dx)),
                                float(np.float32(p.dz)), p.dt, p.xbeg, p.zbeg, p.tbeg, threads)
        shape = (p.nx + 6, p.nz + 6)
        L = p.layers
        arr = lambda a: np.array([getattr(l, a) for l in L], np.float32)
        qp = np.zeros(shape, np.float32)
        qs = np.zeros(shape, np.float32)
        lib.o2d_set_munk(self.o, int(getattr(p, "munk_profile", False)))
        lib.o2d_vmodel_lhm(self.o, len(L), _f(arr("depth")), _f(arr("rho")), _f(arr("vp")), _f(arr("vs")),
                           _f(arr("qp")), _f(arr("qs")), p.vcut, None, p.rhomin, _f(qp), _f(qs))
        lib.o2d_set_stabilize(self.o, int(getattr(p, "stabilize_pml", False)))
        lib.o2d_medium_setup(self.o, _f(qp), _f(qs), p.fq_min, p.fq_max, p.fq_ref)
        lib.o2d_kernel_setup(self.o)
        S = p.sources
        n = len(S)
        sx = np.array([s.x for s in S], np.float32)
        sz = np.array([s.z for s in S], np.float32)
        prm = np.array([[s.tbeg, s.trise] for s in S], np.float32).reshape(n, 2)
        mo = np.array([s.mo for s in S], np.float32)
        m6 = np.array([_moment6(load(variant, "3d"), s) for s in S], np.float32).reshape(n, 6)
        f3 = np.array([[s.fx, s.fy, s.fz] for s in S], np.float32).reshape(n, 3)
        self._hold = [sx, sz, prm, mo, m6, f3]
        if getattr(p, "bddep", None) is not None:
            bd = np.ascontiguousarray(p.bddep, np.float32)
            assert bd.shape == (p.nx + 6, NBD + 1)
            lib.o2d_set_bddep(self.o, _f(bd))
        lib.o2d_set_sdep_fit(self.o, _sdep(p))
        self.nsrc = lib.o2d_source_setup(self.o, int(p.bf_mode), n, _f(sx), _f(sz), _f(prm), _f(mo), _f(m6), _f(f3),
                                         STF[p.stftype])
        if self.nsrc < 0:
            raise ValueError("source depth outside the model after sdep_fit")
        if getattr(p, "abc_type", "pml") == "cerjan":
            lib.o2d_cerjan_setup(self.o)
        else:
            lib.o2d_absorb_setup(self.o, self.scalars()["fcut"])
        self.nst = 0
        if p.stations and (p.sw_wav_v or p.sw_wav_u):
            St = p.stations
            xs = np.array([s.x for s in St], np.float32)
            zs = np.array([s.z for s in St], np.float32)
            zsw = np.array([ZSW.get(s.zsw, 0) for s in St], np.int32)
            self.nst = lib.o2d_wav_setup(self.o, len(St), _f(xs), _f(zs), zsw.ctypes.data_as(_IP), p.ntdec_w,
                                         int(p.sw_wav_v), int(p.sw_wav_u))

    def close(self):
        if self.o:
            self.lib.o2d_destroy(self.o)
            self.o = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def dims(self) -> dict:
        a = (C.c_long * 10)()
        self.lib.o2d_dims(self.o, a)
        return dict(zip(["nk", "ni", "nka", "kbeg_min", "nst", "ntw", "nsrc", "ibeg_k", "iend_k", "kend_k"], list(a)))

    def scalars(self) -> dict:
        a = (C.c_float * 9)()
        self.lib.o2d_scalars(self.o, a)
        return dict(zip(["M0", "UC", "fcut", "vmin", "vmax", "zeta", "ts1", "ts2", "ts3"], list(a)))

    # names -> (id, kind of storage)
    def _spec(self, name: str):
        psv = self.kind == "psv"
        ids = ({"Vx": 0, "Vz": 1, "Sxx": 2, "Szz": 3, "Sxz": 4, "Rxx": 10, "Rzz": 11, "Rxz": 12} if psv else
               {"Vy": 0, "Syz": 2, "Sxy": 3, "Ryz": 10, "Rxy": 11})
        ids.update({"rho": 20, "lam": 21, "mu": 22, "taup": 23, "taus": 24, "frho": 30, "flam": 31, "fmu": 32,
                    "ftaup": 33, "ftaus": 34, "kfs": 50, "kob": 51, "kfs_top": 52, "kfs_bot": 53, "kob_top": 54,
                    "kob_bot": 55, "kbeg_a": 56})
        aux = (["axVx", "azVx", "axVz", "azVz", "axSxx", "azSxz", "axSxz", "azSzz"] if psv else
               ["axVy", "azVy", "axSxy", "azSyz"])
        for n, a in enumerate(aux):
            ids[a] = 60 + n
        ids.update({"gx_c": 110, "gx_b": 111, "gz_c": 114, "gz_b": 115})
        return ids[name]

    def array(self, name: str) -> np.ndarray:
        d = self.dims()
        p = self.p
        fid = self._spec(name)
        ptr = self.lib.o2d_ptr(self.o, fid)
        if fid < 10:
            dt, shape = self.mpr, (d["ni"], d["nk"])
        elif fid < 20:
            dt, shape = self.spr, (d["ni"], d["nk"], max(p.nm, 1))
        elif fid < 30:
            dt, shape = self.spr, (d["ni"], d["nk"])
        elif fid < 50:
            dt, shape = np.float32, (d["ni"], d["nk"])
        elif fid < 60:
            dt, shape = np.int32, (d["ni"],)
        elif fid >= 110:
            dt, shape = self.spr, (p.nx if fid < 114 else p.nz,)
        else:
            dt, shape = self.spr, (p.nx, d["nka"])
        n = int(np.prod(shape))
        buf = (C.c_char * (n * np.dtype(dt).itemsize)).from_address(ptr)
        return np.frombuffer(buf, dtype=dt).reshape(shape).copy()

    def waveforms(self, comp: str = "v") -> np.ndarray:
        d = self.dims()
        nc = 2 if self.kind == "psv" else 1
        ptr = self.lib.o2d_ptr(self.o, 90 if comp == "v" else 91)
        n = d["ntw"] * nc * d["nst"]
        if n == 0:
            return np.zeros((d["nst"], nc, d["ntw"]), np.float32)
        buf = (C.c_float * n).from_address(ptr)
        return np.frombuffer(buf, dtype=np.float32).reshape(d["nst"], nc, d["ntw"]).copy()

    def step(self, it: int):
        self.lib.o2d_step(self.o, it)

    def run(self, it0: int, nsteps: int):
        for it in range(it0, it0 + nsteps):
            self.lib.o2d_step(self.o, it)

    def vmax(self) -> np.ndarray:
        out = np.zeros(2, np.float32)
        self.lib.o2d_vmax(self.o, _f(out))
        return out
