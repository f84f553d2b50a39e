"""Host driver of the 2D solvers (src/swpc_psv/main.f90, src/swpc_sh/main.f90)
and of the batched 2D ensemble.

`Swpc2D` runs the reference's 2D setup sequence (global__setup2,
medium__setup, kernel__setup, source__setup, absorb__setup, wav__setup) with
the library's host routines and exposes the time-loop routines under their
module names.  Arrays use the 2D memory box ``(kbeg_m:kend_m, ibeg_m:iend_m)``
with k fastest: a numpy array of shape ``(nx+6, nz+6)`` indexed
``[i+2, k+2]``.

`Batch2D` joins many set-up 2D runs (same kind and nm) into one persistent
launch per half step, replayed as a CUDA graph (swpc_batch_*).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, fptr, iptr
from .params import Params, bddep_of, sdep_index, zsw_code
from .swpc3d import SourceGrid, _sdr2moment

f32 = np.float32
KINDS = {"psv": _lib.KIND_PSV, "sh": _lib.KIND_SH}


def grid2d(p: Params) -> _lib.Grid:
    return _lib.Grid(p.nx, 1, p.nz, p.na, p.nm, p.dx, p.dx, p.dz, p.dt, p.xbeg, 0.0, p.zbeg, p.tbeg)


def source_grid2d(p: Params, kind: str = "psv") -> SourceGrid:
    """source__setup of the 2D codes (src/swpc_psv/m_source.f90:150-268,
    src/swpc_sh/m_source.f90): cut-off frequency, total moment (P-SV body
    forces: sqrt(sum fx^2 + fz^2); SH: |sum fy|), grid assignment with the
    node sleeve, sdep_fit, normalisation by M0.  ``jsrc`` is all zeros."""
    lib = _lib.load()
    srcs = p.sources
    fcut = f32(0.0)
    for s in srcs:
        fcut = max(fcut, f32(1) / f32(s.trise))
    UC = f32(1e-15)
    if p.bf_mode:
        acc = f32(0.0)
        if kind == "psv":
            for s in srcs:
                acc = acc + (f32(s.fx) * f32(s.fx) + f32(s.fz) * f32(s.fz))
            M0 = np.sqrt(acc, dtype=np.float32)
        else:
            for s in srcs:
                acc = acc + f32(s.fy)
            M0 = np.sqrt(acc * acc, dtype=np.float32)
        UC = UC * f32(1000)
    else:
        M0 = f32(0.0)
        for s in srcs:
            M0 = M0 + f32(s.mo)
    nbd = sdep_index(p)
    bd = bddep_of(p, two_d=True) if nbd >= 0 else None
    zend = f32(p.zbeg) + f32(p.nz) * f32(p.dz)
    rows = []
    for s in srcs:
        i = lib.swpc_x2i(s.x, p.xbeg, p.dx)
        k = lib.swpc_x2i(s.z, p.zbeg, p.dz)
        if -1 <= i <= p.nx + 3 and -1 <= k <= p.nz + 3:
            if bd is not None:
                # sdep_fit = 'bd<n>' (src/swpc_psv/m_source.f90:227-236, inside FDM space :242-245)
                sz = bd[i + 2, nbd]
                k = lib.swpc_x2i(float(sz), p.zbeg, p.dz)
                if not (f32(p.zbeg) <= sz <= zend):
                    raise ValueError(f"sdep_fit={p.sdep_fit}: source depth {float(sz)} outside the model")
            rows.append((i, k, s))
    n = len(rows)
    isrc = np.array([r[0] for r in rows], np.int32)
    ksrc = np.array([r[1] for r in rows], np.int32)
    prm = np.array([[r[2].tbeg, r[2].trise] for r in rows], np.float32).reshape(n, 2)
    if p.bf_mode:
        f3 = np.array([[f32(r[2].fx) / M0, f32(r[2].fy) / M0, f32(r[2].fz) / M0] for r in rows],
                      np.float32).reshape(n, 3)
        mo = np.zeros(n, np.float32)
    else:
        f3 = np.zeros((n, 3), np.float32)
        mo = np.array([f32(r[2].mo) / M0 for r in rows], np.float32)
    sdr = _sdr2moment(lib)
    m6 = np.array([r[2].moment(sdr) for r in rows], np.float32).reshape(n, 6)
    return SourceGrid(isrc, np.zeros(n, np.int32), ksrc, prm, mo, m6, f3, float(M0), float(UC), float(fcut))


def station_grid2d(p: Params, kfs: np.ndarray, kob: np.ndarray):
    """set_stinfo of the 2D codes (src/swpc_psv/m_wav.f90:480-540): station
    cells (ist, kst) with depth modes dep / fsb / obb / oba / bd0-bd9; kfs
    and kob are (nx+6,) maps."""
    lib = _lib.load()
    x1, xn = lib.swpc_i2x(1, p.xbeg, p.dx), lib.swpc_i2x(p.nx, p.xbeg, p.dx)
    cells = []
    bd = None
    for st in p.stations:
        xs, zs = float(f32(st.x)), float(f32(st.z))
        i = lib.swpc_x2i(xs, p.xbeg, p.dx)
        k = lib.swpc_x2i(zs, p.zbeg, p.dz)
        if not (x1 < xs < xn and 1 < k < p.nz and 1 <= i <= p.nx):
            continue
        z = zsw_code(st.zsw, st.name)
        if z == 1:
            k = int(kfs[i + 2]) + 1
        elif z == 2:
            k = int(kob[i + 2]) + 1
        elif z == 3:
            k = int(kob[i + 2]) - 1
        elif z >= 10:
            # bd0-bd9 (src/swpc_psv/m_wav.f90:511-520)
            if bd is None:
                bd = bddep_of(p, two_d=True)
            k = lib.swpc_x2i(float(bd[i + 2, z - 10]), p.zbeg, p.dz)
        k = p.nz - 1 if k > p.nz else (2 if k < 1 else k)
        cells.append((i, k))
    a = np.array(cells, np.int32).reshape(-1, 2)
    return a[:, 0].copy(), a[:, 1].copy()


class Medium2D:
    """Host copy of the 2D medium after medium__setup."""

    FIELDS = ("rho", "lam", "mu", "taup", "taus")
    MAPS = ("kfs", "kob", "kfs_top", "kfs_bot", "kob_top", "kob_bot", "kbeg_a")

    def __init__(self, p: Params):
        lib = _lib.load()
        g = grid2d(p)
        shape = (p.nx + 6, p.nz + 6)
        for name in self.FIELDS:
            setattr(self, name, np.zeros(shape, np.float32))
        self.qp = np.zeros(shape, np.float32)
        self.qs = np.zeros(shape, np.float32)
        for name in self.MAPS:
            setattr(self, name, np.zeros(p.nx + 6, np.int32))
        L = p.layers
        arr = lambda a: np.array([getattr(l, a) for l in L], np.float32)
        rc = lib.swpc_vmodel_lhm_opt(C.byref(g), len(L), fptr(arr("depth")), fptr(arr("rho")), fptr(arr("vp")),
                                 fptr(arr("vs")), fptr(arr("qp")), fptr(arr("qs")), p.vcut, None, p.rhomin,
                                 fptr(self.rho), fptr(self.lam), fptr(self.mu), fptr(self.qp), fptr(self.qs),
                                     int(p.munk_profile))
        if rc:
            raise ValueError("vmodel_lhm failed")
        self.ts = np.zeros(3, np.float32)
        scal = np.zeros(3, np.float32)
        rc = lib.swpc_setup_medium_2d_opt(C.byref(g), p.fq_min, p.fq_max, p.fq_ref, fptr(self.rho), fptr(self.lam),
                                          fptr(self.mu), fptr(self.qp), fptr(self.qs), fptr(self.taup),
                                          fptr(self.taus), iptr(self.kfs), iptr(self.kob), iptr(self.kfs_top),
                                          iptr(self.kfs_bot), iptr(self.kob_top), iptr(self.kob_bot),
                                          fptr(self.ts), fptr(scal), int(p.stabilize_pml))
        if rc:
            raise ValueError("2D medium setup failed")
        self.zeta, self.vmin, self.vmax = (float(x) for x in scal)
        lib.swpc_kbeg_a(C.byref(g), iptr(self.kbeg_a))

    def view(self) -> _lib.MediumView:
        v = _lib.MediumView()
        for name in self.FIELDS:
            setattr(v, name, fptr(getattr(self, name)))
        for name in self.MAPS:
            setattr(v, name, iptr(getattr(self, name)))
        v.ld_k = self.rho.shape[1]
        v.ld_i = self.rho.shape[0]
        v.ld_i2 = self.kfs.shape[0]
        return v


class Swpc2D:
    """One 2D run (kind 'psv' or 'sh') on one GPU."""

    def __init__(self, p: Params, kind: str = "psv", device: int = 0):
        p.check()
        self.p, self.kind = p, kind
        lib = self.lib = _lib.load()
        m = self.medium = Medium2D(p)
        desc = _lib.Desc(KINDS[kind], p.nx, 1, p.nz, p.na, p.nm, p.nt, p.dx, p.dx, p.dz, p.dt, p.tbeg, device)
        ctx = C.c_void_p()
        rc = lib.swpc_create(C.byref(desc), C.byref(ctx))
        self.ctx = ctx
        if rc:
            msg = lib.swpc_last_error(ctx) if ctx else b""
            lib.swpc_destroy(ctx)
            self.ctx = None
            raise _lib.SwpcError(rc, msg.decode() if msg else "swpc_create failed")
        check(ctx, lib.swpc_upload_medium(ctx, C.byref(m.view())))
        check(ctx, lib.swpc_kernel_setup(ctx, fptr(m.ts)))
        # source__setup of the 2D codes (src/swpc_psv/m_source.f90:150-268)
        sg = source_grid2d(p, kind)
        M0, UC, fcut = sg.M0, sg.UC, sg.fcut
        n = len(sg.isrc)
        stf = _lib.STF_CODES[p.stftype]
        if p.bf_mode:
            check(ctx, lib.swpc_bodyforce_setup(ctx, n, iptr(sg.isrc), None, iptr(sg.ksrc), fptr(sg.srcprm),
                                                fptr(sg.f3), stf))
        else:
            check(ctx, lib.swpc_source_setup(ctx, n, iptr(sg.isrc), None, iptr(sg.ksrc), fptr(sg.srcprm),
                                             fptr(sg.mo), fptr(sg.m6), stf))
        self.M0, self.UC, self.fcut = float(M0), float(UC), float(fcut)
        g = grid2d(p)
        if p.abc_type == "cerjan":
            # absorb_c__setup (src/swpc_psv/m_absorb_c.f90, src/swpc_sh/m_absorb_c.f90)
            self.cprof = {k: np.zeros(p.nx if k[1] == "x" else p.nz, np.float32) for k in ("gx_c", "gx_b", "gz_c",
                                                                                          "gz_b")}
            cp = self.cprof
            lib.swpc_cerjan_profiles(C.byref(g), fptr(cp["gx_c"]), fptr(cp["gx_b"]), None, None, fptr(cp["gz_c"]),
                                     fptr(cp["gz_b"]))
            check(ctx, lib.swpc_absorb_setup_cerjan(ctx, fptr(cp["gx_c"]), fptr(cp["gx_b"]), None, None,
                                                    fptr(cp["gz_c"]), fptr(cp["gz_b"])))
        else:
            self.gprof = {k: np.zeros((p.nx if k[1] == "x" else p.nz, 4), np.float32)
                          for k in ("gxc", "gxe", "gzc", "gze")}
            gp = self.gprof
            lib.swpc_damping_profiles(C.byref(g), float(f32(self.fcut)), fptr(gp["gxc"]), fptr(gp["gxe"]), None,
                                      None, fptr(gp["gzc"]), fptr(gp["gze"]))
            check(ctx, lib.swpc_absorb_setup(ctx, fptr(gp["gxc"]), fptr(gp["gxe"]), None, None, fptr(gp["gzc"]),
                                             fptr(gp["gze"])))
        # wav__setup / set_stinfo (src/swpc_psv/m_wav.f90:480-540)
        self.nst = 0
        what = (_lib.WAV_V * p.sw_wav_v) | (_lib.WAV_U * p.sw_wav_u)
        if p.stations and what:
            self.ist, self.kst = station_grid2d(p, m.kfs, m.kob)
            self.nst = len(self.ist)
            check(ctx, lib.swpc_wav_setup(ctx, self.nst, iptr(self.ist), None, iptr(self.kst), p.ntdec_w, what,
                                          self.M0, self.UC))
        self.what = what

    def close(self):
        if self.ctx:
            self.lib.swpc_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, it: int):
        check(self.ctx, self.lib.swpc_step(self.ctx, it))

    def run(self, it0: int = 1, nsteps: int | None = None):
        if nsteps is None:
            nsteps = self.p.nt - it0 + 1
        check(self.ctx, self.lib.swpc_run(self.ctx, it0, nsteps))
        check(self.ctx, self.lib.swpc_sync(self.ctx))

    def kernel__vmax(self) -> np.ndarray:
        out = np.zeros(3, np.float32)
        check(self.ctx, self.lib.swpc_vmax(self.ctx, fptr(out)))
        return out[:2] if self.kind == "psv" else out[:1]

    def download(self, field: int) -> np.ndarray:
        p = self.p
        out = np.zeros((p.nx + 6, p.nz + 6), np.float32)
        check(self.ctx, self.lib.swpc_download_field(self.ctx, field, fptr(out), p.nz + 6, p.nx + 6))
        return out

    def upload(self, field: int, arr: np.ndarray):
        p = self.p
        a = np.ascontiguousarray(arr, np.float32)
        check(self.ctx, self.lib.swpc_upload_field(self.ctx, field, fptr(a), p.nz + 6, p.nx + 6))

    def waveforms(self, what: int = _lib.WAV_V) -> np.ndarray:
        ntw, nst = C.c_int(), C.c_int()
        check(self.ctx, self.lib.swpc_wav_dims(self.ctx, C.byref(ntw), C.byref(nst)))
        nc = 2 if self.kind == "psv" else 1
        out = np.zeros((nst.value, nc, ntw.value), np.float32)
        if nst.value:
            check(self.ctx, self.lib.swpc_wav_fetch(self.ctx, what, fptr(out)))
        return out

    # field ids of this kind
    @property
    def field_ids(self) -> dict:
        if self.kind == "psv":
            return {"Vx": _lib.F_VX, "Vz": _lib.F_VZ, "Sxx": _lib.F_SXX, "Szz": _lib.F_SZZ, "Sxz": _lib.F_SXZ}
        return {"Vy": _lib.F_VY, "Syz": _lib.F_SYZ, "Sxy": _lib.F_SXY}


class Batch2D:
    """Many 2D runs advanced by one persistent launch per half step."""

    def __init__(self, runs: list[Swpc2D]):
        self.runs = runs
        self.lib = _lib.load()
        arr = (C.c_void_p * len(runs))(*[r.ctx.value for r in runs])
        b = C.c_void_p()
        rc = self.lib.swpc_batch_create(arr, len(runs), C.byref(b))
        self.b = b
        if rc:
            msg = self.lib.swpc_batch_last_error(b) if b else b""
            raise _lib.SwpcError(rc, msg.decode() if msg else "swpc_batch_create failed")

    def _check(self, rc):
        if rc:
            raise _lib.SwpcError(rc, self.lib.swpc_batch_last_error(self.b).decode())

    def run(self, it0: int, nsteps: int):
        self._check(self.lib.swpc_batch_run(self.b, it0, nsteps))
        self._check(self.lib.swpc_batch_sync(self.b))

    def step(self, it: int):
        self._check(self.lib.swpc_batch_step(self.b, it))
        self._check(self.lib.swpc_batch_sync(self.b))

    def time_steps(self, it0: int, nsteps: int) -> float:
        ms = C.c_float()
        self._check(self.lib.swpc_batch_time_steps(self.b, it0, nsteps, C.byref(ms)))
        return ms.value

    def set_staged(self, stress_ti: int, vel_ti: int):
        """TMA-staged kernels with stress_ti / vel_ti threads along i (4, 8,
        16), or the tile-walking kernels (0), per phase."""
        self._check(self.lib.swpc_batch_set_staged(self.b, stress_ti, vel_ti))

    def set_shape(self, ti: int, ri: int, bps: int):
        """Tile shape of the tile-walking kernels (ti * ri != 16 also selects
        them for both phases)."""
        self._check(self.lib.swpc_batch_set_shape(self.b, ti, ri, bps))

    def launch(self) -> dict:
        """The current launch: tile shape and staged threads per phase."""
        out = (C.c_int * 5)()
        self._check(self.lib.swpc_batch_get_launch(self.b, out))
        return {"ti": out[0], "ri": out[1], "bps": out[2], "stress_ti": out[3], "vel_ti": out[4]}

    def autotune(self, it0: int, reps: int = 2) -> tuple[int, int, int, int]:
        """Pick the launch while advancing steps it0 ..; returns (steps used,
        threads in i per block, rows per thread, blocks per SM) of the tile
        shape (launch() gives the whole pick)."""
        used, ti, ri, bps = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        self._check(self.lib.swpc_batch_autotune(self.b, it0, reps, C.byref(used), C.byref(ti), C.byref(ri),
                                                 C.byref(bps)))
        self._check(self.lib.swpc_batch_sync(self.b))
        return used.value, ti.value, ri.value, bps.value

    def close(self):
        if self.b:
            self.lib.swpc_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
