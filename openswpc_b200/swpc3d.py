"""Host driver of the 3D solver: the role of src/swpc_3d/main.f90.

`Swpc3D` performs the reference's setup sequence (main.f90:64-78:
global__setup2, medium__setup, kernel__setup, source__setup, absorb__setup,
wav__setup, green__setup) with the library's host setup routines, uploads
everything once, and then exposes the time-loop routines under the
reference's module names.  `run()` replays the loop of main.f90:125-144 as
CUDA-graph launches with report__progress (vmax + divergence abort) every
``ntdec_r`` steps.

Arrays exchanged with the caller use the reference memory-box layout
``(kbeg_m:kend_m, ibeg_m:iend_m, jbeg_m:jend_m)`` with k fastest; in numpy
that is a C-ordered array of shape ``(ny+6, nx+6, nz+6)`` indexed
``[j+2, i+2, k+2]``.
"""
from __future__ import annotations

import ctypes as C
import weakref
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check, fptr, iptr
from .params import Params, bddep_of, sdep_index, zsw_code

f32 = np.float32


@dataclass
class SourceGrid:
    """Result of source__setup (m_source.f90:181-305) for one node."""

    isrc: np.ndarray
    jsrc: np.ndarray
    ksrc: np.ndarray
    srcprm: np.ndarray   # (nsrc, 2) = (tbeg, trise)
    mo: np.ndarray       # normalised by M0
    m6: np.ndarray       # (nsrc, 6) xx yy zz yz xz xy
    f3: np.ndarray       # (nsrc, 3) normalised by M0
    M0: float
    UC: float
    fcut: float


def grid_struct(p: Params) -> _lib.Grid:
    return _lib.Grid(p.nx, p.ny, p.nz, p.na, p.nm, p.dx, p.dy, p.dz, p.dt, p.xbeg, p.ybeg, p.zbeg, p.tbeg)


def _sdr2moment(lib):
    """The library's sdr2moment (m_fdtool.f90:307-336) as a Python callable."""
    def f(strike, dip, rake):
        m6 = (C.c_float * 6)()
        lib.swpc_sdr2moment(strike, dip, rake, m6)
        return tuple(m6)
    return f


def source_grid(p: Params) -> SourceGrid:
    """source__setup (m_source.f90:181-305): cut-off frequency, total moment,
    grid assignment with the node sleeve, sdep_fit, normalisation by M0.
    Double couples get their moment tensor from sdr2moment here."""
    lib = _lib.load()
    srcs = p.sources
    fcut = f32(0.0)
    for s in srcs:
        fcut = max(fcut, f32(1) / f32(s.trise))
    UC = f32(1e-15)
    if p.bf_mode:
        acc = f32(0.0)
        for s in srcs:
            acc = acc + (f32(s.fx) * f32(s.fx) + f32(s.fy) * f32(s.fy) + f32(s.fz) * f32(s.fz))
        M0 = np.sqrt(acc, dtype=np.float32)
        UC = UC * f32(1000)
    else:
        M0 = f32(0.0)
        for s in srcs:
            M0 = M0 + f32(s.mo)
    nbd = sdep_index(p)
    bd = bddep_of(p) if nbd >= 0 else None
    zend = f32(p.zbeg) + f32(p.nz) * f32(p.dz)
    rows = []
    for s in srcs:
        i = lib.swpc_x2i(s.x, p.xbeg, p.dx)
        j = lib.swpc_x2i(s.y, p.ybeg, p.dy)
        k = lib.swpc_x2i(s.z, p.zbeg, p.dz)
        if -1 <= i <= p.nx + 3 and -1 <= j <= p.ny + 3 and -1 <= k <= p.nz + 3:
            if bd is not None:
                # sdep_fit = 'bd<n>' (m_source.f90:262-270); FDM space must contain the depth (:276-280)
                sz = bd[j + 2, i + 2, nbd]
                k = lib.swpc_x2i(float(sz), p.zbeg, p.dz)
                if not (f32(p.zbeg) <= sz <= zend):
                    raise ValueError(f"sdep_fit={p.sdep_fit}: source depth {float(sz)} outside the model")
            rows.append((i, j, k, s))
    n = len(rows)
    isrc = np.array([r[0] for r in rows], np.int32)
    jsrc = np.array([r[1] for r in rows], np.int32)
    ksrc = np.array([r[2] for r in rows], np.int32)
    srcprm = np.array([[r[3].tbeg, r[3].trise] for r in rows], np.float32).reshape(n, 2)
    if p.bf_mode:
        f3 = np.array([[f32(r[3].fx) / M0, f32(r[3].fy) / M0, f32(r[3].fz) / M0] for r in rows], np.float32)
        mo = np.zeros(n, np.float32)
    else:
        f3 = np.zeros((n, 3), np.float32)
        mo = np.array([f32(r[3].mo) / M0 for r in rows], np.float32)
    sdr = _sdr2moment(lib)
    m6 = np.array([r[3].moment(sdr) for r in rows], np.float32).reshape(n, 6)
    return SourceGrid(isrc, jsrc, ksrc, srcprm, mo, m6, f3.reshape(n, 3), float(M0), float(UC), float(fcut))


def station_grid(p: Params, kfs: np.ndarray, kob: np.ndarray):
    """set_stinfo (m_wav.f90:144-274) for a single node: station cells and
    depth mode (dep / fsb / obb / oba / bd0-bd9).  kfs/kob are (ny+6, nx+6)
    maps; the boundary depths come from ``p.bddep`` or vmodel_lhm's rule."""
    lib = _lib.load()
    out = []
    x1, xn = lib.swpc_i2x(1, p.xbeg, p.dx), lib.swpc_i2x(p.nx, p.xbeg, p.dx)
    y1, yn = lib.swpc_i2x(1, p.ybeg, p.dy), lib.swpc_i2x(p.ny, p.ybeg, p.dy)
    bd = None
    for st in p.stations:
        xs, ys, zs = float(f32(st.x)), float(f32(st.y)), float(f32(st.z))
        i = lib.swpc_x2i(xs, p.xbeg, p.dx)
        j = lib.swpc_x2i(ys, p.ybeg, p.dy)
        k = lib.swpc_x2i(zs, p.zbeg, p.dz)
        if not (x1 < xs < xn and y1 < ys < yn and 1 < k < p.nz):
            continue
        if not (1 <= i <= p.nx and 1 <= j <= p.ny):
            continue
        z = zsw_code(st.zsw, st.name)
        if z == 1:
            k = int(kfs[j + 2, i + 2]) + 1
        elif z == 2:
            k = int(kob[j + 2, i + 2]) + 1
        elif z == 3:
            k = int(kob[j + 2, i + 2]) - 1
        elif z >= 10:
            if bd is None:
                bd = bddep_of(p)
            k = lib.swpc_x2i(float(bd[j + 2, i + 2, z - 10]), p.zbeg, p.dz)
        else:
            k = lib.swpc_x2i(zs, p.zbeg, p.dz)
        if k > p.nz:
            k = p.nz - 1
        if k < 1:
            k = 2
        out.append((i, j, k))
    a = np.array(out, np.int32).reshape(-1, 3)
    return a[:, 0].copy(), a[:, 1].copy(), a[:, 2].copy()


def lhm_model(p: Params, xi: np.ndarray | None = None):
    """Per-cell (vp, vs, rho, qp, qs) of the layered model, with the lhm_rmed
    perturbation when ``xi`` is given, over the memory box (vmodel_lhm,
    m_vmodel_lhm.f90:21-169).  The velocities are recovered from the moduli
    the vmodel forms (vs = sqrt(mu/rho), vp = sqrt((lam+2mu)/rho))."""
    lib = _lib.load()
    g = grid_struct(p)
    shape = (p.ny + 6, p.nx + 6, p.nz + 6)
    rho, lam, mu, qp, qs = (np.zeros(shape, np.float32) for _ in range(5))
    L = p.layers
    arr = lambda attr: np.array([getattr(l, attr) for l in L], np.float32)
    if xi is not None:
        xi = np.ascontiguousarray(xi, np.float32)
    rc = lib.swpc_vmodel_lhm_opt(C.byref(g), len(L), fptr(arr("depth")), fptr(arr("rho")), fptr(arr("vp")),
                             fptr(arr("vs")), fptr(arr("qp")), fptr(arr("qs")), p.vcut, fptr(xi), p.rhomin,
                             fptr(rho), fptr(lam), fptr(mu), fptr(qp), fptr(qs), int(p.munk_profile))
    if rc:
        raise ValueError("vmodel_lhm failed")
    vs = np.sqrt(mu / rho).astype(np.float32)
    vp = np.sqrt((lam + 2 * mu) / rho).astype(np.float32)
    return vp, vs, rho, qp, qs


class Medium:
    """Host copy of the medium after medium__setup (m_medium.f90:36-467)."""

    FIELDS = ("rho", "lam", "mu", "taup", "taus", "bx", "by", "bz", "muyz", "muxz", "muxy")
    MAPS = ("kfs", "kob", "kfs_top", "kfs_bot", "kob_top", "kob_bot", "kbeg_a")

    def __init__(self, p: Params, xi: np.ndarray | None = None):
        lib = _lib.load()
        g = grid_struct(p)
        shape = (p.ny + 6, p.nx + 6, p.nz + 6)
        for name in self.FIELDS:
            setattr(self, name, np.zeros(shape, np.float32))
        self.qp = np.zeros(shape, np.float32)
        self.qs = np.zeros(shape, np.float32)
        for name in self.MAPS:
            setattr(self, name, np.zeros(shape[:2], np.int32))
        if not p.layers:
            raise ValueError("a layered (lhm) velocity model is required")
        L = p.layers
        arr = lambda attr: np.array([getattr(l, attr) for l in L], np.float32)
        if xi is not None:
            xi = np.ascontiguousarray(xi, np.float32)
            assert xi.shape == shape
        rc = lib.swpc_vmodel_lhm_opt(C.byref(g), len(L), fptr(arr("depth")), fptr(arr("rho")), fptr(arr("vp")),
                                 fptr(arr("vs")), fptr(arr("qp")), fptr(arr("qs")), p.vcut, fptr(xi), p.rhomin,
                                 fptr(self.rho), fptr(self.lam), fptr(self.mu), fptr(self.qp), fptr(self.qs),
                                     int(p.munk_profile))
        if rc:
            raise ValueError("vmodel_lhm failed")
        self._setup(p)

    @classmethod
    def from_model(cls, p: Params, vp: np.ndarray, vs: np.ndarray, rho: np.ndarray, qp: np.ndarray,
                   qs: np.ndarray) -> "Medium":
        """The medium of per-cell vp, vs, rho, Qp, Qs over the memory box
        (shape (ny+6, nx+6, nz+6), k fastest): the moduli as vmodel_lhm forms
        them (m_vmodel_lhm.f90:158-160, in FP32 with its operation order),
        then medium__setup."""
        self = cls.__new__(cls)
        shape = (p.ny + 6, p.nx + 6, p.nz + 6)
        f = lambda a: np.ascontiguousarray(a, np.float32).reshape(shape)
        vp, vs, rho = f(vp), f(vs), f(rho)
        self.rho = rho.copy()
        self.mu = rho * vs * vs
        self.lam = rho * (vp * vp - 2 * vs * vs)
        self.qp, self.qs = f(qp).copy(), f(qs).copy()
        for name in self.FIELDS[3:]:
            setattr(self, name, np.zeros(shape, np.float32))
        for name in self.MAPS:
            setattr(self, name, np.zeros(shape[:2], np.int32))
        self._setup(p)
        return self

    def _setup(self, p: Params):
        lib = _lib.load()
        g = grid_struct(p)
        self.ts = np.zeros(3, np.float32)
        scal = np.zeros(3, np.float32)
        rc = lib.swpc_setup_medium_opt(C.byref(g), p.fq_min, p.fq_max, p.fq_ref, fptr(self.rho), fptr(self.lam),
                                       fptr(self.mu), fptr(self.qp), fptr(self.qs), fptr(self.taup), fptr(self.taus),
                                       fptr(self.bx), fptr(self.by), fptr(self.bz), fptr(self.muyz),
                                       fptr(self.muxz), fptr(self.muxy), iptr(self.kfs), iptr(self.kob),
                                       iptr(self.kfs_top), iptr(self.kfs_bot), iptr(self.kob_top),
                                       iptr(self.kob_bot), fptr(self.ts), fptr(scal), int(p.stabilize_pml))
        if rc:
            raise ValueError("medium setup failed")
        self.zeta, self.vmin, self.vmax = (float(x) for x in scal)
        lib.swpc_kbeg_a(C.byref(g), iptr(self.kbeg_a))

    def view(self, average_on_device: bool = False) -> _lib.MediumView:
        """The C view of the medium.  With ``average_on_device`` the six
        averaged fields (bx, by, bz, muyz, muxz, muxy) are left out and
        swpc_upload_medium forms them in HBM from rho and mu."""
        v = _lib.MediumView()
        for name in self.FIELDS[:5] if average_on_device else self.FIELDS:
            setattr(v, name, fptr(getattr(self, name)))
        for name in self.MAPS:
            setattr(v, name, iptr(getattr(self, name)))
        v.ld_k = self.rho.shape[2]
        v.ld_i = self.rho.shape[1]
        v.ld_i2 = self.kfs.shape[1]
        return v


class DeviceMedium:
    """The medium built in HBM (swpc_vmodel_lhm_device, then
    swpc_medium_setup_device): vmodel_lhm with the lhm_rmed perturbation
    ``xi`` and medium__setup (m_medium.f90:36-467) run on the device, bitwise
    equal to ``Medium``; the fields stay there and the integer maps, the
    relaxation times and the velocity range come back.  ``xi`` is None, a
    host array or a CUDA tensor of shape (ny+6, nx+6, nz+6)."""

    MAPS = Medium.MAPS

    def __init__(self, lib, ctx, p: Params, xi=None):
        L = p.layers
        if not L:
            raise ValueError("a layered (lhm) velocity model is required")
        arr = lambda attr: np.array([getattr(l, attr) for l in L], np.float32)
        shape = (p.ny + 6, p.nx + 6, p.nz + 6)
        xp = None
        if xi is not None:
            if hasattr(xi, "data_ptr") and getattr(xi, "is_cuda", False):
                import torch

                assert tuple(xi.shape) == shape and xi.dtype == torch.float32 and xi.is_contiguous()
                xp = C.cast(C.c_void_p(xi.data_ptr()), _lib._FP)
            else:
                xi = np.ascontiguousarray(xi, np.float32)
                assert xi.shape == shape
                xp = fptr(xi)
        check(ctx, lib.swpc_vmodel_lhm_device_opt(ctx, len(L), fptr(arr("depth")), fptr(arr("rho")),
                                                  fptr(arr("vp")), fptr(arr("vs")), fptr(arr("qp")), fptr(arr("qs")),
                                                  p.vcut, p.rhomin, p.zbeg, xp, p.nz + 6, p.nx + 6,
                                                  int(p.munk_profile)))
        for name in self.MAPS:
            setattr(self, name, np.zeros(shape[:2], np.int32))
        self.ts = np.zeros(3, np.float32)
        scal = np.zeros(3, np.float32)
        check(ctx, lib.swpc_medium_setup_device_opt(ctx, p.fq_min, p.fq_max, p.fq_ref, fptr(self.ts), fptr(scal),
                                                    *(iptr(getattr(self, n)) for n in self.MAPS), p.nx + 6,
                                                    int(p.stabilize_pml)))
        self.zeta, self.vmin, self.vmax = (float(x) for x in scal)


class Swpc3D:
    """One 3D run on one GPU (the single-node case of the reference)."""

    def __init__(self, p: Params, xi: np.ndarray | None = None, device: int = 0, medium: Medium | None = None,
                 precision: str = "f32", average_on_device: bool = False, medium_on_device: bool = False):
        """``precision`` is the storage of stress and memory variables:
        "f32" (the reference's MP = SP build), "bf16r" (memory variables in
        BF16), "f16r" (memory variables in FP16 with a power-of-two
        scale) or "f16sr" (stress too in FP16); the arithmetic is FP32 in every form.  With
        ``average_on_device`` the upload sends rho instead of the six averaged
        fields, which the library forms in HBM (same bits); with
        ``medium_on_device`` the whole medium is built in HBM from the layers
        and ``xi`` (``DeviceMedium``, same bits)."""
        p.check()
        self.p = p
        self.precision = precision
        self.lib = _lib.load()
        if not medium_on_device:
            self.medium = medium if medium is not None else Medium(p, xi)
        m = self.medium if not medium_on_device else None
        desc = _lib.Desc(_lib.KIND_3D, p.nx, p.ny, p.nz, p.na, p.nm, p.nt, p.dx, p.dy, p.dz, p.dt, p.tbeg, device,
                         _lib.PRECISIONS[precision])
        ctx = C.c_void_p()
        rc = self.lib.swpc_create(C.byref(desc), C.byref(ctx))
        self.ctx = ctx
        if rc:
            msg = self.lib.swpc_last_error(ctx) if ctx else b""
            self.lib.swpc_destroy(ctx)
            self.ctx = None
            raise _lib.SwpcError(rc, msg.decode() if msg else "swpc_create failed")
        self._keep = []
        if medium_on_device:
            m = self.medium = DeviceMedium(self.lib, self.ctx, p, xi)
        else:
            check(self.ctx, self.lib.swpc_upload_medium(self.ctx, C.byref(m.view(average_on_device))))
        check(self.ctx, self.lib.swpc_kernel_setup(self.ctx, fptr(m.ts)))
        # source__setup (m_source.f90) or green__setup (m_green.f90)
        if p.pw_mode and p.green_mode:
            raise ValueError("pw_mode and green_mode exclude each other (m_source.f90:69)")
        self.src = source_grid(Params(**{**p.__dict__, "sources": [], "bf_mode": False})) if p.pw_mode \
            else source_grid(p)
        self.M0, self.UC = self.src.M0, self.src.UC
        stf = _lib.STF_CODES[p.stftype]
        if p.pw_mode:
            self._pw_setup(p, stf)
        elif p.green_mode:
            st = p.stations[p.green_station]
            self.M0 = 1.0
            i, j, k = station_grid(Params(**{**p.__dict__, "stations": [st]}), m.kfs, m.kob)
            if len(i) != 1:
                raise ValueError("green source station outside the domain")
            check(self.ctx, self.lib.swpc_green_setup(self.ctx, int(i[0]), int(j[0]), int(k[0]),
                                                      p.green_cmp.encode()[0:1], 0.0, p.green_trise, stf))
            self.fcut = 1.0 / p.green_trise
        elif p.bf_mode:
            s = self.src
            check(self.ctx, self.lib.swpc_bodyforce_setup(self.ctx, len(s.isrc), iptr(s.isrc), iptr(s.jsrc),
                                                          iptr(s.ksrc), fptr(s.srcprm), fptr(s.f3), stf))
            self.fcut = s.fcut
        else:
            s = self.src
            check(self.ctx, self.lib.swpc_source_setup(self.ctx, len(s.isrc), iptr(s.isrc), iptr(s.jsrc),
                                                       iptr(s.ksrc), fptr(s.srcprm), fptr(s.mo), fptr(s.m6), stf))
            self.fcut = s.fcut
        g = grid_struct(p)
        if p.abc_type == "cerjan":
            # absorb__setup's dispatch (m_absorb.f90:25-41): absorb_c__setup
            n = {"x": p.nx, "y": p.ny, "z": p.nz}
            self.cprof = {a + t: np.zeros(n[a[1]], np.float32) for a in ("gx", "gy", "gz") for t in ("_c", "_b")}
            cp = self.cprof
            names = ("gx_c", "gx_b", "gy_c", "gy_b", "gz_c", "gz_b")
            self.lib.swpc_cerjan_profiles(C.byref(g), *(fptr(cp[k]) for k in names))
            check(self.ctx, self.lib.swpc_absorb_setup_cerjan(self.ctx, *(fptr(cp[k]) for k in names)))
        else:
            # absorb_p__setup with fcut from the source setup (m_absorb_p.f90:528)
            self.gprof = {n: np.zeros((p.nx if n[1] == "x" else p.ny if n[1] == "y" else p.nz, 4), np.float32)
                          for n in ("gxc", "gxe", "gyc", "gye", "gzc", "gze")}
            gp = self.gprof
            self.lib.swpc_damping_profiles(C.byref(g), float(f32(self.fcut)), fptr(gp["gxc"]), fptr(gp["gxe"]),
                                           fptr(gp["gyc"]), fptr(gp["gye"]), fptr(gp["gzc"]), fptr(gp["gze"]))
            check(self.ctx, self.lib.swpc_absorb_setup(self.ctx, fptr(gp["gxc"]), fptr(gp["gxe"]),
                                                       fptr(gp["gyc"]), fptr(gp["gye"]), fptr(gp["gzc"]),
                                                       fptr(gp["gze"])))
        # wav__setup (m_wav.f90:76-142); off in green mode
        self.nst = 0
        what = (_lib.WAV_V * p.sw_wav_v) | (_lib.WAV_U * p.sw_wav_u) | (_lib.WAV_STRESS * p.sw_wav_stress) | \
            (_lib.WAV_STRAIN * p.sw_wav_strain)
        if p.stations and not p.green_mode and what:
            self.ist, self.jst, self.kst = station_grid(p, m.kfs, m.kob)
            self.nst = len(self.ist)
            check(self.ctx, self.lib.swpc_wav_setup(self.ctx, self.nst, iptr(self.ist), iptr(self.jst),
                                                    iptr(self.kst), p.ntdec_w, what, self.M0, self.UC))
        self.what = what
        # snap__setup (m_snap.f90:95-322)
        self.snap_nframes = 0
        if p.snaps:
            self.snap__setup()

    def _pw_setup(self, p: Params, stf: int):
        """pw_setup (m_source.f90:315-465): the plane-wave initial wavefield
        from the host medium, uploaded over the memory box; no source grid,
        M0 = 1 / UC, the PML's fcut from the wave speed at the front, and the
        zero-derivative side boundary switched on."""
        if not isinstance(self.medium, Medium):
            raise ValueError("the plane-wave setup reads the host medium (Medium), not the device-built one")
        if p.pw_ps.lower() not in ("p", "s"):
            raise ValueError("pw_ps must be 'P' or 'S'")
        m = self.medium
        shape = m.rho.shape
        f = [np.zeros(shape, np.float32) for _ in range(9)]
        fcut = C.c_float()
        rc = self.lib.swpc_pw_setup(C.byref(grid_struct(p)), fptr(m.rho), fptr(m.lam), fptr(m.mu), p.pw_ztop,
                                    p.pw_zlen, 0 if p.pw_ps.lower() == "p" else 1, p.pw_strike, p.pw_dip, p.pw_rake,
                                    stf, *(fptr(a) for a in f), C.byref(fcut))
        if rc:
            raise ValueError("pw_setup failed (pw_zlen > 0 and pw_ztop inside the grid are required)")
        for q, a in enumerate(f):
            self.upload(_lib.F_VX + q, a)
        self.M0 = float(f32(1.0) / f32(self.UC))
        self.fcut = float(fcut.value)
        check(self.ctx, self.lib.swpc_set_pw_mode(self.ctx, 1))

    # -- lifetime ---------------------------------------------------------
    def close(self):
        # batches borrow the context: they go first
        for ref in getattr(self, "_dependents", []):
            dep = ref()
            if dep is not None:
                dep.close()
        self._dependents = []
        if self.ctx:
            self.lib.swpc_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- the reference routines --------------------------------------------
    def kernel__update_stress(self):
        check(self.ctx, self.lib.swpc_kernel_update_stress(self.ctx))

    def absorb__update_stress(self):
        check(self.ctx, self.lib.swpc_absorb_update_stress(self.ctx))

    def kernel__update_vel(self):
        check(self.ctx, self.lib.swpc_kernel_update_vel(self.ctx))

    def absorb__update_vel(self):
        check(self.ctx, self.lib.swpc_absorb_update_vel(self.ctx))

    def source__stressglut(self, it: int):
        check(self.ctx, self.lib.swpc_source_stressglut(self.ctx, it))

    def source__bodyforce(self, it: int):
        check(self.ctx, self.lib.swpc_source_bodyforce(self.ctx, it))

    def green__source(self, it: int):
        check(self.ctx, self.lib.swpc_green_source(self.ctx, it))

    def global__comm_stress(self):
        check(self.ctx, self.lib.swpc_comm_stress(self.ctx))

    def global__comm_vel(self):
        check(self.ctx, self.lib.swpc_comm_vel(self.ctx))

    def wav__store(self, it: int):
        check(self.ctx, self.lib.swpc_wav_store(self.ctx, it))

    def snap__setup(self):
        """Enable the snapshot planes named in ``p.snaps`` with the
        reference's defaults for the section positions (m_snap.f90:118-120)."""
        from .params import snap_plane

        p = self.p
        xend = f32(p.xbeg) + f32(p.nx) * f32(p.dx)
        yend = f32(p.ybeg) + f32(p.ny) * f32(p.dy)
        zend = f32(p.zbeg) + f32(p.nz) * f32(p.dz)
        z0 = f32(p.z0_xy) if p.z0_xy is not None else max(min(f32(10.0), zend), f32(p.zbeg))
        x0 = f32(p.x0_yz) if p.x0_yz is not None else max(min(f32(0.0), xend), f32(p.xbeg))
        y0 = f32(p.y0_xz) if p.y0_xz is not None else max(min(f32(0.0), yend), f32(p.ybeg))
        lib = self.lib
        planes = 0
        for name in p.snaps:
            planes |= 1 << snap_plane(name)
        d = _lib.SnapDesc(planes, p.idec, p.jdec, p.kdec, p.ntdec_s, lib.swpc_x2i(float(x0), p.xbeg, p.dx),
                          lib.swpc_x2i(float(y0), p.ybeg, p.dy), lib.swpc_x2i(float(z0), p.zbeg, p.dz),
                          float(f32(self.M0)), float(f32(self.UC)))
        check(self.ctx, lib.swpc_snap_setup(self.ctx, C.byref(d)))
        self.snap_desc = d
        self.snap_nframes = (p.nt - 1) // p.ntdec_s + 1

    def snap__write(self, it: int):
        check(self.ctx, self.lib.swpc_snap_write(self.ctx, it))

    def snapshots(self, name: str) -> np.ndarray:
        """Frames of one plane ("xz_v", "fs_ps", ...): (nframes, nvar, n2, n1)."""
        from .params import snap_plane

        plane = snap_plane(name)
        nv, n1, n2, nf = (C.c_int() for _ in range(4))
        check(self.ctx, self.lib.swpc_snap_dims(self.ctx, plane, C.byref(nv), C.byref(n1), C.byref(n2),
                                                C.byref(nf)))
        out = np.zeros((nf.value, nv.value, n2.value, n1.value), np.float32)
        check(self.ctx, self.lib.swpc_snap_fetch(self.ctx, plane, fptr(out)))
        return out

    def snapshot_max(self, name: str) -> np.ndarray:
        """Running maxima of "fs_v", "fs_u", "ob_v" or "ob_u": (3, nys, nxs)
        = vertical, horizontal, vector."""
        which = {"fs_v": 0, "fs_u": 1, "ob_v": 2, "ob_u": 3}[name]
        nv, n1, n2, nf = (C.c_int() for _ in range(4))
        check(self.ctx, self.lib.swpc_snap_dims(self.ctx, 9, C.byref(nv), C.byref(n1), C.byref(n2), C.byref(nf)))
        out = np.zeros((3, n2.value, n1.value), np.float32)
        check(self.ctx, self.lib.swpc_snap_fetch_max(self.ctx, which, fptr(out)))
        return out

    def kernel__vmax(self) -> np.ndarray:
        out = np.zeros(3, np.float32)
        check(self.ctx, self.lib.swpc_vmax(self.ctx, fptr(out)))
        return out

    def step(self, it: int):
        """One pass of main.f90:128-143 (fused interior + absorber launches)."""
        check(self.ctx, self.lib.swpc_step(self.ctx, it))

    def run(self, it0: int = 1, nsteps: int | None = None, report=None) -> list[tuple[int, np.ndarray]]:
        """The time loop of main.f90:125-144 as CUDA-graph replays.  Every
        ``ntdec_r`` steps kernel__vmax runs before the step (report__progress,
        m_report.f90:134-152); a diverging run raises SwpcError.  Returns the
        list of (it, max|V| * UC * M0) report values."""
        p = self.p
        if nsteps is None:
            nsteps = p.nt - it0 + 1
        last = it0 + nsteps - 1
        reports = []
        it = it0
        while it <= last:
            if it % p.ntdec_r == 0:
                vm = self.kernel__vmax()
                va = vm * f32(self.UC) * f32(self.M0)
                reports.append((it, va))
                if report:
                    report(it, va)
            nxt = (it // p.ntdec_r + 1) * p.ntdec_r
            n = min(nxt, last + 1) - it
            check(self.ctx, self.lib.swpc_run(self.ctx, it, n))
            it += n
        self.sync()
        return reports

    def time_steps(self, it0: int, nsteps: int) -> float:
        ms = C.c_float()
        check(self.ctx, self.lib.swpc_time_steps(self.ctx, it0, nsteps, C.byref(ms)))
        return ms.value

    def rescale(self) -> int:
        """Re-centre the FP16 array scales (precision "f16sr"); returns the
        number of arrays rescaled."""
        n = C.c_int()
        check(self.ctx, self.lib.swpc_rescale(self.ctx, C.byref(n)))
        return n.value

    def sync(self):
        check(self.ctx, self.lib.swpc_sync(self.ctx))

    # -- data ---------------------------------------------------------------
    def green_store_setup(self, ig, jg, kg, bforce: bool = False, ntdec_w: int = 1):
        """green__store (m_green.f90:389-534) at the grid cells (ig, jg, kg):
        reciprocity Green's functions sampled every ntdec_w steps."""
        ip = lambda a: np.ascontiguousarray(a, np.int32)
        self._green = (ip(ig), ip(jg), ip(kg), 9 if bforce else 6, (self.p.nt - 1) // ntdec_w + 1)
        g = self._green
        check(self.ctx, self.lib.swpc_green_store_setup(self.ctx, len(g[0]), *(iptr(a) for a in g[:3]),
                                                        int(bforce), ntdec_w))

    def green_functions(self) -> np.ndarray:
        """gf(ntw, ncmp*ng) (column-major, as the reference) as (ncmp*ng, ntw)."""
        ig, _, _, ncmp, ntw = self._green
        out = np.zeros((ncmp * len(ig), ntw), np.float32)
        check(self.ctx, self.lib.swpc_green_fetch(self.ctx, fptr(out)))
        return out

    def download(self, field: int) -> np.ndarray:
        p = self.p
        out = np.zeros((p.ny + 6, p.nx + 6, p.nz + 6), np.float32)
        check(self.ctx, self.lib.swpc_download_field(self.ctx, field, fptr(out), p.nz + 6, p.nx + 6))
        return out

    def upload(self, field: int, arr: np.ndarray):
        p = self.p
        a = np.ascontiguousarray(arr, np.float32)
        assert a.shape == (p.ny + 6, p.nx + 6, p.nz + 6)
        check(self.ctx, self.lib.swpc_upload_field(self.ctx, field, fptr(a), p.nz + 6, p.nx + 6))

    def record(self, stations=None, what: int = _lib.WAV_V):
        """wav__setup (m_wav.f90:76-142) at ``stations`` (default: the
        parameter file's), also in green mode, where the reference records
        no traces; the traces are scaled by this run's M0 and UC."""
        p = self.p
        q = Params(**{**p.__dict__, "stations": list(p.stations if stations is None else stations)})
        self.ist, self.jst, self.kst = station_grid(q, self.medium.kfs, self.medium.kob)
        self.nst = len(self.ist)
        check(self.ctx, self.lib.swpc_wav_setup(self.ctx, self.nst, iptr(self.ist), iptr(self.jst), iptr(self.kst),
                                                p.ntdec_w, what, self.M0, self.UC))
        self.what = what

    def waveforms(self, what: int = _lib.WAV_V) -> np.ndarray:
        """wav buffer in the reference layout wav(ntw, ncmp, nst), returned as a
        numpy array of shape (nst, ncmp, ntw)."""
        ntw, nst = C.c_int(), C.c_int()
        check(self.ctx, self.lib.swpc_wav_dims(self.ctx, C.byref(ntw), C.byref(nst)))
        ncmp = 3 if what in (_lib.WAV_V, _lib.WAV_U) else 6
        out = np.zeros((nst.value, ncmp, ntw.value), np.float32)
        if nst.value:
            check(self.ctx, self.lib.swpc_wav_fetch(self.ctx, what, fptr(out)))
        return out

    def device_bytes(self) -> int:
        return int(self.lib.swpc_device_bytes(self.ctx))


class ForceBatch3D:
    """Reciprocity batch: one independent wavefield per single force over the
    medium of ``base`` (a 3D run set up in green mode, whose absorber
    profiles and recorder the members share).  ``forces`` lists (station,
    cmp): each member is driven like a green-mode run (green__source,
    m_green.f90:597-632) with a unit force along cmp ('x', 'y', 'z') at the
    station's grid cell and the base's green_trise / stftype.  All members
    advance with one launch per half step."""

    def __init__(self, base: Swpc3D, forces):
        self.base = base
        self.lib = base.lib
        p = base.p
        b = C.c_void_p()
        check(base.ctx, self.lib.swpc_fbatch_create(base.ctx, len(forces), C.byref(b)))
        self.b = b
        if not hasattr(base, "_dependents"):
            base._dependents = []
        base._dependents.append(weakref.ref(self))
        self.n = len(forces)
        stf = _lib.STF_CODES[p.stftype]
        self.cells = []
        for m, (st, cmp) in enumerate(forces):
            i, j, k = station_grid(Params(**{**p.__dict__, "stations": [st]}), base.medium.kfs, base.medium.kob)
            if len(i) != 1:
                raise ValueError(f"force {m}: station outside the domain")
            self.cells.append((int(i[0]), int(j[0]), int(k[0])))
            check(base.ctx, self.lib.swpc_fbatch_green_source(b, m, int(i[0]), int(j[0]), int(k[0]),
                                                              cmp.encode()[0:1], 0.0, p.green_trise, stf))

    def close(self):
        if self.b:
            self.lib.swpc_fbatch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, it: int):
        check(self.base.ctx, self.lib.swpc_fbatch_step(self.b, it))

    def run(self, it0: int, nsteps: int):
        check(self.base.ctx, self.lib.swpc_fbatch_run(self.b, it0, nsteps))
        check(self.base.ctx, self.lib.swpc_fbatch_sync(self.b))

    def time_steps(self, it0: int, nsteps: int) -> float:
        ms = C.c_float()
        check(self.base.ctx, self.lib.swpc_fbatch_time_steps(self.b, it0, nsteps, C.byref(ms)))
        return ms.value

    def set_strip(self, cells: int):
        check(self.base.ctx, self.lib.swpc_fbatch_set_strip(self.b, cells))

    def set_launch(self, kernel: int, mpc: int = 1, bi: int = 4, bj: int = 2):
        """kernel 0: flat kernels; 5 / 6: staged stress / velocity kernels with
        tile (bi, bj) and mpc members per CTA; 7: staged launch order (mpc 1:
        tiles fastest, 0: member groups fastest)."""
        check(self.base.ctx, self.lib.swpc_fbatch_set_launch(self.b, kernel, mpc, bi, bj))

    def launch(self) -> dict:
        out = np.zeros(9, np.int32)
        check(self.base.ctx, self.lib.swpc_fbatch_get_launch(self.b, iptr(out)))
        return {"staged": bool(out[0]), "strip": int(out[1]), "stress": tuple(int(v) for v in out[2:5]),
                "velocity": tuple(int(v) for v in out[5:8]), "tiles_first": bool(out[8])}

    def autotune(self, it0: int, reps: int = 2):
        """Tunes the launch form in use (strip widths, or the staged shapes)
        over steps it0..; returns (steps used, strip)."""
        used, strip = C.c_int(), C.c_int()
        check(self.base.ctx, self.lib.swpc_fbatch_autotune(self.b, it0, reps, C.byref(used), C.byref(strip)))
        return used.value, strip.value

    def waveforms(self, member: int, what: int = _lib.WAV_V) -> np.ndarray:
        base = self.base
        ncmp = 3 if what in (_lib.WAV_V, _lib.WAV_U) else 6
        ntw = (base.p.nt - 1) // base.p.ntdec_w + 1
        out = np.zeros((base.nst, ncmp, ntw), np.float32)
        check(base.ctx, self.lib.swpc_fbatch_wav_fetch(self.b, member, what, fptr(out)))
        return out

    def green_functions(self, member: int) -> np.ndarray:
        """green__store of one member at the base context's green table
        (``Swpc3D.green_store_setup`` before the batch), as (ncmp*ng, ntw)."""
        ig, _, _, ncmp, ntw = self.base._green
        out = np.zeros((ncmp * len(ig), ntw), np.float32)
        check(self.base.ctx, self.lib.swpc_fbatch_green_fetch(self.b, member, fptr(out)))
        return out

    def download(self, member: int, field: int) -> np.ndarray:
        p = self.base.p
        out = np.zeros((p.ny + 6, p.nx + 6, p.nz + 6), np.float32)
        check(self.base.ctx, self.lib.swpc_fbatch_download_field(self.b, member, field, fptr(out), p.nz + 6,
                                                                 p.nx + 6))
        return out

    def device_bytes(self) -> int:
        return int(self.lib.swpc_fbatch_device_bytes(self.b))
