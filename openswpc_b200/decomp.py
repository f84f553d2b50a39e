"""Decomposed 3D runs: the grid split into nproc_x x nproc_y blocks, one
library context per block, with the sleeve exchange of global__comm_stress /
global__comm_vel (src/swpc_3d/m_global.f90:393-609) after each half step.

The blocks follow global__setup2 (m_global.f90:236-300): rank r has block
coordinates (r mod nproc_x, r div nproc_x) and the extents below.  Every
block is one context (``swpc_set_subdomain``) that holds its part of the
medium, sleeve included, the sources whose cell lies in its sleeve range
(m_source.f90:208-211) and the stations inside it (m_wav.f90:206), so a
decomposed run gives the bits of the single-domain run in every cell.

Two ways to move the halos:
* ``Decomposed3D`` keeps all blocks in one process (one GPU or several): the
  messages go through device buffers (a copy across devices where the
  neighbours sit on different GPUs);
* ``BlockRank3D`` is one block per process under torch.distributed (one rank
  per GPU, NCCL point-to-point over NVLink; any backend for the exchange
  logic), trading the same messages with its neighbour ranks.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, fptr, iptr
from .params import Params
from .swpc3d import Medium, grid_struct, source_grid, station_grid

f32 = np.float32

SIDES = 4                      # 0 -x, 1 +x, 2 -y, 3 +y
OPPOSITE = (1, 0, 3, 2)


def block_range(n: int, nproc: int, q: int) -> tuple[int, int]:
    """(beg, end) of block coordinate q when n cells split over nproc blocks
    (global__setup2, m_global.f90:236-249, 276-288): the first nproc - n mod
    nproc blocks get n div nproc cells, the rest one more."""
    m = n % nproc
    if q <= nproc - m - 1:
        return q * (n - m) // nproc + 1, (q + 1) * (n - m) // nproc
    return q * ((n - m) // nproc + 1) - (nproc - m) + 1, (q + 1) * ((n - m) // nproc + 1) - (nproc - m)


def neighbours(px: int, py: int, nproc_x: int, nproc_y: int) -> list[int | None]:
    """Block index (px + py * nproc_x, the rank of m_global.f90:239-240) of
    the neighbour on each side, or None at the grid's faces (MPI_PROC_NULL in
    the reference's itbl)."""
    out = [None] * SIDES
    if px > 0:
        out[0] = (px - 1) + py * nproc_x
    if px < nproc_x - 1:
        out[1] = (px + 1) + py * nproc_x
    if py > 0:
        out[2] = px + (py - 1) * nproc_x
    if py < nproc_y - 1:
        out[3] = px + (py + 1) * nproc_x
    return out


class _Shared:
    """What every block derives from the whole grid: the host medium, the
    source grid (global cells, moments normalised by the total M0), the
    station cells and the absorber profiles."""

    def __init__(self, p: Params, xi=None, medium: Medium | None = None):
        lib = _lib.load()
        self.lib = lib
        self.p = p
        self.medium = medium if medium is not None else Medium(p, xi)
        if p.pw_mode:
            raise ValueError("the plane-wave mode runs on a single domain")
        if p.green_mode:
            raise ValueError("green mode is not decomposed here (one source per run: use Swpc3D or ForceBatch3D)")
        self.src = source_grid(p)
        self.stf = _lib.STF_CODES[p.stftype]
        self.what = (_lib.WAV_V * p.sw_wav_v) | (_lib.WAV_U * p.sw_wav_u) | (_lib.WAV_STRESS * p.sw_wav_stress) | \
            (_lib.WAV_STRAIN * p.sw_wav_strain)
        m = self.medium
        if p.stations and self.what:
            self.ist, self.jst, self.kst = station_grid(p, m.kfs, m.kob)
        else:
            self.ist = self.jst = self.kst = np.zeros(0, np.int32)
        g = grid_struct(p)
        if p.abc_type == "cerjan":
            n = {"x": p.nx, "y": p.ny, "z": p.nz}
            self.cprof = {a + t: np.zeros(n[a[1]], np.float32) for a in ("gx", "gy", "gz") for t in ("_c", "_b")}
            names = ("gx_c", "gx_b", "gy_c", "gy_b", "gz_c", "gz_b")
            lib.swpc_cerjan_profiles(C.byref(g), *(fptr(self.cprof[k]) for k in names))
        else:
            self.gprof = {n: np.zeros((p.nx if n[1] == "x" else p.ny if n[1] == "y" else p.nz, 4), np.float32)
                          for n in ("gxc", "gxe", "gyc", "gye", "gzc", "gze")}
            gp = self.gprof
            lib.swpc_damping_profiles(C.byref(g), float(f32(self.src.fcut)), fptr(gp["gxc"]), fptr(gp["gxe"]),
                                      fptr(gp["gyc"]), fptr(gp["gye"]), fptr(gp["gzc"]), fptr(gp["gze"]))


class Block3D:
    """One block (px, py) of a grid split nproc_x x nproc_y ways: a library
    context over the block with its share of the medium, sources, stations
    and absorber profiles, in block coordinates."""

    def __init__(self, sh: _Shared, px: int, py: int, nproc_x: int, nproc_y: int, device: int = 0,
                 precision: str = "f32"):
        p, lib = sh.p, sh.lib
        self.lib, self.p, self.px, self.py = lib, p, px, py
        self.ib, self.ie = block_range(p.nx, nproc_x, px)
        self.jb, self.je = block_range(p.ny, nproc_y, py)
        self.ioff, self.joff = self.ib - 1, self.jb - 1
        self.nx, self.ny = self.ie - self.ib + 1, self.je - self.jb + 1
        if self.nx < 4 or self.ny < 4:
            raise ValueError("blocks must be at least 4 cells wide")
        self.neighbours = neighbours(px, py, nproc_x, nproc_y)
        self.device = device
        desc = _lib.Desc(_lib.KIND_3D, self.nx, self.ny, p.nz, p.na, p.nm, p.nt, p.dx, p.dy, p.dz, p.dt, p.tbeg,
                         device, _lib.PRECISIONS[precision])
        ctx = C.c_void_p()
        rc = lib.swpc_create(C.byref(desc), C.byref(ctx))
        self.ctx = ctx
        if rc:
            msg = lib.swpc_last_error(ctx) if ctx else b""
            lib.swpc_destroy(ctx)
            self.ctx = None
            raise _lib.SwpcError(rc, msg.decode() if msg else "swpc_create failed")
        check(ctx, lib.swpc_set_subdomain(ctx, p.nx, p.ny, self.ioff, self.joff))
        # the medium over the block's memory box (its sleeve included)
        gm = sh.medium
        js, is_ = slice(self.joff, self.joff + self.ny + 6), slice(self.ioff, self.ioff + self.nx + 6)
        m = Medium.__new__(Medium)
        for name in Medium.FIELDS:
            setattr(m, name, np.ascontiguousarray(getattr(gm, name)[js, is_, :]))
        for name in Medium.MAPS:
            setattr(m, name, np.ascontiguousarray(getattr(gm, name)[js, is_]))
        m.ts = gm.ts
        self.medium = m
        check(ctx, lib.swpc_upload_medium(ctx, C.byref(m.view())))
        check(ctx, lib.swpc_kernel_setup(ctx, fptr(m.ts)))
        # sources whose cell lies in the sleeve range ibeg-2..iend+3 (m_source.f90:208-211)
        s = sh.src
        keep = ((s.isrc >= self.ib - 2) & (s.isrc <= self.ie + 3) & (s.jsrc >= self.jb - 2) &
                (s.jsrc <= self.je + 3))
        isrc = np.ascontiguousarray(s.isrc[keep] - self.ioff, np.int32)
        jsrc = np.ascontiguousarray(s.jsrc[keep] - self.joff, np.int32)
        ksrc = np.ascontiguousarray(s.ksrc[keep], np.int32)
        prm = np.ascontiguousarray(s.srcprm[keep], np.float32)
        if p.bf_mode:
            check(ctx, lib.swpc_bodyforce_setup(ctx, len(isrc), iptr(isrc), iptr(jsrc), iptr(ksrc), fptr(prm),
                                                fptr(np.ascontiguousarray(s.f3[keep], np.float32)), sh.stf))
        else:
            check(ctx, lib.swpc_source_setup(ctx, len(isrc), iptr(isrc), iptr(jsrc), iptr(ksrc), fptr(prm),
                                             fptr(np.ascontiguousarray(s.mo[keep], np.float32)),
                                             fptr(np.ascontiguousarray(s.m6[keep], np.float32)), sh.stf))
        self.nsrc = len(isrc)
        # absorber profiles: the global ones over the block's columns
        ix, iy = slice(self.ioff, self.ioff + self.nx), slice(self.joff, self.joff + self.ny)
        if p.abc_type == "cerjan":
            cp = {k: np.ascontiguousarray(v[ix] if k[1] == "x" else v[iy] if k[1] == "y" else v)
                  for k, v in sh.cprof.items()}
            names = ("gx_c", "gx_b", "gy_c", "gy_b", "gz_c", "gz_b")
            check(ctx, lib.swpc_absorb_setup_cerjan(ctx, *(fptr(cp[k]) for k in names)))
        else:
            gp = {k: np.ascontiguousarray(v[ix] if k[1] == "x" else v[iy] if k[1] == "y" else v)
                  for k, v in sh.gprof.items()}
            check(ctx, lib.swpc_absorb_setup(ctx, *(fptr(gp[k]) for k in ("gxc", "gxe", "gyc", "gye", "gzc", "gze"))))
        # stations inside the block (m_wav.f90:206), in the global station order
        own = (sh.ist >= self.ib) & (sh.ist <= self.ie) & (sh.jst >= self.jb) & (sh.jst <= self.je)
        self.stations = np.nonzero(own)[0]
        self.nst = len(self.stations)
        if self.nst:
            ist = np.ascontiguousarray(sh.ist[own] - self.ioff, np.int32)
            jst = np.ascontiguousarray(sh.jst[own] - self.joff, np.int32)
            kst = np.ascontiguousarray(sh.kst[own], np.int32)
            check(ctx, lib.swpc_wav_setup(ctx, self.nst, iptr(ist), iptr(jst), iptr(kst), p.ntdec_w, sh.what,
                                          s.M0, s.UC))
        self.halo_count = [[0] * SIDES for _ in range(2)]
        n = C.c_longlong()
        for half in (0, 1):
            for side in range(SIDES):
                check(ctx, lib.swpc_halo_count(ctx, half, side, C.byref(n)))
                self.halo_count[half][side] = int(n.value)

    def step_half(self, it: int, half: int):
        check(self.ctx, self.lib.swpc_step_half(self.ctx, it, half))

    def pack(self, half: int, side: int, dst_ptr: int):
        check(self.ctx, self.lib.swpc_halo_pack(self.ctx, half, side, C.c_void_p(dst_ptr)))

    def unpack(self, half: int, side: int, src_ptr: int):
        check(self.ctx, self.lib.swpc_halo_unpack(self.ctx, half, side, C.c_void_p(src_ptr)))

    def sync(self):
        check(self.ctx, self.lib.swpc_sync(self.ctx))

    def vmax(self) -> np.ndarray:
        out = np.zeros(3, np.float32)
        check(self.ctx, self.lib.swpc_vmax(self.ctx, fptr(out)))
        return out

    def download(self, field: int) -> np.ndarray:
        out = np.zeros((self.ny + 6, self.nx + 6, self.p.nz + 6), np.float32)
        check(self.ctx, self.lib.swpc_download_field(self.ctx, field, fptr(out), self.p.nz + 6, self.nx + 6))
        return out

    def waveforms(self, what: int = _lib.WAV_V) -> np.ndarray:
        ntw, nst = C.c_int(), C.c_int()
        check(self.ctx, self.lib.swpc_wav_dims(self.ctx, C.byref(ntw), C.byref(nst)))
        ncmp = 3 if what in (_lib.WAV_V, _lib.WAV_U) else 6
        out = np.zeros((nst.value, ncmp, ntw.value), np.float32)
        if nst.value:
            check(self.ctx, self.lib.swpc_wav_fetch(self.ctx, what, fptr(out)))
        return out

    def close(self):
        if self.ctx:
            self.lib.swpc_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _Run:
    """Time loop, report and gathering shared by both drivers."""

    def run(self, it0: int = 1, nsteps: int | None = None) -> list[tuple[int, np.ndarray]]:
        """main.f90:125-144 over the blocks; every ntdec_r steps the maximum
        of the blocks' kernel__vmax (the mpi_reduce of report__progress,
        m_report.f90:134-152) before the step.  Returns (it, max|V| * UC * M0)."""
        p = self.p
        last = p.nt if nsteps is None else it0 + nsteps - 1
        reports = []
        for it in range(it0, last + 1):
            if it % p.ntdec_r == 0:
                reports.append((it, self.vmax() * f32(self.sh.src.UC) * f32(self.sh.src.M0)))
            self.step(it)
        return reports


class _InProcess(_Run):
    """All blocks in this process.  Every message goes into a receive buffer
    on the receiving block's device: a block's pack kernel stores it there
    directly (NVLink peer stores when the neighbour sits on another GPU), an
    event on the sender's stream marks it complete, and the receiver's stream
    waits for that event before its unpack kernel.  The host never waits.  A
    buffer is overwritten only by the sender's pack two exchanges later, which
    its stream reaches only after waiting for the receiver's own later pack,
    itself after the receiver's unpack: the order holds without more events."""

    def _buffers(self):
        import torch

        # receive buffers: (receiver, half, side the message comes from), on the receiver's device
        self.buf = {}
        for r, b in enumerate(self.blocks):
            for half in (0, 1):
                for side, nbr in enumerate(b.neighbours):
                    if nbr is not None:
                        self.buf[r, half, side] = torch.empty(b.halo_count[half][OPPOSITE[side]],
                                                              dtype=torch.float32, device=f"cuda:{b.device}")
        lib = self.blocks[0].lib if self.blocks else None
        for b in self.blocks:
            for nbr in b.neighbours:
                if nbr is not None and self.blocks[nbr].device != b.device:
                    if lib.swpc_enable_peer_access(b.device, self.blocks[nbr].device):
                        raise RuntimeError(f"no peer access from cuda:{b.device} to cuda:{self.blocks[nbr].device}")
        self.streams = [torch.cuda.ExternalStream(b.lib.swpc_stream(b.ctx), device=f"cuda:{b.device}")
                        for b in self.blocks]

    def _exchange(self, half: int):
        import torch

        packed = []
        for r, b in enumerate(self.blocks):
            for side, nbr in enumerate(b.neighbours):
                if nbr is not None:
                    # into the neighbour's buffer for messages from the opposite side
                    b.pack(half, side, self.buf[nbr, half, OPPOSITE[side]].data_ptr())
            ev = torch.cuda.Event()
            ev.record(self.streams[r])
            packed.append(ev)
        for r, b in enumerate(self.blocks):
            for side, nbr in enumerate(b.neighbours):
                if nbr is None:
                    continue
                self.streams[r].wait_event(packed[nbr])
                b.unpack(half, side, self.buf[r, half, side].data_ptr())

    def step(self, it: int):
        for b in self.blocks:
            b.step_half(it, 0)
        self._exchange(0)
        for b in self.blocks:
            b.step_half(it, 1)
        self._exchange(1)

    def vmax(self) -> np.ndarray:
        return np.max(np.stack([b.vmax() for b in self.blocks]), axis=0)

    def waveforms(self, what: int = _lib.WAV_V) -> np.ndarray:
        """Every block's traces in the global station order."""
        parts = [(b.stations, b.waveforms(what)) for b in self.blocks if b.nst]
        if not parts:
            return np.zeros((0, 0, 0), np.float32)
        ncmp, ntw = parts[0][1].shape[1:]
        out = np.zeros((len(self.sh.ist), ncmp, ntw), np.float32)
        for idx, w in parts:
            out[idx] = w
        return out

    def sync(self):
        for b in self.blocks:
            b.sync()

    def close(self):
        for b in self.blocks:
            b.sync()
        for b in self.blocks:
            b.close()
        self.blocks = []


class Decomposed3D(_InProcess):
    """All blocks of a nproc_x x nproc_y split of a 3D run in this process.
    ``devices`` lists the CUDA device of each block (default: all on device
    0)."""

    def __init__(self, p: Params, nproc_x: int, nproc_y: int, xi=None, devices=None, medium: Medium | None = None,
                 precision: str = "f32"):
        p.check()
        self.p = p
        self.sh = _Shared(p, xi, medium)
        nb = nproc_x * nproc_y
        devices = list(devices) if devices is not None else [0] * nb
        self.blocks = [Block3D(self.sh, r % nproc_x, r // nproc_x, nproc_x, nproc_y, devices[r], precision)
                       for r in range(nb)]
        self._buffers()

    def download(self, field: int) -> np.ndarray:
        """The field over the global memory box (interior cells of every
        block; the sleeve of the grid's faces from the blocks on them)."""
        p = self.p
        out = np.zeros((p.ny + 6, p.nx + 6, p.nz + 6), np.float32)
        for b in self.blocks:
            a = b.download(field)
            # interior columns, plus the grid-face sleeve the block holds
            i0 = 0 if b.ioff == 0 else 3
            i1 = b.nx + 6 if b.ie == p.nx else b.nx + 3
            j0 = 0 if b.joff == 0 else 3
            j1 = b.ny + 6 if b.je == p.ny else b.ny + 3
            out[b.joff + j0:b.joff + j1, b.ioff + i0:b.ioff + i1, :] = a[j0:j1, i0:i1, :]
        return out


class _Shared2D:
    """The whole-grid part of a 2D run's setup (P-SV or SH)."""

    def __init__(self, p: Params, kind: str):
        from .swpc2d import Medium2D, grid2d, source_grid2d, station_grid2d

        lib = _lib.load()
        self.lib, self.p, self.kind = lib, p, kind
        self.medium = Medium2D(p)
        self.src = source_grid2d(p, kind)
        self.stf = _lib.STF_CODES[p.stftype]
        self.what = (_lib.WAV_V * p.sw_wav_v) | (_lib.WAV_U * p.sw_wav_u)
        m = self.medium
        if p.stations and self.what:
            self.ist, self.kst = station_grid2d(p, m.kfs, m.kob)
        else:
            self.ist = self.kst = np.zeros(0, np.int32)
        g = grid2d(p)
        if p.abc_type == "cerjan":
            self.cprof = {k: np.zeros(p.nx if k[1] == "x" else p.nz, np.float32)
                          for k in ("gx_c", "gx_b", "gz_c", "gz_b")}
            cp = self.cprof
            lib.swpc_cerjan_profiles(C.byref(g), fptr(cp["gx_c"]), fptr(cp["gx_b"]), None, None, fptr(cp["gz_c"]),
                                     fptr(cp["gz_b"]))
        else:
            self.gprof = {k: np.zeros((p.nx if k[1] == "x" else p.nz, 4), np.float32)
                          for k in ("gxc", "gxe", "gzc", "gze")}
            gp = self.gprof
            lib.swpc_damping_profiles(C.byref(g), float(f32(self.src.fcut)), fptr(gp["gxc"]), fptr(gp["gxe"]), None,
                                      None, fptr(gp["gzc"]), fptr(gp["gze"]))


class Block2D:
    """Block px of a P-SV or SH grid split nproc_x ways across x (the 2D
    codes' global__setup2, src/swpc_psv/m_global.f90)."""

    def __init__(self, sh: _Shared2D, px: int, nproc_x: int, device: int = 0):
        from .swpc2d import KINDS, Medium2D

        p, lib = sh.p, sh.lib
        self.lib, self.p, self.kind = lib, p, sh.kind
        self.ib, self.ie = block_range(p.nx, nproc_x, px)
        self.ioff, self.nx = self.ib - 1, self.ie - self.ib + 1
        if self.nx < 4:
            raise ValueError("blocks must be at least 4 cells wide")
        self.neighbours = neighbours(px, 0, nproc_x, 1)
        self.device = device
        desc = _lib.Desc(KINDS[sh.kind], self.nx, 1, p.nz, p.na, p.nm, p.nt, p.dx, p.dx, p.dz, p.dt, p.tbeg, device)
        ctx = C.c_void_p()
        rc = lib.swpc_create(C.byref(desc), C.byref(ctx))
        self.ctx = ctx
        if rc:
            msg = lib.swpc_last_error(ctx) if ctx else b""
            lib.swpc_destroy(ctx)
            self.ctx = None
            raise _lib.SwpcError(rc, msg.decode() if msg else "swpc_create failed")
        check(ctx, lib.swpc_set_subdomain(ctx, p.nx, 1, self.ioff, 0))
        gm = sh.medium
        cols = slice(self.ioff, self.ioff + self.nx + 6)
        m = Medium2D.__new__(Medium2D)
        for name in Medium2D.FIELDS:
            setattr(m, name, np.ascontiguousarray(getattr(gm, name)[cols]))
        for name in Medium2D.MAPS:
            setattr(m, name, np.ascontiguousarray(getattr(gm, name)[cols]))
        m.ts = gm.ts
        self.medium = m
        check(ctx, lib.swpc_upload_medium(ctx, C.byref(m.view())))
        check(ctx, lib.swpc_kernel_setup(ctx, fptr(m.ts)))
        s = sh.src
        keep = (s.isrc >= self.ib - 2) & (s.isrc <= self.ie + 3)   # src/swpc_psv/m_source.f90:182
        isrc = np.ascontiguousarray(s.isrc[keep] - self.ioff, np.int32)
        ksrc = np.ascontiguousarray(s.ksrc[keep], np.int32)
        prm = np.ascontiguousarray(s.srcprm[keep], np.float32)
        if p.bf_mode:
            check(ctx, lib.swpc_bodyforce_setup(ctx, len(isrc), iptr(isrc), None, iptr(ksrc), fptr(prm),
                                                fptr(np.ascontiguousarray(s.f3[keep], np.float32)), sh.stf))
        else:
            check(ctx, lib.swpc_source_setup(ctx, len(isrc), iptr(isrc), None, iptr(ksrc), fptr(prm),
                                             fptr(np.ascontiguousarray(s.mo[keep], np.float32)),
                                             fptr(np.ascontiguousarray(s.m6[keep], np.float32)), sh.stf))
        ix = slice(self.ioff, self.ioff + self.nx)
        if p.abc_type == "cerjan":
            cp = {k: np.ascontiguousarray(v[ix] if k[1] == "x" else v) for k, v in sh.cprof.items()}
            check(ctx, lib.swpc_absorb_setup_cerjan(ctx, fptr(cp["gx_c"]), fptr(cp["gx_b"]), None, None,
                                                    fptr(cp["gz_c"]), fptr(cp["gz_b"])))
        else:
            gp = {k: np.ascontiguousarray(v[ix] if k[1] == "x" else v) for k, v in sh.gprof.items()}
            check(ctx, lib.swpc_absorb_setup(ctx, fptr(gp["gxc"]), fptr(gp["gxe"]), None, None, fptr(gp["gzc"]),
                                             fptr(gp["gze"])))
        own = (sh.ist >= self.ib) & (sh.ist <= self.ie)   # src/swpc_psv/m_wav.f90:503
        self.stations = np.nonzero(own)[0]
        self.nst = len(self.stations)
        if self.nst:
            ist = np.ascontiguousarray(sh.ist[own] - self.ioff, np.int32)
            kst = np.ascontiguousarray(sh.kst[own], np.int32)
            check(ctx, lib.swpc_wav_setup(ctx, self.nst, iptr(ist), None, iptr(kst), p.ntdec_w, sh.what, s.M0, s.UC))
        self.halo_count = [[0] * SIDES for _ in range(2)]
        n = C.c_longlong()
        for half in (0, 1):
            for side in (0, 1):
                check(ctx, lib.swpc_halo_count(ctx, half, side, C.byref(n)))
                self.halo_count[half][side] = int(n.value)

    step_half, pack, unpack, sync, close, __del__ = (Block3D.step_half, Block3D.pack, Block3D.unpack, Block3D.sync,
                                                      Block3D.close, Block3D.__del__)

    def vmax(self) -> np.ndarray:
        out = np.zeros(3, np.float32)
        check(self.ctx, self.lib.swpc_vmax(self.ctx, fptr(out)))
        return out[:2] if self.kind == "psv" else out[:1]

    def download(self, field: int) -> np.ndarray:
        out = np.zeros((self.nx + 6, self.p.nz + 6), np.float32)
        check(self.ctx, self.lib.swpc_download_field(self.ctx, field, fptr(out), self.p.nz + 6, self.nx + 6))
        return out

    def waveforms(self, what: int = _lib.WAV_V) -> np.ndarray:
        ntw, nst = C.c_int(), C.c_int()
        check(self.ctx, self.lib.swpc_wav_dims(self.ctx, C.byref(ntw), C.byref(nst)))
        nc = 2 if self.kind == "psv" else 1
        out = np.zeros((nst.value, nc, ntw.value), np.float32)
        if nst.value:
            check(self.ctx, self.lib.swpc_wav_fetch(self.ctx, what, fptr(out)))
        return out


class Decomposed2D(_InProcess):
    """A P-SV or SH run split into nproc_x blocks across x, all in this
    process (``devices``: the CUDA device of each block)."""

    def __init__(self, p: Params, kind: str, nproc_x: int, devices=None):
        p.check()
        self.p = p
        self.sh = _Shared2D(p, kind)
        devices = list(devices) if devices is not None else [0] * nproc_x
        self.blocks = [Block2D(self.sh, q, nproc_x, devices[q]) for q in range(nproc_x)]
        self._buffers()

    def download(self, field: int) -> np.ndarray:
        """The field over the global memory box (nx+6, nz+6)."""
        p = self.p
        out = np.zeros((p.nx + 6, p.nz + 6), np.float32)
        for b in self.blocks:
            a = b.download(field)
            i0 = 0 if b.ioff == 0 else 3
            i1 = b.nx + 6 if b.ie == p.nx else b.nx + 3
            out[b.ioff + i0:b.ioff + i1] = a[i0:i1]
        return out


class HaloTransport:
    """The sleeve messages of one block per rank over torch.distributed:
    every rank posts its sends and receives to its neighbours as one batch of
    point-to-point operations (NCCL over NVLink on GPUs; gloo works for the
    exchange logic on CPU tensors).  Each half step's messages are matched by
    the order of the batch, which every rank builds the same way (sides in
    order 0..3).  With NCCL the waits order the caller's current CUDA stream
    behind the transfers and return at once."""

    def __init__(self, neighbours: list[int | None], group=None):
        self.neighbours = neighbours
        self.group = group

    def exchange(self, send: dict[int, "object"], recv: dict[int, "object"]):
        import torch.distributed as dist

        ops = []
        for side, nbr in enumerate(self.neighbours):
            if nbr is None:
                continue
            ops.append(dist.P2POp(dist.irecv, recv[side], nbr, self.group))
            ops.append(dist.P2POp(dist.isend, send[side], nbr, self.group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()


class BlockRank3D(_Run):
    """One block per process: rank r of torch.distributed's world runs block
    (r mod nproc_x, r div nproc_x) on ``device`` and trades its halos with
    the neighbour ranks through ``HaloTransport``: device buffers with NCCL,
    host copies of them with a backend that moves host tensors (gloo).
    Traces and fields stay with their block; ``vmax`` reduces over the ranks
    (report__progress's mpi_reduce).  ``kind`` "psv" or "sh" runs a 2D block
    of an nproc_x split (nproc_y = 1) the same way."""

    def __init__(self, p: Params, nproc_x: int, nproc_y: int, xi=None, device: int = 0,
                 medium: Medium | None = None, precision: str = "f32", kind: str = "3d"):
        import torch
        import torch.distributed as dist

        p.check()
        self.p = p
        rank, world = dist.get_rank(), dist.get_world_size()
        if world != nproc_x * nproc_y:
            raise ValueError("the world size must equal nproc_x * nproc_y")
        if kind == "3d":
            self.sh = _Shared(p, xi, medium)
            self.block = Block3D(self.sh, rank % nproc_x, rank // nproc_x, nproc_x, nproc_y, device, precision)
        else:
            if nproc_y != 1:
                raise ValueError("the 2D codes split across x only (nproc_y = 1)")
            self.sh = _Shared2D(p, kind)
            self.block = Block2D(self.sh, rank, nproc_x, device)
        self.transport = HaloTransport(self.block.neighbours)
        dev = f"cuda:{device}"
        b = self.block
        self.send = {(h, s): torch.empty(b.halo_count[h][s], dtype=torch.float32, device=dev)
                     for h in (0, 1) for s in range(SIDES) if b.neighbours[s] is not None}
        # what arrives from side s is what this block would send the other way
        self.recv = {(h, s): torch.empty(b.halo_count[h][OPPOSITE[s]], dtype=torch.float32, device=dev)
                     for h in (0, 1) for s in range(SIDES) if b.neighbours[s] is not None}
        self.staged = dist.get_backend() != "nccl"
        # the context's stream as a torch stream, for the stream-ordered NCCL exchange
        self.stream = torch.cuda.ExternalStream(b.lib.swpc_stream(b.ctx), device=dev)

    def _exchange(self, half: int):
        import torch

        b = self.block
        sides = [s for s in range(SIDES) if b.neighbours[s] is not None]
        if not self.staged:
            # NCCL: everything stream-ordered on the block's own stream, no host
            # wait: the sends start after the pack kernels, the unpacks after the
            # receives (work.wait() orders the current stream, not the host)
            with torch.cuda.stream(self.stream):
                for s in sides:
                    b.pack(half, s, self.send[half, s].data_ptr())
                self.transport.exchange({s: self.send[half, s] for s in sides},
                                        {s: self.recv[half, s] for s in sides})
                for s in sides:
                    b.unpack(half, s, self.recv[half, s].data_ptr())
            return
        # a backend that moves host tensors: the messages staged through host memory
        for s in sides:
            b.pack(half, s, self.send[half, s].data_ptr())
        b.sync()
        send = {s: self.send[half, s].cpu() for s in sides}
        recv = {s: self.recv[half, s].cpu() for s in sides}
        self.transport.exchange(send, recv)
        for s in sides:
            self.recv[half, s].copy_(recv[s])
        for s in sides:
            b.unpack(half, s, self.recv[half, s].data_ptr())

    def step(self, it: int):
        self.block.step_half(it, 0)
        self._exchange(0)
        self.block.step_half(it, 1)
        self._exchange(1)

    def vmax(self) -> np.ndarray:
        import torch
        import torch.distributed as dist

        v = torch.from_numpy(self.block.vmax())
        if not self.staged:
            v = v.to(f"cuda:{self.block.device}")
        dist.all_reduce(v, op=dist.ReduceOp.MAX)
        return v.cpu().numpy()

    def waveforms(self, what: int = _lib.WAV_V) -> np.ndarray:
        """This block's traces, rows in the order of ``block.stations``."""
        return self.block.waveforms(what)

    def close(self):
        self.block.close()
