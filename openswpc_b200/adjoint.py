"""Misfit gradient of the 3D viscoelastic run behind ``torch.autograd``.

The misfit is J = 0.5 * sum (v_syn - v_obs)^2 over the three-component
velocity traces that wav__store records (src/swpc_3d/m_wav.f90:530-535) of a
run from rest over steps 1..nt.  Its gradient with respect to per-cell vp, vs
and rho (Q held fixed) comes from the library's discrete adjoint of the step
(``swpc_gradient``: checkpointed forward, recompute per segment, transposed
step, imaging sums in FP32 per checkpoint segment folded into FP64) and the chain rule of ``swpc_gradient_model``.  Both
run on the GPU; this module only moves the model in and the gradient out.

The parameters are the cells of the kernel region: absorber cells copy the
medium of the region's edge (m_medium.f90:124-190) whatever the tensors hold
there, and their medium is held fixed.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import check, fptr
from .params import Params
from .swpc3d import Medium, Swpc3D


class _MediumMaps:
    """Integer maps, relaxation times and velocity range of a medium built in
    HBM (what the host keeps of it)."""

    def __init__(self, p: Params):
        for n in Medium.MAPS:
            setattr(self, n, np.zeros((p.ny + 6, p.nx + 6), np.int32))
        self.ts = np.zeros(3, np.float32)
        self.scal = np.zeros(3, np.float32)


class Misfit3D:
    """A 3D run with its sources, stations and Q fixed, evaluated for any
    per-cell (vp, vs, rho) against observed velocity traces ``obs`` of shape
    (nst, 3, ntw), the layout of ``Swpc3D.waveforms``."""

    def __init__(self, p: Params, vp, vs, rho, qp, qs, obs: np.ndarray, device: int = 0, ckpt: int = 50,
                 slot_memory: int | str = 0):
        self.p = p
        self.qp = np.ascontiguousarray(qp, np.float32)
        self.qs = np.ascontiguousarray(qs, np.float32)
        self.ckpt = int(ckpt)
        self.device = device
        m = Medium.from_model(p, vp, vs, rho, self.qp, self.qs)
        self.solver = Swpc3D(p, device=device, medium=m)
        self.obs = np.ascontiguousarray(obs, np.float32)
        if self.obs.shape != (self.solver.nst, 3, self.ntw):
            raise ValueError(f"observed traces must have shape {(self.solver.nst, 3, self.ntw)}")
        self.set_slot_memory(slot_memory)

    def memory(self) -> tuple[int, int, int, int]:
        """Bytes of one checkpoint, of one kept step, of a kept segment's
        first V and of the working slots of this problem's ckpt."""
        s = self.solver
        ck, st, sg, wk = (C.c_longlong() for _ in range(4))
        check(s.ctx, s.lib.swpc_gradient_memory(s.ctx, C.byref(ck), C.byref(st)))
        check(s.ctx, s.lib.swpc_gradient_segment_bytes(s.ctx, C.byref(sg), C.byref(wk), self.ckpt))
        return ck.value, st.value, sg.value, wk.value

    def _tail(self, budget: int) -> tuple[int, int]:
        """Trailing segments and their steps that `budget` bytes keep (the
        rule of swpc_gradient)."""
        _, st, sg, _ = self.memory()
        nt, k = self.p.nt, self.ckpt
        nseg, t, n = -(-nt // k), 0, 0
        while t < nseg:
            ln = min(k, nt - (nseg - 1 - t) * k)
            if (n + ln) * st + (t + 1) * sg > budget:
                break
            n, t = n + ln, t + 1
        return t, n

    def set_slot_memory(self, nbytes: int | str, reserve: int = 4 << 30) -> int:
        """HBM that the kept steps of trailing segments may take
        (``swpc_gradient_set_slot_memory``): those segments keep what their
        adjoint needs from the first forward pass instead of being
        recomputed, with bitwise the same gradient.  ``"auto"`` keeps the most
        trailing segments that fit, with the working slots and the
        checkpoints of the segments before them, in the device's free memory
        less ``reserve`` bytes (call it before the first gradient, whose
        buffers it would count as used).  Returns the bytes set."""
        s = self.solver
        if nbytes == "auto":
            free, _ = torch.cuda.mem_get_info(self.device)
            ck, st, sg, wk = self.memory()
            nt, k = self.p.nt, self.ckpt
            nseg = -(-nt // k)
            nbytes, steps = 0, 0
            for t in range(1, nseg + 1):
                steps += min(k, nt - (nseg - t) * k)
                keep = steps * st + t * sg
                if keep + max(nseg - t, 1) * ck + wk > free - reserve:
                    break
                nbytes = keep
        check(s.ctx, s.lib.swpc_gradient_set_slot_memory(s.ctx, int(nbytes)))
        self.slot_memory = int(nbytes)
        return self.slot_memory

    def kept_steps(self) -> int:
        """Steps of the trailing segments that the gradient keeps from its
        forward pass."""
        return self._tail(self.slot_memory)[1]

    @property
    def ntw(self) -> int:
        return (self.p.nt - 1) // self.p.ntdec_w + 1

    def close(self):
        self.solver.close()

    def _on_device(self, *ts) -> bool:
        """Whether the model tensors are CUDA tensors on the problem's device
        (the model then stays in HBM)."""
        dev = torch.device(f"cuda:{self.device}" if isinstance(self.device, int) else self.device)
        return all(isinstance(t, torch.Tensor) and t.is_cuda and t.device == dev for t in ts)

    def _dev(self, a) -> torch.Tensor:
        p = self.p
        shape = (p.ny + 6, p.nx + 6, p.nz + 6)
        dev = torch.device(f"cuda:{self.device}" if isinstance(self.device, int) else self.device)
        return torch.as_tensor(a).detach().to(dev, torch.float32).reshape(shape).contiguous()

    def _set_model(self, vp, vs, rho):
        """The medium of per-cell vp, vs, rho: the moduli formed as
        vmodel_lhm forms them (m_vmodel_lhm.f90:158-160, FP32), then
        medium__setup in HBM (swpc_vmodel_upload, swpc_medium_setup_device;
        bitwise the host setup of ``Medium.from_model``).  CUDA tensors on the
        problem's device stay there: swpc_vmodel_velocity_device forms the
        moduli in HBM with the same expressions."""
        s, p = self.solver, self.p
        if self._on_device(vp, vs, rho):
            if not hasattr(self, "_q_dev"):
                self._q_dev = (self._dev(self.qp), self._dev(self.qs))
            vp, vs, rho = (self._dev(t) for t in (vp, vs, rho))
            qp, qs = self._q_dev
            torch.cuda.current_stream(vp.device).synchronize()   # the library works on its own stream
            check(s.ctx, s.lib.swpc_vmodel_velocity_device(s.ctx, *(C.c_void_p(t.data_ptr()) for t in
                                                                    (vp, vs, rho, qp, qs)), p.nz + 6, p.nx + 6))
            m = _MediumMaps(p)
            check(s.ctx, s.lib.swpc_medium_setup_device_opt(s.ctx, p.fq_min, p.fq_max, p.fq_ref, fptr(m.ts),
                                                            fptr(m.scal),
                                                            *(_lib.iptr(getattr(m, n)) for n in Medium.MAPS),
                                                            p.nx + 6, int(p.stabilize_pml)))
            s.medium = m
            return m
        if p.stabilize_pml:
            m = Medium.from_model(p, vp, vs, rho, self.qp, self.qs)
            check(s.ctx, s.lib.swpc_upload_medium(s.ctx, C.byref(m.view(average_on_device=True))))
            s.medium = m
            return m
        shape = (p.ny + 6, p.nx + 6, p.nz + 6)
        f = lambda a: np.ascontiguousarray(a, np.float32).reshape(shape)
        vp, vs, rho = f(vp), f(vs), f(rho)
        mu = rho * vs * vs
        lam = rho * (vp * vp - 2 * vs * vs)
        check(s.ctx, s.lib.swpc_vmodel_upload(s.ctx, fptr(rho), fptr(lam), fptr(mu), fptr(self.qp), fptr(self.qs),
                                              p.nz + 6, p.nx + 6))
        m = _MediumMaps(p)
        check(s.ctx, s.lib.swpc_medium_setup_device(s.ctx, p.fq_min, p.fq_max, p.fq_ref, fptr(m.ts), fptr(m.scal),
                                                    *(_lib.iptr(getattr(m, n)) for n in Medium.MAPS), p.nx + 6))
        s.medium = m
        return m

    def misfit(self, vp, vs, rho) -> float:
        """J of one forward run (no adjoint)."""
        s = self.solver
        self._set_model(vp, vs, rho)
        check(s.ctx, s.lib.swpc_reset_state(s.ctx))
        check(s.ctx, s.lib.swpc_run(s.ctx, 1, self.p.nt))
        r = s.waveforms(_lib.WAV_V).astype(np.float64) - self.obs
        return 0.5 * float(np.sum(r * r))

    def gradient(self, vp, vs, rho):
        """(J, dJ/dvp, dJ/dvs, dJ/drho); the gradients are float64 arrays
        over the memory box, or float64 CUDA tensors when the model is given
        as CUDA tensors on the problem's device (then nothing crosses to the
        host but the traces and the misfit)."""
        s, p = self.solver, self.p
        on_dev = self._on_device(vp, vs, rho)
        self._set_model(vp, vs, rho)
        J = C.c_double()
        check(s.ctx, s.lib.swpc_gradient(s.ctx, fptr(self.obs), self.ckpt, C.byref(J)))
        shape = (p.ny + 6, p.nx + 6, p.nz + 6)
        if on_dev:
            m = [self._dev(t) for t in (vp, vs, rho)]
            out = [torch.empty(shape, dtype=torch.float64, device=m[0].device) for _ in range(3)]
            ptr = lambda t: C.c_void_p(t.data_ptr())
            check(s.ctx, s.lib.swpc_gradient_model_device(s.ctx, ptr(m[0]), ptr(m[1]), ptr(m[2]), p.nz + 6,
                                                          p.nx + 6, ptr(out[0]), ptr(out[1]), ptr(out[2])))
            return J.value, out[0], out[1], out[2]
        f = lambda a: np.ascontiguousarray(a, np.float32).reshape(shape)
        out = [np.zeros(shape, np.float64) for _ in range(3)]
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        check(s.ctx, s.lib.swpc_gradient_model(s.ctx, fptr(f(vp)), fptr(f(vs)), fptr(f(rho)), p.nz + 6, p.nx + 6,
                                               dp(out[0]), dp(out[1]), dp(out[2])))
        return J.value, out[0], out[1], out[2]


def _host(t: torch.Tensor) -> np.ndarray:
    return t.detach().to("cpu", torch.float32).contiguous().numpy()


class WaveformMisfit(torch.autograd.Function):
    """J(vp, vs, rho) of a :class:`Misfit3D` problem as an autograd node.

    ``forward`` runs the forward and, when any input needs a gradient, the
    checkpointed adjoint in the same call (the adjoint needs the residuals of
    the whole forward, so both run together); ``backward`` scales the stored
    gradient by the incoming one.  J is returned as a float64 scalar tensor on
    the device of ``vp``."""

    @staticmethod
    def forward(ctx, vp: torch.Tensor, vs: torch.Tensor, rho: torch.Tensor, problem: Misfit3D):
        # CUDA tensors on the problem's device stay in HBM; others go through host memory
        args = (vp, vs, rho) if problem._on_device(vp, vs, rho) else (_host(vp), _host(vs), _host(rho))
        if any(ctx.needs_input_grad[:3]):
            J, gvp, gvs, grho = problem.gradient(*args)
            as_t = lambda g, t: g.reshape(t.shape) if isinstance(g, torch.Tensor) else torch.from_numpy(g).to(t.device)
            ctx.save_for_backward(*(as_t(g, t) for g, t in ((gvp, vp), (gvs, vs), (grho, rho))))
            ctx.dtypes = (vp.dtype, vs.dtype, rho.dtype)
        else:
            J = problem.misfit(*args)
        return torch.tensor(J, dtype=torch.float64, device=vp.device)

    @staticmethod
    def backward(ctx, gJ: torch.Tensor):
        gvp, gvs, grho = ctx.saved_tensors
        out = [(gJ * g).to(dt) for g, dt in zip((gvp, gvs, grho), ctx.dtypes)]
        return out[0], out[1], out[2], None


def waveform_misfit(vp: torch.Tensor, vs: torch.Tensor, rho: torch.Tensor, problem: Misfit3D) -> torch.Tensor:
    """J = 0.5 sum (v_syn - v_obs)^2, differentiable in vp, vs and rho."""
    return WaveformMisfit.apply(vp, vs, rho, problem)
