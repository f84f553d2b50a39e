"""Random media for the layered model (the lhm_rmed perturbation).

The reference reads a precomputed random-medium volume per layer
(src/swpc_3d/m_vmodel_lhm_rmed.f90:138, read by src/shared/m_rdrmed.f90:73-134
with a cyclic wrap outside 1..n) that gen_rmed3d generates with
rmedia__3dgen (src/shared/m_rmedia.f90:176-307): uniform random numbers,
whitened spectrum filtered by a Gaussian, exponential or von Karman power
spectral density, mean removed, scaled to rms epsil.  Here the same
generation runs in HBM through the library's ``swpc_rmedia_generate`` (cuFFT
for the transforms) and writes the field straight onto the memory box that
``swpc_vmodel_lhm_device`` reads.  Realisations follow a counter-based
stream of the seed (gfortran's random_number stream cannot be reproduced);
every consumer of a run gets the same array.

PSD (3D von Karman, m_rmedia.f90:667-679):
    P(m) = 8 pi^1.5 eps^2 a^3 Gamma(kappa + 3/2) / (Gamma(kappa) (1 + a^2 m^2)^(kappa + 3/2)).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

PTYPES = {"gauss": 1, "exp": 2, "vonkarman": 3}


def rmedia(ptype: str, nx: int, ny: int, nz: int, dx: float, dy: float, dz: float, a: float, eps: float,
           kappa: float, seed: int, device: int | str = 0):
    """A random medium on the GPU as a float32 CUDA tensor over the memory
    box: shape (ny+6, nx+6, nz+6) (k fastest), or (nx+6, nz+6) for ny = 1
    (rmedia__2dgen).  There is no CPU path: the call needs a CUDA device."""
    import torch

    dev = torch.device(device if isinstance(device, str) else f"cuda:{device}")
    if dev.type != "cuda" or not torch.cuda.is_available():
        raise RuntimeError("swpc_rmedia_generate runs on a CUDA device; none is available")
    lib = _lib.load()
    d = _lib.RmediaDesc(PTYPES[ptype], nx, ny, nz, dx, dy, dz, a, eps, kappa, seed)
    shape = (nx + 6, nz + 6) if ny == 1 else (ny + 6, nx + 6, nz + 6)
    with torch.cuda.device(dev):
        xi = torch.empty(shape, dtype=torch.float32, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        rc = lib.swpc_rmedia_generate(C.byref(d), C.cast(C.c_void_p(xi.data_ptr()), _lib._FP), nz + 6, nx + 6,
                                      C.c_void_p(stream))
    if rc:
        raise _lib.SwpcError(rc, "swpc_rmedia_generate failed")
    return xi


def vonkarman_3d(shape_kij: tuple[int, int, int], dx: float, dy: float, dz: float, eps: float, a: float,
                 kappa: float, seed: int, device: int | str = 0, as_numpy: bool = True):
    """The von Karman medium of a 3D run over the memory box of shape
    ``shape_kij`` = (ny+6, nx+6, nz+6): a numpy array (default) or the CUDA
    tensor itself (``as_numpy=False``)."""
    nj, ni, nk = shape_kij
    xi = rmedia("vonkarman", ni - 6, nj - 6, nk - 6, dx, dy, dz, a, eps, kappa, seed, device)
    return xi.cpu().numpy() if as_numpy else xi
