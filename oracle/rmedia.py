"""Random-media generation restated in numpy (TEST INFRASTRUCTURE ONLY).

Follows rmedia__3dgen / rmedia__2dgen (src/shared/m_rmedia.f90:176-307,
:424-) in FP64: uniform random numbers, forward FFT, whitening, filtering by
sqrt(psdf * N * dV) with the PSDFs of m_rmedia.f90:530-679, DC set to zero,
inverse FFT with 1 / (N dV), mean removed, rms scaled to epsil; then the
cyclic mapping onto the memory box of rdrmed__3d (src/shared/m_rdrmed.f90:
100-132).  The uniform numbers are the library's counter-based stream
(splitmix64 of the seed and the cell index, k fastest, then i, then j; top 24
bits), restated here so that the GPU generator is checked value for value.
Only tests/ and bench.py's reference arm (which needs a medium without the
library) use it.
"""
from __future__ import annotations

import math

import numpy as np

GAUSS, EXP, VONKARMAN = 1, 2, 3
PTYPES_BY_NAME = {"gauss": GAUSS, "exp": EXP, "vonkarman": VONKARMAN}


def uniform01(seed: int, n: int) -> np.ndarray:
    """The counter-based uniform stream: value q of seed s (float32 in [0, 1))."""
    with np.errstate(over="ignore"):
        q = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed) + q * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return ((z >> np.uint64(40)).astype(np.float64) / 16777216.0).astype(np.float32)


def psdf(ptype: int, m: np.ndarray, a: float, eps: float, kappa: float, two_d: bool) -> np.ndarray:
    """rmedia__psdf_{gauss,exp,vonKarman}{2d,3d} (m_rmedia.f90:530-679)."""
    pi = math.pi
    am2 = a * a * m * m
    if two_d:
        if ptype == GAUSS:
            return eps * eps * a * a * pi * np.exp(-m * m * a * a * 0.25)
        if ptype == EXP:
            return (2 * eps * eps * a * a * pi) / (1 + am2) ** 1.5
        return (4 * pi * a * a * eps * eps * kappa) / (1 + am2) ** (1 + kappa)
    if ptype == GAUSS:
        return eps * eps * a ** 3 * pi ** 1.5 * np.exp(-m * m * a * a * 0.25)
    if ptype == EXP:
        return (8 * eps * eps * a ** 3 * pi) / (1 + am2) ** 2
    return (8 * pi ** 1.5 * eps * eps * a ** 3 * math.gamma(kappa + 1.5)) / (math.gamma(kappa) * (1 + am2) ** (kappa + 1.5))


def wavenumbers(n: int, d: float) -> np.ndarray:
    """fk__x2k (src/shared/m_fk.f90:269-274): 2 pi q / (n d), negative above n/2."""
    q = np.arange(n)
    return np.where(q <= n // 2, 2 * np.pi * q / (n * d), -2 * np.pi * (n - q) / (n * d))


def volume(ptype: int, nx: int, ny: int, nz: int, dx: float, dy: float, dz: float, a: float, eps: float,
           kappa: float, seed: int) -> np.ndarray:
    """The generated volume, shape (ny, nx, nz) (k fastest); ny = 1 is 2D."""
    two_d = ny == 1
    u = uniform01(seed, nx * ny * nz).astype(np.float64).reshape(ny, nx, nz)
    b = np.fft.rfftn(u, axes=(1, 2) if two_d else (0, 1, 2))
    k1 = wavenumbers(ny, dy)[:, None, None] if not two_d else np.zeros((1, 1, 1))
    k2 = wavenumbers(nx, dx)[None, :, None]
    k3 = (2 * np.pi * np.arange(nz // 2 + 1) / (nz * dz))[None, None, :]
    m = np.sqrt(k1 ** 2 + k2 ** 2 + k3 ** 2)
    ndv = nx * ny * nz * dx * dz * (1.0 if two_d else dy)
    mod = np.abs(b)
    with np.errstate(divide="ignore", invalid="ignore"):
        g = np.where(mod > 0, np.sqrt(psdf(ptype, m, a, eps, kappa, two_d) * ndv) / ndv / mod, 0.0)
    b = b * g
    b[0, 0, 0] = 0.0
    x = np.fft.irfftn(b, s=(nx, nz) if two_d else (ny, nx, nz), axes=(1, 2) if two_d else (0, 1, 2))
    x = x * (nx * ny * nz)   # numpy's inverse divides by N; the 1 / (N dV) is in g
    x = x - x.mean()
    rms = np.sqrt(np.mean(x * x))
    return x * (eps / rms) if rms > 0 else x


def box(vol: np.ndarray) -> np.ndarray:
    """The volume over the memory box with rdrmed__3d's cyclic wrap:
    (ny+6, nx+6, nz+6), or (nx+6, nz+6) for a 2D volume."""
    ny, nx, nz = vol.shape
    wrap = lambda n: (np.arange(-2, n + 4) - 1) % n
    if ny == 1:
        return vol[0][np.ix_(wrap(nx), wrap(nz))]
    return vol[np.ix_(wrap(ny), wrap(nx), wrap(nz))]


def vonkarman_box(shape_kij, dx, dy, dz, eps, a, kappa, seed) -> np.ndarray:
    """The von Karman medium of a 3D run over the memory box, float32."""
    nj, ni, nk = shape_kij
    return box(volume(VONKARMAN, ni - 6, nj - 6, nk - 6, dx, dy, dz, a, eps, kappa, seed)).astype(np.float32)
