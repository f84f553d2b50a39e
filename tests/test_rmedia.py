"""The oracle's restatement of the random-media generator (CPU, no GPU):
its spectrum is the PSDF of m_rmedia.f90 at every wavenumber, its rms is
epsil, and the memory box wraps cyclically as rdrmed__3d reads a volume."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import rmedia as R


def _splitmix_py(seed, q):
    m = (1 << 64) - 1
    z = (seed + q * 0x9E3779B97F4A7C15) & m
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
    z ^= z >> 31
    return (z >> 40) / 16777216.0


def test_uniform_stream_is_the_counter_based_generator():
    u = R.uniform01(12345, 1000)
    ref = np.array([_splitmix_py(12345, q + 1) for q in range(1000)], np.float32)
    assert np.array_equal(u, ref)
    assert 0.0 <= u.min() and u.max() < 1.0 and abs(u.mean() - 0.5) < 0.03


@pytest.mark.parametrize("ptype", [R.GAUSS, R.EXP, R.VONKARMAN])
@pytest.mark.parametrize("shape", [(20, 24, 18), (1, 40, 30)])
def test_spectrum_follows_the_psdf(ptype, shape):
    ny, nx, nz = shape
    dx, dy, dz, a, eps, kappa = 0.25, 0.3, 0.2, 1.5, 0.07, 0.4
    v = R.volume(ptype, nx, ny, nz, dx, dy, dz, a, eps, kappa, seed=99)
    assert v.shape == (ny, nx, nz)
    assert abs(v.mean()) < 1e-12 and abs(np.sqrt(np.mean(v * v)) - eps) < 1e-12
    two_d = ny == 1
    b = np.fft.rfftn(v, axes=(1, 2) if two_d else (0, 1, 2))
    k1 = R.wavenumbers(ny, dy)[:, None, None] if not two_d else np.zeros((1, 1, 1))
    m = np.sqrt(k1 ** 2 + R.wavenumbers(nx, dx)[None, :, None] ** 2 +
                (2 * np.pi * np.arange(nz // 2 + 1) / (nz * dz))[None, None, :] ** 2)
    ps = R.psdf(ptype, m, a, eps, kappa, two_d).ravel()
    keep = ps > 1e-8 * ps.max()     # the Gaussian PSDF underflows at high wavenumbers
    keep[0] = False
    ratio = np.abs(b.ravel()[keep]) ** 2 / ps[keep]
    assert abs(b.ravel()[0]) < 1e-9
    assert keep.sum() > 50 and np.ptp(ratio) <= 1e-8 * ratio.mean()


def test_memory_box_wraps_cyclically():
    v = R.volume(R.VONKARMAN, 10, 8, 12, 0.5, 0.5, 0.5, 2.0, 0.05, 0.5, seed=3)
    b = R.box(v)
    assert b.shape == (14, 16, 18)
    # box cell (k, i, j) sits at [j + 2, i + 2, k + 2] and holds volume cell (wrap(k), wrap(i), wrap(j)), 1-based
    at = lambda k, i, j: b[j + 2, i + 2, k + 2]
    vol = lambda k, i, j: v[j - 1, i - 1, k - 1]
    assert at(1, 1, 1) == vol(1, 1, 1)
    assert at(1, 0, 1) == vol(1, 10, 1)        # i = 0 -> nx
    assert at(-2, 1, 1) == vol(10, 1, 1)       # k = -2 -> nz - 2
    assert at(15, 11, 11) == vol(3, 1, 3)      # k = nz + 3 -> 3, i = nx + 1 -> 1, j = ny + 3 -> 3
    assert at(12, 10, 8) == vol(12, 10, 8)
