"""The random-media generator in HBM (swpc_rmedia_generate) against the
oracle's FP64 restatement of rmedia__3dgen / rmedia__2dgen: the same uniform
stream, so the fields agree to FP32 FFT rounding; the rms is epsil; the
memory box wraps cyclically; a seed gives one realisation."""
from __future__ import annotations

import numpy as np
import pytest

from openswpc_b200.media import rmedia
from oracle import rmedia as R

pytestmark = pytest.mark.gpu

TOL = 2e-5   # rel-L2 of the FP32 generator against the FP64 restatement


def rel_l2(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("ptype", ["gauss", "exp", "vonkarman"])
@pytest.mark.parametrize("shape", [(36, 40, 48), (1, 96, 60)])
def test_generator_matches_oracle(ptype, shape):
    ny, nx, nz = shape
    dx, dy, dz, a, eps, kappa, seed = 0.25, 0.3, 0.2, 1.5, 0.07, 0.4, 2024
    g = rmedia(ptype, nx, ny, nz, dx, dy, dz, a, eps, kappa, seed).cpu().numpy()
    o = R.box(R.volume(R.PTYPES_BY_NAME[ptype], nx, ny, nz, dx, dy, dz, a, eps, kappa, seed))
    assert g.shape == o.shape
    assert rel_l2(g, o) <= TOL, rel_l2(g, o)
    inner = g[3:-3, 3:-3] if ny == 1 else g[3:-3, 3:-3, 3:-3]
    assert abs(float(np.sqrt(np.mean(inner.astype(np.float64) ** 2))) - eps) <= 1e-5 * eps


def test_large_run_medium_statistics():
    """The medium of the large heterogeneous run's parameters (eps = 5 %,
    a = 5 km, kappa = 0.5, dx = 0.1 km) on 256 x 192 x 128 cells: against the
    restatement, rms, and one realisation per seed."""
    nx, ny, nz = 256, 192, 128
    args = ("vonkarman", nx, ny, nz, 0.1, 0.1, 0.1, 5.0, 0.05, 0.5)
    g = rmedia(*args, seed=5).cpu().numpy()
    o = R.box(R.volume(R.VONKARMAN, nx, ny, nz, 0.1, 0.1, 0.1, 5.0, 0.05, 0.5, seed=5))
    assert rel_l2(g, o) <= TOL
    again = rmedia(*args, seed=5).cpu().numpy()
    other = rmedia(*args, seed=6).cpu().numpy()
    assert np.array_equal(g.view(np.uint32), again.view(np.uint32))
    assert rel_l2(other, g) > 0.5
    # the ghost cells repeat the far side of the volume
    assert np.array_equal(g[0], g[ny]) and np.array_equal(g[:, 1], g[:, nx + 1]) and np.array_equal(g[..., 2], g[..., nz + 2])
