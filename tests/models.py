"""Small synthetic configurations shared by the tests.

The layered medium is the four-layer model of the 3D forward benchmark
(vp/vs/rho/Qp/Qs from 0, 5, 18 and 30 km); grids are shrunk so that the
oracle finishes in seconds.
"""
from __future__ import annotations

import numpy as np

from openswpc_b200.params import Layer, Params, Source, Station, dc_source

LAYERS = [Layer(0.0, 2.7, 5.5, 3.2, 300, 150), Layer(5.0, 2.8, 6.0, 3.5, 500, 250),
          Layer(18.0, 2.9, 6.7, 3.9, 600, 300), Layer(30.0, 3.3, 7.8, 4.5, 1000, 500)]


def small3d(nx=40, ny=36, nz=32, na=8, nt=60, dx=0.5, dt=0.02, nm=3, **kw) -> Params:
    """A small layered 3D run: air above z = 0, a double couple at 6 km and
    surface/buried stations."""
    rng = np.random.default_rng(1234)
    xb = -nx // 2 * dx
    yb = -ny // 2 * dx
    st = []
    for n in range(6):
        x = float(rng.uniform(xb + (na + 2) * dx, xb + (nx - na - 2) * dx))
        y = float(rng.uniform(yb + (na + 2) * dx, yb + (ny - na - 2) * dx))
        st.append(Station(x, y, 0.0 if n < 4 else 3.0, f"st{n}", ["fsb", "obb", "oba", "dep", "dep", "dep"][n]))
    args = dict(nx=nx, ny=ny, nz=nz, nt=nt, dx=dx, dy=dx, dz=dx, dt=dt, na=na, nm=nm, xbeg=xb, ybeg=yb,
                zbeg=-3 * dx, fq_min=0.05, fq_max=2.0, layers=list(LAYERS),
                sources=[dc_source(0.0, 0.0, 6.0, 0.0, 1.0, 1e16, 30, 60, 90)], stations=st, ntdec_w=1, ntdec_r=10)
    args.update(kw)
    return Params(**args)


def vonkarman_xi(shape, eps=0.05, seed=7):
    """Cheap seeded random field for tests (white noise smoothed once)."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(shape).astype(np.float32)
    for ax in range(3):
        x = (x + np.roll(x, 1, ax) + np.roll(x, -1, ax)) / 3
    x *= eps / max(float(x.std()), 1e-12)
    return x.astype(np.float32)


def small2d(kind="psv", nx=120, nz=60, na=10, nt=80, dx=0.25, dt=0.02, nm=3, seed=5, **kw) -> Params:
    """A small layered 2D run (P-SV: explosion + double couple; SH: mxy/myz)."""
    rng = np.random.default_rng(seed)
    xb = -nx // 2 * dx
    st = [Station(float(rng.uniform(xb + (na + 2) * dx, xb + (nx - na - 2) * dx)), 0.0,
                  0.0 if n < 3 else 2.0, f"s{n}", ["fsb", "obb", "oba", "dep", "dep"][n]) for n in range(5)]
    if kind == "psv":
        src = [Source(0.3, 0.0, 4.0, 0.0, 0.8, mo=1e15, mxx=1.0, mzz=0.7, mxz=0.4)]
    else:
        src = [Source(0.3, 0.0, 4.0, 0.0, 0.8, mo=1e15, mxy=1.0, myz=0.6)]
    args = dict(nx=nx, ny=1, nz=nz, nt=nt, dx=dx, dy=dx, dz=dx, dt=dt, na=na, nm=nm, xbeg=xb, ybeg=0.0,
                zbeg=-3 * dx, fq_min=0.05, fq_max=2.0, layers=list(LAYERS), sources=src, stations=st, ntdec_w=1,
                ntdec_r=10, sw_wav_u=True)
    args.update(kw)
    return Params(**args)
