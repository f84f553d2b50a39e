"""Parity at the benchmark configurations themselves, not only on small grids.

* The plain 3D forward run (192 x 192 x 96, dx = 0.5 km, dt = 0.02 s, PML 20,
  nt = 1000, the four-layer medium with nm = 3 over 0.05-2 Hz, one double
  couple 30/60/90 of M0 = 1e16 N m at 10 km depth, Kupper T = 2 s, 16
  seeded surface stations in 'fsb' mode) run to the end on the GPU and on the
  f32 oracle: traces, the final V, S, memory variables and PML auxiliaries
  bitwise (rel-L2 <= 1e-5 stated beside), the vmax reports every 50 steps,
  and the error of both against the all-double oracle reported.
* The large heterogeneous run's parameters (dx = 0.1 km, dt = 0.005 s, PML
  32, the von Karman medium with eps = 5 %, a = 5 km, kappa = 0.5, 8 double
  couples at seeded depths 5-15 km, surface stations) on a 160 x 160 x 200
  sub-grid for 400 steps, bitwise against the f32 oracle.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from bench import make_params
from openswpc_b200 import _lib
from openswpc_b200.media import vonkarman_3d
from openswpc_b200.swpc3d import Swpc3D
from oracle.oracle import Oracle3D
from tests.test_gpu_parity3d import REL_L2_TOL, VNAMES, compare_state, rel_l2, same_bits

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


def _traces_and_state(g, o, p):
    a, b = g.waveforms(_lib.WAV_V), o.waveforms("v")
    assert np.linalg.norm(b) > 0
    assert rel_l2(a, b) <= REL_L2_TOL, rel_l2(a, b)
    assert same_bits(a, b)
    compare_state(g, o, p)


def test_plain_forward_config_matches_oracle(record_property):
    p = make_params("c0")
    assert (p.nx, p.ny, p.nz, p.na, p.nt, len(p.sources), len(p.stations)) == (192, 192, 96, 20, 1000, 1, 16)
    assert all(st.zsw == "fsb" for st in p.stations) and p.sources[0].z == 10.0
    g = Swpc3D(p)
    o = Oracle3D(p, threads=THREADS)
    rg = g.run(1, p.nt)
    ro = o.run(1, p.nt, ntdec_r=p.ntdec_r)
    _traces_and_state(g, o, p)
    assert len(rg) == len(ro) == p.nt // p.ntdec_r
    for (ia, va), (ib, vb) in zip(rg, ro):
        assert ia == ib and same_bits(va, vb)
    o.close()
    # the error of the FP32 result against the all-double build of the scheme
    d = Oracle3D(p, variant="f64", threads=THREADS)
    d.run(1, p.nt, ntdec_r=p.ntdec_r)
    errs = {"traces_v": rel_l2(g.waveforms(_lib.WAV_V), d.waveforms("v"))}
    for n, name in enumerate(VNAMES):
        errs[name] = rel_l2(g.download(n), d.array(name))
    for k, v in errs.items():
        record_property(f"rel_l2_vs_f64_{k}", v)
    print("c0 FP32 error against the f64 oracle:", {k: f"{v:.2e}" for k, v in errs.items()})
    assert errs["traces_v"] < 1e-3


def large_run_subgrid(nx=160, ny=160, nz=200, nt=400, nst=64, seed=20241203):
    """The large heterogeneous run's physics on a smaller grid: same spacing,
    time step, PML width, medium statistics and source set (8 double couples
    at seeded xy inside the sub-grid and seeded depths 5-15 km)."""
    from openswpc_b200.params import Station

    p = make_params("c1")
    p.nx, p.ny, p.nz, p.nt = nx, ny, nz, nt
    p.xbeg, p.ybeg = -(nx // 2) * p.dx, -(ny // 2) * p.dy
    rng = np.random.default_rng(seed)
    lo, hi = (p.na + 10) * p.dx, (nx - p.na - 10) * p.dx
    for s in p.sources:
        s.x = float(p.xbeg + rng.uniform(lo, hi))
        s.y = float(p.ybeg + rng.uniform(lo, hi))
    lo, hi = (p.na + 2) * p.dx, (nx - p.na - 2) * p.dx
    p.stations = [Station(float(p.xbeg + rng.uniform(lo, hi)), float(p.ybeg + rng.uniform(lo, hi)), 0.0,
                          f"s{n:03d}", "fsb") for n in range(nst)]
    return p


def test_large_run_parameters_on_a_subgrid_match_oracle():
    p = large_run_subgrid()
    assert (p.dx, p.dt, p.na, len(p.sources)) == (0.1, 0.005, 32, 8)
    assert all(5.0 <= s.z <= 15.0 for s in p.sources)
    xi = vonkarman_3d((p.ny + 6, p.nx + 6, p.nz + 6), p.dx, p.dy, p.dz, 0.05, 5.0, 0.5, 5, "cuda:0")
    assert abs(float(xi.std()) - 0.05) < 5e-3
    g = Swpc3D(p, xi)
    o = Oracle3D(p, xi, threads=THREADS)
    g.run(1, p.nt)
    o.run(1, p.nt, ntdec_r=p.ntdec_r)
    _traces_and_state(g, o, p)
