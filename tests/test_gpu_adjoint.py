"""Discrete adjoint of the 3D step and the misfit gradient.

* dot-product test: <L x, y> = <x, L^T y> for the linear step L (stress then
  velocity update, interior + memory variables + PML, sources off) on random
  states, to FP32 rounding;
* finite differences: the gradient of the L2 velocity misfit with respect to
  single medium values (lam, mu, mu_yz, b_x, ...) against central
  differences of the misfit of the all-double oracle."""
import ctypes as C
import os

import numpy as np
import pytest

from openswpc_b200 import _lib
from openswpc_b200._lib import check, fptr
from openswpc_b200.swpc3d import Swpc3D
from oracle.oracle import Oracle3D
from tests.models import small3d, vonkarman_xi

pytestmark = pytest.mark.gpu

DOT_TOL = 1e-5     # relative mismatch of the two inner products (FP32 arithmetic)
FD_TOL = 1e-3      # relative gradient error against central differences


def domain_mask(p):
    m = np.zeros((p.ny + 6, p.nx + 6, p.nz + 6), bool)
    m[3:-3, 3:-3, 3:-3] = True
    return m


def kernel_mask(p):
    m = np.zeros((p.ny + 6, p.nx + 6, p.nz + 6), bool)
    m[3 + p.na:p.ny + 3 - p.na, 3 + p.na:p.nx + 3 - p.na, 3:p.nz + 3 - p.na] = True
    return m


def fields(p):
    out = [(_lib.F_VX + c, "dom") for c in range(3)] + [(_lib.F_SXX + c, "dom") for c in range(6)]
    out += [(_lib.F_R + 3 * c + m, "ker") for c in range(6) for m in range(p.nm)]
    out += [(_lib.F_AUX + q, "aux") for q in range(18)]
    return out


@pytest.mark.parametrize("nm", [3, 1])
def test_adjoint_dot_product(nm):
    p = small3d(nx=36, ny=30, nz=28, na=6, nt=10, nm=nm)
    xi = vonkarman_xi((p.ny + 6, p.nx + 6, p.nz + 6))
    g = Swpc3D(p, xi)
    lib, ctx = g.lib, g.ctx
    rng = np.random.default_rng(42)
    dom, ker = domain_mask(p), kernel_mask(p)
    shape = dom.shape
    ld_k, ld_i = p.nz + 6, p.nx + 6
    x, y = {}, {}
    for fid, kind in fields(p):
        mask = dom if kind != "ker" else ker
        x[fid] = np.where(mask, rng.standard_normal(shape), 0.0).astype(np.float32)
        y[fid] = np.where(mask, rng.standard_normal(shape), 0.0).astype(np.float32)
    check(ctx, lib.swpc_adj_reset(ctx))
    for fid, _ in fields(p):
        g.upload(fid, x[fid])
        check(ctx, lib.swpc_adj_upload(ctx, fid, fptr(y[fid]), ld_k, ld_i))
    # the effective inputs (uploads keep only cells that are state)
    xe = {fid: g.download(fid) for fid, _ in fields(p)}
    ye = {}
    for fid, _ in fields(p):
        b = np.zeros(shape, np.float32)
        check(ctx, lib.swpc_adj_download(ctx, fid, fptr(b), ld_k, ld_i))
        ye[fid] = b
    check(ctx, lib.swpc_update_stress(ctx))
    check(ctx, lib.swpc_update_vel(ctx))
    check(ctx, lib.swpc_adj_step_linear(ctx))
    lhs = rhs = 0.0
    for fid, kind in fields(p):
        mask = dom if kind != "ker" else ker
        Lx = g.download(fid)
        Lty = np.zeros(shape, np.float32)
        check(ctx, lib.swpc_adj_download(ctx, fid, fptr(Lty), ld_k, ld_i))
        lhs += float(np.sum(Lx[mask].astype(np.float64) * ye[fid][mask]))
        rhs += float(np.sum(xe[fid][mask].astype(np.float64) * Lty[mask]))
    assert abs(lhs - rhs) <= DOT_TOL * max(abs(lhs), abs(rhs)), (lhs, rhs)


def misfit_case():
    p = small3d(nx=40, ny=36, nz=32, na=8, nt=70)
    xi = vonkarman_xi((p.ny + 6, p.nx + 6, p.nz + 6))
    # "observed" data: the same run in a medium with a slower blob
    true = Swpc3D(p, xi)
    m = true.medium
    blob = np.zeros_like(m.mu)
    blob[14:24, 16:26, 14:22] = 1.0
    for f in ("lam", "mu", "muyz", "muxz", "muxy"):
        setattr(m, f, (getattr(m, f) * (1.0 - 0.06 * blob)).astype(np.float32))
    check(true.ctx, true.lib.swpc_upload_medium(true.ctx, C.byref(m.view())))
    true.run(1, p.nt)
    obs = true.waveforms(_lib.WAV_V)
    true.close()
    return p, xi, obs


def forward_misfit(g, p, obs):
    check(g.ctx, g.lib.swpc_upload_medium(g.ctx, C.byref(g.medium.view())))
    for fid in range(9):
        g.upload(fid, np.zeros((p.ny + 6, p.nx + 6, p.nz + 6), np.float32))
    for fid in [_lib.F_R + 3 * c + m for c in range(6) for m in range(p.nm)] + [_lib.F_AUX + q for q in range(18)]:
        g.upload(fid, np.zeros((p.ny + 6, p.nx + 6, p.nz + 6), np.float32))
    g.run(1, p.nt)
    r = g.waveforms(_lib.WAV_V).astype(np.float64) - obs
    return 0.5 * float(np.sum(r * r))


def oracle_misfit(p, medium, obs):
    o = Oracle3D(p, variant="f64", threads=os.cpu_count() or 1, medium=medium)
    o.run(1, p.nt)
    r = o.waveforms("v").astype(np.float64) - obs
    o.close()
    return 0.5 * float(np.sum(r * r))


def test_gradient_matches_finite_differences():
    p, xi, obs = misfit_case()
    g = Swpc3D(p, xi)
    J = C.c_double()
    obsf = np.ascontiguousarray(obs, np.float32)
    check(g.ctx, g.lib.swpc_gradient(g.ctx, fptr(obsf), 16, C.byref(J)))
    J0 = forward_misfit(g, p, obs)
    assert abs(J.value - J0) <= 1e-6 * J0
    names = ["lam", "mu", "muyz", "muxz", "muxy", "bx", "by", "bz"]
    grads = {}
    for w, n in enumerate(names):
        out = np.zeros((p.ny + 6, p.nx + 6, p.nz + 6), np.float64)
        check(g.ctx, g.lib.swpc_gradient_fetch(g.ctx, w, out.ctypes.data_as(C.POINTER(C.c_double)), p.nz + 6,
                                               p.nx + 6))
        grads[n] = out
    ker = kernel_mask(p)
    rows = []
    for n in names:
        arr = getattr(g.medium, n)
        solid = g.medium.mu > 0   # below the air layer
        gr = np.where(ker & solid & (arr != 0), np.abs(grads[n]), 0.0)
        idx = np.unravel_index(np.argmax(gr), gr.shape)   # the most sensitive solid cell of each field
        v0 = float(arr[idx])
        # central differences of the all-double oracle's misfit (free of FP32
        # rounding) at relative steps 1e-2 and 5e-3, combined by Richardson
        # extrapolation, which removes the O(h^2) term
        def central(rel):
            h = rel * abs(v0)
            Js = []
            for sgn in (1.0, -1.0):
                arr[idx] = np.float32(v0 + sgn * h)
                Js.append(oracle_misfit(p, g.medium, obs))
            arr[idx] = np.float32(v0)
            hp = float(np.float32(v0 + h)) - v0
            hm = v0 - float(np.float32(v0 - h))
            return (Js[0] - Js[1]) / (hp + hm)
        fd = (4 * central(5e-3) - central(1e-2)) / 3
        rows.append((n, idx, grads[n][idx], fd))
    bad = [r for r in rows if abs(r[2] - r[3]) > FD_TOL * abs(r[3])]
    print("misfit", J0, "gradient vs central differences:",
          [(r[0], float(r[2]), float(r[3]), abs(float(r[2]) / float(r[3]) - 1)) for r in rows])
    assert not bad, bad
