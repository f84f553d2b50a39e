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


def dot_product(p, staged):
    """<L x, y> and <x, L^T y> on seeded random states x, y (every state
    cell of the domain; memory variables on the kernel region)."""
    xi = vonkarman_xi((p.ny + 6, p.nx + 6, p.nz + 6))
    g = Swpc3D(p, xi)
    lib, ctx = g.lib, g.ctx
    check(ctx, lib.swpc_set_launch(ctx, 8, 1, staged, 1))
    rng = np.random.default_rng(42)
    dom, ker = domain_mask(p), kernel_mask(p)
    shape = dom.shape
    ld_k, ld_i = p.nz + 6, p.nx + 6
    zero = np.float32(0.0)

    def rand(mask):
        return np.where(mask, rng.standard_normal(shape, dtype=np.float32), zero)

    check(ctx, lib.swpc_adj_reset(ctx))
    xe, ye = {}, {}
    for fid, kind in fields(p):
        mask = dom if kind != "ker" else ker
        g.upload(fid, rand(mask))
        check(ctx, lib.swpc_adj_upload(ctx, fid, fptr(rand(mask)), ld_k, ld_i))
        # the effective inputs (uploads keep only cells that are state)
        xe[fid] = g.download(fid)
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
        lhs += float(np.dot(Lx[mask].astype(np.float64), ye[fid][mask].astype(np.float64)))
        rhs += float(np.dot(xe[fid][mask].astype(np.float64), Lty[mask].astype(np.float64)))
    g.close()
    return lhs, rhs


@pytest.mark.parametrize("staged", [1, 0])
@pytest.mark.parametrize("nm", [3, 1])
def test_adjoint_dot_product(nm, staged):
    """staged: the TMA-staged stress-phase weights (1, the default) or the
    one-cell-per-thread kernel (0)."""
    lhs, rhs = dot_product(small3d(nx=36, ny=30, nz=28, na=6, nt=10, nm=nm), staged)
    assert abs(lhs - rhs) <= DOT_TOL * max(abs(lhs), abs(rhs)), (lhs, rhs)


def test_adjoint_dot_product_at_the_gradient_benchmark_grid():
    """The same identity on the gradient benchmark's grid: 256 x 256 x 128
    cells, PML 20, nm = 3, staged stress-phase weights."""
    lhs, rhs = dot_product(small3d(nx=256, ny=256, nz=128, na=20, nt=10, nm=3), 1)
    print("256x256x128 dot product:", lhs, rhs, abs(lhs - rhs) / max(abs(lhs), abs(rhs)))
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


def test_staged_adjoint_weights_give_the_bits_of_the_one_cell_kernel():
    """The gradient (misfit, the eight medium gradients, the final adjoint
    state) with the staged stress-phase weights equals, bit for bit, the
    gradient with the one-cell-per-thread kernel."""
    p, xi, obs = misfit_case()
    obsf = np.ascontiguousarray(obs, np.float32)
    shape = (p.ny + 6, p.nx + 6, p.nz + 6)
    runs = []
    for staged in (1, 0):
        g = Swpc3D(p, xi)
        check(g.ctx, g.lib.swpc_set_launch(g.ctx, 8, 1, staged, 1))
        J = C.c_double()
        check(g.ctx, g.lib.swpc_gradient(g.ctx, fptr(obsf), 16, C.byref(J)))
        grads = []
        for w in range(8):
            out = np.zeros(shape, np.float64)
            check(g.ctx, g.lib.swpc_gradient_fetch(g.ctx, w, out.ctypes.data_as(C.POINTER(C.c_double)), p.nz + 6,
                                                   p.nx + 6))
            grads.append(out)
        adj = []
        for fid, _ in fields(p):
            b = np.zeros(shape, np.float32)
            check(g.ctx, g.lib.swpc_adj_download(g.ctx, fid, fptr(b), p.nz + 6, p.nx + 6))
            adj.append(b)
        runs.append((J.value, grads, adj))
        g.close()
    (J1, g1, a1), (J0, g0, a0) = runs
    assert J1 == J0
    assert any(np.abs(x).max() > 0 for x in g1)
    for w, (x, y) in enumerate(zip(g1, g0)):
        assert np.array_equal(x.view(np.uint64), y.view(np.uint64)), w
    for (fid, _), x, y in zip(fields(p), a1, a0):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), fid


def _gradient_bits(g, p, obsf, ckpt):
    shape = (p.ny + 6, p.nx + 6, p.nz + 6)
    J = C.c_double()
    check(g.ctx, g.lib.swpc_gradient(g.ctx, fptr(obsf), ckpt, C.byref(J)))
    grads = []
    for w in range(8):
        out = np.zeros(shape, np.float64)
        check(g.ctx, g.lib.swpc_gradient_fetch(g.ctx, w, out.ctypes.data_as(C.POINTER(C.c_double)), p.nz + 6,
                                               p.nx + 6))
        grads.append(out)
    adj = []
    for fid, _ in fields(p):
        b = np.zeros(shape, np.float32)
        check(g.ctx, g.lib.swpc_adj_download(g.ctx, fid, fptr(b), p.nz + 6, p.nx + 6))
        adj.append(b)
    return J.value, grads, adj, g.waveforms(_lib.WAV_V)


@pytest.mark.parametrize("body_force", [False, True])
def test_gradient_with_kept_slots_gives_the_bits_of_the_full_recompute(body_force):
    """Steps of trailing segments kept from the first forward pass
    (swpc_gradient_set_slot_memory) replace their recompute: with room for
    none, for the short last segment, for three segments and for every
    segment, the misfit, the eight gradients, the final adjoint state and the
    traces are bit for bit those of the default, on one context and across
    budget changes.  Without body forces a kept step holds V on the shell of
    the kernel region only and the interior V is rebuilt from the kept
    divergences; with body forces (which write V) it holds the whole V."""
    if body_force:
        from openswpc_b200.params import Source
        srcs = [Source(0.2, -0.4, 5.0, 0.0, 1.0, fx=1.0, fy=0.5, fz=-2.0),
                Source(-2.0, 1.5, 3.0, 0.1, 0.8, fx=0.0, fy=1.0, fz=0.0)]
        p = small3d(nx=40, ny=36, nz=32, na=8, nt=70, bf_mode=True, sources=srcs)
        xi = vonkarman_xi((p.ny + 6, p.nx + 6, p.nz + 6))
        rng = np.random.default_rng(5)
        obs = None
    else:
        p, xi, obs = misfit_case()   # nt = 70, ckpt 16: segments of 16, 16, 16, 16 and 6 steps
    ref = Swpc3D(p, xi)
    if obs is None:
        obs = (rng.standard_normal((ref.nst, 3, p.nt)) * 1e-3).astype(np.float32)
    obsf = np.ascontiguousarray(obs, np.float32)
    J0, g0, a0, w0 = _gradient_bits(ref, p, obsf, 16)
    ref.close()
    assert any(np.abs(x).max() > 0 for x in g0)
    g = Swpc3D(p, xi)
    ck, st, sg, wk = (C.c_longlong() for _ in range(4))
    check(g.ctx, g.lib.swpc_gradient_memory(g.ctx, C.byref(ck), C.byref(st)))
    check(g.ctx, g.lib.swpc_gradient_segment_bytes(g.ctx, C.byref(sg), C.byref(wk), 16))
    assert ck.value > 0 and st.value > 0 and sg.value > 0 and wk.value > 0
    budgets = [6 * st.value + sg.value, 38 * st.value + 3 * sg.value, 70 * st.value + 5 * sg.value, 1 << 40, 0]
    for budget in budgets:   # kept steps: 6, 38, 70, 70, none
        check(g.ctx, g.lib.swpc_gradient_set_slot_memory(g.ctx, budget))
        J1, g1, a1, w1 = _gradient_bits(g, p, obsf, 16)
        assert J1 == J0, budget
        for w, (x, y) in enumerate(zip(g1, g0)):
            assert np.array_equal(x.view(np.uint64), y.view(np.uint64)), (budget, w)
        for (fid, _), x, y in zip(fields(p), a1, a0):
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), (budget, fid)
        assert np.array_equal(w1.view(np.uint32), w0.view(np.uint32)), budget
    assert g.lib.swpc_gradient_set_slot_memory(g.ctx, -1) == _lib.SWPC_ERR_ARG
    g.close()


@pytest.mark.parametrize("ntdec_w", [1, 3])
def test_velocity_weights_formed_in_the_stress_gather_give_the_same_bits(ntdec_w):
    """The velocity-phase weights formed inside the stress-phase gather of the
    step before (swpc_set_launch kernel 9, the default) against their own
    kernel in every step: same misfit, gradients, final adjoint state, bit for
    bit.  Stations share cells (i and i+1 neighbours, two at one point), one
    sits in the PML, and with ntdec_w = 3 residuals enter every third step
    only; with and without kept slots."""
    from openswpc_b200.params import Station
    p = small3d(nt=45, ntdec_w=ntdec_w)
    xb, yb = p.xbeg, p.ybeg
    extra = [Station(xb + 14.25, yb + 11.25, 2.0, "a", "dep"), Station(xb + 14.75, yb + 11.25, 2.0, "b", "dep"),
             Station(xb + 14.75, yb + 11.25, 2.0, "c", "dep"), Station(xb + 14.75, yb + 11.75, 2.5, "d", "dep"),
             Station(xb + 1.75, yb + 9.25, 4.0, "pml", "dep")]
    p.stations = list(p.stations) + extra
    xi = vonkarman_xi((p.ny + 6, p.nx + 6, p.nz + 6))
    runs = []
    for fuse, slots in ((0, 0), (1, 0), (1, 20)):
        g = Swpc3D(p, xi)
        check(g.ctx, g.lib.swpc_set_launch(g.ctx, 9, 1, fuse, 1))
        ck, sl = C.c_longlong(), C.c_longlong()
        check(g.ctx, g.lib.swpc_gradient_memory(g.ctx, C.byref(ck), C.byref(sl)))
        check(g.ctx, g.lib.swpc_gradient_set_slot_memory(g.ctx, slots * sl.value))   # some trailing segments
        rng = np.random.default_rng(3)
        obs = (rng.standard_normal((g.nst, 3, (p.nt - 1) // ntdec_w + 1)) * 1e-3).astype(np.float32)
        runs.append(_gradient_bits(g, p, obs, 10))
        g.close()
    J0, g0, a0, _ = runs[0]
    assert any(np.abs(x).max() > 0 for x in g0)
    for J1, g1, a1, _ in runs[1:]:
        assert J1 == J0
        for w, (x, y) in enumerate(zip(g1, g0)):
            assert np.array_equal(x.view(np.uint64), y.view(np.uint64)), w
        for (fid, _), x, y in zip(fields(p), a1, a0):
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), fid


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


def model_case(nt=70):
    """Observed data from a model with a slow Gaussian vs blob; the starting
    model is the layered + random background (both per-cell vp, vs, rho)."""
    from openswpc_b200.swpc3d import Medium, lhm_model
    p = small3d(nx=40, ny=36, nz=32, na=8, nt=nt)
    xi = vonkarman_xi((p.ny + 6, p.nx + 6, p.nz + 6))
    vp, vs, rho, qp, qs = lhm_model(p, xi)
    jj, ii, kk = np.meshgrid(np.arange(p.ny + 6), np.arange(p.nx + 6), np.arange(p.nz + 6), indexing="ij")
    blob = np.exp(-((jj - 21.0) ** 2 + (ii - 23.0) ** 2 + (kk - 19.0) ** 2) / (2 * 3.0 ** 2))
    vs_true = (vs * (1.0 - 0.08 * blob)).astype(np.float32)
    true = Swpc3D(p, medium=Medium.from_model(p, vp, vs_true, rho, qp, qs))
    true.run(1, p.nt)
    obs = true.waveforms(_lib.WAV_V)
    true.close()
    return p, (vp, vs, rho, qp, qs), obs


def oracle_misfit_double_traces(p, medium, obs, stations, scale):
    """Misfit of the all-double oracle with its velocity traces formed in
    double from its FP64 velocity fields (the oracle's own trace buffer is
    FP32, as wav__store's is, and its rounding would swamp the misfit change
    of a 1e-3 perturbation of a weakly sensitive cell).  The traces follow
    wav__store (m_wav.f90:530-535): the two-cell averages of V at the start
    of each step, times M0 UC 1e9, Vz positive up."""
    ist, jst, kst = (np.asarray(a) + 2 for a in stations)
    o = Oracle3D(p, variant="f64", threads=os.cpu_count() or 1, medium=medium)
    syn = np.zeros((len(ist), 3, p.nt))
    for it in range(1, p.nt + 1):
        vx, vy, vz = o.array("Vx"), o.array("Vy"), o.array("Vz")
        syn[:, 0, it - 1] = (vx[jst, ist, kst] + vx[jst, ist - 1, kst]) / 2 * scale
        syn[:, 1, it - 1] = (vy[jst, ist, kst] + vy[jst - 1, ist, kst]) / 2 * scale
        syn[:, 2, it - 1] = -(vz[jst, ist, kst] + vz[jst, ist, kst - 1]) / 2 * scale
        o.step(it)
    o.close()
    r = syn - obs
    return 0.5 * float(np.sum(r * r))


def seeded_cells(p, n, seed=11):
    """n distinct seeded cells of the solid kernel region, two or more cells
    inside its edges (whose medium also feeds the absorber)."""
    rng = np.random.default_rng(seed)
    cells = set()
    while len(cells) < n:
        j = int(rng.integers(p.na + 3, p.ny - p.na - 1))
        i = int(rng.integers(p.na + 3, p.nx - p.na - 1))
        k = int(rng.integers(6, p.nz - p.na - 1))
        cells.add((j + 2, i + 2, k + 2))   # memory-box array index of cell (k, i, j)
    return sorted(cells)


def test_model_gradient_matches_finite_differences_on_20_seeded_cells():
    """dJ/dvp, dJ/dvs, dJ/drho on 20 seeded cells against central differences
    (h = 1e-3 relative) of the all-double oracle's misfit, the medium
    re-derived from the perturbed model each time."""
    from openswpc_b200.adjoint import Misfit3D
    from openswpc_b200.swpc3d import Medium
    p, (vp, vs, rho, qp, qs), obs = model_case()
    prob = Misfit3D(p, vp, vs, rho, qp, qs, obs, ckpt=16)
    J, gvp, gvs, grho = prob.gradient(vp, vs, rho)
    assert abs(J - prob.misfit(vp, vs, rho)) <= 1e-6 * J
    sv = prob.solver
    stations = (sv.ist, sv.jst, sv.kst)
    scale = float(np.float32(sv.M0)) * float(np.float32(sv.UC)) * 1e9
    prob.close()
    model = {"vp": vp, "vs": vs, "rho": rho}
    grads = {"vp": gvp, "vs": gvs, "rho": grho}
    rows = []
    for idx in seeded_cells(p, 20):
        for name in ("vp", "vs", "rho"):
            arr = model[name]
            v0 = float(arr[idx])
            h = 1e-3 * abs(v0)
            Js = []
            for sgn in (1.0, -1.0):
                arr[idx] = np.float32(v0 + sgn * h)
                m = Medium.from_model(p, vp, vs, rho, qp, qs)
                Js.append(oracle_misfit_double_traces(p, m, obs, stations, scale))
            arr[idx] = np.float32(v0)
            step = (float(np.float32(v0 + h)) - v0) + (v0 - float(np.float32(v0 - h)))
            rows.append((name, idx, float(grads[name][idx]), (Js[0] - Js[1]) / step))
    # FD_TOL relative to each cell's own derivative; a cell whose derivative
    # is below 1 % of the largest of its parameter is held to FD_TOL of 1 %
    # of that largest value (the FD noise floor of the FP32 medium setup)
    scale = {n: max(abs(r[3]) for r in rows if r[0] == n) for n in model}
    bad = [r for r in rows if abs(r[2] - r[3]) > FD_TOL * max(abs(r[3]), 1e-2 * scale[r[0]])]
    worst = max(abs(r[2] - r[3]) / max(abs(r[3]), 1e-2 * scale[r[0]]) for r in rows)
    print(f"misfit {J:.6e}; worst relative gradient error over 60 checks {worst:.2e}")
    assert not bad, bad


def test_waveform_misfit_autograd():
    """torch.autograd through WaveformMisfit gives the library's gradient and
    the forward misfit; without grad the forward alone runs."""
    import torch
    from openswpc_b200.adjoint import Misfit3D, waveform_misfit
    p, (vp, vs, rho, qp, qs), obs = model_case(nt=40)
    prob = Misfit3D(p, vp, vs, rho, qp, qs, obs, ckpt=8)
    tv = [torch.tensor(a, requires_grad=True) for a in (vp, vs, rho)]
    J = waveform_misfit(*tv, prob)
    (2.0 * J).backward()
    J_ref, gvp, gvs, grho = prob.gradient(vp, vs, rho)
    assert abs(float(J) - J_ref) <= 1e-12 * J_ref
    for t, g in zip(tv, (gvp, gvs, grho)):
        assert t.grad.dtype == torch.float32
        np.testing.assert_allclose(t.grad.numpy(), (2.0 * g).astype(np.float32), rtol=1e-6, atol=0)
    with torch.no_grad():
        J2 = waveform_misfit(*[t.detach() for t in tv], prob)
    assert abs(float(J2) - J_ref) <= 1e-6 * J_ref
    prob.close()


@pytest.mark.parametrize("stabilize", [False, True])
def test_waveform_misfit_from_cuda_tensors_stays_on_the_device(stabilize):
    """A model given as CUDA tensors is set up and differentiated in HBM
    (swpc_vmodel_velocity_device, swpc_gradient_model_device): the misfit and
    the three gradients are bitwise those of the same model from host
    arrays, and the gradients come back as CUDA tensors."""
    import torch
    from openswpc_b200.adjoint import Misfit3D, waveform_misfit
    p, (vp, vs, rho, qp, qs), obs = model_case(nt=40)
    p.stabilize_pml = stabilize
    prob = Misfit3D(p, vp, vs, rho, qp, qs, obs, ckpt=8)
    J_ref, gvp, gvs, grho = prob.gradient(vp, vs, rho)
    tv = [torch.tensor(a, device="cuda:0", requires_grad=True) for a in (vp, vs, rho)]
    J = waveform_misfit(*tv, prob)
    J.backward()
    assert J.is_cuda and float(J) == J_ref
    for t, g in zip(tv, (gvp, gvs, grho)):
        assert t.grad.is_cuda and t.grad.dtype == torch.float32
        assert np.array_equal(t.grad.cpu().numpy(), g.astype(np.float32))
    J_dev, *g_dev = prob.gradient(*[t.detach() for t in tv])
    assert J_dev == J_ref
    for a, b in zip(g_dev, (gvp, gvs, grho)):
        assert a.is_cuda and a.dtype == torch.float64
        assert np.array_equal(a.cpu().numpy().view(np.uint64), b.view(np.uint64))
    prob.close()


def _recorders(g, ig):
    """Everything the recorders of a run hold: velocity, displacement,
    stress and strain traces, green__store's Green's functions."""
    out = [g.waveforms(w) for w in (_lib.WAV_V, _lib.WAV_U, _lib.WAV_STRESS, _lib.WAV_STRAIN)]
    return out + [g.green_functions()]


def test_recorders_after_gradient_and_reset_equal_a_plain_run():
    """The gradient's recompute advances the wavefield without recording, and
    swpc_reset_state clears every recorder total, so traces and Green's
    functions after either equal those of one plain run from rest, bitwise."""
    p = small3d(nt=40, sw_wav_u=True, sw_wav_stress=True, sw_wav_strain=True)
    xi = vonkarman_xi((p.ny + 6, p.nx + 6, p.nz + 6))
    rng = np.random.default_rng(8)
    ig, jg, kg = (rng.integers(p.na + 2, n - p.na - 2, 16) for n in (p.nx, p.ny, p.nz))
    plain = Swpc3D(p, xi)
    plain.green_store_setup(ig, jg, kg, bforce=True)
    plain.run(1, p.nt)
    ref = _recorders(plain, ig)
    assert all(np.abs(a).max() > 0 for a in ref)
    # a second run from rest on the same context
    check(plain.ctx, plain.lib.swpc_reset_state(plain.ctx))
    plain.run(1, p.nt)
    again = _recorders(plain, ig)
    for a, b in zip(again, ref):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    # the gradient: forward, then checkpointed recompute of every segment
    g = Swpc3D(p, xi)
    g.green_store_setup(ig, jg, kg, bforce=True)
    obs = np.zeros_like(ref[0])
    J = C.c_double()
    check(g.ctx, g.lib.swpc_gradient(g.ctx, fptr(obs), 16, C.byref(J)))
    after = _recorders(g, ig)
    for a, b in zip(after, ref):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
