"""The medium built on the device against the host setup.

swpc_vmodel_lhm_device / swpc_vmodel_upload followed by
swpc_medium_setup_device must give the fields, integer maps, relaxation
times and velocity range of swpc_vmodel_lhm + swpc_setup_medium (which the
CPU tests pin against the oracle) bit for bit, and runs on the two media
must agree bitwise.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from openswpc_b200 import _lib
from openswpc_b200._lib import fptr
from openswpc_b200.params import Layer
from openswpc_b200.swpc3d import Medium, Swpc3D, grid_struct
from tests.models import LAYERS, small3d, vonkarman_xi

pytestmark = pytest.mark.gpu

# water (vs = 0: no vcheck, ocean-bottom detection, harmonic means over zero
# rigidity), a slow layer that the velocity cut-off replaces, then the
# four-layer model
OCEAN = [Layer(0.0, 1.0, 1.5, 0.0, 1e6, 1e6), Layer(1.0, 2.0, 2.0, 0.8, 100, 50)] + \
        [Layer(l.depth + 2.0, l.rho, l.vp, l.vs, l.qp, l.qs) for l in LAYERS]


def same_bits(a, b):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return np.array_equal(a.view(np.uint32), b.view(np.uint32))


def check_same_medium(g, dm, m):
    for q, name in enumerate(Medium.FIELDS[1:], start=1):
        assert same_bits(g.download(_lib.F_MED + q), getattr(m, name)), name
    for name in Medium.MAPS:
        assert np.array_equal(getattr(dm, name), getattr(m, name)), name
    assert same_bits(dm.ts, m.ts)
    assert same_bits(np.array([dm.zeta, dm.vmin, dm.vmax]), np.array([m.zeta, m.vmin, m.vmax]))


def run_and_compare(p, g0, g1, steps):
    for it in range(1, steps + 1):
        g0.step(it)
        g1.step(it)
    for f in list(range(_lib.F_VX, _lib.F_SXY + 1)) + [_lib.F_R, _lib.F_R + 17]:
        assert same_bits(g0.download(f), g1.download(f)), f


# a 1 km low-velocity layer at 3 km depth and a slow top layer, for stabilize_pml
SLOW = [Layer(0.0, 2.2, 2.4, 1.2, 100, 50), Layer(1.0, 2.7, 5.5, 3.2, 300, 150),
        Layer(3.0, 2.4, 3.0, 1.6, 100, 50), Layer(4.0, 2.7, 5.5, 3.2, 300, 150)] + LAYERS[1:]


@pytest.mark.parametrize("case", ["layers", "perturbed", "ocean_clipped", "seawater_munk", "stabilize_pml"])
def test_device_medium_equals_host_setup(case):
    """vmodel_lhm (+ lhm_rmed) and medium__setup in HBM: every field over the
    memory box, the six maps, ts, zeta and the velocity range equal the host
    setup; a run on each agrees bitwise.  "ocean_clipped" adds a water layer,
    a layer removed by vcut and a perturbation strong enough for both vcheck
    bounds and the density floor."""
    kw = {}
    if case == "ocean_clipped":
        kw = dict(layers=OCEAN, vcut=1.0, rhomin=2.75)
    elif case == "stabilize_pml":
        # stabilize_absorber (m_medium.f90:276-340) on the device against the host's
        kw = dict(layers=SLOW, stabilize_pml=True)
    elif case == "seawater_munk":
        # seawater of Munk's profile between z = 0 and depth(1) = 1.8 km (m_vmodel_lhm.f90:123-133)
        kw = dict(layers=[Layer(1.8, 2.7, 5.5, 3.2, 300, 150)] + list(LAYERS[1:]), munk_profile=True)
    p = small3d(nx=56, ny=48, nz=44, na=8, nt=8, **kw)
    shape = (p.ny + 6, p.nx + 6, p.nz + 6)
    xi = None
    if case in ("perturbed", "stabilize_pml"):
        xi = vonkarman_xi(shape)
    elif case == "ocean_clipped":
        xi = vonkarman_xi(shape, eps=0.25, seed=11)
    m = Medium(p, xi)
    if case == "ocean_clipped":
        # the model reaches the velocity ceiling, the velocity floor and the
        # density floor of vcheck
        raw = host_vmodel(p, xi)
        vp = np.sqrt((raw["lam"] + 2 * raw["mu"]) / raw["rho"])
        vs = np.sqrt(raw["mu"] / raw["rho"])
        vmax_r = 6.0 / 7.0 * (1.0 / np.sqrt(3.0 / p.dx ** 2)) / p.dt
        assert np.any(np.isclose(vp, vmax_r, rtol=1e-5)) and float(vp.max()) <= vmax_r * (1 + 1e-5)
        assert np.any(np.isclose(vs, p.vcut, rtol=1e-5))
        assert np.any(raw["rho"] == np.float32(p.rhomin))
    g0 = Swpc3D(p, medium=m)
    g1 = Swpc3D(p, xi, medium_on_device=True)
    check_same_medium(g1, g1.medium, m)
    run_and_compare(p, g0, g1, p.nt)


def test_device_medium_from_a_device_perturbation():
    """xi given as a CUDA tensor (a field generated on the GPU) gives the same
    medium as the host array."""
    import torch

    p = small3d(nx=40, ny=36, nz=32, na=8, nt=4)
    xi = vonkarman_xi((p.ny + 6, p.nx + 6, p.nz + 6))
    m = Medium(p, xi)
    g = Swpc3D(p, torch.from_numpy(xi).cuda(), medium_on_device=True)
    check_same_medium(g, g.medium, m)


def host_vmodel(p, xi):
    """The host vmodel_lhm output (rho, lam, mu, qp, qs) before the setup."""
    lib = _lib.load()
    shape = (p.ny + 6, p.nx + 6, p.nz + 6)
    raw = {n: np.zeros(shape, np.float32) for n in ("rho", "lam", "mu", "qp", "qs")}
    L = p.layers
    arr = lambda a: np.array([getattr(l, a) for l in L], np.float32)
    xp = fptr(np.ascontiguousarray(xi, np.float32)) if xi is not None else None
    assert lib.swpc_vmodel_lhm(C.byref(grid_struct(p)), len(L), fptr(arr("depth")), fptr(arr("rho")),
                               fptr(arr("vp")), fptr(arr("vs")), fptr(arr("qp")), fptr(arr("qs")), p.vcut,
                               xp, p.rhomin, *(fptr(raw[n]) for n in ("rho", "lam", "mu", "qp", "qs"))) == 0
    return raw


def test_setup_of_an_uploaded_model():
    """swpc_vmodel_upload of the host vmodel output, then the setup on the
    device, equals the host setup of the same model."""
    p = small3d(nx=40, ny=36, nz=32, na=8, nt=4)
    shape = (p.ny + 6, p.nx + 6, p.nz + 6)
    xi = vonkarman_xi(shape)
    lib = _lib.load()
    raw = host_vmodel(p, xi)
    m = Medium(p, xi)
    g = Swpc3D(p, medium=m)
    _lib.check(g.ctx, lib.swpc_vmodel_upload(g.ctx, *(fptr(raw[n]) for n in ("rho", "lam", "mu", "qp", "qs")),
                                             p.nz + 6, p.nx + 6))
    maps = {n: np.zeros(shape[:2], np.int32) for n in Medium.MAPS}
    ts = np.zeros(3, np.float32)
    scal = np.zeros(3, np.float32)
    _lib.check(g.ctx, lib.swpc_medium_setup_device(g.ctx, p.fq_min, p.fq_max, p.fq_ref, fptr(ts), fptr(scal),
                                                   *(_lib.iptr(maps[n]) for n in Medium.MAPS), p.nx + 6))
    for q, name in enumerate(Medium.FIELDS[1:], start=1):
        assert same_bits(g.download(_lib.F_MED + q), getattr(m, name)), name
    for n in Medium.MAPS:
        assert np.array_equal(maps[n], getattr(m, n)), n
    assert same_bits(ts, m.ts)
    assert same_bits(scal, np.array([m.zeta, m.vmin, m.vmax], np.float32))


def test_setup_without_a_model_is_refused():
    p = small3d(nx=40, ny=36, nz=32, na=8, nt=4)
    g = Swpc3D(p)
    lib = g.lib
    ts = np.zeros(3, np.float32)
    scal = np.zeros(3, np.float32)
    rc = lib.swpc_medium_setup_device(g.ctx, p.fq_min, p.fq_max, p.fq_ref, fptr(ts), fptr(scal), None, None, None,
                                      None, None, None, None, 0)
    assert rc == _lib.SWPC_ERR_STATE
