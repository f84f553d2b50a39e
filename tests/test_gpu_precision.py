"""Reduced-precision storage forms of the 3D step (BF16 memory variables;
FP16 memory variables; FP16 stress and memory variables; the FP16 arrays with
per-array power-of-two scales).  The
arithmetic stays FP32, so each form is checked against the FP32 form and
against the all-double oracle with a stated tolerance, and the error is
recorded."""
import numpy as np
import pytest

from openswpc_b200 import _lib
from openswpc_b200.swpc3d import Swpc3D
from oracle.oracle import Oracle3D
from tests.models import small3d, vonkarman_xi

pytestmark = pytest.mark.gpu

# rel-L2 bars of the reduced forms against the f64 oracle after 80 steps:
# BF16 keeps 8 significand bits (2^-9 relative rounding) for R, FP16 keeps 11
# (2^-12) for S and R; both stay far below 1e-2 on this case
TOL = {"f32": 1e-5, "bf16r": 1e-2, "f16r": 1e-3, "f16sr": 1e-2}


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def reference():
    p = small3d(nt=80, sw_wav_stress=True)
    xi = vonkarman_xi((p.ny + 6, p.nx + 6, p.nz + 6))
    o = Oracle3D(p, xi, variant="f64")
    o.run(1, p.nt)
    return p, xi, o


@pytest.mark.parametrize("form", ["f32", "bf16r", "f16r", "f16sr"])
def test_precision_form_error_against_f64(form, reference, record_property):
    p, xi, o = reference
    g = Swpc3D(p, xi, precision=form)
    g.run(1, p.nt)
    errs = {"traces_v": rel_l2(g.waveforms(_lib.WAV_V), o.waveforms("v")),
            "traces_stress": rel_l2(g.waveforms(_lib.WAV_STRESS), o.waveforms("stress"))}
    for n, name in enumerate(("Vx", "Vy", "Vz")):
        errs[name] = rel_l2(g.download(n), o.array(name))
    for k, v in errs.items():
        record_property(f"{form}_rel_l2_vs_f64_{k}", v)
    print(form, "rel-L2 against the f64 oracle:", errs)
    assert all(v < TOL[form] for v in errs.values()), errs
    if form != "f32":
        # the reduced form differs from FP32 (it really stores fewer bits)
        f = Swpc3D(p, xi)
        f.run(1, p.nt)
        assert rel_l2(g.download(0), f.download(0)) > 0


def test_reduced_storage_roundtrip_and_rescale():
    """Upload/download through FP16 storage rounds to FP16; re-centring is
    idempotent; a field pushed out of its window is re-centred with its values
    kept; the run goes on as without the forced move."""
    p = small3d(nt=40)
    g = Swpc3D(p, precision="f16sr")
    g.run(1, 30)   # the loop re-centres the scales every 8 steps; the wave still grows in between
    g.rescale()
    assert g.rescale() == 0   # a second call finds every array centred
    before = [g.download(_lib.F_SXX + c) for c in range(6)]
    r_before = g.download(_lib.F_R + 0)
    # every stress 16 times larger: the group's stored maximum leaves the window [2^3, 2^10)
    assert np.abs(before[0]).max() > 0
    for c in range(6):
        g.upload(_lib.F_SXX + c, before[c] * np.float32(16.0))
    d1 = [g.download(_lib.F_SXX + c) for c in range(6)]
    assert g.rescale() == 6   # the six stress arrays move together (one scale per group)
    d2 = [g.download(_lib.F_SXX + c) for c in range(6)]
    for a, b in zip(d1, d2):
        # exact unless a value fell into the FP16 subnormal range
        assert np.abs(a - b).max() <= np.abs(a).max() * 2.0 ** -20
    assert g.rescale() == 0   # centred
    for c in range(6):   # the run's own values again (exact: a power-of-two change of scale)
        g.upload(_lib.F_SXX + c, before[c])
    after = [g.download(_lib.F_SXX + c) for c in range(6)]
    for a, b in zip(before, after):
        assert np.abs(a - b).max() <= np.abs(a).max() * 2.0 ** -20
    assert np.abs(g.download(_lib.F_R + 0) - r_before).max() <= np.abs(r_before).max() * 2.0 ** -20
    # the run continues correctly: same as a run without the uploads
    h = Swpc3D(p, precision="f16sr")
    h.run(1, 30)
    g.run(31, 10)
    h.run(31, 10)
    assert rel_l2(g.download(0), h.download(0)) < 1e-2
    # upload of FP32 values rounds them to FP16 on the device
    # values of the field's own magnitude, so that they fit its current scale
    x = (np.random.default_rng(3).standard_normal(before[0].shape) * np.abs(before[0]).max()).astype(np.float32)
    g.upload(_lib.F_SXX, x)
    y = g.download(_lib.F_SXX)
    inner = (slice(3, -3), slice(3, -3), slice(3, -3))
    assert np.abs(y[inner] - x[inner]).max() <= np.abs(x).max() * 2.0 ** -10


@pytest.mark.parametrize("nm,grid", [(3, (40, 36, 32)), (1, (42, 38, 45)), (0, (42, 38, 45)), (2, (40, 36, 32))])
@pytest.mark.parametrize("form", ["bf16r", "f16r", "f16sr"])
def test_staged_reduced_forms_equal_the_flat_kernels(form, nm, grid):
    """The TMA-staged kernels of the reduced storage forms (2-byte tiles of S
    and R) give the bits of the one-cell kernels of the same form: traces,
    wavefield, memory variables and PML auxiliaries; tiles partial in k, i
    and j, and tiles without interior cells, included."""
    nx, ny, nz = grid
    p = small3d(nx=nx, ny=ny, nz=nz, nt=50, nm=nm, sw_wav_stress=True)
    xi = vonkarman_xi((p.ny + 6, p.nx + 6, p.nz + 6))
    staged = Swpc3D(p, xi, precision=form)   # the default launch
    flat = Swpc3D(p, xi, precision=form)
    _lib.check(flat.ctx, flat.lib.swpc_set_launch(flat.ctx, 0, 2, 2, 1))
    _lib.check(flat.ctx, flat.lib.swpc_set_launch(flat.ctx, 1, 4, 2, 2))
    staged.run(1, p.nt)
    flat.run(1, p.nt)
    for what in (_lib.WAV_V, _lib.WAV_STRESS):
        a, b = staged.waveforms(what), flat.waveforms(what)
        assert np.linalg.norm(b) > 0
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), what
    fields = list(range(9)) + [_lib.F_R + 3 * c + m for c in range(6) for m in range(nm)] + \
        [_lib.F_AUX + q for q in range(18)]
    for fid in fields:
        a, b = staged.download(fid), flat.download(fid)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), fid


@pytest.mark.parametrize("form", ["bf16r", "f16r", "f16sr"])
def test_reduced_forms_on_every_compiled_staged_tile(form):
    """The reduced forms compile stress and velocity tiles (4, 4) and (4, 2):
    each combination gives the bits of the flat kernels."""
    p = small3d(nx=42, ny=38, nz=45, nt=30, nm=3, sw_wav_stress=True)
    xi = vonkarman_xi((p.ny + 6, p.nx + 6, p.nz + 6))
    flat = Swpc3D(p, xi, precision=form)
    _lib.check(flat.ctx, flat.lib.swpc_set_launch(flat.ctx, 0, 2, 2, 1))
    _lib.check(flat.ctx, flat.lib.swpc_set_launch(flat.ctx, 1, 4, 2, 2))
    flat.run(1, p.nt)
    ref = [flat.download(fid) for fid in range(9)]
    for sbj, vbj in ((4, 2), (2, 4), (4, 4), (2, 2)):
        g = Swpc3D(p, xi, precision=form)
        _lib.check(g.ctx, g.lib.swpc_set_launch(g.ctx, 5, 1, 4, sbj))
        _lib.check(g.ctx, g.lib.swpc_set_launch(g.ctx, 6, 1, 4, vbj))
        g.run(1, p.nt)
        for fid in range(9):
            a = g.download(fid)
            assert np.array_equal(a.view(np.uint32), ref[fid].view(np.uint32)), (sbj, vbj, fid)
        g.close()


def test_f16r_keeps_stress_in_fp32_and_rescales_memory_variables():
    """FP16 memory variables with FP32 stress: uploads of S keep every bit,
    R rounds to FP16, and a rescale centres the R scales only."""
    p = small3d(nt=40)
    g = Swpc3D(p, precision="f16r")
    g.run(1, 30)
    x = np.random.default_rng(5).standard_normal((p.ny + 6, p.nx + 6, p.nz + 6)).astype(np.float32)
    inner = (slice(3, -3), slice(3, -3), slice(3, -3))
    g.upload(_lib.F_SXX, x)
    assert np.array_equal(g.download(_lib.F_SXX)[inner].view(np.uint32), x[inner].view(np.uint32))
    r = g.download(_lib.F_R)
    big = np.abs(r).max()
    assert big > 0
    g.rescale()
    assert g.rescale() == 0
    assert np.abs(g.download(_lib.F_R) - r).max() <= big * 2.0 ** -20
