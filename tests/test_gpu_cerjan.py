"""The Cerjan sponge (abc_type = 'cerjan', src/swpc_3d/m_absorb_c.f90)
against the oracle, bitwise.

In this mode the interior update covers the whole domain and the absorber
updates multiply each field by the sponge factors of its staggered
position (m_absorb.f90:43-75 dispatch, m_global.f90:349-378 kernel region).
"""
from __future__ import annotations

import numpy as np
import pytest

from openswpc_b200 import _lib
from openswpc_b200.params import Source
from openswpc_b200.swpc2d import Batch2D, Swpc2D
from openswpc_b200.swpc3d import Swpc3D
from oracle.oracle import Oracle2D, Oracle3D
from tests.models import small2d, small3d, vonkarman_xi
from tests.test_gpu_parity2d import compare as compare2d
from tests.test_gpu_parity2d import set_launch as set_launch2d
from tests.test_gpu_parity3d import compare_state, same_bits

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("launch", ["staged", "flat"])
def test_cerjan_run_matches_oracle_bitwise(launch):
    """Traces, V, S and the memory variables over the whole domain after a
    run with the sponge (free surface undamped, all other faces damped)."""
    p = small3d(nx=48, ny=44, nz=40, na=10, nt=60, abc_type="cerjan", sw_wav_u=True)
    xi = vonkarman_xi((p.ny + 6, p.nx + 6, p.nz + 6))
    g = Swpc3D(p, xi)
    if launch == "flat":
        _lib.check(g.ctx, g.lib.swpc_set_launch(g.ctx, 0, 1, 4, 2))
        _lib.check(g.ctx, g.lib.swpc_set_launch(g.ctx, 1, 1, 4, 2))
    o = Oracle3D(p, xi, threads=8)
    g.run(1, p.nt)
    o.run(1, p.nt, ntdec_r=p.ntdec_r)
    for what, comp in ((_lib.WAV_V, "v"), (_lib.WAV_U, "u")):
        a, b = g.waveforms(what), o.waveforms(comp)
        assert np.linalg.norm(b) > 0, comp
        assert same_bits(a, b), comp
    compare_state(g, o, p)
    # the sponge acted: the absorber holds less energy than without it
    assert np.abs(g.download(_lib.F_VX)[:, 3:13, :]).max() > 0


def test_cerjan_per_routine_calls_equal_graph_steps():
    """swpc_kernel_update_* then swpc_absorb_update_* (the sponge) equal the
    graph-captured step."""
    p = small3d(nx=40, ny=36, nz=32, na=8, nt=12, abc_type="cerjan")
    g0 = Swpc3D(p)
    g1 = Swpc3D(p)
    g0.run(1, p.nt)
    for it in range(1, p.nt + 1):
        g1.step(it)
    for f in list(range(_lib.F_VX, _lib.F_SXY + 1)) + [_lib.F_R + 2]:
        assert same_bits(g0.download(f), g1.download(f)), f


def test_cerjan_context_refuses_pml_adjoint_and_batch():
    p = small3d(nx=40, ny=36, nz=32, na=8, nt=4, abc_type="cerjan")
    g = Swpc3D(p)
    z = np.zeros(64, np.float32)
    rc = g.lib.swpc_absorb_setup(g.ctx, *(_lib.fptr(z) for _ in range(6)))
    assert rc == _lib.SWPC_ERR_STATE
    assert g.lib.swpc_adj_reset(g.ctx) == _lib.SWPC_ERR_STATE
    import ctypes as C

    b = C.c_void_p()
    assert g.lib.swpc_fbatch_create(g.ctx, 2, C.byref(b)) == _lib.SWPC_ERR_STATE


@pytest.mark.parametrize("launch", [(8, 8), (0, 0)], ids=["staged", "tiles"])
@pytest.mark.parametrize("kind", ["psv", "sh"])
def test_cerjan_2d_matches_oracle_bitwise(kind, launch):
    """P-SV and SH with the sponge (src/swpc_psv/m_absorb_c.f90,
    src/swpc_sh/m_absorb_c.f90): traces, fields, memory variables and the
    vmax report over the whole-domain kernel region."""
    p = small2d(kind, nt=100, abc_type="cerjan")
    g = Swpc2D(p, kind)
    set_launch2d(g, *launch)
    o = Oracle2D(p, kind)
    g.run(1, p.nt)
    o.run(1, p.nt)
    for what, comp in ((_lib.WAV_V, "v"), (_lib.WAV_U, "u")):
        a, b = g.waveforms(what), o.waveforms(comp)
        assert np.linalg.norm(b) > 0, comp
        assert same_bits(a, b), comp
    compare2d(g, o, p)
    vm = g.kernel__vmax()
    assert same_bits(vm, o.vmax()[:len(vm)])


@pytest.mark.parametrize("kind", ["psv", "sh"])
def test_cerjan_2d_body_force(kind):
    """Body forces with the sponge: P-SV applies them between the interior
    update and the sponge, SH after the sponge, as the reference does."""
    srcs = [Source(0.4, 0.0, 3.0, 0.0, 0.7, fx=1.0, fy=0.8, fz=-0.5),
            Source(-13.9, 0.0, 1.0, 0.1, 0.6, fx=0.3, fy=1.0, fz=1.0)]
    p = small2d(kind, nt=80, bf_mode=True, sources=srcs, abc_type="cerjan")
    g = Swpc2D(p, kind)
    o = Oracle2D(p, kind)
    g.run(1, p.nt)
    o.run(1, p.nt)
    assert np.linalg.norm(o.waveforms()) > 0
    assert same_bits(g.waveforms(), o.waveforms())
    compare2d(g, o, p)


@pytest.mark.parametrize("staged", [True, False])
@pytest.mark.parametrize("bf", [False, True])
@pytest.mark.parametrize("kind", ["psv", "sh"])
def test_cerjan_2d_batch_members_equal_independent_runs(kind, bf, staged):
    """A batch that mixes Cerjan and PML members of uneven size: every
    member's traces and fields equal its own independent run bitwise, with
    moment sources or body forces (P-SV applies them between the interior
    update and the sponge, SH after the sponge) and with the staged or the
    tile-walking batch kernels."""
    kw = {}
    if bf:
        kw = dict(bf_mode=True, sources=[Source(0.4, 0.0, 3.0, 0.0, 0.7, fx=1.0, fy=0.8, fz=-0.5),
                                         Source(-9.9, 0.0, 1.0, 0.1, 0.6, fx=0.3, fy=1.0, fz=1.0)])
    ps = [small2d(kind, nx=120, nz=60, nt=60, abc_type="cerjan", **kw),
          small2d(kind, nx=96, nz=72, nt=60, seed=9, **kw),
          small2d(kind, nx=140, nz=50, nt=60, seed=11, abc_type="cerjan", **kw)]
    members = [Swpc2D(p, kind) for p in ps]
    batch = Batch2D(members)
    if not staged:
        batch.set_staged(0, 0)
    batch.run(1, 60)
    for p in ps:
        g = Swpc2D(p, kind)
        g.run(1, 60)
        m = members[ps.index(p)]
        assert same_bits(m.waveforms(), g.waveforms())
        for fid in g.field_ids.values():
            assert same_bits(m.download(fid), g.download(fid)), fid
