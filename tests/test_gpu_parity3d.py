"""GPU parity of the 3D time step against the CPU oracle (f32 build).

The CUDA kernels round every operation as the oracle does, so the tests ask
for bitwise equality; the stated bar of rel-L2 <= 1e-5 is checked as well so
that a failure reports how far apart the two are."""
from __future__ import annotations

import numpy as np
import pytest

from openswpc_b200 import _lib
from openswpc_b200.params import Source, Station
from openswpc_b200.swpc3d import Swpc3D
from oracle.oracle import AUX_NAMES, Oracle3D
from tests.models import small3d, vonkarman_xi

pytestmark = pytest.mark.gpu

REL_L2_TOL = 1e-5   # receiver traces and final wavefield (FP32 vs FP32 oracle)
VNAMES = ["Vx", "Vy", "Vz", "Sxx", "Syy", "Szz", "Syz", "Sxz", "Sxy"]
RNAMES = ["Rxx", "Ryy", "Rzz", "Ryz", "Rxz", "Rxy"]


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def same_bits(a, b):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return np.array_equal(a.view(np.uint32), b.view(np.uint32))


def oracle_R_as_box(o, name, m, p):
    """oracle memory variable (njk, nik, nkk, nm) -> GPU box layout."""
    d = o.dims()
    r = o.array(name)[..., m]
    box = np.zeros((p.ny + 6, p.nx + 6, p.nz + 6), np.float32)
    box[d["jbeg_k"] + 2:d["jend_k"] + 3, d["ibeg_k"] + 2:d["iend_k"] + 3, d["kbeg_k"] + 2:d["kend_k"] + 3] = r
    return box


def oracle_aux_as_box(o, name, p):
    d = o.dims()
    a = o.array(name)   # (ny, nx, nka) from kbeg_min
    box = np.zeros((p.ny + 6, p.nx + 6, p.nz + 6), np.float32)
    kb = d["kbeg_min"]
    box[3:p.ny + 3, 3:p.nx + 3, kb + 2:p.nz + 3] = a
    # only absorber cells are defined
    kbeg_a = o.array("kbeg_a")
    mask = np.zeros_like(box, bool)
    kk = np.arange(p.nz + 6)[None, None, :] - 2
    mask[3:p.ny + 3, 3:p.nx + 3, :] = True
    mask &= kk >= kbeg_a[:, :, None]
    mask &= kk <= p.nz
    return np.where(mask, box, 0.0).astype(np.float32)


def compare_state(g: Swpc3D, o: Oracle3D, p, what="all"):
    for n, name in enumerate(VNAMES):
        a = g.download(n)
        b = o.array(name)
        assert rel_l2(a, b) <= REL_L2_TOL, (name, rel_l2(a, b))
        assert same_bits(a, b), (name, np.abs(a - b).max())
    if what == "all":
        for c, name in enumerate(RNAMES):
            for m in range(p.nm):
                a = g.download(_lib.F_R + 3 * c + m)
                b = oracle_R_as_box(o, name, m, p)
                assert same_bits(a, b), (name, m, np.abs(a - b).max())
        if p.na > 0 and p.abc_type == "pml":
            for q, name in enumerate(AUX_NAMES):
                a = g.download(_lib.F_AUX + q)
                b = oracle_aux_as_box(o, name, p)
                assert same_bits(a, b), (name, np.abs(a - b).max())


def test_forward_run_matches_oracle_bitwise():
    p = small3d(nt=80, sw_wav_u=True, sw_wav_stress=True, sw_wav_strain=True)
    xi = vonkarman_xi((p.ny + 6, p.nx + 6, p.nz + 6))
    g = Swpc3D(p, xi)
    o = Oracle3D(p, xi)
    rg = g.run(1, p.nt)
    ro = o.run(1, p.nt, ntdec_r=p.ntdec_r)
    for what, comp in ((_lib.WAV_V, "v"), (_lib.WAV_U, "u"), (_lib.WAV_STRESS, "stress"), (_lib.WAV_STRAIN, "strain")):
        a, b = g.waveforms(what), o.waveforms(comp)
        assert np.linalg.norm(b) > 0, comp
        assert rel_l2(a, b) <= REL_L2_TOL, (comp, rel_l2(a, b))
        assert same_bits(a, b), comp
    compare_state(g, o, p)
    assert len(rg) == len(ro) > 0
    for (ia, va), (ib, vb) in zip(rg, ro):
        assert ia == ib and same_bits(va, vb)


def test_error_against_f64_oracle_is_reported(record_property):
    """The FP32 result's distance to the all-double build of the same scheme
    (the error reference): traces and final velocity, rel-L2."""
    p = small3d(nt=80)
    xi = vonkarman_xi((p.ny + 6, p.nx + 6, p.nz + 6))
    g = Swpc3D(p, xi)
    g.run(1, p.nt)
    o = Oracle3D(p, xi, variant="f64")
    o.run(1, p.nt, ntdec_r=p.ntdec_r)
    errs = {"traces_v": rel_l2(g.waveforms(_lib.WAV_V), o.waveforms("v"))}
    for n, name in enumerate(VNAMES[:3]):
        errs[name] = rel_l2(g.download(n), o.array(name))
    for k, v in errs.items():
        record_property(f"rel_l2_vs_f64_{k}", v)
    print("rel-L2 of the FP32 GPU result against the f64 oracle:", errs)
    # FP32 rounding over 80 steps: far below the 1e-5 bar of the FP32 parity
    assert all(v < 1e-4 for v in errs.values()), errs


def test_random_state_single_step_all_paths():
    """Random V, S, R and absorber auxiliaries exercise every branch of the
    fused kernels (4th-order interior, 2nd-order bands, PML) in one step."""
    p = small3d(nt=4, sources=[], stations=[])
    rng = np.random.default_rng(11)
    g = Swpc3D(p)
    o = Oracle3D(p)
    shape = (p.ny + 6, p.nx + 6, p.nz + 6)
    inside = np.zeros(shape, bool)
    inside[3:p.ny + 3, 3:p.nx + 3, 3:p.nz + 3] = True
    for n, name in enumerate(VNAMES):
        # ghost cells are zero in the reference (nothing but sources writes them)
        v = np.where(inside, rng.standard_normal(shape), 0.0).astype(np.float32)
        g.upload(n, v)
        o.set_array(name, v)
        assert same_bits(g.download(n), o.array(name))
    d = o.dims()
    for c, name in enumerate(RNAMES):
        r = rng.standard_normal((d["njk"], d["nik"], d["nkk"], p.nm)).astype(np.float32)
        o.set_array(name, r)
        for m in range(p.nm):
            g.upload(_lib.F_R + 3 * c + m, oracle_R_as_box(o, name, m, p))
    for q, name in enumerate(AUX_NAMES):
        a = rng.standard_normal((p.ny, p.nx, d["nka"])).astype(np.float32)
        o.set_array(name, a)
        box = oracle_aux_as_box(o, name, p)
        o.set_array(name, box[3:p.ny + 3, 3:p.nx + 3, d["kbeg_min"] + 2:p.nz + 3])   # zero outside the absorber
        g.upload(_lib.F_AUX + q, box)
        assert same_bits(g.download(_lib.F_AUX + q), box)
    for it in (1, 2):
        g.step(it)
        o.step(it)
    compare_state(g, o, p)


def test_separate_routines_equal_fused():
    p = small3d(nt=30)
    g1 = Swpc3D(p)
    g2 = Swpc3D(p)
    for it in range(1, 31):
        g1.step(it)
        g2.wav__store(it)
        g2.kernel__update_stress()
        g2.absorb__update_stress()
        g2.source__stressglut(it)
        g2.global__comm_stress()
        g2.kernel__update_vel()
        g2.absorb__update_vel()
        g2.source__bodyforce(it)
        g2.green__source(it)
        g2.global__comm_vel()
    for n in range(9):
        assert same_bits(g1.download(n), g2.download(n))
    assert same_bits(g1.waveforms(), g2.waveforms())


def test_graph_replay_equals_stepping():
    p = small3d(nt=45)
    g1 = Swpc3D(p)
    g2 = Swpc3D(p)
    g1.run(1, p.nt)
    for it in range(1, p.nt + 1):
        g2.step(it)
    g2.sync()
    for n in range(9):
        assert same_bits(g1.download(n), g2.download(n))
    assert same_bits(g1.waveforms(), g2.waveforms())


@pytest.mark.parametrize("nm", [0, 1, 2])
def test_fewer_memory_variables(nm):
    p = small3d(nt=30, nm=nm)
    g = Swpc3D(p)
    o = Oracle3D(p)
    g.run(1, p.nt)
    o.run(1, p.nt)
    assert same_bits(g.waveforms(), o.waveforms("v"))
    compare_state(g, o, p)


def test_body_force_mode():
    srcs = [Source(0.2, -0.4, 5.0, 0.0, 1.0, fx=1.0, fy=0.5, fz=-2.0),
            Source(-2.0, 1.5, 3.0, 0.1, 0.8, fx=0.0, fy=1.0, fz=0.0)]
    p = small3d(nt=40, bf_mode=True, sources=srcs)
    g = Swpc3D(p)
    o = Oracle3D(p)
    g.run(1, p.nt)
    o.run(1, p.nt)
    assert np.linalg.norm(o.waveforms("v")) > 0
    assert same_bits(g.waveforms(), o.waveforms("v"))
    compare_state(g, o, p)


def test_green_function_source():
    p = small3d(nt=40, green_mode=True, green_cmp="z", green_trise=1.0, green_station=0, sources=[])
    g = Swpc3D(p)
    o = Oracle3D(p)
    g.run(1, p.nt)
    o.run(1, p.nt)
    assert np.abs(o.array("Vz")).max() > 0
    compare_state(g, o, p)


def test_sources_at_domain_edges_and_in_absorber():
    """Sources in the absorber, next to the i/j edges and at k = 1 write into
    ghost cells; the cells that global__comm_* zeroes must stay zero and the
    others keep their values, exactly as in the reference."""
    p = small3d(nt=25)
    xb, yb, zb = p.xbeg, p.ybeg, p.zbeg
    srcs = [Source(xb + 0.2, yb + 0.3, 5.0, 0.0, 0.5, mo=1e15, mxx=1, myy=-1, mzz=0.5, myz=0.3, mxz=0.2, mxy=0.7),
            Source(xb + 19.9, yb + 17.9, 1.0, 0.0, 0.5, mo=2e15, mxy=1, mxz=1, myz=1),
            Source(1.0, 1.0, zb + 0.1, 0.0, 0.5, mo=1e15, mxz=1, myz=-1, mzz=1),
            Source(1.0, 1.0, zb + 0.1, 0.0, 0.7, mo=1e15, mxx=1, mxz=1)]   # same cell: serial injection
    p.sources = srcs
    g = Swpc3D(p)
    o = Oracle3D(p)
    g.run(1, p.nt)
    o.run(1, p.nt)
    compare_state(g, o, p)


def test_vmax_and_divergence_detection():
    p = small3d(nt=30)
    g = Swpc3D(p)
    o = Oracle3D(p)
    g.run(1, 20)
    o.run(1, 20)
    assert same_bits(g.kernel__vmax(), o.vmax())
    v = g.download(_lib.F_VZ)
    v[p.ny // 2 + 2, p.nx // 2 + 2, 3 + 1 + 2] = 1e25   # k = kob + 1 = 4
    g.upload(_lib.F_VZ, v)
    with pytest.raises(_lib.SwpcError) as e:
        g.kernel__vmax()
    assert e.value.code == _lib.SWPC_ERR_DIVERGED


def test_large_box_uploads_through_the_staging_buffer():
    """Boxes of 2^16 floats and more travel to the device in contiguous
    chunks of planes (16 MB) through a staging buffer and are repacked there
    (174 planes here: a full chunk and a short one).  The medium upload of the run and
    a field upload both take that path: the run matches the oracle bitwise,
    and a random field comes back unchanged."""
    p = small3d(nx=168, ny=168, nz=140, na=10, nt=4)
    assert (p.nx + 6) * (p.ny + 6) * (p.nz + 6) >= 1 << 22
    xi = vonkarman_xi((p.ny + 6, p.nx + 6, p.nz + 6))
    g = Swpc3D(p, xi)
    o = Oracle3D(p, xi, threads=8)
    for it in range(1, p.nt + 1):
        g.step(it)
        o.step(it)
    compare_state(g, o, p, what="v")
    x = np.random.default_rng(8).standard_normal((p.ny + 6, p.nx + 6, p.nz + 6)).astype(np.float32)
    g.upload(_lib.F_VY, x)
    assert same_bits(g.download(_lib.F_VY), x)


def test_averaged_medium_formed_on_the_device():
    """With rho given and the six averaged fields left out, swpc_upload_medium
    forms bx, by, bz, muyz, muxz, muxy in HBM (averaged_medium,
    m_medium.f90:432-465): bitwise equal to the host fields over the whole
    memory box, on a perturbed medium with air cells (harmonic means over zero
    rigidity) that is large enough for the chunked upload; runs on either
    medium agree bitwise."""
    p = small3d(nx=90, ny=80, nz=60, na=10, nt=6)
    xi = vonkarman_xi((p.ny + 6, p.nx + 6, p.nz + 6))
    g0 = Swpc3D(p, xi)
    m = g0.medium
    assert float(m.mu.min()) == 0.0 and float(m.mu.max()) > 0.0
    g1 = Swpc3D(p, medium=m, average_on_device=True)
    for q, name in enumerate(m.FIELDS[1:], start=1):
        assert same_bits(g1.download(_lib.F_MED + q), getattr(m, name)), name
    for it in range(1, p.nt + 1):
        g0.step(it)
        g1.step(it)
    for f in list(range(_lib.F_VX, _lib.F_SXY + 1)) + [_lib.F_R, _lib.F_R + 17]:
        assert same_bits(g0.download(f), g1.download(f)), f


def test_larger_grid_against_oracle_few_steps():
    """A grid whose planes exceed one warp row in every direction (k spans
    several 32-cell chunks, absorber/interior boundaries fall mid-warp)."""
    p = small3d(nx=72, ny=64, nz=100, na=12, nt=6)
    g = Swpc3D(p)
    o = Oracle3D(p, threads=8)
    for it in range(1, 7):
        g.step(it)
        o.step(it)
    compare_state(g, o, p)


@pytest.mark.parametrize("variant", [(0, 2, 2, 1, 1, 4, 2, 2), (0, 1, 4, 2, 1, 3, 8, 1), (2, 2, 1, 16, 3, 2, 1, 7),
                                     (2, 1, 1, 64, 3, 1, 1, 3), (0, 2, 2, 1, 4, 2, 2, 2), (0, 2, 2, 1, 4, 1, 4, 1),
                                     (0, 2, 2, 1, 4, 3, 1, 2), (5, 1, 4, 2, 6, 1, 4, 2), (5, 1, 2, 4, 6, 1, 4, 4),
                                     (5, 1, 4, 4, 6, 1, 2, 2)])
def test_launch_variants_are_bitwise_identical(variant):
    """Flat, marching, four-cells-per-thread and TMA-staged kernels (5, 6),
    any block shape, chunk length or tile: same bits.  nz = 70 with na = 8 puts the interior/absorber
    boundary inside a group of four and ends the column mid-group."""
    ks, ms, bis, bjs, kv, mv, biv, bjv = variant
    p = small3d(nx=44, ny=38, nz=70, na=8, nt=25)
    g0 = Swpc3D(p)
    g1 = Swpc3D(p)
    _lib.check(g1.ctx, g1.lib.swpc_set_launch(g1.ctx, ks, ms, bis, bjs))
    _lib.check(g1.ctx, g1.lib.swpc_set_launch(g1.ctx, kv, mv, biv, bjv))
    g0.run(1, p.nt)
    g1.run(1, p.nt)
    for n in range(9):
        assert same_bits(g0.download(n), g1.download(n)), n
    for q in range(18):
        assert same_bits(g0.download(_lib.F_AUX + q), g1.download(_lib.F_AUX + q)), q


@pytest.mark.parametrize("jblock", [1, 3, 5, 0])
def test_staged_launch_order_is_bitwise_identical(jblock):
    """Blocks of jblock j tiles in the staged launch order (a short last
    block for 3 of the 10 j tiles; 0 = the size-dependent default) against
    the flat kernels."""
    p = small3d(nx=44, ny=38, nz=70, na=8, nt=25)
    g0 = Swpc3D(p)
    g1 = Swpc3D(p)
    _lib.check(g0.ctx, g0.lib.swpc_set_launch(g0.ctx, 0, 2, 2, 1))
    _lib.check(g0.ctx, g0.lib.swpc_set_launch(g0.ctx, 1, 4, 2, 2))
    _lib.check(g1.ctx, g1.lib.swpc_set_launch(g1.ctx, 7, 1, jblock, 1))
    g0.run(1, p.nt)
    g1.run(1, p.nt)
    for n in range(9):
        assert same_bits(g0.download(n), g1.download(n)), n
    for q in range(18):
        assert same_bits(g0.download(_lib.F_AUX + q), g1.download(_lib.F_AUX + q)), q


@pytest.mark.parametrize("nm", [0, 1, 2])
def test_staged_kernels_with_fewer_memory_variables(nm):
    """The staged kernels read R from a slab box whose width follows nm."""
    p = small3d(nx=40, ny=36, nz=40, na=8, nt=20, nm=nm)
    g0 = Swpc3D(p)
    g1 = Swpc3D(p)
    _lib.check(g1.ctx, g1.lib.swpc_set_launch(g1.ctx, 5, 1, 4, 2))
    _lib.check(g1.ctx, g1.lib.swpc_set_launch(g1.ctx, 6, 1, 4, 4))
    g0.run(1, p.nt)
    g1.run(1, p.nt)
    fields = list(range(9)) + [_lib.F_R + 3 * c + m for c in range(6) for m in range(nm)]
    for n in fields:
        assert same_bits(g0.download(n), g1.download(n)), n


def test_stabilized_medium_run_matches_oracle():
    """A run on a medium set up with stabilize_pml (a thin low-velocity layer
    in the absorber) equals the oracle bitwise."""
    from openswpc_b200.params import Layer
    from tests.models import LAYERS

    layers = [Layer(0.0, 2.2, 2.4, 1.2, 100, 50), Layer(1.0, 2.7, 5.5, 3.2, 300, 150),
              Layer(3.0, 2.4, 3.0, 1.6, 100, 50), Layer(4.0, 2.7, 5.5, 3.2, 300, 150)] + LAYERS[1:]
    p = small3d(nx=40, ny=36, nz=32, na=8, nt=30, layers=layers, stabilize_pml=True)
    g = Swpc3D(p)
    o = Oracle3D(p, threads=4)
    g.run(1, p.nt)
    o.run(1, p.nt)
    assert same_bits(g.waveforms(), o.waveforms("v"))
    compare_state(g, o, p)


def test_seawater_forward_run_matches_oracle():
    """A run with seawater of Munk's profile above the first layer
    (m_vmodel_lhm.f90:123-133): the ocean bottom lies below the free surface,
    so the ocean-bottom stations ('obb', 'oba') and the 2nd-order bands of
    both surfaces are exercised; traces and final state bitwise."""
    from openswpc_b200.params import Layer
    from tests.models import LAYERS

    p = small3d(nt=60, munk_profile=True, layers=[Layer(1.8, 2.7, 5.5, 3.2, 300, 150)] + list(LAYERS[1:]))
    g = Swpc3D(p)
    o = Oracle3D(p)
    assert (g.medium.kob[4:-4, 4:-4] > g.medium.kfs[4:-4, 4:-4]).all()
    g.run(1, p.nt)
    o.run(1, p.nt, ntdec_r=p.ntdec_r)
    a, b = g.waveforms(_lib.WAV_V), o.waveforms("v")
    assert np.linalg.norm(b) > 0 and same_bits(a, b)
    compare_state(g, o, p)


@pytest.mark.parametrize("ps", ["P", "S"])
def test_plane_wave_run_matches_oracle(ps):
    """Plane-wave mode (pw_setup, m_source.f90:315-465, and the zero-derivative
    side boundary of the PML, m_absorb_p.f90:136-243, 324-431, with the ghost
    planes the single-domain exchange zeroes): traces, final V, S, memory
    variables and PML auxiliaries bitwise; per-routine calls equal graph
    steps."""
    p = small3d(nt=50, pw_mode=True, pw_ztop=8.0, pw_zlen=4.0, pw_ps=ps, pw_strike=30.0, pw_dip=20.0,
                pw_rake=40.0, sources=[], sw_wav_stress=True)
    g = Swpc3D(p)
    o = Oracle3D(p)
    g.run(1, p.nt)
    o.run(1, p.nt, ntdec_r=p.ntdec_r)
    for what, comp in ((_lib.WAV_V, "v"), (_lib.WAV_STRESS, "stress")):
        a, b = g.waveforms(what), o.waveforms(comp)
        assert np.linalg.norm(b) > 0 and same_bits(a, b), comp
    compare_state(g, o, p)
    h = Swpc3D(p)
    for it in range(1, p.nt + 1):
        h.wav__store(it)
        h.kernel__update_stress()
        h.absorb__update_stress()
        h.source__stressglut(it)
        h.global__comm_stress()
        h.kernel__update_vel()
        h.absorb__update_vel()
        h.source__bodyforce(it)
        h.global__comm_vel()
    for n in range(9):
        assert same_bits(h.download(n), g.download(n)), n


def test_failed_tile_copy_is_reported_until_the_state_is_restored():
    """The error word of a timed-out tile wait, raised from the host (no
    kernel made to wait or fault): swpc_sync reports it, keeps reporting it
    across further steps, and a reset to rest (or a restored state and
    swpc_clear_error) clears it; the run from rest then equals a fresh one."""
    p = small3d(nt=20)
    g = Swpc3D(p)
    lib, ctx = g.lib, g.ctx
    g.run(1, 5)
    assert lib.swpc_sync(ctx) == _lib.SWPC_OK
    assert lib.swpc_raise_copy_error(ctx) == _lib.SWPC_OK
    assert lib.swpc_sync(ctx) == _lib.SWPC_ERR_CUDA
    assert b"did not complete" in lib.swpc_last_error(ctx)
    with pytest.raises(_lib.SwpcError):
        g.run(6, 3)     # the run's own sync raises while the word is up
    assert lib.swpc_sync(ctx) == _lib.SWPC_ERR_CUDA
    _lib.check(ctx, lib.swpc_reset_state(ctx))
    assert lib.swpc_sync(ctx) == _lib.SWPC_OK
    g.run(1, p.nt)
    h = Swpc3D(p)
    h.run(1, p.nt)
    for n in range(9):
        assert same_bits(g.download(n), h.download(n))
    assert lib.swpc_raise_copy_error(ctx) == _lib.SWPC_OK
    _lib.check(ctx, lib.swpc_clear_error(ctx))
    assert lib.swpc_sync(ctx) == _lib.SWPC_OK
