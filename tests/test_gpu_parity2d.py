"""GPU parity of the 2D P-SV and SH steps against the CPU oracle, and of the
batched 2D ensemble against independent runs (bitwise)."""
from __future__ import annotations

import numpy as np
import pytest

from openswpc_b200 import _lib
from openswpc_b200.params import Source
from openswpc_b200.swpc2d import Batch2D, Swpc2D
from oracle.oracle import Oracle2D
from tests.models import small2d

pytestmark = pytest.mark.gpu

REL_L2_TOL = 1e-5


def same_bits(a, b):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return np.array_equal(a.view(np.uint32), b.view(np.uint32))


def rel_l2(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def aux_box(o, name, p):
    d = o.dims()
    a = o.array(name)
    box = np.zeros((p.nx + 6, p.nz + 6), np.float32)
    box[3:p.nx + 3, d["kbeg_min"] + 2:p.nz + 3] = a
    kb = o.array("kbeg_a")
    kk = np.arange(p.nz + 6)[None, :] - 2
    mask = np.zeros_like(box, bool)
    mask[3:p.nx + 3, :] = True
    mask &= (kk >= kb[:, None]) & (kk <= p.nz)
    return np.where(mask, box, 0).astype(np.float32)


def compare(g: Swpc2D, o: Oracle2D, p):
    for name, fid in g.field_ids.items():
        a, b = g.download(fid), o.array(name)
        assert rel_l2(a, b) <= REL_L2_TOL, (name, rel_l2(a, b))
        assert same_bits(a, b), (name, np.abs(a - b).max())
    rn = ["Rxx", "Rzz", "Rxz"] if g.kind == "psv" else ["Ryz", "Rxy"]
    rc = [0, 2, 4] if g.kind == "psv" else [3, 5]
    for name, c in zip(rn, rc):
        ref = o.array(name)
        for m in range(p.nm):
            a = g.download(_lib.F_R + 3 * c + m)
            b = np.zeros_like(a)
            d = o.dims()
            b[d["ibeg_k"] + 2:d["iend_k"] + 3, 3:d["kend_k"] + 3] = ref[d["ibeg_k"] + 2:d["iend_k"] + 3, 3:d["kend_k"] + 3, m]
            assert same_bits(a, b), (name, m)
    auxn = (["axVx", "azVx", "axVz", "azVz", "axSxx", "azSxz", "axSxz", "azSzz"] if g.kind == "psv" else
            ["axVy", "azVy", "axSxy", "azSyz"])
    for q, name in enumerate(auxn if p.abc_type == "pml" else []):
        assert same_bits(g.download(_lib.F_AUX + q), aux_box(o, name, p)), name


def set_launch(g: Swpc2D, stress_ti: int, vel_ti: int):
    """Staged kernels with ti threads along i (4, 8, 16), or the tile-walking
    kernels (0), per phase."""
    _lib.check(g.ctx, g.lib.swpc_set_launch(g.ctx, 5 if stress_ti else 0, 1, stress_ti or 1, 1))
    _lib.check(g.ctx, g.lib.swpc_set_launch(g.ctx, 6 if vel_ti else 1, 1, vel_ti or 1, 1))


LAUNCHES = [(8, 8), (4, 16), (16, 4), (0, 0)]


@pytest.mark.parametrize("launch", LAUNCHES, ids=lambda l: f"stress{l[0]}-vel{l[1]}")
@pytest.mark.parametrize("kind", ["psv", "sh"])
def test_2d_forward_matches_oracle(kind, launch):
    """Staged kernels (ti threads along i) and tile-walking kernels (0) give
    the oracle's bits."""
    p = small2d(kind, nt=120)
    g = Swpc2D(p, kind)
    set_launch(g, *launch)
    o = Oracle2D(p, kind)
    g.run(1, p.nt)
    o.run(1, p.nt)
    for what, comp in ((_lib.WAV_V, "v"), (_lib.WAV_U, "u")):
        a, b = g.waveforms(what), o.waveforms(comp)
        assert np.linalg.norm(b) > 0, comp
        assert rel_l2(a, b) <= REL_L2_TOL
        assert same_bits(a, b), comp
    compare(g, o, p)
    vm = g.kernel__vmax()
    assert same_bits(vm, o.vmax()[:len(vm)])


@pytest.mark.parametrize("kind", ["psv", "sh"])
def test_2d_large_box_uploads_through_the_staging_buffer(kind):
    """A 2D box of 2^16 floats or more is uploaded through the staging buffer
    and repacked on the device: the run matches the oracle bitwise and a
    random field comes back unchanged."""
    p = small2d(kind, nx=300, nz=220, na=12, nt=30)
    assert (p.nx + 6) * (p.nz + 6) >= 1 << 16
    g = Swpc2D(p, kind)
    o = Oracle2D(p, kind)
    g.run(1, p.nt)
    o.run(1, p.nt)
    assert same_bits(g.waveforms(), o.waveforms())
    compare(g, o, p)
    fid = next(iter(g.field_ids.values()))
    x = np.random.default_rng(9).standard_normal(g.download(fid).shape).astype(np.float32)
    g.upload(fid, x)
    assert same_bits(g.download(fid), x)


@pytest.mark.parametrize("nm", [0, 1, 2])
@pytest.mark.parametrize("kind", ["psv", "sh"])
def test_2d_staged_thick_absorber_and_fewer_memory_variables(kind, nm):
    """A 20-cell absorber leaves tiles without interior cells (the staged
    stress kernel copies S without R there); nm = 0..2 memory variables."""
    p = small2d(kind, nx=104, nz=70, na=20, nt=90, nm=nm)
    g = Swpc2D(p, kind)
    o = Oracle2D(p, kind)
    g.run(1, p.nt)
    o.run(1, p.nt)
    assert np.linalg.norm(o.waveforms()) > 0
    assert same_bits(g.waveforms(), o.waveforms())
    compare(g, o, p)


@pytest.mark.parametrize("kind", ["psv", "sh"])
def test_2d_body_force_and_absorber_sources(kind):
    """Body forces, one inside the absorber (P-SV injects it between the
    interior and absorber velocity updates, like the reference)."""
    srcs = [Source(0.4, 0.0, 3.0, 0.0, 0.7, fx=1.0, fy=0.8, fz=-0.5),
            Source(-13.9, 0.0, 1.0, 0.1, 0.6, fx=0.3, fy=1.0, fz=1.0)]
    p = small2d(kind, nt=80, bf_mode=True, sources=srcs)
    g = Swpc2D(p, kind)
    o = Oracle2D(p, kind)
    g.run(1, p.nt)
    o.run(1, p.nt)
    assert np.linalg.norm(o.waveforms()) > 0
    assert same_bits(g.waveforms(), o.waveforms())
    compare(g, o, p)


@pytest.mark.parametrize("kind", ["psv", "sh"])
def test_batched_ensemble_equals_independent_runs(kind):
    """Uneven 2D models advanced by one launch per half step give the same
    bits as running each model alone, and as the oracle."""
    sizes = [(96, 48), (160, 40), (72, 90), (128, 64)]
    ps = [small2d(kind, nx=nx, nz=nz, na=8, nt=50, seed=s) for s, (nx, nz) in enumerate(sizes)]
    runs = [Swpc2D(p, kind) for p in ps]
    alone = [Swpc2D(p, kind) for p in ps]
    batch = Batch2D(runs)
    assert batch.launch() == {"ti": 4, "ri": 4, "bps": 0, "stress_ti": 8, "vel_ti": 8}
    batch.run(1, 50)
    for r, a, p in zip(runs, alone, ps):
        a.run(1, 50)
        assert same_bits(r.waveforms(), a.waveforms())
        for fid in r.field_ids.values():
            assert same_bits(r.download(fid), a.download(fid))
    o = Oracle2D(ps[2], kind)
    o.run(1, 50)
    assert same_bits(runs[2].waveforms(), o.waveforms())
    batch.close()


@pytest.mark.parametrize("kind", ["psv", "sh"])
def test_batch_launch_forms_give_the_same_bits(kind):
    """Staged kernels with every thread count, mixed with the tile-walking
    kernels, and tile-walking shapes: all give the bits of independent runs,
    one launch form per ten steps."""
    sizes = [(96, 48), (40, 40), (150, 77)]
    ps = [small2d(kind, nx=nx, nz=nz, na=8, nt=60, seed=20 + s) for s, (nx, nz) in enumerate(sizes)]
    runs = [Swpc2D(p, kind) for p in ps]
    batch = Batch2D(runs)
    forms = [("staged", 4, 16), ("staged", 16, 0), ("shape", 4, 2), ("staged", 0, 8), ("shape", 8, 4),
             ("staged", 8, 4)]
    it = 1
    for what, a, b in forms:
        if what == "staged":
            batch.set_staged(a, b)
            assert batch.launch()["ti"] * batch.launch()["ri"] == 16
        else:
            batch.set_shape(a, b, 0)
            assert batch.launch()["stress_ti"] == 0 and batch.launch()["vel_ti"] == 0
        batch.run(it, 10)
        it += 10
    for r, p in zip(runs, ps):
        a = Swpc2D(p, kind)
        a.run(1, 60)
        assert same_bits(r.waveforms(), a.waveforms())
        for fid in r.field_ids.values():
            assert same_bits(r.download(fid), a.download(fid))
    with pytest.raises(_lib.SwpcError):
        batch.set_staged(6, 8)
    batch.close()


def test_batch_of_more_members_than_one_staged_launch_takes():
    """50 members: the staged kernels take their tensor maps as a kernel
    parameter for at most 48 members per launch, so the batch launches two
    member groups per phase; every member keeps the bits of its own run."""
    ps = [small2d("psv", nx=40 + 8 * (s % 5), nz=32 + 6 * (s % 3), na=6, nt=12, seed=100 + s) for s in range(50)]
    runs = [Swpc2D(p, "psv") for p in ps]
    batch = Batch2D(runs)
    batch.run(1, 12)
    for r, p in zip(runs, ps):
        a = Swpc2D(p, "psv")
        a.run(1, 12)
        assert same_bits(r.waveforms(), a.waveforms())
        for fid in r.field_ids.values():
            assert same_bits(r.download(fid), a.download(fid))
        a.close()
    batch.close()


@pytest.mark.parametrize("kind", ["psv", "sh"])
def test_batch_autotune_steps_are_ordinary_steps(kind):
    """The autotuner advances the run with every candidate launch shape; the
    result equals independent runs bit for bit."""
    sizes = [(200, 40), (64, 120), (150, 77)]
    ps = [small2d(kind, nx=nx, nz=nz, na=8, nt=40, seed=10 + s) for s, (nx, nz) in enumerate(sizes)]
    runs = [Swpc2D(p, kind) for p in ps]
    batch = Batch2D(runs)
    used, ti, ri, bps = batch.autotune(1, reps=2)
    assert used == 24 and ti in (2, 4, 8) and ri in (1, 2, 4, 8) and bps >= 0
    pick = batch.launch()
    assert pick["stress_ti"] in (0, 4, 8, 16) and pick["vel_ti"] in (0, 4, 8, 16)
    batch.run(1 + used, 40 - used)
    for r, p in zip(runs, ps):
        a = Swpc2D(p, kind)
        a.run(1, 40)
        assert same_bits(r.waveforms(), a.waveforms())
        for fid in r.field_ids.values():
            assert same_bits(r.download(fid), a.download(fid))
    batch.close()
