"""Reciprocity batch: every member equals a green-mode run of its own.

Each member of a ForceBatch3D is driven by one unit force (green__source,
src/swpc_3d/m_green.f90:597-632) over the shared medium; its velocity traces
and final V, S, R must be bitwise those of a single green-mode run with the
same force, whatever the launch order (strip width) and whether the steps
run per call or as graph replays."""
import numpy as np
import pytest

from openswpc_b200 import _lib
from openswpc_b200.swpc3d import ForceBatch3D, Swpc3D
from tests.models import small3d, vonkarman_xi

pytestmark = pytest.mark.gpu

FORCES = [(0, "x"), (1, "y"), (2, "z"), (3, "z"), (5, "x")]


def green_params(nt=50, **kw):
    return small3d(nx=44, ny=40, nz=32, na=8, nt=nt, green_mode=True, green_trise=1.2, **kw)


def single(p, xi, station, cmp):
    q = green_params(nt=p.nt)
    q.green_station, q.green_cmp = station, cmp
    g = Swpc3D(q, xi)
    g.record(p.stations)
    g.run(1, q.nt)
    return g


# launch forms: flat kernels with two strip widths; staged kernels with 1, 2
# and 4 members per CTA (5 members: the last group is partial)
LAUNCHES = [("flat", 0), ("flat", 8), ("staged", (4, 4, 1, 4, 2, 1, 0)), ("staged", (4, 2, 2, 4, 2, 2, 0)),
            ("staged", (2, 2, 4, 2, 2, 4, 0)), ("staged", (4, 1, 4, 4, 1, 4, 1)), ("staged", (2, 4, 2, 2, 2, 2, 1)),
            ("staged", (4, 4, 1, 4, 2, 1, 1))]


@pytest.mark.parametrize("launch", LAUNCHES)
def test_members_equal_single_green_runs(launch):
    p = green_params()
    xi = vonkarman_xi((p.ny + 6, p.nx + 6, p.nz + 6))
    base = Swpc3D(p, xi)
    base.record(p.stations)
    fb = ForceBatch3D(base, [(p.stations[s], c) for s, c in FORCES])
    kind, arg = launch
    if kind == "flat":
        fb.set_launch(0)
        fb.set_strip(arg)
    else:
        sbi, sbj, smpc, vbi, vbj, vmpc, order = arg
        fb.set_launch(5, smpc, sbi, sbj)
        fb.set_launch(6, vmpc, vbi, vbj)
        fb.set_launch(7, order)
    fb.run(1, p.nt)
    fields = list(range(9)) + [_lib.F_R + 3 * c + m for c in range(6) for m in range(p.nm)]
    for m, (s, c) in enumerate(FORCES):
        g = single(p, xi, s, c)
        a, b = fb.waveforms(m), g.waveforms(_lib.WAV_V)
        assert np.linalg.norm(b) > 0
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), f"member {m}: traces differ"
        for f in fields:
            x, y = fb.download(m, f), g.download(f)
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), f"member {m}: field {f} differs"
        g.close()
    fb.close()
    base.close()


def test_per_call_steps_equal_graph_replays():
    p = green_params(nt=30)
    xi = vonkarman_xi((p.ny + 6, p.nx + 6, p.nz + 6))
    base = Swpc3D(p, xi)
    base.record(p.stations)
    forces = [(p.stations[s], c) for s, c in FORCES[:3]]
    f1 = ForceBatch3D(base, forces)
    f1.run(1, p.nt)
    f2 = ForceBatch3D(base, forces)
    for it in range(1, p.nt + 1):
        f2.step(it)
    for m in range(3):
        assert np.array_equal(f1.waveforms(m).view(np.uint32), f2.waveforms(m).view(np.uint32))
        for f in range(9):
            assert np.array_equal(f1.download(m, f).view(np.uint32), f2.download(m, f).view(np.uint32))
    f1.close()
    f2.close()
    base.close()


def test_autotune_keeps_results_and_bad_member_is_rejected():
    p = green_params(nt=80)
    base = Swpc3D(p)
    base.record(p.stations)
    fb = ForceBatch3D(base, [(p.stations[0], "z"), (p.stations[1], "x")])
    used, _ = fb.autotune(1, reps=2)
    assert 0 < used <= 56 and fb.launch()["staged"]
    fb.set_launch(0)
    used2, strip = fb.autotune(1 + used, reps=2)
    assert used2 > 0 and strip >= 8
    # a context that still has a batch is not destroyed
    assert base.lib.swpc_destroy(base.ctx) == _lib.SWPC_ERR_STATE
    with pytest.raises(_lib.SwpcError):
        _lib.check(base.ctx, fb.lib.swpc_fbatch_green_source(fb.b, 2, 10, 10, 5, b"z", 0.0, 1.0, 0))
    fb.close()
    base.close()
