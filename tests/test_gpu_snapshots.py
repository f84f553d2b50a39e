"""Snapshot planes (snap__setup / snap__write, src/swpc_3d/m_snap.f90) on the
GPU against the oracle: every plane type, decimation in all three
directions, time decimation, the displacement sums and the free-surface /
ocean-bottom maxima, bitwise."""
import numpy as np
import pytest

from openswpc_b200.params import SNAP_QUANTITIES, SNAP_SECTIONS, dc_source, snap_plane
from openswpc_b200.swpc3d import Swpc3D
from oracle.oracle import Oracle3D
from tests.models import small3d, vonkarman_xi

pytestmark = pytest.mark.gpu

ALL = {f"{s}_{q}" for s in SNAP_SECTIONS for q in SNAP_QUANTITIES}


def same_bits(a, b):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


def oracle_with_snaps(p, xi):
    o = Oracle3D(p, xi)
    planes = sum(1 << snap_plane(n) for n in p.snaps)
    o.snap_setup(planes, p.idec, p.jdec, p.kdec, p.ntdec_s, p.x0_yz, p.y0_xz, p.z0_xy)
    return o


@pytest.mark.parametrize("dec", [(1, 1, 1, 1), (2, 3, 2, 7)])
def test_all_snapshot_planes_bitwise(dec):
    idec, jdec, kdec, ntdec_s = dec
    # a shallow source so that the free-surface planes see the wavefield
    p = small3d(nt=45, snaps=set(ALL), idec=idec, jdec=jdec, kdec=kdec, ntdec_s=ntdec_s,
                x0_yz=1.3, y0_xz=-2.1, z0_xy=4.4, sources=[dc_source(0.5, -0.5, 1.6, 0.0, 0.6, 1e16, 30, 60, 90)])
    xi = vonkarman_xi((p.ny + 6, p.nx + 6, p.nz + 6))
    g = Swpc3D(p, xi)
    g.run(1, p.nt)
    o = oracle_with_snaps(p, xi)
    o.run(1, p.nt)
    d = o.snap_dims()
    assert g.snap_nframes == d["nframes"] == (p.nt - 1) // ntdec_s + 1
    for name in sorted(ALL):
        a = g.snapshots(name)
        b = o.snap_frames(snap_plane(name))
        assert np.abs(b).max() > 0, name
        assert same_bits(a, b), (name, a.shape, b.shape, np.abs(a - b).max())
    # the closing call at nt + 1 (snap__closefiles) updates sums and maxima
    g.snap__write(p.nt + 1)
    o.snap_write(p.nt + 1)
    for w, name in enumerate(("fs_v", "fs_u", "ob_v", "ob_u")):
        a = g.snapshot_max(name)
        b = o.snap_max(w)
        assert np.abs(b).max() > 0, name
        assert same_bits(a, b), name


def test_snapshots_through_separate_routines_equal_graph():
    p = small3d(nt=20, snaps={"xy_ps", "fs_v", "xz_u"}, ntdec_s=3, idec=2, jdec=2, kdec=2)
    g1 = Swpc3D(p)
    g1.run(1, p.nt)
    g2 = Swpc3D(p)
    for it in range(1, p.nt + 1):
        g2.wav__store(it)
        g2.snap__write(it)
        g2.kernel__update_stress()
        g2.absorb__update_stress()
        g2.source__stressglut(it)
        g2.kernel__update_vel()
        g2.absorb__update_vel()
    for name in p.snaps:
        assert same_bits(g1.snapshots(name), g2.snapshots(name)), name
    assert same_bits(g1.snapshot_max("fs_v"), g2.snapshot_max("fs_v"))
