"""green__store (src/swpc_3d/m_green.f90:389-534) on the GPU against the
oracle: the reciprocity Green's functions (displacement derivatives, and
displacements with green_bforce) at a table of grid points, bitwise."""
from __future__ import annotations

import numpy as np
import pytest

from openswpc_b200.swpc3d import ForceBatch3D, Swpc3D, station_grid
from oracle.oracle import Oracle3D
from tests.models import small3d, vonkarman_xi
from tests.test_gpu_parity3d import same_bits

pytestmark = pytest.mark.gpu


def green_table(p, n=40, seed=3):
    """Seeded grid points across the model: near the surface, at depth, next
    to and inside the absorber."""
    rng = np.random.default_rng(seed)
    ig = rng.integers(1, p.nx + 1, n)
    jg = rng.integers(1, p.ny + 1, n)
    kg = rng.integers(1, p.nz + 1, n)
    return ig, jg, kg


@pytest.mark.parametrize("bforce,ntdec", [(False, 1), (True, 3)])
def test_green_store_matches_oracle(bforce, ntdec):
    p = small3d(nt=45, green_mode=True, green_cmp="x", green_trise=1.0, green_station=0, sources=[])
    xi = vonkarman_xi((p.ny + 6, p.nx + 6, p.nz + 6))
    ig, jg, kg = green_table(p)
    g = Swpc3D(p, xi)
    o = Oracle3D(p, xi, threads=8)
    g.green_store_setup(ig, jg, kg, bforce=bforce, ntdec_w=ntdec)
    o.green_store_setup(ig, jg, kg, bforce=bforce, ntdec_w=ntdec)
    g.run(1, p.nt)
    o.run(1, p.nt)
    a, b = g.green_functions(), o.green_functions()
    assert a.shape == ((9 if bforce else 6) * len(ig), (p.nt - 1) // ntdec + 1)
    assert np.abs(b).max() > 0
    assert same_bits(a, b)


def test_green_store_per_step_calls_equal_graph():
    """swpc_step calls green__store beside wav__store; a graph replay of the
    same steps gives the same Green's functions."""
    p = small3d(nt=20, green_mode=True, green_cmp="z", green_trise=1.0, green_station=0, sources=[])
    ig, jg, kg = green_table(p, n=12, seed=5)
    g0, g1 = Swpc3D(p), Swpc3D(p)
    for g in (g0, g1):
        g.green_store_setup(ig, jg, kg, bforce=True)
    g0.run(1, p.nt)
    for it in range(1, p.nt + 1):
        g1.step(it)
    assert same_bits(g0.green_functions(), g1.green_functions())


def test_reciprocity_batch_members_store_their_green_functions():
    """Every member of a reciprocity batch records green__store at the
    context's green table, bitwise as a green-mode run of its own force."""
    p = small3d(nx=44, ny=40, nz=32, na=8, nt=30, green_mode=True, green_trise=1.2, green_cmp="x",
                green_station=0, sources=[])
    xi = vonkarman_xi((p.ny + 6, p.nx + 6, p.nz + 6))
    ig, jg, kg = green_table(p, n=16, seed=7)
    base = Swpc3D(p, xi)
    # and the cells right below the force stations, which the waves reach at once
    si, sj, sk = station_grid(p, base.medium.kfs, base.medium.kob)
    ig, jg, kg = np.r_[ig, si], np.r_[jg, sj], np.r_[kg, np.minimum(sk + 1, p.nz)]
    base.green_store_setup(ig, jg, kg, bforce=True, ntdec_w=2)
    forces = [(0, "x"), (2, "z"), (3, "y")]
    fb = ForceBatch3D(base, [(p.stations[s], c) for s, c in forces])
    fb.run(1, p.nt)
    for m, (s, c) in enumerate(forces):
        q = small3d(nx=44, ny=40, nz=32, na=8, nt=30, green_mode=True, green_trise=1.2, green_cmp=c,
                    green_station=s, sources=[])
        g = Swpc3D(q, xi)
        g.green_store_setup(ig, jg, kg, bforce=True, ntdec_w=2)
        g.run(1, q.nt)
        a, b = fb.green_functions(m), g.green_functions()
        assert np.abs(b).max() > 0
        assert same_bits(a, b), f"member {m}"
        g.close()
    fb.close()


def test_green_store_device_bytes_are_returned_on_reset():
    """A second setup frees the first table's arrays: swpc_device_bytes comes
    back to its value before the first setup when the table is cleared."""
    p = small3d(nt=10, green_mode=True, green_cmp="z", green_trise=1.0, green_station=0, sources=[])
    g = Swpc3D(p)
    b0 = g.lib.swpc_device_bytes(g.ctx)
    ig, jg, kg = green_table(p, n=8)
    g.green_store_setup(ig, jg, kg, bforce=True)
    g.green_store_setup(ig, jg, kg)
    assert g.lib.swpc_device_bytes(g.ctx) > b0
    g.green_store_setup([], [], [])
    assert g.lib.swpc_device_bytes(g.ctx) == b0
