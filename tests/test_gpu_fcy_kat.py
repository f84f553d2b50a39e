"""Known-answer test: the reference's recorded ensemble job.

The first job of the reference's ensemble driver ran work/input_fcy.inf: 400 x
400 x 270 cells of 10 m, dt = 1 ms, PML 20, a uniform medium (vmodel_type
'uni': vp 3.5, vs 2.0 km/s, rho 2.5, Qp 200, Qs 100 below topo0 = 0, air
above) and one double couple of moment magnitude 1.0 at 0.6 km depth
(work/source_fcy.dat, Kupper time function).  Its log
(work/joblog/20250529_113331.log) holds the medium's minimum and maximum
velocity and max |V| at the surface every 100 steps up to step 700, with 3
significant digits; the fixture tests/golden/fcy_run.json (written by
tests/golden/make_fcy_golden.py) carries them.

The uniform model is run as a layered model of one layer whose top is topo0:
vmodel_uni (src/swpc_3d/m_vmodel_uni.f90:95-128) puts the medium where
z > topo0 and air (rho 0.001, Q 10) elsewhere, vmodel_lhm
(src/swpc_3d/m_vmodel_lhm.f90:109-149) puts the first layer where z >= its
depth and the same air above; the two differ only at a cell centre exactly on
topo0, and this grid has none (z = -0.1 + (k - 0.5) * 0.01 km).  The run used
the reference's default mixed precision, so each value is compared to one
unit of its last printed digit, as in the example known-answer test."""
import json
import math
from pathlib import Path

import numpy as np
import pytest

from openswpc_b200.params import Layer, Params, dc_source

GOLDEN = Path(__file__).resolve().parent / "golden" / "fcy_run.json"


def fcy_params() -> tuple[Params, dict]:
    g = json.loads(GOLDEN.read_text())
    kv = g["params"]
    f = lambda k: float(kv[k])
    layers = [Layer(f("topo0"), f("rho0"), f("vp0"), f("vs0"), f("qp0"), f("qs0"))]
    x, y, z, tbeg, trise, mw, strike, dip, rake = g["sources"][0]
    # seismic moment of a moment magnitude (m_fdtool.f90:302), in the precision of the reference's reals
    mo = float(np.float32(10.0) ** (np.float32(1.5) * np.float32(mw) + np.float32(9.05)))
    src = dc_source(x, y, z, tbeg, trise, mo, strike, dip, rake)
    p = Params(nx=int(kv["nx"]), ny=int(kv["ny"]), nz=int(kv["nz"]), nt=int(kv["nt"]), dx=f("dx"), dy=f("dy"),
               dz=f("dz"), dt=f("dt"), vcut=f("vcut"), xbeg=f("xbeg"), ybeg=f("ybeg"), zbeg=f("zbeg"),
               tbeg=f("tbeg"), fq_min=f("fq_min"), fq_max=f("fq_max"), fq_ref=f("fq_ref"), na=int(kv["na"]),
               ntdec_r=int(kv["ntdec_r"]), stftype=kv["stftype"], sdep_fit=kv["sdep_fit"], nm=3, layers=layers,
               sources=[src], stations=[])
    return p, g


def test_fcy_fixture_is_consistent():
    p, g = fcy_params()
    kv = g["params"]
    assert (p.nx, p.ny, p.nz, p.na, p.ntdec_r) == (400, 400, 270, 20, 100)
    assert kv["vmodel_type"] == "uni" and kv["stf_format"] == "xymwdc" and kv["abc_type"] == "pml"
    assert kv["is_ocean"] == ".false." and kv["earth_flattening"] == ".false." and kv["stabilize_pml"] == ".false."
    assert [r[0] for r in g["reports"]] == list(range(100, 701, 100))
    # no cell centre lies on topo0, where vmodel_uni and vmodel_lhm would differ
    zc = np.float32(p.zbeg) + (np.arange(-2, p.nz + 4, dtype=np.float32) - np.float32(0.5)) * np.float32(p.dz)
    assert not np.any(zc == np.float32(kv["topo0"]))


def last_digit(v: float) -> float:
    """One unit in the 3rd significant digit of v."""
    return 10.0 ** (math.floor(math.log10(abs(v))) - 2)


@pytest.mark.gpu
def test_fcy_run_matches_recorded_progress():
    from openswpc_b200.swpc3d import Swpc3D

    p, g = fcy_params()
    last = g["reports"][-1][0]
    with Swpc3D(p) as sim:
        hdr = g["header"]
        assert abs(sim.medium.vmin - hdr["Minimum velocity"]) <= 1e-3 + 1e-6, sim.medium.vmin
        assert abs(sim.medium.vmax - hdr["Maximum velocity"]) <= 1e-3 + 1e-6, sim.medium.vmax
        got = dict((it, va) for it, va in sim.run(1, last))
    bad = []
    for it, *want in g["reports"]:
        for c in range(3):
            v = float(got[it][c])
            if want[c] == 0.0:
                if v != 0.0:
                    bad.append((it, c, v, want[c]))
            elif abs(v - want[c]) > last_digit(want[c]):
                bad.append((it, c, v, want[c]))
    print({it: [float(x) for x in va] for it, va in got.items()})
    assert not bad, bad
