"""Known-answer test: the reference's recorded example run.

The reference ships no test suite; its one recorded numerical output is
example/example.out, the progress lines of the example (384^3 cells, 1000
steps, eight-layer lhm model, one moment-tensor source): max |V| on the
surface every 50 steps, printed with 3 significant digits.  That run used the
default mixed precision (velocity and stress in double); this library is
FP32, so each value is compared to one unit of its last printed digit.  The
parameters come from tests/golden/example_run.json (written by
tests/golden/make_example_golden.py from the reference's example files)."""
import json
import math
from pathlib import Path

import numpy as np
import pytest

from openswpc_b200.params import Layer, Params, Source

GOLDEN = Path(__file__).resolve().parent / "golden" / "example_run.json"


def example_params() -> tuple[Params, list]:
    g = json.loads(GOLDEN.read_text())
    kv = g["params"]
    f = lambda k: float(kv[k])
    layers = [Layer(*row[:6]) for row in g["layers"]]
    s = g["sources"][0]
    src = Source(*s[:5], mo=s[5], mxx=s[6], myy=s[7], mzz=s[8], myz=s[9], mxz=s[10], mxy=s[11])
    p = Params(nx=int(kv["nx"]), ny=int(kv["ny"]), nz=int(kv["nz"]), nt=int(kv["nt"]), dx=f("dx"), dy=f("dy"),
               dz=f("dz"), dt=f("dt"), vcut=f("vcut"), xbeg=f("xbeg"), ybeg=f("ybeg"), zbeg=f("zbeg"),
               tbeg=f("tbeg"), fq_min=f("fq_min"), fq_max=f("fq_max"), fq_ref=f("fq_ref"), na=int(kv["na"]),
               ntdec_r=int(kv["ntdec_r"]), stftype=kv["stftype"], nm=3, layers=layers, sources=[src],
               stations=[])
    return p, g["reports"]


def test_example_fixture_is_consistent():
    p, reports = example_params()
    assert (p.nx, p.ny, p.nz, p.nt, p.na) == (384, 384, 384, 1000, 20)
    assert [r[0] for r in reports] == list(range(50, 1001, 50))


def last_digit(v: float) -> float:
    """One unit in the 3rd significant digit of v."""
    return 10.0 ** (math.floor(math.log10(abs(v))) - 2)


@pytest.mark.gpu
def test_example_run_matches_recorded_progress():
    from openswpc_b200.swpc3d import Swpc3D

    p, reports = example_params()
    with Swpc3D(p) as sim:
        got = dict((it, va) for it, va in sim.run(1, p.nt))
    bad = []
    for it, *want in reports:
        for c in range(3):
            if abs(float(got[it][c]) - want[c]) > last_digit(want[c]):
                bad.append((it, c, float(got[it][c]), want[c]))
    assert not bad, bad
