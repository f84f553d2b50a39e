"""The bench's reference arm on CPU: `bench.py --impl reference` prints one
JSON line with the keys the measurement contract names (small workloads, a
bounded sample of a few oracle steps)."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
KEYS = {"impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"}


# runs bench.py in this interpreter, then lists the shared objects of the package it mapped
_WRAP = ("import runpy, sys; sys.argv = ['bench.py'] + sys.argv[1:]; runpy.run_path('bench.py', run_name='__main__'); "
         "print('MAPPED', sorted({l.split()[-1] for l in open('/proc/self/maps') if 'openswpc_b200' in l}))")


def run_reference(workload: str, mapped: list | None = None) -> dict:
    out = subprocess.run([sys.executable, "-c", _WRAP, "--impl", "reference", "--workload", workload,
                          "--steps", "3", "--warmup", "3", "--cpu-budget", "2"],
                         cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    if mapped is not None:
        mapped += eval(next(l for l in out.stdout.splitlines() if l.startswith("MAPPED"))[len("MAPPED"):])
    return json.loads(lines[0])


@pytest.mark.parametrize("workload", ["c0", "c2a"])
def test_reference_arm_prints_the_contract_line(workload):
    mapped = []
    line = run_reference(workload, mapped)
    # the reference arm runs the oracle alone: no library of the package is loaded
    assert not mapped, mapped
    assert KEYS <= set(line), KEYS - set(line)
    assert line["impl"] == "reference" and line["value"] > 0 and line["steps"] >= 1
    assert line["cpu_baseline"]["kind"] in ("port", "reference") and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert isinstance(line["config"], dict) and "workload" in line["config"]


def test_reference_arm_without_an_adjoint_says_so():
    line = run_reference("c3")
    assert line == {"impl": "reference", "unavailable": "the reference has no adjoint or gradient path"}


def test_reference_arm_of_the_decomposition_says_so():
    line = run_reference("decomp")
    assert line["impl"] == "reference" and "MPI" in line["unavailable"]
