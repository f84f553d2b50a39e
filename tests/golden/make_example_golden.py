"""Generate tests/golden/example_run.json from the reference's example run.

The reference ships no test suite; its only recorded numerical output is
example/example.out (the progress lines of example/input.inf: max |V| at the
surface every 50 steps, 3 significant digits).  This script reads that log
and the example's input files from a checkout of the reference and writes the
parameters and the recorded values as a fixture, so the GPU known-answer test
needs no reference checkout at run time.

Usage: python tests/golden/make_example_golden.py /path/to/OpenSWPC
"""
import json
import re
import sys
from pathlib import Path


def main(ref: Path) -> None:
    ex = ref / "example"
    kv = {}
    for line in (ex / "input.inf").read_text().splitlines():
        line = re.sub(r"!!.*$", "", line).strip()
        if "=" in line and not line.startswith("#"):
            k, v = line.split("=", 1)
            kv[k.strip()] = v.strip().strip("'\"")
    keys = ["nx", "ny", "nz", "nt", "dx", "dy", "dz", "dt", "vcut", "xbeg", "ybeg", "zbeg", "tbeg", "fq_min",
            "fq_max", "fq_ref", "na", "ntdec_r", "stftype", "stf_format", "vmodel_type"]
    params = {k: kv[k] for k in keys}
    layers = []
    for line in (ex / "lhm.dat").read_text().splitlines():
        s = line.strip()
        if s and not s.startswith("#"):
            layers.append([float(x) for x in s.split()[:6]])
    sources = []
    for line in (ex / "source.dat").read_text().splitlines():
        s = line.strip()
        if s and not s.startswith("#"):
            sources.append([float(x) for x in s.split()[:12]])
    reports = []
    for line in (ex / "example.out").read_text().splitlines():
        m = re.match(r"\s*it=(\d+),.*\(\s*(\S+)\s+(\S+)\s+(\S+)\s*\)", line)
        if m:
            reports.append([int(m.group(1))] + [float(m.group(q)) for q in (2, 3, 4)])
    header = [l.strip() for l in (ex / "example.out").read_text().splitlines()[:14] if ":" in l]
    out = {"source": "example/input.inf, example/lhm.dat, example/source.dat, example/example.out",
           "params": params, "layers": layers, "sources": sources, "reports": reports, "header": header}
    dst = Path(__file__).resolve().parent / "example_run.json"
    dst.write_text(json.dumps(out, indent=1) + "\n")
    print(dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_example_golden.py /path/to/OpenSWPC")
    main(Path(sys.argv[1]))
