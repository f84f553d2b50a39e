"""Generate tests/golden/fcy_run.json from the reference's recorded ensemble job.

Besides example/example.out, the reference holds one more recorded run: the
first job of its ensemble driver (work/auto_chengyu.py), whose progress lines
are in work/joblog/20250529_113331.log.  That job ran work/input_fcy.inf
(400 x 400 x 270 cells, dx = 10 m, dt = 1 ms, uniform medium, PML 20) with
work/source_fcy.dat (one double couple given by moment magnitude and strike,
dip, rake) and printed max |V| at the surface every 100 steps with 3
significant digits until it was killed after step 700, plus the minimum and
maximum velocity of the medium in its header.  This script reads those files
from a checkout of the reference and writes them as a fixture, so the GPU
known-answer test needs no reference checkout at run time.

Usage: python tests/golden/make_fcy_golden.py /path/to/OpenSWPC
"""
import json
import re
import sys
from pathlib import Path


def read_inf(path: Path) -> dict:
    kv = {}
    for line in path.read_text().splitlines():
        line = re.sub(r"!!.*$", "", line).strip()
        if "=" in line and not line.startswith("#"):
            k, v = line.split("=", 1)
            kv[k.strip()] = v.strip().strip("'\"")
    return kv


def main(ref: Path) -> None:
    work = ref / "work"
    kv = read_inf(work / "input_fcy.inf")
    keys = ["nx", "ny", "nz", "nt", "dx", "dy", "dz", "dt", "vcut", "xbeg", "ybeg", "zbeg", "tbeg", "fq_min",
            "fq_max", "fq_ref", "na", "ntdec_r", "stftype", "stf_format", "sdep_fit", "vmodel_type", "vp0", "vs0",
            "rho0", "qp0", "qs0", "topo0", "abc_type", "is_ocean", "munk_profile", "earth_flattening",
            "stabilize_pml"]
    params = {k: kv[k] for k in keys}
    sources = []
    for line in (work / "source_fcy.dat").read_text().splitlines():
        s = line.strip()
        if s and not s.startswith("#"):
            sources.append([float(x) for x in s.split()[:9]])
    log = (work / "joblog" / "20250529_113331.log").read_text()
    reports = []
    for line in log.splitlines():
        m = re.match(r"\s*it=(\d+),.*\(\s*(\S+)\s+(\S+)\s+(\S+)\s*\)", line)
        if m:
            reports.append([int(m.group(1))] + [float(m.group(q)) for q in (2, 3, 4)])
    header = {}
    for line in log.splitlines():
        m = re.match(r"\s*(Minimum velocity|Maximum velocity|Stability  Condition c|Maximum frequency)\s*:\s*(\S+)",
                     line)
        if m:
            header[m.group(1)] = float(m.group(2))
    out = {"source": "work/input_fcy.inf, work/source_fcy.dat, work/joblog/20250529_113331.log",
           "params": params, "sources": sources, "reports": reports, "header": header}
    dst = Path(__file__).resolve().parent / "fcy_run.json"
    dst.write_text(json.dumps(out, indent=1) + "\n")
    print(dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fcy_golden.py /path/to/OpenSWPC")
    main(Path(sys.argv[1]))
