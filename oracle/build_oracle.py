"""Build recipe for the CPU oracle (test infrastructure only).

Compiles the C restatements in this directory into ``oracle/lib``:
    liboracle3d_f32.so    MP = SP build (the FP32 parity reference)
    liboracle3d_mixed.so  MP = DP, SP medium/memory variables (reference default)
    liboracle3d_f64.so    all double (error reference)
All builds use -ffp-contract=off so that the f32 build rounds every
operation as the Fortran source spells it out.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "lib"

VARIANTS = {
    "f32": ("float", "float"),
    "mixed": ("double", "float"),
    "f64": ("double", "double"),
}
SOURCES = {"3d": "swpc3d_oracle.c", "2d": "swpc2d_oracle.c"}


def build(verbose: bool = False) -> list[Path]:
    LIB.mkdir(exist_ok=True)
    out = []
    for kind, src in SOURCES.items():
        s = HERE / src
        if not s.exists():
            continue
        for name, (mpr, spr) in VARIANTS.items():
            so = LIB / f"liboracle{kind}_{name}.so"
            if so.exists() and so.stat().st_mtime > s.stat().st_mtime:
                out.append(so)
                continue
            cmd = ["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
                   f"-DMPR={mpr}", f"-DSPR={spr}", "-o", str(so), str(s), "-lm"]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
            out.append(so)
    return out


if __name__ == "__main__":
    for p in build(verbose="-v" in sys.argv):
        print(p)
