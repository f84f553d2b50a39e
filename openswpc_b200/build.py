"""Build the in-tree shared library ``openswpc_b200/lib/libswpc_gpu.so``.

The CUDA sources are compiled for sm_100a only.  The time-step kernels are
compiled with ``-fmad=false`` so that every product and sum is rounded
separately, as the single-precision Fortran expressions of the reference spell
them out; the host setup code is compiled with ``-ffp-contract=off`` for the
same reason.  Run ``python -m openswpc_b200.build`` (or call :func:`build`).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "lib"
OBJDIR = PKG / "lib" / "obj"
LIBNAME = "libswpc_gpu.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC,-fopenmp",
              "-Xptxas", "-O3"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off", "-Wall", "-Wno-unused-function"]

CU_SOURCES = ["swpc3d_kernels.cu", "swpc3d_march.cu", "swpc3d_vec.cu", "swpc2d_kernels.cu", "swpc_api.cu", "swpc2d_api.cu", "swpc_noalloc.cu", "swpc_snap.cu", "swpc_prec.cu", "swpc_adjoint.cu", "swpc_fbatch.cu", "swpc3d_tma.cu", "swpc2d_tma.cu", "swpc_medium.cu", "swpc_green.cu", "swpc_rmedia.cu", "swpc_pw.cu", "swpc_decomp.cu"]
CPP_SOURCES = ["swpc_host.cpp", "swpc_io.cpp"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libswpc_gpu.so")


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout)


def _stale(obj: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build(verbose: bool = False, force: bool = False) -> Path:
    """Compile every source that changed and link the shared library."""
    nvcc = _nvcc()
    OBJDIR.mkdir(parents=True, exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list((PKG.parent / "include").glob("*.h"))
    objs = []
    for src in CU_SOURCES:
        s = CSRC / src
        if not s.exists():
            continue
        o = OBJDIR / (s.stem + ".o")
        if force or _stale(o, [s] + headers):
            cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-c", str(s), "-o", str(o)]
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
        objs.append(o)
    for src in CPP_SOURCES:
        s = CSRC / src
        o = OBJDIR / (s.stem + ".o")
        if force or _stale(o, [s] + headers):
            cmd = ["g++", *CXX_FLAGS, "-c", str(s), "-o", str(o)]
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
        objs.append(o)
    lib = LIBDIR / LIBNAME
    if force or _stale(lib, objs):
        cmd = [nvcc, *ARCH, "-shared", "-Xcompiler", "-fopenmp", "-o", str(lib), *map(str, objs), "-lcudart", "-lcufft"]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
