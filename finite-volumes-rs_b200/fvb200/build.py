"""Build libfvb200.so (CUDA for sm_100a + host C++) in-tree.

The library is compiled with --fmad=false and -ffp-contract=off: the
reference's Rust arithmetic never fuses a*b+c, and bit-level parity of
assembly, SpMV, factorisation and the triangular sweeps depends on keeping
both roundings.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent          # .../finite-volumes-rs_b200/fvb200
ROOT = PKG.parent.parent                         # repository root
CSRC = PKG.parent / "csrc"
INCLUDE = ROOT / "include"
LIB = PKG / "libfvb200.so"

CUDA_SOURCES = ["fv_assembly.cu", "fv_precond.cu", "fv_solvers.cu", "fv_batch.cu", "fv_dist.cu", "fv_tiles.cu", "fv_fill.cu", "fv_meshbuild.cu", "fv_vector.cu"]
HOST_SOURCES = ["meshgen.cpp", "fv_order.cpp"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "--fmad=false", "--extended-lambda",
    "-Xcompiler", "-fPIC,-fopenmp,-ffp-contract=off,-O2",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def sources() -> list[Path]:
    out = [CSRC / s for s in CUDA_SOURCES + HOST_SOURCES if (CSRC / s).exists()]
    return out


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    deps = sources() + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h")) + [Path(__file__)]
    return all(d.stat().st_mtime <= t for d in deps)


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    if not force and up_to_date():
        return LIB
    objdir = PKG.parent / "_build"
    objdir.mkdir(exist_ok=True)
    nvcc = _nvcc()
    cmds, objs = [], []
    for src in sources():
        obj = objdir / (src.stem + ".o")
        cmd = [nvcc, *NVCC_FLAGS, *(extra or []), "-I", str(INCLUDE), "-I", str(CSRC), "-c", str(src), "-o", str(obj)]
        if src.suffix == ".cpp":
            cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-fopenmp", "-ffp-contract=off",
                   "-I", str(INCLUDE), "-I", "/usr/local/cuda/include", "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        cmds.append(cmd)
        objs.append(str(obj))
    # the translation units compile independently: run them side by side
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for r in list(ex.map(lambda c: subprocess.run(c, check=False), cmds)):
            if r.returncode != 0:
                raise subprocess.CalledProcessError(r.returncode, r.args)
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", str(tmp),
           "-Xcompiler", "-fopenmp", "-lgomp"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
