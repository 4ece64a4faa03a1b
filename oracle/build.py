"""Build the CPU oracle (test infrastructure) as oracle/liboracle.so.

gcc, -O2, -ffp-contract=off: x86-64 SSE2 doubles with no fused multiply-add,
the same arithmetic as the reference's Rust build.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
SRC = [HERE / "oracle.c", HERE / "oracle_mpi.c", HERE / "oracle_mesh.c"]


def build(force: bool = False) -> Path:
    srcs = [s for s in SRC if s.exists()]
    if not force and LIB.exists() and all(s.stat().st_mtime <= LIB.stat().st_mtime for s in srcs + [Path(__file__)]):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = ["gcc", "-O2", "-std=c11", "-ffp-contract=off", "-fPIC", "-shared", "-fopenmp",
           *map(str, srcs), "-o", str(tmp), "-lm"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
