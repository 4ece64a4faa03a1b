"""Generate the golden fixtures of tests/golden/ from the CPU oracle.

    python tests/golden/make_golden.py            (FV_REFERENCE_DIR=<reference checkout> also
                                                   writes square_su2_input.npz)

The reference crate cannot be built in this environment (no Rust toolchain,
no MPI), so these vectors come from the oracle (oracle/oracle.c, a
restatement of the reference's algorithms): they freeze the oracle's
outputs on small seeded inputs, and the GPU tests compare against them
without needing the oracle library.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "finite-volumes-rs_b200"))
sys.path.insert(0, str(HERE.parent))

CASES = ["square8_diffusion", "cube3_convdiff"]


def compute(fv, orc, name):
    from cases import convdiff_3d, diffusion_2d, oracle_system
    if name == "square8_diffusion":
        case = diffusion_2d(fv, 8, seed=21)
        kind, solve = "ic", orc.cg
    else:
        case = convdiff_3d(fv, 3, seed=22)
        kind, solve = "ilu", orc.bicgstab
    ptr, cols, vals, rhs = oracle_system(orc, case)
    pc = orc.Precond(kind, ptr, cols, vals)
    fp, fc, fv_, _, nd = pc.export()
    x, info = solve(ptr, cols, vals, pc, rhs, rtol=1e-10, atol=1e-10, maxit=500)
    lev, _ = orc.levels(ptr, cols)
    blev, _ = orc.levels(ptr, cols, upper=True)
    return {
        "row_ptr": ptr, "cols": cols, "vals": vals, "rhs": rhs,
        "f_ptr": fp, "f_cols": fc, "f_vals": fv_, "n_dropped": np.array([nd]),
        "fwd_level": lev, "bwd_level": blev,
        "x_solve": x, "iterations": np.array([info["iterations"]]),
        "z_apply": pc.apply(rhs),
    }


def square_su2_input():
    """The parsed contents of the reference's square.su2 (the input of its mesh
    known-answer test, core/mesh/io.rs:569-590), read from the reference
    checkout named by FV_REFERENCE_DIR; None when it is not available."""
    import os
    from oracle import mesh_ref
    base = os.environ.get("FV_REFERENCE_DIR")
    path = Path(base) / "src/core/mesh/examples/square.su2" if base else None
    if path is None or not path.exists():
        return None
    dim, nodes, elements, boundaries = mesh_ref.read_su2(path.read_text())
    bkeys = list(boundaries.items())
    return {
        "dim": np.array(dim), "nodes": np.array(nodes),
        "elem_kind": np.array([k for k, _ in elements], np.int32),
        "elem_ptr": np.concatenate([[0], np.cumsum([len(n) for _, n in elements])]).astype(np.int32),
        "elem_nodes": np.array([v for _, n in elements for v in n], np.int32),
        "bnd_ptr": np.concatenate([[0], np.cumsum([len(k) for k, _ in bkeys])]).astype(np.int32),
        "bnd_nodes": np.array([v for k, _ in bkeys for v in k], np.int32),
        "bnd_marker": np.array([mk for _, mk in bkeys], np.int32),
    }


def main():
    su2 = square_su2_input()
    if su2 is not None:
        np.savez_compressed(HERE / "square_su2_input.npz", **su2)
        print("square_su2_input", {k: v.shape for k, v in su2.items()})
    if "--su2-only" in sys.argv:
        return
    from fvb200.build import build
    build()
    import fvb200 as fv
    import oracle as orc
    for name in CASES:
        out = compute(fv, orc, name)
        np.savez_compressed(HERE / f"{name}.npz", **out)
        print(name, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
