"""CPU tests: the oracle and the host-side mesh builder.

- the reference's own known-answer test on square.su2 (core/mesh/io.rs:564-590)
- the C++ mesh builder against the pure-Python restatement, bit for bit
- the oracle against SciPy (direct solve, factor residuals) and hand values
- committed golden vectors (tests/golden/, made by make_golden.py)
"""
import os
import sys
from pathlib import Path

import numpy as np
import pytest
from conftest import reference_file
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from cases import convdiff_3d, diffusion_2d, oracle_system

SQUARE_SU2 = reference_file("src/core/mesh/examples/square.su2")
GOLDEN = Path(__file__).resolve().parent / "golden"


def _mesh_arrays_equal(m, ref):
    assert m.n_faces == len(ref["face_nodes"])
    assert m.n_cells == len(ref["cell_faces"])
    fn = [list(m.face_nodes[m.face_node_ptr[f]:m.face_node_ptr[f + 1]]) for f in range(m.n_faces)]
    assert fn == [list(x) for x in ref["face_nodes"]]
    cf = [list(m.cell_faces[m.cell_face_ptr[c]:m.cell_face_ptr[c + 1]]) for c in range(m.n_cells)]
    assert cf == ref["cell_faces"]
    assert list(m.face_owner) == ref["face_owner"]
    assert list(m.face_neighbor) == ref["face_neighbor"]
    assert np.array_equal(m.face_area, np.array(ref["face_area"]))
    assert np.array_equal(m.face_normal, np.array(ref["face_normal"]))
    assert np.array_equal(m.face_center, np.array(ref["face_center"]))
    assert np.array_equal(m.cell_center, np.array(ref["cell_center"]))
    assert np.array_equal(m.cell_volume, np.array(ref["cell_volume"]))


def _square_su2_input():
    """The reference's square.su2 as (dim, nodes, elements, boundaries): read
    from the reference checkout when FV_REFERENCE_DIR names one, else from the
    committed fixture of its parsed contents (tests/golden/square_su2_input.npz,
    written by tests/golden/make_golden.py from that file)."""
    from oracle import mesh_ref
    if SQUARE_SU2 is not None:
        return mesh_ref.read_su2(SQUARE_SU2.read_text())
    z = np.load(GOLDEN / "square_su2_input.npz")
    eptr, en = z["elem_ptr"], z["elem_nodes"]
    elements = [(int(k), [int(v) for v in en[eptr[e]:eptr[e + 1]]]) for e, k in enumerate(z["elem_kind"])]
    bptr, bn = z["bnd_ptr"], z["bnd_nodes"]
    boundaries = {tuple(int(v) for v in bn[bptr[b]:bptr[b + 1]]): int(mk) for b, mk in enumerate(z["bnd_marker"])}
    return int(z["dim"]), [list(map(float, p)) for p in z["nodes"]], elements, boundaries


def test_square_su2_known_answer(fv):
    """core/mesh/io.rs:569-590: 121 nodes, 220 faces, 100 cells, total volume 1
    within 10 eps, closed boundary sum(n A) ~ 0 within 10 eps."""
    from oracle import mesh_ref
    dim, nodes, elements, boundaries = _square_su2_input()
    assert dim == 2
    kinds = np.array([k for k, _ in elements], np.int32)
    eptr = np.concatenate([[0], np.cumsum([len(n) for _, n in elements])]).astype(np.int32)
    en = np.array([v for _, n in elements for v in n], np.int32)
    bkeys = list(boundaries.items())
    bptr = np.arange(0, 2 * len(bkeys) + 1, 2, dtype=np.int32)
    bn = np.array([v for k, _ in bkeys for v in k], np.int32)
    bm = np.array([mk for _, mk in bkeys], np.int32)
    m = fv.Mesh.from_elements(2, np.array(nodes), kinds, eptr, en, bptr, bn, bm)
    assert m.n_nodes == 121 and m.n_faces == 220 and m.n_cells == 100
    total_volume = 0.0
    for v in m.cell_volume:
        total_volume += v
    assert abs(total_volume - 1.0) < np.finfo(float).eps * 10
    sf = np.zeros(2)
    for f in range(m.n_faces):
        if m.face_patch[f] >= 0:
            sf += m.face_normal[f] * m.face_area[f]
    assert np.linalg.norm(sf) < np.finfo(float).eps * 10
    ref = mesh_ref.build(2, nodes, elements, boundaries)
    _mesh_arrays_equal(m, ref)


@pytest.mark.skipif(SQUARE_SU2 is None, reason="FV_REFERENCE_DIR unset: reference checkout not available")
def test_square_su2_reader(fv):
    """The library's own SU2 reader on the reference's file gives the restated mesh."""
    from oracle import mesh_ref
    dim, nodes, elements, boundaries = mesh_ref.read_su2(SQUARE_SU2.read_text())
    _mesh_arrays_equal(fv.Mesh.read_su2(SQUARE_SU2), mesh_ref.build(2, nodes, elements, boundaries))


def _square_elements(n):
    el = []
    for j in range(n):
        for i in range(n):
            a = j * (n + 1) + i
            b, c, d = a + 1, a + n + 2, a + n + 1
            el += [(5, [a, b, c]), (5, [a, c, d])]
    return el


def _cube_elements(n):
    n1 = n + 1
    stride = [1, n1, n1 * n1]
    perms = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]
    el = []
    for k in range(n):
        for j in range(n):
            for i in range(n):
                base = (k * n1 + j) * n1 + i
                for p in perms:
                    v = [base]
                    for s in p:
                        v.append(v[-1] + stride[s])
                    el.append((10, v))
    return el


def _boundary_by_count(elements):
    from oracle.mesh_ref import VTK_FACES
    cnt = {}
    for kind, n in elements:
        loc, st = VTK_FACES[kind]
        for i in range(len(st) - 1):
            key = tuple(sorted(n[loc[q]] for q in range(st[i], st[i + 1])))
            cnt[key] = cnt.get(key, 0) + 1
    return {k: 0 for k, c in cnt.items() if c == 1}


@pytest.mark.parametrize("dim,n", [(2, 5), (3, 2)])
def test_generator_matches_restatement(fv, dim, n):
    from oracle import mesh_ref
    m = fv.Mesh.square(n, 0.2, 17) if dim == 2 else fv.Mesh.cube(n, 0.15, 17)
    el = _square_elements(n) if dim == 2 else _cube_elements(n)
    ref = mesh_ref.build(dim, m.nodes.tolist(), el, _boundary_by_count(el))
    _mesh_arrays_equal(m, ref)


def test_benchmark_mesh_sizes(fv):
    """Sizes of the 2D benchmark family: N = 2 n^2, F_b = 4n, nnz = N + 2 F_int."""
    m = fv.Mesh.square(32, 0.2, 1)
    assert m.n_cells == 2 * 32 * 32 and m.n_boundary_faces == 128
    assert m.n_faces == 3 * 32 * 32 + 2 * 32
    m3 = fv.Mesh.cube(4, 0.15, 1)
    assert m3.n_cells == 6 * 64 and m3.n_boundary_faces == 6 * 2 * 16
    assert abs(m3.cell_volume.sum() - 1.0 / 3.0) < 1e-12  # |n| = 1/3 quirk of the reference normal


def test_oracle_assembly_hand_values(fv, orc):
    """Unperturbed 2x2 square, kappa = 1: the two triangles of a square share a
    diagonal of length h*sqrt(2) at centroid distance h*sqrt(2)/3 -> coefficient 3."""
    m = fv.Mesh.square(2, 0.0, 0)
    nb = m.n_boundary_faces
    ptr, cols, vals, rhs = orc.assemble(m, -1.0, 0.0, -1.0, kappa=np.ones(m.n_faces), source=np.ones(m.n_cells),
                                        bndi=np.zeros(nb), bnde=np.zeros(nb))
    A = sp.csr_matrix((vals, cols, ptr))
    assert abs(A[0, 1] + 3.0) < 1e-14 and abs(A[1, 0] + 3.0) < 1e-14
    assert np.allclose(rhs, m.cell_volume)           # f = 1: rhs = f V
    assert np.allclose(A.sum(axis=1).A1[[0]], A.sum(axis=1).A1[[0]])
    assert (A.diagonal() > 0).all()


def test_oracle_cg_ic0_vs_scipy(fv, orc):
    case = diffusion_2d(fv, 24, seed=2)
    ptr, cols, vals, rhs = oracle_system(orc, case)
    A = sp.csr_matrix((vals, cols, ptr))
    assert abs(A - A.T).max() == 0.0
    xs = spla.spsolve(A.tocsc(), rhs)
    pc = orc.Precond("ic", ptr, cols, vals)
    x, info = orc.cg(ptr, cols, vals, pc, rhs, rtol=1e-12, atol=1e-12, maxit=2000)
    assert np.linalg.norm(x - xs) / np.linalg.norm(xs) < 1e-9
    assert len(info["history"]) == info["iterations"]
    # IC(0): L L^T equals A on the pattern of A
    lp, lc, lv, inv, _ = pc.export()
    L = sp.csr_matrix((lv, lc, lp), shape=A.shape)
    R = (L @ L.T - A).tocoo()
    mask = np.asarray(A[R.row, R.col] != 0).ravel()
    assert np.abs(R.data[mask]).max() < 1e-12 * abs(A).max()
    assert np.allclose(inv, 1.0 / L.diagonal(), rtol=0, atol=0)


def test_oracle_bicgstab_ilu0_vs_scipy(fv, orc):
    case = convdiff_3d(fv, 5, seed=3)
    ptr, cols, vals, rhs = oracle_system(orc, case)
    A = sp.csr_matrix((vals, cols, ptr))
    assert abs(A - A.T).max() > 0  # upwind convection is non-symmetric
    xs = spla.spsolve(A.tocsc(), rhs)
    pc = orc.Precond("ilu", ptr, cols, vals)
    x, info = orc.bicgstab(ptr, cols, vals, pc, rhs, rtol=1e-12, atol=1e-12, maxit=2000)
    assert np.linalg.norm(x - xs) / np.linalg.norm(xs) < 1e-9
    # ILU(0): L U equals A on the pattern (unit lower L)
    p, c, v, _, nd = pc.export()
    LU = sp.csr_matrix((v, c, p), shape=A.shape)
    L = sp.tril(LU, -1) + sp.eye(A.shape[0])
    U = sp.triu(LU)
    R = (L @ U - A).tocoo()
    mask = np.asarray(A[R.row, R.col] != 0).ravel()
    assert np.abs(R.data[mask]).max() < 1e-12 * abs(A).max()
    assert nd == 0


def test_oracle_ic_rejects_nonsymmetric(fv, orc):
    case = convdiff_3d(fv, 3, seed=1)
    ptr, cols, vals, _ = oracle_system(orc, case)
    pc = orc.Precond("ic", ptr, cols, vals)
    assert not pc.ok() and pc.status == 6


def test_oracle_levels(fv, orc):
    """Forward levels of the natural ordering: every dependency sits in an earlier level."""
    case = diffusion_2d(fv, 16)
    ptr, cols, vals, _ = oracle_system(orc, case)
    lev, nl = orc.levels(ptr, cols)
    for i in range(len(ptr) - 1):
        for k in range(ptr[i], ptr[i + 1]):
            if cols[k] < i:
                assert lev[cols[k]] < lev[i]
    assert nl == lev.max() + 1


def test_golden_vectors(fv, orc):
    """Oracle outputs match the committed fixtures (tests/golden/make_golden.py)."""
    sys.path.insert(0, str(GOLDEN))
    import make_golden
    for name in make_golden.CASES:
        path = GOLDEN / f"{name}.npz"
        assert path.exists(), f"missing fixture {path}"
        want = np.load(path)
        got = make_golden.compute(fv, orc, name)
        for key in want.files:
            a, b = want[key], got[key]
            if a.dtype.kind == "f" and key.startswith("x_"):
                assert np.linalg.norm(a - b) <= 1e-13 * max(np.linalg.norm(a), 1e-300), key
            else:
                assert np.array_equal(a, b), key


def test_cabi_exports_every_declared_symbol():
    """libfvb200.so exports every function include/fv_b200.h declares (no GPU call)."""
    import re
    root = Path(__file__).resolve().parents[1]
    from fvb200.build import build
    lib = build()
    decl = set()
    for h in (root / "include").glob("*.h"):
        decl |= set(re.findall(r"^\s*(?:const\s+)?\w[\w\s\*]*?\b(fv_\w+)\s*\(", h.read_text(), re.M))
    assert len(decl) > 20
    import ctypes
    L = ctypes.CDLL(str(lib))
    missing = [s for s in sorted(decl) if not hasattr(L, s)]
    assert not missing, missing


def test_graft_entry_build(fv):
    """The entry point's build() runs end to end (library, oracle, package import)."""
    import __graft_entry__
    __graft_entry__.build()


def test_term_algebra(fv):
    k = np.ones(4)
    e = -fv.laplacian(fv.Orthogonal(), k) - fv.source(k)
    assert e.coefficients() == (-1.0, 0.0, -1.0)
    e = fv.convection(fv.Upwind(k), k) - fv.laplacian(fv.Orthogonal(), k) - fv.source(k)
    assert e.coefficients() == (-1.0, 1.0, -1.0)
    e = fv.laplacian(fv.Orthogonal(), k) + fv.source(k)
    assert e.coefficients() == (1.0, 0.0, 1.0)
    with pytest.raises(NotImplementedError):
        fv.laplacian(fv.Orthogonal(), k) + fv.laplacian(fv.Orthogonal(), k)
    with pytest.raises(NotImplementedError):
        fv.laplacian(object(), k)


def test_host_builder_rejects_bad_node_ids(fv):
    """Element or boundary node ids outside [0, n_nodes) are FV_ERR_INVALID, not a read out of bounds."""
    from fvb200._lib import FvError
    nodes = np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]])
    kinds, eptr = np.array([5], np.int32), np.array([0, 3], np.int32)
    bptr = np.array([0, 2, 4, 6], np.int32)
    bm = np.zeros(3, np.int32)
    good_bn = np.array([0, 1, 1, 2, 2, 0], np.int32)
    m = fv.Mesh.from_elements(2, nodes, kinds, eptr, np.array([0, 1, 2], np.int32), bptr, good_bn, bm)
    assert m.n_cells == 1 and m.n_boundary_faces == 3
    for en, bn in ((np.array([0, 1, 3], np.int32), good_bn), (np.array([0, 1, 2], np.int32),
                                                                np.array([0, 1, 1, 2, 2, -1], np.int32))):
        with pytest.raises(FvError) as ei:
            fv.Mesh.from_elements(2, nodes, kinds, eptr, en, bptr, bn, bm)
        assert "FV_ERR_INVALID" in str(ei.value)


def test_oracle_diagonal_preconditioner(fv, orc):
    """DiagonalPreconditioner restated: z = (1 / a_ii) r; a missing diagonal is refused."""
    case = diffusion_2d(fv, 6, seed=4)
    ptr, cols, vals, _ = oracle_system(orc, case)
    A = sp.csr_matrix((vals, cols, ptr))
    r = np.random.default_rng(1).standard_normal(A.shape[0])
    z = orc.Precond("diag", ptr, cols, vals).apply(r)
    assert np.array_equal(z, (1.0 / A.diagonal()) * r)
    bad = orc.Precond("diag", np.array([0, 2, 3]), np.array([0, 1, 0]), np.ones(3))
    assert not bad.ok() and bad.status == 1


def test_face_constraints(fv):
    """FaceConstraints (fvm/bcs/mod.rs): indexed by face id from the first boundary face, (0, 0) by default,
    set per face or for many faces at once; as_bc() is the (bndi, bnde) pair assemble takes."""
    m = fv.Mesh.square(4, 0.0, 0)
    fc = fv.FaceConstraints.from_mesh(m)
    fb0 = m.n_faces - m.n_boundary_faces
    assert fc[fb0] == (0.0, 0.0)
    fc[fb0 + 1] = (1.0, 0.0)
    bottom = [f for f in range(fb0, m.n_faces) if abs(m.face_center[f, 1]) < 1e-12]
    fc[bottom] = (0.0, 2.5)
    bi, be = fc.as_bc()
    assert len(bi) == m.n_boundary_faces and bi[1] == 1.0
    assert np.all(be[np.array(bottom) - fb0] == 2.5)
    with pytest.raises(IndexError):
        fc[0]
