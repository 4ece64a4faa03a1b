"""Edge cases on the GPU, with the reference's behaviour as the bar.

- ILU(0) with a pivot below 1e-16 that a later row uses: FV_ERR_SINGULAR_PIVOT
  (the reference panics, incomplete_lower_upper.rs:234-235); a small last
  pivot nobody uses is not an error
- IC(0) of a non-symmetric matrix: FV_ERR_NOT_SYMMETRIC (incomplete_cholesky.rs:153)
- a one-cell mesh: assembly, IC(0) and CG give the oracle's answer
- max_iterations 0, 1, 2: the same iteration counts and iterates as the
  oracle (the loop guard is `iter > max_iter`, so max 0 still runs one)
- a batch of a single problem equals the plain solver
"""
import numpy as np
import pytest

from cases import diffusion_2d, oracle_system

pytestmark = pytest.mark.gpu


def test_ilu0_singular_pivot(fv):
    from fvb200._lib import FV_ERR_SINGULAR_PIVOT, FvError
    ptr = np.array([0, 2, 4], np.int32)
    cols = np.array([0, 1, 0, 1], np.int32)
    A = fv.DistributedMatrix.from_csr(ptr, cols, np.array([0.0, 1.0, 1.0, 1.0]))
    with pytest.raises(FvError) as e:
        fv.IncompleteLowerUpper.from_matrix(A, 0)
    assert e.value.status == FV_ERR_SINGULAR_PIVOT
    B = fv.DistributedMatrix.from_csr(ptr, cols, np.array([2.0, 1.0, 1.0, 0.0]))
    P = fv.IncompleteLowerUpper.from_matrix(B, 0)  # u_11 = -0.5 is never a pivot
    assert P.factors()[2].shape[0] == 4


def test_ic0_rejects_nonsymmetric(fv):
    from fvb200._lib import FV_ERR_NOT_SYMMETRIC, FvError
    ptr = np.array([0, 2, 4], np.int32)
    cols = np.array([0, 1, 0, 1], np.int32)
    A = fv.DistributedMatrix.from_csr(ptr, cols, np.array([4.0, 1.0, 1.5, 4.0]))
    with pytest.raises(FvError) as e:
        fv.IncompleteCholesky.from_matrix(A, 0)
    assert e.value.status == FV_ERR_NOT_SYMMETRIC


def test_symbolic_analysis_rejects_bad_patterns(fv):
    """The reference indexes [[i, i]] and walks sorted rows: a row without its diagonal, or with
    unsorted / repeated columns, is FV_ERR_INVALID; IC(0) of a structurally unsymmetric pattern is
    FV_ERR_NOT_SYMMETRIC."""
    from fvb200._lib import FV_ERR_INVALID, FV_ERR_NOT_SYMMETRIC, FvError
    for name, (ptr, cols) in {"unsorted": ([0, 2, 4], [1, 0, 0, 1]), "repeated": ([0, 2, 4], [0, 0, 0, 1])}.items():
        with pytest.raises(FvError) as e:  # refused when the matrix is created
            fv.DistributedMatrix.from_csr(np.array(ptr, np.int32), np.array(cols, np.int32), np.ones(len(cols)))
        assert e.value.status == FV_ERR_INVALID, name
    A = fv.DistributedMatrix.from_csr(np.array([0, 2, 3], np.int32), np.array([0, 1, 0], np.int32), np.ones(3))
    for cls in (fv.IncompleteLowerUpper, fv.IncompleteCholesky):
        with pytest.raises(FvError) as e:  # no diagonal in row 1: refused by the symbolic analysis
            cls.from_matrix(A, 0)
        assert e.value.status == FV_ERR_INVALID
    A = fv.DistributedMatrix.from_csr(np.array([0, 2, 3], np.int32), np.array([0, 1, 1], np.int32),
                                      np.array([4.0, 1.0, 4.0]))
    with pytest.raises(FvError) as e:
        fv.IncompleteCholesky.from_matrix(A, 0)
    assert e.value.status == FV_ERR_NOT_SYMMETRIC
    P = fv.IncompleteLowerUpper.from_matrix(A, 0)  # ILU(0) takes it
    z = fv.DistributedVector.from_size(2)
    P.precondition(z, fv.DistributedVector(np.array([1.0, 2.0])))
    assert np.allclose(z.numpy(), np.linalg.solve([[4.0, 1.0], [0.0, 4.0]], [1.0, 2.0]), rtol=1e-15)


def test_one_cell_mesh(fv, orc):
    nodes = np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]])
    bp = np.array([0, 2, 4, 6], np.int32)
    bn = np.array([0, 1, 1, 2, 2, 0], np.int32)
    m = fv.Mesh.from_elements(2, nodes, np.array([5], np.int32), np.array([0, 3], np.int32),
                              np.array([0, 1, 2], np.int32), bp, bn, np.zeros(3, np.int32))
    assert m.n_cells == 1 and m.n_faces == 3 and m.n_boundary_faces == 3
    kf, f = np.ones(3), np.array([2.0])
    bi, be = np.zeros(3), np.array([0.5, 1.0, 1.5])
    A, b = fv.assemble(-fv.laplacian(fv.Orthogonal(), kf) - fv.source(f), (bi, be), m)
    ptr, cols, vals, rhs = orc.assemble(m, -1.0, 0.0, -1.0, kappa=kf, source=f, bndi=bi, bnde=be)
    assert np.array_equal(A.to_csr()[2], vals) and np.array_equal(b.numpy(), rhs)
    P = fv.IncompleteCholesky.from_matrix(A, 0)
    x = fv.DistributedVector.from_size(1)
    info = fv.conjugate_gradient(x, A, b, P, None, fv.LinearSolverOptions(1e-12, 1e-12, 10))
    assert info.iterations == 1
    assert abs(x.numpy()[0] - rhs[0] / vals[0]) <= 1e-15 * abs(rhs[0] / vals[0])


@pytest.mark.parametrize("maxit", [0, 1, 2])
def test_max_iterations_semantics(fv, orc, maxit):
    case = diffusion_2d(fv, 16, seed=21)
    ptr, cols, vals, rhs = oracle_system(orc, case)
    A = fv.DistributedMatrix.from_csr(ptr, cols, vals)
    P = fv.IncompleteCholesky.from_matrix(A, 0)
    x = fv.DistributedVector.from_size(len(rhs))
    info = fv.conjugate_gradient(x, A, fv.DistributedVector(rhs), P, None,
                                 fv.LinearSolverOptions(1e-14, 1e-14, maxit))
    xo, io = orc.cg(ptr, cols, vals, orc.Precond("ic", ptr, cols, vals), rhs, rtol=1e-14, atol=1e-14, maxit=maxit)
    assert info.iterations == io["iterations"] == maxit + 1
    assert np.linalg.norm(x.numpy() - xo) <= 1e-12 * np.linalg.norm(xo)
    xb = fv.DistributedVector.from_size(len(rhs))
    ib = fv.bi_conjugate_gradient_stab(xb, A, fv.DistributedVector(rhs), P, None,
                                       fv.LinearSolverOptions(1e-14, 1e-14, maxit))
    xbo, ibo = orc.bicgstab(ptr, cols, vals, orc.Precond("ic", ptr, cols, vals), rhs, rtol=1e-14, atol=1e-14,
                            maxit=maxit)
    assert ib.iterations == ibo["iterations"]
    assert np.linalg.norm(xb.numpy() - xbo) <= 1e-12 * np.linalg.norm(xbo)


def test_batch_of_one_equals_plain_solver(fv):
    from fvb200.batch import BatchCG, MeshBatch
    case = diffusion_2d(fv, 20, seed=22)
    m = case["mesh"]
    mb = MeshBatch([m])
    nb = m.n_boundary_faces
    eq = -fv.laplacian(fv.Orthogonal(), case["kappa"]) - fv.source(case["source"])
    A, b = fv.assemble(eq, (np.zeros(nb), np.zeros(nb)), mb)
    P = fv.IncompleteCholesky.from_matrix(A, 0)
    x = fv.DistributedVector.from_size(m.n_cells)
    out = BatchCG(A, mb.cell_offsets, 256).solve(P, b, x, precision="fp64", relative_tolerance=1e-10,
                                                 absolute_tolerance=1e-10, max_iterations=2000)
    A1, b1 = fv.assemble(eq, (np.zeros(nb), np.zeros(nb)), m)
    P1 = fv.IncompleteCholesky.from_matrix(A1, 0)
    x1 = fv.DistributedVector.from_size(m.n_cells)
    i1 = fv.conjugate_gradient(x1, A1, b1, P1, None, fv.LinearSolverOptions(1e-10, 1e-10, 2000))
    assert abs(int(out["iterations"][0]) - i1.iterations) <= 2
    assert np.linalg.norm(x.numpy() - x1.numpy()) <= 1e-10 * np.linalg.norm(x1.numpy())
