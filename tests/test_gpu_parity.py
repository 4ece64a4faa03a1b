"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

Bars: CSR pattern and level schedules bit-exact; assembled coefficients,
SpMV, IC(0)/ILU(0) factors and a preconditioner apply bit-exact (same
operation order, no FMA); Krylov solutions within 1e-10 relative L2 of the
oracle's at tolerance 1e-12, iteration counts within +-2.
"""
import numpy as np
import pytest

from cases import convdiff_3d, diffusion_2d, equation, oracle_system

pytestmark = pytest.mark.gpu


def _gpu_system(fv, case):
    A, b = fv.assemble(equation(fv, case), (case["bndi"], case["bnde"]), case["mesh"])
    return A, b


@pytest.mark.parametrize("which", ["2d", "3d"])
def test_assembly_bit_exact(fv, orc, which):
    case = diffusion_2d(fv, 16) if which == "2d" else convdiff_3d(fv, 5)
    ptr, cols, vals, rhs = oracle_system(orc, case)
    A, b = _gpu_system(fv, case)
    gp, gc, gv = A.to_csr()
    assert np.array_equal(gp, ptr)
    assert np.array_equal(gc, cols)
    assert np.array_equal(gv, vals), np.abs(gv - vals).max()
    assert np.array_equal(b.numpy(), rhs)


def test_boundary_closure_nonzero(fv, orc):
    """Dirichlet g != 0 and zero-gradient faces exercise both bndi and bnde."""
    case = convdiff_3d(fv, 4, seed=11)
    nb = case["mesh"].n_boundary_faces
    rng = np.random.default_rng(0)
    case["bndi"] = (rng.random(nb) < 0.3).astype(np.float64)
    case["bnde"] = np.where(case["bndi"] == 0.0, rng.standard_normal(nb), 0.0)
    ptr, cols, vals, rhs = oracle_system(orc, case)
    A, b = _gpu_system(fv, case)
    gp, gc, gv = A.to_csr()
    assert np.array_equal(gv, vals)
    assert np.array_equal(b.numpy(), rhs)


@pytest.mark.parametrize("which", ["2d", "3d"])
def test_spmv_bit_exact(fv, orc, which):
    case = diffusion_2d(fv, 16) if which == "2d" else convdiff_3d(fv, 5)
    ptr, cols, vals, _ = oracle_system(orc, case)
    A = fv.DistributedMatrix.from_csr(ptr, cols, vals)
    x = np.random.default_rng(1).standard_normal(len(ptr) - 1)
    y = fv.DistributedVector.from_size(len(x))
    A.imul(y, x)
    assert np.array_equal(y.numpy(), orc.spmv(ptr, cols, vals, x))


def test_ic0_factor_and_apply_bit_exact(fv, orc):
    case = diffusion_2d(fv, 20)
    ptr, cols, vals, rhs = oracle_system(orc, case)
    A = fv.DistributedMatrix.from_csr(ptr, cols, vals)
    P = fv.IncompleteCholesky.from_matrix(A, 0)
    o = orc.Precond("ic", ptr, cols, vals)
    op, oc, ov, _, _ = o.export()
    gp, gc, gv, _ = P.factors()
    assert np.array_equal(gp, op) and np.array_equal(gc, oc)
    assert np.array_equal(gv, ov), np.abs(gv - ov).max()
    z = fv.DistributedVector.from_size(len(rhs))
    P.precondition(z, fv.DistributedVector(rhs))
    assert np.array_equal(z.numpy(), o.apply(rhs))
    # levels bit-exact against the oracle's schedule of the same pattern
    fl, bl, nf, nb = P.levels()
    lo, nlo = orc.levels(ptr, cols, upper=False)
    up, nup = orc.levels(ptr, cols, upper=True)
    assert np.array_equal(fl, lo) and nf == nlo
    assert np.array_equal(bl, up) and nb == nup


def test_ilu0_factor_and_apply_bit_exact(fv, orc):
    case = convdiff_3d(fv, 6)
    ptr, cols, vals, rhs = oracle_system(orc, case)
    A = fv.DistributedMatrix.from_csr(ptr, cols, vals)
    P = fv.IncompleteLowerUpper.from_matrix(A, 0)
    o = orc.Precond("ilu", ptr, cols, vals)
    op, oc, ov, _, ond = o.export()
    gp, gc, gv, gnd = P.factors()
    assert gnd == ond
    assert np.array_equal(gp, op) and np.array_equal(gc, oc)
    assert np.array_equal(gv, ov), np.abs(gv - ov).max()
    z = fv.DistributedVector.from_size(len(rhs))
    P.precondition(z, fv.DistributedVector(rhs))
    assert np.array_equal(z.numpy(), o.apply(rhs))
    # a second apply reuses the sentinel-reset buffers
    r2 = np.random.default_rng(2).standard_normal(len(rhs))
    P.precondition(z, fv.DistributedVector(r2))
    assert np.array_equal(z.numpy(), o.apply(r2))


def test_ilu0_drop_rule(fv, orc):
    """A matrix with tiny off-diagonals: the 1e-6 drop rule removes entries."""
    case = convdiff_3d(fv, 4, seed=9)
    ptr, cols, vals, rhs = oracle_system(orc, case)
    vals = vals.copy()
    rng = np.random.default_rng(4)
    for i in range(len(ptr) - 1):
        for k in range(ptr[i], ptr[i + 1]):
            if cols[k] != i and rng.random() < 0.2:
                vals[k] *= 1e-9
    A = fv.DistributedMatrix.from_csr(ptr, cols, vals)
    P = fv.IncompleteLowerUpper.from_matrix(A, 0)
    o = orc.Precond("ilu", ptr, cols, vals)
    op, oc, ov, _, ond = o.export()
    gp, gc, gv, gnd = P.factors()
    assert ond > 0 and gnd == ond
    assert np.array_equal(gp, op) and np.array_equal(gc, oc) and np.array_equal(gv, ov)
    z = fv.DistributedVector.from_size(len(rhs))
    P.precondition(z, fv.DistributedVector(rhs))
    assert np.array_equal(z.numpy(), o.apply(rhs))


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_cg_ic0_matches_oracle(fv, orc):
    case = diffusion_2d(fv, 32)
    ptr, cols, vals, rhs = oracle_system(orc, case)
    o = orc.Precond("ic", ptr, cols, vals)
    xo, io = orc.cg(ptr, cols, vals, o, rhs, rtol=1e-12, atol=1e-12, maxit=2000)
    A, b = _gpu_system(fv, case)
    P = fv.IncompleteCholesky.from_matrix(A, 0)
    x = fv.DistributedVector.from_size(case["mesh"].n_cells)
    opts = fv.LinearSolverOptions(1e-12, 1e-12, 2000)
    info = fv.conjugate_gradient(x, A, b, P, None, opts)
    assert info.status == 0
    assert abs(info.iterations - io["iterations"]) <= 2
    assert _rel(x.numpy(), xo) <= 1e-10
    assert abs(info.initial_residual - io["initial_residual"]) <= 1e-12 * io["initial_residual"]
    assert len(info.history) == info.iterations


def test_bicgstab_ilu0_matches_oracle(fv, orc):
    case = convdiff_3d(fv, 8)
    ptr, cols, vals, rhs = oracle_system(orc, case)
    o = orc.Precond("ilu", ptr, cols, vals)
    xo, io = orc.bicgstab(ptr, cols, vals, o, rhs, rtol=1e-12, atol=1e-12, maxit=2000)
    A, b = _gpu_system(fv, case)
    P = fv.IncompleteLowerUpper.from_matrix(A, 0)
    x = fv.DistributedVector.from_size(case["mesh"].n_cells)
    info = fv.bi_conjugate_gradient_stab(x, A, b, P, None, fv.LinearSolverOptions(1e-12, 1e-12, 2000))
    assert info.status == 0
    assert abs(info.iterations - io["iterations"]) <= 2
    assert _rel(x.numpy(), xo) <= 1e-10


def test_solvers_at_benchmark_tolerance(fv, orc):
    """rtol = atol = 1e-8 as in the benchmark configs: iterations within +-2,
    and the solution within 1e-10 of the oracle's."""
    case = diffusion_2d(fv, 48, seed=8)
    ptr, cols, vals, rhs = oracle_system(orc, case)
    xo, io = orc.cg(ptr, cols, vals, orc.Precond("ic", ptr, cols, vals), rhs, rtol=1e-8, atol=1e-8, maxit=5000)
    A, b = _gpu_system(fv, case)
    x = fv.DistributedVector.from_size(case["mesh"].n_cells)
    info = fv.conjugate_gradient(x, A, b, fv.IncompleteCholesky.from_matrix(A, 0), None,
                                 fv.LinearSolverOptions(1e-8, 1e-8, 5000))
    assert abs(info.iterations - io["iterations"]) <= 2
    assert _rel(x.numpy(), xo) <= 1e-10


def test_identity_preconditioner_and_zero_rhs(fv, orc):
    case = diffusion_2d(fv, 12)
    ptr, cols, vals, rhs = oracle_system(orc, case)
    A = fv.DistributedMatrix.from_csr(ptr, cols, vals)
    xo, io = orc.cg(ptr, cols, vals, None, rhs, rtol=1e-10, atol=1e-10, maxit=1000)
    x = fv.DistributedVector.from_size(len(rhs))
    info = fv.conjugate_gradient(x, A, fv.DistributedVector(rhs), None, None, fv.LinearSolverOptions(1e-10, 1e-10))
    assert abs(info.iterations - io["iterations"]) <= 2
    assert _rel(x.numpy(), xo) <= 1e-9
    # |b| < 1e-14: x = 0, zero iterations (conjugate_gradient.rs:31-36)
    x = fv.DistributedVector(np.ones(len(rhs)))
    info = fv.conjugate_gradient(x, A, fv.DistributedVector(np.zeros(len(rhs))), None)
    assert info.iterations == 0 and np.all(x.numpy() == 0.0) and info.history == [0.0]


@pytest.mark.parametrize("kind", ["2d", "3d"])
def test_diagonal_preconditioner_matches_oracle(fv, orc, kind):
    """DiagonalPreconditioner: apply bit for bit, the exported inverse diagonal, and a
    CG (2D) / BiCGStab (3D) solve against the oracle (<=1e-10, iterations +-2)."""
    case = diffusion_2d(fv, 20, seed=12) if kind == "2d" else convdiff_3d(fv, 5, seed=12)
    ptr, cols, vals, rhs = oracle_system(orc, case)
    A = fv.DistributedMatrix.from_csr(ptr, cols, vals)
    P = fv.DiagonalPreconditioner.from_matrix(A)
    o = orc.Precond("diag", ptr, cols, vals)
    r = np.random.default_rng(3).standard_normal(len(rhs))
    z = fv.DistributedVector.from_size(len(rhs))
    P.precondition(z, fv.DistributedVector(r))
    assert np.array_equal(z.numpy(), o.apply(r))
    dp, dc, dv, _ = P.factors()
    diag = np.array([vals[k] for i in range(len(rhs)) for k in range(ptr[i], ptr[i + 1]) if cols[k] == i])
    assert np.array_equal(dc, np.arange(len(rhs))) and np.array_equal(dv, 1.0 / diag)
    opts = fv.LinearSolverOptions(1e-10, 1e-10, 5000)
    x = fv.DistributedVector.from_size(len(rhs))
    if kind == "2d":
        info = fv.conjugate_gradient(x, A, fv.DistributedVector(rhs), P, None, opts)
        xo, io = orc.cg(ptr, cols, vals, o, rhs, rtol=1e-10, atol=1e-10, maxit=5000)
    else:
        info = fv.bi_conjugate_gradient_stab(x, A, fv.DistributedVector(rhs), P, None, opts)
        xo, io = orc.bicgstab(ptr, cols, vals, o, rhs, rtol=1e-10, atol=1e-10, maxit=5000)
    assert abs(info.iterations - io["iterations"]) <= 2
    assert np.linalg.norm(x.numpy() - xo) <= 1e-10 * np.linalg.norm(xo)
    # another matrix on the same pattern
    A2 = fv.DistributedMatrix.from_csr(ptr, cols, 2.0 * np.asarray(vals))
    P2 = fv.DiagonalPreconditioner.from_matrix(A2)
    P2.precondition(z, fv.DistributedVector(r))
    assert np.array_equal(z.numpy(), orc.Precond("diag", ptr, cols, 2.0 * np.asarray(vals)).apply(r))


def test_face_constraints_as_boundary_condition(fv, orc):
    """A FaceConstraints passed to assemble gives the same system as its (bndi, bnde) arrays and the oracle."""
    case = diffusion_2d(fv, 12, seed=21)
    m = case["mesh"]
    fc = fv.FaceConstraints.from_mesh(m)
    fb0 = m.n_faces - m.n_boundary_faces
    for f in range(fb0, m.n_faces):
        fc[f] = (1.0, 0.0) if m.face_center[f, 0] > 0.999 else (0.0, float(m.face_center[f, 1]))
    bi, be = fc.as_bc()
    A, b = fv.assemble(equation(fv, case), fc, m)
    ptr, cols, vals, rhs = orc.assemble(m, case["c_lap"], case["c_conv"], case["c_src"], kappa=case["kappa"],
                                        flux=case["flux"], source=case["source"], bndi=bi, bnde=be)
    gp, gc, gv = A.to_csr()
    assert np.array_equal(gp, ptr) and np.array_equal(gc, cols) and np.array_equal(gv, vals)
    assert np.array_equal(b.numpy(), rhs)
