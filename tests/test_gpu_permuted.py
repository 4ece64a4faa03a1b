"""Permuted systems on the GPU: B = Q A Q^T built on the device
(fv_csr_permute), factorised and solved in B's numbering.

- B's CSR equals the oracle's permutation of A, bit for bit; re-permuting
  after A's values changed (fv_csr_permute_values) too
- with the box order, B's rows are sorted by level, so its IC(0)/ILU(0)
  sweeps consecutive rows (schedule 4): factors equal the oracle's on B, and
  the apply equals the oracle's on B and the level-chunk apply, bit for bit
- the apply in B's numbering equals the reordered preconditioner applied in
  A's numbering (fv_*_factor_perm), bit for bit
- CG / BiCGStab on B: solution within 1e-10 of the oracle's solve on B,
  iterations +-2, and unpermuted it solves A x = b
- vector permutation round trip; a non-permutation is rejected
"""
import numpy as np
import pytest

from cases import convdiff_3d, diffusion_2d, equation, oracle_system

pytestmark = pytest.mark.gpu

SOL_TOL = 1e-10  # relative L2 bound on solutions (the FP64 parity bar)


def _case(fv, which, n=None):
    if which == 0:
        return "ic", diffusion_2d(fv, n or 24, seed=41)
    return "ilu", convdiff_3d(fv, n or 8, seed=42)


def _permuted(fv, case):
    A, b = fv.assemble(equation(fv, case), (case["bndi"], case["bnde"]), case["mesh"])
    perm, _ = fv.order_boxes(A)
    return A, b, perm, A.permuted(perm)


@pytest.mark.parametrize("which", [0, 1])
def test_permuted_matrix_factors_and_apply(fv, orc, which):
    kind, case = _case(fv, which)
    ptr, cols, vals, rhs = oracle_system(orc, case)
    A, b, perm, B = _permuted(fv, case)
    bp, bc, bv = orc.permute(ptr, cols, vals, perm)
    gp, gc, gv = B.to_csr()
    assert np.array_equal(gp, bp) and np.array_equal(gc, bc) and np.array_equal(gv, bv)
    cls = fv.IncompleteCholesky if kind == "ic" else fv.IncompleteLowerUpper
    P = cls.from_matrix(B, 0)
    assert P.schedule()[0] == 4  # rows sorted by level: consecutive-row sweeps
    o = orc.Precond(kind, bp, bc, bv)
    fp, fc, fvv, fd = P.factors()
    op_, oc, ov, _, od = o.export()
    assert np.array_equal(fp, op_) and np.array_equal(fc, oc) and np.array_equal(fvv, ov) and fd == od
    Pq = cls.from_matrix(A, 0, ordering=perm)  # the same factorisation applied in A's numbering
    rng = np.random.default_rng(11)
    n = len(rhs)
    for grid, rpt in ((0, 0), (148, 1), (1184, 2), (37, 8), (0, 0)):
        P.set_grid(grid, rpt)
        r = rng.standard_normal(n)
        z = fv.DistributedVector.from_size(n)
        P.precondition(z, fv.DistributedVector(r))
        zb = z.numpy()
        assert np.array_equal(zb, o.apply(r))
        # level chunks give the same bits
        P.schedule(1)
        z1 = fv.DistributedVector.from_size(n)
        P.precondition(z1, fv.DistributedVector(r))
        assert np.array_equal(z1.numpy(), zb)
        P.schedule(4)
        # A's numbering: Q^T M_B^-1 Q r
        ra = np.empty(n)
        ra[perm] = r
        za = fv.DistributedVector.from_size(n)
        Pq.precondition(za, fv.DistributedVector(ra))
        assert np.array_equal(za.numpy()[perm], zb)


@pytest.mark.parametrize("which", [0, 1])
def test_permuted_solve_matches_oracle(fv, orc, which):
    kind, case = _case(fv, which, n=40 if which == 0 else 12)
    ptr, cols, vals, rhs = oracle_system(orc, case)
    A, b, perm, B = _permuted(fv, case)
    bp, bc, bv = orc.permute(ptr, cols, vals, perm)
    n = len(rhs)
    bq = fv.DistributedVector.from_size(n)
    B.to_permuted(b, bq)
    assert np.array_equal(bq.numpy(), rhs[perm])
    cls = fv.IncompleteCholesky if kind == "ic" else fv.IncompleteLowerUpper
    P = cls.from_matrix(B, 0)
    y = fv.DistributedVector.from_size(n)
    opts = fv.LinearSolverOptions(1e-8, 1e-8, 5000)
    o = orc.Precond(kind, bp, bc, bv)
    if kind == "ic":
        info = fv.conjugate_gradient(y, B, bq, P, None, opts)
        yo, io = orc.cg(bp, bc, bv, o, rhs[perm], rtol=1e-8, atol=1e-8, maxit=5000)
    else:
        info = fv.bi_conjugate_gradient_stab(y, B, bq, P, None, opts)
        yo, io = orc.bicgstab(bp, bc, bv, o, rhs[perm], rtol=1e-8, atol=1e-8, maxit=5000)
    assert info.status == 0
    assert abs(info.iterations - io["iterations"]) <= 2
    assert np.linalg.norm(y.numpy() - yo) <= SOL_TOL * np.linalg.norm(yo)
    x = fv.DistributedVector.from_size(n)
    B.from_permuted(y, x)
    assert np.array_equal(x.numpy()[perm], y.numpy())
    import scipy.sparse as sp
    Ah = sp.csr_matrix((vals, cols, ptr))
    assert np.linalg.norm(rhs - Ah @ x.numpy()) <= 1.01e-8 * np.linalg.norm(rhs)


def test_permuted_values_follow_reassembly(fv, orc):
    kind, case = _case(fv, 1)
    A, b, perm, B = _permuted(fv, case)
    P = fv.IncompleteLowerUpper.from_matrix(B, 0)
    case2 = dict(case, kappa=case["kappa"] * 1.7, flux=case["flux"] * 0.6)
    fv.assemble(equation(fv, case2), (case2["bndi"], case2["bnde"]), case2["mesh"], lhs=A)
    B.refresh_permuted()
    P.refactor()
    ptr, cols, vals, _ = oracle_system(orc, case2)
    bp, bc, bv = orc.permute(ptr, cols, vals, perm)
    assert np.array_equal(B.to_csr()[2], bv)
    _, oc, ov, _, od = orc.Precond("ilu", bp, bc, bv).export()
    _, gc, gv, gd = P.factors()
    assert np.array_equal(gv, ov) and np.array_equal(gc, oc) and gd == od


def test_permuted_rejects_non_permutation(fv):
    _, case = _case(fv, 1)
    A, _ = fv.assemble(equation(fv, case), (case["bndi"], case["bnde"]), case["mesh"])
    n = A.nrows()
    bad = np.arange(n, dtype=np.int32)
    bad[3] = 5
    with pytest.raises(fv.FvError):
        A.permuted(bad)
    with pytest.raises(ValueError):
        A.permuted(np.arange(n - 1, dtype=np.int32))


def test_permuted_system_helper(fv, orc):
    """fvb200.PermutedSystem: the same bits as the steps done by hand, and a
    refresh after re-assembly gives the solve of the new system."""
    kind, case = _case(fv, 1, n=12)
    A, b = fv.assemble(equation(fv, case), (case["bndi"], case["bnde"]), case["mesh"])
    n = A.nrows()
    opts = fv.LinearSolverOptions(1e-8, 1e-8, 5000)
    S = fv.PermutedSystem(A, "ilu")
    assert S.P.schedule()[0] == 4 and S.order_info["n_colours"] == 2
    x = fv.DistributedVector.from_size(n)
    info = S.solve(x, b, opts, initial_guess=False)
    A2, b2, perm2, B2 = _permuted(fv, case)
    P2 = fv.IncompleteLowerUpper.from_matrix(B2, 0)
    bq = fv.DistributedVector.from_size(n)
    B2.to_permuted(b2, bq)
    y = fv.DistributedVector.from_size(n)
    info2 = fv.bi_conjugate_gradient_stab(y, B2, bq, P2, None, opts)
    x2 = fv.DistributedVector.from_size(n)
    B2.from_permuted(y, x2)
    assert info.iterations == info2.iterations and np.array_equal(x.numpy(), x2.numpy())
    # new values: refresh, then solve from the previous solution
    case2 = dict(case, kappa=case["kappa"] * 1.3)
    _, b3 = fv.assemble(equation(fv, case2), (case2["bndi"], case2["bnde"]), case2["mesh"], lhs=A)
    S.refresh()
    S.solve(x, b3, opts)
    ptr, cols, vals, rhs = oracle_system(orc, case2)
    import scipy.sparse as sp
    Ah = sp.csr_matrix((vals, cols, ptr))
    assert np.linalg.norm(rhs - Ah @ x.numpy()) <= 1.01e-8 * np.linalg.norm(rhs)
