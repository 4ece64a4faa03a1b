"""Reordered (perf-mode) factorisations on the GPU against the oracle run on
the same permuted matrix B = Q A Q^T:

- the device ordering equals the host ordering
- IC(0) / ILU(0) factors of B, the dropped-entry count and the level
  schedules: bit for bit
- the preconditioner apply z = Q^T M_B^{-1} Q r: bit for bit, on repeated
  applies, for the box ordering and for an arbitrary permutation, at any
  sweep grid
- CG / BiCGStab with it: solution within 1e-10 of the oracle's, iterations +-2
- value-only refactorisation after the matrix changed: bit for bit
- a non-permutation is rejected
"""
import numpy as np
import pytest

from cases import convdiff_3d, diffusion_2d, equation, oracle_system

pytestmark = pytest.mark.gpu

SOL_TOL = 1e-10  # relative L2 bound on solutions (the FP64 parity bar)


def _system(fv, case):
    return fv.assemble(equation(fv, case), (case["bndi"], case["bnde"]), case["mesh"])


def _case(fv, which):
    return ("ic", diffusion_2d(fv, 24, seed=31)) if which == 0 else ("ilu", convdiff_3d(fv, 8, seed=32))


@pytest.mark.parametrize("which", [0, 1])
def test_reordered_factors_levels_and_apply_bit_exact(fv, orc, which):
    kind, case = _case(fv, which)
    ptr, cols, vals, rhs = oracle_system(orc, case)
    A, b = _system(fv, case)
    d = case["mesh"].dim
    perm, info = fv.order_boxes(A)
    hp, hinfo = fv.order_boxes_host(case["mesh"].cell_center, ptr, cols, 0, np.zeros(d), np.ones(d))
    assert np.array_equal(perm, hp) and info == hinfo and info["n_colours"] == 2
    cls = fv.IncompleteCholesky if kind == "ic" else fv.IncompleteLowerUpper
    P = cls.from_matrix(A, 0, ordering="boxes")
    assert np.array_equal(P.perm, perm)
    o = orc.Precond.reordered(kind, ptr, cols, vals, perm)
    gp, gc, gv, gd = P.factors()
    op_, oc, ov, _, od = o.export()
    assert np.array_equal(gp, op_) and np.array_equal(gc, oc) and np.array_equal(gv, ov) and gd == od
    bp, bc, _ = orc.permute(ptr, cols, vals, perm)
    fl, bl, nf, nb = P.levels()
    of, onf = orc.levels(bp, bc)
    ob, onb = orc.levels(bp, bc, upper=True)
    assert np.array_equal(fl, of) and np.array_equal(bl, ob) and (nf, nb) == (onf, onb)
    assert nf == info["n_levels"]
    rng = np.random.default_rng(7)
    for grid, rpt in ((0, 0), (148, 1), (1184, 2), (37, 8), (0, 0)):  # repeated applies at several shapes
        P.set_grid(grid, rpt)
        r = rng.standard_normal(len(rhs))
        z = fv.DistributedVector.from_size(len(rhs))
        P.precondition(z, fv.DistributedVector(r))
        assert np.array_equal(z.numpy(), o.apply(r))


def test_reordered_apply_arbitrary_permutation(fv, orc):
    _, case = _case(fv, 1)
    ptr, cols, vals, _ = oracle_system(orc, case)
    A, _ = _system(fv, case)
    perm = np.random.default_rng(3).permutation(len(ptr) - 1).astype(np.int32)
    P = fv.IncompleteLowerUpper.from_matrix(A, 0, ordering=perm)
    o = orc.Precond.reordered("ilu", ptr, cols, vals, perm)
    r = np.random.default_rng(4).standard_normal(len(ptr) - 1)
    z = fv.DistributedVector.from_size(len(r))
    P.precondition(z, fv.DistributedVector(r))
    assert np.array_equal(z.numpy(), o.apply(r))


@pytest.mark.parametrize("which", [0, 1])
def test_reordered_solve_matches_oracle(fv, orc, which):
    kind, case = _case(fv, which)
    ptr, cols, vals, rhs = oracle_system(orc, case)
    A, b = _system(fv, case)
    cls = fv.IncompleteCholesky if kind == "ic" else fv.IncompleteLowerUpper
    P = cls.from_matrix(A, 0, ordering="boxes")
    o = orc.Precond.reordered(kind, ptr, cols, vals, P.perm)
    x = fv.DistributedVector.from_size(len(rhs))
    opts = fv.LinearSolverOptions(1e-8, 1e-8, 5000)
    if kind == "ic":
        info = fv.conjugate_gradient(x, A, b, P, None, opts)
        xo, io = orc.cg(ptr, cols, vals, o, rhs, rtol=1e-8, atol=1e-8, maxit=5000)
    else:
        info = fv.bi_conjugate_gradient_stab(x, A, b, P, None, opts)
        xo, io = orc.bicgstab(ptr, cols, vals, o, rhs, rtol=1e-8, atol=1e-8, maxit=5000)
    assert info.status == 0
    assert abs(info.iterations - io["iterations"]) <= 2
    assert np.linalg.norm(x.numpy() - xo) <= SOL_TOL * np.linalg.norm(xo)


def test_reordered_refactor_after_new_values(fv, orc):
    _, case = _case(fv, 1)
    A, _ = _system(fv, case)
    P = fv.IncompleteLowerUpper.from_matrix(A, 0, ordering="boxes")
    case2 = dict(case, kappa=case["kappa"] * 1.7, flux=case["flux"] * 0.6)
    fv.assemble(equation(fv, case2), (case2["bndi"], case2["bnde"]), case2["mesh"], lhs=A)
    P.refactor()
    ptr, cols, vals, _ = oracle_system(orc, case2)
    o = orc.Precond.reordered("ilu", ptr, cols, vals, P.perm)
    _, gc, gv, gd = P.factors()
    _, oc, ov, _, od = o.export()
    assert np.array_equal(gv, ov) and np.array_equal(gc, oc) and gd == od
    r = np.random.default_rng(9).standard_normal(len(ptr) - 1)
    z = fv.DistributedVector.from_size(len(r))
    P.precondition(z, fv.DistributedVector(r))
    assert np.array_equal(z.numpy(), o.apply(r))


def test_reordered_rejects_non_permutation(fv):
    _, case = _case(fv, 1)
    A, _ = _system(fv, case)
    n = A.nrows()
    bad = np.arange(n, dtype=np.int32)
    bad[3] = 5  # 5 twice, 3 missing
    with pytest.raises(fv.FvError):
        fv.IncompleteLowerUpper.from_matrix(A, 0, ordering=bad)
    with pytest.raises(fv.FvError):
        fv.IncompleteLowerUpper.from_matrix(A, 0, ordering=np.full(n, n, np.int32))
