"""IC(k) / ILU(k) with fill, oracle side (CPU).

- the oracle's level-k patterns equal a pure-Python restatement of the
  reference's depth-first walks (row_i_u_sparsity / row_i_l_sparsity /
  row_i_sparsity_edit), including the visiting order
- IC(1) has the pattern of A (the reference's walk adds nothing at level 1)
- IC(2): L L^T equals A on the factor pattern; ILU(1): L U equals A on the
  pattern up to the drop rule (|v| <= 1e-6 |u_ii| removed)
- level 1 fill lowers the BiCGStab iteration count of the 3D case
"""
import numpy as np
import pytest
import scipy.sparse as sp

from cases import convdiff_3d, diffusion_2d, oracle_system


def _walk(mode, i, level, ptr, cols):
    """Pure-Python restatement: mode 'u', 'l' (ILU) or 'ball' (IC)."""
    s, q, visited, length = set(), [i], {i: i}, {i: 0}
    while q:
        k = q.pop()
        lk = length[k]
        for t in range(ptr[k], ptr[k + 1]):
            j = int(cols[t])
            if j == k or visited.get(j) == i:
                continue
            visited[j] = i
            if mode == "ball":
                if lk < level:
                    q.append(j)
                    length[j] = lk + 1
                    s.add(j)
            elif mode == "u":
                if j < i and lk < level:
                    q.append(j)
                    length[j] = lk + 1
                elif j > i:
                    s.add(j)
            else:
                if j > i and lk < level:
                    q.append(j)
                    length[j] = lk + 1
                elif j < i:
                    s.add(j)
    return s


def _py_pattern(kind, level, ptr, cols):
    rows = []
    for i in range(len(ptr) - 1):
        if kind == "ilu":
            r = _walk("l", i, level, ptr, cols) | {i} | _walk("u", i, level, ptr, cols)
        else:
            r = _walk("ball", i, level, ptr, cols) | set(int(c) for c in cols[ptr[i]:ptr[i + 1]])
        rows.append(sorted(r))
    return rows


@pytest.mark.parametrize("kind,level", [("ilu", 1), ("ilu", 2), ("ilu", 3), ("ic", 2), ("ic", 3)])
def test_fill_pattern_equals_python_walks(fv, orc, kind, level):
    case = convdiff_3d(fv, 3, seed=1) if kind == "ilu" else diffusion_2d(fv, 6, seed=1)
    ptr, cols, vals, _ = oracle_system(orc, case)
    fptr, fcol, fill = orc.fill_pattern(kind, level, ptr, cols)
    want = _py_pattern(kind, level, ptr, cols)
    got = [list(fcol[fptr[i]:fptr[i + 1]]) for i in range(len(ptr) - 1)]
    assert got == want
    for i in range(len(ptr) - 1):
        a = set(cols[ptr[i]:ptr[i + 1]].tolist())
        assert [bool(f) for f in fill[fptr[i]:fptr[i + 1]]] == [c not in a for c in got[i]]
    assert fill.sum() > 0


def test_ic1_is_ic0(fv, orc):
    ptr, cols, vals, _ = oracle_system(orc, diffusion_2d(fv, 12, seed=2))
    fptr, fcol, fill = orc.fill_pattern("ic", 1, ptr, cols)
    assert np.array_equal(fptr, ptr) and np.array_equal(fcol, cols) and fill.sum() == 0
    r = np.random.default_rng(0).standard_normal(len(ptr) - 1)
    a = orc.Precond("ic", ptr, cols, vals, level=1).apply(r)
    b = orc.Precond("ic", ptr, cols, vals, level=0).apply(r)
    assert np.array_equal(a, b)


def test_ic2_factor_reproduces_a_on_its_pattern(fv, orc):
    ptr, cols, vals, _ = oracle_system(orc, diffusion_2d(fv, 10, seed=3))
    n = len(ptr) - 1
    pc = orc.Precond("ic", ptr, cols, vals, level=2)
    assert pc.ok()
    lp, lc, lv, inv, _ = pc.export()
    L = sp.csr_matrix((lv, lc, lp), shape=(n, n))
    fptr, fcol, _ = orc.fill_pattern("ic", 2, ptr, cols)
    A = sp.csr_matrix((vals, cols, ptr), shape=(n, n)).toarray()
    R = (L @ L.T).toarray() - A
    mask = sp.csr_matrix((np.ones(len(fcol)), fcol, fptr), shape=(n, n)).toarray() > 0
    assert np.abs(R[mask]).max() < 1e-12 * np.abs(A).max()


def test_ilu1_factor_and_iterations(fv, orc):
    case = convdiff_3d(fv, 6, seed=4)
    ptr, cols, vals, rhs = oracle_system(orc, case)
    n = len(ptr) - 1
    p1 = orc.Precond("ilu", ptr, cols, vals, level=1)
    lp, lc, lv, _, nd = p1.export()
    LU = sp.csr_matrix((lv, lc, lp), shape=(n, n)).toarray()
    L = np.tril(LU, -1) + np.eye(n)
    U = np.triu(LU)
    A = sp.csr_matrix((vals, cols, ptr), shape=(n, n)).toarray()
    stored = LU != 0
    R = (L @ U - A)[stored]
    assert np.abs(R).max() < 1e-5 * np.abs(A).max()
    _, i0 = orc.bicgstab(ptr, cols, vals, orc.Precond("ilu", ptr, cols, vals), rhs, rtol=1e-10, atol=1e-10,
                         maxit=2000)
    _, i1 = orc.bicgstab(ptr, cols, vals, p1, rhs, rtol=1e-10, atol=1e-10, maxit=2000)
    assert i1["iterations"] < i0["iterations"]


@pytest.mark.parametrize("kind,level", [("ilu", 1), ("ilu", 2), ("ic", 2), ("ic", 3)])
def test_library_fill_pattern_equals_oracle(fv, orc, kind, level):
    """The library's own walk (rows split over host threads, joined in row
    order) gives the oracle's arrays; amap places every entry of A."""
    case = convdiff_3d(fv, 12, seed=7) if kind == "ilu" else diffusion_2d(fv, 40, seed=7)
    ptr, cols, vals, _ = oracle_system(orc, case)
    fptr, fcol, fill = orc.fill_pattern(kind, level, ptr, cols)
    cls = fv.IncompleteLowerUpper if kind == "ilu" else fv.IncompleteCholesky
    got = cls.fill_pattern(ptr, cols, level)
    assert np.array_equal(got[0], fptr) and np.array_equal(got[1], fcol)
    if kind == "ic":
        assert np.array_equal(got[3], fill)
    amap = got[2]
    rows = np.repeat(np.arange(len(ptr) - 1), np.diff(ptr))
    assert np.array_equal(fcol[amap], cols)
    assert (amap >= fptr[rows]).all() and (amap < fptr[rows + 1]).all()


def test_library_fill_pattern_rejects_bad_patterns(fv):
    from fvb200._lib import FvError
    ptr = np.array([0, 2, 4], np.int32)
    with pytest.raises(FvError):
        fv.IncompleteLowerUpper.fill_pattern(ptr, np.array([1, 0, 0, 1], np.int32), 1)  # unsorted row
    with pytest.raises(FvError):
        fv.IncompleteLowerUpper.fill_pattern(ptr, np.array([0, 2, 0, 1], np.int32), 1)  # column out of range
    empty = fv.IncompleteLowerUpper.fill_pattern(np.zeros(1, np.int32), np.zeros(0, np.int32), 1)
    assert len(empty[0]) == 1 and len(empty[1]) == 0
