"""Transient and extra terms, oracle side (CPU).

- time(Euler) with a zero-gradient boundary keeps a constant field constant
- time(Backward) with equal steps is BDF2: lhs 3/(2dt), rhs (2u1 - u0/2)/dt
- linear_source adds its coefficient to the diagonal; divergence(F) adds -F A
  to the owner's rhs and +F A to the neighbour's
- the term algebra keeps the new terms with their signs
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from cases import diffusion_2d


def test_euler_keeps_a_constant_field(fv, orc):
    case = diffusion_2d(fv, 12, seed=1)
    m = case["mesh"]
    nb = m.n_boundary_faces
    u0 = np.full(m.n_cells, 3.25)
    ptr, cols, vals, rhs = orc.assemble(m, -1.0, 0.0, 0.0, kappa=case["kappa"], bndi=np.ones(nb),
                                        bnde=np.zeros(nb), extra=dict(c_time=1.0, time_scheme="euler", dt=0.01,
                                                                      previous=u0))
    x = spla.spsolve(sp.csr_matrix((vals, cols, ptr)).tocsc(), rhs)
    assert np.abs(x - u0).max() < 1e-12


def test_backward_equal_steps_is_bdf2(fv, orc):
    m = fv.Mesh.square(4, 0.1, 2)
    nb = m.n_boundary_faces
    u1 = np.linspace(1.0, 2.0, m.n_cells)
    u0 = np.linspace(0.5, 0.7, m.n_cells)
    dt = 0.125
    ptr, cols, vals, rhs = orc.assemble(m, 0.0, 0.0, 0.0, bndi=np.zeros(nb), bnde=np.zeros(nb),
                                        extra=dict(c_time=1.0, time_scheme="backward", dt=dt, dt_2=dt,
                                                   previous=u1, previous_2=u0))
    A = sp.csr_matrix((vals, cols, ptr)).toarray()
    V = m.cell_volume
    assert np.allclose(np.diag(A), 1.5 / dt * V, rtol=1e-15)
    assert np.allclose(rhs, (2.0 * u1 - 0.5 * u0) / dt * V, rtol=1e-14)


def test_linear_source_and_divergence(fv, orc):
    m = fv.Mesh.square(5, 0.1, 3)
    nb = m.n_boundary_faces
    c = np.linspace(0.1, 0.9, m.n_cells)
    F = np.linspace(-1.0, 1.0, m.n_faces)
    ptr, cols, vals, rhs = orc.assemble(m, 0.0, 0.0, 0.0, bndi=np.zeros(nb), bnde=np.zeros(nb),
                                        extra=dict(c_lin=-1.0, lin=c, c_div=1.0, divflux=F))
    A = sp.csr_matrix((vals, cols, ptr)).toarray()
    assert np.allclose(np.diag(A), -c * m.cell_volume, rtol=1e-15)
    want = np.zeros(m.n_cells)
    for f in range(m.n_faces):
        want[m.face_owner[f]] += -F[f] * m.face_area[f]
        if m.face_neighbor[f] >= 0:
            want[m.face_neighbor[f]] -= -F[f] * m.face_area[f]
    assert np.allclose(rhs, want, rtol=1e-13, atol=1e-15)


def test_term_algebra_with_transient_terms(fv):
    k = np.ones(4)
    e = fv.time(fv.Euler(k, 0.1)) - fv.laplacian(fv.Orthogonal(), k) + fv.linear_source(k) - fv.divergence(k)
    assert e.coefficient("time") == 1.0 and e.coefficient("linear_source") == 1.0
    assert e.coefficient("divergence") == -1.0 and e.coefficients() == (-1.0, 0.0, 0.0)
    with pytest.raises(NotImplementedError):
        fv.time(object())
