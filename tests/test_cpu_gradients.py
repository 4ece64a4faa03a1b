"""Gradients and the Corrected scheme, oracle side (CPU).

- the C oracle's gradient coefficients equal an independent pure-Python
  restatement of Mesh::compute + Matrix::inv bit for bit
- least-squares gradients reproduce a linear field exactly (to rounding)
- on a uniform quad mesh (orthogonal: n parallel to d, |n| = 1) Corrected
  equals Orthogonal and its explicit correction vanishes
"""
import numpy as np
import pytest

from cases import diffusion_2d


def _linear(mesh, a, b0):
    u = mesh.cell_center @ a + b0
    fb0 = mesh.n_faces - mesh.n_boundary_faces
    ub = mesh.face_center[fb0:] @ a + b0
    return u, np.zeros(mesh.n_boundary_faces), ub


@pytest.mark.parametrize("dim", [2, 3])
def test_oracle_grad_coeffs_equal_python_restatement(fv, orc, dim):
    from oracle import mesh_ref
    m = fv.Mesh.square(5, 0.2, 3) if dim == 2 else fv.Mesh.cube(2, 0.15, 3)
    gc, gd = orc.grad_coeffs(m)
    pc, pd = mesh_ref.grad_coeffs(dim, m.cell_face_ptr.tolist(), m.cell_faces.tolist(), m.face_owner.tolist(),
                                  m.face_neighbor.tolist(), m.face_center.tolist(), m.cell_center.tolist())
    assert np.array_equal(gc, np.array(pc))
    assert np.array_equal(gd, np.array(pd))


@pytest.mark.parametrize("dim", [2, 3])
def test_oracle_gradient_of_linear_field_is_exact(fv, orc, dim):
    m = fv.Mesh.square(12, 0.2, 5) if dim == 2 else fv.Mesh.cube(4, 0.15, 5)
    a = np.array([0.7, -1.3, 0.4][:dim])
    u, bi, be = _linear(m, a, 2.5)
    g = orc.gradients(m, u, bi, be)
    assert np.abs(g - a).max() < 1e-10


def test_corrected_equals_orthogonal_on_uniform_quads(fv, orc):
    n = 6
    nodes = np.array([[i / n, j / n] for j in range(n + 1) for i in range(n + 1)])
    quads = [[j * (n + 1) + i, j * (n + 1) + i + 1, (j + 1) * (n + 1) + i + 1, (j + 1) * (n + 1) + i]
             for j in range(n) for i in range(n)]
    kinds = np.full(len(quads), 9, np.int32)
    eptr = np.arange(0, 4 * len(quads) + 1, 4, dtype=np.int32)
    cnt = {}
    for q in quads:
        for e in range(4):
            key = tuple(sorted((q[e], q[(e + 1) % 4])))
            cnt[key] = cnt.get(key, 0) + 1
    bnd = [k for k, v in cnt.items() if v == 1]
    m = fv.Mesh.from_elements(2, nodes, kinds, eptr, np.array(quads, np.int32).ravel(),
                              np.arange(0, 2 * len(bnd) + 1, 2, dtype=np.int32), np.array(bnd, np.int32).ravel(),
                              np.zeros(len(bnd), np.int32))
    nb = m.n_boundary_faces
    kf = np.linspace(1.0, 2.0, m.n_faces)
    u = np.sin(m.cell_center[:, 0] * 3.0) + m.cell_center[:, 1]
    g = orc.gradients(m, u, np.zeros(nb), np.zeros(nb))
    o = orc.assemble(m, -1.0, 0.0, -1.0, kappa=kf, source=np.ones(m.n_cells), bndi=np.zeros(nb), bnde=np.zeros(nb))
    c = orc.assemble(m, -1.0, 0.0, -1.0, kappa=kf, source=np.ones(m.n_cells), bndi=np.zeros(nb), bnde=np.zeros(nb),
                     corrected=(g, 1.0))
    assert np.array_equal(o[0], c[0]) and np.array_equal(o[1], c[1])
    assert np.allclose(o[2], c[2], rtol=1e-13, atol=1e-13 * np.abs(o[2]).max())
    assert np.allclose(o[3], c[3], rtol=1e-13, atol=1e-13 * np.abs(o[3]).max())


def test_corrected_changes_a_distorted_mesh(fv, orc):
    case = diffusion_2d(fv, 10, seed=2)
    m = case["mesh"]
    nb = m.n_boundary_faces
    u = m.cell_center[:, 0] ** 2
    g = orc.gradients(m, u, np.zeros(nb), np.zeros(nb))
    o = orc.assemble(m, -1.0, 0.0, -1.0, kappa=case["kappa"], source=case["source"], bndi=np.zeros(nb),
                     bnde=np.zeros(nb))
    c = orc.assemble(m, -1.0, 0.0, -1.0, kappa=case["kappa"], source=case["source"], bndi=np.zeros(nb),
                     bnde=np.zeros(nb), corrected=(g, 1.0))
    c0 = orc.assemble(m, -1.0, 0.0, -1.0, kappa=case["kappa"], source=case["source"], bndi=np.zeros(nb),
                      bnde=np.zeros(nb), corrected=(g, 0.0))
    assert not np.allclose(o[2], c[2])                 # 1/(n.d) differs from 1/|d|
    assert np.array_equal(c[2], c0[2])                 # the reduction only scales the rhs
    assert not np.array_equal(c[3], c0[3])
