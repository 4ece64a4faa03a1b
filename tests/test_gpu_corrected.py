"""Gradients and the Corrected scheme on the GPU, against the oracle.

- fv_compute_gradients equals the oracle's compute_gradients bit for bit
  (coefficients of Mesh::compute built at mesh upload)
- assembly with laplacian(Corrected(grad, r), kappa): pattern, coefficients
  and rhs bit-exact, for r = 1 and r = 0.5, 2D diffusion and 3D
  convection-diffusion
- a CG + IC(0) solve of the corrected system matches the oracle (<=1e-10,
  iterations +-2)
"""
import numpy as np
import pytest

from cases import convdiff_3d, diffusion_2d

pytestmark = pytest.mark.gpu


def _grad(fv, m, u, bi, be):
    g = fv.DistributedVector.from_size(m.n_cells * m.dim)
    fv.compute_gradients(g, u, (bi, be), m)
    return g


@pytest.mark.parametrize("kind", ["2d", "3d"])
def test_gradients_equal_oracle(fv, orc, kind):
    case = diffusion_2d(fv, 20, seed=7) if kind == "2d" else convdiff_3d(fv, 6, seed=7)
    m = case["mesh"]
    nb = m.n_boundary_faces
    rng = np.random.default_rng(3)
    u = rng.standard_normal(m.n_cells)
    bi, be = rng.uniform(0, 1, nb), rng.standard_normal(nb)
    g = _grad(fv, m, u, bi, be).numpy().reshape(m.n_cells, m.dim)
    assert np.array_equal(g, orc.gradients(m, u, bi, be))


@pytest.mark.parametrize("kind,red", [("2d", 1.0), ("2d", 0.5), ("3d", 1.0)])
def test_corrected_assembly_equals_oracle(fv, orc, kind, red):
    case = diffusion_2d(fv, 20, seed=8) if kind == "2d" else convdiff_3d(fv, 6, seed=8)
    m = case["mesh"]
    nb = m.n_boundary_faces
    u = np.cos(3.0 * m.cell_center[:, 0]) + m.cell_center[:, 1] ** 2
    g = _grad(fv, m, u, case["bndi"], case["bnde"])
    lap = fv.laplacian(fv.Corrected(g, red), case["kappa"])
    src = fv.source(case["source"])
    if case["c_conv"] != 0.0:
        eq = fv.convection(fv.Upwind(case["flux"]), case["flux"]) - lap - src
    else:
        eq = -lap - src
    A, b = fv.assemble(eq, (case["bndi"], case["bnde"]), m)
    gp, gc, gv = A.to_csr()
    ptr, cols, vals, rhs = orc.assemble(m, case["c_lap"], case["c_conv"], case["c_src"], kappa=case["kappa"],
                                        flux=case["flux"], source=case["source"], bndi=case["bndi"],
                                        bnde=case["bnde"], corrected=(g.numpy().reshape(m.n_cells, m.dim), red))
    assert np.array_equal(gp, ptr) and np.array_equal(gc, cols)
    assert np.array_equal(gv, vals)
    assert np.array_equal(b.numpy(), rhs)


def test_corrected_solve_matches_oracle(fv, orc):
    case = diffusion_2d(fv, 32, seed=9)
    m = case["mesh"]
    u = np.zeros(m.n_cells)
    g = _grad(fv, m, u + m.cell_center[:, 0], case["bndi"], case["bnde"])
    eq = -fv.laplacian(fv.Corrected(g, 1.0), case["kappa"]) - fv.source(case["source"])
    A, b = fv.assemble(eq, (case["bndi"], case["bnde"]), m)
    P = fv.IncompleteCholesky.from_matrix(A, 0)
    x = fv.DistributedVector.from_size(m.n_cells)
    info = fv.conjugate_gradient(x, A, b, P, None, fv.LinearSolverOptions(1e-12, 1e-12, 3000))
    ptr, cols, vals, rhs = orc.assemble(m, -1.0, 0.0, -1.0, kappa=case["kappa"], source=case["source"],
                                        bndi=case["bndi"], bnde=case["bnde"],
                                        corrected=(g.numpy().reshape(m.n_cells, m.dim), 1.0))
    xo, io = orc.cg(ptr, cols, vals, orc.Precond("ic", ptr, cols, vals), rhs, rtol=1e-12, atol=1e-12, maxit=3000)
    assert abs(info.iterations - io["iterations"]) <= 2
    assert np.linalg.norm(x.numpy() - xo) <= 1e-10 * np.linalg.norm(xo)
