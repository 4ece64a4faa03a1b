"""Transient and extra terms on the GPU, against the oracle.

- assembly with time(Euler / Backward, with densities), linear_source and
  divergence: coefficients and rhs bit-exact
- a time loop (implicit Euler heat equation, 5 steps): value-only
  re-assembly into the resident pattern, IC(0) refactorisation, CG; every
  step's solution within 1e-10 of the oracle's loop
"""
import numpy as np
import pytest

from cases import convdiff_3d, diffusion_2d

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("variant", ["euler", "euler_density", "backward", "backward_density"])
def test_transient_assembly_equals_oracle(fv, orc, variant):
    case = convdiff_3d(fv, 5, seed=13)
    m = case["mesh"]
    n = m.n_cells
    rng = np.random.default_rng(5)
    u1, u0 = rng.standard_normal(n), rng.standard_normal(n)
    dens = (rng.uniform(1, 2, n), rng.uniform(1, 2, n), rng.uniform(1, 2, n))
    lin = rng.uniform(-1, 0, n)
    divf = rng.standard_normal(m.n_faces)
    if variant.startswith("euler"):
        sch = fv.Euler(u1, 0.05, *(dens[:2] if variant.endswith("density") else (None, None)))
        ex = dict(time_scheme="euler", dt=0.05, previous=u1,
                  densities=dens[:2] if variant.endswith("density") else None)
    else:
        sch = fv.Backward(u1, u0, 0.05, 0.07, dens if variant.endswith("density") else None)
        ex = dict(time_scheme="backward", dt=0.05, dt_2=0.07, previous=u1, previous_2=u0,
                  densities=dens if variant.endswith("density") else None)
    eq = (fv.time(sch) + fv.convection(fv.Upwind(case["flux"]), case["flux"])
          - fv.laplacian(fv.Orthogonal(), case["kappa"]) - fv.source(case["source"])
          - fv.linear_source(lin) + fv.divergence(divf))
    A, b = fv.assemble(eq, (case["bndi"], case["bnde"]), m)
    gp, gc, gv = A.to_csr()
    ptr, cols, vals, rhs = orc.assemble(m, -1.0, 1.0, -1.0, kappa=case["kappa"], flux=case["flux"],
                                        source=case["source"], bndi=case["bndi"], bnde=case["bnde"],
                                        extra=dict(ex, c_time=1.0, c_lin=-1.0, lin=lin, c_div=1.0, divflux=divf))
    assert np.array_equal(gp, ptr) and np.array_equal(gc, cols)
    assert np.array_equal(gv, vals)
    assert np.array_equal(b.numpy(), rhs)


def test_heat_equation_time_loop(fv, orc):
    case = diffusion_2d(fv, 24, seed=14)
    m = case["mesh"]
    nb = m.n_boundary_faces
    dt = 1e-3
    u = np.exp(-((m.cell_center[:, 0] - 0.5) ** 2 + (m.cell_center[:, 1] - 0.5) ** 2) / 0.02)
    uo = u.copy()
    A = P = None
    opts = fv.LinearSolverOptions(1e-12, 1e-12, 2000)
    for _ in range(5):
        eq = fv.time(fv.Euler(u, dt)) - fv.laplacian(fv.Orthogonal(), case["kappa"])
        if A is None:
            A, b = fv.assemble(eq, (np.zeros(nb), np.zeros(nb)), m)
            P = fv.IncompleteCholesky.from_matrix(A, 0)
        else:
            _, b = fv.assemble(eq, (np.zeros(nb), np.zeros(nb)), m, lhs=A)
            P.refactor()
        x = fv.DistributedVector(u)
        fv.conjugate_gradient(x, A, b, P, None, opts)
        u = x.numpy()
        ptr, cols, vals, rhs = orc.assemble(m, -1.0, 0.0, 0.0, kappa=case["kappa"], bndi=np.zeros(nb),
                                            bnde=np.zeros(nb),
                                            extra=dict(c_time=1.0, time_scheme="euler", dt=dt, previous=uo))
        xo, _ = orc.cg(ptr, cols, vals, orc.Precond("ic", ptr, cols, vals), rhs, rtol=1e-12, atol=1e-12,
                       maxit=2000, x0=uo)
        uo = xo
        assert np.linalg.norm(u - uo) <= 1e-10 * np.linalg.norm(uo)
