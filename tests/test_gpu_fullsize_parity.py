"""GPU against the oracle at the benchmark sizes.

Config "square256": unit square, 256 x 256 squares x 2 triangles (131,072
cells), jitter 0.2h, lognormal(0, 1) diffusivity, f = 1, u = 0 on the
boundary, CG + IC(0) at rtol = atol = 1e-8 (seed 1000, the benchmark's).
Config "cube128": unit cube, 128^3 hexes x 6 tetrahedra (12,582,912 cells),
jitter 0.15h, lognormal(0, 0.5) diffusivity, upwind convection with
v = (1, 0.5, 0.25), f ~ U(0, 1), BiCGStab + ILU(0) at rtol = atol = 1e-8.

For each, in the reference's natural order and in the box-colour order of
the perf mode (the oracle factorising the same permuted matrix):

- the mesh: the device build equals the oracle's own generator, bit for bit
- pattern, assembled coefficients and right-hand side: bit for bit
- factors, dropped-entry count and level schedules: bit for bit
- one preconditioner apply: bit for bit
- CG at rtol = atol = 1e-8: solution within 1e-10 (relative L2) of the
  oracle's, iterations within +-2, true residual below the tolerance
- BiCGStab: the iterate after 10 iterations (tolerance 0) within 1e-10 of
  the oracle's; at rtol = atol = 1e-8 the true residual below the tolerance

Why BiCGStab is held to less at this size: the reference restarts whenever
|rho| <= 1e-15 |b| (bi_conjugate_gradient_stab.rs:155-169), and here |b| is
about 5e-5, so restarts fire all through the solve (39-44 of them) at
moments set by the last bits of the dot products.  The GPU's and the
oracle's residual histories (the same factors, bit for bit; dot products
summed in different orders) agree to 1e-14 at first, drift past 1e-6 by
iteration ~20 and are unrelated by iteration ~100; perturbing the right-hand
side by 1e-15 moves the oracle's own count on the 64^3 cube from 87 to 123.
The stopping iteration of this solver is not a reproducible quantity, so it
is only bounded (at most 1.5x the oracle's + 2), and the strict comparison
is made where the two runs are still in step.

The oracle's solves run on host threads side by side (ctypes releases the
GIL); the config-1 ones take two to three minutes each.
"""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SOL_TOL = 1e-10  # relative L2 bound on solutions (the FP64 parity bar)
RTOL = 1e-8
SEED = 1000
V = (1.0, 0.5, 0.25)
# iterations of the fixed-count comparison (see the module docstring for BiCGStab's 10)
FIXED_ITERATIONS = {"cube128": 10}
MESH_ARRAYS = ("cell_face_ptr", "cell_faces", "face_owner", "face_neighbor", "face_area", "face_normal",
               "face_center", "cell_center", "cell_volume")


def _build(fv, kind):
    from oracle import gen
    if kind == "square256":
        m = fv.Mesh.square(256, 0.2, SEED, on_device=True)
        om = gen.Mesh.square(256, 0.2, SEED)
        kf, _, sc = m.fields(SEED, 1.0, 1.0, source_const=1.0)
        fl = None
        coef = (-1.0, 0.0, -1.0)
        eq = -fv.laplacian(fv.Orthogonal(), kf) - fv.source(sc)
    else:
        m = fv.Mesh.cube(128, 0.15, SEED, on_device=True)
        om = gen.Mesh.cube(128, 0.15, SEED)
        kf, fl, sc = m.fields(SEED, float(np.linalg.norm(V)) / 128 / 3.0, 0.5, velocity=V, source_uniform=True)
        coef = (-1.0, 1.0, -1.0)
        eq = fv.convection(fv.Upwind(fl), fl) - fv.laplacian(fv.Orthogonal(), kf) - fv.source(sc)
    nb = m.n_boundary_faces
    bc = (np.zeros(nb), np.zeros(nb))
    return m, om, eq, bc, dict(kappa=kf, flux=fl, source=sc, bndi=bc[0], bnde=bc[1]), coef


@pytest.fixture(scope="module", params=["square256", "cube128"])
def problem(request, fv, orc):
    kind = request.param
    m, om, eq, bc, fields, coef = _build(fv, kind)
    A, b = fv.assemble(eq, bc, m)
    ptr, cols, vals, rhs = orc.assemble(om, coef[0], coef[1], coef[2], **fields)
    yield dict(kind=kind, m=m, om=om, A=A, b=b, sys=(ptr, cols, vals, rhs))


def test_mesh_and_system_bit_exact(problem):
    m, om = problem["m"], problem["om"]
    assert (m.n_cells, m.n_faces, m.n_boundary_faces) == (om.n_cells, om.n_faces, om.n_boundary_faces)
    for name in MESH_ARRAYS:
        a, o = getattr(m, name), getattr(om, name)
        assert a.shape == o.shape and a.tobytes() == o.tobytes(), name
    ptr, cols, vals, rhs = problem["sys"]
    gp, gc, gv = problem["A"].to_csr()
    assert np.array_equal(gp, ptr) and np.array_equal(gc, cols)
    assert gv.tobytes() == vals.tobytes()
    assert problem["b"].numpy().tobytes() == rhs.tobytes()


def _factor_checks(fv, orc, problem, ordering):
    ptr, cols, vals, rhs = problem["sys"]
    pk = "ic" if problem["kind"] == "square256" else "ilu"
    cls = fv.IncompleteCholesky if pk == "ic" else fv.IncompleteLowerUpper
    P = cls.from_matrix(problem["A"], 0, ordering=ordering)
    if ordering is None:
        o = orc.Precond(pk, ptr, cols, vals)
        lp, lc = ptr, cols
    else:
        o = orc.Precond.reordered(pk, ptr, cols, vals, P.perm)
        lp, lc, _ = orc.permute(ptr, cols, vals, P.perm)
    gp, gc, gv, gd = P.factors()
    op_, oc, ov, _, od = o.export()
    assert np.array_equal(gp, op_) and np.array_equal(gc, oc) and gd == od
    assert gv.tobytes() == ov.tobytes()
    fl, bl, nf, nb = P.levels()
    of, onf = orc.levels(lp, lc)
    ob, onb = orc.levels(lp, lc, upper=True)
    assert (nf, nb) == (onf, onb)
    assert np.array_equal(fl, of) and np.array_equal(bl, ob)
    z = fv.DistributedVector.from_size(len(rhs))
    P.precondition(z, fv.DistributedVector(rhs))
    assert z.numpy().tobytes() == o.apply(rhs).tobytes()
    return P, o


def test_factors_levels_apply_and_solves(fv, orc, problem):
    """Both orderings: factors, levels and an apply bit for bit, then the GPU
    solves against the oracle's (run concurrently on the host): at rtol 1e-8,
    and for a fixed number of iterations."""
    ptr, cols, vals, rhs = problem["sys"]
    A, b = problem["A"], problem["b"]
    cg = problem["kind"] == "square256"
    solve = fv.conjugate_gradient if cg else fv.bi_conjugate_gradient_stab
    osolve = orc.cg if cg else orc.bicgstab
    runs = {"rtol": (RTOL, 10000)}
    if not cg:
        runs["fixed"] = (0.0, FIXED_ITERATIONS[problem["kind"]])
    pairs = {o: _factor_checks(fv, orc, problem, o) for o in (None, "boxes")}
    pk = "ic" if cg else "ilu"

    def oracle_precond(o, P, first):
        # a solve of its own for every concurrent oracle run: the reordered
        # wrapper's work vectors belong to one object and one thread
        if first:
            return pairs[o][1]
        return orc.Precond(pk, ptr, cols, vals) if o is None else orc.Precond.reordered(pk, ptr, cols, vals, P.perm)

    with ThreadPoolExecutor(max_workers=4) as ex:
        futs = {(o, k): ex.submit(osolve, ptr, cols, vals, oracle_precond(o, P, j == 0), rhs, rtol=tol, atol=tol,
                                  maxit=it)
                for o, (P, _) in pairs.items() for j, (k, (tol, it)) in enumerate(runs.items())}
        gpu = {}
        for o, (P, _) in pairs.items():
            for k, (tol, it) in runs.items():
                x = fv.DistributedVector.from_size(len(rhs))
                info = solve(x, A, b, P, None, fv.LinearSolverOptions(tol, tol, it))
                r = fv.DistributedVector.from_size(len(rhs))
                A.imul(r, x)
                relres = float(np.linalg.norm(r.numpy() - rhs) / np.linalg.norm(rhs))
                gpu[(o, k)] = (x.numpy(), info, relres)
        for (o, k), f in futs.items():
            xo, io = f.result()
            xg, info, relres = gpu[(o, k)]
            assert info.status == 0
            if k == "rtol":
                if cg:
                    assert abs(info.iterations - io["iterations"]) <= 2, (o, info.iterations, io["iterations"])
                    assert np.linalg.norm(xg - xo) <= SOL_TOL * np.linalg.norm(xo), (o, k)
                else:
                    assert info.iterations <= 1.5 * io["iterations"] + 2, (o, info.iterations, io["iterations"])
                assert relres <= RTOL, (o, relres)
            else:
                assert info.iterations == io["iterations"]
                assert np.linalg.norm(xg - xo) <= SOL_TOL * np.linalg.norm(xo), (o, k)
