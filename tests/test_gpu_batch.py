"""Batched solves (block-diagonal union of independent meshes) on the GPU.

- the union's assembly and IC(0) are the per-problem ones, bit for bit
- FP64 batched CG matches the oracle per problem (<=1e-10, iterations +-2)
- each problem's result is identical alone and in a mix (per-problem reductions)
- mixed precision (FP32 CG inside FP64 refinement) reaches the FP64 tolerance and
  an error <= 1e-8 against a tight FP64 oracle solve
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problems(fv, sides, seed0=100):
    out = []
    for k, s in enumerate(sides):
        m = fv.Mesh.square(s, 0.2, seed0 + k)
        sigma = 0.5 + 1.5 * ((k * 0.37) % 1.0)
        kf, _, sc = m.fields(seed0 + k, 1.0, sigma, source_const=1.0)
        out.append((m, kf, sc))
    return out


def _union_system(fv, probs):
    from fvb200.batch import MeshBatch
    mb = MeshBatch([p[0] for p in probs])
    kf = mb.face_field([p[1] for p in probs])
    sc = mb.cell_field([p[2] for p in probs])
    nb = mb.n_boundary_faces
    eq = -fv.laplacian(fv.Orthogonal(), kf) - fv.source(sc)
    A, b = fv.assemble(eq, (np.zeros(nb), np.zeros(nb)), mb)
    return mb, A, b


def test_union_assembly_and_ic0_are_per_problem(fv, orc):
    probs = _problems(fv, [6, 9, 4])
    mb, A, b = _union_system(fv, probs)
    gp, gc, gv = A.to_csr()
    P = fv.IncompleteCholesky.from_matrix(A, 0)
    fp, fc, fvv, _ = P.factors()
    bb = b.numpy()
    for k, (m, kf, sc) in enumerate(probs):
        r0, r1 = mb.cell_offsets[k], mb.cell_offsets[k + 1]
        nb = m.n_boundary_faces
        ptr, cols, vals, rhs = orc.assemble(m, -1.0, 0.0, -1.0, kappa=kf, source=sc, bndi=np.zeros(nb),
                                            bnde=np.zeros(nb))
        a0, a1 = gp[r0], gp[r1]
        assert np.array_equal(gp[r0:r1 + 1] - a0, ptr)
        assert np.array_equal(gc[a0:a1] - r0, cols)
        assert np.array_equal(gv[a0:a1], vals)
        assert np.array_equal(bb[r0:r1], rhs)
        op, oc, ov, _, _ = orc.Precond("ic", ptr, cols, vals).export()
        f0, f1 = fp[r0], fp[r1]
        assert np.array_equal(fc[f0:f1] - r0, oc) and np.array_equal(fvv[f0:f1], ov)


def test_batch_fp64_matches_oracle(fv, orc):
    from fvb200.batch import BatchCG
    probs = _problems(fv, [12, 20, 7, 16])
    mb, A, b = _union_system(fv, probs)
    P = fv.IncompleteCholesky.from_matrix(A, 0)
    x = fv.DistributedVector.from_size(mb.n_cells)
    bc = BatchCG(A, mb.cell_offsets, 256)
    out = bc.solve(P, b, x, precision="fp64", relative_tolerance=1e-12, absolute_tolerance=1e-12, max_iterations=3000)
    xs = x.numpy()
    for k, (m, kf, sc) in enumerate(probs):
        nb = m.n_boundary_faces
        ptr, cols, vals, rhs = orc.assemble(m, -1.0, 0.0, -1.0, kappa=kf, source=sc, bndi=np.zeros(nb),
                                            bnde=np.zeros(nb))
        xo, io = orc.cg(ptr, cols, vals, orc.Precond("ic", ptr, cols, vals), rhs, rtol=1e-12, atol=1e-12, maxit=3000)
        r0, r1 = mb.cell_offsets[k], mb.cell_offsets[k + 1]
        assert abs(int(out["iterations"][k]) - io["iterations"]) <= 2
        assert np.linalg.norm(xs[r0:r1] - xo) <= 1e-10 * np.linalg.norm(xo)
        assert out["status"][k] == 0


def test_batch_result_same_alone_and_in_mix(fv):
    from fvb200.batch import BatchCG
    probs = _problems(fv, [10, 15, 6, 13, 8], seed0=300)
    target = 3
    results = {}
    for name, subset in (("alone", [target]), ("mix", list(range(len(probs))))):
        sel = [probs[i] for i in subset]
        mb, A, b = _union_system(fv, sel)
        P = fv.IncompleteCholesky.from_matrix(A, 0)
        for precision in ("fp64", "mixed"):
            x = fv.DistributedVector.from_size(mb.n_cells)
            out = BatchCG(A, mb.cell_offsets, 512).solve(P, b, x, precision=precision, relative_tolerance=1e-8,
                                                        absolute_tolerance=1e-8, outer_tolerance=1e-10)
            k = subset.index(target)
            r0, r1 = mb.cell_offsets[k], mb.cell_offsets[k + 1]
            results[(name, precision)] = (x.numpy()[r0:r1].copy(), int(out["iterations"][k]))
    for precision in ("fp64", "mixed"):
        xa, ia = results[("alone", precision)]
        xm, im = results[("mix", precision)]
        assert ia == im
        assert np.array_equal(xa, xm)


def test_batch_mixed_precision_accuracy(fv, orc):
    from fvb200.batch import BatchCG
    probs = _problems(fv, [24, 32, 18], seed0=500)
    mb, A, b = _union_system(fv, probs)
    P = fv.IncompleteCholesky.from_matrix(A, 0)
    x = fv.DistributedVector.from_size(mb.n_cells)
    out = BatchCG(A, mb.cell_offsets, 1024).solve(P, b, x, precision="mixed", outer_tolerance=1e-10,
                                                  inner_relative_tolerance=1e-4, max_outer=30)
    xs = x.numpy()
    for k, (m, kf, sc) in enumerate(probs):
        nb = m.n_boundary_faces
        ptr, cols, vals, rhs = orc.assemble(m, -1.0, 0.0, -1.0, kappa=kf, source=sc, bndi=np.zeros(nb),
                                            bnde=np.zeros(nb))
        xo, _ = orc.cg(ptr, cols, vals, orc.Precond("ic", ptr, cols, vals), rhs, rtol=1e-13, atol=1e-13, maxit=5000)
        r0, r1 = mb.cell_offsets[k], mb.cell_offsets[k + 1]
        assert out["final_residual"][k] <= 1e-10
        assert out["outer_steps"][k] >= 1 or out["fp64_fallback"][k] == 1
        assert np.linalg.norm(xs[r0:r1] - xo) <= 1e-8 * np.linalg.norm(xo)
        # the true FP64 residual of the returned solution
        import scipy.sparse as sp
        Ak = sp.csr_matrix((vals, cols, ptr))
        assert np.linalg.norm(rhs - Ak @ xs[r0:r1]) <= 1.0001e-10 * np.linalg.norm(rhs)


def _cube_problems(fv, sides, seed0=700):
    out = []
    for k, n in enumerate(sides):
        m = fv.Mesh.cube(n, 0.15, seed0 + k)
        kappa0 = float(np.linalg.norm((1.0, 0.5, 0.25))) / n / 3.0
        kf, fl, sc = m.fields(seed0 + k, kappa0, 0.5, velocity=(1.0, 0.5, 0.25), source_uniform=True)
        out.append((m, kf, fl, sc))
    return out


def test_batch_bicgstab_fp64_and_mixed(fv, orc):
    """Convection-diffusion problems, BiCGStab + ILU(0): FP64 batched matches the
    oracle per problem; mixed precision (FP32 BiCGStab + FP32 ILU(0) inside FP64
    refinement) reaches |b-Ax|/|b| <= 1e-10 and error <= 1e-8."""
    from fvb200.batch import BatchCG, MeshBatch
    probs = _cube_problems(fv, [5, 7, 4])
    mb = MeshBatch([p[0] for p in probs])
    kf = mb.face_field([p[1] for p in probs])
    fl = mb.face_field([p[2] for p in probs])
    sc = mb.cell_field([p[3] for p in probs])
    nb = mb.n_boundary_faces
    eq = fv.convection(fv.Upwind(fl), fl) - fv.laplacian(fv.Orthogonal(), kf) - fv.source(sc)
    A, b = fv.assemble(eq, (np.zeros(nb), np.zeros(nb)), mb)
    P = fv.IncompleteLowerUpper.from_matrix(A, 0)
    bc = BatchCG(A, mb.cell_offsets, 256)
    x64 = fv.DistributedVector.from_size(mb.n_cells)
    o64 = bc.solve(P, b, x64, precision="fp64", relative_tolerance=1e-12, absolute_tolerance=1e-12,
                   max_iterations=2000, solver="bicgstab")
    xm = fv.DistributedVector.from_size(mb.n_cells)
    om = bc.solve(P, b, xm, precision="mixed", outer_tolerance=1e-10, inner_relative_tolerance=1e-4,
                  max_iterations=2000, solver="bicgstab")
    a64, am = x64.numpy(), xm.numpy()
    for k, (m, kfk, flk, sck) in enumerate(probs):
        nbk = m.n_boundary_faces
        ptr, cols, vals, rhs = orc.assemble(m, -1.0, 1.0, -1.0, kappa=kfk, flux=flk, source=sck, bndi=np.zeros(nbk),
                                            bnde=np.zeros(nbk))
        o = orc.Precond("ilu", ptr, cols, vals)
        xo, io = orc.bicgstab(ptr, cols, vals, o, rhs, rtol=1e-12, atol=1e-12, maxit=2000)
        r0, r1 = mb.cell_offsets[k], mb.cell_offsets[k + 1]
        assert abs(int(o64["iterations"][k]) - io["iterations"]) <= 2
        assert np.linalg.norm(a64[r0:r1] - xo) <= 1e-10 * np.linalg.norm(xo)
        assert om["final_residual"][k] <= 1e-10
        assert np.linalg.norm(am[r0:r1] - xo) <= 1e-8 * np.linalg.norm(xo)


def test_union_of_resident_meshes_equals_host_union(fv):
    """Parts already on the GPU are joined there (fv_mesh_concat): the same system as the host-built union."""
    sides = [6, 9, 4, 13]
    host = _problems(fv, sides, seed0=300)
    dev = []
    for k, s in enumerate(sides):
        m = fv.Mesh.square(s, 0.2, 300 + k, on_device=True)
        dev.append((m, host[k][1], host[k][2]))
    mbh, Ah, bh = _union_system(fv, host)
    mbd, Ad, bd = _union_system(fv, dev)
    for x, y in zip(Ah.to_csr(), Ad.to_csr()):
        assert np.array_equal(x, y)
    assert np.array_equal(bh.numpy(), bd.numpy())
    Ph = fv.IncompleteCholesky.from_matrix(Ah, 0)
    Pd = fv.IncompleteCholesky.from_matrix(Ad, 0)
    for x, y in zip(Ph.factors()[:3], Pd.factors()[:3]):
        assert np.array_equal(x, y)
    # a 3D union mixing device-built and uploaded parts
    cubes = [fv.Mesh.cube(3, 0.1, 5, on_device=True), fv.Mesh.cube(4, 0.1, 6)]
    cubes[1].device()
    from fvb200.batch import MeshBatch
    mb = MeshBatch(cubes)
    flux = mb.face_field([np.linspace(-1, 1, m.n_faces) for m in cubes])
    kap = mb.face_field([np.full(m.n_faces, 0.3) for m in cubes])
    nb = mb.n_boundary_faces
    eq = fv.convection(fv.Upwind(flux), flux) - fv.laplacian(fv.Orthogonal(), kap)
    A1, b1 = fv.assemble(eq, (np.zeros(nb), np.ones(nb)), mb)
    mb2 = MeshBatch([fv.Mesh.cube(3, 0.1, 5), fv.Mesh.cube(4, 0.1, 6)])
    A2, b2 = fv.assemble(eq, (np.zeros(nb), np.ones(nb)), mb2)
    for x, y in zip(A1.to_csr(), A2.to_csr()):
        assert np.array_equal(x, y)
    assert np.array_equal(b1.numpy(), b2.numpy())


def test_batch_with_diagonal_preconditioner(fv, orc):
    """DiagonalPreconditioner in the batched CG (FP64 and mixed): per problem against the oracle's
    plain CG with the same preconditioner (<=1e-10 rel, iterations +-2 in FP64), same alone and in a mix."""
    from fvb200.batch import BatchCG
    probs = _problems(fv, [7, 11, 5], seed0=500)
    mb, A, b = _union_system(fv, probs)
    P = fv.DiagonalPreconditioner.from_matrix(A)
    x = fv.DistributedVector.from_size(mb.n_cells)
    out = BatchCG(A, mb.cell_offsets, 256).solve(P, b, x, precision="fp64", relative_tolerance=1e-10,
                                                 absolute_tolerance=1e-10, max_iterations=5000)
    xs = x.numpy()
    for k, (m, kf, sc) in enumerate(probs):
        nb = m.n_boundary_faces
        ptr, cols, vals, rhs = orc.assemble(m, -1.0, 0.0, -1.0, kappa=kf, source=sc, bndi=np.zeros(nb),
                                            bnde=np.zeros(nb))
        xo, io = orc.cg(ptr, cols, vals, orc.Precond("diag", ptr, cols, vals), rhs, rtol=1e-10, atol=1e-10,
                        maxit=5000)
        r0, r1 = mb.cell_offsets[k], mb.cell_offsets[k + 1]
        assert abs(int(out["iterations"][k]) - io["iterations"]) <= 2
        assert np.linalg.norm(xs[r0:r1] - xo) <= 1e-10 * np.linalg.norm(xo)
    x2 = fv.DistributedVector.from_size(mb.n_cells)
    o2 = BatchCG(A, mb.cell_offsets, 256).solve(P, b, x2, precision="mixed", outer_tolerance=1e-10)
    assert max(o2["final_residual"]) <= 1e-10
    mb1, A1, b1 = _union_system(fv, [probs[1]])
    P1 = fv.DiagonalPreconditioner.from_matrix(A1)
    x1 = fv.DistributedVector.from_size(mb1.n_cells)
    o1 = BatchCG(A1, mb1.cell_offsets, 256).solve(P1, b1, x1, precision="mixed", outer_tolerance=1e-10)
    r0, r1 = mb.cell_offsets[1], mb.cell_offsets[2]
    assert np.array_equal(x1.numpy(), x2.numpy()[r0:r1]) and int(o1["iterations"][0]) == int(o2["iterations"][1])


def test_batch_reordered_per_problem_and_same_alone_and_in_mix(fv, orc):
    """Box ordering per problem (offsets): each problem's factors are the
    oracle's on that problem's own reordered matrix, the union has the largest
    problem's level count, batched FP64 CG matches the oracle per problem, and
    a problem's result is the same bits alone and in a mix (FP64 and mixed)."""
    from fvb200.batch import BatchCG
    probs = _problems(fv, [12, 20, 8, 16], seed0=700)
    target = 2
    results = {}
    for name, subset in (("alone", [target]), ("mix", list(range(len(probs))))):
        sel = [probs[i] for i in subset]
        mb, A, b = _union_system(fv, sel)
        P = fv.IncompleteCholesky.from_matrix(A, 0, ordering="boxes", offsets=mb.cell_offsets)
        if name == "mix":
            levels = []
            xs = None
            x = fv.DistributedVector.from_size(mb.n_cells)
            out = BatchCG(A, mb.cell_offsets, 256).solve(P, b, x, precision="fp64", relative_tolerance=1e-10,
                                                         absolute_tolerance=1e-10, max_iterations=3000)
            xs = x.numpy()
            for k, (m, kf, sc) in enumerate(sel):
                nb = m.n_boundary_faces
                ptr, cols, vals, rhs = orc.assemble(m, -1.0, 0.0, -1.0, kappa=kf, source=sc, bndi=np.zeros(nb),
                                                    bnde=np.zeros(nb))
                perm, info = fv.order_boxes_host(m.cell_center, ptr, cols, 0, np.zeros(2), np.ones(2))
                levels.append(info["n_levels"])
                o = orc.Precond.reordered("ic", ptr, cols, vals, perm)
                xo, io = orc.cg(ptr, cols, vals, o, rhs, rtol=1e-10, atol=1e-10, maxit=3000)
                r0, r1 = mb.cell_offsets[k], mb.cell_offsets[k + 1]
                assert abs(int(out["iterations"][k]) - io["iterations"]) <= 2
                assert np.linalg.norm(xs[r0:r1] - xo) <= 1e-10 * np.linalg.norm(xo)
                # this problem's rows of the union's permutation, in order, are its own ordering
                own = P.perm[(P.perm >= r0) & (P.perm < r1)] - r0
                assert np.array_equal(own, perm)
            assert P.levels()[2] == max(levels) == P.order_info["n_levels"]
        for precision in ("fp64", "mixed"):
            x = fv.DistributedVector.from_size(mb.n_cells)
            out = BatchCG(A, mb.cell_offsets, 512).solve(P, b, x, precision=precision, relative_tolerance=1e-8,
                                                        absolute_tolerance=1e-8, outer_tolerance=1e-10)
            k = subset.index(target)
            r0, r1 = mb.cell_offsets[k], mb.cell_offsets[k + 1]
            results[(name, precision)] = (x.numpy()[r0:r1].copy(), int(out["iterations"][k]))
    for precision in ("fp64", "mixed"):
        xa, ia = results[("alone", precision)]
        xm, im = results[("mix", precision)]
        assert ia == im
        assert np.array_equal(xa, xm)
