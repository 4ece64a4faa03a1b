"""Box-tiled sweeps, and level chunks with the next chunk prefetched, on the
GPU: the same bits as the level-ordered sweeps.

A matrix assembled on a mesh gets a box tiling at factorisation; the tiled
sweeps must reproduce the level-chunk sweeps (and so the oracle) bit for bit,
in FP64 and in the FP32 sweeps of the mixed-precision batch.
"""
import numpy as np
import pytest

from cases import convdiff_3d, diffusion_2d, equation, oracle_system

pytestmark = pytest.mark.gpu


def _system(fv, case):
    return fv.assemble(equation(fv, case), (case["bndi"], case["bnde"]), case["mesh"])


@pytest.mark.parametrize("kind", ["3d", "2d"])
def test_tiled_apply_equals_level_apply_and_oracle(fv, orc, kind):
    case = convdiff_3d(fv, 10, seed=4) if kind == "3d" else diffusion_2d(fv, 48, seed=4)
    A, b = _system(fv, case)
    P = (fv.IncompleteLowerUpper if kind == "3d" else fv.IncompleteCholesky).from_matrix(A, 0)
    assert P.schedule()[0] == 1  # level chunks by default
    act, st = P.schedule(2)
    assert act == 2 and st[0] > 0 and st[1] > 1
    r = fv.DistributedVector(np.random.default_rng(5).standard_normal(A.nrows()))
    z_tiles = fv.DistributedVector.from_size(A.nrows())
    P.precondition(z_tiles, r)
    P.schedule(1)
    assert P.schedule()[0] == 1
    z_levels = fv.DistributedVector.from_size(A.nrows())
    P.precondition(z_levels, r)
    assert np.array_equal(z_tiles.numpy(), z_levels.numpy())
    ptr, cols, vals, _ = oracle_system(orc, case)
    want = orc.Precond("ilu" if kind == "3d" else "ic", ptr, cols, vals).apply(r.numpy())
    assert np.array_equal(z_tiles.numpy(), want)
    # level chunks with the next chunk prefetched: same bits
    assert P.schedule(3)[0] == 3
    z_pf = fv.DistributedVector.from_size(A.nrows())
    for _ in range(3):
        P.precondition(z_pf, r)
    assert np.array_equal(z_pf.numpy(), want)
    # repeated applies keep the sentinel protocol intact
    P.schedule(2)
    for _ in range(3):
        P.precondition(z_tiles, r)
    assert np.array_equal(z_tiles.numpy(), want)


def test_tiled_solve_equals_level_solve(fv):
    case = convdiff_3d(fv, 12, seed=6)
    A, b = _system(fv, case)
    P = fv.IncompleteLowerUpper.from_matrix(A, 0)
    opts = fv.LinearSolverOptions(1e-10, 1e-10, 2000)
    out = {}
    for req in (2, 3, 1):
        P.schedule(req)
        x = fv.DistributedVector.from_size(A.nrows())
        info = fv.bi_conjugate_gradient_stab(x, A, b, P, None, opts)
        out[req] = (x.numpy(), info.iterations, info.history)
    for req in (2, 3):
        assert out[req][1] == out[1][1]
        assert np.array_equal(out[req][0], out[1][0])
        assert out[req][2] == out[1][2]


def test_tiled_fp32_batch_equals_level_batch(fv):
    """Mixed-precision batch (FP32 sweeps): both schedules, same result."""
    from fvb200.batch import BatchCG, MeshBatch
    ms = [fv.Mesh.square(s, 0.2, 60 + s) for s in (20, 33, 9)]
    mb = MeshBatch(ms)
    kf = mb.face_field([m.fields(3 + k, 1.0, 1.0)[0] for k, m in enumerate(ms)])
    sc = mb.cell_field([np.ones(m.n_cells) for m in ms])
    nb = mb.n_boundary_faces
    A, b = fv.assemble(-fv.laplacian(fv.Orthogonal(), kf) - fv.source(sc), (np.zeros(nb), np.zeros(nb)), mb)
    P = fv.IncompleteCholesky.from_matrix(A, 0)
    assert P.schedule(2)[0] == 2
    res = {}
    for req in (2, 3, 1):
        P.schedule(req)
        x = fv.DistributedVector.from_size(mb.n_cells)
        o = BatchCG(A, mb.cell_offsets, 256).solve(P, b, x, precision="mixed", outer_tolerance=1e-10)
        res[req] = (x.numpy(), list(o["iterations"]))
    for req in (2, 3):
        assert res[req][1] == res[1][1]
        assert np.array_equal(res[req][0], res[1][0])
