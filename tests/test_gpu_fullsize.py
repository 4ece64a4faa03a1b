"""The 12.6M-cell benchmark problem (unit cube 128^3 x 6 Kuhn tetrahedra,
convection-diffusion, BiCGStab + ILU(0)) checked through properties that do
not need an oracle run at this size:

- the mesh built on the GPU equals the host builder's, every array bit for bit
- the triangular sweeps give the same bits under both level-chunk schedules,
  and applying the preconditioner twice gives the same bits (sentinel resets)
- the preconditioner inverts its own factors: L U z = r row by row, within
  rounding, checked on the host with the exported factors
- BiCGStab reaches the requested tolerance on the true residual |b - A x| / |b|
"""
import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu

N = 128


@pytest.fixture(scope="module")
def system(fv):
    m = fv.Mesh.cube(N, 0.15, 1000, on_device=True)
    v = (1.0, 0.5, 0.25)
    kf, fl, sc = m.fields(1000, float(np.linalg.norm(v)) / N / 3.0, 0.5, velocity=v, source_uniform=True)
    nb = m.n_boundary_faces
    eq = fv.convection(fv.Upwind(fl), fl) - fv.laplacian(fv.Orthogonal(), kf) - fv.source(sc)
    A, b = fv.assemble(eq, (np.zeros(nb), np.zeros(nb)), m)
    P = fv.IncompleteLowerUpper.from_matrix(A, 0)
    return m, A, b, P


def test_device_mesh_equals_host_mesh(fv, system):
    m = system[0]
    h = fv.Mesh.cube(N, 0.15, 1000)
    assert (m.n_cells, m.n_faces, m.n_boundary_faces) == (6 * N ** 3, h.n_faces, 6 * 2 * N * N)
    for name in ("face_node_ptr", "face_nodes", "face_patch", "cell_face_ptr", "cell_faces", "face_owner",
                 "face_neighbor", "face_area", "face_normal", "face_center", "cell_center", "cell_volume"):
        assert getattr(m, name).tobytes() == getattr(h, name).tobytes(), name


def test_sweeps_same_bits_across_schedules_and_repeats(fv, system):
    m, A, b, P = system
    r = fv.DistributedVector(np.random.default_rng(3).standard_normal(m.n_cells))
    out = []
    for sched in (1, 3, 1):
        P.schedule(sched)
        z = fv.DistributedVector.from_size(m.n_cells)
        P.precondition(z, r)
        out.append(z.numpy())
    P.schedule(1)
    assert out[0].tobytes() == out[1].tobytes() == out[2].tobytes()
    # L U z = r on the exported factors (unit lower L, U with the diagonal)
    fp, fc, fvv, nd = P.factors()
    assert nd == 0
    n = m.n_cells
    F = sp.csr_matrix((fvv, fc, fp), shape=(n, n))
    L = sp.tril(F, -1, format="csr") + sp.eye(n, format="csr")
    U = sp.triu(F, 0, format="csr")
    res = L @ (U @ out[0]) - r.numpy()
    assert np.linalg.norm(res) <= 1e-12 * np.linalg.norm(r.numpy())


def test_bicgstab_reaches_tolerance(fv, system):
    m, A, b, P = system
    x = fv.DistributedVector.from_size(m.n_cells)
    info = fv.bi_conjugate_gradient_stab(x, A, b, P, None, fv.LinearSolverOptions(1e-8, 1e-8, 10000))
    assert info.status == 0 and 100 < info.iterations < 400
    ptr, cols, vals = A.to_csr()
    Ah = sp.csr_matrix((vals, cols, ptr), shape=(m.n_cells, m.n_cells))
    bb = b.numpy()
    true_rel = np.linalg.norm(bb - Ah @ x.numpy()) / np.linalg.norm(bb)
    assert true_rel <= 2e-8
