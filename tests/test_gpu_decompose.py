"""One problem split over ranks, the device path (fv_dist_cg / fv_dist_bicgstab).

Only one GPU is available to these tests, so the ranks are host threads on
that GPU, each with its own stream, local matrix and block preconditioner.
Their collect / reduce_add callbacks meet at a host barrier: every rank
finishes its own stream, then copies the peers' packed send buffers into its
ghost tail (collect) or sums the peers' partial sums in rank order
(reduce_add).  No kernel ever waits for another rank's kernel.

Checked against the block-Jacobi oracle (the reference's MPI algorithm with
the same contiguous partition): solution <= 1e-10 rel, iterations +-2.
"""
import threading

import numpy as np
import pytest

from cases import convdiff_3d, diffusion_2d, oracle_system

pytestmark = pytest.mark.gpu


class EmulatedRanks:
    def __init__(self, plans):
        self.plans = plans
        self.P = len(plans)
        self.bar = threading.Barrier(self.P, timeout=120)
        self.send_ptr = [0] * self.P
        self.sums = [None] * self.P

    def comm(self, r):
        import torch

        from fvb200.decompose import _cuda_tensor, make_fv_comm
        plan = self.plans[r]

        def collect(ctx, send, ghost, stream):
            try:
                torch.cuda.synchronize()
                self.send_ptr[r] = send or 0
                self.bar.wait()
                g = _cuda_tensor(ghost, plan.n_ghost) if plan.n_ghost else None
                rd = plan.recv_displs
                for q in range(self.P):
                    cnt = int(plan.recv_counts[q])
                    if q == r or cnt == 0:
                        continue
                    off = int(self.plans[q].send_displs[r])
                    src = _cuda_tensor(self.send_ptr[q] + 8 * off, cnt)
                    g[rd[q]:rd[q + 1]].copy_(src)
                torch.cuda.synchronize()
                self.bar.wait()
                return 0
            except Exception:
                self.bar.abort()
                return 1

        def reduce_add(ctx, buf, count, stream):
            try:
                torch.cuda.synchronize()
                t = _cuda_tensor(buf, count)
                self.sums[r] = t.cpu().numpy().copy()
                self.bar.wait()
                s = self.sums[0].copy()
                for q in range(1, self.P):
                    s = s + self.sums[q]
                self.bar.wait()
                t.copy_(torch.from_numpy(s))
                torch.cuda.synchronize()
                return 0
            except Exception:
                self.bar.abort()
                return 1

        return make_fv_comm(collect, reduce_add)


def _run(fv, orc, case, world, solver, kind):
    import torch

    from fvb200.decompose import HaloPlan, RankSystem, contiguous_partition
    from oracle import mpi as ompi
    ptr, cols, vals, rhs = oracle_system(orc, case)
    n = len(ptr) - 1
    bounds = contiguous_partition(n, world)
    plans = [HaloPlan.from_global(ptr, cols, vals, bounds, r) for r in range(world)]
    emu = EmulatedRanks(plans)
    opts = fv.LinearSolverOptions(1e-10, 1e-10, 3000)
    out = [None] * world
    systems, precs, comms = [], [], []
    for r, p in enumerate(plans):
        comms.append(emu.comm(r))
        systems.append(RankSystem(p, comms[-1]))
        blk = systems[-1].square_block()
        precs.append((fv.IncompleteCholesky if kind == "ic" else fv.IncompleteLowerUpper).from_matrix(blk, 0))
        precs[-1]._blk = blk

    def rank_main(r):
        try:
            st = torch.cuda.Stream()
            p = plans[r]
            b = fv.DistributedVector(rhs[p.lo:p.hi])
            x = fv.DistributedVector.from_size(p.n_own)
            torch.cuda.synchronize()
            info = systems[r].solve(solver, x, b, precs[r], opts, stream=st)
            st.synchronize()
            out[r] = (x.numpy(), info)
        except Exception as e:  # surfaced by the assertions below
            out[r] = e
            emu.bar.abort()

    th = [threading.Thread(target=rank_main, args=(r,)) for r in range(world)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=300)
    for o in out:
        assert not isinstance(o, Exception), o
    x = np.concatenate([o[0] for o in out])
    its = {o[1].iterations for o in out}
    assert len(its) == 1  # every rank took the same steps
    bj = ompi.BlockJacobi(kind, ptr, cols, vals, world)
    xo, io = ompi.solve(solver, ptr, cols, vals, bj, rhs, 1e-10, 1e-10, 3000)
    return x, out[0][1], xo, io


@pytest.mark.parametrize("world", [2, 3])
def test_dist_cg_ic0_matches_block_jacobi_oracle(fv, orc, world):
    x, info, xo, io = _run(fv, orc, diffusion_2d(fv, 40, seed=6), world, "cg", "ic")
    assert abs(info.iterations - io["iterations"]) <= 2
    assert np.linalg.norm(x - xo) <= 1e-10 * np.linalg.norm(xo)
    assert info.status == 0


def test_dist_bicgstab_ilu0_matches_block_jacobi_oracle(fv, orc):
    x, info, xo, io = _run(fv, orc, convdiff_3d(fv, 7, seed=9), 2, "bicgstab", "ilu")
    assert abs(info.iterations - io["iterations"]) <= 2
    assert np.linalg.norm(x - xo) <= 1e-10 * np.linalg.norm(xo)


def test_single_rank_dist_equals_plain_solver(fv, orc):
    """One rank, no communicator: the distributed loop is the plain solver."""
    from fvb200.decompose import HaloPlan, RankSystem, contiguous_partition
    case = diffusion_2d(fv, 24, seed=8)
    ptr, cols, vals, rhs = oracle_system(orc, case)
    plan = HaloPlan.from_global(ptr, cols, vals, contiguous_partition(len(ptr) - 1, 1), 0)
    rs = RankSystem(plan, None)
    assert plan.n_ghost == 0
    P = fv.IncompleteCholesky.from_matrix(rs.square_block(), 0)
    opts = fv.LinearSolverOptions(1e-10, 1e-10, 2000)
    x1 = fv.DistributedVector.from_size(len(rhs))
    i1 = rs.solve("cg", x1, fv.DistributedVector(rhs), P, opts)
    A = fv.DistributedMatrix.from_csr(ptr, cols, vals)
    P0 = fv.IncompleteCholesky.from_matrix(A, 0)
    x0 = fv.DistributedVector.from_size(len(rhs))
    i0 = fv.conjugate_gradient(x0, A, fv.DistributedVector(rhs), P0, None, opts)
    assert abs(i1.iterations - i0.iterations) <= 1
    assert np.linalg.norm(x1.numpy() - x0.numpy()) <= 1e-10 * np.linalg.norm(x0.numpy())
