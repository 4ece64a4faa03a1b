"""One problem split over ranks (domain decomposition), host side, on CPU.

- HaloPlan: each rank's local matrix (owned + ghost columns) reproduces the
  global SpMV rows; send and receive lists agree between every pair of ranks
- Communicator.collect / reduce_add over a world_size-2 gloo process group
  deliver the owners' ghost values and the global sums
- the square block of a rank's matrix is the block the block-Jacobi oracle
  factorises
"""
import os
import sys
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp

from cases import convdiff_3d, diffusion_2d, oracle_system

ROOT = Path(__file__).resolve().parents[1]


def _system(fv, orc, kind):
    case = diffusion_2d(fv, 14, seed=4) if kind == "2d" else convdiff_3d(fv, 4, seed=2)
    return oracle_system(orc, case)


@pytest.mark.parametrize("kind,world", [("2d", 2), ("2d", 3), ("3d", 4)])
def test_halo_plan_reproduces_global_spmv(fv, orc, kind, world):
    from fvb200.decompose import HaloPlan, contiguous_partition
    ptr, cols, vals, _ = _system(fv, orc, kind)
    n = len(ptr) - 1
    A = sp.csr_matrix((vals, cols, ptr), shape=(n, n))
    x = np.random.default_rng(1).standard_normal(n)
    want = A @ x
    bounds = contiguous_partition(n, world)
    plans = [HaloPlan.from_global(ptr, cols, vals, bounds, r) for r in range(world)]
    for p in plans:
        assert p.n_own == bounds[p.rank + 1] - bounds[p.rank]
        assert np.all(np.diff(p.ghosts) > 0)
        assert not np.any((p.ghosts >= p.lo) & (p.ghosts < p.hi))
        for i in range(p.n_own):  # rows sorted by local column
            assert np.all(np.diff(p.cols[p.row_ptr[i]:p.row_ptr[i + 1]]) > 0)
        xl = np.concatenate([x[p.lo:p.hi], x[p.ghosts]])
        L = sp.csr_matrix((p.vals, p.cols, p.row_ptr), shape=(p.n_own, p.n_own + p.n_ghost))
        assert np.allclose(L @ xl, want[p.lo:p.hi], rtol=1e-14, atol=1e-14 * np.abs(want).max())
        # square block: the owned columns only
        sq = L[:, :p.n_own].toarray()
        assert np.array_equal(sq, A[p.lo:p.hi, p.lo:p.hi].toarray())
    # what q sends to r is what r receives from q, in the same order
    for r in plans:
        for q in plans:
            if q.rank == r.rank:
                continue
            sent = q.send_idx[q.send_displs[r.rank]:q.send_displs[r.rank + 1]] + q.lo
            got = r.ghosts[r.recv_displs[q.rank]:r.recv_displs[q.rank + 1]]
            assert np.array_equal(sent, got)
    assert sum(len(p.ghosts) for p in plans) == sum(len(p.send_idx) for p in plans)


def _worker(rank, world, port, q):
    sys.path.insert(0, str(ROOT / "finite-volumes-rs_b200"))
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    import fvb200 as fv
    import oracle
    from fvb200.decompose import Communicator, HaloPlan, contiguous_partition
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ptr, cols, vals, _ = _system(fv, oracle, "3d")
        n = len(ptr) - 1
        bounds = contiguous_partition(n, world)
        plan = HaloPlan.from_global(ptr, cols, vals, bounds, rank)
        comm = Communicator()
        xg = np.arange(n, dtype=np.float64) * 0.5 + 1.0        # the global vector every rank could see
        x_own = torch.tensor(xg[plan.lo:plan.hi])
        send = x_own[torch.as_tensor(plan.send_idx.astype(np.int64))].contiguous()
        ghost = torch.full((plan.n_ghost,), -1.0, dtype=torch.float64)
        comm.collect(plan, send, ghost)
        ok_ghost = bool(np.array_equal(ghost.numpy(), xg[plan.ghosts]))
        buf = torch.tensor([float(rank + 1), float(plan.n_own)], dtype=torch.float64)
        comm.reduce_add(buf)
        ok_sum = bool(buf[0].item() == world * (world + 1) / 2 and buf[1].item() == n)
        q.put((rank, ok_ghost, ok_sum, plan.n_ghost))
    finally:
        dist.destroy_process_group()


def test_collect_and_reduce_add_two_gloo_ranks():
    import multiprocessing as mp
    import socket
    ctx = mp.get_context("spawn")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    q = ctx.Queue()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=240) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ok_ghost, ok_sum, ng in res:
        assert ok_ghost and ok_sum and ng > 0
