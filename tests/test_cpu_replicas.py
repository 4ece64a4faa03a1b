"""Replica sharding across ranks, run as world_size-2 gloo process groups on CPU."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _worker(rank, world, port, q):
    sys.path.insert(0, str(ROOT / "finite-volumes-rs_b200"))
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch.distributed as dist

    from fvb200 import replicas
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(0)
        cells = 2 * np.rint(np.exp(rng.uniform(np.log(32), np.log(512), 64))).astype(int) ** 2
        assign = replicas.assign_greedy(cells, world)
        mine = assign[rank]
        # every rank computed the same assignment
        import torch
        gathered = [None] * world
        dist.all_gather_object(gathered, assign)
        t = replicas.max_over_ranks(1.0 + rank)
        # per-rank work: the oracle solves this rank's two smallest problems
        import oracle
        import fvb200 as fv
        solved = 0
        for k in sorted(mine, key=lambda k: cells[k])[:2]:
            side = int(round(np.sqrt(cells[k] / 2)))
            m = fv.Mesh.square(side, 0.2, replicas.rank_seed(10, rank) + k)
            kf, _, sc = m.fields(k, 1.0, 1.0)
            nb = m.n_boundary_faces
            ptr, cols, vals, rhs = oracle.assemble(m, -1.0, 0.0, -1.0, kappa=kf, source=sc, bndi=np.zeros(nb),
                                                   bnde=np.zeros(nb))
            x, info = oracle.cg(ptr, cols, vals, oracle.Precond("ic", ptr, cols, vals), rhs, rtol=1e-8, atol=1e-8,
                                maxit=5000)
            solved += int(info["final_residual"] < 1e-8)
        q.put((rank, mine, all(g == assign for g in gathered), t, solved, replicas.imbalance(cells, assign)))
    finally:
        dist.destroy_process_group()


def test_replicas_two_gloo_ranks():
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
    (r0, m0, same0, t0, s0, imb), (r1, m1, same1, t1, s1, _) = res
    assert same0 and same1
    assert sorted(m0 + m1) == list(range(64)) and not set(m0) & set(m1)
    assert t0 == t1 == 2.0          # max over ranks
    assert s0 == 2 and s1 == 2      # each rank solved its own problems
    assert imb < 1.05               # greedy by cells balances the load


def test_assign_greedy_properties():
    sys.path.insert(0, str(ROOT / "finite-volumes-rs_b200"))
    from fvb200.replicas import assign_greedy
    cells = [5, 1, 9, 3, 3, 7]
    a = assign_greedy(cells, 3)
    assert sorted(sum(a, [])) == list(range(6))
    assert assign_greedy(cells, 1) == [list(range(6))]
    with pytest.raises(Exception):
        assign_greedy(cells, 0)[0]
