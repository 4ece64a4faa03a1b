"""Serving: continuous batching of independent requests on one GPU."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_request_same_alone_and_in_a_wave(fv):
    import torch

    from fvb200.serve import MeshCache, Request, solve_wave
    cache = MeshCache(fv)
    reqs = [Request(0, 0.0, "2d", 20, 11, cells=800), Request(1, 0.0, "2d", 33, 12, cells=2178),
            Request(2, 0.0, "2d", 9, 13, cells=162)]
    st = torch.cuda.Stream()
    solve_wave(fv, cache, reqs, st, tile_rows=256, keep_solution=True)
    mixed = {r.rid: (r.solution.copy(), r.iterations) for r in reqs}
    alone = Request(1, 0.0, "2d", 33, 12, cells=2178)
    solve_wave(fv, cache, [alone], st, tile_rows=256, keep_solution=True)
    assert np.array_equal(alone.solution, mixed[1][0])
    assert alone.iterations == mixed[1][1]
    r3 = [Request(3, 0.0, "3d", 5, 21, cells=750), Request(4, 0.0, "3d", 4, 22, cells=384)]
    solve_wave(fv, cache, r3, st, tile_rows=256, keep_solution=True)
    a = Request(4, 0.0, "3d", 4, 22, cells=384)
    solve_wave(fv, cache, [a], st, tile_rows=256, keep_solution=True)
    assert np.array_equal(a.solution, r3[1].solution)
    assert max(r.residual for r in reqs + r3) <= 1e-10


def test_server_completes_a_small_stream(fv):
    from fvb200.serve import Server, request_stream
    reqs = request_stream(rate=200.0, duration=0.25, seed=3, lo=2e3, hi=4e4)
    assert len(reqs) > 10
    srv = Server(fv, workers=2, max_wave_cells=200_000, max_wave_requests=16)
    stats = srv.run(reqs, time_limit=120.0)
    assert stats["completed"] == len(reqs)
    assert stats["max_residual"] <= 1e-10
    assert stats["waves"] >= 2
    assert stats["p99_ms"] >= stats["p50_ms"] > 0
