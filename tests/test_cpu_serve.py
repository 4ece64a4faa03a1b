"""Request server scheduling on CPU (fake solver; no GPU)."""
import threading
import time

import numpy as np


class _Stream:
    def synchronize(self):
        pass


def _fake_solve(delay_per_cell=2e-8, fail_rid=None):
    lock = threading.Lock()
    state = {"in_flight": 0, "max_in_flight": 0}

    def solve(fv, cache, wave, stream):
        with lock:
            state["in_flight"] += 1
            state["max_in_flight"] = max(state["max_in_flight"], state["in_flight"])
        try:
            if fail_rid is not None and any(r.rid == fail_rid for r in wave):
                raise RuntimeError("injected failure")
            time.sleep(sum(r.cells for r in wave) * delay_per_cell)
            for r in wave:
                r.iterations = 10
                r.residual = 1e-11
        finally:
            with lock:
                state["in_flight"] -= 1

    return solve, state


def test_request_stream_statistics():
    from fvb200.serve import request_stream
    reqs = request_stream(rate=2000.0, duration=2.0, seed=1)
    assert 3600 < len(reqs) < 4400                       # Poisson count around 4000
    cells = np.array([r.cells for r in reqs], float)
    assert cells.min() >= 9_000 and cells.max() <= 2_100_000
    p1, p99 = np.percentile(cells, [1, 99])
    assert 7e3 < p1 < 2e4 and 1.2e6 < p99 <= 2.1e6
    frac3d = np.mean([r.kind == "3d" for r in reqs])
    assert 0.45 < frac3d < 0.55
    gaps = np.diff([r.arrival for r in reqs])
    assert abs(gaps.mean() - 1 / 2000.0) < 1e-4


def test_server_admission_respects_budget_and_survives_a_failure(fv):
    """A wave whose solve raises fails its own requests only; admission never
    reserves more than the memory budget; waves overlap."""
    from fvb200.serve import BYTES_PER_CELL, Request, Server
    rng = np.random.default_rng(0)
    reqs = []
    for k in range(60):
        kind = "2d" if k % 2 else "3d"
        cells = int(rng.integers(2_000, 40_000))
        reqs.append(Request(k, 0.002 * k, kind, 10, k, cells=cells))
    budget = 40 * 40_000 * max(BYTES_PER_CELL.values())  # room for a few waves only
    solve, state = _fake_solve(delay_per_cell=3e-7, fail_rid=17)
    srv = Server(fv, workers=3, budget_bytes=budget, max_wave_cells=120_000, max_wave_requests=8,
                 solve_fn=solve, make_stream=_Stream)
    stats = srv.run(reqs, time_limit=60.0, warm=False)
    failed = [r for r in reqs if r.error]
    assert len(failed) >= 1 and any(r.rid == 17 for r in failed)
    assert stats["completed"] + stats["failed"] == len(reqs)
    assert stats["peak_reserved_bytes"] <= budget
    assert state["max_in_flight"] >= 2                   # waves overlap
    assert all(r.finish >= r.arrival for r in reqs)
    by_wave = {}
    for r in reqs:
        by_wave.setdefault(r.wave, []).append(r)
    for w in by_wave.values():
        assert len({r.kind for r in w}) == 1 and len(w) <= 8
