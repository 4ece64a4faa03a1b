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


def test_size_class_waves_finish_small_requests_early(fv):
    """wave_order "size": every wave is one size class of one kind, worker 0
    starts with the largest request, and when a wave lasts as long as its
    largest problem, the median latency drops well below FIFO packing while
    the span stays that of the largest solve."""
    from fvb200.serve import Request, Server
    rng = np.random.default_rng(3)
    reqs = []
    for k in range(120):
        cells = int(np.exp(rng.uniform(np.log(2e3), np.log(4e5))))
        reqs.append(Request(k, 0.0, "2d" if k % 3 else "3d", 10, k, cells=cells))  # one burst

    def solve(fv, cache, wave, stream):  # a wave lasts as long as its largest problem
        time.sleep(max(r.cells for r in wave) * 2e-6)
        for r in wave:
            r.iterations, r.residual = 10, 1e-11

    out = {}
    for order in ("fifo", "size"):
        for r in reqs:
            r.finish, r.wave, r.error = -1.0, -1, None
        srv = Server(fv, workers=2, budget_bytes=1 << 40, max_wave_cells=4_000_000, max_wave_requests=64,
                     solve_fn=solve, make_stream=_Stream, wave_order=order, size_ratio=4.0, aging_s=30.0)
        out[order] = srv.run(reqs, time_limit=60.0, warm=False)
        assert out[order]["completed"] == len(reqs)
        if order == "size":
            by_wave = {}
            for r in reqs:
                by_wave.setdefault(r.wave, []).append(r)
            for w in by_wave.values():
                c = [r.cells for r in w]
                assert len({r.kind for r in w}) == 1 and max(c) <= 4.0 * min(c)
            biggest = max(reqs, key=lambda r: r.cells)
            assert biggest.wave in (0, 1)  # among the first waves taken
    assert out["size"]["p50_ms"] < 0.6 * out["fifo"]["p50_ms"]
    assert out["size"]["wall_s"] < 1.5 * out["fifo"]["wall_s"]


def test_wave_order_is_checked(fv):
    import pytest
    from fvb200.serve import Server
    with pytest.raises(ValueError):
        Server(fv, budget_bytes=1, solve_fn=lambda *a: None, make_stream=_Stream, wave_order="random")


def test_batching_window_groups_early_arrivals(fv):
    """The first arrival waits up to batch_window_s for requests that arrive
    right after it, so they share its wave."""
    from fvb200.serve import Request, Server
    reqs = [Request(0, 0.0, "2d", 10, 0, cells=1000)] + [Request(k, 0.02, "2d", 10, k, cells=1000)
                                                          for k in range(1, 6)]

    def solve(fv, cache, wave, stream):
        time.sleep(0.01)

    srv = Server(fv, workers=1, budget_bytes=1 << 40, solve_fn=solve, make_stream=_Stream, batch_window_s=0.1)
    stats = srv.run(reqs, time_limit=30.0, warm=False)
    assert stats["completed"] == 6 and stats["waves"] == 1


def test_mesh_cache_builds_each_key_once_under_concurrent_gets():
    """Threads asking for the same (kind, side) at once get one mesh object,
    built once, and the cache's cell count holds it once."""
    import threading
    import time as _time
    from types import SimpleNamespace

    from fvb200.serve import MeshCache

    builds = []

    class FakeMesh:
        @staticmethod
        def square(side, jitter, seed, on_device=True):
            builds.append(side)
            _time.sleep(0.05)  # a slow build: the other threads arrive meanwhile
            return SimpleNamespace(n_cells=2 * side * side)

    cache = MeshCache(SimpleNamespace(Mesh=FakeMesh), capacity_cells=10_000)
    got = []
    ts = [threading.Thread(target=lambda: got.append(cache.get("2d", 16))) for _ in range(6)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert builds == [16]
    assert len(got) == 6 and all(g is got[0] for g in got)
    assert cache.cells == 2 * 16 * 16
    # eviction keeps the count equal to the meshes held
    cache.get("2d", 40)
    cache.get("2d", 60)
    assert cache.cells == sum(m.n_cells for m in cache.d.values()) and cache.cells <= 10_000


def test_capped_run_stops_at_the_cap_and_reports_the_backlog():
    """drain=False: at the wall cap admission stops, running waves finish,
    nothing new starts, and every request is either completed or backlog."""
    from fvb200.serve import Server, request_stream
    reqs = request_stream(rate=400.0, duration=2.0, seed=3)
    solve, _ = _fake_solve(delay_per_cell=1e-7)  # slower than the arrivals: a backlog builds
    srv = Server(None, workers=2, budget_bytes=10 ** 12, solve_fn=solve, make_stream=_Stream)
    t0 = time.perf_counter()
    st = srv.run(reqs, time_limit=1.0, warm=False, drain=False)
    wall = time.perf_counter() - t0
    assert st["backlog"] > 0
    assert st["completed"] + st["backlog"] + st["failed"] == st["offered"] == len(reqs)
    assert st["arrived_by_cap"] < len(reqs)
    # the last waves started before the cap; no wave is longer than a few seconds here
    assert wall < 1.0 + 10.0


class _FakeRun:
    """A stepwise wave: request r needs r.seed % 5 + 1 advances in total; a
    carried request keeps what it has done (a restart would show as extra
    advances); rid 7 stagnates, a wave holding rid 13 fails to build."""
    builds = []

    def __init__(self, fv, cache, reqs, stream, prev=None):
        if any(r.rid == 13 for r in reqs):
            raise RuntimeError("injected build failure")
        assert len({r.kind for r in reqs}) == 1
        self.kind = reqs[0].kind
        self.reqs = list(reqs)
        self.steps = {r.rid: (prev.steps[r.rid] if prev is not None and r.rid in prev.steps else 0) for r in reqs}
        carried = [r.rid for r in reqs if prev is not None and r.rid in prev.steps]
        if prev is not None:
            assert all(not prev.finished.get(rid, False) for rid in carried)
        self.finished = {}
        _FakeRun.builds.append(([r.rid for r in reqs], carried))

    @property
    def cells(self):
        return sum(r.cells for r in self.running())

    def running(self):
        return [r for r in self.reqs if not self.finished.get(r.rid)]

    def advance(self, iterations):
        time.sleep(0.002)
        fin, stalled = [], []
        for r in self.running():
            self.steps[r.rid] += 1
            if self.steps[r.rid] == r.seed % 5 + 1:
                self.finished[r.rid] = True
                r.iterations = self.steps[r.rid]
                r.residual = 1e-11
                (stalled if r.rid == 7 else fin).append(r)
        return fin, stalled

    def close(self):
        pass


def test_refill_carries_running_requests_and_refills_freed_slots(fv):
    """Refill mode: finished requests leave at once, waiting requests of the
    same kind join the running wave, carried requests never restart, every
    wave has one kind and at most max_wave_requests requests, a failed build
    fails only the newly admitted requests, a stagnated request is solved by
    the fallback."""
    from fvb200.serve import Request, Server
    _FakeRun.builds = []
    reqs = [Request(k, 0.001 * k, "2d" if k % 3 else "3d", 10, k, cells=1000 + 10 * k) for k in range(80)]
    fell_back = []

    def fallback(fv_, cache_, wave, stream):
        fell_back.extend(r.rid for r in wave)
        for r in wave:
            r.residual = 1e-12

    srv = Server(None, workers=2, budget_bytes=10 ** 12, refill=True, run_fn=_FakeRun, fallback_fn=fallback,
                 make_stream=_Stream, max_wave_requests=6, max_wave_cells=10 ** 9, refill_fraction=0.2,
                 batch_window_s=0.0)
    st = srv.run(reqs, time_limit=60.0, warm=False)
    assert st["refills"] > 0
    assert st["completed"] + st["failed"] == len(reqs)
    failed = {r.rid for r in reqs if r.error}
    assert 13 in failed and len(failed) <= 6       # only the build that held 13 failed (its new requests)
    assert fell_back == [7]
    for r in reqs:
        if r.error is None:
            assert r.iterations == r.seed % 5 + 1, r.rid   # carried over, never restarted
            assert r.finish >= r.start >= r.arrival
    seen_carried = False
    for rids, carried in _FakeRun.builds:
        assert len(rids) <= 6
        kinds = {reqs[i].kind for i in rids}
        assert len(kinds) == 1
        seen_carried |= bool(carried)
    assert seen_carried
