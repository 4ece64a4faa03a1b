"""Request server: continuous batching of independent solves on one GPU.

Requests (a mesh size, a seed, a tolerance) arrive as a Poisson stream.  An
arrived request is admitted when its estimated device memory fits the free
budget; admitted requests of one kind (2D diffusion -> CG + IC(0), 3D
convection-diffusion -> BiCGStab + ILU(0)) are packed into a wave, a
block-diagonal batch solved with per-problem scalars in mixed precision
(fvb200.batch).  Several waves are in flight at once, each on its own CUDA
stream driven by its own host thread, so work of requests that arrived while
others were running overlaps on the device; a worker that finishes a wave
immediately takes the next admitted requests (slots are refilled as they
free up).  Per-problem reductions never mix problems, so a request's result
is the same alone and in any wave.

A wave lasts as long as its slowest problem, which grows with the problem's
size, and every request of a wave completes when the wave does.  With
wave_order "size" (the default) waves are therefore built from one size
class: worker 0 takes the largest admitted requests first (the longest solves
start at once, which keeps the stream's span short), the other workers the
smallest (short waves, so most requests complete early); a request that has
waited longer than `aging_s` is taken first by any worker.  wave_order "fifo"
packs requests in arrival order.  A wave is formed once its oldest request
has waited `batch_window_s` (or the admitted requests fill a wave, or no
more requests are due), so a wave does not start with the first arrival alone.

Meshes are built on the host per (kind, size) and cached; the request's seed
drives its diffusivity and source fields.
"""
from __future__ import annotations

import collections
import dataclasses
import threading
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from .batch import BatchCG, MeshBatch


@dataclasses.dataclass
class Request:
    rid: int
    arrival: float         # seconds from the start of the stream
    kind: str              # "2d" or "3d"
    side: int              # 2D: squares per side; 3D: hexes per side
    seed: int
    rtol: float = 1e-8
    cells: int = 0
    # filled by the server
    start: float = -1.0
    finish: float = -1.0
    wave: int = -1
    iterations: int = 0
    residual: float = float("nan")
    solution: np.ndarray | None = None
    error: str | None = None


def request_stream(rate: float, duration: float, seed: int, mix_3d: float = 0.5, lo: float = 1e4,
                   hi: float = 2e6) -> list[Request]:
    """Poisson arrivals; cells lognormal with 1st/99th percentiles lo/hi,
    clipped to [lo, hi]; 2D side = round(sqrt(cells/2)), 3D n = round((cells/6)^(1/3))."""
    rng = np.random.default_rng(seed)
    mu = 0.5 * (np.log(lo) + np.log(hi))
    sigma = (np.log(hi) - mu) / 2.3263478740408408
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        cells = float(np.clip(np.exp(rng.normal(mu, sigma)), lo, hi))
        if rng.random() < mix_3d:
            n = max(2, int(round((cells / 6.0) ** (1.0 / 3.0))))
            out.append(Request(len(out), t, "3d", n, int(rng.integers(1 << 30)), cells=6 * n ** 3))
        else:
            s = max(2, int(round(np.sqrt(cells / 2.0))))
            out.append(Request(len(out), t, "2d", s, int(rng.integers(1 << 30)), cells=2 * s * s))
    return out


class MeshCache:
    """Meshes per (kind, side), built on the GPU (faces, geometry and the
    resident fv_mesh on the device; the host arrays read back); geometry
    jitter seeded by the size.  A wave joins its meshes on the device."""

    def __init__(self, fv, capacity_cells: int = 60_000_000, on_device: bool = True):
        self.fv = fv
        self.on_device = on_device
        self.cap = capacity_cells
        self.d = collections.OrderedDict()
        self.cells = 0
        self.lock = threading.Lock()
        self.building = {}  # key -> Event of the one thread building that mesh

    def _build(self, kind, side):
        return (self.fv.Mesh.square(side, 0.2, 17 + side, on_device=self.on_device) if kind == "2d"
                else self.fv.Mesh.cube(side, 0.15, 17 + side, on_device=self.on_device))

    def get(self, kind, side):
        """The mesh of (kind, side): built by the first thread that asks for it
        (outside the lock); threads asking for the same key meanwhile wait for
        that build instead of building it again, so each mesh is built, counted
        and inserted once."""
        key = (kind, side)
        while True:
            with self.lock:
                if key in self.d:
                    self.d.move_to_end(key)
                    return self.d[key]
                ev = self.building.get(key)
                owner = ev is None
                if owner:
                    ev = threading.Event()
                    self.building[key] = ev
            if not owner:
                ev.wait()
                continue  # built (or its build failed: then this thread tries)
            try:
                m = self._build(kind, side)
                with self.lock:
                    self.d[key] = m
                    self.cells += m.n_cells
                    while self.cells > self.cap and len(self.d) > 1:
                        _, old = self.d.popitem(last=False)
                        self.cells -= old.n_cells
                return m
            finally:
                with self.lock:
                    del self.building[key]
                ev.set()


def request_fields(m, req: Request):
    if req.kind == "2d":
        kf, _, sc = m.fields(req.seed, 1.0, 1.0, source_const=1.0)
        return kf, None, sc
    v = (1.0, 0.5, 0.25)
    kappa0 = float(np.linalg.norm(v)) / req.side / 3.0
    return m.fields(req.seed, kappa0, 0.5, velocity=v, source_uniform=True)


BYTES_PER_CELL = {"2d": 700, "3d": 1100}   # resident estimate: mesh, CSR, factors, FP32 copies, vectors


def solve_wave(fv, cache, reqs: list[Request], stream, tile_rows=1024, outer_tol=1e-10, keep_solution=False,
               precision="mixed", ordering="boxes"):
    """Pack requests of one kind into one batch and solve it on `stream` to
    |b - A x| / |b| <= outer_tol per request: FP32 Krylov inside FP64
    refinement (precision "mixed") or FP64 throughout ("fp64").  ordering
    "boxes": every request's IC(0)/ILU(0) in its own box-colour order (the
    union then has the largest request's level count); None: natural order."""
    import torch
    kind = reqs[0].kind
    with torch.cuda.stream(stream):
        meshes = [cache.get(r.kind, r.side) for r in reqs]
        # per-request fields on host threads (the generator releases the GIL)
        with ThreadPoolExecutor(max_workers=min(8, len(reqs))) as ex:
            fields = list(ex.map(lambda mr: request_fields(*mr), zip(meshes, reqs)))
        kfs, fls, scs = (list(x) for x in zip(*fields))
        mb = MeshBatch(meshes)
        kf = mb.face_field(kfs)
        sc = mb.cell_field(scs)
        nb = mb.n_boundary_faces
        bc = (np.zeros(nb), np.zeros(nb))
        if kind == "2d":
            eq = -fv.laplacian(fv.Orthogonal(), kf) - fv.source(sc)
        else:
            fl = mb.face_field(fls)
            eq = fv.convection(fv.Upwind(fl), fl) - fv.laplacian(fv.Orthogonal(), kf) - fv.source(sc)
        A, b = fv.assemble(eq, bc, mb, stream=stream)
        P = (fv.IncompleteCholesky if kind == "2d" else fv.IncompleteLowerUpper).from_matrix(
            A, 0, stream=stream, ordering=ordering, offsets=mb.cell_offsets if ordering else None)
        x = fv.DistributedVector.from_size(mb.n_cells)
        solver = BatchCG(A, mb.cell_offsets, tile_rows, stream=stream)
        if precision == "mixed":
            out = solver.solve(P, b, x, precision="mixed", outer_tolerance=outer_tol, inner_relative_tolerance=1e-2,
                               max_outer=30, max_iterations=20000, stream=stream,
                               solver="cg" if kind == "2d" else "bicgstab")
        else:
            out = solver.solve(P, b, x, precision="fp64", relative_tolerance=outer_tol,
                               absolute_tolerance=outer_tol, max_iterations=20000, stream=stream,
                               solver="cg" if kind == "2d" else "bicgstab")
        xs = x.data.cpu().numpy() if keep_solution else None
        stream.synchronize()
        for k, r in enumerate(reqs):
            r.iterations = int(out["iterations"][k])
            r.residual = float(out["final_residual"][k])
            if keep_solution:
                r.solution = xs[mb.cell_offsets[k]:mb.cell_offsets[k + 1]].copy()
        # release device objects in this thread (frees are stream ordered per object)
        solver.close()
        P.close()
        A.close()
        del mb
    return out


class Server:
    """solve_fn(fv, cache, wave, stream) solves a wave in place (default: solve_wave);
    it is a parameter so the scheduling can be exercised without a GPU."""

    def __init__(self, fv, workers: int = 2, budget_bytes: int | None = None, max_wave_cells: int = 48_000_000,
                 max_wave_requests: int = 512, solve_fn=None, make_stream=None, wave_order: str = "size",
                 size_ratio: float = 4.0, aging_s: float = 30.0,
                 batch_window_s: float = 0.05):
        if wave_order not in ("size", "fifo"):
            raise ValueError(f"wave_order must be 'size' or 'fifo', not {wave_order!r}")
        self.wave_order = wave_order
        self.size_ratio = float(size_ratio)
        self.aging_s = float(aging_s)
        self.batch_window_s = float(batch_window_s)
        self.fv = fv
        self.cache = MeshCache(fv)
        self.workers = workers
        self.solve_fn = solve_fn or solve_wave
        if make_stream is None:
            import torch
            make_stream = torch.cuda.Stream
        self.make_stream = make_stream
        if budget_bytes is None:
            import torch
            free, total = torch.cuda.mem_get_info()
            budget_bytes = int(free * 0.7)
        self.budget = budget_bytes
        self.peak_reserved = 0
        self.failed = 0
        self.max_wave_cells = max_wave_cells
        self.max_wave_requests = max_wave_requests
        self.lock = threading.Condition()
        self.reserved = 0
        self.admitted = collections.deque()
        self.done = []
        self.waves = 0

    def _cost(self, r: Request) -> int:
        return BYTES_PER_CELL[r.kind] * r.cells

    def _take_wave(self, worker: int, now: float) -> list[Request]:
        """Remove the next wave from self.admitted (caller holds the lock)."""
        q = self.admitted
        if self.wave_order == "fifo" or now - q[0].arrival > self.aging_s:
            kind = q[0].kind
            order = [r for r in q if r.kind == kind]
            fits = lambda r, first: True  # noqa: E731
        elif worker == 0:  # the largest requests, down to size_ratio below the largest
            kind = max(q, key=lambda r: r.cells).kind
            order = sorted((r for r in q if r.kind == kind), key=lambda r: -r.cells)
            fits = lambda r, first: r.cells * self.size_ratio >= first.cells  # noqa: E731
        else:  # the smallest requests, up to size_ratio above the smallest
            kind = min(q, key=lambda r: r.cells).kind
            order = sorted((r for r in q if r.kind == kind), key=lambda r: r.cells)
            fits = lambda r, first: r.cells <= first.cells * self.size_ratio  # noqa: E731
        wave, cells = [], 0
        for r in order:
            if len(wave) == self.max_wave_requests:
                break
            if wave and (cells + r.cells > self.max_wave_cells or not fits(r, wave[0])):
                if self.wave_order == "fifo":
                    continue
                break
            wave.append(r)
            cells += r.cells
        taken = {id(r) for r in wave}
        self.admitted = collections.deque(r for r in q if id(r) not in taken)
        return wave

    def run(self, requests: list[Request], time_limit: float = 120.0, warm: bool = True, drain: bool = True) -> dict:
        """Serve `requests` (arrival times relative to now).  Returns latency and
        throughput statistics over the completed requests.  At time_limit
        admission stops; with drain the workers still solve every admitted
        request, without it they finish their current wave and stop, and the
        requests left (admitted or still to arrive) are the backlog."""
        if warm:  # one small wave of each kind brings the driver and the caches up
            for kind, side in (("2d", 8), ("3d", 3)):
                self.solve_fn(self.fv, self.cache, [Request(-1, 0.0, kind, side, 1, cells=1)], self.make_stream())
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        t0 = time.perf_counter()
        stop = threading.Event()

        def admit_loop():
            while not stop.is_set():
                now = time.perf_counter() - t0
                with self.lock:
                    while pending and pending[0].arrival <= now:
                        r = pending[0]
                        c = self._cost(r)
                        if self.reserved + c > self.budget and self.reserved > 0:
                            break  # admission by free device memory
                        pending.popleft()
                        self.reserved += c
                        self.peak_reserved = max(self.peak_reserved, self.reserved)
                        self.admitted.append(r)
                        self.lock.notify_all()
                    if not pending and not self.admitted:
                        pass
                time.sleep(0.0005)

        def worker(index):
            stream = self.make_stream()
            while True:
                with self.lock:
                    while not stop.is_set():
                        if self.admitted:
                            # a batching window: the oldest request waits up to
                            # batch_window_s for others to join its wave
                            wait = self.admitted[0].arrival + self.batch_window_s - (time.perf_counter() - t0)
                            full = sum(r.cells for r in self.admitted) >= self.max_wave_cells
                            if wait <= 0 or full or not pending:
                                break
                            self.lock.wait(min(wait, 0.01))
                        else:
                            self.lock.wait(0.01)
                    if stop.is_set() and (not drain or not self.admitted):
                        return
                    wave = self._take_wave(index, time.perf_counter() - t0)
                    wid = self.waves
                    self.waves += 1
                start = time.perf_counter() - t0
                for r in wave:
                    r.start = start
                    r.wave = wid
                try:
                    self.solve_fn(self.fv, self.cache, wave, stream)
                except Exception as e:  # a failed wave fails its requests, not the server
                    for r in wave:
                        r.error = f"{type(e).__name__}: {e}"
                        r.residual = float("nan")
                    with self.lock:
                        self.failed += len(wave)
                fin = time.perf_counter() - t0
                with self.lock:
                    for r in wave:
                        r.finish = fin
                        self.reserved -= self._cost(r)
                    self.done.extend(wave)
                    self.lock.notify_all()

        adm = threading.Thread(target=admit_loop, daemon=True)
        ws = [threading.Thread(target=worker, args=(k,), daemon=True) for k in range(self.workers)]
        adm.start()
        for w in ws:
            w.start()
        deadline = t0 + time_limit
        while time.perf_counter() < deadline:
            with self.lock:
                if len(self.done) == len(requests):
                    break
            time.sleep(0.01)
        stop.set()
        with self.lock:
            self.lock.notify_all()
        for w in ws:
            w.join(timeout=max(1.0, deadline - time.perf_counter() + 600))
        wall = time.perf_counter() - t0
        fin = [r for r in self.done if r.finish >= 0 and r.error is None]
        lat = np.array([r.finish - r.arrival for r in fin]) if fin else np.zeros(0)
        span = (max(r.finish for r in fin) - min(r.arrival for r in fin)) if fin else 0.0
        return {
            "completed": len(fin), "offered": len(requests), "failed": self.failed, "waves": self.waves,
            "backlog": len(requests) - len(fin) - self.failed,
            "arrived_by_cap": sum(1 for r in requests if r.arrival <= time_limit),
            "wall_s": wall, "peak_reserved_bytes": self.peak_reserved, "budget_bytes": self.budget,
            "solves_per_s": len(fin) / span if span > 0 else 0.0,
            "p50_ms": float(np.percentile(lat, 50) * 1e3) if len(lat) else None,
            "p99_ms": float(np.percentile(lat, 99) * 1e3) if len(lat) else None,
            "max_residual": float(max((r.residual for r in fin), default=float("nan"))),
            "cells_per_s": float(sum(r.cells for r in fin) / span) if span > 0 else 0.0,
        }
