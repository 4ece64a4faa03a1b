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

Slot refill (Server(refill=True), what the bench serves with): a worker's
wave runs stepwise (fv_batch_begin / fv_batch_advance); a request leaves as
soon as it has finished, and the wave is rebuilt over its running requests
-- which carry their Krylov state over, bit for bit -- plus waiting requests
of its kind (WaveRun), so freed slots are refilled while the others run.

Meshes are built on the device per (kind, size) and cached; the request's
seed drives its diffusivity and source fields.
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
    fields: tuple | None = dataclasses.field(default=None, repr=False, compare=False)  # while in a run


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


def mesh_order(fv, m, stream=None):
    """The box-colour order of mesh m alone and the level of every reordered
    row (fvb200.order_boxes(..., levels=True) on the mesh's pattern), computed
    once and kept on the mesh: a wave merges its requests' orders
    (fvb200.merge_orders) instead of ordering the whole union again."""
    o = getattr(m, "_box_order", None)
    if o is None:
        nb = m.n_boundary_faces
        A, _ = fv.assemble(-fv.laplacian(fv.Orthogonal(), np.ones(m.n_faces)), (np.zeros(nb), np.zeros(nb)), m,
                           stream=stream)
        perm, _, lev = fv.order_boxes(A, levels=True, stream=stream)
        A.close()
        o = (perm, lev)
        m._box_order = o
    return o


def request_fields(m, req: Request):
    if req.kind == "2d":
        kf, _, sc = m.fields(req.seed, 1.0, 1.0, source_const=1.0)
        return kf, None, sc
    v = (1.0, 0.5, 0.25)
    kappa0 = float(np.linalg.norm(v)) / req.side / 3.0
    return m.fields(req.seed, kappa0, 0.5, velocity=v, source_uniform=True)


BYTES_PER_CELL = {"2d": 700, "3d": 1100}   # resident estimate: mesh, CSR, factors, FP32 copies, vectors


def wave_system(fv, cache, reqs: list[Request], stream, ordering="boxes", keep_fields=False):
    """The block-diagonal system of requests of one kind on `stream`: the
    joined mesh, A, b and the IC(0) (2D) / ILU(0) (3D) of A.  ordering "boxes":
    every request's factor in its own box-colour order (the union then has the
    largest request's level count); None: natural order.  Every request's rows
    are the same bits in any wave.  keep_fields: the request's generated fields
    stay on it (r.fields) for the next wave it joins."""
    kind = reqs[0].kind
    meshes = [cache.get(r.kind, r.side) for r in reqs]
    todo = [k for k, r in enumerate(reqs) if r.fields is None]
    if todo:  # per-request fields on host threads (the generator releases the GIL)
        with ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            got = list(ex.map(lambda k: request_fields(meshes[k], reqs[k]), todo))
    else:
        got = []
    fields = [r.fields for r in reqs]
    for k, f in zip(todo, got):
        fields[k] = f
        if keep_fields:
            reqs[k].fields = f
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
    make = fv.IncompleteCholesky if kind == "2d" else fv.IncompleteLowerUpper
    if ordering == "boxes":  # the union's order from the meshes' own (the order fv_order_boxes gives the union)
        perm = fv.merge_orders([mesh_order(fv, m, stream) for m in meshes], mb.cell_offsets)
        P = make.from_matrix(A, 0, stream=stream, ordering=perm)
    else:
        P = make.from_matrix(A, 0, stream=stream, ordering=ordering)
    return mb, A, b, P


def solve_wave(fv, cache, reqs: list[Request], stream, tile_rows=1024, outer_tol=1e-10, keep_solution=False,
               precision="mixed", ordering="boxes"):
    """Pack requests of one kind into one batch and solve it on `stream` to
    |b - A x| / |b| <= outer_tol per request: FP32 Krylov inside FP64
    refinement (precision "mixed") or FP64 throughout ("fp64")."""
    import torch
    kind = reqs[0].kind
    with torch.cuda.stream(stream):
        mb, A, b, P = wave_system(fv, cache, reqs, stream, ordering)
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


class WaveRun:
    """A running wave of requests of one kind, solved stepwise
    (fv_batch_begin / fv_batch_advance).  Built over `reqs`; the requests that
    were running in `prev` continue from their state there (their rows of x and
    of the Krylov vectors and their scalars are carried over bit for bit), the
    others start from x0 = 0.  So a request admitted into a running wave, and
    the requests it joins, give the same result as alone."""

    def __init__(self, fv, cache, reqs: list[Request], stream, prev: "WaveRun | None" = None, tile_rows=1024,
                 outer_tol=1e-10, precision="mixed", ordering="boxes", keep_solution=False):
        import torch
        self.fv, self.stream, self.reqs = fv, stream, list(reqs)
        self.kind = reqs[0].kind
        self.keep_solution = keep_solution
        self.precision = precision
        self.index = {r.rid: k for k, r in enumerate(self.reqs)}
        self.done = np.zeros(len(self.reqs), bool)
        with torch.cuda.stream(stream):
            self.mb, self.A, self.b, self.P = wave_system(fv, cache, self.reqs, stream, ordering, keep_fields=True)
            self.x = fv.DistributedVector.from_size(self.mb.n_cells)
            self.solver = BatchCG(self.A, self.mb.cell_offsets, tile_rows, stream=stream)
            carry = None
            if prev is not None:
                carry = np.array([prev.index.get(r.rid, -1) for r in self.reqs], np.int32)
                for k, q in enumerate(carry):
                    if q >= 0 and prev.done[q]:
                        raise ValueError(f"request {self.reqs[k].rid} has finished in the previous wave")
            common = dict(max_iterations=20000, stream=stream, solver="cg" if self.kind == "2d" else "bicgstab",
                          carry_from=prev.solver if prev is not None else None, carry=carry)
            if precision == "mixed":
                self.solver.begin(self.P, self.b, self.x, precision="mixed", outer_tolerance=outer_tol,
                                  inner_relative_tolerance=1e-2, **common)
            else:
                self.solver.begin(self.P, self.b, self.x, precision="fp64", relative_tolerance=outer_tol,
                                  absolute_tolerance=outer_tol, **common)

    @property
    def cells(self) -> int:
        return int(sum(r.cells for r, d in zip(self.reqs, self.done) if not d))

    def running(self) -> list[Request]:
        return [r for r, d in zip(self.reqs, self.done) if not d]

    def advance(self, iterations: int):
        """Up to `iterations` more iterations.  Returns (finished, stalled): the
        requests that finished (iterations, residual and, with keep_solution,
        the solution recorded on them) and those whose FP32 run stagnated
        (mixed precision; to be solved again in FP64)."""
        running, done = self.solver.advance(iterations, stream=self.stream)
        new = np.flatnonzero(done & ~self.done)
        if len(new) == 0:
            return [], []
        rep = self.solver.report()
        off = self.mb.cell_offsets
        finished, stalled = [], []
        for k in new:
            r = self.reqs[k]
            r.iterations = int(rep["iterations"][k])
            r.residual = float(rep["final_residual"][k])
            r.fields = None
            if rep["status"][k] != 0:
                r.error = f"status {int(rep['status'][k])}"
            if self.keep_solution:
                r.solution = self.x.data[off[k]:off[k + 1]].cpu().numpy()
            (stalled if rep["fp64_fallback"][k] else finished).append(r)
        self.done[new] = True
        return finished, stalled

    def close(self):
        self.solver.close()
        self.P.close()
        self.A.close()
        self.mb = None


class Server:
    """solve_fn(fv, cache, wave, stream) solves a wave in place (default: solve_wave);
    it is a parameter so the scheduling can be exercised without a GPU.

    refill=True serves with slot refill instead of whole waves: a worker runs
    a WaveRun (run_fn(fv, cache, reqs, stream, prev=...), default WaveRun) of
    one kind, advancing it `advance_iterations` iterations at a time; every
    request that finished leaves at once, and when the requests finished since
    the wave was last built hold `refill_fraction` of its cells (or of its
    requests) and admitted requests of the same kind wait, the wave is rebuilt
    over its running requests -- which continue from their state -- plus the
    waiting requests, in arrival order, up to max_wave_cells /
    max_wave_requests.  A wave takes refills for `run_max_s` seconds, then
    drains, so that the other kind is served too; worker k prefers kind
    ("3d", "2d")[k % 2].  A rebuild also waits until the wave has run
    `rebuild_ratio` times as long as its last build took, which bounds the
    share of a worker's time spent rebuilding.  A request whose FP32 run stagnated is solved again
    with fallback_fn (default: solve_wave in FP64)."""

    def __init__(self, fv, workers: int = 2, budget_bytes: int | None = None, max_wave_cells: int = 48_000_000,
                 max_wave_requests: int = 512, solve_fn=None, make_stream=None, wave_order: str = "size",
                 size_ratio: float = 4.0, aging_s: float = 30.0,
                 batch_window_s: float = 0.05, refill: bool = False, run_fn=None, fallback_fn=None,
                 refill_fraction: float = 0.25, advance_iterations: int = 32, run_max_s: float = 10.0,
                 rebuild_ratio: float = 3.0):
        if wave_order not in ("size", "fifo"):
            raise ValueError(f"wave_order must be 'size' or 'fifo', not {wave_order!r}")
        self.refill = bool(refill)
        self.run_fn = run_fn or WaveRun
        if fallback_fn is None:
            def fallback_fn(fv_, cache_, reqs_, stream_):
                return solve_wave(fv_, cache_, reqs_, stream_, precision="fp64")
        self.fallback_fn = fallback_fn
        self.refill_fraction = float(refill_fraction)
        self.advance_iterations = int(advance_iterations)
        self.run_max_s = float(run_max_s)
        self.rebuild_ratio = float(rebuild_ratio)
        self.refills = 0
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

    def _take_first(self, worker: int) -> list[Request]:
        """Refill mode: the first requests of a new wave -- the worker's
        preferred kind if any is admitted, else the other -- in arrival order
        (caller holds the lock)."""
        kinds = {r.kind for r in self.admitted}
        pref = ("3d", "2d")[worker % 2]
        kind = pref if pref in kinds else next(iter(sorted(kinds)))
        return self._take_kind(kind, self.max_wave_cells, self.max_wave_requests)

    def _take_kind(self, kind: str, room_cells: int, room_requests: int) -> list[Request]:
        """Admitted requests of `kind` in arrival order while they fit (caller holds the lock)."""
        out, cells = [], 0
        for r in self.admitted:
            if len(out) == room_requests:
                break
            if r.kind != kind:
                continue
            if out and cells + r.cells > room_cells:
                continue
            if not out and r.cells > room_cells and room_cells < self.max_wave_cells:
                continue  # a refill takes only what fits; a new wave takes its first request whatever its size
            out.append(r)
            cells += r.cells
        taken = {id(r) for r in out}
        self.admitted = collections.deque(r for r in self.admitted if id(r) not in taken)
        return out

    def run(self, requests: list[Request], time_limit: float = 120.0, warm: bool = True, drain: bool = True) -> dict:
        """Serve `requests` (arrival times relative to now).  Returns latency and
        throughput statistics over the completed requests.  At time_limit
        admission stops; with drain the workers still solve every admitted
        request, without it they finish their current wave and stop, and the
        requests left (admitted or still to arrive) are the backlog."""
        if warm:  # one small wave of each kind brings the driver and the caches up
            for kind, side in (("2d", 8), ("3d", 3)):
                w = [Request(-1, 0.0, kind, side, 1, cells=1)]
                if self.refill:
                    wr = self.run_fn(self.fv, self.cache, w, self.make_stream(), prev=None)
                    while wr.running():
                        wr.advance(self.advance_iterations)
                    wr.close()
                else:
                    self.solve_fn(self.fv, self.cache, w, self.make_stream())
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

        def finish(reqs):
            fin = time.perf_counter() - t0
            with self.lock:
                for r in reqs:
                    r.finish = fin
                    self.reserved -= self._cost(r)
                    if r.error is not None:
                        self.failed += 1
                self.done.extend(reqs)
                self.lock.notify_all()

        def worker_refill(index):
            stream = self.make_stream()
            run = None
            built_cells = built_count = freed_cells = freed_count = 0
            run_t0 = built_at = build_s = 0.0
            while True:
                new = []
                with self.lock:
                    if run is None:
                        while not stop.is_set():
                            if self.admitted:
                                wait = self.admitted[0].arrival + self.batch_window_s - (time.perf_counter() - t0)
                                full = sum(r.cells for r in self.admitted) >= self.max_wave_cells
                                if wait <= 0 or full or not pending:
                                    break
                                self.lock.wait(min(wait, 0.01))
                            else:
                                self.lock.wait(0.01)
                        if stop.is_set() and (not drain or not self.admitted):
                            return
                        new = self._take_first(index)
                        run_t0 = time.perf_counter()
                    elif (self.admitted and not stop.is_set() and time.perf_counter() - run_t0 < self.run_max_s
                          and time.perf_counter() - built_at >= self.rebuild_ratio * build_s
                          and (freed_cells >= self.refill_fraction * built_cells
                               or freed_count >= self.refill_fraction * built_count)):
                        new = self._take_kind(run.kind, self.max_wave_cells - run.cells,
                                              self.max_wave_requests - len(run.running()))
                        if new:
                            self.refills += 1
                    if new:
                        wid = self.waves
                        self.waves += 1
                if new:
                    start = time.perf_counter() - t0
                    for r in new:
                        r.start = start
                        r.wave = wid
                    try:
                        tb = time.perf_counter()
                        nxt = self.run_fn(self.fv, self.cache, (run.running() if run is not None else []) + new,
                                          stream, prev=run)
                        built_at = time.perf_counter()
                        build_s = built_at - tb
                    except Exception as e:  # the new requests fail; a running wave carries on
                        for r in new:
                            r.error = f"{type(e).__name__}: {e}"
                            r.residual = float("nan")
                        finish(new)
                        if run is None:
                            continue
                    else:
                        if run is not None:
                            run.close()
                        run = nxt
                        built_cells, built_count = run.cells, len(run.running())
                        freed_cells = freed_count = 0
                try:
                    finished, stalled = run.advance(self.advance_iterations)
                except Exception as e:  # a failed wave fails its running requests, not the server
                    lost = run.running()
                    for r in lost:
                        r.error = f"{type(e).__name__}: {e}"
                        r.residual = float("nan")
                    finish(lost)
                    try:
                        run.close()
                    finally:
                        run = None
                    continue
                for r in stalled:  # the FP32 run stagnated: FP64 from x0 = 0
                    try:
                        r.error = None
                        self.fallback_fn(self.fv, self.cache, [r], stream)
                    except Exception as e:
                        r.error = f"{type(e).__name__}: {e}"
                        r.residual = float("nan")
                out = finished + stalled
                if out:
                    freed_cells += sum(r.cells for r in out)
                    freed_count += len(out)
                    finish(out)
                if not run.running():
                    run.close()
                    run = None

        adm = threading.Thread(target=admit_loop, daemon=True)
        ws = [threading.Thread(target=worker_refill if self.refill else worker, args=(k,), daemon=True)
              for k in range(self.workers)]
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
            "refills": self.refills,
            "backlog": len(requests) - len(fin) - self.failed,
            "arrived_by_cap": sum(1 for r in requests if r.arrival <= time_limit),
            "wall_s": wall, "peak_reserved_bytes": self.peak_reserved, "budget_bytes": self.budget,
            "solves_per_s": len(fin) / span if span > 0 else 0.0,
            "p50_ms": float(np.percentile(lat, 50) * 1e3) if len(lat) else None,
            "p99_ms": float(np.percentile(lat, 99) * 1e3) if len(lat) else None,
            "max_residual": float(max((r.residual for r in fin), default=float("nan"))),
            "cells_per_s": float(sum(r.cells for r in fin) / span) if span > 0 else 0.0,
        }
