"""Batched solves: many independent meshes as one block-diagonal system.

MeshBatch concatenates host meshes into one mesh whose faces are ordered
interior faces of every problem first, then the boundary faces of every
problem (each problem keeps its own relative face order, so every cell sees
its faces in the same order as alone).  assemble() on a MeshBatch therefore
yields exactly the per-problem matrices on the diagonal, IC(0) of the union is
the per-problem IC(0), and BatchCG solves all problems at once with
per-problem scalars (fv_batch_cg).
"""
from __future__ import annotations

import ctypes as C
import functools
import time

import numpy as np

from ._lib import BatchInfo, BatchOptions, check, exiting, lib
from .streams import stream_handle

FV_BATCH_FP64, FV_BATCH_MIXED = 0, 1


class MeshBatch:
    def __init__(self, meshes):
        assert meshes and len({m.dim for m in meshes}) == 1
        self.meshes = list(meshes)
        self.dim = meshes[0].dim
        self.n_problems = len(meshes)
        nc = np.array([m.n_cells for m in meshes], np.int64)
        fi = np.array([m.n_faces - m.n_boundary_faces for m in meshes], np.int64)
        fb = np.array([m.n_boundary_faces for m in meshes], np.int64)
        self.cell_offsets = np.concatenate([[0], np.cumsum(nc)])
        self.int_offsets = np.concatenate([[0], np.cumsum(fi)])
        self.bnd_offsets = np.concatenate([[0], np.cumsum(fb)])
        self.n_cells = int(self.cell_offsets[-1])
        self.n_boundary_faces = int(self.bnd_offsets[-1])
        self.n_faces = int(self.int_offsets[-1]) + self.n_boundary_faces
        self._fi, self._fb = fi, fb
        self._device = {}

    # union arrays on the host, built on first use (a union whose parts are
    # resident on the GPU is joined there by fv_mesh_concat without them)
    @functools.cached_property
    def face_owner(self):
        co, fi = self.cell_offsets, self._fi
        own_i = [m.face_owner[: fi[p]].astype(np.int64) + co[p] for p, m in enumerate(self.meshes)]
        own_b = [m.face_owner[fi[p]:].astype(np.int64) + co[p] for p, m in enumerate(self.meshes)]
        return np.concatenate(own_i + own_b).astype(np.int32)

    @functools.cached_property
    def face_neighbor(self):
        co, fi, fb = self.cell_offsets, self._fi, self._fb
        nb_i = [m.face_neighbor[: fi[p]].astype(np.int64) + co[p] for p, m in enumerate(self.meshes)]
        return np.concatenate(nb_i + [np.full(fb[p], -1, np.int64) for p in range(self.n_problems)]).astype(np.int32)

    @functools.cached_property
    def face_area(self):
        return self.face_field([m.face_area for m in self.meshes])

    @functools.cached_property
    def face_center(self):
        return self.face_field([m.face_center for m in self.meshes])

    @functools.cached_property
    def cell_center(self):
        return np.ascontiguousarray(np.concatenate([m.cell_center for m in self.meshes]))

    @functools.cached_property
    def cell_volume(self):
        return np.ascontiguousarray(np.concatenate([m.cell_volume for m in self.meshes]))

    def face_field(self, per_problem):
        """Concatenate per-problem face arrays into the union face order."""
        fi = [m.n_faces - m.n_boundary_faces for m in self.meshes]
        parts = [a[: fi[p]] for p, a in enumerate(per_problem)] + [a[fi[p]:] for p, a in enumerate(per_problem)]
        return np.ascontiguousarray(np.concatenate(parts))

    def boundary_field(self, per_problem):
        """Concatenate per-problem boundary-face arrays (bndi, bnde)."""
        return np.ascontiguousarray(np.concatenate(per_problem))

    def cell_field(self, per_problem):
        return np.ascontiguousarray(np.concatenate(per_problem))

    def device(self, stream=None):
        import torch

        from .mesh import DeviceMesh
        dev = torch.cuda.current_device()
        if dev not in self._device:
            parts = [getattr(m, "_device", {}).get(dev) for m in self.meshes]
            if all(p is not None and p.handle for p in parts):  # every part resident: join on the device
                arr = (C.c_void_p * len(parts))(*[p.handle.value for p in parts])
                h = C.c_void_p()
                check(lib().fv_mesh_concat(arr, len(parts), stream_handle(stream), C.byref(h)), "fv_mesh_concat")
                self._device[dev] = DeviceMesh.adopt(self, h)
            else:
                self._device[dev] = DeviceMesh(self, stream)
        return self._device[dev]

    def __del__(self):
        try:
            if exiting():  # module globals may already be gone at interpreter teardown
                return
            for dm in self._device.values():
                dm.close()
        except Exception:
            pass


class BatchCG:
    """fv_batch handle over a block-diagonal matrix with row_offsets per problem
    (solve(..., solver="cg"|"bicgstab"))."""

    def __init__(self, A, row_offsets, tile_rows: int = 0, stream=None):
        self.A = A
        self.row_offsets = np.ascontiguousarray(row_offsets, dtype=np.int64)
        self.n_problems = len(self.row_offsets) - 1
        self.tile_rows = tile_rows
        self.handle = C.c_void_p()
        check(lib().fv_batch_create(A.handle, self.n_problems, self.row_offsets.ctypes.data_as(C.POINTER(C.c_int64)),
                                    tile_rows, stream_handle(stream), C.byref(self.handle)), "fv_batch_create")

    @staticmethod
    def _options(precision, relative_tolerance, absolute_tolerance, max_iterations, inner_relative_tolerance,
                 outer_tolerance, max_outer):
        if precision not in ("mixed", "fp64"):
            raise ValueError(f"precision must be 'mixed' or 'fp64', not {precision!r}")
        return BatchOptions(FV_BATCH_MIXED if precision == "mixed" else FV_BATCH_FP64, relative_tolerance,
                            absolute_tolerance, max_iterations, inner_relative_tolerance, outer_tolerance, max_outer)

    def _info(self):
        n = self.n_problems
        arrs = dict(iterations=np.zeros(n, np.int64), outer_steps=np.zeros(n, np.int32), final_residual=np.zeros(n),
                    status=np.zeros(n, np.int32), fp64_fallback=np.zeros(n, np.int32))
        info = BatchInfo(0.0, 0, arrs["iterations"].ctypes.data_as(C.POINTER(C.c_int64)),
                         arrs["outer_steps"].ctypes.data_as(C.POINTER(C.c_int32)),
                         arrs["final_residual"].ctypes.data_as(C.POINTER(C.c_double)),
                         arrs["status"].ctypes.data_as(C.POINTER(C.c_int32)),
                         arrs["fp64_fallback"].ctypes.data_as(C.POINTER(C.c_int32)))
        return info, arrs

    def solve(self, P, b, x, precision: str = "mixed", relative_tolerance=1e-8, absolute_tolerance=1e-8,
              max_iterations=10000, inner_relative_tolerance=1e-2, outer_tolerance=1e-10, max_outer=30,
              stream=None, solver: str = "cg"):
        if solver not in ("cg", "bicgstab"):
            raise ValueError(f"solver must be 'cg' or 'bicgstab', not {solver!r}")
        o = self._options(precision, relative_tolerance, absolute_tolerance, max_iterations,
                          inner_relative_tolerance, outer_tolerance, max_outer)
        info, arrs = self._info()
        fn = lib().fv_batch_bicgstab if solver == "bicgstab" else lib().fv_batch_cg
        check(fn(self.handle, P.handle, C.c_void_p(b.data.data_ptr()), C.c_void_p(x.data.data_ptr()), C.byref(o),
                 C.byref(info), stream_handle(stream)), "fv_batch_" + solver)
        return dict(arrs, device_ms=info.device_ms, launched_iterations=info.launched_iterations)

    # ---- stepwise runs (continuous batching): fv_batch_begin / _advance / _report
    def begin(self, P, b, x, precision: str = "mixed", relative_tolerance=1e-8, absolute_tolerance=1e-8,
              max_iterations=10000, inner_relative_tolerance=1e-2, outer_tolerance=1e-10, stream=None,
              solver: str = "cg", carry_from: "BatchCG | None" = None, carry=None):
        """Start a run.  carry[p] = q >= 0 continues problem q of the running
        batch `carry_from` as problem p (its state copied bit for bit); -1
        starts p from x0 = 0.  P, b and x must stay alive for the whole run."""
        if solver not in ("cg", "bicgstab"):
            raise ValueError(f"solver must be 'cg' or 'bicgstab', not {solver!r}")
        o = self._options(precision, relative_tolerance, absolute_tolerance, max_iterations,
                          inner_relative_tolerance, outer_tolerance, 0)
        cmap = None
        if carry is not None:
            cmap = np.ascontiguousarray(carry, dtype=np.int32)
            if cmap.shape != (self.n_problems,) or carry_from is None:
                raise ValueError("carry needs one entry per problem and carry_from")
        method = 1 if solver == "bicgstab" else 0
        check(lib().fv_batch_begin(self.handle, P.handle, method, C.c_void_p(b.data.data_ptr()),
                                   C.c_void_p(x.data.data_ptr()), C.byref(o),
                                   carry_from.handle if carry_from is not None else None,
                                   cmap.ctypes.data_as(C.POINTER(C.c_int32)) if cmap is not None else None,
                                   stream_handle(stream)), "fv_batch_begin")
        self._run = (P, b, x)  # keep the run's operands alive

    def advance(self, max_iterations: int, stream=None):
        """Up to max_iterations more iterations; returns (running count, done flags)."""
        done = np.zeros(self.n_problems, np.int32)
        running = C.c_int32(0)
        check(lib().fv_batch_advance(self.handle, int(max_iterations), C.byref(running),
                                     done.ctypes.data_as(C.POINTER(C.c_int32)), stream_handle(stream)),
              "fv_batch_advance")
        return int(running.value), done.astype(bool)

    def report(self):
        """Per-problem iterations / residuals / status of the current run
        (fp64_fallback: the FP32 run stagnated and left the problem unfinished)."""
        info, arrs = self._info()
        check(lib().fv_batch_report(self.handle, C.byref(info)), "fv_batch_report")
        return dict(arrs, launched_iterations=info.launched_iterations)

    def close(self):
        if self.handle:
            lib().fv_batch_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            if exiting():  # module globals may already be gone at interpreter teardown
                return
            self.close()
        except Exception:
            pass


def autotune_tile(A, row_offsets, P, b, x, candidates=(256, 512, 1024, 2048), iters=10):
    """Pick the tile size (rows per problem-aligned reduction tile) that runs a
    fixed number of FP64 CG iterations fastest on this batch."""
    import torch
    best, best_t = None, float("inf")
    timings = {}
    for tile in candidates:
        bc = BatchCG(A, row_offsets, tile)
        bc.solve(P, b, x, precision="fp64", relative_tolerance=0.0, absolute_tolerance=0.0, max_iterations=2)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        bc.solve(P, b, x, precision="fp64", relative_tolerance=0.0, absolute_tolerance=0.0, max_iterations=iters)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        timings[tile] = dt
        bc.close()
        if dt < best_t:
            best, best_t = tile, dt
    return best, timings


def autotune_schedule(P, b, x, candidates=(1, 3), reps=3, stream=None):
    """Pick the faster sweep schedule for this preconditioner (level chunks, or
    level chunks with the next chunk prefetched: the same bits either way) by
    timing a few applies of each; returns (chosen, {schedule: ms per apply})."""
    import torch
    times = {}
    for sch in candidates:
        P.schedule(sch)
        P.precondition(x, b, stream=stream)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        torch.cuda.synchronize()
        ev[0].record()
        for _ in range(reps):
            P.precondition(x, b, stream=stream)
        ev[1].record()
        torch.cuda.synchronize()
        times[sch] = ev[0].elapsed_time(ev[1]) / reps
    best = min(times, key=times.get)
    P.schedule(best)
    return best, times
