"""One problem split over several ranks (one GPU each): the reference's MPI design.

The crate runs one MPI rank per partition of the mesh
(src/core/mesh/decompose.rs).  A rank owns a set of cells/rows; its matrix has
a column for each owned cell followed by ghost columns for the cells of other
ranks that share a face with an owned cell.  Two communication steps keep the
ranks consistent (src/core/communicator.rs):

  collect ...... refresh the ghost values before an SpMV      (:226-266)
  reduce_add ... sum a local dot product over the ranks         (:282-290)

and the preconditioners factorise only the square block of owned columns
(DistributedMatrix::square_block, src/linalg/dmatrix.rs:214-229), i.e. block
Jacobi across ranks.

Here the rows are split into contiguous ranges of the global numbering
(METIS, which the reference uses through core/mesh/decompose.rs:32, is not
available; contiguous ranges of the generators' lexicographic numbering are
slabs of the domain).  `HaloPlan` computes, for one rank, the local matrix in
local numbering (owned columns first, ghost columns after them, sorted by
global id), the ghost list and the send list.  `Communicator` carries out
collect / reduce_add over a torch.distributed process group (NCCL with device
tensors, gloo with host tensors) and hands both to the library as the C
callbacks of `fv_comm`, so the Krylov loops of libfvb200 (fv_dist_cg,
fv_dist_bicgstab) call them in the reference's places.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import COLLECT_FN, REDUCE_FN, FvComm, FvError, SolverInfo, check, exiting, lib
from .linalg import DistributedMatrix, LinearSolverInfo, LinearSolverOptions, _dev_f64
from .streams import stream_handle


def contiguous_partition(n: int, world: int) -> np.ndarray:
    """Row bounds of `world` contiguous parts: part t owns [n t / P, n (t+1) / P)."""
    return np.array([(n * t) // world for t in range(world + 1)], dtype=np.int64)


@dataclass
class HaloPlan:
    """What one rank needs to run its part of a distributed solve.

    ghosts[k]       global id of ghost column n_own + k (ascending)
    recv_counts[q]  how many ghosts rank q owns (ghosts are grouped by owner,
                    since the parts are contiguous and ghosts are sorted)
    send_idx        local rows whose values other ranks need, grouped by the
                    receiving rank in rank order, ascending within a group
    send_counts[q]  how many of them go to rank q
    row_ptr, cols, vals: the rank's matrix in local numbering; each row sorted
                    by local column (owned columns, then ghost columns)
    """
    rank: int
    world: int
    lo: int
    hi: int
    ghosts: np.ndarray
    recv_counts: np.ndarray
    send_idx: np.ndarray
    send_counts: np.ndarray
    row_ptr: np.ndarray
    cols: np.ndarray
    vals: np.ndarray | None

    @property
    def n_own(self) -> int:
        return self.hi - self.lo

    @property
    def n_ghost(self) -> int:
        return len(self.ghosts)

    @property
    def recv_displs(self) -> np.ndarray:
        return np.concatenate([[0], np.cumsum(self.recv_counts)]).astype(np.int64)

    @property
    def send_displs(self) -> np.ndarray:
        return np.concatenate([[0], np.cumsum(self.send_counts)]).astype(np.int64)

    @classmethod
    def from_global(cls, row_ptr, cols, vals, bounds, rank: int) -> "HaloPlan":
        """Plan of `rank` from the global CSR (pattern and optionally values).
        Every rank can build its own plan from the global pattern; the send
        list of rank r is the set of r's rows that appear as ghost columns in
        the other ranks' rows."""
        row_ptr = np.asarray(row_ptr, dtype=np.int64)
        cols = np.asarray(cols, dtype=np.int64)
        bounds = np.asarray(bounds, dtype=np.int64)
        world = len(bounds) - 1
        lo, hi = int(bounds[rank]), int(bounds[rank + 1])
        a0, a1 = int(row_ptr[lo]), int(row_ptr[hi])
        lc = cols[a0:a1]
        owned = (lc >= lo) & (lc < hi)
        ghosts = np.unique(lc[~owned])
        owner_of_ghost = np.searchsorted(bounds, ghosts, side="right") - 1
        recv_counts = np.bincount(owner_of_ghost, minlength=world).astype(np.int64)
        # local column ids: owned -> c - lo, ghost -> n_own + position in ghosts
        local = np.empty_like(lc)
        local[owned] = lc[owned] - lo
        local[~owned] = (hi - lo) + np.searchsorted(ghosts, lc[~owned])
        lptr = (row_ptr[lo:hi + 1] - a0).astype(np.int64)
        # sort every row by local column (a stable sort on (row, local col))
        row_of = np.repeat(np.arange(hi - lo), np.diff(lptr))
        order = np.lexsort((local, row_of))
        lcols = local[order].astype(np.int32)
        lvals = None if vals is None else np.asarray(vals, dtype=np.float64)[a0:a1][order]
        # send list: for every other rank q (ascending), the rows of this rank
        # that q's rows reference, ascending
        send, counts = [], np.zeros(world, np.int64)
        for q in range(world):
            if q == rank:
                continue
            q0, q1 = int(bounds[q]), int(bounds[q + 1])
            qc = cols[row_ptr[q0]:row_ptr[q1]]
            need = np.unique(qc[(qc >= lo) & (qc < hi)])
            send.append(need - lo)
            counts[q] = len(need)
        send_idx = np.concatenate(send).astype(np.int32) if send else np.zeros(0, np.int32)
        return cls(rank, world, lo, hi, ghosts.astype(np.int64), recv_counts, send_idx, counts,
                   lptr.astype(np.int32), lcols, lvals)


def _cuda_tensor(ptr: int, n: int):
    """Zero-copy float64 CUDA tensor over a device pointer (no ownership)."""
    import torch

    class _View:
        __cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (int(ptr), False), "version": 3,
                                    "strides": None}
    return torch.as_tensor(_View(), device="cuda")


def _stream(ptr):
    import torch
    return torch.cuda.ExternalStream(int(ptr)) if ptr else torch.cuda.default_stream()


class Communicator:
    """collect / reduce_add over a torch.distributed process group
    (core/communicator.rs:226-290).  Works on device tensors with NCCL and on
    host tensors with gloo; ranks must call in the same order."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)

    def collect(self, plan: HaloPlan, send, ghost) -> None:
        """ghost[...] = the owners' values of this rank's ghost columns;
        send = this rank's packed values (plan.send_idx order)."""
        dist = self.dist
        ops = []
        sd, rd = plan.send_displs, plan.recv_displs
        for q in range(self.size):
            if q == self.rank:
                continue
            if plan.send_counts[q]:
                ops.append(dist.P2POp(dist.isend, send[sd[q]:sd[q + 1]], q, self.group))
            if plan.recv_counts[q]:
                ops.append(dist.P2POp(dist.irecv, ghost[rd[q]:rd[q + 1]], q, self.group))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()

    def reduce_add(self, buf) -> None:
        self.dist.all_reduce(buf, op=self.dist.ReduceOp.SUM, group=self.group)

    def fv_comm(self, plan: HaloPlan) -> FvComm:
        """The fv_comm callbacks for the library (device buffers, NCCL)."""
        import torch

        def collect(ctx, send, ghost, stream):  # noqa: ARG001
            try:
                with torch.cuda.stream(_stream(stream)):
                    self.collect(plan, _cuda_tensor(send or 0, len(plan.send_idx)),
                                 _cuda_tensor(ghost or 0, plan.n_ghost))
                return 0
            except Exception:  # reported to the caller as FV_ERR_COMM
                return 1

        def reduce_add(ctx, buf, count, stream):
            try:
                with torch.cuda.stream(_stream(stream)):
                    self.reduce_add(_cuda_tensor(buf, count))
                return 0
            except Exception:
                return 1

        return make_fv_comm(collect, reduce_add)


def make_fv_comm(collect, reduce_add) -> FvComm:
    """fv_comm from two Python callables (ctx, send, ghost, stream) -> int and
    (ctx, buf, count, stream) -> int.  Keep the returned object alive while
    the library may call it."""
    c = FvComm(None, COLLECT_FN(collect), REDUCE_FN(reduce_add))
    c._keep = (c.collect, c.reduce_add)
    return c


class RankSystem:
    """This rank's share of a distributed linear system: the local matrix with
    ghost columns, its square block, and the halo/reduction plumbing."""

    def __init__(self, plan: HaloPlan, comm: FvComm | None, stream=None):
        if plan.vals is None:
            raise ValueError("the plan carries no matrix values")
        self.plan = plan
        self.matrix = DistributedMatrix.from_csr(plan.row_ptr, plan.cols, plan.vals,
                                                 ncols=plan.n_own + plan.n_ghost, stream=stream)
        self._comm = comm
        self.handle = C.c_void_p()
        sidx = np.ascontiguousarray(plan.send_idx, dtype=np.int32)
        check(lib().fv_dist_create(self.matrix.handle, plan.n_ghost, sidx.ctypes.data_as(C.POINTER(C.c_int32)),
                                   len(sidx), C.byref(comm) if comm is not None else None, C.byref(self.handle)),
              "fv_dist_create")

    def square_block(self, stream=None) -> DistributedMatrix:
        """DistributedMatrix::square_block (dmatrix.rs:214-229)."""
        h = C.c_void_p()
        check(lib().fv_csr_square_block(self.matrix.handle, stream_handle(stream), C.byref(h)), "square_block")
        return DistributedMatrix(h)

    def spmv(self, y, x_with_ghosts, stream=None) -> None:
        check(lib().fv_dist_spmv(self.handle, C.c_void_p(x_with_ghosts.data_ptr()), C.c_void_p(y.data_ptr()),
                                 stream_handle(stream)), "fv_dist_spmv")

    def dot(self, x, y, stream=None) -> float:
        out = C.c_double()
        check(lib().fv_dist_dot(self.handle, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), C.byref(out),
                                stream_handle(stream)), "fv_dist_dot")
        return out.value

    def solve(self, solver: str, solution, rhs, preconditioner=None, options: LinearSolverOptions | None = None,
              stream=None) -> LinearSolverInfo:
        """conjugate_gradient / bi_conjugate_gradient_stab on all ranks together."""
        fn, name = ((lib().fv_dist_cg, "ConjugateGradient") if solver == "cg"
                    else (lib().fv_dist_bicgstab, "BiConjugateGradientStab"))
        options = options or LinearSolverOptions()
        cap = int(options.max_iterations) + 2
        hist = np.zeros(cap, np.float64)
        info = SolverInfo()
        info.history = hist.ctypes.data_as(C.POINTER(C.c_double))
        info.history_cap = cap
        b = _dev_f64(rhs)
        ph = preconditioner.handle if preconditioner is not None else C.c_void_p()
        st = fn(self.handle, ph, C.c_void_p(b.data_ptr()), solution.ptr(), options.c(), C.byref(info),
                stream_handle(stream))
        if st not in (0, 4):
            raise FvError(st, name)
        return LinearSolverInfo(name, int(info.iterations), float(info.initial_residual),
                                float(info.final_residual), hist[: min(int(info.history_len), cap)].tolist(),
                                int(info.status), int(info.restarts), float(info.device_ms))

    def close(self):
        if self.handle:
            lib().fv_dist_destroy(self.handle)
            self.handle = C.c_void_p()
        self.matrix.close()

    def __del__(self):
        try:
            if exiting():  # module globals may already be gone at interpreter teardown
                return
            self.close()
        except Exception:
            pass
