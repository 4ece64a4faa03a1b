"""DistributedMatrix / DistributedVector, assemble(), the preconditioners and
the Krylov solvers, mirroring the reference crate's Rust API on the device.

  assemble ................... src/fvm/assembly.rs:11
  DistributedMatrix::imul .... src/linalg/dmatrix.rs:136
  IncompleteCholesky ......... src/linalg/preconditioners/incomplete_cholesky.rs:205
  IncompleteLowerUpper ....... src/linalg/preconditioners/incomplete_lower_upper.rs:266
  conjugate_gradient ......... src/linalg/solvers/conjugate_gradient.rs:12
  bi_conjugate_gradient_stab . src/linalg/solvers/bi_conjugate_gradient_stab.rs:13
  LinearSolverOptions/Info ... src/linalg/solvers/mod.rs:11-42

Error behaviour: where the reference panics (missing matrix entry, ILU pivot
below 1e-16, IC on a non-symmetric matrix) these raise FvError; solvers
return a LinearSolverInfo and never raise for non-convergence.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from ._lib import BcDesc, FvError, OrderInfo, SolverInfo, SolverOptions, TermsDesc, check, exiting, lib
from .streams import stream_handle


def _torch():
    import torch
    return torch


def _dev_f64(a):
    """Device float64 tensor for an array-like (numpy / torch / DistributedVector)."""
    torch = _torch()
    if isinstance(a, DistributedVector):
        return a.data
    if isinstance(a, torch.Tensor):
        t = a.to(device="cuda", dtype=torch.float64)
        return t.contiguous()
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


class DistributedVector:
    """Dense FP64 vector resident on the GPU (torch tensor)."""

    def __init__(self, data):
        self.data = _dev_f64(data)

    @classmethod
    def from_size(cls, n: int) -> "DistributedVector":
        torch = _torch()
        return cls(torch.zeros(n, dtype=torch.float64, device="cuda"))

    @classmethod
    def from_data(cls, data) -> "DistributedVector":
        return cls(data)

    def __len__(self):
        return int(self.data.numel())

    def len(self):
        return len(self)

    def numpy(self) -> np.ndarray:
        return self.data.detach().cpu().numpy()

    # DistributedVector operations (linalg/dvector.rs:46-160) on the device
    def dot(self, rhs: "DistributedVector", stream=None) -> float:
        if len(self) != len(rhs):
            raise ValueError("dot: lengths differ (the reference asserts)")
        return self.dot_smaller(rhs, stream)

    def dot_smaller(self, rhs: "DistributedVector", stream=None) -> float:
        out = C.c_double()
        check(lib().fv_vec_dot(min(len(self), len(rhs)), self.ptr(), rhs.ptr(), stream_handle(stream),
                               C.byref(out)), "dot")
        return out.value

    def sum(self, stream=None) -> float:
        out = C.c_double()
        check(lib().fv_vec_sum(len(self), self.ptr(), stream_handle(stream), C.byref(out)), "sum")
        return out.value

    def _update(self, other, a, op, n=None, stream=None):
        x = other.ptr() if other is not None else None
        check(lib().fv_vec_update(len(self) if n is None else n, self.ptr(), x, float(a), op,
                                  stream_handle(stream)), "vector update")
        return self

    def __iadd__(self, rhs: "DistributedVector"):
        if len(self) != len(rhs):
            raise ValueError("+=: lengths differ")
        return self._update(rhs, 0.0, 0)

    def __isub__(self, rhs: "DistributedVector"):
        if len(self) != len(rhs):
            raise ValueError("-=: lengths differ")
        return self._update(rhs, 0.0, 1)

    def __imul__(self, a: float):
        return self._update(None, a, 2)

    def inv(self) -> "DistributedVector":
        return self._update(None, 0.0, 3)

    def set(self, rhs: "DistributedVector"):
        if len(rhs) < len(self):
            raise ValueError("set: source shorter than the vector")
        return self._update(rhs, 0.0, 4)

    def set_smaller(self, rhs: "DistributedVector"):
        return self._update(rhs, 0.0, 4, n=min(len(self), len(rhs)))

    def __getitem__(self, i):
        return float(self.data[i].item())

    def __setitem__(self, i, v):
        self.data[i] = float(v)

    def ptr(self) -> C.c_void_p:
        return C.c_void_p(self.data.data_ptr())


class DistributedMatrix:
    """CSR matrix on the GPU (fv_csr handle), FP64 values, int32 indices."""

    def __init__(self, handle: C.c_void_p, keepalive=None):
        self.handle = handle
        self._keep = keepalive

    @classmethod
    def from_csr(cls, row_ptr, cols, vals, ncols=None, stream=None) -> "DistributedMatrix":
        rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
        cc = np.ascontiguousarray(cols, dtype=np.int32)
        vv = np.ascontiguousarray(vals, dtype=np.float64)
        n = len(rp) - 1
        h = C.c_void_p()
        check(lib().fv_csr_create_host(n, n if ncols is None else ncols, rp.ctypes.data_as(C.POINTER(C.c_int32)),
                                       cc.ctypes.data_as(C.POINTER(C.c_int32)),
                                       vv.ctypes.data_as(C.POINTER(C.c_double)), stream_handle(stream),
                                       C.byref(h)), "DistributedMatrix.from_csr")
        return cls(h)

    def shape(self):
        nr, nc, nz = C.c_int64(), C.c_int64(), C.c_int64()
        check(lib().fv_csr_info(self.handle, C.byref(nr), C.byref(nc), C.byref(nz)), "fv_csr_info")
        return nr.value, nc.value, nz.value

    def nrows(self):
        return self.shape()[0]

    def ncols(self):
        return self.shape()[1]

    def nnz(self):
        return self.shape()[2]

    def to_csr(self, stream=None):
        """(row_ptr, cols, vals) as numpy arrays."""
        n, _, nz = self.shape()
        rp = np.empty(n + 1, np.int32)
        cc = np.empty(max(nz, 1), np.int32)
        vv = np.empty(max(nz, 1), np.float64)
        check(lib().fv_csr_download(self.handle, rp.ctypes.data_as(C.POINTER(C.c_int32)),
                                    cc.ctypes.data_as(C.POINTER(C.c_int32)),
                                    vv.ctypes.data_as(C.POINTER(C.c_double)), stream_handle(stream)),
              "fv_csr_download")
        return rp, cc[:nz], vv[:nz]

    def imul(self, result: DistributedVector, rhs, stream=None) -> None:
        """result = self * rhs (dmatrix.rs:136-146), bit-exact per row."""
        x = _dev_f64(rhs)
        check(lib().fv_spmv(self.handle, C.c_void_p(x.data_ptr()), result.ptr(), stream_handle(stream)), "fv_spmv")

    def permuted(self, perm, stream=None) -> "DistributedMatrix":
        """Q A Q^T (fv_csr_permute): row i is this matrix's row perm[i], columns
        renumbered the same way.  The copy keeps this matrix alive and takes its
        current values again with refresh_permuted()."""
        p = np.ascontiguousarray(perm, np.int32)
        if p.shape != (self.nrows(),):
            raise ValueError("perm needs one entry per row")
        h = C.c_void_p()
        check(lib().fv_csr_permute(self.handle, p.ctypes.data_as(C.POINTER(C.c_int32)), stream_handle(stream),
                                   C.byref(h)), "fv_csr_permute")
        B = DistributedMatrix(h, keepalive=self)
        B.perm = p
        return B

    def refresh_permuted(self, stream=None) -> None:
        """A permuted copy takes the current values of the matrix it was made from."""
        check(lib().fv_csr_permute_values(self.handle, stream_handle(stream)), "fv_csr_permute_values")

    def to_permuted(self, x, out: "DistributedVector", stream=None) -> None:
        """out[i] = x[perm[i]]: a vector of the source numbering in this permuted copy's numbering."""
        xs = _dev_f64(x)
        check(lib().fv_vec_permute(self.handle, C.c_void_p(xs.data_ptr()), out.ptr(), 0, stream_handle(stream)),
              "fv_vec_permute")

    def from_permuted(self, y, out: "DistributedVector", stream=None) -> None:
        """out[perm[i]] = y[i]: back to the source numbering."""
        ys = _dev_f64(y)
        check(lib().fv_vec_permute(self.handle, C.c_void_p(ys.data_ptr()), out.ptr(), 1, stream_handle(stream)),
              "fv_vec_permute")

    def close(self):
        if self.handle:
            lib().fv_csr_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            if exiting():  # module globals may already be gone at interpreter teardown
                return
            self.close()
        except Exception:
            pass


def _bc_arrays(boundary_condition, mesh):
    """(bndi, bnde) over the boundary faces from a FaceConstraints, a callable
    face id -> (bndi, bnde), or the pair of arrays itself."""
    if hasattr(boundary_condition, "as_bc"):
        return boundary_condition.as_bc()
    if callable(boundary_condition):
        nb = mesh.n_boundary_faces
        fb0 = mesh.n_faces - nb
        pairs = [boundary_condition(fb0 + k) for k in range(nb)]
        return (np.array([p[0] for p in pairs], dtype=np.float64),
                np.array([p[1] for p in pairs], dtype=np.float64))
    return boundary_condition


def assemble(equation, boundary_condition, mesh, lhs: DistributedMatrix | None = None, stream=None):
    """assemble(equation, boundary_condition, mesh) -> (DistributedMatrix, DistributedVector).

    boundary_condition: a FaceConstraints, a callable face_id -> (bndi, bnde)
    as in the reference (evaluated once per boundary face on the host), or a
    pair of arrays (bndi, bnde) over the boundary faces.  Passing `lhs` from an earlier call
    on the same mesh refills its values in place (value-only re-assembly).
    """
    dm, t, bc, keep = _assembly_descriptors(equation, boundary_condition, mesh, stream)
    rhs = DistributedVector.from_size(mesh.n_cells)
    h = lhs.handle if lhs is not None else C.c_void_p()
    check(lib().fv_assemble(dm.handle, C.byref(t), C.byref(bc), C.byref(h), rhs.ptr(), stream_handle(stream)),
          "assemble")
    # torch's caching allocator is stream ordered: the temporaries in `keep`
    # are not reused before the assembly kernel has consumed them
    del keep
    if lhs is None:
        lhs = DistributedMatrix(h, keepalive=dm)
    return lhs, rhs


def assembly_launcher(equation, boundary_condition, mesh, lhs: DistributedMatrix, rhs: DistributedVector,
                      stream=None):
    """A zero-argument callable that re-assembles `equation` into `lhs` and
    `rhs` (value-only, resident pattern) with one fv_assemble call: the term
    descriptors are built once, so each call is the C call alone (for timing
    the assembly kernel)."""
    dm, t, bc, keep = _assembly_descriptors(equation, boundary_condition, mesh, stream)
    h = lhs.handle
    sh = stream_handle(stream)

    def run():
        check(lib().fv_assemble(dm.handle, C.byref(t), C.byref(bc), C.byref(h), rhs.ptr(), sh), "assemble")

    run.keep = keep  # the descriptors' device arrays live as long as the callable
    return run


def _assembly_descriptors(equation, boundary_condition, mesh, stream):
    """(device mesh, TermsDesc, BcDesc, tensors the descriptors point into)."""
    dm = mesh.device(stream)
    c_lap, c_conv, c_src = equation.coefficients()
    keep = []

    def dptr(kind):
        if kind not in equation.data:
            return None
        t = _dev_f64(equation.data[kind])
        keep.append(t)
        return t.data_ptr()

    t = TermsDesc()
    t.laplacian_coef, t.convection_coef, t.source_coef = c_lap, c_conv, c_src
    t.diffusivity = dptr("laplacian")
    t.flux = dptr("convection")
    t.source = dptr("source")
    sch = equation.data.get("laplacian_scheme")
    if sch is not None and sch.__class__.__name__ == "Corrected":
        g = sch.gradients.data if isinstance(sch.gradients, DistributedVector) else _dev_f64(sch.gradients)
        g = g.reshape(-1).contiguous()
        if g.numel() != mesh.n_cells * mesh.dim:
            raise ValueError("Corrected: gradients must hold n_cells * dim values")
        keep.append(g)
        t.scheme = 1
        t.corrector_reduction = sch.corrector_reduction
        t.gradients = g.data_ptr()
    def arr(a):
        t = _dev_f64(a)
        keep.append(t)
        return t.data_ptr()

    ts = equation.data.get("time")
    if ts is not None:
        t.time_coef = equation.coefficient("time")
        t.dt = ts.dt
        t.previous = arr(ts.previous)
        if ts.__class__.__name__ == "Euler":
            t.time_scheme = 1
            if ts.densities is not None:
                t.density, t.density_previous = arr(ts.densities[0]), arr(ts.densities[1])
        else:
            t.time_scheme = 2
            t.dt_2 = ts.dt_2
            t.previous_2 = arr(ts.previous_2)
            if ts.densities is not None:
                t.density, t.density_previous, t.density_previous_2 = (arr(d) for d in ts.densities)
    if "linear_source" in equation.data:
        t.linear_source_coef = equation.coefficient("linear_source")
        t.linear_source = arr(equation.data["linear_source"])
    if "divergence" in equation.data:
        t.divergence_coef = equation.coefficient("divergence")
        t.divergence_flux = arr(equation.data["divergence"])
    bndi, bnde = _bc_arrays(boundary_condition, mesh)
    bi = _dev_f64(bndi)
    be = _dev_f64(bnde)
    keep += [bi, be]
    bc = BcDesc(bi.data_ptr(), be.data_ptr())
    return dm, t, bc, keep


def compute_gradients(gradients: DistributedVector, values, boundary_condition, mesh, stream=None) -> None:
    """compute_gradients (fvm/tools/gradients.rs:48-86): least-squares cell
    gradients of a cell field into `gradients` (n_cells*dim, cell-major).
    boundary_condition as in assemble (callable face id -> (bndi, bnde), or a
    pair of arrays over the boundary faces)."""
    dm = mesh.device(stream)
    v = _dev_f64(values)
    bndi, bnde = _bc_arrays(boundary_condition, mesh)
    bi, be = _dev_f64(bndi), _dev_f64(bnde)
    if len(gradients) != mesh.n_cells * mesh.dim:
        raise ValueError("gradients must hold n_cells * dim values")
    bc = BcDesc(bi.data_ptr(), be.data_ptr())
    check(lib().fv_compute_gradients(dm.handle, C.c_void_p(v.data_ptr()), C.byref(bc), gradients.ptr(),
                                     stream_handle(stream)), "compute_gradients")
    del v, bi, be


class Preconditioner:
    handle = C.c_void_p()
    perm = None          # reordered factorisations: perm[i] = the row of A that is row i of the factors
    order_info = None

    def precondition(self, solution: DistributedVector, rhs: DistributedVector, comm=None, stream=None) -> None:
        """solution = M^-1 rhs (Preconditioner::precondition, preconditioners/mod.rs:13-17)."""
        check(lib().fv_precond_apply(self.handle, rhs.ptr(), solution.ptr(), stream_handle(stream)), "precondition")

    def factors(self, stream=None):
        """Stored factors as CSR numpy arrays: IC -> the reference's `l`,
        ILU -> the reference's `lu` (dropped entries removed); and n_dropped."""
        nz = C.c_int64()
        nd = C.c_int32()
        check(lib().fv_precond_export(self.handle, C.byref(nz), None, None, None, C.byref(nd),
                                      stream_handle(stream)), "factors")
        n = self.n
        rp = np.empty(n + 1, np.int32)
        cc = np.empty(max(nz.value, 1), np.int32)
        vv = np.empty(max(nz.value, 1), np.float64)
        check(lib().fv_precond_export(self.handle, C.byref(nz), rp.ctypes.data_as(C.POINTER(C.c_int32)),
                                      cc.ctypes.data_as(C.POINTER(C.c_int32)),
                                      vv.ctypes.data_as(C.POINTER(C.c_double)), C.byref(nd),
                                      stream_handle(stream)), "factors")
        return rp, cc[: nz.value], vv[: nz.value], nd.value

    def levels(self):
        n = self.n
        fl = np.empty(n, np.int32)
        bl = np.empty(n, np.int32)
        nf, nb = C.c_int32(), C.c_int32()
        check(lib().fv_precond_levels(self.handle, fl.ctypes.data_as(C.POINTER(C.c_int32)),
                                      bl.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(nf), C.byref(nb), None),
              "levels")
        return fl, bl, nf.value, nb.value

    def schedule(self, request: int = -1):
        """Sweep schedule: request -1 = query, 0 or 1 = level chunks (default),
        2 = box tiles (matrices assembled on a mesh), 3 = level chunks with
        the next chunk prefetched, 4 = consecutive rows (the default when the
        rows are sorted by level, e.g. a matrix permuted by order_boxes'
        order).  Returns (active, stats) with active 1..4 and stats = (box
        edge in cell sizes, boxes, lane use fwd/bwd, ring share fwd/bwd)."""
        act = C.c_int32()
        st = np.zeros(6)
        check(lib().fv_precond_schedule(self.handle, int(request), C.byref(act),
                                        st.ctypes.data_as(C.POINTER(C.c_double))), "schedule")
        return act.value, st

    def set_grid(self, blocks: int, rows_per_thread: int = 0):
        """Sweep launch shape (fv_precond_set_grid): blocks per launch and rows
        per thread of the reordered sweeps, 0 = defaults; same results for any shape."""
        check(lib().fv_precond_set_grid(self.handle, int(blocks), int(rows_per_thread)), "set_grid")

    def refactor(self, stream=None):
        """Value-only refactorisation after the matrix values changed."""
        check(lib().fv_precond_refactor(self.handle, stream_handle(stream)), "refactor")

    def close(self):
        if self.handle:
            lib().fv_precond_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            if exiting():  # module globals may already be gone at interpreter teardown
                return
            self.close()
        except Exception:
            pass


def _fill_pattern(kind: int, level: int, row_ptr, cols):
    """Host level-k factor pattern (fv_fill_pattern_host): (fptr, fcol, amap, fill)."""
    ip = C.POINTER(C.c_int32)
    ptr = np.ascontiguousarray(row_ptr, np.int32)
    col = np.ascontiguousarray(cols, np.int32)
    n = len(ptr) - 1
    nnz = C.c_int64()
    check(lib().fv_fill_pattern_host(kind, int(level), n, ptr.ctypes.data_as(ip), col.ctypes.data_as(ip),
                                     C.byref(nnz), None, None, None, None), "fill pattern")
    fptr = np.zeros(n + 1, np.int32)
    fcol = np.zeros(max(nnz.value, 1), np.int32)
    amap = np.zeros(max(len(col), 1), np.int32)
    fill = np.zeros(max(nnz.value, 1), np.uint8)
    check(lib().fv_fill_pattern_host(kind, int(level), n, ptr.ctypes.data_as(ip), col.ctypes.data_as(ip),
                                     C.byref(nnz), fptr.ctypes.data_as(ip), fcol.ctypes.data_as(ip),
                                     amap.ctypes.data_as(ip), fill.ctypes.data_as(C.POINTER(C.c_uint8))),
          "fill pattern")
    return fptr, fcol[:nnz.value], amap[:len(col)], fill[:nnz.value]


def order_boxes(matrix: "DistributedMatrix", rows_per_box: int = 0, offsets=None, stream=None, levels=False):
    """Box-colour ordering of a matrix assembled on a mesh (fv_order_boxes):
    (perm, info) with perm[i] = the row of the matrix that becomes row i of
    the reordered one, info = dict(n_boxes, boxes_per_axis, n_colours,
    n_levels).  rows_per_box 0: 32 in 2D, 384 in 3D.  offsets: the row
    offsets of the independent problems of a batch (each ordered on its own).
    levels (one problem only): also return level[i] of row i of the
    reordered matrix (fv_order_boxes_levels), for merge_orders."""
    n = matrix.nrows()
    perm = np.empty(n, np.int32)
    info = OrderInfo()
    if levels:
        if offsets is not None and len(offsets) > 2:
            raise ValueError("levels: one problem only")
        lev = np.empty(n, np.int32)
        ip = C.POINTER(C.c_int32)
        check(lib().fv_order_boxes_levels(matrix.handle, int(rows_per_box), perm.ctypes.data_as(ip),
                                          lev.ctypes.data_as(ip), C.byref(info), stream_handle(stream)),
              "order_boxes_levels")
        return perm, _order_info(info), lev
    np_, offp = 1, None
    if offsets is not None:
        off = np.ascontiguousarray(offsets, np.int64)
        np_, offp = len(off) - 1, off.ctypes.data_as(C.POINTER(C.c_int64))
    check(lib().fv_order_boxes(matrix.handle, np_, offp, int(rows_per_box),
                               perm.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(info), stream_handle(stream)),
          "order_boxes")
    return perm, _order_info(info)


def order_boxes_host(cell_center, row_ptr, cols, rows_per_box: int = 0, lo=None, hi=None, levels=False):
    """The same ordering from host arrays (fv_order_boxes_host): cell_center
    n x dim, a CSR pattern, optional domain box lo / hi; levels: also the
    level of every reordered row (fv_order_boxes_host_levels)."""
    cc = np.ascontiguousarray(cell_center, np.float64)
    n, dim = cc.shape
    ptr = np.ascontiguousarray(row_ptr, np.int32)
    col = np.ascontiguousarray(cols, np.int32)
    perm = np.empty(n, np.int32)
    info = OrderInfo()
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int32)
    lo_a = np.ascontiguousarray(lo, np.float64) if lo is not None else None
    hi_a = np.ascontiguousarray(hi, np.float64) if hi is not None else None
    box = (lo_a.ctypes.data_as(dp) if lo_a is not None else None, hi_a.ctypes.data_as(dp) if hi_a is not None else None)
    if levels:
        lev = np.empty(n, np.int32)
        check(lib().fv_order_boxes_host_levels(n, dim, cc.ctypes.data_as(dp), dim, *box, ptr.ctypes.data_as(ip),
                                               col.ctypes.data_as(ip), int(rows_per_box), perm.ctypes.data_as(ip),
                                               lev.ctypes.data_as(ip), C.byref(info)), "order_boxes_host_levels")
        return perm, _order_info(info), lev
    check(lib().fv_order_boxes_host(n, dim, cc.ctypes.data_as(dp), dim, *box, ptr.ctypes.data_as(ip),
                                    col.ctypes.data_as(ip), int(rows_per_box), perm.ctypes.data_as(ip),
                                    C.byref(info)), "order_boxes_host")
    return perm, _order_info(info)


def merge_orders(parts, offsets):
    """The union order of independent problems from each problem's own order:
    parts[k] = (perm_k, level_k) as order_boxes(..., levels=True) gives them
    for problem k alone, offsets = the problems' first rows in the union.
    For each level, every problem's rows of that level in problem order --
    the order fv_order_boxes gives the union (rows sorted stably by level,
    then problem, then position)."""
    ptrs = []
    nlev = 0
    for perm_k, lev_k in parts:
        top = int(lev_k[-1]) + 1 if len(lev_k) else 0
        ptrs.append(np.searchsorted(lev_k, np.arange(top + 1), side="left"))
        nlev = max(nlev, top)
    segs = []
    for lv in range(nlev):
        for k, (perm_k, _) in enumerate(parts):
            lp = ptrs[k]
            if lv + 1 < len(lp) and lp[lv + 1] > lp[lv]:
                segs.append(perm_k[lp[lv]:lp[lv + 1]] + np.int32(offsets[k]))
    return np.concatenate(segs).astype(np.int32) if segs else np.zeros(0, np.int32)


def _order_info(info):
    return {"n_boxes": int(info.n_boxes), "boxes_per_axis": [int(v) for v in info.boxes_per_axis],
            "n_colours": int(info.n_colours), "n_levels": int(info.n_levels)}


def _factor(kind: str, matrix, level, ordering, stream, offsets=None):
    """Natural order (the reference's factorisation) when ordering is None;
    else the reordered factorisation of Q A Q^T with ordering = "boxes" (the
    box-colour ordering; per problem with `offsets`) or a permutation array
    (perm[i] = the row of A that becomes row i).  Returns (handle, perm or
    None, order info or None)."""
    h = C.c_void_p()
    if ordering is None:
        fn = lib().fv_ic_factor if kind == "ic" else lib().fv_ilu_factor
        check(fn(matrix.handle, int(level), stream_handle(stream), C.byref(h)),
              "IncompleteCholesky" if kind == "ic" else "IncompleteLowerUpper")
        return h, None, None
    if level != 0:
        raise FvError(8, "reordered factorisation: level 0 only")
    info = None
    if isinstance(ordering, str):
        if ordering != "boxes":
            raise ValueError(f"unknown ordering {ordering!r}")
        perm, info = order_boxes(matrix, offsets=offsets, stream=stream)
    else:
        perm = np.ascontiguousarray(ordering, np.int32)
    fn = lib().fv_ic0_factor_perm if kind == "ic" else lib().fv_ilu0_factor_perm
    check(fn(matrix.handle, perm.ctypes.data_as(C.POINTER(C.c_int32)), stream_handle(stream), C.byref(h)),
          "reordered factorisation")
    return h, perm, info


class IncompleteCholesky(Preconditioner):
    def __init__(self, handle, n, matrix):
        self.handle, self.n, self._m = handle, n, matrix

    @staticmethod
    def fill_pattern(row_ptr, cols, level: int):
        """The IC(level) factor pattern from_matrix builds (row_i_sparsity_edit,
        incomplete_cholesky.rs:35-85), from a host CSR pattern: (fptr, fcol,
        amap = position of every entry of A, fill = 1 for fill entries)."""
        return _fill_pattern(1, level, row_ptr, cols)

    @classmethod
    def from_matrix(cls, matrix: DistributedMatrix, level: int = 0, stream=None, ordering=None,
                    offsets=None) -> "IncompleteCholesky":
        """IncompleteCholesky::from_matrix(A, level) (incomplete_cholesky.rs:205).
        ordering: None = the reference's natural row order; "boxes" or a
        permutation = the reordered factorisation (fv_ic0_factor_perm);
        offsets: a batch's problem row offsets for "boxes"."""
        h, perm, info = _factor("ic", matrix, level, ordering, stream, offsets)
        P = cls(h, matrix.nrows(), matrix)
        P.perm, P.order_info = perm, info
        return P


class IncompleteLowerUpper(Preconditioner):
    def __init__(self, handle, n, matrix):
        self.handle, self.n, self._m = handle, n, matrix

    @staticmethod
    def fill_pattern(row_ptr, cols, level: int):
        """The ILU(level) factor pattern from_matrix builds (row_i_l_sparsity /
        row_i_u_sparsity, incomplete_lower_upper.rs:30-137), from a host CSR
        pattern: (fptr, fcol, amap = position of every entry of A)."""
        return _fill_pattern(2, level, row_ptr, cols)[:3]

    @classmethod
    def from_matrix(cls, matrix: DistributedMatrix, level: int = 0, stream=None, ordering=None,
                    offsets=None) -> "IncompleteLowerUpper":
        """IncompleteLowerUpper::from_matrix(A, level) (incomplete_lower_upper.rs:266).
        ordering: None = the reference's natural row order; "boxes" or a
        permutation = the reordered factorisation (fv_ilu0_factor_perm);
        offsets: a batch's problem row offsets for "boxes"."""
        h, perm, info = _factor("ilu", matrix, level, ordering, stream, offsets)
        P = cls(h, matrix.nrows(), matrix)
        P.perm, P.order_info = perm, info
        return P


class DiagonalPreconditioner(Preconditioner):
    """DiagonalPreconditioner (preconditioners/mod.rs:38-68): z = r / diag(A)."""

    def __init__(self, handle, n, matrix):
        self.handle, self.n, self._m = handle, n, matrix

    @classmethod
    def from_matrix(cls, matrix: DistributedMatrix, stream=None) -> "DiagonalPreconditioner":
        h = C.c_void_p()
        check(lib().fv_diag_factor(matrix.handle, stream_handle(stream), C.byref(h)), "DiagonalPreconditioner")
        return cls(h, matrix.nrows(), matrix)


class IdentityPreconditioner(Preconditioner):
    handle = C.c_void_p()


@dataclass
class LinearSolverOptions:
    relative_tolerance: float = 1e-6
    absolute_tolerance: float = 1e-6
    max_iterations: int = 1000

    def c(self) -> SolverOptions:
        return SolverOptions(self.relative_tolerance, self.absolute_tolerance, self.max_iterations)


@dataclass
class LinearSolverInfo:
    solver_identifier: str
    iterations: int
    initial_residual: float
    final_residual: float
    history: list = field(default_factory=list)
    status: int = 0
    restarts: int = 0
    device_ms: float = 0.0

    def __str__(self):
        return (f"(solver={self.solver_identifier}, iterations={self.iterations}, "
                f"initial_residual={self.initial_residual:.3e}, final_residual={self.final_residual:.3e})")


def _solve(fn, name, solution, lhs, rhs, preconditioner, options, stream):
    options = options or LinearSolverOptions()
    cap = int(options.max_iterations) + 2
    hist = np.zeros(cap, np.float64)
    info = SolverInfo()
    info.history = hist.ctypes.data_as(C.POINTER(C.c_double))
    info.history_cap = cap
    b = _dev_f64(rhs)
    ph = preconditioner.handle if preconditioner is not None else C.c_void_p()
    st = fn(lhs.handle, ph, C.c_void_p(b.data_ptr()), solution.ptr(), options.c(), C.byref(info),
            stream_handle(stream))
    if st not in (0, 4):  # breakdown is reported in the info, as the reference returns Ok with NaN residuals
        raise FvError(st, name)
    return LinearSolverInfo(name, int(info.iterations), float(info.initial_residual), float(info.final_residual),
                            hist[: min(int(info.history_len), cap)].tolist(), int(info.status), int(info.restarts),
                            float(info.device_ms))


def conjugate_gradient(solution: DistributedVector, lhs: DistributedMatrix, rhs, preconditioner=None, comm=None,
                       options: LinearSolverOptions | None = None, stream=None) -> LinearSolverInfo:
    return _solve(lib().fv_cg, "ConjugateGradient", solution, lhs, rhs, preconditioner, options, stream)


def bi_conjugate_gradient_stab(solution: DistributedVector, lhs: DistributedMatrix, rhs, preconditioner=None,
                               comm=None, options: LinearSolverOptions | None = None,
                               stream=None) -> LinearSolverInfo:
    return _solve(lib().fv_bicgstab, "BiConjugateGradientStab", solution, lhs, rhs, preconditioner, options, stream)


class PermutedSystem:
    """The box-colour order as a permuted system: B = Q A Q^T (rows sorted by
    level) factorised with IC(0) ("ic") or ILU(0) ("ilu") and solved in its
    own numbering; b is permuted in and x back on every solve, so callers
    keep A's numbering.  After A is re-assembled, refresh() takes its new
    values and refactorises.  perm: an explicit permutation instead of
    order_boxes' (any permutation; the sweeps are fastest when it sorts the
    rows by level)."""

    def __init__(self, A: DistributedMatrix, kind: str = "ilu", perm=None, stream=None):
        if kind not in ("ic", "ilu"):
            raise ValueError(f"kind must be 'ic' or 'ilu', not {kind!r}")
        if perm is None:
            perm, self.order_info = order_boxes(A, stream=stream)
        else:
            self.order_info = None
        self.kind = kind
        self.A = A
        self.B = A.permuted(perm, stream=stream)
        cls = IncompleteCholesky if kind == "ic" else IncompleteLowerUpper
        self.P = cls.from_matrix(self.B, 0, stream=stream)
        n = A.nrows()
        self._b = DistributedVector.from_size(n)
        self._y = DistributedVector.from_size(n)

    @property
    def perm(self):
        return self.B.perm

    def refresh(self, stream=None) -> None:
        """Take A's current values (after a re-assembly) and refactorise."""
        self.B.refresh_permuted(stream=stream)
        self.P.refactor(stream=stream)

    def solve(self, solution: DistributedVector, rhs, options: LinearSolverOptions | None = None,
              initial_guess: bool = True, stream=None) -> LinearSolverInfo:
        """CG (IC) or BiCGStab (ILU) on B y = Q rhs from y0 = Q solution
        (initial_guess) or 0; solution = Q^T y."""
        self.B.to_permuted(rhs, self._b, stream=stream)
        if initial_guess:
            self.B.to_permuted(solution.data, self._y, stream=stream)
        else:
            self._y.data.zero_()
        fn = conjugate_gradient if self.kind == "ic" else bi_conjugate_gradient_stab
        info = fn(self._y, self.B, self._b, self.P, None, options, stream=stream)
        self.B.from_permuted(self._y, solution, stream=stream)
        return info
