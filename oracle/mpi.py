"""MPI-semantics oracle (block-Jacobi over P contiguous partitions, one OpenMP
thread per rank) -- TEST AND CPU-BASELINE INFRASTRUCTURE ONLY.  See oracle_mpi.c."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import OrInfo, _d, _i, _pd, _pi, dp, i64, ip, lib as _lib

_done = False


def lib():
    global _done
    L = _lib()
    if not _done:
        L.or_bj_create.argtypes = [C.c_int, i64, ip, ip, dp, C.c_int, C.POINTER(C.c_int)]
        L.or_bj_create.restype = C.c_void_p
        L.or_bj_free.argtypes = [C.c_void_p]
        L.or_bj_free.restype = None
        for f in (L.or_bj_cg, L.or_bj_bicgstab):
            f.argtypes = [i64, ip, ip, dp, C.c_void_p, dp, dp, C.c_double, C.c_double, i64, C.POINTER(OrInfo)]
            f.restype = C.c_int
        L.or_pattern_par.argtypes = [i64, ip, ip, ip, ip, C.c_int, ip, ip, C.POINTER(i64)]
        L.or_pattern_par.restype = C.c_int
        L.or_assemble_par.argtypes = [C.c_int32, i64, i64, i64, ip, ip, dp, dp, dp, dp, C.c_double, C.c_double,
                                      C.c_double, dp, dp, dp, dp, dp, ip, ip, C.c_int, dp, dp]
        L.or_assemble_par.restype = C.c_int
        _done = True
    return L


def assemble(mesh, c_lap, c_conv, c_src, kappa, flux, source, bndi, bnde, P):
    """assemble() on P ranks (one thread each, contiguous cell partitions): the
    pattern and Orthogonal / Upwind / source values of every rank's own rows.
    Returns (row_ptr, cols, vals, rhs), equal bit for bit to oracle.assemble."""
    N, F, Fb = mesh.n_cells, mesh.n_faces, mesh.n_boundary_faces
    cfp, cf = _i(mesh.cell_face_ptr), _i(mesh.cell_faces)
    ow, nb = _i(mesh.face_owner), _i(mesh.face_neighbor)
    ptr = np.zeros(N + 1, np.int32)
    nnz = C.c_int64()
    rc = lib().or_pattern_par(N, _pi(cfp), _pi(cf), _pi(ow), _pi(nb), int(P), _pi(ptr), None, C.byref(nnz))
    if rc != 0:
        raise RuntimeError("oracle pattern failed")
    cols = np.empty(max(nnz.value, 1), np.int32)
    lib().or_pattern_par(N, _pi(cfp), _pi(cf), _pi(ow), _pi(nb), int(P), _pi(ptr), _pi(cols), C.byref(nnz))
    cols = cols[: nnz.value]
    z = lambda n: np.zeros(max(n, 1))  # noqa: E731
    kappa = _d(kappa) if kappa is not None else z(F)
    flux = _d(flux) if flux is not None else z(F)
    source = _d(source) if source is not None else z(N)
    bndi = _d(bndi) if bndi is not None and len(bndi) else z(Fb)
    bnde = _d(bnde) if bnde is not None and len(bnde) else z(Fb)
    vals = np.empty(max(len(cols), 1))
    rhs = np.empty(N)
    rc = lib().or_assemble_par(mesh.dim, N, F, Fb, _pi(ow), _pi(nb), _pd(_d(mesh.face_area)),
                               _pd(_d(mesh.face_center)), _pd(_d(mesh.cell_center)), _pd(_d(mesh.cell_volume)),
                               c_lap, c_conv, c_src, _pd(kappa), _pd(flux), _pd(source), _pd(bndi), _pd(bnde),
                               _pi(ptr), _pi(cols), int(P), _pd(vals), _pd(rhs))
    if rc != 0:
        raise RuntimeError(f"oracle parallel assemble failed: {rc}")
    return ptr, cols, vals[: len(cols)], rhs


class BlockJacobi:
    def __init__(self, kind, ptr, cols, vals, P):
        self._keep = (_i(ptr), _i(cols), _d(vals))
        st = C.c_int()
        self.h = lib().or_bj_create(1 if kind == "ic" else 2, len(ptr) - 1, _pi(self._keep[0]), _pi(self._keep[1]),
                                    _pd(self._keep[2]), int(P), C.byref(st))
        self.status = st.value
        self.P = P

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_bj_free(self.h)
            self.h = None


def solve(solver, ptr, cols, vals, bj, b, rtol, atol, maxit, threads=None):
    ptr, cols, vals, b = _i(ptr), _i(cols), _d(vals), _d(b)
    x = np.zeros(len(b))
    info = OrInfo()
    f = lib().or_bj_bicgstab if solver == "bicgstab" else lib().or_bj_cg
    rc = f(len(b), _pi(ptr), _pi(cols), _pd(vals), bj.h, _pd(b), _pd(x), rtol, atol, maxit, C.byref(info))
    assert rc == 0
    return x, {"iterations": info.iterations, "initial_residual": info.initial_residual,
               "final_residual": info.final_residual, "restarts": info.restarts}
