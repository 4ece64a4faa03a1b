"""MPI-semantics oracle (block-Jacobi over P contiguous partitions, one OpenMP
thread per rank) -- TEST AND CPU-BASELINE INFRASTRUCTURE ONLY.  See oracle_mpi.c."""
from __future__ import annotations

import ctypes as C
import time

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
        _done = True
    return L


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


def iterations_estimate(solver, kind, ptr, cols, vals, b, rtol, P, budget_s=60.0):
    """Iteration count of the P-rank block-Jacobi solve to rtol.  Runs the full
    solve when it fits in budget_s (timed on the first 3 iterations), else
    extrapolates from the residual decay of a bounded run."""
    bj = BlockJacobi(kind, ptr, cols, vals, P)
    t0 = time.perf_counter()
    _, info = solve(solver, ptr, cols, vals, bj, b, 1e-30, 1e-30, 2)
    t_it = (time.perf_counter() - t0) / max(info["iterations"], 1)
    cap = max(3, int(budget_s / max(t_it, 1e-9)))
    _, info = solve(solver, ptr, cols, vals, bj, b, rtol, rtol, cap)
    if info["final_residual"] <= rtol or info["iterations"] <= cap:
        return int(info["iterations"])
    # not converged in budget: geometric extrapolation of the residual history
    rate = (info["final_residual"] / max(info["initial_residual"], 1e-300)) ** (1.0 / info["iterations"])
    return int(np.ceil(np.log(rtol) / np.log(max(rate, 1e-12))))
