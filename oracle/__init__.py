"""CPU oracle -- TEST INFRASTRUCTURE ONLY.

ctypes wrapper of oracle/liboracle.so, the single-threaded FP64 C
restatement of the finite-volumes crate's assemble / SpMV / IC(0) / ILU(0) /
CG / BiCGStab (see oracle/oracle.c for the file:line map).  Used only by
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, as the
checker and the timed CPU baseline; the product library never calls it.

Parity status: assembly, factorisation and Krylov results are parity-unpinned
against the reference itself (the reference has no tests for them and cannot
be built here); the oracle is cross-checked against SciPy and hand-derived
coefficients in tests/, and the mesh geometry it consumes is pinned by the
reference's square.su2 known-answer test.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from .build import LIB, build

_L = None
P = C.POINTER
dp, ip, i64, vp = P(C.c_double), P(C.c_int32), C.c_int64, C.c_void_p


class OrExtra(C.Structure):
    _fields_ = [("c_time", C.c_double), ("c_lin", C.c_double), ("c_div", C.c_double), ("time_scheme", C.c_int),
                ("dt", C.c_double), ("dt_2", C.c_double), ("prev", dp), ("prev2", dp), ("dens", dp), ("densp", dp),
                ("densp2", dp), ("lin", dp), ("divflux", dp)]


class OrInfo(C.Structure):
    _fields_ = [("iterations", i64), ("initial_residual", C.c_double), ("final_residual", C.c_double),
                ("history_len", i64), ("restarts", C.c_int32)]


def lib():
    global _L
    if _L is None:
        build()
        L = C.CDLL(str(LIB))
        sig = {
            "or_pattern": ([i64, ip, ip, ip, ip, ip, ip, P(i64)], C.c_int),
            "or_assemble": ([C.c_int32, i64, i64, i64, ip, ip, dp, dp, dp, dp, C.c_double, C.c_double, C.c_double,
                             dp, dp, dp, dp, dp, ip, ip, dp, dp], C.c_int),
            "or_assemble_scheme": ([C.c_int32, i64, i64, i64, ip, ip, dp, dp, dp, dp, C.c_double, C.c_double,
                                    C.c_double, dp, dp, dp, dp, dp, ip, ip, dp, dp, C.c_int, dp, dp, C.c_double],
                                   C.c_int),
            "or_assemble_full": ([C.c_int32, i64, i64, i64, ip, ip, dp, dp, dp, dp, C.c_double, C.c_double,
                                  C.c_double, dp, dp, dp, dp, dp, ip, ip, dp, dp, C.c_int, dp, dp, C.c_double,
                                  P(OrExtra)], C.c_int),
            "or_grad_coeffs": ([C.c_int32, i64, ip, ip, dp, dp, ip, ip, dp, dp], C.c_int),
            "or_gradients": ([C.c_int32, i64, i64, i64, ip, ip, ip, ip, dp, dp, dp, dp, dp, dp], None),
            "or_spmv": ([i64, ip, ip, dp, dp, dp], None),
            "or_dot": ([i64, dp, dp], C.c_double),
            "or_ic0_create": ([i64, ip, ip, dp, P(C.c_int)], vp),
            "or_ic_create_fill": ([i64, ip, ip, dp, P(C.c_ubyte), P(C.c_int)], vp),
            "or_fill_pattern": ([C.c_int, C.c_int, i64, ip, ip, ip, ip, P(C.c_ubyte)], i64),
            "or_ilu0_create": ([i64, ip, ip, dp, P(C.c_int)], vp),
            "or_precond_apply": ([vp, dp, dp], None),
            "or_diag_create": ([i64, ip, ip, dp, P(C.c_int)], vp),
            "or_precond_free": ([vp], None),
            "or_precond_nnz": ([vp], i64),
            "or_perm_create": ([i64, ip, vp], vp),
            "or_precond_ndropped": ([vp], i64),
            "or_precond_export": ([vp, ip, ip, dp, dp], None),
            "or_levels": ([i64, ip, ip, C.c_int32, ip], C.c_int32),
            "or_cg": ([i64, ip, ip, dp, vp, dp, dp, C.c_double, C.c_double, i64, dp, i64, P(OrInfo)], C.c_int),
            "or_bicgstab": ([i64, ip, ip, dp, vp, dp, dp, C.c_double, C.c_double, i64, dp, i64, P(OrInfo)],
                            C.c_int),
        }
        for k, (a, r) in sig.items():
            f = getattr(L, k)
            f.argtypes = a
            f.restype = r
        _L = L
    return _L


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _pi(a):
    return a.ctypes.data_as(ip)


def _pd(a):
    return a.ctypes.data_as(dp)


def pattern(mesh):
    """CSR pattern of cell_to_cell (rows sorted)."""
    cfp, cf, ow, nb = _i(mesh.cell_face_ptr), _i(mesh.cell_faces), _i(mesh.face_owner), _i(mesh.face_neighbor)
    nnz = C.c_int64()
    rc = lib().or_pattern(mesh.n_cells, _pi(cfp), _pi(cf), _pi(ow), _pi(nb), None, None, C.byref(nnz))
    assert rc == 0
    ptr = np.empty(mesh.n_cells + 1, np.int32)
    cols = np.empty(max(nnz.value, 1), np.int32)
    rc = lib().or_pattern(mesh.n_cells, _pi(cfp), _pi(cf), _pi(ow), _pi(nb), _pi(ptr), _pi(cols), C.byref(nnz))
    assert rc == 0
    return ptr, cols[: nnz.value]


def grad_coeffs(mesh):
    """Gradient coefficients of Mesh::compute: (per cell-face entry in mesh
    order, n_entries x dim; per cell, n_cells x dim)."""
    d, N = mesh.dim, mesh.n_cells
    cfp, cf = _i(mesh.cell_face_ptr), _i(mesh.cell_faces)
    gcoef = np.empty((max(int(cfp[-1]), 1), d))
    gdiag = np.empty((N, d))
    rc = lib().or_grad_coeffs(d, N, _pi(_i(mesh.face_owner)), _pi(_i(mesh.face_neighbor)),
                              _pd(_d(mesh.face_center)), _pd(_d(mesh.cell_center)), _pi(cfp), _pi(cf), _pd(gcoef),
                              _pd(gdiag))
    if rc != 0:
        raise RuntimeError("oracle gradient coefficients: singular cell matrix")
    return gcoef[: int(cfp[-1])], gdiag


def gradients(mesh, values, bndi, bnde):
    """compute_gradients restated: n_cells x dim."""
    gcoef, gdiag = grad_coeffs(mesh)
    d, N = mesh.dim, mesh.n_cells
    out = np.empty((N, d))
    gc = _d(gcoef) if len(gcoef) else np.zeros((1, d))
    lib().or_gradients(d, N, mesh.n_faces, mesh.n_boundary_faces, _pi(_i(mesh.face_owner)),
                       _pi(_i(mesh.face_neighbor)), _pi(_i(mesh.cell_face_ptr)), _pi(_i(mesh.cell_faces)), _pd(gc),
                       _pd(_d(gdiag)), _pd(_d(values)), _pd(_d(bndi) if len(bndi) else np.zeros(1)),
                       _pd(_d(bnde) if len(bnde) else np.zeros(1)), _pd(out))
    return out


def assemble(mesh, c_lap, c_conv, c_src, kappa=None, flux=None, source=None, bndi=None, bnde=None,
             corrected=None, extra=None):
    """assemble() restated: returns (row_ptr, cols, vals, rhs).  corrected =
    (gradients n_cells x dim, corrector_reduction) selects the Corrected
    face-normal gradient scheme for the laplacian (Orthogonal otherwise).
    extra = dict(c_time, time_scheme ("euler" | "backward"), dt, dt_2,
    previous, previous_2, densities, c_lin, lin, c_div, divflux) adds the
    transient / linear-source / divergence terms."""
    if extra is not None:
        return _assemble_full(mesh, c_lap, c_conv, c_src, kappa, flux, source, bndi, bnde, corrected, extra)
    ptr, cols = pattern(mesh)
    F, N, Fb = mesh.n_faces, mesh.n_cells, mesh.n_boundary_faces
    z = lambda n: np.zeros(max(n, 1))  # noqa: E731
    kappa = _d(kappa) if kappa is not None else z(F)
    flux = _d(flux) if flux is not None else z(F)
    source = _d(source) if source is not None else z(N)
    bndi = _d(bndi) if bndi is not None else z(Fb)
    bnde = _d(bnde) if bnde is not None else z(Fb)
    vals = np.empty(len(cols))
    rhs = np.empty(N)
    if corrected is None:
        rc = lib().or_assemble(mesh.dim, N, F, Fb, _pi(_i(mesh.face_owner)), _pi(_i(mesh.face_neighbor)),
                               _pd(_d(mesh.face_area)), _pd(_d(mesh.face_center)), _pd(_d(mesh.cell_center)),
                               _pd(_d(mesh.cell_volume)), c_lap, c_conv, c_src, _pd(kappa), _pd(flux), _pd(source),
                               _pd(bndi), _pd(bnde), _pi(ptr), _pi(cols), _pd(vals), _pd(rhs))
    else:
        grad, red = corrected
        rc = lib().or_assemble_scheme(mesh.dim, N, F, Fb, _pi(_i(mesh.face_owner)), _pi(_i(mesh.face_neighbor)),
                                      _pd(_d(mesh.face_area)), _pd(_d(mesh.face_center)),
                                      _pd(_d(mesh.cell_center)), _pd(_d(mesh.cell_volume)), c_lap, c_conv, c_src,
                                      _pd(kappa), _pd(flux), _pd(source), _pd(bndi), _pd(bnde), _pi(ptr), _pi(cols),
                                      _pd(vals), _pd(rhs), 1, _pd(_d(mesh.face_normal)), _pd(_d(grad)), float(red))
    if rc != 0:
        raise RuntimeError(f"oracle assemble failed: {rc}")
    return ptr, cols, vals, rhs


def _assemble_full(mesh, c_lap, c_conv, c_src, kappa, flux, source, bndi, bnde, corrected, extra):
    ptr, cols = pattern(mesh)
    F, N, Fb = mesh.n_faces, mesh.n_cells, mesh.n_boundary_faces
    z = lambda n: np.zeros(max(n, 1))  # noqa: E731
    kappa = _d(kappa) if kappa is not None else z(F)
    flux = _d(flux) if flux is not None else z(F)
    source = _d(source) if source is not None else z(N)
    bndi = _d(bndi) if bndi is not None else z(Fb)
    bnde = _d(bnde) if bnde is not None else z(Fb)
    keep = []

    def arr(a):
        if a is None:
            return None
        t = _d(a)
        keep.append(t)
        return _pd(t)

    ex = OrExtra()
    ex.c_time = float(extra.get("c_time", 0.0))
    ex.c_lin = float(extra.get("c_lin", 0.0))
    ex.c_div = float(extra.get("c_div", 0.0))
    ex.time_scheme = 1 if extra.get("time_scheme", "euler") == "euler" else 2
    ex.dt = float(extra.get("dt", 0.0))
    ex.dt_2 = float(extra.get("dt_2", 0.0))
    ex.prev = arr(extra.get("previous"))
    ex.prev2 = arr(extra.get("previous_2"))
    dens = extra.get("densities")
    if dens is not None:
        ex.dens, ex.densp = arr(dens[0]), arr(dens[1])
        if len(dens) > 2:
            ex.densp2 = arr(dens[2])
    ex.lin = arr(extra.get("lin"))
    ex.divflux = arr(extra.get("divflux"))
    scheme, grad, red = (0, z(N * mesh.dim), 0.0) if corrected is None else (1, _d(corrected[0]), corrected[1])
    vals = np.empty(len(cols))
    rhs = np.empty(N)
    rc = lib().or_assemble_full(mesh.dim, N, F, Fb, _pi(_i(mesh.face_owner)), _pi(_i(mesh.face_neighbor)),
                                _pd(_d(mesh.face_area)), _pd(_d(mesh.face_center)), _pd(_d(mesh.cell_center)),
                                _pd(_d(mesh.cell_volume)), c_lap, c_conv, c_src, _pd(kappa), _pd(flux), _pd(source),
                                _pd(bndi), _pd(bnde), _pi(ptr), _pi(cols), _pd(vals), _pd(rhs), scheme,
                                _pd(_d(mesh.face_normal)) if scheme else None, _pd(_d(grad)), float(red),
                                C.byref(ex))
    if rc != 0:
        raise RuntimeError(f"oracle assemble failed: {rc}")
    return ptr, cols, vals, rhs


def spmv(ptr, cols, vals, x):
    ptr, cols, vals, x = _i(ptr), _i(cols), _d(vals), _d(x)
    y = np.empty(len(ptr) - 1)
    lib().or_spmv(len(ptr) - 1, _pi(ptr), _pi(cols), _pd(vals), _pd(x), _pd(y))
    return y


def dot(a, b):
    a, b = _d(a), _d(b)
    return lib().or_dot(len(a), _pd(a), _pd(b))


def fill_pattern(kind, level, ptr, cols):
    """Sorted level-k factor pattern (kind "ic" / "ilu") of the reference's
    depth-first walks, and a 0/1 fill flag per entry."""
    ptr, cols = _i(ptr), _i(cols)
    n = len(ptr) - 1
    k = 1 if kind == "ic" else 2
    tot = lib().or_fill_pattern(k, int(level), n, _pi(ptr), _pi(cols), None, None, None)
    fptr = np.zeros(n + 1, np.int32)
    fcol = np.zeros(max(tot, 1), np.int32)
    fill = np.zeros(max(tot, 1), np.uint8)
    lib().or_fill_pattern(k, int(level), n, _pi(ptr), _pi(cols), _pi(fptr), _pi(fcol),
                          fill.ctypes.data_as(P(C.c_ubyte)))
    return fptr, fcol[:tot], fill[:tot]


class Precond:
    """IncompleteCholesky / IncompleteLowerUpper / DiagonalPreconditioner ("diag") restated.  level >= 1: the
    level-0 numerics on the level-k pattern with zeros at fill positions (IC
    sums a row's fill entries after its matrix entries in the backward sweep,
    as the reference's sp_t does)."""

    def __init__(self, kind, ptr, cols, vals, level=0):
        self.n = len(ptr) - 1
        st = C.c_int()
        fill = None
        if level > 0 and not (kind == "ic" and level == 1):
            fptr, fcol, fill = fill_pattern(kind, level, ptr, cols)
            fv_ = np.zeros(len(fcol))
            ptr_, cols_, vals_ = _i(ptr), _i(cols), _d(vals)
            for i in range(self.n):
                a0, a1, f0, f1 = ptr_[i], ptr_[i + 1], fptr[i], fptr[i + 1]
                pos = np.searchsorted(fcol[f0:f1], cols_[a0:a1]) + f0
                fv_[pos] = vals_[a0:a1]
            ptr, cols, vals = fptr, fcol, fv_
        self._keep = (_i(ptr), _i(cols), _d(vals), fill)
        if kind == "diag":
            self.h = lib().or_diag_create(self.n, _pi(self._keep[0]), _pi(self._keep[1]), _pd(self._keep[2]),
                                          C.byref(st))
        elif kind == "ic":
            fl = fill.ctypes.data_as(P(C.c_ubyte)) if fill is not None else None
            self.h = lib().or_ic_create_fill(self.n, _pi(self._keep[0]), _pi(self._keep[1]), _pd(self._keep[2]),
                                             fl, C.byref(st))
        else:
            self.h = lib().or_ilu0_create(self.n, _pi(self._keep[0]), _pi(self._keep[1]), _pd(self._keep[2]),
                                          C.byref(st))
        self.status = st.value
        self.kind = kind

    @classmethod
    def reordered(cls, kind, ptr, cols, vals, perm):
        """The product's reordered preconditioner restated: `kind` factorised on
        B = Q A Q^T (perm[i] = the row of A that is row i of B), applied in A's
        numbering as z = Q^T M_B^{-1} Q r.  Factors (export) are B's.  The object
        owns one pair of work vectors: apply it from one thread at a time."""
        bp, bc, bv = permute(ptr, cols, vals, perm)
        inner = cls(kind, bp, bc, bv)
        if not inner.h:
            return inner
        p = np.ascontiguousarray(perm, np.int32)
        self = cls.__new__(cls)
        self.n, self.kind, self.status = inner.n, kind, inner.status
        self._keep = inner._keep + (p,)
        self.h = lib().or_perm_create(inner.n, _pi(p), inner.h)
        inner.h = None  # owned by the wrapper now
        return self

    def ok(self):
        return bool(self.h)

    def apply(self, r):
        r = _d(r)
        z = np.zeros(self.n)
        lib().or_precond_apply(self.h, _pd(r), _pd(z))
        return z

    def export(self):
        nz = lib().or_precond_nnz(self.h)
        ptr = np.empty(self.n + 1, np.int32)
        cols = np.empty(max(nz, 1), np.int32)
        vals = np.empty(max(nz, 1))
        inv = np.empty(self.n)
        lib().or_precond_export(self.h, _pi(ptr), _pi(cols), _pd(vals), _pd(inv))
        return ptr, cols[:nz], vals[:nz], inv, lib().or_precond_ndropped(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib().or_precond_free(self.h)
            except Exception:  # interpreter teardown: module globals may be gone already
                pass
            self.h = None


def permute(ptr, cols, vals, perm):
    """B = Q A Q^T as CSR with sorted rows: row i of B is row perm[i] of A, every
    column j renumbered to the position of j in perm."""
    ptr, cols, vals = _i(ptr), _i(cols), _d(vals)
    perm = np.ascontiguousarray(perm, np.int64)
    n = len(ptr) - 1
    inv = np.empty(n, np.int64)
    inv[perm] = np.arange(n)
    lens = np.diff(ptr)[perm]
    bptr = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=bptr[1:])
    src = np.repeat(ptr[perm].astype(np.int64) - bptr[:-1], lens) + np.arange(bptr[-1])
    rows = np.repeat(np.arange(n), lens)
    bc = inv[cols[src]]
    order = np.lexsort((bc, rows))
    return bptr.astype(np.int32), bc[order].astype(np.int32), vals[src][order]


def levels(ptr, cols, upper=False):
    ptr, cols = _i(ptr), _i(cols)
    lev = np.empty(len(ptr) - 1, np.int32)
    nl = lib().or_levels(len(ptr) - 1, _pi(ptr), _pi(cols), 1 if upper else 0, _pi(lev))
    return lev, nl


def _solve(fn, ptr, cols, vals, pc, b, x0, rtol, atol, maxit):
    ptr, cols, vals, b = _i(ptr), _i(cols), _d(vals), _d(b)
    x = _d(x0).copy() if x0 is not None else np.zeros(len(b))
    hist = np.zeros(maxit + 3)
    info = OrInfo()
    rc = fn(len(b), _pi(ptr), _pi(cols), _pd(vals), pc.h if pc is not None else None, _pd(b), _pd(x), rtol, atol,
            maxit, _pd(hist), len(hist), C.byref(info))
    assert rc == 0
    return x, {"iterations": info.iterations, "initial_residual": info.initial_residual,
               "final_residual": info.final_residual, "history": hist[: info.history_len].tolist(),
               "restarts": info.restarts}


def cg(ptr, cols, vals, pc, b, x0=None, rtol=1e-6, atol=1e-6, maxit=1000):
    return _solve(lib().or_cg, ptr, cols, vals, pc, b, x0, rtol, atol, maxit)


def bicgstab(ptr, cols, vals, pc, b, x0=None, rtol=1e-6, atol=1e-6, maxit=1000):
    return _solve(lib().or_bicgstab, ptr, cols, vals, pc, b, x0, rtol, atol, maxit)
