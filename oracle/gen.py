"""The oracle's own synthetic inputs -- TEST AND CPU-BASELINE INFRASTRUCTURE ONLY.

Seeded square / cube meshes and their fields generated by oracle_mesh.c (the
reference's face numbering and geometry restated in C), without the product
library, so that the CPU reference arm never loads it.  The CPU suite checks
every array against the library's host builder bit for bit.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import lib as _lib

P = C.POINTER
dp, ip = P(C.c_double), P(C.c_int32)
_done = False


def lib():
    global _done
    L = _lib()
    if not _done:
        L.or_mesh_generate.argtypes = [C.c_int, C.c_int, C.c_double, C.c_uint64, P(C.c_void_p)]
        L.or_mesh_generate.restype = C.c_int
        L.or_mesh_free.argtypes = [C.c_void_p]
        L.or_mesh_free.restype = None
        L.or_mesh_sizes.argtypes = [C.c_void_p, P(C.c_int64)]
        L.or_mesh_sizes.restype = None
        L.or_mesh_arrays.argtypes = [C.c_void_p, dp, ip, ip, ip, ip, dp, dp, dp, dp, dp]
        L.or_mesh_arrays.restype = None
        L.or_fields_generate.argtypes = [C.c_void_p, C.c_uint64, C.c_double, C.c_double, dp, C.c_double, C.c_int,
                                         dp, dp, dp]
        L.or_fields_generate.restype = C.c_int
        _done = True
    return L


class Mesh:
    """A generated mesh with the attributes oracle.assemble reads (the same
    names and layouts as the library's host mesh)."""

    def __init__(self, dim: int, n: int, jitter: float, seed: int):
        h = C.c_void_p()
        rc = lib().or_mesh_generate(dim, n, jitter, seed, C.byref(h))
        if rc != 0:
            raise RuntimeError(f"or_mesh_generate failed: {rc}")
        self._h = h
        s = (C.c_int64 * 6)()
        lib().or_mesh_sizes(h, s)
        self.dim, self.n_nodes, self.n_cells, self.n_faces, self.n_boundary_faces, ncf = (int(v) for v in s)
        d, N, F = self.dim, self.n_cells, self.n_faces
        self.nodes = np.empty((self.n_nodes, d))
        self.cell_face_ptr = np.empty(N + 1, np.int32)
        self.cell_faces = np.empty(ncf, np.int32)
        self.face_owner = np.empty(F, np.int32)
        self.face_neighbor = np.empty(F, np.int32)
        self.face_area = np.empty(F)
        self.face_normal = np.empty((F, d))
        self.face_center = np.empty((F, d))
        self.cell_center = np.empty((N, d))
        self.cell_volume = np.empty(N)
        pi = lambda a: a.ctypes.data_as(ip)  # noqa: E731
        pd = lambda a: a.ctypes.data_as(dp)  # noqa: E731
        lib().or_mesh_arrays(h, pd(self.nodes), pi(self.cell_face_ptr), pi(self.cell_faces), pi(self.face_owner),
                             pi(self.face_neighbor), pd(self.face_area), pd(self.face_normal), pd(self.face_center),
                             pd(self.cell_center), pd(self.cell_volume))

    @classmethod
    def square(cls, n: int, jitter: float = 0.0, seed: int = 0) -> "Mesh":
        return cls(2, n, jitter, seed)

    @classmethod
    def cube(cls, n: int, jitter: float = 0.0, seed: int = 0) -> "Mesh":
        return cls(3, n, jitter, seed)

    def fields(self, seed: int, kappa0: float = 1.0, sigma: float = 1.0, velocity=(0.0, 0.0, 0.0),
               source_const: float = 1.0, source_uniform: bool = False):
        kf, fl, sc = np.empty(self.n_faces), np.empty(self.n_faces), np.empty(self.n_cells)
        v = np.ascontiguousarray(np.asarray(velocity, dtype=np.float64)[: max(self.dim, 3)])
        pd = lambda a: a.ctypes.data_as(dp)  # noqa: E731
        rc = lib().or_fields_generate(self._h, seed, kappa0, sigma, pd(v), source_const, 1 if source_uniform else 0,
                                      pd(kf), pd(fl), pd(sc))
        if rc != 0:
            raise RuntimeError("or_fields_generate failed")
        return kf, fl, sc

    def __del__(self):
        if getattr(self, "_h", None):
            lib().or_mesh_free(self._h)
            self._h = None
