"""FaceConstraints (fvm/bcs/mod.rs:7-57): one (lhs, value) pair per boundary
face, indexed by face id, (0, 0) until set.  `as_bc()` gives what
`assemble` takes as the boundary condition: the pair of arrays (bndi, bnde)
over the boundary faces, in face order.  For a scalar unknown: Dirichlet
u = g is (0, g); zero gradient is (1, 0).
"""
from __future__ import annotations

import numpy as np


class FaceConstraints:
    def __init__(self, mesh):
        self.face_start = int(mesh.n_faces - mesh.n_boundary_faces)
        nb = int(mesh.n_boundary_faces)
        self.lhs = np.zeros(nb)
        self.value = np.zeros(nb)

    @classmethod
    def from_mesh(cls, mesh) -> "FaceConstraints":
        return cls(mesh)

    def _slot(self, face) -> np.ndarray | int:
        f = np.asarray(face, dtype=np.int64) - self.face_start
        if np.any(f < 0) or np.any(f >= len(self.lhs)):
            raise IndexError("FaceConstraints: not a boundary face")  # the reference asserts
        return f if f.ndim else int(f)

    def __getitem__(self, face):
        k = self._slot(face)
        return self.lhs[k], self.value[k]

    def __setitem__(self, face, pair):
        k = self._slot(face)
        self.lhs[k], self.value[k] = pair

    def as_bc(self):
        return self.lhs, self.value
