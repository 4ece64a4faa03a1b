"""Host mesh (stand-in for the reference's Mesh<DIM> after Mesh::compute) and
its device upload.

Numbering and geometry follow core/mesh/io.rs:364-533 (SU2 reading,
compute_vtk_faces), core/mesh/mod.rs:451-529 (add_face / add_cell) and
core/mesh/compute.rs:12-375; the work is done in C++ (csrc/meshgen.cpp).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import HostMesh_, MeshDesc, check, exiting, lib

VTK_TRIANGLE, VTK_QUAD, VTK_TETRA, VTK_HEXAHEDRON = 5, 9, 10, 12


def _view(ptr, n, dtype):
    if n == 0:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(int(n),)).view(dtype)


class Mesh:
    """A computed unstructured mesh with reference-identical numbering.

    Attributes are numpy arrays (views owned by this object):
    face_owner, face_neighbor (-1 = boundary), face_area, face_normal,
    face_center, cell_center, cell_volume, cell_face_ptr, cell_faces, nodes, ...
    """

    def __init__(self, handle):
        self._h = handle
        m = handle.contents
        self.dim = int(m.dim)
        d = self.dim
        self.n_nodes = int(m.n_nodes)
        self.n_faces = int(m.n_faces)
        self.n_cells = int(m.n_cells)
        self.n_boundary_faces = int(m.n_boundary_faces)
        F, N = self.n_faces, self.n_cells
        self.nodes = _view(m.nodes, self.n_nodes * d, np.float64).reshape(-1, d)
        self.face_node_ptr = _view(m.face_node_ptr, F + 1, np.int32)
        self.face_nodes = _view(m.face_nodes, int(self.face_node_ptr[-1]), np.int32)
        self.face_patch = _view(m.face_patch, F, np.int32)
        self.cell_face_ptr = _view(m.cell_face_ptr, N + 1, np.int32)
        self.cell_faces = _view(m.cell_faces, int(self.cell_face_ptr[-1]), np.int32)
        self.face_owner = _view(m.face_owner, F, np.int32)
        self.face_neighbor = _view(m.face_neighbor, F, np.int32)
        self.face_area = _view(m.face_area, F, np.float64)
        self.face_normal = _view(m.face_normal, F * d, np.float64).reshape(-1, d)
        self.face_center = _view(m.face_center, F * d, np.float64).reshape(-1, d)
        self.cell_center = _view(m.cell_center, N * d, np.float64).reshape(-1, d)
        self.cell_volume = _view(m.cell_volume, N, np.float64)
        self._device = {}

    def __del__(self):
        try:
            if exiting():  # module globals may already be gone at interpreter teardown
                return
            for dm in self._device.values():
                dm.close()
            if self._h:
                lib().fv_host_mesh_free(self._h)
                self._h = None
        except Exception:
            pass

    # -- construction ------------------------------------------------------
    # Every constructor takes on_device: False builds faces and geometry on the
    # host (fv_host_mesh_*); True builds them on the current GPU
    # (fv_mesh_build_*), keeps that device mesh for assemble and reads the same
    # arrays back into this object.
    @classmethod
    def _built_on_device(cls, call, what, stream) -> "Mesh":
        import torch

        from .streams import stream_handle
        dev = torch.cuda.current_device()
        h = C.c_void_p()
        out = C.POINTER(HostMesh_)()
        check(call(stream_handle(stream), C.byref(h), C.byref(out)), what)
        m = cls(out)
        m._device[dev] = DeviceMesh.adopt(m, h)
        return m

    @classmethod
    def from_elements(cls, dim, nodes, elem_kind, elem_node_ptr, elem_nodes, bface_node_ptr=None,
                      bface_nodes=None, bface_marker=None, on_device: bool = False, stream=None) -> "Mesh":
        nodes = np.ascontiguousarray(nodes, dtype=np.float64).reshape(-1)
        ek = np.ascontiguousarray(elem_kind, dtype=np.int32)
        ep = np.ascontiguousarray(elem_node_ptr, dtype=np.int32)
        en = np.ascontiguousarray(elem_nodes, dtype=np.int32)
        if bface_node_ptr is None:
            bp = np.zeros(1, np.int32)
            bn = np.zeros(1, np.int32)
            bm = np.zeros(1, np.int32)
            nb = 0
        else:
            bp = np.ascontiguousarray(bface_node_ptr, dtype=np.int32)
            bn = np.ascontiguousarray(bface_nodes, dtype=np.int32)
            bm = np.ascontiguousarray(bface_marker, dtype=np.int32)
            nb = len(bm)
        P = lambda a, t: a.ctypes.data_as(C.POINTER(t))  # noqa: E731
        if on_device:
            return cls._built_on_device(
                lambda st, h, o: lib().fv_mesh_build_elements(
                    dim, len(nodes) // dim, P(nodes, C.c_double), len(ek), P(ek, C.c_int32), P(ep, C.c_int32),
                    P(en, C.c_int32), nb, P(bp, C.c_int32), P(bn, C.c_int32), P(bm, C.c_int32), st, h, o),
                "Mesh.from_elements(on_device)", stream)
        out = C.POINTER(HostMesh_)()
        check(lib().fv_host_mesh_from_elements(dim, len(nodes) // dim, P(nodes, C.c_double), len(ek),
                                               P(ek, C.c_int32), P(ep, C.c_int32), P(en, C.c_int32), nb,
                                               P(bp, C.c_int32), P(bn, C.c_int32), P(bm, C.c_int32),
                                               C.byref(out)), "Mesh.from_elements")
        return cls(out)

    @classmethod
    def read_su2(cls, path, dim: int = 0, on_device: bool = False, stream=None) -> "Mesh":
        """Mesh::read_su2 (core/mesh/io.rs:489-533); dim 0 = NDIME of the file."""
        if on_device:
            return cls._built_on_device(lambda st, h, o: lib().fv_mesh_build_su2(str(path).encode(), int(dim), st, h, o),
                                        "Mesh.read_su2(on_device)", stream)
        out = C.POINTER(HostMesh_)()
        check(lib().fv_host_mesh_read_su2(str(path).encode(), int(dim), C.byref(out)), "Mesh.read_su2")
        return cls(out)

    @classmethod
    def from_faces(cls, dim, nodes, face_node_ptr, face_nodes, face_patch, cell_face_ptr, cell_faces,
                   on_device: bool = False, stream=None) -> "Mesh":
        """Explicit faces and cells (add_face / add_cell, core/mesh/mod.rs:451-529) + Mesh::compute.
        face_patch: boundary tag per face, -1 untagged; tagged faces last."""
        nodes = np.ascontiguousarray(nodes, dtype=np.float64).reshape(-1)
        fp = np.ascontiguousarray(face_node_ptr, dtype=np.int32)
        fn = np.ascontiguousarray(face_nodes, dtype=np.int32)
        pa = np.ascontiguousarray(face_patch, dtype=np.int32)
        cp = np.ascontiguousarray(cell_face_ptr, dtype=np.int32)
        cf = np.ascontiguousarray(cell_faces, dtype=np.int32)
        P = lambda a, t: a.ctypes.data_as(C.POINTER(t))  # noqa: E731
        I = lambda a: P(a, C.c_int32)  # noqa: E731
        args = (dim, len(nodes) // dim, P(nodes, C.c_double), len(pa), I(fp), I(fn), I(pa), len(cp) - 1, I(cp), I(cf))
        if on_device:
            return cls._built_on_device(lambda st, h, o: lib().fv_mesh_build_faces(*args, st, h, o),
                                        "Mesh.from_faces(on_device)", stream)
        out = C.POINTER(HostMesh_)()
        check(lib().fv_host_mesh_from_faces(*args, C.byref(out)), "Mesh.from_faces")
        return cls(out)

    @classmethod
    def read(cls, path, dim: int = 0, on_device: bool = False, stream=None) -> "Mesh":
        """Mesh::read (core/mesh/io.rs:68-225): the crate's own .msh format; dim 0 = NDIME of the file."""
        if on_device:
            return cls._built_on_device(lambda st, h, o: lib().fv_mesh_build_msh(str(path).encode(), int(dim), st, h, o),
                                        "Mesh.read(on_device)", stream)
        out = C.POINTER(HostMesh_)()
        check(lib().fv_host_mesh_read_msh(str(path).encode(), int(dim), C.byref(out)), "Mesh.read")
        return cls(out)

    def write(self, path, patch_names=None) -> None:
        """Mesh::write (core/mesh/io.rs:10-66); patch_names[p] names boundary tag p ("patch_<p>" otherwise)."""
        names = list(patch_names or [])
        arr = (C.c_char_p * max(len(names), 1))(*[str(x).encode() for x in names])
        check(lib().fv_host_mesh_write_msh(self._h, str(path).encode(), arr, len(names)), "Mesh.write")

    @classmethod
    def square(cls, n: int, jitter: float = 0.0, seed: int = 0, on_device: bool = False, stream=None) -> "Mesh":
        if on_device:
            return cls._built_on_device(lambda st, h, o: lib().fv_mesh_build_square(n, jitter, seed, st, h, o),
                                        "Mesh.square(on_device)", stream)
        out = C.POINTER(HostMesh_)()
        check(lib().fv_host_mesh_generate_square(n, jitter, seed, C.byref(out)), "Mesh.square")
        return cls(out)

    @classmethod
    def cube(cls, n: int, jitter: float = 0.0, seed: int = 0, on_device: bool = False, stream=None) -> "Mesh":
        if on_device:
            return cls._built_on_device(lambda st, h, o: lib().fv_mesh_build_cube(n, jitter, seed, st, h, o),
                                        "Mesh.cube(on_device)", stream)
        out = C.POINTER(HostMesh_)()
        check(lib().fv_host_mesh_generate_cube(n, jitter, seed, C.byref(out)), "Mesh.cube")
        return cls(out)

    # -- accessors mirroring the reference ---------------------------------
    def n_interior_faces(self) -> int:
        return self.n_faces - self.n_boundary_faces

    def boundary_faces(self) -> np.ndarray:
        return np.arange(self.n_interior_faces(), self.n_faces, dtype=np.int64)

    def cell_to_cell(self):
        """CSR of cell_to_cell with sorted rows (dmatrix.rs:38-50)."""
        rows = []
        for c in range(self.n_cells):
            s = {c}
            for f in self.cell_faces[self.cell_face_ptr[c]:self.cell_face_ptr[c + 1]]:
                nb = self.face_neighbor[f]
                if nb >= 0:
                    s.add(int(self.face_owner[f]) if nb == c else int(nb))
            rows.append(sorted(s))
        ptr = np.zeros(self.n_cells + 1, np.int32)
        ptr[1:] = np.cumsum([len(r) for r in rows])
        return ptr, np.array([c for r in rows for c in r], np.int32)

    # -- synthetic fields ---------------------------------------------------
    def fields(self, seed: int, kappa0: float = 1.0, sigma: float = 1.0, velocity=(0.0, 0.0, 0.0),
               source_const: float = 1.0, source_uniform: bool = False):
        """Seeded face diffusivity, face flux v.n and cell source (fv_host_fields_generate)."""
        kf = np.empty(self.n_faces)
        fl = np.empty(self.n_faces)
        sc = np.empty(self.n_cells)
        v = np.ascontiguousarray(np.asarray(velocity, dtype=np.float64)[: max(self.dim, 3)])
        Pd = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
        check(lib().fv_host_fields_generate(self._h, seed, kappa0, sigma, Pd(v), source_const,
                                            1 if source_uniform else 0, Pd(kf), Pd(fl), Pd(sc)),
              "Mesh.fields")
        return kf, fl, sc

    # -- device --------------------------------------------------------------
    def device(self, stream=None) -> "DeviceMesh":
        import torch
        dev = torch.cuda.current_device()
        if dev not in self._device:
            self._device[dev] = DeviceMesh(self, stream)
        return self._device[dev]


class DeviceMesh:
    """fv_mesh handle: geometry and cell->face table resident on one GPU."""

    def __init__(self, mesh: Mesh, stream=None):
        from .streams import stream_handle
        self.mesh = mesh
        d = MeshDesc()
        d.dim = mesh.dim
        d.n_cells = mesh.n_cells
        d.n_faces = mesh.n_faces
        d.n_boundary_faces = mesh.n_boundary_faces
        Pi = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))  # noqa: E731
        Pd = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
        d.face_owner = Pi(mesh.face_owner)
        d.face_neighbor = Pi(mesh.face_neighbor)
        d.face_area = Pd(mesh.face_area)
        d.face_center = Pd(mesh.face_center)
        d.cell_center = Pd(mesh.cell_center)
        d.cell_volume = Pd(mesh.cell_volume)
        # normals and the mesh-order cell faces: gradients and the Corrected scheme
        self._keep = []
        if getattr(mesh, "face_normal", None) is not None and getattr(mesh, "cell_faces", None) is not None:
            fn = np.ascontiguousarray(mesh.face_normal, dtype=np.float64)
            cp = np.ascontiguousarray(mesh.cell_face_ptr, dtype=np.int32)
            cf = np.ascontiguousarray(mesh.cell_faces, dtype=np.int32)
            self._keep = [fn, cp, cf]
            d.face_normal = Pd(fn)
            d.cell_face_ptr = Pi(cp)
            d.cell_faces = Pi(cf)
        self.handle = C.c_void_p()
        check(lib().fv_mesh_upload(C.byref(d), stream_handle(stream), C.byref(self.handle)), "fv_mesh_upload")

    @classmethod
    def adopt(cls, mesh: Mesh, handle: C.c_void_p) -> "DeviceMesh":
        """Wrap an fv_mesh built on the device (fv_mesh_build_*) for this mesh."""
        dm = cls.__new__(cls)
        dm.mesh = mesh
        dm._keep = []
        dm.handle = handle
        return dm

    def close(self):
        if self.handle:
            lib().fv_mesh_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            if exiting():  # module globals may already be gone at interpreter teardown
                return
            self.close()
        except Exception:
            pass
