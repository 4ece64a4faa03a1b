"""Mesh built on the device (fv_mesh_build_*) against the host builder.

The host builder (fv_host_mesh_from_elements) is pinned to the pure-Python
restatement of Mesh::read_su2 + Mesh::compute and to the reference's
square.su2 known answer by the CPU tests; here every array of the device
build must equal it bit for bit:
- face numbering, face node lists, patches, owner/neighbour, cell faces
- face area / normal / centre, cell centre / volume
on triangles, tetrahedra, a triangle+quad mix with four markers in
scrambled order, hexahedra, elements in shuffled order, an SU2 file, and
the 1.5M-cell cube.  The device mesh then assembles (Corrected scheme, so
the gradient coefficients built with it are used too) exactly the system the
host-built mesh assembles.  Bad input fails with FV_ERR_INVALID as on the
host.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

_FIELDS = ("face_node_ptr", "face_nodes", "face_patch", "cell_face_ptr", "cell_faces", "face_owner",
           "face_neighbor", "face_area", "face_normal", "face_center", "cell_center", "cell_volume", "nodes")


def _same_mesh(a, b):
    assert (a.dim, a.n_nodes, a.n_faces, a.n_cells, a.n_boundary_faces) == \
        (b.dim, b.n_nodes, b.n_faces, b.n_cells, b.n_boundary_faces)
    for name in _FIELDS:
        x, y = getattr(a, name), getattr(b, name)
        assert x.dtype == y.dtype and x.shape == y.shape and x.tobytes() == y.tobytes(), name


def _both(fv, *args, **kw):
    host = fv.Mesh.from_elements(*args, **kw)
    dev = fv.Mesh.from_elements(*args, on_device=True, **kw)
    _same_mesh(host, dev)
    return host, dev


def _grid_nodes(n, dim, jitter, rng):
    ax = np.linspace(0.0, 1.0, n + 1)
    pts = np.stack(np.meshgrid(*([ax] * dim), indexing="ij"), -1).reshape(-1, dim)[:, ::-1].copy()
    inner = np.all((pts > 0) & (pts < 1), axis=1)
    pts[inner] += rng.uniform(-jitter, jitter, (inner.sum(), dim)) / n
    return pts


def _mixed_2d(n, rng):
    """Quads where (i + j) % 3 == 0, two triangles elsewhere; markers 2, 0, 1, 3 for the
    bottom, right, top and left sides (not in input order)."""
    nodes = _grid_nodes(n, 2, 0.25, rng)
    v = lambda i, j: j * (n + 1) + i  # noqa: E731
    el = []
    for j in range(n):
        for i in range(n):
            a, b, c, d = v(i, j), v(i + 1, j), v(i + 1, j + 1), v(i, j + 1)
            el += [(9, [a, b, c, d])] if (i + j) % 3 == 0 else [(5, [a, b, c]), (5, [a, c, d])]
    bf = []
    for i in range(n):
        bf += [([v(i, 0), v(i + 1, 0)], 2), ([v(n, i), v(n, i + 1)], 0), ([v(i + 1, n), v(i, n)], 1),
               ([v(0, i + 1), v(0, i)], 3)]
    return nodes, el, bf


def _hex_3d(n, rng):
    nodes = _grid_nodes(n, 3, 0.2, rng)
    v = lambda i, j, k: (k * (n + 1) + j) * (n + 1) + i  # noqa: E731
    el = []
    for k in range(n):
        for j in range(n):
            for i in range(n):
                el.append((12, [v(i, j, k), v(i + 1, j, k), v(i + 1, j + 1, k), v(i, j + 1, k),
                                v(i, j, k + 1), v(i + 1, j, k + 1), v(i + 1, j + 1, k + 1), v(i, j + 1, k + 1)]))
    bf = []
    for a in range(n):
        for b in range(n):
            bf += [([v(0, a, b), v(0, a + 1, b), v(0, a + 1, b + 1), v(0, a, b + 1)], 4),
                   ([v(n, a, b), v(n, a + 1, b), v(n, a + 1, b + 1), v(n, a, b + 1)], 1),
                   ([v(a, 0, b), v(a + 1, 0, b), v(a + 1, 0, b + 1), v(a, 0, b + 1)], 5),
                   ([v(a, n, b), v(a + 1, n, b), v(a + 1, n, b + 1), v(a, n, b + 1)], 0),
                   ([v(a, b, 0), v(a + 1, b, 0), v(a + 1, b + 1, 0), v(a, b + 1, 0)], 3),
                   ([v(a, b, n), v(a + 1, b, n), v(a + 1, b + 1, n), v(a, b + 1, n)], 2)]
    return nodes, el, bf


def _arrays(dim, nodes, el, bf):
    kinds = np.array([k for k, _ in el], np.int32)
    eptr = np.concatenate([[0], np.cumsum([len(x) for _, x in el])]).astype(np.int32)
    en = np.array([q for _, x in el for q in x], np.int32)
    bptr = np.concatenate([[0], np.cumsum([len(x) for x, _ in bf])]).astype(np.int32)
    bn = np.array([q for x, _ in bf for q in x], np.int32)
    bm = np.array([mk for _, mk in bf], np.int32)
    return dim, nodes, kinds, eptr, en, bptr, bn, bm


@pytest.mark.parametrize("n,jitter", [(1, 0.0), (9, 0.2), (40, 0.3)])
def test_square_equals_host(fv, n, jitter):
    _same_mesh(fv.Mesh.square(n, jitter, 11), fv.Mesh.square(n, jitter, 11, on_device=True))


@pytest.mark.parametrize("n", [1, 5, 12])
def test_cube_equals_host(fv, n):
    _same_mesh(fv.Mesh.cube(n, 0.15, 4), fv.Mesh.cube(n, 0.15, 4, on_device=True))


def test_mixed_triangles_and_quads_with_scrambled_markers(fv):
    rng = np.random.default_rng(5)
    host, dev = _both(fv, *_arrays(2, *_mixed_2d(13, rng)))
    assert set(np.unique(host.face_patch)) == {-1, 0, 1, 2, 3}
    # boundary faces by ascending marker after the interior faces
    p = host.face_patch[host.n_interior_faces():]
    assert np.all(np.diff(p) >= 0)


def test_hexahedra(fv):
    rng = np.random.default_rng(6)
    host, dev = _both(fv, *_arrays(3, *_hex_3d(6, rng)))
    assert host.n_cells == 216 and host.n_boundary_faces == 6 * 36


def test_shuffled_elements_and_boundary_list(fv):
    """Discovery order follows the element order: a shuffled list numbers faces differently, on both builders."""
    rng = np.random.default_rng(7)
    nodes, el, bf = _mixed_2d(11, rng)
    el = [el[i] for i in rng.permutation(len(el))]
    bf = [bf[i] for i in rng.permutation(len(bf))]
    _both(fv, *_arrays(2, nodes, el, bf))
    m = fv.Mesh.cube(4, 0.1, 2)
    ne = m.n_cells
    perm = rng.permutation(ne)
    cube_el = []
    for c in range(ne):  # rebuild each tet's nodes from the host mesh (any order of its four nodes)
        faces = m.cell_faces[m.cell_face_ptr[c]:m.cell_face_ptr[c + 1]]
        vs = sorted({int(q) for f in faces for q in m.face_nodes[m.face_node_ptr[f]:m.face_node_ptr[f + 1]]})
        cube_el.append((10, vs))
    cube_el = [cube_el[i] for i in perm]
    bfaces = [(list(m.face_nodes[m.face_node_ptr[f]:m.face_node_ptr[f + 1]]), 0)
              for f in range(m.n_interior_faces(), m.n_faces)]
    _both(fv, *_arrays(3, m.nodes.copy(), cube_el, bfaces))


def test_su2_file_equals_host(fv, tmp_path):
    rng = np.random.default_rng(8)
    nodes, el, bf = _mixed_2d(7, rng)
    lines = ["NDIME= 2", f"NELEM= {len(el)}"]
    lines += [" ".join(str(q) for q in [k, *x, i]) for i, (k, x) in enumerate(el)]
    lines += [f"NPOIN= {len(nodes)}"] + [f"{float(p[0])!r} {float(p[1])!r} {i}" for i, p in enumerate(nodes)]
    lines += ["NMARK= 4"]
    for mk in range(4):
        side = [x for x, m_ in bf if m_ == mk]
        lines += [f"MARKER_TAG= side{mk}", f"MARKER_ELEMS= {len(side)}"] + [f"3 {a} {b}" for a, b in side]
    path = tmp_path / "mixed.su2"
    path.write_text("\n".join(lines) + "\n")
    host = fv.Mesh.read_su2(path)
    dev = fv.Mesh.read_su2(path, on_device=True)
    _same_mesh(host, dev)
    assert host.n_cells == len(el) and np.array_equal(host.nodes, nodes)
    assert np.isfinite(host.face_normal).all() and abs(host.cell_volume.sum() - 1.0) < 1e-12


def test_large_cube_equals_host(fv):
    _same_mesh(fv.Mesh.cube(64, 0.15, 1), fv.Mesh.cube(64, 0.15, 1, on_device=True))


@pytest.mark.parametrize("kind", ["2d", "3d"])
def test_device_mesh_assembles_the_same_system(fv, kind):
    if kind == "2d":
        mh, md = fv.Mesh.square(24, 0.25, 3), fv.Mesh.square(24, 0.25, 3, on_device=True)
    else:
        mh, md = fv.Mesh.cube(7, 0.15, 3), fv.Mesh.cube(7, 0.15, 3, on_device=True)
    kf, fl, sc = mh.fields(3, 0.3, 0.5, velocity=(1.0, 0.5, 0.25))
    nb = mh.n_boundary_faces
    bc = (np.zeros(nb), np.linspace(0.0, 1.0, nb))
    u = np.sin(2.0 * mh.cell_center[:, 0]) + mh.cell_center[:, 1]
    out = []
    for m in (mh, md):
        g = fv.DistributedVector.from_size(m.n_cells * m.dim)
        fv.compute_gradients(g, u, bc, m)
        eq = fv.convection(fv.Upwind(fl), fl) - fv.laplacian(fv.Corrected(g, 1.0), kf) - fv.source(sc)
        A, b = fv.assemble(eq, bc, m)
        out.append((g.numpy(), *A.to_csr(), b.numpy()))
    for x, y in zip(*out):
        assert np.array_equal(x, y)


def test_bad_input_is_rejected_as_on_the_host(fv):
    from fvb200._lib import FvError
    rng = np.random.default_rng(9)
    dim, nodes, kinds, eptr, en, bptr, bn, bm = _arrays(2, *_mixed_2d(4, rng))
    cases = {
        "missing marker": (kinds, en, bptr[:-4], bn[:-8], bm[:-4]),
        "unknown kind": (np.where(np.arange(len(kinds)) == 3, 7, kinds).astype(np.int32), en, bptr, bn, bm),
        "node out of range": (kinds, np.where(np.arange(len(en)) == 5, len(nodes) + 3, en).astype(np.int32),
                              bptr, bn, bm),
    }
    for name, (k, e, bp, bnn, bmm) in cases.items():
        for on_device in (False, True):
            with pytest.raises(FvError) as ei:
                fv.Mesh.from_elements(dim, nodes, k, eptr, e, bp, bnn, bmm, on_device=on_device)
            assert "FV_ERR_INVALID" in str(ei.value), (name, on_device)


def test_msh_file_and_explicit_faces_on_device(fv, tmp_path):
    """Mesh::read of the crate's own format, and explicit faces/cells: device build == host build."""
    rng = np.random.default_rng(10)
    meshes = [fv.Mesh.square(9, 0.2, 5), fv.Mesh.cube(4, 0.15, 6),
              fv.Mesh.from_elements(*_arrays(2, *_mixed_2d(6, rng))), fv.Mesh.from_elements(*_arrays(3, *_hex_3d(3, rng)))]
    for k, m in enumerate(meshes):
        path = tmp_path / f"m{k}.msh"
        m.write(path)
        host = fv.Mesh.read(path)
        dev = fv.Mesh.read(path, on_device=True)
        _same_mesh(host, m)
        _same_mesh(dev, m)
        dev2 = fv.Mesh.from_faces(m.dim, m.nodes, m.face_node_ptr, m.face_nodes, m.face_patch, m.cell_face_ptr,
                                  m.cell_faces, on_device=True)
        _same_mesh(dev2, m)


def test_msh_errors_on_device(fv, tmp_path):
    from fvb200._lib import FvError
    m = fv.Mesh.square(3, 0.0, 0)
    path = tmp_path / "g.msh"
    m.write(path)
    lines = path.read_text().splitlines()
    ci = lines.index(f"NCELLS={m.n_cells}") + 1
    fi = lines.index(f"NFACES={m.n_faces}") + 1
    cases = {"remote": ("\n".join(lines[:ci] + [lines[ci][:-1] + "1"] + lines[ci + 1:]), "FV_ERR_UNSUPPORTED"),
             "node": ("\n".join(lines[:fi] + ["2 0 999 - 0 -"] + lines[fi + 1:]), "FV_ERR_INVALID"),
             # an interior face that no cell lists any more: its cell now lists face 0 twice
             "open": ("\n".join(lines[:ci] + [" ".join([lines[ci].split(" ")[0], "0", "0"] + lines[ci].split(" ")[3:])]
                                + lines[ci + 1:]), "FV_ERR_INVALID")}
    for name, (text, want) in cases.items():
        p = tmp_path / f"{name}.msh"
        p.write_text(text)
        for on_device in (False, True):
            with pytest.raises(FvError) as ei:
                fv.Mesh.read(p, on_device=on_device)
            assert want in str(ei.value), (name, on_device)
