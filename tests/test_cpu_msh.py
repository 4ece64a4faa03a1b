"""The crate's own mesh format (Mesh::write / Mesh::read, core/mesh/io.rs:10-225)
and meshes given as explicit faces and cells, on the host.

- the writer's text equals the pure-Python restatement (oracle/mesh_ref.py),
  doubles printed as Rust's Display prints them
- read(write(m)) gives m back bit for bit; reading equals the restatement's
  add_face / add_cell + Mesh::compute
- the reference's read_write_square_mesh test (io.rs:592-608) on square.su2
- malformed files fail with FV_ERR_INVALID, ghost entries with
  FV_ERR_UNSUPPORTED
"""
import math
from pathlib import Path

import numpy as np
import pytest
from conftest import reference_file

SQUARE_SU2 = reference_file("src/core/mesh/examples/square.su2")

_FIELDS = ("face_node_ptr", "face_nodes", "face_patch", "cell_face_ptr", "cell_faces", "face_owner",
           "face_neighbor", "face_area", "face_normal", "face_center", "cell_center", "cell_volume", "nodes")


def _same(a, b):
    assert (a.dim, a.n_nodes, a.n_faces, a.n_cells, a.n_boundary_faces) == \
        (b.dim, b.n_nodes, b.n_faces, b.n_cells, b.n_boundary_faces)
    for name in _FIELDS:
        x, y = getattr(a, name), getattr(b, name)
        assert x.shape == y.shape and x.tobytes() == y.tobytes(), name


def _lists(m):
    fn = [list(m.face_nodes[m.face_node_ptr[f]:m.face_node_ptr[f + 1]]) for f in range(m.n_faces)]
    cf = [list(m.cell_faces[m.cell_face_ptr[c]:m.cell_face_ptr[c + 1]]) for c in range(m.n_cells)]
    return fn, [int(p) for p in m.face_patch], cf


def _meshes(fv):
    return [fv.Mesh.square(6, 0.25, 3), fv.Mesh.cube(3, 0.15, 4), fv.Mesh.square(1, 0.0, 0)]


def test_rust_display_of_doubles():
    from oracle.mesh_ref import rust_f64
    cases = {1.0: "1", 0.1: "0.1", 1e-7: "0.0000001", 1e21: "1000000000000000000000", -0.0: "-0", 2.5: "2.5",
             100.0: "100", 0.30000000000000004: "0.30000000000000004", -1.25e-3: "-0.00125",
             math.inf: "inf", -math.inf: "-inf"}
    for x, want in cases.items():
        assert rust_f64(x) == want, x
    rng = np.random.default_rng(1)
    for x in np.concatenate([rng.standard_normal(200), rng.standard_normal(50) * 1e-12, rng.standard_normal(50) * 1e17]):
        assert float(rust_f64(float(x))) == float(x)


def test_writer_text_equals_restatement(fv, tmp_path):
    from oracle import mesh_ref
    for k, m in enumerate(_meshes(fv)):
        path = tmp_path / f"m{k}.msh"
        names = ["wall", "inlet"] if k == 0 else None
        m.write(path, names)
        fn, fp, cf = _lists(m)
        want = mesh_ref.write_msh(m.dim, m.nodes.tolist(), fn, fp, cf, names)
        assert path.read_text() == want


def test_writer_prints_extreme_coordinates_like_rust(fv, tmp_path):
    """Node coordinates far from 1 (tiny, huge, negative zero) in one small mesh."""
    from oracle import mesh_ref
    m = fv.Mesh.square(2, 0.0, 0)
    nodes = m.nodes.copy()
    nodes[:, 0] *= np.array([1e-300, 1e22, 3.0, 1.0 / 3.0, 7e-9, 1.0, 123456789.0, 2.0 ** -30, 1e15])
    nodes[0, 1] = -0.0
    fn, fp, cf = _lists(m)
    fptr = np.concatenate([[0], np.cumsum([len(x) for x in fn])]).astype(np.int32)
    cptr = np.concatenate([[0], np.cumsum([len(x) for x in cf])]).astype(np.int32)
    m2 = fv.Mesh.from_faces(2, nodes, fptr, np.concatenate(fn), fp, cptr, np.concatenate(cf))
    path = tmp_path / "x.msh"
    m2.write(path)
    assert path.read_text() == mesh_ref.write_msh(2, nodes.tolist(), fn, fp, cf)
    back = fv.Mesh.read(path)
    assert back.nodes.tobytes() == nodes.tobytes()


def test_read_write_round_trip(fv, tmp_path):
    for k, m in enumerate(_meshes(fv)):
        path = tmp_path / f"r{k}.msh"
        m.write(path)
        _same(fv.Mesh.read(path), m)
        _same(fv.Mesh.read(path, dim=m.dim), m)


def test_reader_equals_restatement(fv, tmp_path):
    from oracle import mesh_ref
    m = fv.Mesh.square(5, 0.3, 9)
    path = tmp_path / "s.msh"
    m.write(path)
    dim, nodes, fnodes, tags, cells = mesh_ref.read_msh(path.read_text())
    ref = mesh_ref.build_topology(dim, nodes, fnodes, tags, cells)
    got = fv.Mesh.read(path)
    assert [list(x) for x in fnodes] == _lists(got)[0]
    assert list(got.face_owner) == ref["face_owner"] and list(got.face_neighbor) == ref["face_neighbor"]
    for key in ("face_area", "face_normal", "face_center", "cell_center", "cell_volume"):
        assert np.array_equal(getattr(got, key), np.array(ref[key])), key


def test_from_faces_equals_element_build(fv):
    """Feeding a mesh's own faces and cells back gives the same mesh (owner = first listing cell)."""
    for m in _meshes(fv):
        m2 = fv.Mesh.from_faces(m.dim, m.nodes, m.face_node_ptr, m.face_nodes, m.face_patch, m.cell_face_ptr,
                                m.cell_faces)
        _same(m2, m)


@pytest.mark.skipif(SQUARE_SU2 is None, reason="FV_REFERENCE_DIR unset: reference checkout not available")
def test_reference_read_write_square_mesh(fv, tmp_path):
    """io.rs:592-608: square.su2 -> write -> read; 121 nodes, 220 faces, 100 cells,
    total volume 1 and a closed boundary within 10 eps, before and after."""
    def check(m):
        assert m.n_nodes == 121 and m.n_faces == 220 and m.n_cells == 100
        tv = 0.0
        for v in m.cell_volume:
            tv += v
        assert abs(tv - 1.0) < np.finfo(float).eps * 10
        sf = np.zeros(2)
        for f in range(m.n_faces):
            if m.face_patch[f] >= 0:
                sf += m.face_normal[f] * m.face_area[f]
        assert np.linalg.norm(sf) < np.finfo(float).eps * 10
    m = fv.Mesh.read_su2(SQUARE_SU2)
    check(m)
    path = tmp_path / "square.msh"
    m.write(path)
    m2 = fv.Mesh.read(path)
    check(m2)
    _same(m2, m)


def test_malformed_files(fv, tmp_path):
    from fvb200._lib import FvError
    m = fv.Mesh.square(2, 0.0, 0)
    good = tmp_path / "g.msh"
    m.write(good)
    text = good.read_text()
    lines = text.splitlines()
    fi = lines.index(f"NFACES={m.n_faces}") + 1
    ci = lines.index(f"NCELLS={m.n_cells}") + 1
    bad = {
        "dimension": (text, 3, "FV_ERR_INVALID"),
        "tag": ("\n".join(lines[:fi] + [lines[fi].replace(" - 0 -", " x 0 -")] + lines[fi + 1:]), 0,
                "FV_ERR_INVALID"),
        "long face": ("\n".join(lines[:fi] + ["65 " + " ".join(["0"] * 65) + " - 0 -"] + lines[fi + 1:]), 0,
                      "FV_ERR_INVALID"),
        "remote cell": ("\n".join(lines[:ci] + [lines[ci][:-1] + "1"] + lines[ci + 1:]), 0, "FV_ERR_UNSUPPORTED"),
        "node index": ("\n".join(lines[:fi] + ["2 0 999 - 0 -"] + lines[fi + 1:]), 0, "FV_ERR_INVALID"),
    }
    assert lines[fi].endswith(" - 0 -") and lines[ci].endswith(" -")
    for name, (t, dim, want) in bad.items():
        p = tmp_path / f"{name.replace(' ', '_')}.msh"
        p.write_text(t)
        with pytest.raises(FvError) as ei:
            fv.Mesh.read(p, dim=dim)
        assert want in str(ei.value), name
