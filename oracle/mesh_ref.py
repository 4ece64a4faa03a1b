"""Pure-Python restatement of the reference's mesh numbering and geometry --
TEST INFRASTRUCTURE ONLY, small meshes.

Used to pin the C++ mesh builder (csrc/meshgen.cpp) bit for bit:
  compute_vtk_faces ..... core/mesh/io.rs:364-486
  VTK face tables ....... core/mesh/vtk.rs:56-125
  add_face / add_cell ... core/mesh/mod.rs:451-529
  calc_face_data ........ core/mesh/compute.rs:267-321
  calc_cell_data ........ core/mesh/compute.rs:325-375
  orientation ........... core/mesh/compute.rs:97-131
Python floats are IEEE doubles and every expression below keeps the
reference's evaluation order, so the results are the Rust results.
"""
from __future__ import annotations

import math

VTK_FACES = {
    5: ([0, 1, 1, 2, 2, 0], [0, 2, 4, 6]),
    9: ([0, 1, 1, 2, 2, 3, 3, 0], [0, 2, 4, 6, 8]),
    10: ([0, 2, 1, 0, 1, 3, 1, 2, 3, 0, 3, 2], [0, 3, 6, 9, 12]),
    12: ([0, 3, 2, 1, 4, 5, 6, 7, 0, 1, 5, 4, 1, 2, 6, 5, 2, 3, 7, 6, 3, 0, 4, 7], [0, 4, 8, 12, 16, 20, 24]),
}


def compute_vtk_faces(elements, boundaries):
    """elements: list of (kind, [nodes]); boundaries: {sorted node tuple: marker}.
    Returns (face_nodes, face_boundaries, elem_faces) in final numbering."""
    face_nodes, bnd_face_nodes, elem_faces = [], [], []
    face_hash, face_boundaries, u2f = {}, [], []
    unique_b = set()
    for kind, n in elements:
        loc, starts = VTK_FACES[kind]
        ef = []
        for i in range(len(starts) - 1):
            fi = [n[loc[k]] for k in range(starts[i], starts[i + 1])]
            key = tuple(sorted(fi))
            if key in face_hash:
                fid = face_hash[key]
            else:
                fid = len(face_boundaries)
                bnd = boundaries.get(key)
                face_boundaries.append(bnd)
                face_hash[key] = fid
                if bnd is not None:
                    unique_b.add(bnd)
                    u2f.append(len(bnd_face_nodes))
                    bnd_face_nodes.append(fi)
                else:
                    u2f.append(len(face_nodes))
                    face_nodes.append(fi)
            ef.append(fid)
        elem_faces.append(ef)
    running = len(face_nodes)
    new_bnd = []
    for b in sorted(unique_b):
        for i in range(len(u2f)):
            if face_boundaries[i] == b:
                old = u2f[i]
                u2f[i] = running
                running += 1
                new_bnd.append(bnd_face_nodes[old])
    face_nodes = face_nodes + new_bnd
    elem_faces = [[u2f[f] for f in ef] for ef in elem_faces]
    fb = [None] * len(face_boundaries)
    for i, b in enumerate(face_boundaries):
        fb[u2f[i]] = b
    return face_nodes, fb, elem_faces


def _dot(a, b):
    x = 0.0
    for i in range(len(a)):
        x += a[i] * b[i]
    return x


def _face_data(dim, nodes, fn):
    size = len(fn)
    c = [0.0] * dim
    for n in fn:
        for d in range(dim):
            c[d] += nodes[n][d]
    c = [c[d] / float(size) for d in range(dim)]
    if dim == 2:
        n0, n1 = nodes[fn[0]], nodes[fn[1]]
        dn = [n1[0] - n0[0], n1[1] - n0[1]]
        dsn = [-dn[1], dn[0]]
        area = math.sqrt(_dot(dsn, dsn))
        return area, [dsn[0] / area, dsn[1] / area], [(n0[0] + n1[0]) * 0.5, (n0[1] + n1[1]) * 0.5]
    center = [0.0] * 3
    normal = [0.0] * 3
    area = 0.0
    for i in range(size):
        n0 = nodes[fn[i]]
        n1 = nodes[fn[0 if i == size - 1 else i + 1]]
        d0 = [n0[k] - c[k] for k in range(3)]
        d1 = [n1[k] - c[k] for k in range(3)]
        dsn = [d0[1] * d1[2] - d0[2] * d1[1], d0[2] * d1[0] - d0[0] * d1[2], d0[0] * d1[1] - d0[1] * d1[0]]
        dsn = [v * 0.5 for v in dsn]
        ai = math.sqrt(_dot(dsn, dsn))
        area += ai
        normal = dsn
        for k in range(3):
            center[k] += ((((n0[k] + n1[k]) + c[k]) * 1.0) / 3.0) * ai
    return area, [v / area for v in normal], [v / area for v in center]


def build(dim, nodes, elements, boundaries):
    """Mesh::read_su2 + Mesh::compute for a small element list."""
    face_nodes, fbnd, elem_faces = compute_vtk_faces(elements, boundaries)
    return build_topology(dim, nodes, face_nodes, fbnd, elem_faces)


def build_topology(dim, nodes, face_nodes, fbnd, elem_faces):
    """add_face / add_cell (mod.rs:451-529) + Mesh::compute for explicit faces
    (fbnd: tag or None per face) and cells (lists of faces)."""
    F = len(face_nodes)
    owner, neigh = [-1] * F, [-1] * F
    for c, ef in enumerate(elem_faces):
        for f in ef:
            if owner[f] < 0:
                owner[f] = c
            elif fbnd[f] is None and neigh[f] < 0:
                neigh[f] = c
    area, normal, fcenter = [], [], []
    for fn in face_nodes:
        a, n, c = _face_data(dim, nodes, fn)
        area.append(a)
        normal.append(n)
        fcenter.append(c)
    vdiv, cmul, cdiv = (2.0, 2.0, 3.0) if dim == 2 else (3.0, 3.0, 4.0)
    ccenter, volume = [], []
    for ef in elem_faces:
        ave = [0.0] * dim
        for f in ef:
            for d in range(dim):
                ave[d] += fcenter[f][d]
        ave = [v / float(len(ef)) for v in ave]
        ctr = [0.0] * dim
        vol = 0.0
        for f in ef:
            dfc = [fcenter[f][d] - ave[d] for d in range(dim)]
            h = abs(_dot(dfc, normal[f]))
            vi = h * area[f] / vdiv
            for d in range(dim):
                ctr[d] += ((fcenter[f][d] * cmul + ave[d]) / cdiv) * vi
            vol += vi
        volume.append(vol)
        ccenter.append([v / vol for v in ctr])
    for f in range(F):
        ip = ccenter[owner[f]]
        if _dot(normal[f], [fcenter[f][d] - ip[d] for d in range(dim)]) < 0.0:
            normal[f] = [v * -1.0 for v in normal[f]]
    return dict(face_nodes=face_nodes, face_patch=fbnd, cell_faces=elem_faces, face_owner=owner,
                face_neighbor=neigh, face_area=area, face_normal=normal, face_center=fcenter,
                cell_center=ccenter, cell_volume=volume)


def read_su2(text):
    """Minimal SU2 reader (NDIME, NELEM, NPOIN, NMARK blocks) as used by
    Mesh::read_su2 (io.rs:489-533): returns dim, nodes, elements, boundaries
    (markers numbered 0.. in file order)."""
    lines = [ln.strip() for ln in text.splitlines()]
    dim = None
    nodes, elements, boundaries = [], [], {}
    i = 0
    marker = -1
    while i < len(lines):
        ln = lines[i]
        if ln.startswith("NDIME="):
            dim = int(ln.split("=")[1])
        elif ln.startswith("NELEM="):
            ne = int(ln.split("=")[1])
            for k in range(ne):
                t = [int(v) for v in lines[i + 1 + k].split()]
                kind = t[0]
                nn = {5: 3, 9: 4, 10: 4, 12: 8, 3: 2}[kind]
                elements.append((kind, t[1:1 + nn]))
            i += ne
        elif ln.startswith("NPOIN="):
            npn = int(ln.split("=")[1].split()[0])
            for k in range(npn):
                t = lines[i + 1 + k].split()
                nodes.append([float(v) for v in t[:dim]])
            i += npn
        elif ln.startswith("MARKER_TAG="):
            marker += 1
        elif ln.startswith("MARKER_ELEMS="):
            nm = int(ln.split("=")[1])
            for k in range(nm):
                t = [int(v) for v in lines[i + 1 + k].split()]
                nn = {3: 2, 5: 3, 9: 4}[t[0]]
                boundaries[tuple(sorted(t[1:1 + nn]))] = marker
            i += nm
        i += 1
    return dim, nodes, elements, boundaries


def _mat_inv(a):
    """Matrix::inv (core/matrix.rs:320-380) on a list of rows."""
    n = len(a)
    a = [row[:] for row in a]
    out = [[1.0 if i == j else 0.0 for j in range(n)] for i in range(n)]
    for k in range(n - 1):
        piv = a[k][k]
        if abs(piv) < 1e-14:
            maxi, maxp = k, abs(piv)
            for j in range(k + 1, n):
                pj = abs(a[k][j])
                if pj > maxp:
                    maxi, maxp = j, pj
            if maxi == k:
                raise ZeroDivisionError("singular")
            a[k], a[maxi] = a[maxi], a[k]
            out[k], out[maxi] = out[maxi], out[k]
        piv = a[k][k]
        for i in range(k + 1, n):
            f = (-a[i][k]) / piv
            a[i] = [a[i][j] + a[k][j] * f for j in range(n)]
            out[i] = [out[i][j] + out[k][j] * f for j in range(n)]
    for k in range(n):
        piv = a[k][k]
        if abs(piv) < 1e-14:
            raise ZeroDivisionError("singular")
        a[k] = [v / piv for v in a[k]]
        out[k] = [v / piv for v in out[k]]
    for k in range(n - 1, 0, -1):
        piv = a[k][k]
        for i in range(k):
            f = (-a[i][k]) / piv
            a[i] = [a[i][j] + a[k][j] * f for j in range(n)]
            out[i] = [out[i][j] + out[k][j] * f for j in range(n)]
    return out


def grad_coeffs(dim, cell_face_ptr, cell_faces, face_owner, face_neighbor, face_center, cell_center):
    """Gradient coefficients of Mesh::compute (core/mesh/compute.rs:155-203):
    per cell-face entry (mesh order) and per cell, as lists of vectors."""
    gco, gdg = [], []
    for c in range(len(cell_face_ptr) - 1):
        xc = cell_center[c]
        dg = []
        for k in range(cell_face_ptr[c], cell_face_ptr[c + 1]):
            f = cell_faces[k]
            if face_neighbor[f] < 0:
                p = face_center[f]
            else:
                p = cell_center[face_owner[f] if face_neighbor[f] == c else face_neighbor[f]]
            dg.append([p[d] - xc[d] for d in range(dim)])
        g = [[0.0] * dim for _ in range(dim)]
        for v in dg:
            for i in range(dim):
                for j in range(dim):
                    g[i][j] += v[i] * v[j]
        gi = _mat_inv(g)
        own = [0.0] * dim
        for v in dg:
            w = [_dot(gi[i], v) for i in range(dim)]
            gco.append(w)
            own = [own[i] - w[i] for i in range(dim)]
        gdg.append(own)
    return gco, gdg


# ------------------------------------------------------------------ .msh
# Mesh::write / Mesh::read (core/mesh/io.rs:10-225), the crate's own format.

def rust_f64(x):
    """Rust's Display for f64: the shortest digits that read back to x (Python's
    repr finds the same digits), written out without an exponent."""
    if x != x:
        return "NaN"
    if x == math.inf:
        return "inf"
    if x == -math.inf:
        return "-inf"
    if x == 0.0:
        return "-0" if math.copysign(1.0, x) < 0 else "0"
    r = repr(float(x))
    sign = "-" if r.startswith("-") else ""
    r = r.lstrip("-")
    mant, exp = (r.split("e") + ["0"])[:2]
    ip, fp = (mant.split(".") + [""])[:2]
    digits, point = ip + fp, len(ip) + int(exp)
    while len(digits) > 1 and digits[0] == "0":
        digits, point = digits[1:], point - 1
    digits = digits.rstrip("0") or "0"
    if point <= 0:
        body = "0." + "0" * (-point) + digits
    elif point >= len(digits):
        body = digits + "0" * (point - len(digits))
    else:
        body = digits[:point] + "." + digits[point:]
    return sign + body


def write_msh(dim, nodes, face_nodes, face_patch, cell_faces, names=None):
    """Text of Mesh::write for a serial mesh (every face and cell owned, global
    id = index); boundary faces grouped by tag in face order are the patches."""
    patches = []
    for f, p in enumerate(face_patch):
        if p is None or p < 0:
            continue
        if not patches or patches[-1][0] != p:
            patches.append([p, f, 0])
        patches[-1][2] += 1
    names = list(names or [])
    out = [f"NDIME={dim}", f"NPATCH={len(patches)}"]
    for p, first, cnt in patches:
        nm = names[p] if p < len(names) else f"patch_{p}"
        out.append(f"{nm} {p} {first} {cnt}")
    out.append(f"NNODES={len(nodes)}")
    out += [" ".join(rust_f64(float(v)) for v in n[:dim]) for n in nodes]
    out.append(f"NFACES={len(face_nodes)}")
    for f, fn in enumerate(face_nodes):
        tag = face_patch[f]
        tag = "-" if tag is None or tag < 0 else str(int(tag))
        out.append(" ".join([str(len(fn))] + [str(int(v)) for v in fn] + [tag, str(f), "-"]))
    out.append(f"NCELLS={len(cell_faces)}")
    for c, cf in enumerate(cell_faces):
        out.append(" ".join([str(len(cf))] + [str(int(v)) for v in cf] + [str(c), "-"]))
    return "\n".join(out) + "\n"


def read_msh(text, dim=0):
    """Mesh::read: (dim, nodes, face_nodes, face_tags, cell_faces); ValueError on
    a malformed line, NotImplementedError on remote (ghost) entries."""
    section = "none"
    left = {"NNODES": 0, "NFACES": 0, "NCELLS": 0, "NPATCH": 0}
    nodes, face_nodes, tags, cells = [], [], [], []
    for line in text.splitlines():
        ls = line.strip()
        if not ls:
            continue
        if ls[0] == "N":
            parts = ls.split("=")
            if len(parts) < 2:
                raise ValueError(ls)
            section, val = parts[0], int(parts[1])
            if section == "NDIME":
                dim = dim or val
                if val != dim:
                    raise ValueError("NDIME")
            elif section in left:
                left[section] = val
            continue
        if section not in left or left[section] == 0:
            continue
        tok = ls.split(" ")
        if section == "NNODES":
            x = [0.0] * dim
            for i, t in enumerate(tok[:dim]):
                x[i] = float(t.strip())
            nodes.append(x)
        elif section in ("NFACES", "NCELLS"):
            size = int(tok[0])
            if size > 64:
                raise ValueError("size")
            idx = [int(v) for v in tok[1:1 + size]]
            rest = tok[1 + size:]
            if section == "NFACES":
                tags.append(None if rest[0] == "-" else int(rest[0]))
                rest = rest[1:]
                face_nodes.append(idx)
            else:
                cells.append(idx)
            int(rest[0])
            if rest[1] != "-":
                raise NotImplementedError("remote entries")
        left[section] -= 1
    return dim, nodes, face_nodes, tags, cells
