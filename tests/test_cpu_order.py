"""The box-colour ordering of the reordered (perf-mode) factorisations, on the
host (fv_order_boxes_host, fv_order_boxes_batch_host):

- the result is a permutation, and the reordered matrix's forward dependency
  levels are non-decreasing along its rows (every level a contiguous range),
  with as many levels as reported
- boxes of one colour are never coupled by a matrix entry
- on the square / cube generators with aligned boxes two colours suffice and
  the sweeps have far fewer levels than in natural order
- a batch of independent problems has the largest problem's level count, and
  each problem keeps its own ordering
"""
import numpy as np
import pytest

from cases import convdiff_3d, diffusion_2d, oracle_system


def _order(fv, case, rows_per_box=0, aligned=True):
    m = case["mesh"]
    from oracle import pattern
    ptr, cols = pattern(m)
    d = m.dim
    lo, hi = (np.zeros(d), np.ones(d)) if aligned else (None, None)
    perm, info = fv.order_boxes_host(m.cell_center, ptr, cols, rows_per_box, lo, hi)
    return ptr, cols, perm, info


@pytest.mark.parametrize("kind,n", [("2d", 16), ("2d", 24), ("3d", 8), ("3d", 12)])
def test_box_ordering_properties(fv, orc, kind, n):
    case = diffusion_2d(fv, n, seed=4) if kind == "2d" else convdiff_3d(fv, n, seed=4)
    ptr, cols, vals, _ = oracle_system(orc, case)
    _, _, perm, info = _order(fv, case)
    N = len(ptr) - 1
    assert np.array_equal(np.sort(perm), np.arange(N))
    bp, bc, _ = orc.permute(ptr, cols, vals, perm)
    lev, nl = orc.levels(bp, bc)
    assert np.all(np.diff(lev) >= 0) and nl == info["n_levels"]
    nat_levels = orc.levels(ptr, cols)[1]
    assert info["n_colours"] == 2
    # two colours of 4 x 4 squares (2D) / 4^3 hexes (3D): at most twice the levels inside one box
    assert nl <= (16 if kind == "2d" else 28) and nl <= nat_levels
    # boxes of one colour are not coupled: recompute the grid's boxes; colours are their parity
    K = info["boxes_per_axis"][:case["mesh"].dim]
    key = np.floor(case["mesh"].cell_center * np.array(K)).astype(int)
    parity = key.sum(1) % 2
    rows = np.repeat(np.arange(N), np.diff(ptr))
    box = np.ravel_multi_index(key.T, K)
    other = box[rows] != box[cols]
    assert np.all(parity[rows][other] != parity[cols][other])


def test_box_ordering_unaligned_and_defaults(fv, orc):
    """Without a domain box (the centres' bounding box) the boxes cut elements:
    possibly more colours, still a valid level-sorted permutation; rows_per_box
    changes the grid."""
    case = convdiff_3d(fv, 10, seed=6)
    ptr, cols, perm, info = _order(fv, case, aligned=False)
    assert np.array_equal(np.sort(perm), np.arange(len(ptr) - 1))
    assert info["n_colours"] >= 2
    vals = np.ones(len(cols))
    lev, nl = orc.levels(*orc.permute(ptr, cols, vals, perm)[:2])
    assert np.all(np.diff(lev) >= 0) and nl == info["n_levels"]
    _, _, _, info2 = _order(fv, case, rows_per_box=48)
    assert np.prod(info2["boxes_per_axis"]) > np.prod(info["boxes_per_axis"])


def test_box_ordering_batch(fv, orc):
    """A block-diagonal union: each problem's rows keep their own relative
    order, the union's levels are the deepest problem's, level-sorted."""
    import ctypes as C

    from fvb200._lib import OrderInfo, lib
    from oracle import pattern
    meshes = [fv.Mesh.square(s, 0.2, 10 + s) for s in (8, 16, 12)]
    parts, offs, cc = [], [0], []
    for m in meshes:
        ptr, cols = pattern(m)
        parts.append((ptr, cols))
        offs.append(offs[-1] + m.n_cells)
        cc.append(m.cell_center)
    N = offs[-1]
    uptr = np.concatenate([[0]] + [p[0][1:] + sum(len(q[1]) for q in parts[:k]) for k, p in enumerate(parts)])
    ucol = np.concatenate([p[1] + offs[k] for k, p in enumerate(parts)]).astype(np.int32)
    uptr = uptr.astype(np.int32)
    cen = np.ascontiguousarray(np.concatenate(cc))
    off = np.array(offs, np.int64)
    lo, hi = np.zeros(2 * len(meshes)), np.ones(2 * len(meshes))
    perm = np.empty(N, np.int32)
    info = OrderInfo()
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int32)
    st = lib().fv_order_boxes_batch_host(len(meshes), off.ctypes.data_as(C.POINTER(C.c_int64)), 2,
                                         cen.ctypes.data_as(dp), 2, lo.ctypes.data_as(dp), hi.ctypes.data_as(dp),
                                         uptr.ctypes.data_as(ip), ucol.ctypes.data_as(ip), 0,
                                         perm.ctypes.data_as(ip), C.byref(info))
    assert st == 0
    assert np.array_equal(np.sort(perm), np.arange(N))
    lev, nl = orc.levels(*orc.permute(uptr, ucol, np.ones(len(ucol)), perm)[:2])
    assert np.all(np.diff(lev) >= 0) and nl == info.n_levels
    for k, m in enumerate(meshes):
        own = perm[(perm >= offs[k]) & (perm < offs[k + 1])] - offs[k]
        single, sinfo = fv.order_boxes_host(m.cell_center, *parts[k], 0, np.zeros(2), np.ones(2))
        assert np.array_equal(own, single)
    assert nl == max(fv.order_boxes_host(m.cell_center, *parts[k], 0, np.zeros(2), np.ones(2))[1]["n_levels"]
                     for k, m in enumerate(meshes))


def test_merged_orders_equal_the_batch_order(fv, orc):
    """merge_orders over each problem's own order and levels (computed alone,
    fv_order_boxes_host_levels) is the batch order of the union, 2D and 3D;
    the levels are those of the reordered matrix."""
    import ctypes as C

    from fvb200._lib import OrderInfo, lib
    from oracle import pattern
    for dim, meshes in ((2, [fv.Mesh.square(s, 0.2, 10 + s) for s in (8, 16, 12, 5)]),
                        (3, [fv.Mesh.cube(n, 0.15, 20 + n) for n in (4, 6, 3)])):
        parts, offs, cc, own = [], [0], [], []
        for m in meshes:
            ptr, cols = pattern(m)
            parts.append((ptr, cols))
            offs.append(offs[-1] + m.n_cells)
            cc.append(m.cell_center)
            perm_k, info_k, lev_k = fv.order_boxes_host(m.cell_center, ptr, cols, 0, np.zeros(dim), np.ones(dim),
                                                        levels=True)
            lv, nl = orc.levels(*orc.permute(ptr, cols, np.ones(len(cols)), perm_k)[:2])
            assert np.array_equal(lev_k, lv) and nl == info_k["n_levels"] == lev_k[-1] + 1
            own.append((perm_k, lev_k))
        N = offs[-1]
        uptr = np.concatenate([[0]] + [p[0][1:] + sum(len(q[1]) for q in parts[:k]) for k, p in enumerate(parts)])
        ucol = np.concatenate([p[1] + offs[k] for k, p in enumerate(parts)]).astype(np.int32)
        uptr = uptr.astype(np.int32)
        cen = np.ascontiguousarray(np.concatenate(cc))
        off = np.array(offs, np.int64)
        lo, hi = np.zeros(dim * len(meshes)), np.ones(dim * len(meshes))
        perm = np.empty(N, np.int32)
        info = OrderInfo()
        dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int32)
        st = lib().fv_order_boxes_batch_host(len(meshes), off.ctypes.data_as(C.POINTER(C.c_int64)), dim,
                                             cen.ctypes.data_as(dp), dim, lo.ctypes.data_as(dp),
                                             hi.ctypes.data_as(dp), uptr.ctypes.data_as(ip), ucol.ctypes.data_as(ip),
                                             0, perm.ctypes.data_as(ip), C.byref(info))
        assert st == 0
        assert np.array_equal(fv.merge_orders(own, offs[:-1]), perm)


def test_box_ordering_rejects_bad_input(fv):
    from fvb200 import FvError
    with pytest.raises(FvError):
        fv.order_boxes_host(np.zeros((3, 2)), np.array([0, 1, 2, 3]), np.array([0, 5, 2]))
