"""Box-tile plans of the triangular sweeps, checked on the CPU.

The plan (fv_tile_plan_host: the planner fv_ic0_factor / fv_ilu0_factor use
for a matrix assembled on a mesh) must be a valid schedule:
- every row once; a step holds at most 32 rows of one level; a box's steps
  ascend in level
- every dependency that is not read from the shared-memory ring points to a
  row of an earlier box, or of the same box at least RING steps earlier
- every ring read names the slot its producer wrote, within the last RING-1
  steps of the same box
An emulation of the tiled sweeps (boxes in dispatch order, a ring that is
really overwritten) reproduces the oracle's preconditioner apply bit for bit.
"""
import ctypes as C

import numpy as np
import pytest

from cases import convdiff_3d, diffusion_2d, oracle_system

RING = 8


def _plan(n, dim, cells, ptr, cols, direction):
    from fvb200._lib import lib
    c4 = np.zeros((n, 4))
    c4[:, :dim] = cells
    c4 = np.ascontiguousarray(c4)
    ptr = np.ascontiguousarray(ptr, np.int32)
    cols = np.ascontiguousarray(cols, np.int32)
    sizes = np.zeros(3, np.int64)
    ip = C.POINTER(C.c_int32)
    st = lib().fv_tile_plan_host(n, dim, c4.ctypes.data_as(C.POINTER(C.c_double)), ptr.ctypes.data_as(ip),
                                 cols.ctypes.data_as(ip), direction, sizes.ctypes.data_as(C.POINTER(C.c_int64)),
                                 None, None, None, None, None)
    assert st == 0, st
    nb, ns, ne = (int(v) for v in sizes)
    box_step = np.zeros(nb + 1, np.int32)
    sptr = np.zeros(ns + 1, np.int32)
    trow = np.zeros(n, np.int32)
    dsrc = np.zeros(max(ne, 1), np.int32)
    stats = np.zeros(4)
    st = lib().fv_tile_plan_host(n, dim, c4.ctypes.data_as(C.POINTER(C.c_double)), ptr.ctypes.data_as(ip),
                                 cols.ctypes.data_as(ip), direction, sizes.ctypes.data_as(C.POINTER(C.c_int64)),
                                 box_step.ctypes.data_as(ip), sptr.ctypes.data_as(ip), trow.ctypes.data_as(ip),
                                 dsrc.ctypes.data_as(ip), stats.ctypes.data_as(C.POINTER(C.c_double)))
    assert st == 0
    return box_step, sptr, trow, dsrc[:ne], stats


def _side(ptr, cols, upper):
    """Strict lower (upper) part in row order, as the sweeps store it."""
    sp, sc = [0], []
    for i in range(len(ptr) - 1):
        for k in range(ptr[i], ptr[i + 1]):
            if (cols[k] > i) if upper else (cols[k] < i):
                sc.append(cols[k])
        sp.append(len(sc))
    return np.array(sp), np.array(sc, dtype=np.int64)


def _levels(sp, sc, n, upper):
    lev = np.zeros(n, np.int64)
    rng = range(n - 1, -1, -1) if upper else range(n)
    for i in rng:
        d = sc[sp[i]:sp[i + 1]]
        if len(d):
            lev[i] = lev[d].max() + 1
    return lev


def _check_plan(n, sp, sc, lev, plan):
    box_step, sptr, trow, dsrc, _ = plan
    assert np.array_equal(np.sort(trow), np.arange(n))
    nb = len(box_step) - 1
    box_of = np.empty(n, np.int64)
    lstep = np.empty(n, np.int64)
    lane = np.empty(n, np.int64)
    for b in range(nb):
        prev = -1
        for s in range(box_step[b], box_step[b + 1]):
            rows = trow[sptr[s]:sptr[s + 1]]
            assert 1 <= len(rows) <= 32
            assert len(set(lev[rows])) == 1 and lev[rows[0]] >= prev
            prev = lev[rows[0]]
            box_of[rows] = b
            lstep[rows] = s - box_step[b]
            lane[rows] = np.arange(len(rows))
    for i in range(n):
        for k in range(sp[i], sp[i + 1]):
            j = sc[k]
            if dsrc[k] < 0:
                slot = -dsrc[k] - 1
                assert box_of[j] == box_of[i] and 1 <= lstep[i] - lstep[j] <= RING - 1
                assert slot == (lstep[j] % RING) * 32 + lane[j]
            else:
                assert dsrc[k] == j
                assert box_of[j] < box_of[i] or (box_of[j] == box_of[i] and lstep[i] - lstep[j] >= RING)
    return box_of


def _emulate(n, sp, sc, vals, diag_inv, rhs, plan):
    """Tiled sweep in dispatch order with a real ring: x_i = d_i (rhs_i - sum v x_j)."""
    box_step, sptr, trow, dsrc, _ = plan
    x = [None] * n
    for b in range(len(box_step) - 1):
        ring = [None] * (RING * 32)
        for s in range(box_step[b], box_step[b + 1]):
            out = []
            for ln, i in enumerate(trow[sptr[s]:sptr[s + 1]]):
                acc = float(rhs[i])
                for k in range(sp[i], sp[i + 1]):
                    v = ring[-dsrc[k] - 1] if dsrc[k] < 0 else x[dsrc[k]]
                    assert v is not None and v == x[sc[k]]
                    acc = acc - float(vals[k]) * v
                r = acc if diag_inv is None else float(diag_inv[i]) * acc
                out.append((ln, i, r))
            for ln, i, r in out:
                x[i] = r
                ring[((s - box_step[b]) % RING) * 32 + ln] = r
    return np.array(x)


@pytest.mark.parametrize("kind", ["3d", "2d"])
def test_tile_plan_is_a_valid_schedule_and_reproduces_the_apply(fv, orc, kind):
    case = convdiff_3d(fv, 8, seed=3) if kind == "3d" else diffusion_2d(fv, 40, seed=3)
    m = case["mesh"]
    ptr, cols, vals, rhs = oracle_system(orc, case)
    n = len(ptr) - 1
    dim = 3 if kind == "3d" else 2
    pc = orc.Precond("ilu" if kind == "3d" else "ic", ptr, cols, vals)
    fp, fc, fvv, inv, _ = pc.export()
    r = np.random.default_rng(2).standard_normal(n)
    want = pc.apply(r)
    planf = _plan(n, dim, m.cell_center, ptr, cols, 0)
    planb = _plan(n, dim, m.cell_center, ptr, cols, 1)
    lp, lc = _side(ptr, cols, False)
    up, uc = _side(ptr, cols, True)
    _check_plan(n, lp, lc, _levels(lp, lc, n, False), planf)
    _check_plan(n, up, uc, _levels(up, uc, n, True), planb)
    assert planf[4][0] > 0 and planf[4][2] > 0.3  # boxes larger than one cell, most reads from the ring
    if kind == "3d":  # ILU: unit lower; the factor CSR holds strict L, then U with the diagonal
        Lv = np.array([fvv[k] for i in range(n) for k in range(fp[i], fp[i + 1]) if fc[k] < i])
        Uv = np.array([fvv[k] for i in range(n) for k in range(fp[i], fp[i + 1]) if fc[k] > i])
        dg = np.array([fvv[k] for i in range(n) for k in range(fp[i], fp[i + 1]) if fc[k] == i])
        y = _emulate(n, lp, lc, Lv, None, r, planf)
        z = _emulate(n, up, uc, Uv, 1.0 / dg, y, planb)
    else:  # IC: L with the diagonal in inv (1/l_ii); backward over L^T
        Lv = np.array([fvv[k] for i in range(n) for k in range(fp[i], fp[i + 1]) if fc[k] < i])
        LT = {}
        for i in range(n):
            for k in range(fp[i], fp[i + 1]):
                if fc[k] < i:
                    LT[(fc[k], i)] = fvv[k]
        Uv = np.array([LT[(i, j)] for i in range(n) for j in uc[up[i]:up[i + 1]]])
        y = _emulate(n, lp, lc, Lv, inv, r, planf)
        z = _emulate(n, up, uc, Uv, inv, y, planb)
    assert np.array_equal(z, want)


def test_tile_plan_keeps_batch_problems_apart(fv, orc):
    """A block-diagonal union (a batch): boxes never mix problems."""
    import scipy.sparse as sp
    from fvb200.batch import MeshBatch
    ms = [fv.Mesh.square(s, 0.2, 40 + s) for s in (12, 20, 7)]
    mb = MeshBatch(ms)
    blocks = []
    for m in ms:
        nbf = m.n_boundary_faces
        p_, c_, v_, _ = orc.assemble(m, -1.0, 0.0, -1.0, kappa=np.ones(m.n_faces), source=np.ones(m.n_cells),
                                     bndi=np.zeros(nbf), bnde=np.zeros(nbf))
        blocks.append(sp.csr_matrix((v_, c_, p_)))
    U = sp.block_diag(blocks, format="csr")
    U.sort_indices()
    ptr, cols = U.indptr, U.indices
    n = len(ptr) - 1
    plan = _plan(n, 2, mb.cell_center, ptr, cols, 0)
    lp, lc = _side(ptr, cols, False)
    box_of = _check_plan(n, lp, lc, _levels(lp, lc, n, False), plan)
    prob = np.searchsorted(np.asarray(mb.cell_offsets), np.arange(n), side="right") - 1
    for b in np.unique(box_of):
        assert len(set(prob[box_of == b])) == 1
