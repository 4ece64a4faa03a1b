// Box tiles for the triangular sweeps (host-side planning).
//
// The level-ordered sweep (k_sweep) hands every level of the dependency DAG to
// different warps, so each level costs one trip through L2: a value is
// published by one SM and polled by another.  On a mesh, a row's dependencies
// are its face neighbours, so a spatially compact group of cells keeps most of
// a dependency chain inside itself.  Here the cells are grouped into boxes of
// the cell-centre coordinates (per connected component of the matrix graph,
// so the problems of a batch never share a box); one warp sweeps a whole box in
// level order, passing values between its own steps through a small ring in
// shared memory, and only dependencies that cross a box face go through L2.
//
// Deadlock freedom does not depend on how many warps are resident: boxes are
// dispatched in an order in which every box comes after all boxes it depends
// on (checked here; no tiling is produced when the order does not exist), and
// inside a box the rows are swept in level order.
//
// The arithmetic of every row is unchanged (same entries, same order), so the
// tiled sweep returns the same bits as the level-ordered one.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "fv_internal.cuh"

namespace {

int32_t find(std::vector<int32_t> &p, int32_t a) {
    while (p[a] != a) {
        p[a] = p[p[a]];
        a = p[a];
    }
    return a;
}

// Geometric boxes: box coordinates of every row for boxes of edge k * h_c in
// component c (h_c: the component's mean cell size), and the rank of every
// box in the wavefront order (component, bx+by+bz, bz, by, bx).
struct Boxes {
    std::vector<int64_t> rank;  // rank of the geometric box of every row
    int64_t nbox = 0;           // number of ranks (boxes of all components)
};

Boxes make_boxes(int64_t n, int dim, const double *cell, const std::vector<int32_t> &comp, int32_t ncomp,
                 const std::vector<double> &lo, const std::vector<double> &hi, const std::vector<double> &hc,
                 double k) {
    Boxes B;
    std::vector<int64_t> nbd((size_t)ncomp * 3, 1), off((size_t)ncomp + 1, 0);
    for (int32_t c = 0; c < ncomp; ++c) {
        const double e = k * hc[c];
        int64_t tot = 1;
        for (int d = 0; d < dim; ++d) {
            const double ext = hi[(size_t)c * 3 + d] - lo[(size_t)c * 3 + d];
            nbd[(size_t)c * 3 + d] = std::max<int64_t>(1, (int64_t)std::floor(ext / e) + 1);
            tot *= nbd[(size_t)c * 3 + d];
        }
        off[c + 1] = off[c] + tot;
        if (off[c + 1] > 4 * n + 64) return B;  // far finer than the cells: not useful
    }
    // rank of every box id: sort by (component, coordinate sum, z, y, x)
    const int64_t total = off[ncomp];
    std::vector<int64_t> ids((size_t)total);
    std::iota(ids.begin(), ids.end(), 0);
    auto coords = [&](int64_t id, int32_t &c, int64_t *q) {
        c = (int32_t)(std::upper_bound(off.begin(), off.end(), id) - off.begin() - 1);
        int64_t r = id - off[c];
        for (int d = 0; d < 3; ++d) {
            q[d] = d < dim ? r % nbd[(size_t)c * 3 + d] : 0;
            if (d < dim) r /= nbd[(size_t)c * 3 + d];
        }
    };
    std::vector<int64_t> key((size_t)total * 2);
    for (int64_t id = 0; id < total; ++id) {
        int32_t c;
        int64_t q[3];
        coords(id, c, q);
        key[2 * id] = (int64_t)c << 40 | (q[0] + q[1] + q[2]);
        key[2 * id + 1] = (q[2] << 42) | (q[1] << 21) | q[0];
    }
    std::sort(ids.begin(), ids.end(), [&](int64_t a, int64_t b) {
        return key[2 * a] != key[2 * b] ? key[2 * a] < key[2 * b] : key[2 * a + 1] < key[2 * b + 1];
    });
    std::vector<int64_t> rank_of((size_t)total);
    for (int64_t r = 0; r < total; ++r) rank_of[ids[r]] = r;
    B.rank.resize((size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        const int32_t c = comp[i];
        const double e = k * hc[c];
        int64_t id = 0;
        for (int d = dim - 1; d >= 0; --d) {
            int64_t q = (int64_t)std::floor((cell[4 * i + d] - lo[(size_t)c * 3 + d]) / e);
            q = std::min<int64_t>(std::max<int64_t>(q, 0), nbd[(size_t)c * 3 + d] - 1);
            id = id * nbd[(size_t)c * 3 + d] + q;
        }
        B.rank[i] = rank_of[off[c] + id];
    }
    B.nbox = total;
    return B;
}

// Box of every row for one sweep direction: its geometric box, or the latest
// box (in dispatch order) of its dependencies when that comes later, so that
// every dependency lies in the row's own box or in an earlier one.  Forward:
// rows in ascending order (dependencies j < i), boxes in ascending rank;
// backward: rows descending (j > i), boxes in descending rank.  Returns dense
// box ids in dispatch order and their count.
std::vector<int32_t> assign_boxes(int64_t n, const Boxes &B, const int32_t *ptr, const int32_t *col, bool backward,
                                  int64_t &nb) {
    std::vector<int64_t> r((size_t)n);
    auto geo = [&](int64_t i) { return backward ? B.nbox - 1 - B.rank[i] : B.rank[i]; };
    if (!backward) {
        for (int64_t i = 0; i < n; ++i) {
            int64_t v = geo(i);
            for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k) v = std::max(v, r[col[k]]);
            r[i] = v;
        }
    } else {
        for (int64_t i = n - 1; i >= 0; --i) {
            int64_t v = geo(i);
            for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k) v = std::max(v, r[col[k]]);
            r[i] = v;
        }
    }
    std::vector<int64_t> used(r);
    std::sort(used.begin(), used.end());
    used.erase(std::unique(used.begin(), used.end()), used.end());
    nb = (int64_t)used.size();
    std::vector<int32_t> box((size_t)n);
    for (int64_t i = 0; i < n; ++i)
        box[i] = (int32_t)(std::lower_bound(used.begin(), used.end(), r[i]) - used.begin());
    return box;
}

// Largest number of rows one box holds at one level.
int32_t max_rows_per_box_level(const std::vector<int32_t> &box, int64_t nb, const int32_t *order,
                               const int32_t *level, int64_t n) {
    std::vector<int32_t> mark((size_t)nb, -1), cnt((size_t)nb, 0);
    int32_t mx = 0;
    for (int64_t t = 0; t < n; ++t) {
        const int32_t i = order[t];
        const int32_t b = box[i];
        if (mark[b] != level[i]) {
            mark[b] = level[i];
            cnt[b] = 0;
        }
        mx = std::max(mx, ++cnt[b]);
    }
    return mx;
}

// One sweep direction: the steps of each box (boxes in dispatch order) and
// where each dependency is read from.
bool plan_direction(int64_t n, const std::vector<int32_t> &box, int64_t nb, const int32_t *ptr, const int32_t *col,
                    const int32_t *level, const int32_t *order, int ring, fv_tile_plan &P) {
    for (int64_t i = 0; i < n; ++i)
        for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k)
            if (box[col[k]] > box[i]) return false;  // not reached: assign_boxes orders them
    // rows of each box in level order (order[] is level-sorted)
    std::vector<int64_t> start((size_t)nb + 1, 0);
    for (int64_t i = 0; i < n; ++i) start[box[i] + 1]++;
    for (int64_t r = 0; r < nb; ++r) start[r + 1] += start[r];
    P.trow.assign((size_t)n, 0);
    {
        std::vector<int64_t> fill(start.begin(), start.end() - 1);
        for (int64_t t = 0; t < n; ++t) {
            const int32_t i = order[t];
            P.trow[(size_t)fill[box[i]]++] = i;
        }
    }
    // steps: a new step when the level changes or 32 rows are taken
    std::vector<int32_t> lstep((size_t)n), lane((size_t)n);
    P.box_step.assign((size_t)nb + 1, 0);
    P.sptr.clear();
    for (int64_t r = 0; r < nb; ++r) {
        P.box_step[r] = (int32_t)P.sptr.size();
        int32_t st = -1, ln = 32, lev = -1;
        for (int64_t t = start[r]; t < start[r + 1]; ++t) {
            const int32_t i = P.trow[t];
            if (level[i] != lev || ln == 32) {
                P.sptr.push_back((int32_t)t);
                ++st;
                ln = 0;
                lev = level[i];
            }
            lstep[i] = st;
            lane[i] = ln++;
        }
    }
    P.box_step[nb] = (int32_t)P.sptr.size();
    P.nsteps = (int32_t)P.sptr.size();
    P.sptr.push_back((int32_t)n);
    P.nb = (int32_t)nb;
    P.lane_use = P.nsteps ? (double)n / (32.0 * (double)P.nsteps) : 0.0;
    // dependency sources: recent steps of the same box from the shared-memory
    // ring, everything else from the vector in global memory
    const int64_t nnz = ptr[n];
    P.dsrc.assign((size_t)(nnz ? nnz : 1), 0);
    int64_t in_ring = 0;
    for (int64_t i = 0; i < n; ++i)
        for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k) {
            const int32_t j = col[k];
            if (box[j] == box[i] && lstep[i] - lstep[j] <= ring - 1) {
                P.dsrc[k] = -(((lstep[j] % ring) * 32 + lane[j]) + 1);
                ++in_ring;
            } else {
                P.dsrc[k] = j;
            }
        }
    P.ring_share = nnz ? (double)in_ring / (double)nnz : 0.0;
    return true;
}

// Critical path of a plan in units of one L2 round trip: a step costs
// kStepCost, a dependency read from the vector costs one round trip after its
// producer finished, a ring read costs nothing beyond the step.
constexpr double kStepCost = 0.1;
double critical_path(int64_t n, const fv_tile_plan &P, const int32_t *ptr) {
    std::vector<double> T((size_t)n, 0.0);
    double worst = 0.0;
    for (int32_t b = 0; b < P.nb; ++b) {
        double t = 0.0;
        for (int32_t q = P.box_step[b]; q < P.box_step[b + 1]; ++q) {
            double start = t;
            for (int32_t u = P.sptr[q]; u < P.sptr[q + 1]; ++u) {
                const int32_t i = P.trow[u];
                for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k)
                    if (P.dsrc[k] >= 0) start = std::max(start, T[P.dsrc[k]] + 1.0);
            }
            t = start + kStepCost;
            for (int32_t u = P.sptr[q]; u < P.sptr[q + 1]; ++u) T[P.trow[u]] = t;
        }
        worst = std::max(worst, t);
    }
    return worst;
}

}  // namespace

bool fv_build_tile_plans(int64_t n, int dim, const double *cell, const int32_t *lp, const int32_t *lc,
                         const int32_t *up, const int32_t *uc, const int32_t *fwd_level, const int32_t *bwd_level,
                         const int32_t *fwd_order, const int32_t *bwd_order, int ring, fv_tile_plan &fwd,
                         fv_tile_plan &bwd) {
    if (n <= 0 || (dim != 2 && dim != 3)) return false;
    // connected components of the matrix graph (a batch's problems)
    std::vector<int32_t> parent((size_t)n);
    std::iota(parent.begin(), parent.end(), 0);
    for (int64_t i = 0; i < n; ++i)
        for (int32_t k = lp[i]; k < lp[i + 1]; ++k) {
            int32_t a = find(parent, (int32_t)i), b = find(parent, lc[k]);
            if (a != b) parent[std::max(a, b)] = std::min(a, b);
        }
    std::vector<int32_t> comp((size_t)n), label((size_t)n, -1);
    int32_t ncomp = 0;
    for (int64_t i = 0; i < n; ++i) {
        int32_t r = find(parent, (int32_t)i);
        if (label[r] < 0) label[r] = ncomp++;
        comp[i] = label[r];
    }
    std::vector<double> lo((size_t)ncomp * 3, INFINITY), hi((size_t)ncomp * 3, -INFINITY), hc((size_t)ncomp, 0.0);
    std::vector<int64_t> cnt((size_t)ncomp, 0);
    for (int64_t i = 0; i < n; ++i) {
        const int32_t c = comp[i];
        cnt[c]++;
        for (int d = 0; d < dim; ++d) {
            const double v = cell[4 * i + d];
            if (!std::isfinite(v)) return false;
            lo[(size_t)c * 3 + d] = std::min(lo[(size_t)c * 3 + d], v);
            hi[(size_t)c * 3 + d] = std::max(hi[(size_t)c * 3 + d], v);
        }
    }
    for (int32_t c = 0; c < ncomp; ++c) {
        double vol = 1.0;
        int dd = 0;
        for (int d = 0; d < dim; ++d) {
            const double ext = hi[(size_t)c * 3 + d] - lo[(size_t)c * 3 + d];
            if (ext > 0) {
                vol *= ext;
                ++dd;
            }
        }
        hc[c] = dd ? std::pow(vol / (double)cnt[c], 1.0 / dd) : 1.0;
        if (!(hc[c] > 0) || !std::isfinite(hc[c])) hc[c] = 1.0;
    }
    // Box edge: from coarse to fine, among the sizes at which no level of a box
    // holds more than 64 rows, the one with the shortest estimated critical
    // path (the estimate falls and then rises as boxes shrink: stop at the
    // first rise).  Tiles are used only when they beat the level schedule,
    // whose critical path is one round trip per level.
    static const double kEdges[] = {128, 96, 64, 48, 32, 24, 16, 12, 9, 7, 5, 4, 3, 2};
    int32_t nlev_f = 0, nlev_b = 0;
    for (int64_t i = 0; i < n; ++i) {
        nlev_f = std::max(nlev_f, fwd_level[i] + 1);
        nlev_b = std::max(nlev_b, bwd_level[i] + 1);
    }
    double best = 0.8 * (double)(nlev_f + nlev_b);
    bool found = false;
    for (double k : kEdges) {
        Boxes B = make_boxes(n, dim, cell, comp, ncomp, lo, hi, hc, k);
        if (B.nbox == 0) break;
        int64_t nbf = 0, nbb = 0;
        std::vector<int32_t> bf = assign_boxes(n, B, lp, lc, false, nbf);
        std::vector<int32_t> bb = assign_boxes(n, B, up, uc, true, nbb);
        if (nbf < 2 && n > 64) continue;
        if (max_rows_per_box_level(bf, nbf, fwd_order, fwd_level, n) > 64 ||
            max_rows_per_box_level(bb, nbb, bwd_order, bwd_level, n) > 64)
            continue;
        fv_tile_plan f, b;
        if (!plan_direction(n, bf, nbf, lp, lc, fwd_level, fwd_order, ring, f)) return false;
        if (!plan_direction(n, bb, nbb, up, uc, bwd_level, bwd_order, ring, b)) return false;
        const double cp = critical_path(n, f, lp) + critical_path(n, b, up);
        if (cp < best) {
            best = cp;
            f.edge = b.edge = k;
            f.est = b.est = cp / (double)(nlev_f + nlev_b);
            fwd = std::move(f);
            bwd = std::move(b);
            found = true;
        } else if (found) {
            break;
        }
    }
    return found;
}

// Host entry point for inspection and tests: the plan fv_ic0_factor /
// fv_ilu0_factor build for a matrix assembled on a mesh, from host arrays.
// sizes[0..2] receive (boxes, steps, entries of the swept side); the arrays
// may be NULL to query the sizes first.
static fv_status tile_plan_host_impl(int64_t n, int32_t dim, const double *cell, const int32_t *row_ptr,
                                     const int32_t *cols, int32_t direction, int64_t *sizes, int32_t *box_step,
                                     int32_t *sptr, int32_t *trow, int32_t *dsrc, double *stats) {
    if (n <= 0 || !cell || !row_ptr || !cols || !sizes || (direction != 0 && direction != 1)) return FV_ERR_INVALID;
    std::vector<int32_t> lp((size_t)n + 1), up((size_t)n + 1), lc, uc;
    for (int64_t i = 0; i < n; ++i) {
        lp[i] = (int32_t)lc.size();
        up[i] = (int32_t)uc.size();
        for (int32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
            if (cols[k] < 0 || cols[k] >= n) return FV_ERR_INVALID;
            if (cols[k] < i) lc.push_back(cols[k]);
            if (cols[k] > i) uc.push_back(cols[k]);
        }
    }
    lp[n] = (int32_t)lc.size();
    up[n] = (int32_t)uc.size();
    std::vector<int32_t> lev[2], ord[2];
    for (int d = 0; d < 2; ++d) {
        lev[d].assign((size_t)n, 0);
        int32_t nlev = 0;
        if (d == 0) {
            for (int64_t i = 0; i < n; ++i) {
                int32_t l = 0;
                for (int32_t k = lp[i]; k < lp[i + 1]; ++k) l = std::max(l, lev[0][lc[k]] + 1);
                lev[0][i] = l;
                nlev = std::max(nlev, l + 1);
            }
        } else {
            for (int64_t i = n - 1; i >= 0; --i) {
                int32_t l = 0;
                for (int32_t k = up[i]; k < up[i + 1]; ++k) l = std::max(l, lev[1][uc[k]] + 1);
                lev[1][i] = l;
                nlev = std::max(nlev, l + 1);
            }
        }
        std::vector<int64_t> start((size_t)nlev + 1, 0);
        for (int64_t i = 0; i < n; ++i) start[lev[d][i] + 1]++;
        for (int32_t l = 0; l < nlev; ++l) start[l + 1] += start[l];
        ord[d].assign((size_t)n, 0);
        for (int64_t i = 0; i < n; ++i) ord[d][start[lev[d][i]]++] = (int32_t)i;
    }
    if (lc.empty()) lc.push_back(0);
    if (uc.empty()) uc.push_back(0);
    fv_tile_plan tp[2];
    if (!fv_build_tile_plans(n, dim, cell, lp.data(), lc.data(), up.data(), uc.data(), lev[0].data(), lev[1].data(),
                             ord[0].data(), ord[1].data(), FV_TILE_RING, tp[0], tp[1]))
        return FV_ERR_UNSUPPORTED;
    const fv_tile_plan &P = tp[direction];
    const int64_t nside = direction == 0 ? lp[n] : up[n];
    sizes[0] = P.nb;
    sizes[1] = P.nsteps;
    sizes[2] = nside;
    if (box_step) std::copy(P.box_step.begin(), P.box_step.end(), box_step);
    if (sptr) std::copy(P.sptr.begin(), P.sptr.end(), sptr);
    if (trow) std::copy(P.trow.begin(), P.trow.end(), trow);
    if (dsrc) std::copy(P.dsrc.begin(), P.dsrc.begin() + nside, dsrc);
    if (stats) {
        stats[0] = P.edge;
        stats[1] = P.lane_use;
        stats[2] = P.ring_share;
        stats[3] = P.est;
    }
    return FV_OK;
}

extern "C" fv_status fv_tile_plan_host(int64_t n, int32_t dim, const double *cell, const int32_t *row_ptr,
                                       const int32_t *cols, int32_t direction, int64_t *sizes, int32_t *box_step,
                                       int32_t *sptr, int32_t *trow, int32_t *dsrc, double *stats) {
    return fv_host_guard([&] {
        return tile_plan_host_impl(n, dim, cell, row_ptr, cols, direction, sizes, box_step, sptr, trow, dsrc, stats);
    });
}
