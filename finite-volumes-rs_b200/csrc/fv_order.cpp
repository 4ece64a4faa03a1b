// Box-colour ordering of a matrix's rows for the reordered (perf-mode)
// triangular sweeps.  Host code, O(n + nnz).
//
// The reference factorises in the natural row order
// (src/linalg/preconditioners/incomplete_lower_upper.rs:200-261,
// incomplete_cholesky.rs:87-145), whose dependency graph on a 3D mesh has a
// level count proportional to the mesh's extent (512 levels per sweep on a
// 128^3 cube): every level costs one SM-to-SM handoff on the GPU, so the
// sweeps are latency-bound.  This ordering groups the cells into boxes of
// their centres, colours the boxes so that no two coupled boxes share a
// colour, and numbers the rows colour by colour, box by box, keeping the
// natural order inside a box.  The ILU/IC factorisation of that reordered
// matrix has dependencies only inside a box and on boxes of earlier colours,
// so its level count is about (colours) x (levels inside one box), and every
// level spans all boxes of a colour.  Finally the rows are sorted by level
// (stable): that keeps every dependency before its dependent (rows of one
// level are never coupled), so the factor's dependency graph is unchanged,
// and each level becomes a contiguous range of rows.
//
// On meshes whose boxes align with the element grid (the square / cube
// generators with box counts dividing the element counts) the box graph is
// the grid graph and two colours suffice; other meshes get a few more.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "fv_b200.h"

namespace {

// Per-problem result: the rows of one problem in the final order and the
// level of each of them.
fv_status order_one(int64_t n, int32_t dim, const double *center, int64_t center_stride, const double *lo_in,
                    const double *hi_in, const int32_t *row_ptr, const int32_t *cols, int32_t col_base,
                    int32_t rows_per_box, int32_t *perm, int32_t *level_out, fv_order_info *info) {
    if (n <= 0 || (dim != 2 && dim != 3) || !center || !row_ptr || !cols || !perm || center_stride < dim)
        return FV_ERR_INVALID;
    // default box: 4 x 4 squares of 2 triangles in 2D, 4^3 hexes of 6 tetrahedra in 3D
    if (rows_per_box <= 0) rows_per_box = dim == 2 ? 32 : 384;
    const int64_t k_first = row_ptr[0];
    for (int64_t i = 0; i < n; ++i)
        if (row_ptr[i + 1] < row_ptr[i]) return FV_ERR_INVALID;
    for (int64_t k = k_first; k < row_ptr[n]; ++k)
        if (cols[k] - col_base < 0 || cols[k] - col_base >= n) return FV_ERR_INVALID;
    // domain box: given, or the centres' bounding box
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (int d = 0; d < dim; ++d) {
        if (lo_in && hi_in) {
            lo[d] = lo_in[d];
            hi[d] = hi_in[d];
        } else {
            lo[d] = hi[d] = center[d];
            for (int64_t i = 0; i < n; ++i) {
                lo[d] = std::min(lo[d], center[i * center_stride + d]);
                hi[d] = std::max(hi[d], center[i * center_stride + d]);
            }
        }
        if (!(hi[d] >= lo[d])) return FV_ERR_INVALID;
    }
    // boxes per axis: about n / rows_per_box boxes, shaped like the domain
    double ext[3] = {0, 0, 0}, gm = 1.0;
    int dims_pos = 0;
    for (int d = 0; d < dim; ++d) {
        ext[d] = hi[d] - lo[d];
        if (ext[d] > 0) {
            gm *= ext[d];
            ++dims_pos;
        }
    }
    const double target = std::max(1.0, (double)n / rows_per_box);
    int32_t K[3] = {1, 1, 1};
    if (dims_pos > 0) {
        gm = std::pow(gm, 1.0 / dims_pos);
        const double per_axis = std::pow(target, 1.0 / dims_pos);
        for (int d = 0; d < dim; ++d)
            if (ext[d] > 0) K[d] = (int32_t)std::max(1.0, std::min(65536.0, std::round(per_axis * ext[d] / gm)));
    }
    const int64_t nbox = (int64_t)K[0] * K[1] * K[2];
    if (nbox > (int64_t)1 << 31) return FV_ERR_INVALID;
    // Box boundaries: each interior boundary moves from its uniform position to
    // the sparsest slice of cell centres within a quarter box of it.  On a mesh
    // built on a grid (the square and cube generators, any side) those slices
    // are the grid lines, so no element is cut and the box graph stays the
    // grid graph (two colours) even when the side does not divide evenly;
    // elsewhere fewer cells straddle the boundaries.
    constexpr int kBins = 128;  // histogram bins per box
    constexpr int kWin = 2;     // a candidate's score: the centres within +-kWin bins (wide gaps win)
    std::vector<double> cut[3];
    for (int d = 0; d < dim; ++d) {
        if (K[d] <= 1) continue;
        const int64_t nbins = (int64_t)K[d] * kBins;
        std::vector<int64_t> hist((size_t)nbins, 0);
        for (int64_t i = 0; i < n; ++i) {
            int64_t q = (int64_t)std::floor((center[i * center_stride + d] - lo[d]) / ext[d] * nbins);
            ++hist[(size_t)std::min<int64_t>(std::max<int64_t>(q, 0), nbins - 1)];
        }
        cut[d].resize((size_t)K[d] - 1);
        for (int k = 1; k < K[d]; ++k) {
            const int64_t mid = (int64_t)k * kBins;
            auto score = [&](int64_t q) {
                int64_t c = 0;
                for (int64_t u = q - kWin; u <= q + kWin; ++u)
                    if (u >= 0 && u < nbins) c += hist[(size_t)u];
                return c;
            };
            int64_t best = mid, best_score = score(mid);
            for (int64_t q = mid - kBins / 4; q <= mid + kBins / 4; ++q) {
                if (q <= 0 || q >= nbins) continue;
                // fewest centres nearby; ties go to the bin nearest the uniform position
                const int64_t sc = score(q);
                if (sc < best_score || (sc == best_score && std::llabs(q - mid) < std::llabs(best - mid))) {
                    best = q;
                    best_score = sc;
                }
            }
            cut[d][k - 1] = lo[d] + ((double)best + 0.5) / nbins * ext[d];
        }
    }
    std::vector<int32_t> box((size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        int64_t b = 0;
        for (int d = 0; d < dim; ++d) {
            int64_t q = 0;
            if (K[d] > 1)
                q = std::upper_bound(cut[d].begin(), cut[d].end(), center[i * center_stride + d]) - cut[d].begin();
            b = b * K[d] + q;
        }
        box[i] = (int32_t)b;
    }
    // occupied boxes, ranked by their first (smallest) row
    std::vector<int32_t> rank((size_t)nbox, -1);
    int32_t nb = 0;
    for (int64_t i = 0; i < n; ++i)
        if (rank[box[i]] < 0) rank[box[i]] = nb++;
    for (int64_t i = 0; i < n; ++i) box[i] = rank[box[i]];  // box rank of every row
    std::vector<int32_t>().swap(rank);
    // rows grouped by box (counting sort, rows ascending inside a box)
    std::vector<int64_t> bptr((size_t)nb + 1, 0);
    for (int64_t i = 0; i < n; ++i) ++bptr[box[i] + 1];
    for (int32_t b = 0; b < nb; ++b) bptr[b + 1] += bptr[b];
    std::vector<int32_t> brow((size_t)n);
    {
        std::vector<int64_t> fill(bptr.begin(), bptr.end() - 1);
        for (int64_t i = 0; i < n; ++i) brow[fill[box[i]]++] = (int32_t)i;
    }
    // box adjacency (both directions of every coupling), deduplicated per scan
    std::vector<std::vector<int32_t>> adj((size_t)nb);
    {
        std::vector<int32_t> stamp((size_t)nb, -1);
        for (int32_t b = 0; b < nb; ++b) {
            stamp[b] = b;
            for (int64_t u = bptr[b]; u < bptr[b + 1]; ++u) {
                const int32_t i = brow[u];
                for (int32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
                    const int32_t c = box[cols[k] - col_base];
                    if (stamp[c] != b) {
                        stamp[c] = b;
                        adj[b].push_back(c);
                        adj[c].push_back(b);  // a coupling seen from one side only still separates colours
                    }
                }
            }
        }
    }
    // greedy colouring in box-rank order (smallest colour unused by coloured neighbours)
    std::vector<int32_t> colour((size_t)nb, -1);
    int32_t ncol = 0;
    {
        std::vector<char> used;
        for (int32_t b = 0; b < nb; ++b) {
            used.assign((size_t)ncol + 1, 0);
            for (int32_t c : adj[b])
                if (colour[c] >= 0) used[colour[c]] = 1;
            int32_t k = 0;
            while (used[k]) ++k;
            colour[b] = k;
            ncol = std::max(ncol, k + 1);
        }
    }
    std::vector<std::vector<int32_t>>().swap(adj);
    // first ordering: colour, box rank, row
    std::vector<int64_t> cptr((size_t)ncol + 1, 0);
    for (int32_t b = 0; b < nb; ++b) cptr[colour[b] + 1] += bptr[b + 1] - bptr[b];
    for (int32_t c = 0; c < ncol; ++c) cptr[c + 1] += cptr[c];
    std::vector<int32_t> q0((size_t)n);
    {
        std::vector<int64_t> fill(cptr.begin(), cptr.end() - 1);
        for (int32_t b = 0; b < nb; ++b)
            for (int64_t u = bptr[b]; u < bptr[b + 1]; ++u) q0[fill[colour[b]]++] = brow[u];
    }
    std::vector<int32_t>().swap(brow);
    std::vector<int32_t> pos((size_t)n);  // row -> position in q0
    for (int64_t p = 0; p < n; ++p) pos[q0[p]] = (int32_t)p;
    // level of every row in the first ordering's forward dependency graph
    std::vector<int32_t> level((size_t)n, 0);
    int32_t nlev = 0;
    for (int64_t p = 0; p < n; ++p) {
        const int32_t i = q0[p];
        int32_t l = 0;
        for (int32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
            const int32_t j = cols[k] - col_base;
            if (pos[j] < p) l = std::max(l, level[j] + 1);
        }
        level[i] = l;
        nlev = std::max(nlev, l + 1);
    }
    // final ordering: level, then the first ordering (stable counting sort)
    std::vector<int64_t> lptr((size_t)nlev + 1, 0);
    for (int64_t i = 0; i < n; ++i) ++lptr[level[i] + 1];
    for (int32_t l = 0; l < nlev; ++l) lptr[l + 1] += lptr[l];
    for (int64_t p = 0; p < n; ++p) {
        const int32_t i = q0[p];
        const int64_t at = lptr[level[i]]++;
        perm[at] = i;
        if (level_out) level_out[at] = level[i];
    }
    if (info) {
        info->n_boxes = nb;
        for (int d = 0; d < 3; ++d) info->boxes_per_axis[d] = d < dim ? K[d] : 1;
        info->n_colours = ncol;
        info->n_levels = nlev;
    }
    return FV_OK;
}

}  // namespace

extern "C" fv_status fv_order_boxes_host(int64_t n, int32_t dim, const double *cell_center, int64_t center_stride,
                                         const double *lo, const double *hi, const int32_t *row_ptr,
                                         const int32_t *cols, int32_t rows_per_box, int32_t *perm,
                                         fv_order_info *info) {
    if (!row_ptr || row_ptr[0] != 0) return FV_ERR_INVALID;
    try {
        return order_one(n, dim, cell_center, center_stride, lo, hi, row_ptr, cols, 0, rows_per_box, perm, nullptr,
                         info);
    } catch (const std::bad_alloc &) {
        return FV_ERR_ALLOC;
    }
}

extern "C" fv_status fv_order_boxes_host_levels(int64_t n, int32_t dim, const double *cell_center,
                                                int64_t center_stride, const double *lo, const double *hi,
                                                const int32_t *row_ptr, const int32_t *cols, int32_t rows_per_box,
                                                int32_t *perm, int32_t *level, fv_order_info *info) {
    if (!row_ptr || row_ptr[0] != 0 || !level) return FV_ERR_INVALID;
    try {
        return order_one(n, dim, cell_center, center_stride, lo, hi, row_ptr, cols, 0, rows_per_box, perm, level,
                         info);
    } catch (const std::bad_alloc &) {
        return FV_ERR_ALLOC;
    }
}

// A block-diagonal union of independent problems (rows [off[p], off[p+1]) of
// problem p, coupled to nothing outside): every problem ordered on its own,
// with its own domain box (lo/hi per problem, or NULL for the centres'
// bounding boxes), then all rows sorted stably by (level, problem, position):
// the union's level count is the largest problem's.
extern "C" fv_status fv_order_boxes_batch_host(int32_t n_problems, const int64_t *offsets, int32_t dim,
                                               const double *cell_center, int64_t center_stride, const double *lo,
                                               const double *hi, const int32_t *row_ptr, const int32_t *cols,
                                               int32_t rows_per_box, int32_t *perm, fv_order_info *info) {
    if (n_problems < 1 || !offsets || !row_ptr || offsets[0] != 0 || row_ptr[0] != 0) return FV_ERR_INVALID;
    try {
        const int64_t n = offsets[n_problems];
        for (int32_t p = 0; p < n_problems; ++p)
            if (offsets[p + 1] <= offsets[p]) return FV_ERR_INVALID;
        std::vector<int32_t> lperm((size_t)n), lev((size_t)n);
        std::vector<fv_order_info> one((size_t)n_problems);
        std::vector<int> st((size_t)n_problems, FV_OK);
        // the problems are independent: ordered side by side on the host's cores
#pragma omp parallel for schedule(dynamic, 1)
        for (int32_t p = 0; p < n_problems; ++p) {
            const int64_t a = offsets[p], b = offsets[p + 1];
            try {
                st[p] = order_one(b - a, dim, cell_center + a * center_stride, center_stride,
                                  lo ? lo + (int64_t)p * dim : nullptr, hi ? hi + (int64_t)p * dim : nullptr,
                                  row_ptr + a, cols, (int32_t)a, rows_per_box, lperm.data() + a, lev.data() + a,
                                  &one[p]);
            } catch (const std::bad_alloc &) {
                st[p] = FV_ERR_ALLOC;
            }
            if (st[p] == FV_OK)
                for (int64_t i = a; i < b; ++i) lperm[i] += (int32_t)a;
        }
        fv_order_info tot{};
        int32_t nlev = 0;
        for (int32_t p = 0; p < n_problems; ++p) {
            if (st[p] != FV_OK) return (fv_status)st[p];
            tot.n_boxes += one[p].n_boxes;
            tot.n_colours = std::max(tot.n_colours, one[p].n_colours);
            nlev = std::max(nlev, one[p].n_levels);
        }
        for (int d = 0; d < 3; ++d) tot.boxes_per_axis[d] = one[0].boxes_per_axis[d];
        std::vector<int64_t> lptr((size_t)nlev + 1, 0);
        for (int64_t i = 0; i < n; ++i) ++lptr[lev[i] + 1];
        for (int32_t l = 0; l < nlev; ++l) lptr[l + 1] += lptr[l];
        for (int64_t i = 0; i < n; ++i) perm[lptr[lev[i]]++] = lperm[i];
        tot.n_levels = nlev;
        if (info) *info = tot;
        return FV_OK;
    } catch (const std::bad_alloc &) {
        return FV_ERR_ALLOC;
    }
}
