// Level-k fill patterns of IncompleteCholesky / IncompleteLowerUpper (host).
//
// The reference builds a factor's row pattern by a depth-first walk from the
// row over the matrix graph (a stack, a visited map keyed by the row, and a
// path length per pushed node):
//   ILU U part, row_i_u_sparsity (incomplete_lower_upper.rs:30-83): nodes
//     j > i reached through at most `level` intermediate nodes below i;
//   ILU L part, row_i_l_sparsity (:86-137): nodes j < i reached through at
//     most `level` intermediate nodes above i;
//   IC, row_i_sparsity_edit (incomplete_cholesky.rs:35-85): every node the
//     walk pushes, i.e. the nodes within `level` steps (pushed in walk order,
//     first visit wins).
// The walk order matters for levels where a node can be reached by paths of
// different lengths, so it is restated exactly: neighbours in ascending
// order, last pushed popped first, a node marked on its first visit.
//
// Rows are independent, so the rows are split into contiguous ranges walked
// by host threads, each with its own visited marks; the ranges are joined in
// row order, which gives the same arrays as one sequential pass.
#include <algorithm>
#include <cstring>
#include <thread>
#include <vector>

#include "fv_internal.cuh"

namespace {

enum Walk { kUpperThroughLower, kLowerThroughUpper, kBall };

struct Walker {
    std::vector<uint32_t> mark;  // mark[j] == gen: j visited by the current walk
    uint32_t gen = 0;
    std::vector<int32_t> stack;  // (node, path length) pairs, last pushed on top

    // Appends the walk's result set (unsorted) to out.
    void walk(Walk w, int32_t i, int level, const int32_t *ptr, const int32_t *col, std::vector<int32_t> &out) {
        ++gen;
        stack.clear();
        stack.push_back(i);
        stack.push_back(0);
        mark[i] = gen;
        while (!stack.empty()) {
            const int32_t lk = stack.back();
            stack.pop_back();
            const int32_t k = stack.back();
            stack.pop_back();
            for (int32_t t = ptr[k]; t < ptr[k + 1]; ++t) {
                const int32_t j = col[t];
                if (j == k) continue;
                if (mark[j] == gen) continue;
                mark[j] = gen;
                const bool down = w == kBall || (w == kUpperThroughLower ? j < i : j > i);
                if (down && lk < level) {
                    stack.push_back(j);
                    stack.push_back(lk + 1);
                    if (w == kBall) out.push_back(j);
                } else if (w == kUpperThroughLower ? j > i : w == kLowerThroughUpper && j < i) {
                    out.push_back(j);
                }
            }
        }
    }
};

struct Part {
    int64_t r0 = 0, r1 = 0;
    std::vector<int32_t> len;   // entries per row
    std::vector<int32_t> col;   // the rows' sorted patterns, concatenated
    std::vector<int32_t> amap;  // A entry -> index into col
    std::vector<uint8_t> fill;  // 1 for entries not in A (IC only)
    fv_status status = FV_OK;
};

void walk_rows(int kind, int level, int64_t n, const int32_t *ptr, const int32_t *col, Part &p) {
    Walker wk;
    wk.mark.assign((size_t)n, 0);
    std::vector<int32_t> row;
    p.len.resize((size_t)(p.r1 - p.r0));
    p.amap.resize((size_t)(ptr[p.r1] - ptr[p.r0]));
    for (int64_t i = p.r0; i < p.r1; ++i) {
        row.clear();
        if (kind == 2) {
            wk.walk(kLowerThroughUpper, (int32_t)i, level, ptr, col, row);
            row.push_back((int32_t)i);
            wk.walk(kUpperThroughLower, (int32_t)i, level, ptr, col, row);
        } else {
            wk.walk(kBall, (int32_t)i, level, ptr, col, row);
            row.insert(row.end(), col + ptr[i], col + ptr[i + 1]);
        }
        std::sort(row.begin(), row.end());
        row.erase(std::unique(row.begin(), row.end()), row.end());
        const size_t base = p.col.size();
        if (kind == 1) p.fill.insert(p.fill.end(), row.size(), (uint8_t)1);
        // the matrix's own entries must be part of the pattern
        size_t q = 0;
        for (int32_t t = ptr[i]; t < ptr[i + 1]; ++t) {
            while (q < row.size() && row[q] < col[t]) ++q;
            if (q == row.size() || row[q] != col[t]) {
                p.status = FV_ERR_UNSUPPORTED;
                return;
            }
            p.amap[(size_t)(t - ptr[p.r0])] = (int32_t)(base + q);
            if (kind == 1) p.fill[base + q] = 0;
        }
        p.col.insert(p.col.end(), row.begin(), row.end());
        p.len[(size_t)(i - p.r0)] = (int32_t)row.size();
        if ((int64_t)p.col.size() > 0x7fffffffLL - 64) {
            p.status = FV_ERR_UNSUPPORTED;
            return;
        }
    }
}

void walk_rows_caught(int kind, int level, int64_t n, const int32_t *ptr, const int32_t *col, Part &p) {
    try {
        walk_rows(kind, level, n, ptr, col, p);
    } catch (...) {  // std::bad_alloc: no exception may leave a thread
        p.status = FV_ERR_ALLOC;
    }
}

// Runs f(0) .. f(nt - 1), one thread each where a thread can be started and
// on the calling thread otherwise.
template <typename F>
void run_parts(int64_t nt, F f) {
    std::vector<std::thread> th;
    try {
        th.reserve((size_t)nt);
        for (int64_t p = 1; p < nt; ++p) th.emplace_back(f, p);
    } catch (...) {
    }
    f(0);
    for (int64_t p = (int64_t)th.size() + 1; p < nt; ++p) f(p);
    for (auto &t : th) t.join();
}

}  // namespace

/* fill is filled for IC (kind 1) only: 1 for pattern entries that are not
 * entries of A.  FV_ERR_UNSUPPORTED when A's own entries are not all in the
 * pattern (a pattern without its diagonal) or the pattern would not fit
 * 32-bit offsets; FV_ERR_ALLOC when host memory runs out. */
fv_status fv_fill_pattern(int kind, int level, int64_t n, const int32_t *ptr, const int32_t *col,
                          std::vector<int32_t> &fptr, std::vector<int32_t> &fcol, std::vector<int32_t> &amap,
                          std::vector<uint8_t> &fill) {
    try {
        // one range per thread, at least 256 rows each, at most 16 threads;
        // each thread holds 4 bytes of visited marks per row of A, and all
        // threads' marks together stay within 1 GiB
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const int64_t by_memory = (int64_t(1) << 30) / std::max<int64_t>(1, 4 * n);
        const int64_t nt = std::max<int64_t>(1, std::min<int64_t>({(int64_t)hw, 16, n / 256, by_memory}));
        std::vector<Part> parts((size_t)nt);
        for (int64_t p = 0; p < nt; ++p) {
            parts[(size_t)p].r0 = n * p / nt;
            parts[(size_t)p].r1 = n * (p + 1) / nt;
        }
        run_parts(nt, [&](int64_t p) { walk_rows_caught(kind, level, n, ptr, col, parts[(size_t)p]); });
        int64_t total = 0;
        std::vector<int64_t> base((size_t)nt);
        for (int64_t p = 0; p < nt; ++p) {
            if (parts[(size_t)p].status != FV_OK) return parts[(size_t)p].status;
            base[(size_t)p] = total;
            total += (int64_t)parts[(size_t)p].col.size();
            if (total > 0x7fffffffLL - 64) return FV_ERR_UNSUPPORTED;
        }
        fptr.assign((size_t)n + 1, 0);
        fcol.resize((size_t)total);
        amap.resize((size_t)ptr[n]);
        fill.resize(kind == 1 ? (size_t)total : 0);
        run_parts(nt, [&](int64_t p) {
            const Part &q = parts[(size_t)p];
            const int32_t b = (int32_t)base[(size_t)p];
            int32_t acc = b;
            for (int64_t i = q.r0; i < q.r1; ++i) fptr[(size_t)i + 1] = acc += q.len[(size_t)(i - q.r0)];
            std::copy(q.col.begin(), q.col.end(), fcol.begin() + b);
            if (kind == 1) std::copy(q.fill.begin(), q.fill.end(), fill.begin() + b);
            for (size_t t = 0; t < q.amap.size(); ++t) amap[(size_t)ptr[q.r0] + t] = b + q.amap[t];
        });
        return FV_OK;
    } catch (...) {
        return FV_ERR_ALLOC;
    }
}

extern "C" fv_status fv_fill_pattern_host(int32_t kind, int32_t level, int64_t n, const int32_t *row_ptr,
                                          const int32_t *cols, int64_t *nnz, int32_t *fptr, int32_t *fcol,
                                          int32_t *amap, uint8_t *fill) {
    if ((kind != 1 && kind != 2) || level < 0 || n < 0 || n > 0x7fffffffLL || !row_ptr || !nnz) return FV_ERR_INVALID;
    if (row_ptr[0] != 0 || (row_ptr[n] > 0 && !cols)) return FV_ERR_INVALID;
    for (int64_t i = 0; i < n; ++i) {
        if (row_ptr[i + 1] < row_ptr[i]) return FV_ERR_INVALID;
        for (int32_t t = row_ptr[i]; t < row_ptr[i + 1]; ++t)
            if (cols[t] < 0 || cols[t] >= n || (t > row_ptr[i] && cols[t] <= cols[t - 1])) return FV_ERR_INVALID;
    }
    return fv_host_guard([&]() -> fv_status {
        std::vector<int32_t> p, c, a;
        std::vector<uint8_t> f;
        FV_TRY(fv_fill_pattern(kind, level, n, row_ptr, cols, p, c, a, f));
        *nnz = (int64_t)c.size();
        if (!fcol) return FV_OK;
        if (!fptr) return FV_ERR_INVALID;
        std::memcpy(fptr, p.data(), sizeof(int32_t) * (size_t)(n + 1));
        if (!c.empty()) std::memcpy(fcol, c.data(), sizeof(int32_t) * c.size());
        if (amap && !a.empty()) std::memcpy(amap, a.data(), sizeof(int32_t) * a.size());
        if (fill && kind == 1 && !f.empty()) std::memcpy(fill, f.data(), f.size());
        return FV_OK;
    });
}
