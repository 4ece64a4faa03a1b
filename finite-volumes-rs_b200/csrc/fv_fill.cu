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
#include <algorithm>
#include <vector>

#include "fv_internal.cuh"

namespace {

enum Walk { kUpperThroughLower, kLowerThroughUpper, kBall };

// Returns the walk's result set (unsorted); stamp/len/stack are scratch of
// size n; gen is a value no earlier walk used (a fresh visited set).
void walk(Walk w, int32_t i, int level, const int32_t *ptr, const int32_t *col, std::vector<int64_t> &stamp,
          int64_t gen, std::vector<int32_t> &len, std::vector<int32_t> &stack, std::vector<int32_t> &out) {
    out.clear();
    stack.clear();
    stack.push_back(i);
    stamp[i] = gen;
    len[i] = 0;
    while (!stack.empty()) {
        const int32_t k = stack.back();
        stack.pop_back();
        const int32_t lk = len[k];
        for (int32_t t = ptr[k]; t < ptr[k + 1]; ++t) {
            const int32_t j = col[t];
            if (j == k) continue;
            if (stamp[j] == gen) continue;
            stamp[j] = gen;
            if (w == kBall) {
                if (lk < level) {
                    stack.push_back(j);
                    len[j] = lk + 1;
                    out.push_back(j);
                }
            } else if (w == kUpperThroughLower) {
                if (j < i && lk < level) {
                    stack.push_back(j);
                    len[j] = lk + 1;
                } else if (j > i) {
                    out.push_back(j);
                }
            } else {
                if (j > i && lk < level) {
                    stack.push_back(j);
                    len[j] = lk + 1;
                } else if (j < i) {
                    out.push_back(j);
                }
            }
        }
    }
}

}  // namespace

bool fv_fill_pattern(int kind, int level, int64_t n, const int32_t *ptr, const int32_t *col,
                     std::vector<int32_t> &fptr, std::vector<int32_t> &fcol, std::vector<int32_t> &amap,
                     std::vector<uint8_t> &fill) {
    std::vector<int64_t> stamp((size_t)n, -1);
    std::vector<int32_t> len((size_t)n, 0), stack, a, b, row;
    fptr.assign((size_t)n + 1, 0);
    fcol.clear();
    fill.clear();
    amap.assign((size_t)ptr[n], 0);
    for (int64_t i = 0; i < n; ++i) {
        row.clear();
        if (kind == 2) {
            walk(kLowerThroughUpper, (int32_t)i, level, ptr, col, stamp, 2 * i, len, stack, a);
            walk(kUpperThroughLower, (int32_t)i, level, ptr, col, stamp, 2 * i + 1, len, stack, b);
            row.insert(row.end(), a.begin(), a.end());
            row.push_back((int32_t)i);
            row.insert(row.end(), b.begin(), b.end());
        } else {
            walk(kBall, (int32_t)i, level, ptr, col, stamp, 2 * i, len, stack, a);
            row.insert(row.end(), a.begin(), a.end());
            for (int32_t t = ptr[i]; t < ptr[i + 1]; ++t) row.push_back(col[t]);
        }
        std::sort(row.begin(), row.end());
        row.erase(std::unique(row.begin(), row.end()), row.end());
        // the matrix's own entries must be part of the pattern
        size_t q = 0;
        for (int32_t t = ptr[i]; t < ptr[i + 1]; ++t) {
            while (q < row.size() && row[q] < col[t]) ++q;
            if (q == row.size() || row[q] != col[t]) return false;
            amap[t] = (int32_t)(fcol.size() + q);
        }
        for (size_t u = 0; u < row.size(); ++u) {
            fcol.push_back(row[u]);
            bool in_a = false;
            for (int32_t t = ptr[i]; t < ptr[i + 1] && !in_a; ++t) in_a = col[t] == row[u];
            fill.push_back(in_a ? 0 : 1);
        }
        fptr[i + 1] = (int32_t)fcol.size();
        if ((int64_t)fcol.size() > 0x7fffffffLL - 64) return false;
    }
    return true;
}
