// IC(0) / ILU(0) factorisation and the triangular sweeps that apply them.
//
// Reference: src/linalg/preconditioners/incomplete_cholesky.rs (build :148-202,
// compute :87-145, precondition :217-255) and incomplete_lower_upper.rs
// (build_and_compute_row_by_row :200-261 with the drop rule of
// src/linalg/sparse_array.rs:48-50, precondition :287-329).
//
// Design.  Both the numeric factorisation and the sweeps are dependency
// graphs over rows (row i needs the rows j of its strict lower part forward,
// of its strict upper part backward).  Rows are processed in level order
// (a stable sort by level of the DAG), handed out 32 at a time to warps via an
// atomic ticket, one row per lane.  A row waits only for the rows it depends
// on, through the produced values themselves (sweeps: a slot holds the
// all-ones sentinel until written) or through per-row done flags
// (factorisation).  Because tickets are taken in order by running warps, the
// oldest unfinished row always belongs to a running warp whose inputs are
// ready: the scheme cannot deadlock whatever the grid size or the other work
// on the GPU, and every wait is bounded in time anyway.
//
// Each row is computed in the reference's own order (ascending column, same
// reciprocal-then-multiply, no FMA), so the factors and the sweep results are
// the reference's bits.  ILU entries dropped by the 1e-6 rule are stored as
// exact zeros in place: subtracting lik*0 or l_ij*0 leaves every later value
// unchanged, which is what skipping them does in the reference.
#include <algorithm>
#include <cmath>
#include <new>
#include <type_traits>
#include <vector>

#include <cub/cub.cuh>

#include "fv_internal.cuh"

struct fv_symbolic {
    int64_t n = 0, nnz_l = 0, nnz_u = 0;
    int32_t *l_ptr = nullptr, *l_col = nullptr;  // strict lower part of the pattern
    int32_t *u_ptr = nullptr, *u_col = nullptr;  // strict upper part
    int32_t *fwd_order = nullptr, *bwd_order = nullptr;
    int32_t *l_tpos = nullptr;                   // L entry (i,j) -> slot of (j,i) in U (IC only)
    int32_t n_fwd_levels = 0, n_bwd_levels = 0;
    int32_t max_row = 0;                         // longest row of the pattern
    int32_t max_lower = 0, max_upper = 0;        // longest strict-lower / strict-upper row
    bool symmetric_pattern = false;
    std::vector<int32_t> h_fwd_level, h_bwd_level;   // host copies (filled on demand for device-built schedules)
    int32_t *d_fwd_level = nullptr, *d_bwd_level = nullptr;  // device-built schedules only
    // box tiling of the two sweeps ([0] forward over L, [1] backward over U);
    // absent (tiled = false) for matrices without mesh geometry or without an
    // acyclic box order
    // Steps are laid out as 32 slots each (slot = 32 * step + lane); per slot
    // the row (-1 idle), the entries' positions in the swept side's value
    // array and their dependency sources (4 per slot, FV_TILE_PAD when unused),
    // and the slot of the row in the other direction's plan.
    bool tiled = false, tiles_tried = false;
    int32_t t_nb[2] = {0, 0};
    int64_t t_nslots[2] = {0, 0};
    int32_t *t_box_step[2] = {nullptr, nullptr};
    int32_t *t_slot_row[2] = {nullptr, nullptr}, *t_slot_src[2] = {nullptr, nullptr};
    int32_t *t_slot_ds[2] = {nullptr, nullptr}, *t_slot_next[2] = {nullptr, nullptr};
    double t_lane_use[2] = {0, 0}, t_ring_share[2] = {0, 0}, t_edge = 0;
};

void fv_symbolic_free(fv_symbolic *s) {
    if (!s) return;
    cudaFree(s->l_ptr);
    cudaFree(s->l_col);
    cudaFree(s->u_ptr);
    cudaFree(s->u_col);
    cudaFree(s->fwd_order);
    cudaFree(s->bwd_order);
    cudaFree(s->l_tpos);
    cudaFree(s->d_fwd_level);
    cudaFree(s->d_bwd_level);
    for (int d = 0; d < 2; ++d) {
        cudaFree(s->t_box_step[d]);
        cudaFree(s->t_slot_row[d]);
        cudaFree(s->t_slot_src[d]);
        cudaFree(s->t_slot_ds[d]);
        cudaFree(s->t_slot_next[d]);
    }
    delete s;
}

struct fv_precond {
    int kind = 0;  // 1 = IC(0), 2 = ILU(0)
    int64_t n = 0;
    const fv_csr *A = nullptr;
    fv_symbolic *sym = nullptr;  // owned by A
    double *l_val = nullptr, *u_val = nullptr, *diag = nullptr, *dinv = nullptr;
    double *tmp = nullptr;        // forward-sweep output, kept at sentinel between applies
    unsigned *done = nullptr;     // factorisation flags
    unsigned epoch = 0;
    int schedule = 1;             // 1: level chunks (default); 2: box tiles (when planned);
                                  // 3: level chunks, next chunk prefetched; 4: consecutive rows
                                  // (the default when the rows are sorted by forward level)
    bool contiguous = false;      // the rows are sorted by forward level
    int sweep_blocks = 0;         // blocks of 8 warps per sweep launch (0: the kernels' default)
    int sweep_rpt = 0;            // rows per thread of the reordered sweeps (0: default)
    unsigned *ctrl = nullptr;     // [0,1] fwd ticket/exit  [2,3] bwd ticket/exit  [4,5] factor ticket/exit
    int *err = nullptr;
    int64_t n_dropped = 0;
    // FP32 copies of the factors for mixed-precision inner solves
    float *l32 = nullptr, *u32 = nullptr, *dinv32 = nullptr, *tmp32 = nullptr;
    // level k >= 1 with fill: the factorised matrix is `fill` (the pattern of
    // the level-k factor holding the values of `orig`, zeros elsewhere);
    // amap[k] is the position of orig's entry k in it
    fv_csr *fill = nullptr;
    const fv_csr *orig = nullptr;
    int32_t *amap = nullptr;
    int level = 0;
    // reordered factorisation (fv_*_factor_perm): `fill` is B = Q A Q^T, perm[i]
    // = the row of A that is B's row i; the sweeps gather the right-hand side
    // through perm and scatter the result back, the backward sweep's own output
    // (B's numbering, polled by its dependants) lives in zint / zint32
    int32_t *perm = nullptr;
    double *zint = nullptr;
    float *zint32 = nullptr;
    // box-tiled sweeps: per-slot records (factor values in slot order) and
    // slot-ordered right-hand sides, FP64 and FP32; rebuilt when the factors change
    void *t_rec64[2] = {nullptr, nullptr}, *t_rec32[2] = {nullptr, nullptr};
    double *t_rhs64[2] = {nullptr, nullptr};
    float *t_rhs32[2] = {nullptr, nullptr};
    unsigned t_rec64_epoch = 0, t_rec32_version = 0;
    unsigned f32_version = 0;  // incremented by every fv_precond_make_f32
};

// ------------------------------------------------------------------ symbolic
static fv_status build_symbolic_impl(const fv_csr *A, cudaStream_t st, fv_symbolic **out) {
    const int64_t n = A->nrows, nnz = A->nnz;
    std::vector<int32_t> ptr((size_t)n + 1), col((size_t)(nnz ? nnz : 1));
    FV_CUDA_TRY(cudaMemcpyAsync(ptr.data(), A->row_ptr, sizeof(int32_t) * (n + 1), cudaMemcpyDeviceToHost, st));
    if (nnz) FV_CUDA_TRY(cudaMemcpyAsync(col.data(), A->cols, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost, st));
    FV_CUDA_TRY(cudaStreamSynchronize(st));
    fv_symbolic *s = new fv_symbolic();
    s->n = n;
    std::vector<int32_t> lp((size_t)n + 1), up((size_t)n + 1);
    int64_t nl = 0, nu = 0;
    int32_t maxrow = 0;
    for (int64_t i = 0; i < n; ++i) {
        lp[i] = (int32_t)nl;
        up[i] = (int32_t)nu;
        bool has_diag = false;
        maxrow = std::max(maxrow, ptr[i + 1] - ptr[i]);
        for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k) {
            if (k > ptr[i] && col[k] <= col[k - 1]) {
                delete s;
                return FV_ERR_INVALID;  // columns must be sorted and unique
            }
            if (col[k] < i)
                ++nl;
            else if (col[k] > i)
                ++nu;
            else
                has_diag = true;
        }
        if (!has_diag) {  // the reference indexes [[i,i]] and panics
            delete s;
            return FV_ERR_INVALID;
        }
    }
    lp[n] = (int32_t)nl;
    up[n] = (int32_t)nu;
    for (int64_t i = 0; i < n; ++i) {
        s->max_lower = std::max(s->max_lower, lp[i + 1] - lp[i]);
        s->max_upper = std::max(s->max_upper, up[i + 1] - up[i]);
    }
    s->nnz_l = nl;
    s->nnz_u = nu;
    s->max_row = maxrow;
    std::vector<int32_t> lc((size_t)(nl ? nl : 1)), uc((size_t)(nu ? nu : 1));
    const bool fill_order = !A->fill_mask.empty();
    for (int64_t i = 0; i < n; ++i) {
        int32_t a = lp[i], b = up[i];
        for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k) {
            if (col[k] < i) lc[a++] = col[k];
            if (col[k] > i && !(fill_order && A->fill_mask[k])) uc[b++] = col[k];
        }
        // IC(k) fill: a row's fill entries come after the matrix's own entries
        // in the backward sweep (the reference's sp_t order)
        if (fill_order)
            for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k)
                if (col[k] > i && A->fill_mask[k]) uc[b++] = col[k];
    }
    // level schedules (stable: rows of a level keep ascending order)
    auto schedule = [&](bool upper, std::vector<int32_t> &level, std::vector<int32_t> &order) -> int32_t {
        level.assign((size_t)n, 0);
        int32_t nlev = 0;
        if (!upper) {
            for (int64_t i = 0; i < n; ++i) {
                int32_t l = 0;
                for (int32_t k = lp[i]; k < lp[i + 1]; ++k) l = std::max(l, level[lc[k]] + 1);
                level[i] = l;
                nlev = std::max(nlev, l + 1);
            }
        } else {
            for (int64_t i = n - 1; i >= 0; --i) {
                int32_t l = 0;
                for (int32_t k = up[i]; k < up[i + 1]; ++k) l = std::max(l, level[uc[k]] + 1);
                level[i] = l;
                nlev = std::max(nlev, l + 1);
            }
        }
        std::vector<int64_t> start((size_t)nlev + 1, 0);
        for (int64_t i = 0; i < n; ++i) start[level[i] + 1]++;
        for (int32_t l = 0; l < nlev; ++l) start[l + 1] += start[l];
        order.assign((size_t)n, 0);
        for (int64_t i = 0; i < n; ++i) order[start[level[i]]++] = (int32_t)i;
        return nlev;
    };
    std::vector<int32_t> fo, bo;
    s->n_fwd_levels = schedule(false, s->h_fwd_level, fo);
    s->n_bwd_levels = schedule(true, s->h_bwd_level, bo);
    // transpose map L(i,j) -> U(j,i); also tells whether the pattern is symmetric
    std::vector<int32_t> tpos((size_t)(nl ? nl : 1)), cur(up.begin(), up.end() - 1);
    bool sym = (nl == nu);
    for (int64_t i = 0; i < n && sym; ++i)
        for (int32_t k = lp[i]; k < lp[i + 1]; ++k) {
            int32_t j = lc[k];
            int32_t p = -1;
            if (!fill_order) {  // U rows ascending: the entries of row j appear in order of i
                p = cur[j]++;
                if (p >= up[j + 1] || uc[p] != i) p = -1;
            } else {
                for (int32_t t = up[j]; t < up[j + 1]; ++t)
                    if (uc[t] == i) p = t;
            }
            if (p < 0) {
                sym = false;
                break;
            }
            tpos[k] = p;
        }
    s->symmetric_pattern = sym;
    cudaError_t e = cudaSuccess;
    auto up_load = [&](int32_t **d, const std::vector<int32_t> &h, size_t cnt) {
        if (e != cudaSuccess) return;
        e = cudaMalloc(d, sizeof(int32_t) * (cnt ? cnt : 1));
        if (e == cudaSuccess && cnt) e = cudaMemcpyAsync(*d, h.data(), sizeof(int32_t) * cnt, cudaMemcpyHostToDevice, st);
    };
    up_load(&s->l_ptr, lp, (size_t)n + 1);
    up_load(&s->u_ptr, up, (size_t)n + 1);
    up_load(&s->l_col, lc, (size_t)nl);
    up_load(&s->u_col, uc, (size_t)nu);
    up_load(&s->fwd_order, fo, (size_t)n);
    up_load(&s->bwd_order, bo, (size_t)n);
    if (sym) up_load(&s->l_tpos, tpos, (size_t)nl);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        fv_internal_set_cuda_error(e, "symbolic upload");
        fv_symbolic_free(s);
        return e == cudaErrorMemoryAllocation ? FV_ERR_ALLOC : FV_ERR_CUDA;
    }
    *out = s;
    return FV_OK;
}

static fv_status build_symbolic(const fv_csr *A, cudaStream_t st, fv_symbolic **out) {
    return fv_host_guard([&] { return build_symbolic_impl(A, st, out); });
}

static fv_status ensure_host_levels(fv_symbolic *s, cudaStream_t st);

// Box tiles of the two sweeps, planned on first request when the matrix was
// assembled on a mesh (cell centres known); s->tiled says whether a plan exists.
static fv_status build_tiles_impl(fv_symbolic *s, const fv_csr *A, cudaStream_t st) {
    if (s->tiles_tried) return FV_OK;
    s->tiles_tried = true;
    const int64_t n = s->n;
    if (!A->mesh || A->mesh->n_cells != n || n <= 0) return FV_OK;
    std::vector<int32_t> lp((size_t)n + 1), up((size_t)n + 1), lc((size_t)(s->nnz_l ? s->nnz_l : 1)),
        uc((size_t)(s->nnz_u ? s->nnz_u : 1)), fo((size_t)n), bo((size_t)n);
    std::vector<double4> cells((size_t)n);
    FV_CUDA_TRY(cudaMemcpyAsync(lp.data(), s->l_ptr, sizeof(int32_t) * (n + 1), cudaMemcpyDeviceToHost, st));
    FV_CUDA_TRY(cudaMemcpyAsync(up.data(), s->u_ptr, sizeof(int32_t) * (n + 1), cudaMemcpyDeviceToHost, st));
    if (s->nnz_l)
        FV_CUDA_TRY(cudaMemcpyAsync(lc.data(), s->l_col, sizeof(int32_t) * s->nnz_l, cudaMemcpyDeviceToHost, st));
    if (s->nnz_u)
        FV_CUDA_TRY(cudaMemcpyAsync(uc.data(), s->u_col, sizeof(int32_t) * s->nnz_u, cudaMemcpyDeviceToHost, st));
    FV_CUDA_TRY(cudaMemcpyAsync(fo.data(), s->fwd_order, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st));
    FV_CUDA_TRY(cudaMemcpyAsync(bo.data(), s->bwd_order, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st));
    FV_CUDA_TRY(cudaMemcpyAsync(cells.data(), A->mesh->cell, sizeof(double4) * n, cudaMemcpyDeviceToHost, st));
    FV_CUDA_TRY(cudaStreamSynchronize(st));
    fv_tile_plan tp[2];
    if (s->max_lower > FV_TILE_MAXL || s->max_upper > FV_TILE_MAXL) return FV_OK;
    FV_TRY(ensure_host_levels(s, st));
    if (!fv_build_tile_plans(n, A->mesh->dim, (const double *)cells.data(), lp.data(), lc.data(), up.data(),
                             uc.data(), s->h_fwd_level.data(), s->h_bwd_level.data(), fo.data(), bo.data(),
                             FV_TILE_RING, tp[0], tp[1]))
        return FV_OK;
    // slot layout of both directions
    std::vector<int32_t> srow[2], ssrc[2], sds[2], snext[2], row_slot[2];
    for (int d = 0; d < 2; ++d) {
        const int64_t nslots = 32LL * tp[d].nsteps;
        srow[d].assign((size_t)nslots, -1);
        ssrc[d].assign((size_t)nslots * FV_TILE_MAXL, -1);
        sds[d].assign((size_t)nslots * FV_TILE_MAXL, FV_TILE_PAD);
        row_slot[d].assign((size_t)n, -1);
        const std::vector<int32_t> &ptr = d == 0 ? lp : up;
        for (int32_t st = 0; st < tp[d].nsteps; ++st)
            for (int32_t u = tp[d].sptr[st]; u < tp[d].sptr[st + 1]; ++u) {
                const int64_t slot = 32LL * st + (u - tp[d].sptr[st]);
                const int32_t row = tp[d].trow[u];
                srow[d][slot] = row;
                row_slot[d][row] = (int32_t)slot;
                for (int32_t k = ptr[row]; k < ptr[row + 1]; ++k) {
                    ssrc[d][slot * FV_TILE_MAXL + (k - ptr[row])] = k;
                    sds[d][slot * FV_TILE_MAXL + (k - ptr[row])] = tp[d].dsrc[k];
                }
            }
        if (32LL * tp[d].nsteps >= 0x7fffffffLL) return FV_OK;
    }
    for (int d = 0; d < 2; ++d) {  // the forward sweep writes the backward sweep's rhs in its slot order
        snext[d].assign(srow[d].size(), -1);
        for (size_t slot = 0; slot < srow[d].size(); ++slot)
            if (d == 0 && srow[d][slot] >= 0) snext[d][slot] = row_slot[1][srow[d][slot]];
    }
    cudaError_t e = cudaSuccess;
    auto up_load = [&](int32_t **dp, const std::vector<int32_t> &h) {
        if (e != cudaSuccess) return;
        e = cudaMalloc(dp, sizeof(int32_t) * (h.size() ? h.size() : 1));
        if (e == cudaSuccess && h.size())
            e = cudaMemcpyAsync(*dp, h.data(), sizeof(int32_t) * h.size(), cudaMemcpyHostToDevice, st);
    };
    for (int d = 0; d < 2; ++d) {
        up_load(&s->t_box_step[d], tp[d].box_step);
        up_load(&s->t_slot_row[d], srow[d]);
        up_load(&s->t_slot_src[d], ssrc[d]);
        up_load(&s->t_slot_ds[d], sds[d]);
        up_load(&s->t_slot_next[d], snext[d]);
        s->t_nb[d] = tp[d].nb;
        s->t_nslots[d] = 32LL * tp[d].nsteps;
        s->t_lane_use[d] = tp[d].lane_use;
        s->t_ring_share[d] = tp[d].ring_share;
    }
    s->t_edge = tp[0].edge;
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        fv_internal_set_cuda_error(e, "tile plan upload");
        return e == cudaErrorMemoryAllocation ? FV_ERR_ALLOC : FV_ERR_CUDA;
    }
    s->tiled = true;
    return FV_OK;
}

static fv_status build_tiles(fv_symbolic *s, const fv_csr *A, cudaStream_t st) {
    return fv_host_guard([&] { return build_tiles_impl(s, A, st); });
}

static fv_status build_symbolic_device(const fv_csr *A, cudaStream_t st, fv_symbolic **out);

// The device analysis serves every pattern without IC(k) fill entries; the
// host one keeps the fill entries' special place in the backward sweep.
fv_status fv_get_symbolic(fv_csr *A, cudaStream_t st, fv_symbolic **out) {
    if (!A->sym) {
        if (A->fill_mask.empty())
            FV_TRY(build_symbolic_device(A, st, &A->sym));
        else
            FV_TRY(build_symbolic(A, st, &A->sym));
    }
    *out = A->sym;
    return FV_OK;
}

// Host copies of the level of every row (box-tile planning, fv_precond_levels).
static fv_status ensure_host_levels_impl(fv_symbolic *s, cudaStream_t st) {
    if (!s->h_fwd_level.empty() || s->n == 0 || !s->d_fwd_level) return FV_OK;
    s->h_fwd_level.resize((size_t)s->n);
    s->h_bwd_level.resize((size_t)s->n);
    FV_CUDA_TRY(cudaMemcpyAsync(s->h_fwd_level.data(), s->d_fwd_level, sizeof(int32_t) * s->n,
                                cudaMemcpyDeviceToHost, st));
    FV_CUDA_TRY(cudaMemcpyAsync(s->h_bwd_level.data(), s->d_bwd_level, sizeof(int32_t) * s->n,
                                cudaMemcpyDeviceToHost, st));
    FV_CUDA_TRY(cudaStreamSynchronize(st));
    return FV_OK;
}

static fv_status ensure_host_levels(fv_symbolic *s, cudaStream_t st) {
    return fv_host_guard([&] { return ensure_host_levels_impl(s, st); });
}

// ------------------------------------------------------------------ kernels
namespace {

__device__ __forceinline__ bool take_chunk(unsigned *ticket, int64_t nchunks, int64_t &chunk) {
    unsigned c = 0;
    if ((threadIdx.x & 31) == 0) c = atomicAdd(ticket, 1u);
    c = __shfl_sync(0xffffffffu, c, 0);
    chunk = c;
    return (int64_t)c < nchunks;
}

__device__ __forceinline__ void leave(unsigned *ticket, unsigned *exits) {
    if ((threadIdx.x & 31) == 0) {
        unsigned total = gridDim.x * (blockDim.x >> 5);
        if (atomicAdd(exits, 1u) == total - 1) {
            *ticket = 0;
            *exits = 0;
        }
    }
}

// ILU(0) numeric, one row per lane (incomplete_lower_upper.rs:207-261).
template <int MAXR>
__global__ void __launch_bounds__(128) k_ilu0(int64_t n, const int32_t *__restrict__ order,
                                              const int32_t *__restrict__ a_ptr, const double *__restrict__ a_val,
                                              const int32_t *__restrict__ l_ptr, const int32_t *__restrict__ l_col,
                                              const int32_t *__restrict__ u_ptr, const int32_t *__restrict__ u_col,
                                              double *l_val, double *u_val, double *diag, double *dinv,
                                              unsigned *done, unsigned epoch, unsigned *ctrl, int *err) {
    const int64_t nchunks = (n + 31) / 32;
    int64_t chunk;
    while (take_chunk(&ctrl[0], nchunks, chunk)) {
        const int64_t idx = chunk * 32 + (threadIdx.x & 31);
        if (idx >= n) continue;
        const int i = order[idx];
        const int l0 = l_ptr[i], nl = l_ptr[i + 1] - l0;
        const int u0 = u_ptr[i], nu = u_ptr[i + 1] - u0;
        const int m = nl + 1 + nu;
        const int a0 = a_ptr[i];
        int c[MAXR];
        double v[MAXR];
        for (int q = 0; q < m; ++q) {
            v[q] = a_val[a0 + q];
            c[q] = q < nl ? l_col[l0 + q] : (q == nl ? i : u_col[u0 + q - nl - 1]);
        }
        for (int q = 0; q < nl; ++q) {
            const int k = c[q];
            fv_wait_flag(&done[k], epoch, err);
            const double lukk = __ldcg(&diag[k]);
            if (fabs(lukk) < 1e-16) atomicOr(err, FV_DEV_SINGULAR);
            const double lukkinv = 1.0 / lukk;
            v[q] = lukkinv * v[q];
            const double lik = v[q];
            int p = q + 1;
            for (int s = u_ptr[k]; s < u_ptr[k + 1]; ++s) {
                const int j = u_col[s];
                const double term = lik * __ldcg(&u_val[s]);
                while (p < m && c[p] < j) ++p;
                if (p < m && c[p] == j) v[p] -= term;
            }
        }
        const double tol = fabs(v[nl]) * 1e-6;
        for (int q = 0; q < m; ++q)
            if (q != nl && !(fabs(v[q]) > tol)) v[q] = 0.0;
        for (int q = 0; q < nl; ++q) l_val[l0 + q] = v[q];
        for (int q = 0; q < nu; ++q) u_val[u0 + q] = v[nl + 1 + q];
        diag[i] = v[nl];
        dinv[i] = 1.0 / v[nl];
        __threadfence();
        fv_st_release_u32(&done[i], epoch);
    }
    leave(&ctrl[0], &ctrl[1]);
}

// k_ilu0 for short rows (at most MAXR entries: tetrahedra, triangles): the
// same arithmetic in the same order, with the loads rearranged so that one
// level costs about one flag round trip: the row bounds of every U_k are
// read before waiting, all flags are polled together, and then diag[k] and
// every u_kj are loaded at once into registers before the elimination runs.
template <int MAXR>
__global__ void __launch_bounds__(128) k_ilu0s(int64_t n, const int32_t *__restrict__ order,
                                               const int32_t *__restrict__ a_ptr, const double *__restrict__ a_val,
                                               const int32_t *__restrict__ l_ptr, const int32_t *__restrict__ l_col,
                                               const int32_t *__restrict__ u_ptr, const int32_t *__restrict__ u_col,
                                               double *l_val, double *u_val, double *diag, double *dinv,
                                               unsigned *done, unsigned epoch, unsigned *ctrl, int *err) {
    constexpr int MU = MAXR - 1;  // a strict-upper row holds at most MAXR - 1 entries
    const int64_t nchunks = (n + 31) / 32;
    int64_t chunk;
    while (take_chunk(&ctrl[0], nchunks, chunk)) {
        const int64_t idx = chunk * 32 + (threadIdx.x & 31);
        if (idx >= n) continue;
        const int i = __ldg(&order[idx]);
        const int l0 = __ldg(&l_ptr[i]), nl = __ldg(&l_ptr[i + 1]) - l0;
        const int u0 = __ldg(&u_ptr[i]), nu = __ldg(&u_ptr[i + 1]) - u0;
        const int m = nl + 1 + nu;
        const int a0 = __ldg(&a_ptr[i]);
        int c[MAXR];
        double v[MAXR];
#pragma unroll
        for (int q = 0; q < MAXR; ++q)
            if (q < m) {
                v[q] = a_val[a0 + q];
                c[q] = q < nl ? __ldg(&l_col[l0 + q]) : (q == nl ? i : __ldg(&u_col[u0 + q - nl - 1]));
            }
        // static parts of the rows k the elimination reads
        int ub[MAXR], ul[MAXR], ucol[MAXR][MU];
#pragma unroll
        for (int q = 0; q < MAXR; ++q)
            if (q < nl) {
                ub[q] = __ldg(&u_ptr[c[q]]);
                ul[q] = __ldg(&u_ptr[c[q] + 1]) - ub[q];
            }
#pragma unroll
        for (int q = 0; q < MAXR; ++q)
#pragma unroll
            for (int t = 0; t < MU; ++t)
                if (q < nl && t < ul[q]) ucol[q][t] = __ldg(&u_col[ub[q] + t]);
        // every dependency's flag, polled together (bounded)
        unsigned pending = 0;
#pragma unroll
        for (int q = 0; q < MAXR; ++q)
            if (q < nl && fv_ld_acquire_u32(&done[c[q]]) != epoch) pending |= 1u << q;
        if (pending) {
            const unsigned long long t0 = fv_globaltimer();
            for (unsigned it = 1; pending; ++it) {
#pragma unroll
                for (int q = 0; q < MAXR; ++q)
                    if (((pending >> q) & 1u) && fv_ld_acquire_u32(&done[c[q]]) == epoch) pending &= ~(1u << q);
                if (pending && (it & 255u) == 0 &&
                    (*(volatile int *)err || fv_globaltimer() - t0 > FV_WAIT_LIMIT_NS)) {
                    if (!*(volatile int *)err) atomicOr(err, FV_DEV_TIMEOUT);
                    pending = 0;
                }
            }
        }
        // the factored values of those rows, loaded together
        double dk[MAXR], uv[MAXR][MU];
#pragma unroll
        for (int q = 0; q < MAXR; ++q)
            if (q < nl) dk[q] = __ldcg(&diag[c[q]]);
#pragma unroll
        for (int q = 0; q < MAXR; ++q)
#pragma unroll
            for (int t = 0; t < MU; ++t)
                if (q < nl && t < ul[q]) uv[q][t] = __ldcg(&u_val[ub[q] + t]);
        // elimination in the order of k_ilu0
#pragma unroll
        for (int q = 0; q < MAXR; ++q) {
            if (q < nl) {
                const double lukk = dk[q];
                if (fabs(lukk) < 1e-16) atomicOr(err, FV_DEV_SINGULAR);
                const double lukkinv = 1.0 / lukk;
                v[q] = lukkinv * v[q];
                const double lik = v[q];
#pragma unroll
                for (int t = 0; t < MU; ++t) {
                    if (t < ul[q]) {
                        const int j = ucol[q][t];
                        const double term = lik * uv[q][t];
#pragma unroll
                        for (int p = q + 1; p < MAXR; ++p)
                            if (p < m && c[p] == j) v[p] -= term;
                    }
                }
            }
        }
        const double tol = fabs(v[nl]) * 1e-6;
#pragma unroll
        for (int q = 0; q < MAXR; ++q)
            if (q < m && q != nl && !(fabs(v[q]) > tol)) v[q] = 0.0;
#pragma unroll
        for (int q = 0; q < MAXR; ++q) {
            if (q < nl) l_val[l0 + q] = v[q];
            if (q > nl && q < m) u_val[u0 + q - nl - 1] = v[q];
        }
        diag[i] = v[nl];
        dinv[i] = 1.0 / v[nl];
        __threadfence();
        fv_st_release_u32(&done[i], epoch);
    }
    leave(&ctrl[0], &ctrl[1]);
}

// IC(0) numeric, up-looking form of the reference's right-looking loop
// (incomplete_cholesky.rs:87-135): every l_ij receives the same updates
// l_ik*l_jk in ascending k and the same final scaling by 1/l_jj.
template <int MAXR>
__global__ void __launch_bounds__(128) k_ic0(int64_t n, const int32_t *__restrict__ order,
                                             const int32_t *__restrict__ a_ptr, const double *__restrict__ a_val,
                                             const int32_t *__restrict__ l_ptr, const int32_t *__restrict__ l_col,
                                             const int32_t *__restrict__ l_tpos, double *l_val, double *u_val,
                                             double *diag, double *dinv, unsigned *done, unsigned epoch,
                                             unsigned *ctrl, int *err) {
    const int64_t nchunks = (n + 31) / 32;
    int64_t chunk;
    while (take_chunk(&ctrl[0], nchunks, chunk)) {
        const int64_t idx = chunk * 32 + (threadIdx.x & 31);
        if (idx >= n) continue;
        const int i = order[idx];
        const int l0 = l_ptr[i], nl = l_ptr[i + 1] - l0;
        const int a0 = a_ptr[i];
        int c[MAXR];
        double v[MAXR];
        for (int q = 0; q < nl; ++q) {
            c[q] = l_col[l0 + q];
            v[q] = a_val[a0 + q];
        }
        double vd = a_val[a0 + nl];
        for (int q = 0; q < nl; ++q) {
            const int j = c[q];
            fv_wait_flag(&done[j], epoch, err);
            // merge row i (k < j) with row j's strict lower part
            int p = 0;
            const int s1 = l_ptr[j + 1];
            for (int s = l_ptr[j]; s < s1 && p < q; ++s) {
                const int k = l_col[s];
                while (p < q && c[p] < k) ++p;
                if (p < q && c[p] == k) v[q] -= v[p] * __ldcg(&l_val[s]);
            }
            v[q] = __ldcg(&dinv[j]) * v[q];
        }
        for (int q = 0; q < nl; ++q) vd -= v[q] * v[q];
        const double lii = sqrt(vd);
        for (int q = 0; q < nl; ++q) {
            l_val[l0 + q] = v[q];
            u_val[l_tpos[l0 + q]] = v[q];
        }
        diag[i] = lii;
        dinv[i] = 1.0 / lii;
        __threadfence();
        fv_st_release_u32(&done[i], epoch);
    }
    leave(&ctrl[0], &ctrl[1]);
}

// k_ic0 for short rows, rearranged like k_ilu0s: row j's lower bounds and
// columns before the wait, all flags polled together, dinv[j] and row j's
// lower values loaded at once; the arithmetic and its order are k_ic0's.
template <int MAXR>
__global__ void __launch_bounds__(128) k_ic0s(int64_t n, const int32_t *__restrict__ order,
                                              const int32_t *__restrict__ a_ptr, const double *__restrict__ a_val,
                                              const int32_t *__restrict__ l_ptr, const int32_t *__restrict__ l_col,
                                              const int32_t *__restrict__ l_tpos, double *l_val, double *u_val,
                                              double *diag, double *dinv, unsigned *done, unsigned epoch,
                                              unsigned *ctrl, int *err) {
    constexpr int ML = MAXR - 1;  // a strict-lower row holds at most MAXR - 1 entries
    const int64_t nchunks = (n + 31) / 32;
    int64_t chunk;
    while (take_chunk(&ctrl[0], nchunks, chunk)) {
        const int64_t idx = chunk * 32 + (threadIdx.x & 31);
        if (idx >= n) continue;
        const int i = __ldg(&order[idx]);
        const int l0 = __ldg(&l_ptr[i]), nl = __ldg(&l_ptr[i + 1]) - l0;
        const int a0 = __ldg(&a_ptr[i]);
        int c[ML];
        double v[ML];
#pragma unroll
        for (int q = 0; q < ML; ++q)
            if (q < nl) {
                c[q] = __ldg(&l_col[l0 + q]);
                v[q] = a_val[a0 + q];
            }
        double vd = a_val[a0 + nl];
        int lb[ML], ln[ML], lc[ML][ML];
#pragma unroll
        for (int q = 0; q < ML; ++q)
            if (q < nl) {
                lb[q] = __ldg(&l_ptr[c[q]]);
                ln[q] = __ldg(&l_ptr[c[q] + 1]) - lb[q];
            }
#pragma unroll
        for (int q = 0; q < ML; ++q)
#pragma unroll
            for (int t = 0; t < ML; ++t)
                if (q < nl && t < ln[q]) lc[q][t] = __ldg(&l_col[lb[q] + t]);
        unsigned pending = 0;
#pragma unroll
        for (int q = 0; q < ML; ++q)
            if (q < nl && fv_ld_acquire_u32(&done[c[q]]) != epoch) pending |= 1u << q;
        if (pending) {
            const unsigned long long t0 = fv_globaltimer();
            for (unsigned it = 1; pending; ++it) {
#pragma unroll
                for (int q = 0; q < ML; ++q)
                    if (((pending >> q) & 1u) && fv_ld_acquire_u32(&done[c[q]]) == epoch) pending &= ~(1u << q);
                if (pending && (it & 255u) == 0 &&
                    (*(volatile int *)err || fv_globaltimer() - t0 > FV_WAIT_LIMIT_NS)) {
                    if (!*(volatile int *)err) atomicOr(err, FV_DEV_TIMEOUT);
                    pending = 0;
                }
            }
        }
        double dj[ML], lv[ML][ML];
#pragma unroll
        for (int q = 0; q < ML; ++q)
            if (q < nl) dj[q] = __ldcg(&dinv[c[q]]);
#pragma unroll
        for (int q = 0; q < ML; ++q)
#pragma unroll
            for (int t = 0; t < ML; ++t)
                if (q < nl && t < ln[q]) lv[q][t] = __ldcg(&l_val[lb[q] + t]);
        // k_ic0's merge: for each dependency j (ascending) the row's own k < j
        // against row j's lower part, ascending k
#pragma unroll
        for (int q = 0; q < ML; ++q) {
            if (q < nl) {
#pragma unroll
                for (int t = 0; t < ML; ++t) {
                    if (t < ln[q]) {
                        const int k = lc[q][t];
#pragma unroll
                        for (int p = 0; p < ML; ++p)
                            if (p < q && c[p] == k) v[q] -= v[p] * lv[q][t];
                    }
                }
                v[q] = dj[q] * v[q];
            }
        }
#pragma unroll
        for (int q = 0; q < ML; ++q)
            if (q < nl) vd -= v[q] * v[q];
        const double lii = sqrt(vd);
#pragma unroll
        for (int q = 0; q < ML; ++q)
            if (q < nl) {
                l_val[l0 + q] = v[q];
                u_val[__ldg(&l_tpos[l0 + q])] = v[q];
            }
        diag[i] = lii;
        dinv[i] = 1.0 / lii;
        __threadfence();
        fv_st_release_u32(&done[i], epoch);
    }
    leave(&ctrl[0], &ctrl[1]);
}

// |a_ij - a_ji| < 1e-14 for every stored pair (is_symmetric, dmatrix.rs:76-88)
__global__ void k_check_symmetric(int64_t n, const int32_t *__restrict__ a_ptr, const double *__restrict__ a_val,
                                  const int32_t *__restrict__ l_ptr, const int32_t *__restrict__ l_col,
                                  const int32_t *__restrict__ u_ptr, const int32_t *__restrict__ l_tpos, int *bad) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int l0 = l_ptr[i], nl = l_ptr[i + 1] - l0, a0 = a_ptr[i];
    for (int q = 0; q < nl; ++q) {
        // the transposed entry (j,i) sits in U slot p of row j, i.e. at A position
        // a_ptr[j] + (number of strict-lower entries of row j) + 1 + (p - u_ptr[j])
        const int j = l_col[l0 + q];
        const int p = l_tpos[l0 + q];
        const double aji = a_val[a_ptr[j] + (l_ptr[j + 1] - l_ptr[j]) + 1 + (p - u_ptr[j])];
        const double aij = a_val[a0 + q];
        if (!(fabs(aij - aji) < 1e-14)) atomicOr(bad, 1);
    }
}

__global__ void k_count_dropped(int64_t nl, const double *__restrict__ l_val, int64_t nu,
                                const double *__restrict__ u_val, unsigned long long *cnt) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned c = 0;
    for (int64_t k = t; k < nl; k += (int64_t)gridDim.x * blockDim.x) c += (l_val[k] == 0.0);
    for (int64_t k = t; k < nu; k += (int64_t)gridDim.x * blockDim.x) c += (u_val[k] == 0.0);
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(cnt, (unsigned long long)c);
}

}  // namespace

// Triangular sweep (one row per lane, level order, values as readiness).
//   x_i = [dinv_i *] (rhs_i - sum_{j in row} val * x_j), ascending j.
// After reading rhs_i the lane may reset it to the sentinel (rhs_reset), and
// it may pre-fill a later sweep's output slot (next_reset) with the sentinel.
//
// Everything a row needs apart from its dependencies' values (its position in
// the level order, row bounds, columns, coefficients, rhs, 1/diagonal) is
// loaded before the first wait, and all dependencies are polled together, so
// the critical path from one level to the next is one store plus one L2 read.
// MAXL bounds the off-diagonal count of a row on the swept side; rows are
// held in registers.
template <typename T>
__device__ __forceinline__ bool fv_slot_ready(const T *p, T &v);
template <>
__device__ __forceinline__ bool fv_slot_ready<double>(const double *p, double &v) {
    unsigned long long b = fv_ld_relaxed_u64(p);
    v = __longlong_as_double((long long)b);
    return b != FV_SENTINEL_U64;
}
template <>
__device__ __forceinline__ bool fv_slot_ready<float>(const float *p, float &v) {
    unsigned b = fv_ld_relaxed_u32(p);
    v = __uint_as_float(b);
    return b != FV_SENTINEL_U32;
}

// The permutation of a reordered factorisation (fv_ilu0_factor_perm and
// friends): the factor's row i is row nat[i] of the caller's vectors.  The
// forward sweep reads its right-hand side at nat[i] (gather); the backward
// sweep also stores its result at out[nat[i]] (scatter).  Row groups of a
// batch are indexed in the caller's numbering.  nat == nullptr: no
// permutation.
template <typename T>
struct SweepPerm {
    const int32_t *nat = nullptr;
    bool gather = false;
    T *out = nullptr;
};

template <typename T, bool UNIT, int MAXL>
__global__ void __launch_bounds__(256) k_sweep(int64_t n, const int32_t *__restrict__ order,
                                               const int32_t *__restrict__ ptr, const int32_t *__restrict__ col,
                                               const T *__restrict__ val, const T *__restrict__ dinv,
                                               const T *rhs, T *x, T *rhs_reset, T *next_reset, unsigned *ctrl,
                                               int *err, const int *skip, fv_row_skip rs, SweepPerm<T> pm) {
    if (skip && *(volatile const int *)skip) return;  // a converged solve: no warp takes a ticket
    const int64_t nchunks = (n + 31) / 32;
    int64_t chunk;
    while (take_chunk(&ctrl[0], nchunks, chunk)) {
        const int64_t idx = chunk * 32 + (threadIdx.x & 31);
        if (idx >= n) continue;
        const int i = order ? __ldg(&order[idx]) : (int)idx;
        const int nat = pm.nat ? __ldg(&pm.nat[i]) : i;  // the row in the caller's numbering
        // a converged problem's rows (and all their dependencies) are skipped together
        if (rs.group && rs.done[(int64_t)__ldg(&rs.group[nat]) * rs.stride]) continue;
        const int k0 = __ldg(&ptr[i]);
        const int m = __ldg(&ptr[i + 1]) - k0;
        int c[MAXL];
        T v[MAXL], xv[MAXL];
#pragma unroll
        for (int q = 0; q < MAXL; ++q)
            if (q < m) {
                c[q] = __ldg(&col[k0 + q]);
                v[q] = __ldg(&val[k0 + q]);
            }
        T s = rhs[pm.gather ? nat : i];
        const T d = UNIT ? T(1) : __ldg(&dinv[i]);
        unsigned pending = 0;
#pragma unroll
        for (int q = 0; q < MAXL; ++q)
            if (q < m && !fv_slot_ready(&x[c[q]], xv[q])) pending |= 1u << q;
        if (pending) {
            const unsigned long long t0 = fv_globaltimer();
            for (unsigned it = 1; pending; ++it) {
#pragma unroll
                for (int q = 0; q < MAXL; ++q)
                    if ((pending >> q) & 1u)
                        if (fv_slot_ready(&x[c[q]], xv[q])) pending &= ~(1u << q);
                if (pending && (it & 255u) == 0) {
                    if (*(volatile int *)err || fv_globaltimer() - t0 > FV_WAIT_LIMIT_NS) {
                        if (!*(volatile int *)err) atomicOr(err, FV_DEV_TIMEOUT);
#pragma unroll
                        for (int q = 0; q < MAXL; ++q)
                            if ((pending >> q) & 1u) xv[q] = T(NAN);
                        pending = 0;
                    }
                }
            }
        }
#pragma unroll
        for (int q = 0; q < MAXL; ++q)
            if (q < m) s = s - v[q] * xv[q];
        const T r = UNIT ? s : d * s;
        fv_publish(&x[i], r);
        if (pm.out) pm.out[nat] = r;
        // sentinel resets come after the publish: a store to the slot just
        // read would otherwise sit on the row's critical path
        if (rhs_reset) fv_reset_slot(&rhs_reset[i]);
        if (next_reset) fv_reset_slot(&next_reset[i]);
    }
    leave(&ctrl[0], &ctrl[1]);
}

// k_sweep with the next chunk's static data loaded before the current chunk
// waits: each warp holds two tickets, so twice the rows' independent loads
// (order -> row bounds -> entries, rhs, 1/diagonal) are in flight while the
// frontier waits for values.  Tickets are taken and processed in increasing
// order per warp, so the lowest unfinished ticket is always some warp's
// current chunk and its dependencies (earlier tickets) are finished.
template <typename T, int MAXL>
struct SweepRow {
    int i, m, nat;
    bool live;
    int c[MAXL];
    T v[MAXL];
    T s, d;
};

template <typename T, bool UNIT, int MAXL>
__device__ __forceinline__ void sweep_stage(SweepRow<T, MAXL> &r, int64_t chunk, int64_t n,
                                            const int32_t *__restrict__ order, const int32_t *__restrict__ ptr,
                                            const int32_t *__restrict__ col, const T *__restrict__ val,
                                            const T *__restrict__ dinv, const T *rhs, const fv_row_skip &rs,
                                            const SweepPerm<T> &pm) {
    const int64_t idx = chunk * 32 + (threadIdx.x & 31);
    r.live = idx < n;
    if (!r.live) return;
    r.i = order ? __ldg(&order[idx]) : (int)idx;
    r.nat = pm.nat ? __ldg(&pm.nat[r.i]) : r.i;
    if (rs.group && rs.done[(int64_t)__ldg(&rs.group[r.nat]) * rs.stride]) {
        r.live = false;
        return;
    }
    const int k0 = __ldg(&ptr[r.i]);
    r.m = __ldg(&ptr[r.i + 1]) - k0;
#pragma unroll
    for (int q = 0; q < MAXL; ++q)
        if (q < r.m) {
            r.c[q] = __ldg(&col[k0 + q]);
            r.v[q] = __ldg(&val[k0 + q]);
        }
    r.s = rhs[pm.gather ? r.nat : r.i];
    r.d = UNIT ? T(1) : __ldg(&dinv[r.i]);
}

template <typename T, bool UNIT, int MAXL>
__global__ void __launch_bounds__(256) k_sweep_pf(int64_t n, const int32_t *__restrict__ order,
                                                  const int32_t *__restrict__ ptr, const int32_t *__restrict__ col,
                                                  const T *__restrict__ val, const T *__restrict__ dinv,
                                                  const T *rhs, T *x, T *rhs_reset, T *next_reset, unsigned *ctrl,
                                                  int *err, const int *skip, fv_row_skip rs, SweepPerm<T> pm) {
    if (skip && *(volatile const int *)skip) return;
    const int64_t nchunks = (n + 31) / 32;
    int64_t chunk;
    bool have = take_chunk(&ctrl[0], nchunks, chunk);
    SweepRow<T, MAXL> a, b;
    if (have) sweep_stage<T, UNIT, MAXL>(a, chunk, n, order, ptr, col, val, dinv, rhs, rs, pm);
    while (have) {
        int64_t next;
        const bool have_next = take_chunk(&ctrl[0], nchunks, next);
        if (have_next) sweep_stage<T, UNIT, MAXL>(b, next, n, order, ptr, col, val, dinv, rhs, rs, pm);
        if (a.live) {
            T xv[MAXL];
            unsigned pending = 0;
#pragma unroll
            for (int q = 0; q < MAXL; ++q)
                if (q < a.m && !fv_slot_ready(&x[a.c[q]], xv[q])) pending |= 1u << q;
            if (pending) {
                const unsigned long long t0 = fv_globaltimer();
                for (unsigned it = 1; pending; ++it) {
#pragma unroll
                    for (int q = 0; q < MAXL; ++q)
                        if ((pending >> q) & 1u)
                            if (fv_slot_ready(&x[a.c[q]], xv[q])) pending &= ~(1u << q);
                    if (pending && (it & 255u) == 0) {
                        if (*(volatile int *)err || fv_globaltimer() - t0 > FV_WAIT_LIMIT_NS) {
                            if (!*(volatile int *)err) atomicOr(err, FV_DEV_TIMEOUT);
#pragma unroll
                            for (int q = 0; q < MAXL; ++q)
                                if ((pending >> q) & 1u) xv[q] = T(NAN);
                            pending = 0;
                        }
                    }
                }
            }
            T s = a.s;
#pragma unroll
            for (int q = 0; q < MAXL; ++q)
                if (q < a.m) s = s - a.v[q] * xv[q];
            const T r = UNIT ? s : a.d * s;
            fv_publish(&x[a.i], r);
            if (pm.out) pm.out[a.nat] = r;
            if (rhs_reset) fv_reset_slot(&rhs_reset[a.i]);
            if (next_reset) fv_reset_slot(&next_reset[a.i]);
        }
        a = b;
        have = have_next;
    }
    leave(&ctrl[0], &ctrl[1]);
}

// Sweep of a reordered factorisation (fv_*_factor_perm with a level-sorted
// ordering such as fv_order_boxes): every level is a contiguous range of rows
// and rows of one level are never coupled, so rows are taken in index order
// (forward) or reverse index order (backward: the forward levels descending
// are a valid schedule of the upper triangle, whose dependencies always lie at
// higher indices).  A block takes 256 * RPT consecutive rows per ticket (one
// atomic per block chunk instead of one per warp), every thread loads the
// static data of all its RPT rows before it polls any dependency, and there is
// no level-order indirection, so a wide level streams at memory speed.
// Deadlock-free for any grid: tickets are taken in order by running blocks,
// every dependency lies at a lower position (earlier chunk, or earlier row of
// the same chunk, which its thread handles first), so the lowest unfinished
// row always belongs to a running block and has its inputs.
template <typename T, bool UNIT, int MAXL, int RPT, bool REV>
__global__ void __launch_bounds__(256, RPT == 1 ? 5 : 1) k_sweep_seq(int64_t n, const int32_t *__restrict__ ptr,
                                                   const int32_t *__restrict__ col, const T *__restrict__ val,
                                                   const T *__restrict__ dinv, const T *rhs, T *x, T *rhs_reset,
                                                   T *next_reset, unsigned *ctrl, int *err, const int *skip,
                                                   fv_row_skip rs, SweepPerm<T> pm) {
    if (skip && *(volatile const int *)skip) return;
    constexpr int CH = 256 * RPT;
    const int64_t nchunks = (n + CH - 1) / CH;
    // tickets alternate between two slots: thread 0 writes slot k%2 at chunk k,
    // and every thread reads it before the barrier of chunk k+1
    __shared__ unsigned s_ticket[2];
    if (threadIdx.x == 0) s_ticket[0] = atomicAdd(&ctrl[0], 1u);
    __syncthreads();
    int64_t chunk = s_ticket[0];
    // row bounds and caller-numbered rows of a chunk, loaded one chunk ahead
    int i[RPT], nat[RPT], k0[RPT], k1[RPT];
    auto addresses = [&](int64_t ch) {
#pragma unroll
        for (int q = 0; q < RPT; ++q) {
            const int64_t idx = ch * CH + q * 256 + threadIdx.x;
            k0[q] = 0;
            k1[q] = -1;  // not live
            if (ch >= nchunks || idx >= n) continue;
            i[q] = REV ? (int)(n - 1 - idx) : (int)idx;
            nat[q] = pm.nat ? __ldg(&pm.nat[i[q]]) : i[q];
            k0[q] = __ldg(&ptr[i[q]]);
            k1[q] = __ldg(&ptr[i[q] + 1]);
        }
    };
    addresses(chunk);
    for (unsigned k = 1; chunk < nchunks; ++k) {
        // the next ticket is taken now, so its atomic overlaps this chunk's
        // work; a block's tickets increase, so the lowest unfinished row is
        // always in some block's current chunk
        if (threadIdx.x == 0) s_ticket[k & 1] = atomicAdd(&ctrl[0], 1u);
        int ci[RPT], cnat[RPT], m[RPT], c[RPT][MAXL];
        T v[RPT][MAXL], sr[RPT], d[RPT];
#pragma unroll
        for (int q = 0; q < RPT; ++q) {
            ci[q] = i[q];
            cnat[q] = nat[q];
            m[q] = k1[q] - k0[q];
            if (m[q] < 0) continue;
            // a converged problem's rows (and all their dependencies) are skipped together
            if (rs.group && rs.done[(int64_t)__ldg(&rs.group[cnat[q]]) * rs.stride]) {
                m[q] = -1;
                continue;
            }
#pragma unroll
            for (int t = 0; t < MAXL; ++t)
                if (t < m[q]) {
                    c[q][t] = __ldg(&col[k0[q] + t]);
                    v[q][t] = __ldg(&val[k0[q] + t]);
                }
            sr[q] = rhs[pm.gather ? cnat[q] : ci[q]];
            d[q] = UNIT ? T(1) : __ldg(&dinv[ci[q]]);
        }
        __syncthreads();
        const int64_t next = s_ticket[k & 1];
        addresses(next);  // the next chunk's bounds load while this chunk waits and computes
#pragma unroll
        for (int q = 0; q < RPT; ++q) {
            if (m[q] < 0) continue;
            T xv[MAXL];
            unsigned pending = 0;
#pragma unroll
            for (int t = 0; t < MAXL; ++t)
                if (t < m[q] && !fv_slot_ready(&x[c[q][t]], xv[t])) pending |= 1u << t;
            if (pending) {
                const unsigned long long t0 = fv_globaltimer();
                for (unsigned it = 1; pending; ++it) {
#pragma unroll
                    for (int t = 0; t < MAXL; ++t)
                        if ((pending >> t) & 1u)
                            if (fv_slot_ready(&x[c[q][t]], xv[t])) pending &= ~(1u << t);
                    if (pending && (it & 255u) == 0) {
                        if (*(volatile int *)err || fv_globaltimer() - t0 > FV_WAIT_LIMIT_NS) {
                            if (!*(volatile int *)err) atomicOr(err, FV_DEV_TIMEOUT);
#pragma unroll
                            for (int t = 0; t < MAXL; ++t)
                                if ((pending >> t) & 1u) xv[t] = T(NAN);
                            pending = 0;
                        }
                    }
                }
            }
            T s = sr[q];
#pragma unroll
            for (int t = 0; t < MAXL; ++t)
                if (t < m[q]) s = s - v[q][t] * xv[t];
            const T r = UNIT ? s : d[q] * s;
            fv_publish(&x[ci[q]], r);
            if (pm.out) pm.out[cnat[q]] = r;
            if (rhs_reset) fv_reset_slot(&rhs_reset[ci[q]]);
            if (next_reset) fv_reset_slot(&next_reset[ci[q]]);
        }
        chunk = next;
    }
    leave(&ctrl[0], &ctrl[1]);
}

// Rows longer than 32 entries on the swept side: one dependency at a time.
template <typename T, bool UNIT>
__global__ void __launch_bounds__(256) k_sweep_long(int64_t n, const int32_t *__restrict__ order,
                                                    const int32_t *__restrict__ ptr, const int32_t *__restrict__ col,
                                                    const T *__restrict__ val, const T *__restrict__ dinv,
                                                    const T *rhs, T *x, T *rhs_reset, T *next_reset, unsigned *ctrl,
                                                    int *err, const int *skip, fv_row_skip rs, SweepPerm<T> pm) {
    if (skip && *(volatile const int *)skip) return;
    const int64_t nchunks = (n + 31) / 32;
    int64_t chunk;
    while (take_chunk(&ctrl[0], nchunks, chunk)) {
        const int64_t idx = chunk * 32 + (threadIdx.x & 31);
        if (idx >= n) continue;
        const int i = order ? order[idx] : (int)idx;
        const int nat = pm.nat ? pm.nat[i] : i;
        if (rs.group && rs.done[(int64_t)rs.group[nat] * rs.stride]) continue;
        T s = rhs[pm.gather ? nat : i];
        if (rhs_reset) fv_reset_slot(&rhs_reset[i]);
        if (next_reset) fv_reset_slot(&next_reset[i]);
        const int k1 = ptr[i + 1];
        for (int k = ptr[i]; k < k1; ++k) {
            const T xj = fv_wait_value(&x[col[k]], err);
            s = s - val[k] * xj;
        }
        const T r = UNIT ? s : dinv[i] * s;
        fv_publish(&x[i], r);
        if (pm.out) pm.out[nat] = r;
    }
    leave(&ctrl[0], &ctrl[1]);
}

template <typename T, bool UNIT>
static void launch_sweep(int maxl, int G, cudaStream_t st, int64_t n, const int32_t *order, const int32_t *ptr,
                         const int32_t *col, const T *val, const T *dinv, const T *rhs, T *x, T *rhs_reset,
                         T *next_reset, unsigned *ctrl, int *err, const int *skip, fv_row_skip rs = {},
                         bool prefetch = false, SweepPerm<T> pm = {}) {
#define FV_SWEEP(...)                                                                                           \
    fv_note_launch(), __VA_ARGS__<<<G, 256, 0, st>>>(n, order, ptr, col, val, dinv, rhs, x, rhs_reset, next_reset, \
                                                     ctrl, err, skip, rs, pm)
    if (prefetch && maxl <= 4)
        FV_SWEEP(k_sweep_pf<T, UNIT, 4>);
    else if (prefetch && maxl <= 8)
        FV_SWEEP(k_sweep_pf<T, UNIT, 8>);
    else if (maxl <= 4)
        FV_SWEEP(k_sweep<T, UNIT, 4>);
    else if (maxl <= 8)
        FV_SWEEP(k_sweep<T, UNIT, 8>);
    else if (maxl <= 16)
        FV_SWEEP(k_sweep<T, UNIT, 16>);
    else if (maxl <= 32)
        FV_SWEEP(k_sweep<T, UNIT, 32>);
    else
        FV_SWEEP(k_sweep_long<T, UNIT>);
#undef FV_SWEEP
}

// The same sweep over box tiles (fv_tiles.cu).  A warp takes a box (tickets
// in the boxes' dispatch order, every box after the boxes it depends on) and
// runs its steps in level order, one row per lane.  All static data of a step
// -- the row, its factor entries, where each dependency comes from, the slot
// of the row in the next sweep -- sits in one record per (step, lane), and
// the step's right-hand side in a slot-ordered array; both are streamed into
// shared memory with cp.async D steps ahead, so a step waits only for the
// values it depends on: from the warp's ring of its last FV_TILE_RING steps
// (rows of the same box) or, polled like k_sweep, from the vector.
struct __align__(16) TileRec64 {
    double v[FV_TILE_MAXL];
    double d;
    int32_t ds[FV_TILE_MAXL];
    int32_t row, next;
};
struct __align__(16) TileRec32 {
    float v[FV_TILE_MAXL];
    float d;
    int32_t row, next, pad;
    int32_t ds[FV_TILE_MAXL];
};
static_assert(sizeof(TileRec64) == 64 && sizeof(TileRec32) == 48, "tile record layout");
template <typename T>
using TileRec = typename std::conditional<sizeof(T) == 8, TileRec64, TileRec32>::type;

constexpr int kTileWarps = 4;  // warps per block
constexpr int kTileDepth = 6;  // steps in flight per warp

template <typename T>
constexpr size_t tile_smem() {
    return (size_t)kTileWarps * 32 * (kTileDepth * (sizeof(TileRec<T>) + sizeof(T)) + FV_TILE_RING * sizeof(T));
}

template <typename T>
__global__ void k_tile_records(int64_t nslots, const int32_t *__restrict__ slot_row,
                               const int32_t *__restrict__ slot_src, const int32_t *__restrict__ slot_ds,
                               const int32_t *__restrict__ slot_next, const T *__restrict__ val,
                               const T *__restrict__ dinv, TileRec<T> *__restrict__ rec) {
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < nslots; u += (int64_t)gridDim.x * blockDim.x) {
        TileRec<T> r;
        r.row = slot_row[u];
        r.next = slot_next[u];
#pragma unroll
        for (int q = 0; q < FV_TILE_MAXL; ++q) {
            const int32_t src = slot_src[u * FV_TILE_MAXL + q];
            r.v[q] = src >= 0 ? val[src] : T(0);
            r.ds[q] = slot_ds[u * FV_TILE_MAXL + q];
        }
        r.d = (dinv && r.row >= 0) ? dinv[r.row] : T(1);
        if constexpr (sizeof(T) == 4) r.pad = 0;
        rec[u] = r;
    }
}

template <typename T>
__global__ void k_tile_rhs(int64_t nslots, const int32_t *__restrict__ slot_row, const T *__restrict__ r,
                           T *__restrict__ out) {
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < nslots; u += (int64_t)gridDim.x * blockDim.x) {
        const int32_t row = slot_row[u];
        out[u] = row >= 0 ? r[row] : T(0);
    }
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(a), "l"(gmem) : "memory");
}
template <int BYTES>
__device__ __forceinline__ void cp_async_small(void *smem, const void *gmem) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(a), "l"(gmem), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// The reordered factorisation's sweeps (k_sweep_seq, 1, 2, 4 or 8 rows per
// thread); rows longer than 8 entries on the swept side fall back to the
// level-chunk kernels.
template <typename T, bool UNIT, bool REV>
static void launch_sweep_seq(int maxl, int rpt, int G, cudaStream_t st, int64_t n, const int32_t *order,
                             const int32_t *ptr, const int32_t *col, const T *val, const T *dinv, const T *rhs, T *x,
                             T *rhs_reset, T *next_reset, unsigned *ctrl, int *err, const int *skip, fv_row_skip rs,
                             SweepPerm<T> pm) {
    if (maxl > 8) {
        launch_sweep<T, UNIT>(maxl, G, st, n, order, ptr, col, val, dinv, rhs, x, rhs_reset, next_reset, ctrl, err,
                              skip, rs, false, pm);
        return;
    }
#define FV_SEQ(ML, R)                                                                                               \
    fv_note_launch(), k_sweep_seq<T, UNIT, ML, R, REV><<<G, 256, 0, st>>>(n, ptr, col, val, dinv, rhs, x, rhs_reset, \
                                                                          next_reset, ctrl, err, skip, rs, pm)
#define FV_SEQ_R(ML)          \
    if (rpt <= 1)             \
        FV_SEQ(ML, 1);        \
    else if (rpt <= 2)        \
        FV_SEQ(ML, 2);        \
    else if (rpt <= 4)        \
        FV_SEQ(ML, 4);        \
    else                      \
        FV_SEQ(ML, 8)
    if (maxl <= 4) {
        FV_SEQ_R(4);
    } else {
        FV_SEQ_R(8);
    }
#undef FV_SEQ_R
#undef FV_SEQ
}

template <typename T, bool UNIT>
__global__ void __launch_bounds__(kTileWarps * 32) k_sweep_tiled(int64_t nb, const int32_t *__restrict__ box_step,
                                                                 const TileRec<T> *__restrict__ rec,
                                                                 const T *__restrict__ rhs_slot, T *x, T *next_rhs,
                                                                 T *rhs_reset, T *next_reset, unsigned *ctrl,
                                                                 int *err, const int *skip, fv_row_skip rs) {
    using R = TileRec<T>;
    extern __shared__ __align__(16) unsigned char tile_smem_raw[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    R *recbuf = reinterpret_cast<R *>(tile_smem_raw) + (size_t)w * kTileDepth * 32;
    T *rhsbuf = reinterpret_cast<T *>(tile_smem_raw + (size_t)kTileWarps * kTileDepth * 32 * sizeof(R)) +
                (size_t)w * kTileDepth * 32;
    T *ring = reinterpret_cast<T *>(tile_smem_raw + (size_t)kTileWarps * kTileDepth * 32 * (sizeof(R) + sizeof(T))) +
              (size_t)w * FV_TILE_RING * 32;
    if (skip && *(volatile const int *)skip) return;
    int64_t b;
    while (take_chunk(&ctrl[0], nb, b)) {
        const int s0 = __ldg(&box_step[b]), s1 = __ldg(&box_step[b + 1]);
        // a box holds rows of one connected component: one problem of a batch
        if (rs.group) {
            const int row0 = rec[(int64_t)32 * s0].row;
            if (rs.done[(int64_t)__ldg(&rs.group[row0]) * rs.stride]) continue;
        }
        auto issue = [&](int step, int bi) {
            if (step < s1) {
                const int64_t u = (int64_t)32 * step + lane;
                const unsigned char *src = reinterpret_cast<const unsigned char *>(&rec[u]);
                unsigned char *dst = reinterpret_cast<unsigned char *>(&recbuf[bi * 32 + lane]);
#pragma unroll
                for (int c = 0; c < (int)(sizeof(R) / 16); ++c) cp_async16(dst + 16 * c, src + 16 * c);
                cp_async_small<sizeof(T)>(&rhsbuf[bi * 32 + lane], &rhs_slot[u]);
            }
            cp_async_commit();
        };
#pragma unroll
        for (int k = 0; k < kTileDepth; ++k) issue(s0 + k, k);
        for (int st = s0; st < s1; ++st) {
            cp_async_wait<kTileDepth - 1>();
            const int bi = (st - s0) % kTileDepth;
            const R r = recbuf[bi * 32 + lane];
            const T rh = rhsbuf[bi * 32 + lane];
            issue(st + kTileDepth, bi);
            if (r.row >= 0) {
                T xv[FV_TILE_MAXL];
                unsigned pending = 0;
#pragma unroll
                for (int q = 0; q < FV_TILE_MAXL; ++q) {
                    xv[q] = T(0);
                    if (r.ds[q] >= 0 && !fv_slot_ready(&x[r.ds[q]], xv[q])) pending |= 1u << q;
                }
                if (pending) {
                    const unsigned long long t0 = fv_globaltimer();
                    for (unsigned it = 1; pending; ++it) {
#pragma unroll
                        for (int q = 0; q < FV_TILE_MAXL; ++q)
                            if ((pending >> q) & 1u)
                                if (fv_slot_ready(&x[r.ds[q]], xv[q])) pending &= ~(1u << q);
                        if (pending && (it & 255u) == 0) {
                            if (*(volatile int *)err || fv_globaltimer() - t0 > FV_WAIT_LIMIT_NS) {
                                if (!*(volatile int *)err) atomicOr(err, FV_DEV_TIMEOUT);
#pragma unroll
                                for (int q = 0; q < FV_TILE_MAXL; ++q)
                                    if ((pending >> q) & 1u) xv[q] = T(NAN);
                                pending = 0;
                            }
                        }
                    }
                }
                T s = rh;
#pragma unroll
                for (int q = 0; q < FV_TILE_MAXL; ++q)
                    if (r.ds[q] != FV_TILE_PAD) s = s - r.v[q] * (r.ds[q] < 0 ? ring[-r.ds[q] - 1] : xv[q]);
                const T res = UNIT ? s : r.d * s;
                ring[((st - s0) % FV_TILE_RING) * 32 + lane] = res;
                fv_publish(&x[r.row], res);
                if (next_rhs) next_rhs[r.next] = res;
                if (rhs_reset) fv_reset_slot(&rhs_reset[r.row]);
                if (next_reset) fv_reset_slot(&next_reset[r.row]);
            }
            __syncwarp();
        }
    }
    cp_async_wait<0>();
    leave(&ctrl[0], &ctrl[1]);
}

template <typename T, bool UNIT>
static int tile_grid(int64_t nb) {
    static int per_sm = -1;
    if (per_sm < 0) {
        cudaFuncSetAttribute(k_sweep_tiled<T, UNIT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tile_smem<T>());
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep_tiled<T, UNIT>, kTileWarps * 32,
                                                          tile_smem<T>()) != cudaSuccess ||
            per_sm < 1)
            per_sm = 1;
    }
    return (int)std::max<int64_t>(1, std::min<int64_t>((nb + kTileWarps - 1) / kTileWarps, 148LL * per_sm));
}

static bool use_tiles(const fv_precond *P) {
    const fv_symbolic *s = P->sym;
    return P->schedule == 2 && s->tiled;
}

// Records of both directions for precision T, rebuilt when the factors changed.
template <typename T>
static fv_status tile_prepare(fv_precond *P, cudaStream_t st) {
    const fv_symbolic *s = P->sym;
    void **rec = sizeof(T) == 8 ? P->t_rec64 : P->t_rec32;
    T **rhs = reinterpret_cast<T **>(sizeof(T) == 8 ? (void **)P->t_rhs64 : (void **)P->t_rhs32);
    const unsigned version = sizeof(T) == 8 ? P->epoch : P->f32_version;
    unsigned &seen = sizeof(T) == 8 ? P->t_rec64_epoch : P->t_rec32_version;
    for (int d = 0; d < 2; ++d) {
        if (!rec[d]) {
            FV_CUDA_TRY(cudaMalloc(&rec[d], sizeof(TileRec<T>) * (s->t_nslots[d] ? s->t_nslots[d] : 1)));
            FV_CUDA_TRY(cudaMalloc(&rhs[d], sizeof(T) * (s->t_nslots[d] ? s->t_nslots[d] : 1)));
            seen = version - 1;
        }
    }
    if (seen != version) {
        const T *lv, *uv, *dv;
        if constexpr (sizeof(T) == 8) {
            lv = P->l_val;
            uv = P->u_val;
            dv = P->dinv;
        } else {
            lv = P->l32;
            uv = P->u32;
            dv = P->dinv32;
        }
        for (int d = 0; d < 2; ++d) {
            const int64_t ns = s->t_nslots[d];
            if (!ns) continue;
            const unsigned G = (unsigned)std::min<int64_t>((ns + 255) / 256, 148 * 16);
            const T *dinv = (d == 0 && P->kind == 2) ? nullptr : dv;  // ILU's forward sweep has a unit diagonal
            fv_note_launch(), k_tile_records<T><<<G, 256, 0, st>>>(ns, s->t_slot_row[d], s->t_slot_src[d],
                                                                   s->t_slot_ds[d], s->t_slot_next[d],
                                                                   d == 0 ? lv : uv, dinv,
                                                                   reinterpret_cast<TileRec<T> *>(rec[d]));
            FV_CUDA_TRY(cudaGetLastError());
        }
        seen = version;
    }
    return FV_OK;
}

// Both tiled sweeps: z = M^-1 r (same contract as the level-chunk sweeps).
template <typename T>
static fv_status tiled_apply(fv_precond *P, const T *r, T *z, T *tmp, cudaStream_t st, const int *skip,
                             const fv_row_skip &rs) {
    const fv_symbolic *s = P->sym;
    FV_TRY(tile_prepare<T>(P, st));
    void **rec = sizeof(T) == 8 ? P->t_rec64 : P->t_rec32;
    T **rhs = reinterpret_cast<T **>(sizeof(T) == 8 ? (void **)P->t_rhs64 : (void **)P->t_rhs32);
    const int64_t ns0 = s->t_nslots[0];
    if (ns0) {
        const unsigned G = (unsigned)std::min<int64_t>((ns0 + 255) / 256, 148 * 16);
        fv_note_launch(), k_tile_rhs<T><<<G, 256, 0, st>>>(ns0, s->t_slot_row[0], r, rhs[0]);
        FV_CUDA_TRY(cudaGetLastError());
    }
    const size_t smem = tile_smem<T>();
    if (P->kind == 2) {
        const int G = tile_grid<T, true>(s->t_nb[0]);
        fv_note_launch(), k_sweep_tiled<T, true><<<G, kTileWarps * 32, smem, st>>>(
                              s->t_nb[0], s->t_box_step[0], reinterpret_cast<const TileRec<T> *>(rec[0]), rhs[0], tmp,
                              rhs[1], nullptr, z, P->ctrl, P->err, skip, rs);
    } else {
        const int G = tile_grid<T, false>(s->t_nb[0]);
        fv_note_launch(), k_sweep_tiled<T, false><<<G, kTileWarps * 32, smem, st>>>(
                              s->t_nb[0], s->t_box_step[0], reinterpret_cast<const TileRec<T> *>(rec[0]), rhs[0], tmp,
                              rhs[1], nullptr, z, P->ctrl, P->err, skip, rs);
    }
    FV_CUDA_TRY(cudaGetLastError());
    const int G = tile_grid<T, false>(s->t_nb[1]);
    fv_note_launch(), k_sweep_tiled<T, false><<<G, kTileWarps * 32, smem, st>>>(
                          s->t_nb[1], s->t_box_step[1], reinterpret_cast<const TileRec<T> *>(rec[1]), rhs[1], z,
                          nullptr, tmp, nullptr, P->ctrl + 2, P->err, skip, rs);
    FV_CUDA_TRY(cudaGetLastError());
    return FV_OK;
}

static int sweep_grid(int64_t n);

// ------------------------------------------------------------------ symbolic on the device
// The same analysis as build_symbolic: strict lower / upper parts, the level
// of every row (longest dependency chain), rows ordered by level (ascending
// row within a level), and the transpose map of IC.  Levels come from a
// sync-free sweep in natural row order (reverse order for the upper part):
// a row's dependencies are lower (higher) rows, so they sit in earlier
// chunks or earlier lanes of the same chunk.
namespace {

enum : int { kSymUnsorted = 1, kSymNoDiag = 2, kSymRange = 4, kSymAsym = 8 };

__global__ void k_sym_count(int64_t n, const int32_t *__restrict__ ptr, const int32_t *__restrict__ col,
                            int32_t *__restrict__ cl, int32_t *__restrict__ cu, int *flags, int *maxes) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int nl = 0, nu = 0, len = 0, bad = 0;
    if (i < n) {
        bool diag = false;
        const int k0 = ptr[i], k1 = ptr[i + 1];
        len = k1 - k0;
        for (int k = k0; k < k1; ++k) {
            const int c = col[k];
            if (c < 0 || c >= n) bad |= kSymRange;
            if (k > k0 && c <= col[k - 1]) bad |= kSymUnsorted;
            if (c < i)
                ++nl;
            else if (c > i)
                ++nu;
            else
                diag = true;
        }
        if (!diag) bad |= kSymNoDiag;
        cl[i] = nl;
        cu[i] = nu;
    }
    const int ml = __reduce_max_sync(0xffffffffu, nl), mu = __reduce_max_sync(0xffffffffu, nu);
    const int mr = __reduce_max_sync(0xffffffffu, len), bo = __reduce_or_sync(0xffffffffu, bad);
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&maxes[0], ml);
        atomicMax(&maxes[1], mu);
        atomicMax(&maxes[2], mr);
        if (bo) atomicOr(flags, bo);
    }
}

__global__ void k_sym_split(int64_t n, const int32_t *__restrict__ ptr, const int32_t *__restrict__ col,
                            const int32_t *__restrict__ lp, const int32_t *__restrict__ up,
                            int32_t *__restrict__ lc, int32_t *__restrict__ uc) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int a = lp[i], b = up[i];
    for (int k = ptr[i]; k < ptr[i + 1]; ++k) {
        const int c = col[k];
        if (c < i) lc[a++] = c;
        if (c > i) uc[b++] = c;
    }
}

// level[i] = 1 + max level of the row's dependencies (0 without any); slots
// start at all-ones (no level yet).  Bounded waits as in the sweeps.
__global__ void __launch_bounds__(256) k_sym_levels(int64_t n, int upper, const int32_t *__restrict__ ptr,
                                                    const int32_t *__restrict__ col, int32_t *level,
                                                    unsigned *ctrl, int *err, int *nlev) {
    const int64_t nchunks = (n + 31) / 32;
    int64_t chunk;
    int top = -1;
    while (take_chunk(&ctrl[0], nchunks, chunk)) {
        const int64_t idx = chunk * 32 + (threadIdx.x & 31);
        if (idx >= n) continue;
        const int64_t i = upper ? n - 1 - idx : idx;
        int lev = 0;
        for (int k = __ldg(&ptr[i]); k < __ldg(&ptr[i + 1]); ++k) {
            const int32_t c = __ldg(&col[k]);
            unsigned v = fv_ld_relaxed_u32(&level[c]);
            if (v == 0xFFFFFFFFu) {
                const unsigned long long t0 = fv_globaltimer();
                for (unsigned it = 1; v == 0xFFFFFFFFu; ++it) {
                    v = fv_ld_relaxed_u32(&level[c]);
                    if (v == 0xFFFFFFFFu && (it & 255u) == 0 &&
                        (*(volatile int *)err || fv_globaltimer() - t0 > FV_WAIT_LIMIT_NS)) {
                        if (!*(volatile int *)err) atomicOr(err, FV_DEV_TIMEOUT);
                        v = 0;
                    }
                }
            }
            lev = max(lev, (int)v + 1);
        }
        asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(&level[i]), "r"((unsigned)lev) : "memory");
        top = max(top, lev);
    }
    top = __reduce_max_sync(0xffffffffu, top);
    if ((threadIdx.x & 31) == 0) atomicMax(nlev, top + 1);
    leave(&ctrl[0], &ctrl[1]);
}

__global__ void k_sym_iota(int64_t n, int32_t *__restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (int32_t)i;
}

// L entry (i, j) -> position of (j, i) among U's entries; a missing mirror
// entry marks the pattern unsymmetric.
__global__ void k_sym_tpos(int64_t n, const int32_t *__restrict__ lp, const int32_t *__restrict__ lc,
                           const int32_t *__restrict__ up, const int32_t *__restrict__ uc,
                           int32_t *__restrict__ tpos, int *flags) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int bad = 0;
    if (i < n) {
        for (int k = lp[i]; k < lp[i + 1]; ++k) {
            const int j = lc[k];
            int lo = up[j], hi = up[j + 1];
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (uc[mid] < i)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            if (lo < up[j + 1] && uc[lo] == i)
                tpos[k] = lo;
            else
                bad = kSymAsym;
        }
    }
    if (__reduce_or_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flags, kSymAsym);
}

}  // namespace

static fv_status build_symbolic_device(const fv_csr *A, cudaStream_t st, fv_symbolic **out) {
    const int64_t n = A->nrows;
    if (n <= 0 || n >= 0x7fffffffLL || A->nnz >= 0x7fffffffLL) return FV_ERR_INVALID;
    const unsigned G = (unsigned)((n + 255) / 256);
    fv_symbolic *s = new fv_symbolic();
    s->n = n;
    int *dw = nullptr;  // [0] flags [1..3] max lower / upper / row [4] err [5,6] levels fwd / bwd
    unsigned *ctrl = nullptr;
    int32_t *cnt = nullptr, *keys = nullptr, *iota = nullptr;
    void *tmp = nullptr;
    auto cleanup = [&]() {  // scratch from the stream-ordered pool: no device-wide synchronisation
        for (void *q : {(void *)dw, (void *)ctrl, (void *)cnt, (void *)keys, (void *)iota, tmp})
            if (q) cudaFreeAsync(q, st);
    };
    auto fail = [&](cudaError_t e, const char *what) {
        fv_internal_set_cuda_error(e, what);
        cleanup();
        fv_symbolic_free(s);
        return e == cudaErrorMemoryAllocation ? FV_ERR_ALLOC : FV_ERR_CUDA;
    };
    auto reject = [&](fv_status code) {
        cleanup();
        fv_symbolic_free(s);
        return code;
    };
    cudaError_t e = fv_malloc_async(&dw, sizeof(int) * 8, st);
    if (e == cudaSuccess) e = fv_malloc_async(&ctrl, sizeof(unsigned) * 4, st);
    if (e == cudaSuccess) e = fv_malloc_async(&cnt, sizeof(int32_t) * 2 * (n + 1), st);
    if (e == cudaSuccess) e = cudaMalloc(&s->l_ptr, sizeof(int32_t) * (n + 1));
    if (e == cudaSuccess) e = cudaMalloc(&s->u_ptr, sizeof(int32_t) * (n + 1));
    if (e == cudaSuccess) e = cudaMemsetAsync(dw, 0, sizeof(int) * 8, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(ctrl, 0, sizeof(unsigned) * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(cnt, 0, sizeof(int32_t) * 2 * (n + 1), st);
    if (e == cudaSuccess) {
        fv_note_launch();
        k_sym_count<<<G, 256, 0, st>>>(n, A->row_ptr, A->cols, cnt, cnt + (n + 1), dw, dw + 1);
        e = cudaGetLastError();
    }
    size_t tb = 0, tb2 = 0;
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, s->l_ptr, (int)(n + 1), st);
    if (e == cudaSuccess)
        e = cub::DeviceRadixSort::SortPairs(nullptr, tb2, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                            (const int32_t *)nullptr, (int32_t *)nullptr, (int)n, 0, 32, st);
    tb = std::max(tb, tb2);
    if (e == cudaSuccess) e = fv_malloc_async(&tmp, tb, st);
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp, tb, cnt, s->l_ptr, (int)(n + 1), st);
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp, tb, cnt + (n + 1), s->u_ptr, (int)(n + 1), st);
    int h[8] = {0};
    int32_t nl = 0, nu = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, dw, sizeof(int) * 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&nl, s->l_ptr + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&nu, s->u_ptr + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(e, "symbolic (counts)");
    if (h[0]) return reject(FV_ERR_INVALID);  // unsorted / duplicate columns, no diagonal (the reference panics)
    s->nnz_l = nl;
    s->nnz_u = nu;
    s->max_lower = h[1];
    s->max_upper = h[2];
    s->max_row = h[3];
    e = cudaMalloc(&s->l_col, sizeof(int32_t) * (nl ? nl : 1));
    if (e == cudaSuccess) e = cudaMalloc(&s->u_col, sizeof(int32_t) * (nu ? nu : 1));
    if (e == cudaSuccess) e = cudaMalloc(&s->d_fwd_level, sizeof(int32_t) * n);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_bwd_level, sizeof(int32_t) * n);
    if (e == cudaSuccess) e = cudaMalloc(&s->fwd_order, sizeof(int32_t) * n);
    if (e == cudaSuccess) e = cudaMalloc(&s->bwd_order, sizeof(int32_t) * n);
    if (e == cudaSuccess) e = fv_malloc_async(&keys, sizeof(int32_t) * n, st);
    if (e == cudaSuccess) e = fv_malloc_async(&iota, sizeof(int32_t) * n, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->d_fwd_level, 0xFF, sizeof(int32_t) * n, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->d_bwd_level, 0xFF, sizeof(int32_t) * n, st);
    if (e == cudaSuccess) {
        fv_note_launch();
        k_sym_split<<<G, 256, 0, st>>>(n, A->row_ptr, A->cols, s->l_ptr, s->u_ptr, s->l_col, s->u_col);
        fv_note_launch();
        k_sym_iota<<<G, 256, 0, st>>>(n, iota);
        const int SG = sweep_grid(n);
        fv_note_launch();
        k_sym_levels<<<SG, 256, 0, st>>>(n, 0, s->l_ptr, s->l_col, s->d_fwd_level, ctrl, dw + 4, dw + 5);
        fv_note_launch();
        k_sym_levels<<<SG, 256, 0, st>>>(n, 1, s->u_ptr, s->u_col, s->d_bwd_level, ctrl + 2, dw + 4, dw + 6);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, dw, sizeof(int) * 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(e, "symbolic (levels)");
    if (h[4]) {
        fv_internal_set_error_text("symbolic analysis: level sweep timed out");
        return reject(FV_ERR_TIMEOUT);
    }
    s->n_fwd_levels = h[5];
    s->n_bwd_levels = h[6];
    // rows by level, ascending row within a level (the radix sort is stable)
    for (int d = 0; d < 2 && e == cudaSuccess; ++d) {
        const int32_t nlev = d == 0 ? s->n_fwd_levels : s->n_bwd_levels;
        int bits = 1;
        while (bits < 31 && (1 << bits) < nlev) ++bits;
        size_t need = 0;
        e = cub::DeviceRadixSort::SortPairs(nullptr, need, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                            (const int32_t *)nullptr, (int32_t *)nullptr, (int)n, 0, bits, st);
        if (e == cudaSuccess && need > tb) {
            cudaFreeAsync(tmp, st);
            tmp = nullptr;
            tb = need;
            e = fv_malloc_async(&tmp, tb, st);
        }
        if (e != cudaSuccess) break;
        e = cub::DeviceRadixSort::SortPairs(tmp, tb, (const uint32_t *)(d == 0 ? s->d_fwd_level : s->d_bwd_level),
                                            (uint32_t *)keys, iota, d == 0 ? s->fwd_order : s->bwd_order, (int)n, 0,
                                            bits, st);
    }
    // transpose map (IC) when the pattern is structurally symmetric
    if (e == cudaSuccess && nl == nu) {
        e = cudaMalloc(&s->l_tpos, sizeof(int32_t) * (nl ? nl : 1));
        if (e == cudaSuccess) {
            fv_note_launch();
            k_sym_tpos<<<G, 256, 0, st>>>(n, s->l_ptr, s->l_col, s->u_ptr, s->u_col, s->l_tpos, dw);
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, dw, sizeof(int) * 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(e, "symbolic (orders)");
    s->symmetric_pattern = nl == nu && !(h[0] & kSymAsym);
    if (!s->symmetric_pattern) {
        cudaFree(s->l_tpos);
        s->l_tpos = nullptr;
    }
    cleanup();
    *out = s;
    return FV_OK;
}

static int sweep_grid(int64_t n) {
    int64_t warps = (n + 31) / 32;
    int64_t blocks = (warps + 7) / 8;
    // 296 blocks of 8 warps (2 per SM): enough chunks in flight to keep the
    // level frontier busy; more warps only add pollers that compete with it
    // for L2 (measured on a 12.6M-row ILU(0): 1.23 ms per apply at 296
    // blocks, 1.25 at 592, 1.29 at 1184)
    return (int)std::max<int64_t>(1, std::min<int64_t>(blocks, 148 * 2));
}

// DiagonalPreconditioner (preconditioners/mod.rs:38-68): dinv[i] = 1.0 / a_ii
// (Inverse for f64, linalg/mod.rs:48-52); z_i = dinv_i * r_i.  A row without its
// diagonal is an error (the reference indexes [[i, i]] and panics).
namespace {
__global__ void k_diag_inverse(int64_t n, const int32_t *__restrict__ ptr, const int32_t *__restrict__ col,
                               const double *__restrict__ val, double *__restrict__ dinv, int *err) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int lo = ptr[i], hi = ptr[i + 1];
    while (lo < hi) {  // columns ascending
        const int mid = (lo + hi) >> 1;
        if (col[mid] < i)
            lo = mid + 1;
        else
            hi = mid;
    }
    if (lo < ptr[i + 1] && col[lo] == i)
        dinv[i] = 1.0 / val[lo];
    else
        atomicOr(err, FV_DEV_SINGULAR);
}

template <typename T>
__global__ void k_diag_apply(int64_t n, const T *__restrict__ dinv, const T *__restrict__ r, T *__restrict__ z,
                             const int *skip, fv_row_skip rs) {
    if (skip && *(volatile const int *)skip) return;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (rs.group && rs.done[(int64_t)rs.group[i] * rs.stride]) continue;
        z[i] = dinv[i] * r[i];
    }
}

static fv_status diag_compute(fv_precond *P, cudaStream_t st) {
    const int64_t n = P->n;
    FV_CUDA_TRY(cudaMemsetAsync(P->err, 0, sizeof(int), st));
    fv_note_launch(), k_diag_inverse<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, P->A->row_ptr, P->A->cols,
                                                                                  P->A->vals, P->dinv, P->err);
    FV_CUDA_TRY(cudaGetLastError());
    int bad = 0;
    FV_CUDA_TRY(cudaMemcpyAsync(&bad, P->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    FV_CUDA_TRY(cudaStreamSynchronize(st));
    if (bad) {
        FV_CUDA_TRY(cudaMemsetAsync(P->err, 0, sizeof(int), st));
        fv_internal_set_error_text("DiagonalPreconditioner: a row without its diagonal entry");
        return FV_ERR_INVALID;
    }
    return FV_OK;
}

static int diag_grid(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 8)); }
}  // namespace

extern "C" fv_status fv_diag_factor(const fv_csr *A, void *stream, fv_precond **out) {
    if (!A || !out || A->nrows <= 0) return FV_ERR_INVALID;
    *out = nullptr;
    cudaStream_t st = fv_stream(stream);
    fv_precond *P = new fv_precond();
    P->kind = 3;
    P->n = A->nrows;
    P->A = A;
    cudaError_t e = cudaMalloc(&P->dinv, sizeof(double) * P->n);
    if (e == cudaSuccess) e = cudaMalloc(&P->err, sizeof(int));
    if (e != cudaSuccess) {
        fv_internal_set_cuda_error(e, "fv_diag_factor");
        fv_precond_destroy(P);
        return e == cudaErrorMemoryAllocation ? FV_ERR_ALLOC : FV_ERR_CUDA;
    }
    const fv_status s = diag_compute(P, st);
    if (s != FV_OK) {
        fv_precond_destroy(P);
        return s;
    }
    *out = P;
    return FV_OK;
}

// Rows per thread and blocks of the reordered sweeps unless set by
// fv_precond_set_grid: one row per thread and up to 8 blocks of 256 threads
// per SM (measured on the 12.6M-row ILU(0) apply: 0.47 ms at 1 row / 1184
// blocks, 0.51-0.52 at 2 rows, 0.75 at 4 rows, 1.28 at 8 rows: a block waits
// for its slowest row at every ticket, so short chunks keep more rows moving).
static int seq_rpt(const fv_precond *P) { return P->sweep_rpt > 0 ? P->sweep_rpt : 1; }
static int seq_grid(const fv_precond *P, int64_t n, int rpt) {
    if (P->sweep_blocks > 0) return P->sweep_blocks;
    const int64_t chunks = (n + 256LL * rpt - 1) / (256LL * rpt);
    return (int)std::max<int64_t>(1, std::min<int64_t>(chunks, 148 * 8));
}

// z = M^-1 r.  r must not alias z.  The forward sweep writes P->tmp and
// pre-fills z with the sentinel; the backward sweep consumes tmp (resetting it
// to the sentinel for the next apply) and writes z.
fv_status fv_precond_apply_dev(fv_precond *P, const double *r, double *z, cudaStream_t st, const int *skip,
                               const fv_row_skip *rskip) {
    const fv_symbolic *s = P->sym;
    const int64_t n = P->n;
    const fv_row_skip rs = rskip ? *rskip : fv_row_skip{};
    if (P->kind == 3) {
        fv_note_launch(), k_diag_apply<double><<<diag_grid(n), 256, 0, st>>>(n, P->dinv, r, z, skip, rs);
        FV_CUDA_TRY(cudaGetLastError());
        return FV_OK;
    }
    const int G = P->sweep_blocks > 0 ? P->sweep_blocks : sweep_grid(n);
    if (P->perm) {  // reordered factorisation: gather r, sweep in B's numbering, scatter z
        const bool pf = P->schedule == 3;
        SweepPerm<double> fwd, bwd;
        fwd.nat = bwd.nat = P->perm;
        fwd.gather = true;
        bwd.out = z;
        (void)pf;
        const int R = seq_rpt(P), Gs = seq_grid(P, n, R);
        if (P->kind == 2)
            launch_sweep_seq<double, true, false>(s->max_lower, R, Gs, st, n, s->fwd_order, s->l_ptr, s->l_col,
                                                  P->l_val, nullptr, r, P->tmp, nullptr, P->zint, P->ctrl, P->err,
                                                  skip, rs, fwd);
        else
            launch_sweep_seq<double, false, false>(s->max_lower, R, Gs, st, n, s->fwd_order, s->l_ptr, s->l_col,
                                                   P->l_val, P->dinv, r, P->tmp, nullptr, P->zint, P->ctrl, P->err,
                                                   skip, rs, fwd);
        FV_CUDA_TRY(cudaGetLastError());
        launch_sweep_seq<double, false, true>(s->max_upper, R, Gs, st, n, s->bwd_order, s->u_ptr, s->u_col, P->u_val,
                                              P->dinv, P->tmp, P->zint, P->tmp, nullptr, P->ctrl + 2, P->err, skip, rs,
                                              bwd);
        FV_CUDA_TRY(cudaGetLastError());
        return FV_OK;
    }
    if (P->schedule == 4) {  // rows in index order: consecutive chunks, block tickets
        const int R = seq_rpt(P), Gs = seq_grid(P, n, R);
        const SweepPerm<double> none;
        if (P->kind == 2)
            launch_sweep_seq<double, true, false>(s->max_lower, R, Gs, st, n, s->fwd_order, s->l_ptr, s->l_col,
                                                  P->l_val, nullptr, r, P->tmp, nullptr, z, P->ctrl, P->err, skip,
                                                  rs, none);
        else
            launch_sweep_seq<double, false, false>(s->max_lower, R, Gs, st, n, s->fwd_order, s->l_ptr, s->l_col,
                                                   P->l_val, P->dinv, r, P->tmp, nullptr, z, P->ctrl, P->err, skip,
                                                   rs, none);
        FV_CUDA_TRY(cudaGetLastError());
        launch_sweep_seq<double, false, true>(s->max_upper, R, Gs, st, n, s->bwd_order, s->u_ptr, s->u_col, P->u_val,
                                              P->dinv, P->tmp, z, P->tmp, nullptr, P->ctrl + 2, P->err, skip, rs,
                                              none);
        FV_CUDA_TRY(cudaGetLastError());
        return FV_OK;
    }
    if (use_tiles(P)) return tiled_apply<double>(P, r, z, P->tmp, st, skip, rs);
    const bool pf = P->schedule == 3;
    if (P->kind == 2)
        launch_sweep<double, true>(s->max_lower, G, st, n, s->fwd_order, s->l_ptr, s->l_col, P->l_val, nullptr, r,
                                   P->tmp, nullptr, z, P->ctrl, P->err, skip, rs, pf);
    else
        launch_sweep<double, false>(s->max_lower, G, st, n, s->fwd_order, s->l_ptr, s->l_col, P->l_val, P->dinv, r,
                                    P->tmp, nullptr, z, P->ctrl, P->err, skip, rs, pf);
    FV_CUDA_TRY(cudaGetLastError());
    launch_sweep<double, false>(s->max_upper, G, st, n, s->bwd_order, s->u_ptr, s->u_col, P->u_val, P->dinv, P->tmp,
                                z, P->tmp, nullptr, P->ctrl + 2, P->err, skip, rs, pf);
    FV_CUDA_TRY(cudaGetLastError());
    return FV_OK;
}

fv_status fv_precond_check_error(fv_precond *P, cudaStream_t st) {
    int e = 0;
    FV_CUDA_TRY(cudaMemcpyAsync(&e, P->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    FV_CUDA_TRY(cudaStreamSynchronize(st));
    if (e) {
        FV_CUDA_TRY(cudaMemsetAsync(P->err, 0, sizeof(int), st));
        if (e & FV_DEV_TIMEOUT) return FV_ERR_TIMEOUT;
        if (e & FV_DEV_SINGULAR) return FV_ERR_SINGULAR_PIVOT;
        return FV_ERR_BREAKDOWN;
    }
    return FV_OK;
}

int *fv_precond_err_ptr(fv_precond *P) { return P->err; }
int64_t fv_precond_rows(const fv_precond *P) { return P->n; }

namespace {
__global__ void k_to_f32(int64_t n, const double *__restrict__ a, float *__restrict__ b) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}
}  // namespace

// FP32 copies of the current factors (rounded from the FP64 factorisation).
fv_status fv_precond_make_f32(fv_precond *P, cudaStream_t st) {
    const fv_symbolic *s = P->sym;
    const int64_t n = P->n;
    if (P->kind == 3) {
        if (!P->dinv32) FV_CUDA_TRY(cudaMalloc(&P->dinv32, sizeof(float) * n));
        fv_note_launch(), k_to_f32<<<148 * 8, 256, 0, st>>>(n, P->dinv, P->dinv32);
        FV_CUDA_TRY(cudaGetLastError());
        P->f32_version += 1;
        return FV_OK;
    }
    if (!P->l32) {
        FV_CUDA_TRY(cudaMalloc(&P->l32, sizeof(float) * (s->nnz_l ? s->nnz_l : 1)));
        FV_CUDA_TRY(cudaMalloc(&P->u32, sizeof(float) * (s->nnz_u ? s->nnz_u : 1)));
        FV_CUDA_TRY(cudaMalloc(&P->dinv32, sizeof(float) * n));
        FV_CUDA_TRY(cudaMalloc(&P->tmp32, sizeof(float) * n));
        FV_CUDA_TRY(cudaMemsetAsync(P->tmp32, 0xFF, sizeof(float) * n, st));
        if (P->perm) {
            FV_CUDA_TRY(cudaMalloc(&P->zint32, sizeof(float) * n));
            FV_CUDA_TRY(cudaMemsetAsync(P->zint32, 0xFF, sizeof(float) * n, st));
        }
    }
    const int G = 148 * 8;
    if (s->nnz_l) fv_note_launch(), k_to_f32<<<G, 256, 0, st>>>(s->nnz_l, P->l_val, P->l32);
    if (s->nnz_u) fv_note_launch(), k_to_f32<<<G, 256, 0, st>>>(s->nnz_u, P->u_val, P->u32);
    fv_note_launch(), k_to_f32<<<G, 256, 0, st>>>(n, P->dinv, P->dinv32);
    FV_CUDA_TRY(cudaGetLastError());
    P->f32_version += 1;
    return FV_OK;
}

// z = M^-1 r in FP32 with the FP32 factor copies (fv_precond_make_f32 first).
fv_status fv_precond_apply_dev_f32(fv_precond *P, const float *r, float *z, cudaStream_t st, const int *skip,
                                   const fv_row_skip *rskip) {
    const fv_symbolic *s = P->sym;
    const int64_t n = P->n;
    const fv_row_skip rs = rskip ? *rskip : fv_row_skip{};
    if (P->kind == 3) {
        if (!P->dinv32) return FV_ERR_INVALID;
        fv_note_launch(), k_diag_apply<float><<<diag_grid(n), 256, 0, st>>>(n, P->dinv32, r, z, skip, rs);
        FV_CUDA_TRY(cudaGetLastError());
        return FV_OK;
    }
    if (!P->l32) return FV_ERR_INVALID;
    const int G = P->sweep_blocks > 0 ? P->sweep_blocks : sweep_grid(n);
    if (P->perm) {  // reordered factorisation: gather r, sweep in B's numbering, scatter z
        const bool pf = P->schedule == 3;
        SweepPerm<float> fwd, bwd;
        fwd.nat = bwd.nat = P->perm;
        fwd.gather = true;
        bwd.out = z;
        (void)pf;
        const int R = seq_rpt(P), Gs = seq_grid(P, n, R);
        if (P->kind == 2)
            launch_sweep_seq<float, true, false>(s->max_lower, R, Gs, st, n, s->fwd_order, s->l_ptr, s->l_col,
                                                 P->l32, nullptr, r, P->tmp32, nullptr, P->zint32, P->ctrl, P->err,
                                                 skip, rs, fwd);
        else
            launch_sweep_seq<float, false, false>(s->max_lower, R, Gs, st, n, s->fwd_order, s->l_ptr, s->l_col,
                                                  P->l32, P->dinv32, r, P->tmp32, nullptr, P->zint32, P->ctrl,
                                                  P->err, skip, rs, fwd);
        FV_CUDA_TRY(cudaGetLastError());
        launch_sweep_seq<float, false, true>(s->max_upper, R, Gs, st, n, s->bwd_order, s->u_ptr, s->u_col, P->u32,
                                             P->dinv32, P->tmp32, P->zint32, P->tmp32, nullptr, P->ctrl + 2, P->err,
                                             skip, rs, bwd);
        FV_CUDA_TRY(cudaGetLastError());
        return FV_OK;
    }
    if (P->schedule == 4) {  // rows in index order: consecutive chunks, block tickets
        const int R = seq_rpt(P), Gs = seq_grid(P, n, R);
        const SweepPerm<float> none;
        if (P->kind == 2)
            launch_sweep_seq<float, true, false>(s->max_lower, R, Gs, st, n, s->fwd_order, s->l_ptr, s->l_col,
                                                 P->l32, nullptr, r, P->tmp32, nullptr, z, P->ctrl, P->err, skip, rs,
                                                 none);
        else
            launch_sweep_seq<float, false, false>(s->max_lower, R, Gs, st, n, s->fwd_order, s->l_ptr, s->l_col,
                                                  P->l32, P->dinv32, r, P->tmp32, nullptr, z, P->ctrl, P->err, skip,
                                                  rs, none);
        FV_CUDA_TRY(cudaGetLastError());
        launch_sweep_seq<float, false, true>(s->max_upper, R, Gs, st, n, s->bwd_order, s->u_ptr, s->u_col, P->u32,
                                             P->dinv32, P->tmp32, z, P->tmp32, nullptr, P->ctrl + 2, P->err, skip, rs,
                                             none);
        FV_CUDA_TRY(cudaGetLastError());
        return FV_OK;
    }
    if (use_tiles(P)) return tiled_apply<float>(P, r, z, P->tmp32, st, skip, rs);
    const bool pf = P->schedule == 3;
    if (P->kind == 2)
        launch_sweep<float, true>(s->max_lower, G, st, n, s->fwd_order, s->l_ptr, s->l_col, P->l32, nullptr, r,
                                  P->tmp32, nullptr, z, P->ctrl, P->err, skip, rs, pf);
    else
        launch_sweep<float, false>(s->max_lower, G, st, n, s->fwd_order, s->l_ptr, s->l_col, P->l32, P->dinv32, r,
                                   P->tmp32, nullptr, z, P->ctrl, P->err, skip, rs, pf);
    FV_CUDA_TRY(cudaGetLastError());
    launch_sweep<float, false>(s->max_upper, G, st, n, s->bwd_order, s->u_ptr, s->u_col, P->u32, P->dinv32,
                               P->tmp32, z, P->tmp32, nullptr, P->ctrl + 2, P->err, skip, rs, pf);
    FV_CUDA_TRY(cudaGetLastError());
    return FV_OK;
}

extern "C" fv_status fv_precond_schedule(fv_precond *P, int32_t request, int32_t *active, double *stats) {
    if (!P || request < -1 || request > 4) return FV_ERR_INVALID;
    if (P->kind == 3) {  // no sweeps to schedule
        if (active) *active = 1;
        if (stats) std::fill(stats, stats + 6, 0.0);
        return FV_OK;
    }
    fv_symbolic *s = P->sym;
    if (request == 2) FV_TRY(build_tiles(s, P->A, fv_stream(nullptr)));
    if (request == 2 && !s->tiled) return FV_ERR_UNSUPPORTED;
    if (request == 4 && (P->perm || P->fill)) return FV_ERR_UNSUPPORTED;
    if (request >= 0) P->schedule = request <= 1 ? 1 : request;
    if (active) *active = use_tiles(P) ? 2 : (P->schedule == 3 || P->schedule == 4 ? P->schedule : 1);
    if (stats) {
        stats[0] = s->t_edge;
        stats[1] = s->t_nb[0];
        stats[2] = s->t_lane_use[0];
        stats[3] = s->t_lane_use[1];
        stats[4] = s->t_ring_share[0];
        stats[5] = s->t_ring_share[1];
    }
    return FV_OK;
}

extern "C" fv_status fv_precond_destroy(fv_precond *P) {
    if (!P) return FV_OK;
    cudaFree(P->l_val);
    cudaFree(P->u_val);
    cudaFree(P->diag);
    cudaFree(P->dinv);
    cudaFree(P->tmp);
    cudaFree(P->done);
    cudaFree(P->ctrl);
    cudaFree(P->err);
    cudaFree(P->l32);
    cudaFree(P->u32);
    cudaFree(P->dinv32);
    cudaFree(P->tmp32);
    cudaFree(P->amap);
    cudaFree(P->perm);
    cudaFree(P->zint);
    cudaFree(P->zint32);
    for (int d = 0; d < 2; ++d) {
        cudaFree(P->t_rec64[d]);
        cudaFree(P->t_rec32[d]);
        cudaFree(P->t_rhs64[d]);
        cudaFree(P->t_rhs32[d]);
    }
    fv_csr *F = P->fill;
    delete P;
    if (F) fv_csr_destroy(F);
    return FV_OK;
}

static fv_status precond_alloc(fv_precond *P, cudaStream_t st) {
    const int64_t n = P->n;
    FV_CUDA_TRY(cudaMalloc(&P->l_val, sizeof(double) * (P->sym->nnz_l ? P->sym->nnz_l : 1)));
    FV_CUDA_TRY(cudaMalloc(&P->u_val, sizeof(double) * (P->sym->nnz_u ? P->sym->nnz_u : 1)));
    FV_CUDA_TRY(cudaMalloc(&P->diag, sizeof(double) * n));
    FV_CUDA_TRY(cudaMalloc(&P->dinv, sizeof(double) * n));
    FV_CUDA_TRY(cudaMalloc(&P->tmp, sizeof(double) * n));
    FV_CUDA_TRY(cudaMalloc(&P->done, sizeof(unsigned) * n));
    FV_CUDA_TRY(cudaMalloc(&P->ctrl, sizeof(unsigned) * 8));
    FV_CUDA_TRY(cudaMalloc(&P->err, sizeof(int)));
    FV_CUDA_TRY(cudaMemsetAsync(P->tmp, 0xFF, sizeof(double) * n, st));
    FV_CUDA_TRY(cudaMemsetAsync(P->done, 0, sizeof(unsigned) * n, st));
    FV_CUDA_TRY(cudaMemsetAsync(P->ctrl, 0, sizeof(unsigned) * 8, st));
    FV_CUDA_TRY(cudaMemsetAsync(P->err, 0, sizeof(int), st));
    return FV_OK;
}

namespace {
__global__ void k_order_not_identity(int64_t n, const int32_t *__restrict__ order, int *flag) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (order[i] != (int32_t)i) *flag = 1;
}
}  // namespace

static fv_status factor_common(const fv_csr *Ac, int kind, cudaStream_t st, fv_precond **out) {
    if (!Ac || !out) return FV_ERR_INVALID;
    if (Ac->nrows != Ac->ncols) return FV_ERR_INVALID;
    fv_csr *A = const_cast<fv_csr *>(Ac);
    fv_symbolic *sym = nullptr;
    FV_TRY(fv_get_symbolic(A, st, &sym));
    if (sym->max_row > 32) return FV_ERR_UNSUPPORTED;
    if (kind == 1 && !sym->symmetric_pattern) return FV_ERR_NOT_SYMMETRIC;
    fv_precond *P = *out;
    const bool fresh = (P == nullptr);
    if (fresh) {
        P = new fv_precond();
        P->kind = kind;
        P->n = A->nrows;
        P->A = A;
        P->sym = sym;
        fv_status s = precond_alloc(P, st);
        if (s != FV_OK) {
            fv_precond_destroy(P);
            return s;
        }
        // rows already sorted by forward level (a matrix permuted by a level-sorted
        // order): the sweeps take consecutive rows (schedule 4), no order array
        if (A->fill_mask.empty() && sym->max_lower <= 8 && sym->max_upper <= 8) {
            int notid = 0;
            FV_CUDA_TRY(cudaMemsetAsync(P->err, 0, sizeof(int), st));
            fv_note_launch(), k_order_not_identity<<<(unsigned)std::min<int64_t>((A->nrows + 255) / 256, 148 * 8), 256,
                                                     0, st>>>(A->nrows, sym->fwd_order, P->err);
            FV_CUDA_TRY(cudaGetLastError());
            FV_CUDA_TRY(cudaMemcpyAsync(&notid, P->err, sizeof(int), cudaMemcpyDeviceToHost, st));
            FV_CUDA_TRY(cudaMemsetAsync(P->err, 0, sizeof(int), st));
            FV_CUDA_TRY(cudaStreamSynchronize(st));
            if (!notid) P->schedule = 4;
            P->contiguous = !notid;
        }
    } else if (P->A != A || P->kind != kind) {
        return FV_ERR_INVALID;
    }
    const int64_t n = P->n;
    if (kind == 1 && A->fill_mask.empty()) {  // a fill pattern: checked on the matrix it came from
        FV_CUDA_TRY(cudaMemsetAsync(P->err, 0, sizeof(int), st));
        fv_note_launch(), k_check_symmetric<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, A->row_ptr, A->vals, sym->l_ptr, sym->l_col,
                                                                      sym->u_ptr, sym->l_tpos, P->err);
        FV_CUDA_TRY(cudaGetLastError());
        int bad = 0;
        FV_CUDA_TRY(cudaMemcpyAsync(&bad, P->err, sizeof(int), cudaMemcpyDeviceToHost, st));
        FV_CUDA_TRY(cudaStreamSynchronize(st));
        if (bad) {
            FV_CUDA_TRY(cudaMemsetAsync(P->err, 0, sizeof(int), st));
            if (fresh) fv_precond_destroy(P);
            return FV_ERR_NOT_SYMMETRIC;
        }
    }
    P->epoch += 1;
    if (P->epoch == 0) {  // wrapped: clear the flags
        FV_CUDA_TRY(cudaMemsetAsync(P->done, 0, sizeof(unsigned) * n, st));
        P->epoch = 1;
    }
    const int G = sweep_grid(n) * 2;  // 128-thread blocks
    const int mr = sym->max_row;
    if (kind == 2) {
#define FV_ILU(MR)                                                                                          \
    fv_note_launch(), k_ilu0<MR><<<G, 128, 0, st>>>(n, sym->fwd_order, A->row_ptr, A->vals, sym->l_ptr, sym->l_col, sym->u_ptr, \
                                  sym->u_col, P->l_val, P->u_val, P->diag, P->dinv, P->done, P->epoch,        \
                                  P->ctrl + 4, P->err)
        if (mr <= 6)
            fv_note_launch(), k_ilu0s<6><<<G, 128, 0, st>>>(n, sym->fwd_order, A->row_ptr, A->vals, sym->l_ptr,
                                                             sym->l_col, sym->u_ptr, sym->u_col, P->l_val, P->u_val,
                                                             P->diag, P->dinv, P->done, P->epoch, P->ctrl + 4, P->err);
        else if (mr <= 8)
            FV_ILU(8);
        else if (mr <= 16)
            FV_ILU(16);
        else
            FV_ILU(32);
#undef FV_ILU
    } else {
#define FV_IC(MR)                                                                                             \
    fv_note_launch(), k_ic0<MR><<<G, 128, 0, st>>>(n, sym->fwd_order, A->row_ptr, A->vals, sym->l_ptr, sym->l_col, sym->l_tpos, \
                                 P->l_val, P->u_val, P->diag, P->dinv, P->done, P->epoch, P->ctrl + 4, P->err)
        if (mr <= 6)
            fv_note_launch(), k_ic0s<6><<<G, 128, 0, st>>>(n, sym->fwd_order, A->row_ptr, A->vals, sym->l_ptr,
                                                            sym->l_col, sym->l_tpos, P->l_val, P->u_val, P->diag,
                                                            P->dinv, P->done, P->epoch, P->ctrl + 4, P->err);
        else if (mr <= 8)
            FV_IC(8);
        else if (mr <= 16)
            FV_IC(16);
        else
            FV_IC(32);
#undef FV_IC
    }
    FV_CUDA_TRY(cudaGetLastError());
    fv_status es = fv_precond_check_error(P, st);
    if (es != FV_OK) {
        if (fresh) fv_precond_destroy(P);
        return es;
    }
    if (kind == 2) {
        unsigned long long *cnt = nullptr;
        FV_CUDA_TRY(fv_malloc_async(&cnt, sizeof(unsigned long long), st));
        FV_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), st));
        fv_note_launch(), k_count_dropped<<<592, 256, 0, st>>>(sym->nnz_l, P->l_val, sym->nnz_u, P->u_val, cnt);
        unsigned long long h = 0;
        FV_CUDA_TRY(cudaMemcpyAsync(&h, cnt, sizeof(h), cudaMemcpyDeviceToHost, st));
        FV_CUDA_TRY(cudaFreeAsync(cnt, st));
        FV_CUDA_TRY(cudaStreamSynchronize(st));
        P->n_dropped = (int64_t)h;
    }
    *out = P;
    return FV_OK;
}

namespace {
__global__ void k_scatter_vals(int64_t nnz, const int32_t *__restrict__ amap, const double *__restrict__ a,
                               double *__restrict__ f) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x)
        f[amap[k]] = a[k];
}
}  // namespace

// is_symmetric (dmatrix.rs:76-88) of a matrix, as IncompleteCholesky::build asserts it
static fv_status check_symmetric(fv_csr *A, cudaStream_t st) {
    fv_symbolic *sym = nullptr;
    FV_TRY(fv_get_symbolic(A, st, &sym));
    if (!sym->symmetric_pattern) return FV_ERR_NOT_SYMMETRIC;
    int *bad = nullptr;
    FV_CUDA_TRY(fv_malloc_async(&bad, sizeof(int), st));
    FV_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(int), st));
    const int64_t n = A->nrows;
    fv_note_launch(), k_check_symmetric<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(
                          n, A->row_ptr, A->vals, sym->l_ptr, sym->l_col, sym->u_ptr, sym->l_tpos, bad);
    FV_CUDA_TRY(cudaGetLastError());
    int h = 0;
    FV_CUDA_TRY(cudaMemcpyAsync(&h, bad, sizeof(int), cudaMemcpyDeviceToHost, st));
    FV_CUDA_TRY(cudaFreeAsync(bad, st));
    FV_CUDA_TRY(cudaStreamSynchronize(st));
    return h ? FV_ERR_NOT_SYMMETRIC : FV_OK;
}

// Scatter the values of P->orig into the fill pattern.
static fv_status scatter_fill(fv_precond *P, cudaStream_t st) {
    fv_csr *F = P->fill;
    FV_CUDA_TRY(cudaMemsetAsync(F->vals, 0, sizeof(double) * (F->nnz ? F->nnz : 1), st));
    if (P->orig->nnz) {
        fv_note_launch(), k_scatter_vals<<<592, 256, 0, st>>>(P->orig->nnz, P->amap, P->orig->vals, F->vals);
        FV_CUDA_TRY(cudaGetLastError());
    }
    return FV_OK;
}

// IC(k) / ILU(k) with fill (k >= 1; IC(1) has the pattern of A, see fv_ic_factor).
static fv_status fill_factor(const fv_csr *Ac, int kind, int level, cudaStream_t st, fv_precond **out) {
    fv_csr *A = const_cast<fv_csr *>(Ac);
    if (A->nrows != A->ncols) return FV_ERR_INVALID;
    if (kind == 1) FV_TRY(check_symmetric(A, st));
    const int64_t n = A->nrows, nnz = A->nnz;
    std::vector<int32_t> ptr, col, fptr, fcol, amap;
    std::vector<uint8_t> fill;
    try {
        ptr.resize((size_t)n + 1);
        col.resize((size_t)(nnz ? nnz : 1));
    } catch (const std::bad_alloc &) {
        return FV_ERR_ALLOC;
    }
    FV_CUDA_TRY(cudaMemcpyAsync(ptr.data(), A->row_ptr, sizeof(int32_t) * (n + 1), cudaMemcpyDeviceToHost, st));
    if (nnz) FV_CUDA_TRY(cudaMemcpyAsync(col.data(), A->cols, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost, st));
    FV_CUDA_TRY(cudaStreamSynchronize(st));
    FV_TRY(fv_fill_pattern(kind, level, n, ptr.data(), col.data(), fptr, fcol, amap, fill));
    fv_csr *F = new (std::nothrow) fv_csr();
    if (!F) return FV_ERR_ALLOC;
    F->nrows = F->ncols = n;
    F->nnz = (int64_t)fcol.size();
    if (kind == 1) F->fill_mask = std::move(fill);
    int32_t *damap = nullptr;
    cudaError_t e = cudaMalloc(&F->row_ptr, sizeof(int32_t) * (n + 1));
    if (e == cudaSuccess) e = cudaMalloc(&F->cols, sizeof(int32_t) * (F->nnz ? F->nnz : 1));
    if (e == cudaSuccess) e = cudaMalloc(&F->vals, sizeof(double) * (F->nnz ? F->nnz : 1));
    if (e == cudaSuccess) e = cudaMalloc(&damap, sizeof(int32_t) * (nnz ? nnz : 1));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(F->row_ptr, fptr.data(), sizeof(int32_t) * (n + 1), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && F->nnz)
        e = cudaMemcpyAsync(F->cols, fcol.data(), sizeof(int32_t) * F->nnz, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && nnz)
        e = cudaMemcpyAsync(damap, amap.data(), sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        fv_internal_set_cuda_error(e, "fill pattern upload");
        cudaFree(damap);
        fv_csr_destroy(F);
        return e == cudaErrorMemoryAllocation ? FV_ERR_ALLOC : FV_ERR_CUDA;
    }
    fv_precond tmp;  // scatter through a stand-in so the values are in place before factorising
    tmp.fill = F;
    tmp.orig = A;
    tmp.amap = damap;
    fv_status s = scatter_fill(&tmp, st);
    tmp.fill = nullptr;
    tmp.amap = nullptr;
    fv_precond *P = nullptr;
    if (s == FV_OK) s = factor_common(F, kind, st, &P);
    if (s == FV_OK) P->schedule = 1;  // fill patterns keep the level chunks
    if (s != FV_OK) {
        cudaFree(damap);
        fv_csr_destroy(F);
        return s;
    }
    P->fill = F;
    P->orig = A;
    P->amap = damap;
    P->level = level;
    *out = P;
    return FV_OK;
}

/* IncompleteCholesky::from_matrix(A, level).  The reference's IC pattern of
 * row i is A's row plus every node the walk of row_i_sparsity_edit pushes,
 * i.e. the nodes within `level - 1` neighbour steps of A's neighbours; for
 * level 1 that is A's own pattern, so IC(1) is IC(0). */
extern "C" fv_status fv_ic_factor(const fv_csr *A, int32_t level, void *stream, fv_precond **out) {
    if (!out || !A || level < 0) return FV_ERR_INVALID;
    *out = nullptr;
    if (level <= 1) return factor_common(A, 1, fv_stream(stream), out);
    return fill_factor(A, 1, level, fv_stream(stream), out);
}
/* IncompleteLowerUpper::from_matrix(A, level): the factor pattern of
 * row_i_l_sparsity / row_i_u_sparsity, then the row-by-row IKJ elimination
 * with the drop rule of level 0 on that pattern. */
extern "C" fv_status fv_ilu_factor(const fv_csr *A, int32_t level, void *stream, fv_precond **out) {
    if (!out || !A || level < 0) return FV_ERR_INVALID;
    *out = nullptr;
    if (level == 0) return factor_common(A, 2, fv_stream(stream), out);
    return fill_factor(A, 2, level, fv_stream(stream), out);
}

extern "C" fv_status fv_ic0_factor(const fv_csr *A, void *stream, fv_precond **out) {
    if (!out) return FV_ERR_INVALID;
    *out = nullptr;
    return factor_common(A, 1, fv_stream(stream), out);
}
extern "C" fv_status fv_ilu0_factor(const fv_csr *A, void *stream, fv_precond **out) {
    if (!out) return FV_ERR_INVALID;
    *out = nullptr;
    return factor_common(A, 2, fv_stream(stream), out);
}
// ------------------------------------------------------------------ reordered factorisation
// IC(0) / ILU(0) of B = Q A Q^T (row i of B is row perm[i] of A, columns
// renumbered the same way and sorted), applied in A's numbering:
// z = Q^T M_B^{-1} Q r.  B lives in P->fill with amap[k] = the position in B
// of A's entry k, so refactorisation is the fill path's scatter.
namespace {
__global__ void k_perm_inverse(int64_t n, const int32_t *__restrict__ perm, int32_t *__restrict__ iperm,
                               int *__restrict__ bad) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t p = perm[i];
        if (p < 0 || p >= n) {
            atomicOr(bad, 1);
            continue;
        }
        if (atomicExch(&iperm[p], (int32_t)i) != -1) atomicOr(bad, 1);  // p listed twice
    }
}
__global__ void k_perm_rowlen(int64_t n, const int32_t *__restrict__ perm, const int32_t *__restrict__ aptr,
                              int32_t *__restrict__ len) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += (int64_t)gridDim.x * blockDim.x)
        len[i] = i < n ? aptr[perm[i] + 1] - aptr[perm[i]] : 0;
}
// rows of at most 32 entries (factor_common's limit)
__global__ void k_perm_rows(int64_t n, const int32_t *__restrict__ perm, const int32_t *__restrict__ iperm,
                            const int32_t *__restrict__ aptr, const int32_t *__restrict__ acol,
                            const int32_t *__restrict__ bptr, int32_t *__restrict__ bcol, int32_t *__restrict__ amap,
                            int *__restrict__ bad) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t old = perm[i];
        const int32_t k0 = aptr[old], m = aptr[old + 1] - k0, b0 = bptr[i];
        if (m > 32) {
            atomicOr(bad, 2);
            continue;
        }
        int32_t c[32], src[32];
        for (int t = 0; t < m; ++t) {  // insertion sort by the new column
            const int32_t ct = iperm[acol[k0 + t]];
            int q = t;
            while (q > 0 && c[q - 1] > ct) {
                c[q] = c[q - 1];
                src[q] = src[q - 1];
                --q;
            }
            c[q] = ct;
            src[q] = k0 + t;
        }
        for (int t = 0; t < m; ++t) {
            bcol[b0 + t] = c[t];
            amap[src[t]] = b0 + t;
        }
    }
}
}  // namespace

// B = Q A Q^T (B's row i is A's row perm[i], columns renumbered and sorted):
// its pattern, the permutation on the device and amap (A's entry k sits at
// B's entry amap[k]); B's values are not filled.
static fv_status build_permuted(fv_csr *A, const int32_t *perm_host, cudaStream_t st, fv_csr **Bout,
                                int32_t **perm_out, int32_t **amap_out) {
    if (!A || !perm_host || A->nrows != A->ncols || A->nrows <= 0) return FV_ERR_INVALID;
    const int64_t n = A->nrows, nnz = A->nnz;
    fv_csr *B = new (std::nothrow) fv_csr();
    if (!B) return FV_ERR_ALLOC;
    B->nrows = B->ncols = n;
    B->nnz = nnz;
    int32_t *perm = nullptr, *iperm = nullptr, *len = nullptr, *amap = nullptr;
    int *bad = nullptr;
    void *scan_tmp = nullptr;
    size_t scan_bytes = 0;
    int hbad = 0;
    cudaError_t e = cudaMalloc(&perm, sizeof(int32_t) * n);
    if (e == cudaSuccess) e = cudaMalloc(&B->row_ptr, sizeof(int32_t) * (n + 1));
    if (e == cudaSuccess) e = cudaMalloc(&B->cols, sizeof(int32_t) * (nnz ? nnz : 1));
    if (e == cudaSuccess) e = cudaMalloc(&B->vals, sizeof(double) * (nnz ? nnz : 1));
    if (e == cudaSuccess) e = cudaMalloc(&amap, sizeof(int32_t) * (nnz ? nnz : 1));
    if (e == cudaSuccess) e = fv_malloc_async(&iperm, sizeof(int32_t) * n, st);
    if (e == cudaSuccess) e = fv_malloc_async(&len, sizeof(int32_t) * (n + 1), st);
    if (e == cudaSuccess) e = fv_malloc_async(&bad, sizeof(int), st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(perm, perm_host, sizeof(int32_t) * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(iperm, 0xFF, sizeof(int32_t) * n, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(bad, 0, sizeof(int), st);
    const int G = (int)std::max<int64_t>(1, std::min<int64_t>((n + 256) / 256, 148 * 8));
    if (e == cudaSuccess) {
        fv_note_launch(), k_perm_inverse<<<G, 256, 0, st>>>(n, perm, iperm, bad);
        fv_note_launch(), k_perm_rowlen<<<G, 256, 0, st>>>(n, perm, A->row_ptr, len);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, len, B->row_ptr, n + 1, st);
    if (e == cudaSuccess) e = fv_malloc_async(&scan_tmp, scan_bytes ? scan_bytes : 1, st);
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, len, B->row_ptr, n + 1, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess && !hbad) {  // columns only once perm is known to be a permutation
        fv_note_launch(), k_perm_rows<<<G, 256, 0, st>>>(n, perm, iperm, A->row_ptr, A->cols, B->row_ptr, B->cols,
                                                        amap, bad);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (iperm) cudaFreeAsync(iperm, st);
    if (len) cudaFreeAsync(len, st);
    if (bad) cudaFreeAsync(bad, st);
    if (scan_tmp) cudaFreeAsync(scan_tmp, st);
    if (e != cudaSuccess || hbad) {
        if (e != cudaSuccess) fv_internal_set_cuda_error(e, "matrix permutation");
        if (hbad & 1) fv_internal_set_error_text("perm is not a permutation of 0..n-1");
        if (hbad & 2) fv_internal_set_error_text("a row has more than 32 entries");
        cudaFree(perm);
        cudaFree(amap);
        fv_csr_destroy(B);
        if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? FV_ERR_ALLOC : FV_ERR_CUDA;
        return (hbad & 2) ? FV_ERR_UNSUPPORTED : FV_ERR_INVALID;
    }
    *Bout = B;
    *perm_out = perm;
    *amap_out = amap;
    return FV_OK;
}

static fv_status perm_factor_impl(const fv_csr *Ac, const int32_t *perm_host, int kind, cudaStream_t st,
                                  fv_precond **out) {
    fv_csr *A = const_cast<fv_csr *>(Ac);
    if (!A || !perm_host || !out || A->nrows != A->ncols || A->nrows <= 0) return FV_ERR_INVALID;
    const int64_t n = A->nrows;
    fv_csr *B = nullptr;
    int32_t *perm = nullptr, *amap = nullptr;
    FV_TRY(build_permuted(A, perm_host, st, &B, &perm, &amap));
    cudaError_t e = cudaSuccess;
    fv_precond tmp;  // scatter through a stand-in so the values are in place before factorising
    tmp.fill = B;
    tmp.orig = A;
    tmp.amap = amap;
    fv_status s = scatter_fill(&tmp, st);
    tmp.fill = nullptr;
    tmp.amap = nullptr;
    fv_precond *P = nullptr;
    if (s == FV_OK) s = factor_common(B, kind, st, &P);
    if (s == FV_OK) P->schedule = 1;  // the reordered sweeps have their own kernels (P->perm)
    if (s == FV_OK) {
        e = cudaMalloc(&P->zint, sizeof(double) * n);
        if (e == cudaSuccess) e = cudaMemsetAsync(P->zint, 0xFF, sizeof(double) * n, st);
        if (e != cudaSuccess) {
            fv_internal_set_cuda_error(e, "reordered factorisation");
            fv_precond_destroy(P);
            P = nullptr;
            s = e == cudaErrorMemoryAllocation ? FV_ERR_ALLOC : FV_ERR_CUDA;
        }
    }
    if (s != FV_OK) {
        cudaFree(perm);
        cudaFree(amap);
        fv_csr_destroy(B);
        return s;
    }
    P->fill = B;
    P->orig = A;
    P->amap = amap;
    P->perm = perm;
    *out = P;
    return FV_OK;
}

namespace {
// y[i] = x[perm[i]] (to the permuted numbering) or y[perm[i]] = x[i] (back)
__global__ void k_vec_permute(int64_t n, const int32_t *__restrict__ perm, const double *__restrict__ x,
                              double *__restrict__ y, int back) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (back)
            y[perm[i]] = x[i];
        else
            y[i] = x[perm[i]];
    }
}
}  // namespace

static fv_status csr_permute_impl(const fv_csr *Ac, const int32_t *perm_host, cudaStream_t st, fv_csr **out) {
    fv_csr *A = const_cast<fv_csr *>(Ac);
    if (!A || !out || A->perm_src) return FV_ERR_INVALID;
    fv_csr *B = nullptr;
    int32_t *perm = nullptr, *amap = nullptr;
    FV_TRY(build_permuted(A, perm_host, st, &B, &perm, &amap));
    B->perm_src = A;
    B->perm = perm;
    B->perm_amap = amap;
    if (A->nnz) fv_note_launch(), k_scatter_vals<<<592, 256, 0, st>>>(A->nnz, amap, A->vals, B->vals);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        fv_internal_set_cuda_error(e, "fv_csr_permute");
        fv_csr_destroy(B);
        return FV_ERR_CUDA;
    }
    *out = B;
    return FV_OK;
}

extern "C" fv_status fv_csr_permute(const fv_csr *A, const int32_t *perm, void *stream, fv_csr **out) {
    if (!out) return FV_ERR_INVALID;
    *out = nullptr;
    return fv_host_guard([&] { return csr_permute_impl(A, perm, fv_stream(stream), out); });
}

extern "C" fv_status fv_csr_permute_values(fv_csr *B, void *stream) {
    if (!B || !B->perm_src || !B->perm_amap) return FV_ERR_INVALID;
    cudaStream_t st = fv_stream(stream);
    if (B->perm_src->nnz)
        fv_note_launch(), k_scatter_vals<<<592, 256, 0, st>>>(B->perm_src->nnz, B->perm_amap, B->perm_src->vals,
                                                               B->vals);
    FV_CUDA_TRY(cudaGetLastError());
    return FV_OK;
}

extern "C" fv_status fv_vec_permute(const fv_csr *B, const double *x, double *y, int32_t back, void *stream) {
    if (!B || !B->perm || !x || !y || x == y) return FV_ERR_INVALID;
    const int64_t n = B->nrows;
    const unsigned G = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 8));
    fv_note_launch(), k_vec_permute<<<G, 256, 0, fv_stream(stream)>>>(n, B->perm, x, y, back ? 1 : 0);
    FV_CUDA_TRY(cudaGetLastError());
    return FV_OK;
}

static fv_status perm_factor(const fv_csr *A, const int32_t *perm_host, int kind, void *stream, fv_precond **out) {
    if (!out) return FV_ERR_INVALID;
    *out = nullptr;
    return fv_host_guard([&] { return perm_factor_impl(A, perm_host, kind, fv_stream(stream), out); });
}

extern "C" fv_status fv_ic0_factor_perm(const fv_csr *A, const int32_t *perm, void *stream, fv_precond **out) {
    return perm_factor(A, perm, 1, stream, out);
}
extern "C" fv_status fv_ilu0_factor_perm(const fv_csr *A, const int32_t *perm, void *stream, fv_precond **out) {
    return perm_factor(A, perm, 2, stream, out);
}
extern "C" fv_status fv_precond_perm(const fv_precond *P, int32_t *perm_host, void *stream) {
    if (!P || !perm_host || !P->perm) return FV_ERR_INVALID;
    cudaStream_t st = fv_stream(stream);
    FV_CUDA_TRY(cudaMemcpyAsync(perm_host, P->perm, sizeof(int32_t) * P->n, cudaMemcpyDeviceToHost, st));
    FV_CUDA_TRY(cudaStreamSynchronize(st));
    return FV_OK;
}

// The box-colour ordering (fv_order.cpp) of a matrix assembled on a mesh:
// cell centres from the mesh, the domain box of every problem from its
// boundary faces' centres (a face belongs to its owner's problem).
static fv_status order_boxes_impl(const fv_csr *A, int32_t n_problems, const int64_t *offsets,
                                  int32_t rows_per_box, int32_t *perm_host, int32_t *level_host, fv_order_info *info,
                                  cudaStream_t st) {
    if (!A || !perm_host || A->nrows != A->ncols || A->nrows <= 0) return FV_ERR_INVALID;
    if (level_host && n_problems > 1) return FV_ERR_INVALID;
    const fv_mesh *m = A->mesh;
    if (!m || m->n_cells != A->nrows) {
        fv_internal_set_error_text("fv_order_boxes: the matrix was not assembled on a mesh (use fv_order_boxes_host)");
        return FV_ERR_INVALID;
    }
    const int64_t n = A->nrows, nnz = A->nnz, nbf = m->n_bfaces, fb0 = m->n_faces - m->n_bfaces;
    const int np = n_problems > 1 ? n_problems : 1;
    std::vector<int64_t> off((size_t)np + 1);
    if (np > 1) {
        if (!offsets || offsets[0] != 0 || offsets[np] != n) return FV_ERR_INVALID;
        for (int p = 0; p < np; ++p)
            if (offsets[p + 1] <= offsets[p]) return FV_ERR_INVALID;
        std::copy(offsets, offsets + np + 1, off.begin());
    } else {
        off[0] = 0;
        off[1] = n;
    }
    std::vector<int32_t> ptr((size_t)n + 1), col((size_t)(nnz ? nnz : 1));
    std::vector<double4> cell((size_t)n), bfc((size_t)(nbf ? nbf : 1));
    std::vector<int2> bfo((size_t)(nbf ? nbf : 1));
    FV_CUDA_TRY(cudaMemcpyAsync(ptr.data(), A->row_ptr, sizeof(int32_t) * (n + 1), cudaMemcpyDeviceToHost, st));
    if (nnz) FV_CUDA_TRY(cudaMemcpyAsync(col.data(), A->cols, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost, st));
    FV_CUDA_TRY(cudaMemcpyAsync(cell.data(), m->cell, sizeof(double4) * n, cudaMemcpyDeviceToHost, st));
    if (nbf) {
        FV_CUDA_TRY(cudaMemcpyAsync(bfc.data(), m->bface_center, sizeof(double4) * nbf, cudaMemcpyDeviceToHost, st));
        FV_CUDA_TRY(cudaMemcpyAsync(bfo.data(), m->face_cells + fb0, sizeof(int2) * nbf, cudaMemcpyDeviceToHost, st));
    }
    FV_CUDA_TRY(cudaStreamSynchronize(st));
    const int dim = m->dim;
    std::vector<double> lo((size_t)np * dim), hi((size_t)np * dim);
    std::vector<char> seen((size_t)np, 0);
    for (int64_t f = 0; f < nbf; ++f) {  // the boundary's face centres span each problem's domain
        const int64_t c = bfo[f].x;
        const int p = (int)(std::upper_bound(off.begin(), off.end(), c) - off.begin()) - 1;
        if (p < 0 || p >= np) continue;
        const double *x = &bfc[f].x;
        for (int d = 0; d < dim; ++d) {
            double &l = lo[(size_t)p * dim + d], &h = hi[(size_t)p * dim + d];
            if (!seen[p] || x[d] < l) l = x[d];
            if (!seen[p] || x[d] > h) h = x[d];
        }
        seen[p] = 1;
    }
    bool all_seen = true;
    for (int p = 0; p < np; ++p) all_seen = all_seen && seen[p];
    const double *lo_p = all_seen ? lo.data() : nullptr, *hi_p = all_seen ? hi.data() : nullptr;
    if (np == 1 && level_host)
        return fv_order_boxes_host_levels(n, dim, &cell[0].x, 4, lo_p, hi_p, ptr.data(), col.data(), rows_per_box,
                                          perm_host, level_host, info);
    if (np == 1)
        return fv_order_boxes_host(n, dim, &cell[0].x, 4, lo_p, hi_p, ptr.data(), col.data(), rows_per_box,
                                   perm_host, info);
    return fv_order_boxes_batch_host(np, off.data(), dim, &cell[0].x, 4, lo_p, hi_p, ptr.data(), col.data(),
                                     rows_per_box, perm_host, info);
}

extern "C" fv_status fv_order_boxes(const fv_csr *A, int32_t n_problems, const int64_t *offsets,
                                    int32_t rows_per_box, int32_t *perm_host, fv_order_info *info, void *stream) {
    return fv_host_guard([&] {
        return order_boxes_impl(A, n_problems, offsets, rows_per_box, perm_host, nullptr, info, fv_stream(stream));
    });
}

extern "C" fv_status fv_order_boxes_levels(const fv_csr *A, int32_t rows_per_box, int32_t *perm_host,
                                           int32_t *level_host, fv_order_info *info, void *stream) {
    if (!level_host) return FV_ERR_INVALID;
    return fv_host_guard([&] {
        return order_boxes_impl(A, 1, nullptr, rows_per_box, perm_host, level_host, info, fv_stream(stream));
    });
}

// Blocks (of 8 warps) per sweep launch and rows per thread of the reordered
// sweeps; 0 restores the defaults.  Any setting gives the same results: rows
// are handed out by ticket in a dependency-respecting order.
extern "C" fv_status fv_precond_set_grid(fv_precond *P, int32_t blocks, int32_t rows_per_thread) {
    if (!P || blocks < 0 || blocks > 148 * 32 || rows_per_thread < 0 || rows_per_thread > 8) return FV_ERR_INVALID;
    P->sweep_blocks = blocks;
    P->sweep_rpt = rows_per_thread;
    return FV_OK;
}

// Value-only refactorisation into an existing preconditioner (same matrix object).
extern "C" fv_status fv_precond_refactor(fv_precond *P, void *stream) {
    if (!P) return FV_ERR_INVALID;
    fv_precond *q = P;
    cudaStream_t st = fv_stream(stream);
    if (P->kind == 3) return diag_compute(P, st);
    if (P->fill) {  // level k / reordered: new values of the original matrix into the factorised one
        if (P->kind == 1 && !P->perm) FV_TRY(check_symmetric(const_cast<fv_csr *>(P->orig), st));
        FV_TRY(scatter_fill(P, st));
    }
    return factor_common(P->A, P->kind, st, &q);
}

extern "C" fv_status fv_precond_apply(fv_precond *P, const double *r, double *z, void *stream) {
    if (!P || !r || !z || r == z) return FV_ERR_INVALID;
    cudaStream_t st = fv_stream(stream);
    FV_TRY(fv_precond_apply_dev(P, r, z, st, nullptr, nullptr));
    return fv_precond_check_error(P, st);
}

extern "C" fv_status fv_precond_apply_host(fv_precond *P, const double *r_host, double *z_host, void *stream) {
    if (!P || !r_host || !z_host) return FV_ERR_INVALID;
    cudaStream_t st = fv_stream(stream);
    double *buf = nullptr;
    FV_CUDA_TRY(fv_malloc_async(&buf, sizeof(double) * 2 * P->n, st));
    FV_CUDA_TRY(cudaMemcpyAsync(buf, r_host, sizeof(double) * P->n, cudaMemcpyHostToDevice, st));
    fv_status s = fv_precond_apply_dev(P, buf, buf + P->n, st, nullptr, nullptr);
    if (s == FV_OK) s = fv_precond_check_error(P, st);
    if (s == FV_OK)
        FV_CUDA_TRY(cudaMemcpyAsync(z_host, buf + P->n, sizeof(double) * P->n, cudaMemcpyDeviceToHost, st));
    cudaFreeAsync(buf, st);
    FV_CUDA_TRY(cudaStreamSynchronize(st));
    return s;
}

static fv_status precond_export_impl(const fv_precond *P, int64_t *nnz, int32_t *row_ptr, int32_t *cols,
                                      double *vals, int32_t *n_dropped, void *stream) {
    if (!P || !nnz) return FV_ERR_INVALID;
    cudaStream_t st = fv_stream(stream);
    const fv_symbolic *s = P->sym;
    const int64_t n = P->n;
    if (n_dropped) *n_dropped = (int32_t)P->n_dropped;
    if (P->kind == 3) {  // the reference's `diagonal`: 1 / a_ii on the diagonal
        *nnz = n;
        if (!row_ptr || !cols || !vals) return FV_OK;
        FV_CUDA_TRY(cudaMemcpyAsync(vals, P->dinv, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
        FV_CUDA_TRY(cudaStreamSynchronize(st));
        for (int64_t i = 0; i <= n; ++i) row_ptr[i] = (int32_t)i;
        for (int64_t i = 0; i < n; ++i) cols[i] = (int32_t)i;
        return FV_OK;
    }
    // IC: the reference's `l` (lower incl. diagonal); ILU: the reference's `lu` (dropped entries removed)
    const int64_t total = P->kind == 1 ? s->nnz_l + n : s->nnz_l + s->nnz_u + n - P->n_dropped;
    if (!row_ptr || !cols || !vals) {
        *nnz = total;
        return FV_OK;
    }
    std::vector<int32_t> lp(n + 1), lc(s->nnz_l ? s->nnz_l : 1), up(n + 1), uc(s->nnz_u ? s->nnz_u : 1);
    std::vector<double> lv(s->nnz_l ? s->nnz_l : 1), uv(s->nnz_u ? s->nnz_u : 1), dg(n);
    FV_CUDA_TRY(cudaMemcpyAsync(lp.data(), s->l_ptr, sizeof(int32_t) * (n + 1), cudaMemcpyDeviceToHost, st));
    FV_CUDA_TRY(cudaMemcpyAsync(up.data(), s->u_ptr, sizeof(int32_t) * (n + 1), cudaMemcpyDeviceToHost, st));
    if (s->nnz_l) {
        FV_CUDA_TRY(cudaMemcpyAsync(lc.data(), s->l_col, sizeof(int32_t) * s->nnz_l, cudaMemcpyDeviceToHost, st));
        FV_CUDA_TRY(cudaMemcpyAsync(lv.data(), P->l_val, sizeof(double) * s->nnz_l, cudaMemcpyDeviceToHost, st));
    }
    if (s->nnz_u) {
        FV_CUDA_TRY(cudaMemcpyAsync(uc.data(), s->u_col, sizeof(int32_t) * s->nnz_u, cudaMemcpyDeviceToHost, st));
        FV_CUDA_TRY(cudaMemcpyAsync(uv.data(), P->u_val, sizeof(double) * s->nnz_u, cudaMemcpyDeviceToHost, st));
    }
    FV_CUDA_TRY(cudaMemcpyAsync(dg.data(), P->diag, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    FV_CUDA_TRY(cudaStreamSynchronize(st));
    int64_t o = 0;
    for (int64_t i = 0; i < n; ++i) {
        row_ptr[i] = (int32_t)o;
        for (int32_t k = lp[i]; k < lp[i + 1]; ++k) {
            if (P->kind == 2 && lv[k] == 0.0) continue;
            cols[o] = lc[k];
            vals[o++] = lv[k];
        }
        cols[o] = (int32_t)i;
        vals[o++] = dg[i];
        if (P->kind == 2)
            for (int32_t k = up[i]; k < up[i + 1]; ++k) {
                if (uv[k] == 0.0) continue;
                cols[o] = uc[k];
                vals[o++] = uv[k];
            }
    }
    row_ptr[n] = (int32_t)o;
    *nnz = o;
    return FV_OK;
}

extern "C" fv_status fv_precond_export(const fv_precond *P, int64_t *nnz, int32_t *row_ptr, int32_t *cols,
                                       double *vals, int32_t *n_dropped, void *stream) {
    return fv_host_guard([&] { return precond_export_impl(P, nnz, row_ptr, cols, vals, n_dropped, stream); });
}

extern "C" fv_status fv_precond_levels(const fv_precond *P, int32_t *fwd_level, int32_t *bwd_level,
                                       int32_t *n_fwd_levels, int32_t *n_bwd_levels, void *stream) {
    if (!P) return FV_ERR_INVALID;
    fv_symbolic *s = P->sym;
    if (!s) return FV_ERR_UNSUPPORTED;  // the diagonal preconditioner has no sweeps
    if (fwd_level || bwd_level) FV_TRY(ensure_host_levels(s, fv_stream(stream)));
    if (fwd_level) std::copy(s->h_fwd_level.begin(), s->h_fwd_level.end(), fwd_level);
    if (bwd_level) std::copy(s->h_bwd_level.begin(), s->h_bwd_level.end(), bwd_level);
    if (n_fwd_levels) *n_fwd_levels = s->n_fwd_levels;
    if (n_bwd_levels) *n_bwd_levels = s->n_bwd_levels;
    return FV_OK;
}
