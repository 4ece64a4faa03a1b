// Internal definitions shared by the CUDA translation units of libfvb200.
//
// Numerics: the whole library is compiled with --fmad=false so that every
// a*b+c keeps two roundings, as the reference's Rust code does; sqrt and
// division are CUDA's IEEE-rounded double operations.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include <new>

#include "fv_b200.h"

#define FV_CUDA_TRY(expr)                                  \
    do {                                                   \
        cudaError_t _e = (expr);                           \
        if (_e != cudaSuccess) {                           \
            fv_internal_set_cuda_error(_e, #expr);         \
            return (_e == cudaErrorMemoryAllocation) ? FV_ERR_ALLOC : FV_ERR_CUDA; \
        }                                                  \
    } while (0)

#define FV_TRY(expr)                     \
    do {                                 \
        fv_status _s = (expr);           \
        if (_s != FV_OK) return _s;      \
    } while (0)

void fv_internal_set_cuda_error(cudaError_t e, const char *what);
void fv_internal_set_error_text(const char *what);

// Runs f() so that no C++ exception crosses the C ABI: a failed host
// allocation (std::bad_alloc from a std::vector) returns FV_ERR_ALLOC, any
// other exception (a size the host containers reject) FV_ERR_INVALID.
template <typename F>
inline fv_status fv_host_guard(F &&f) noexcept {
    try {
        return f();
    } catch (const std::bad_alloc &) {
        fv_internal_set_error_text("host memory allocation failed");
        return FV_ERR_ALLOC;
    } catch (...) {
        fv_internal_set_error_text("host container size rejected");
        return FV_ERR_INVALID;
    }
}
// Counts kernel launches made by this library (fv_launch_count).
// cudaMallocAsync from the device's default pool, which is first told to keep
// freed memory (release threshold = max): without that the pool hands memory
// back to the driver at synchronisations and re-maps it on the next request,
// which showed up as rare ~1 s stalls in repeated solves.
cudaError_t fv_malloc_async_raw(void **p, size_t bytes, cudaStream_t st);
template <typename T>
static inline cudaError_t fv_malloc_async(T **p, size_t bytes, cudaStream_t st) {
    return fv_malloc_async_raw(reinterpret_cast<void **>(p), bytes, st);
}
void fv_note_launch();
void fv_note_launches(long long delta);  // graph replays add, captures (not run) subtract
unsigned long long fv_launches_now();

static inline cudaStream_t fv_stream(void *s) { return (cudaStream_t)s; }

// Device-side error word (one per object that runs bounded waits).
enum : int { FV_DEV_OK = 0, FV_DEV_TIMEOUT = 1, FV_DEV_SINGULAR = 2, FV_DEV_BREAKDOWN = 4 };

// ------------------------------------------------------------------ objects
struct fv_mesh {
    int dim = 0;
    int64_t n_cells = 0, n_faces = 0, n_bfaces = 0;
    int maxf = 0;                      // max faces of a cell
    int2 *face_cells = nullptr;        // (owner, neighbour) per face
    double *face_area = nullptr;       // per face
    double4 *bface_center = nullptr;   // per boundary face (x, y, z|0, 0)
    double4 *cell = nullptr;           // (cx, cy, cz|0, volume)
    int32_t *cf_ptr = nullptr;         // cell -> faces CSR, faces ascending
    int32_t *cf_face = nullptr;        // face id, bit 31 set when the cell is the face's neighbour
    int32_t *cf_other = nullptr;       // the other cell, -1 for boundary faces
    int2 *cf_pad = nullptr;            // (cf_face, cf_other) at cell * padf + slot, padded with (0, -2)
    int padf = 0;                      // 4 or 8 (0: no padded copy, cells with more than 8 faces)
    int64_t ncf = 0;                   // entries of cf_face / cf_other
    // Corrected scheme / gradients (present when uploaded with normals and cell_faces)
    double4 *face_normal = nullptr;    // per face (x, y, z|0, 0)
    double4 *face_center = nullptr;    // per face, all faces
    int32_t *gcf_ptr = nullptr;        // the cells' faces in mesh order (Mesh::cell_faces)
    int32_t *gcf_face = nullptr;
    double4 *gcoef = nullptr;          // gradient coefficient of each (cell, face) in that order
    double4 *gdiag = nullptr;          // gradient coefficient of the cell itself
    // Orthogonal-scheme geometry cached on the first assembly that uses it:
    // (area, 1/|d|) per face (|d| from the owner centre to the neighbour centre
    // or boundary face centre) and the cells' volumes
    double2 *face_geo = nullptr;
    double *cell_vol = nullptr;
    // CSR pattern of cell_to_cell (built on the first assemble)
    int32_t *row_ptr = nullptr;
    int32_t *cols = nullptr;
    int64_t nnz = -1;
};

// Gradient coefficients of Mesh::compute (compute.rs:155-203) for a mesh whose
// cell, face_cells, face_center, gcf_ptr and gcf_face are resident; a cell with
// a singular gradient matrix sets *dbad.
cudaError_t fv_mesh_launch_grad_coeffs(fv_mesh *m, int *dbad, cudaStream_t st);

struct fv_symbolic;  // triangular split + level schedules of a pattern (fv_precond.cu)

// Level-k fill patterns of the reference (fv_fill.cu).  From the host CSR
// pattern of A (sorted rows with diagonal), the sorted pattern of the factor
// and, for every entry of A, its position in that pattern.
//   kind 2 (ILU): row i = row_i_l_sparsity ∪ {i} ∪ row_i_u_sparsity
//                 (incomplete_lower_upper.rs:30-137)
//   kind 1 (IC):  row i = entries of A ∪ the level-ball of i
//                 (incomplete_cholesky.rs:35-85, 148-192); fill[k] marks fill
fv_status fv_fill_pattern(int kind, int level, int64_t n, const int32_t *ptr, const int32_t *col,
                          std::vector<int32_t> &fptr, std::vector<int32_t> &fcol, std::vector<int32_t> &amap,
                          std::vector<uint8_t> &fill);

// Box tiling of one sweep direction (fv_tiles.cu): boxes in dispatch order,
// each a run of steps (rows of one level, at most 32); trow lists the rows in
// that order; dsrc[k] (aligned with the swept side's entries) is the column j
// when the dependency is read from the vector, or -(slot + 1) when it comes
// from the warp's shared-memory ring of its last `ring` steps.
struct fv_tile_plan {
    std::vector<int32_t> box_step, sptr, trow, dsrc;
    int32_t nb = 0, nsteps = 0;
    double lane_use = 0.0, ring_share = 0.0, edge = 0.0;
    double est = 0.0;  // estimated critical path of both sweeps / that of the level schedule
};
bool fv_build_tile_plans(int64_t n, int dim, const double *cell, const int32_t *lp, const int32_t *lc,
                         const int32_t *up, const int32_t *uc, const int32_t *fwd_level, const int32_t *bwd_level,
                         const int32_t *fwd_order, const int32_t *bwd_order, int ring, fv_tile_plan &fwd,
                         fv_tile_plan &bwd);
#define FV_TILE_RING 8
#define FV_TILE_MAXL 4              // entries per row on the swept side in the tiled layout
#define FV_TILE_PAD (-2147483647 - 1)  // unused entry of a slot

// Rows a sweep may skip: row i is skipped when done[group[i] * stride] != 0
// (rows of the problems of a batch that have converged).
struct fv_row_skip {
    const int32_t *group;
    const int *done;
    int stride;
};

struct fv_csr {
    int64_t nrows = 0, ncols = 0, nnz = 0;
    int32_t *row_ptr = nullptr;   // device
    int32_t *cols = nullptr;      // device
    double *vals = nullptr;       // device
    bool owns_pattern = true;     // false when the pattern belongs to an fv_mesh
    // IC(k) fill patterns: per stored entry, 1 when it is fill (not in the
    // matrix it was built from); the backward sweep then visits a row's
    // entries of the matrix first and its fill after them, as the reference
    // does (incomplete_cholesky.rs:167-192, 235-244).  Empty otherwise.
    std::vector<uint8_t> fill_mask;
    const fv_mesh *mesh = nullptr;
    fv_symbolic *sym = nullptr;   // cached symbolic analysis (value independent)
    // a permuted copy Q A Q^T (fv_csr_permute): the matrix its values come from,
    // the permutation (row i = src row perm[i]) and src's entry k's position here
    const fv_csr *perm_src = nullptr;
    int32_t *perm = nullptr;
    int32_t *perm_amap = nullptr;
};

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ unsigned long long fv_ld_relaxed_u64(const void *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void fv_st_relaxed_u64(void *p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned fv_ld_relaxed_u32(const void *p) {
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned fv_ld_acquire_u32(const void *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void fv_st_release_u32(void *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long fv_globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// A value slot that has not been produced yet holds all-ones bits (memset
// 0xFF).  Producers never store that pattern: a computed all-ones NaN is
// replaced by the canonical quiet NaN.
#define FV_SENTINEL_U64 0xFFFFFFFFFFFFFFFFULL
#define FV_SENTINEL_U32 0xFFFFFFFFu
// Bounded waits give up after this many nanoseconds of wall time.
#define FV_WAIT_LIMIT_NS 2000000000ULL

__device__ __forceinline__ unsigned long long fv_pack_value(double v) {
    unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return b == FV_SENTINEL_U64 ? 0x7FF8000000000000ULL : b;
}
__device__ __forceinline__ unsigned fv_pack_value(float v) {
    unsigned b = (unsigned)__float_as_uint(v);
    return b == FV_SENTINEL_U32 ? 0x7FC00000u : b;
}

// Wait until *p holds a produced value.  Gives up (returns NaN and raises
// FV_DEV_TIMEOUT in *err) after FV_WAIT_LIMIT_NS, or as soon as another
// thread has raised an error, so one failure cannot cascade into long waits.
__device__ __forceinline__ double fv_wait_value(const double *p, int *err) {
    unsigned long long v = fv_ld_relaxed_u64(p);
    if (v != FV_SENTINEL_U64) return __longlong_as_double((long long)v);
    unsigned long long t0 = fv_globaltimer();
    for (unsigned it = 1;; ++it) {
        v = fv_ld_relaxed_u64(p);
        if (v != FV_SENTINEL_U64) return __longlong_as_double((long long)v);
        if ((it & 255u) == 0) {
            if (*(volatile int *)err) return __longlong_as_double(0x7FF8000000000000LL);
            if (fv_globaltimer() - t0 > FV_WAIT_LIMIT_NS) {
                atomicOr(err, FV_DEV_TIMEOUT);
                return __longlong_as_double(0x7FF8000000000000LL);
            }
        }
    }
}
__device__ __forceinline__ float fv_wait_value(const float *p, int *err) {
    unsigned v = fv_ld_relaxed_u32(p);
    if (v != FV_SENTINEL_U32) return __uint_as_float(v);
    unsigned long long t0 = fv_globaltimer();
    for (unsigned it = 1;; ++it) {
        v = fv_ld_relaxed_u32(p);
        if (v != FV_SENTINEL_U32) return __uint_as_float(v);
        if ((it & 255u) == 0) {
            if (*(volatile int *)err) return __uint_as_float(0x7FC00000u);
            if (fv_globaltimer() - t0 > FV_WAIT_LIMIT_NS) {
                atomicOr(err, FV_DEV_TIMEOUT);
                return __uint_as_float(0x7FC00000u);
            }
        }
    }
}
__device__ __forceinline__ void fv_publish(double *p, double v) { fv_st_relaxed_u64(p, fv_pack_value(v)); }
__device__ __forceinline__ void fv_publish(float *p, float v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(fv_pack_value(v)) : "memory");
}

__device__ __forceinline__ void fv_reset_slot(double *p) { fv_st_relaxed_u64(p, FV_SENTINEL_U64); }
__device__ __forceinline__ void fv_reset_slot(float *p) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(FV_SENTINEL_U32) : "memory");
}

// Wait until flag == want (acquire).  Same bounded policy as fv_wait_value.
__device__ __forceinline__ bool fv_wait_flag(const unsigned *flag, unsigned want, int *err) {
    if (fv_ld_acquire_u32(flag) == want) return true;
    unsigned long long t0 = fv_globaltimer();
    for (unsigned it = 1;; ++it) {
        if (fv_ld_acquire_u32(flag) == want) return true;
        if ((it & 255u) == 0) {
            if (*(volatile int *)err) return false;
            if (fv_globaltimer() - t0 > FV_WAIT_LIMIT_NS) {
                atomicOr(err, FV_DEV_TIMEOUT);
                return false;
            }
        }
    }
}

// Deterministic block reduction of NV doubles (fixed shuffle tree, fixed
// warp order).  Result valid in thread 0.
template <int NV>
__device__ __forceinline__ void fv_block_reduce(double (&v)[NV], double *smem /* [NV*32] */) {
#pragma unroll
    for (int q = 0; q < NV; ++q)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; ++q) smem[q * 32 + warp] = v[q];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            v[q] = lane < nw ? smem[q * 32 + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
        }
    }
}

// Fixed launch geometry for reductions: the grid size depends only on n, so
// partial sums (and therefore results) are reproducible run to run and do not
// depend on what else runs on the GPU.
static inline int fv_reduce_grid(int64_t n, int block) {
    int64_t g = (n + (int64_t)block * 4 - 1) / ((int64_t)block * 4);
    if (g < 1) g = 1;
    if (g > 1184) g = 1184;  // 148 SMs x 8
    return (int)g;
}
