// CSR matrix objects, SpMV and the Krylov solvers.
//
// Reference: DistributedMatrix::imul (src/linalg/dmatrix.rs:136-146),
// DistributedVector::dot (src/linalg/dvector.rs:63-79),
// conjugate_gradient (src/linalg/solvers/conjugate_gradient.rs:12-111),
// bi_conjugate_gradient_stab (src/linalg/solvers/bi_conjugate_gradient_stab.rs:13-178),
// LinearSolverOptions / LinearSolverInfo (src/linalg/solvers/mod.rs:11-42).
//
// Design.  Every vector pass of an iteration is one kernel that also produces
// the dot products that follow it: the block partials are written to a fixed
// slot per block and the last block to finish reduces them in block order and
// runs the scalar update of the iteration (alpha, omega, beta, the
// convergence test, the restart decision) on the device.  The grid size
// depends only on n, so results are reproducible and independent of other
// work on the GPU.  Scalars never travel to the host inside the loop; the
// host enqueues iterations in batches and reads one `done` word per batch.
// Kernels of an iteration that follows convergence return immediately.
#include <algorithm>
#include <cmath>
#include <vector>

#include "fv_internal.cuh"

struct fv_symbolic;
struct fv_precond;
fv_status fv_precond_apply_dev(fv_precond *P, const double *r, double *z, cudaStream_t st, const int *skip,
                               const fv_row_skip *rskip);
fv_status fv_precond_check_error(fv_precond *P, cudaStream_t st);
void fv_symbolic_free(fv_symbolic *s);

// ------------------------------------------------------------------ CSR API
extern "C" fv_status fv_csr_create_host(int64_t nrows, int64_t ncols, const int32_t *row_ptr, const int32_t *cols,
                                        const double *vals, void *stream, fv_csr **out) {
    if (!out || nrows < 0 || ncols < 0 || !row_ptr || nrows >= 0x7fffffffLL) return FV_ERR_INVALID;
    *out = nullptr;
    if (row_ptr[0] != 0) return FV_ERR_INVALID;
    for (int64_t i = 0; i < nrows; ++i) {
        if (row_ptr[i + 1] < row_ptr[i]) return FV_ERR_INVALID;
        for (int32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
            if (cols[k] < 0 || cols[k] >= ncols) return FV_ERR_INVALID;
            if (k > row_ptr[i] && cols[k] <= cols[k - 1]) return FV_ERR_INVALID;
        }
    }
    const int64_t nnz = row_ptr[nrows];
    cudaStream_t st = fv_stream(stream);
    fv_csr *a = new fv_csr();
    a->nrows = nrows;
    a->ncols = ncols;
    a->nnz = nnz;
    cudaError_t e = cudaMalloc(&a->row_ptr, sizeof(int32_t) * (nrows + 1));
    if (e == cudaSuccess) e = cudaMalloc(&a->cols, sizeof(int32_t) * (nnz ? nnz : 1));
    if (e == cudaSuccess) e = cudaMalloc(&a->vals, sizeof(double) * (nnz ? nnz : 1));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(a->row_ptr, row_ptr, sizeof(int32_t) * (nrows + 1), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && nnz) e = cudaMemcpyAsync(a->cols, cols, sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && nnz) e = cudaMemcpyAsync(a->vals, vals, sizeof(double) * nnz, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        fv_internal_set_cuda_error(e, "fv_csr_create_host");
        fv_csr_destroy(a);
        return e == cudaErrorMemoryAllocation ? FV_ERR_ALLOC : FV_ERR_CUDA;
    }
    *out = a;
    return FV_OK;
}

extern "C" fv_status fv_csr_info(const fv_csr *A, int64_t *nrows, int64_t *ncols, int64_t *nnz) {
    if (!A) return FV_ERR_INVALID;
    if (nrows) *nrows = A->nrows;
    if (ncols) *ncols = A->ncols;
    if (nnz) *nnz = A->nnz;
    return FV_OK;
}

extern "C" fv_status fv_csr_download(const fv_csr *A, int32_t *row_ptr, int32_t *cols, double *vals, void *stream) {
    if (!A) return FV_ERR_INVALID;
    cudaStream_t st = fv_stream(stream);
    if (row_ptr)
        FV_CUDA_TRY(cudaMemcpyAsync(row_ptr, A->row_ptr, sizeof(int32_t) * (A->nrows + 1), cudaMemcpyDeviceToHost, st));
    if (cols && A->nnz)
        FV_CUDA_TRY(cudaMemcpyAsync(cols, A->cols, sizeof(int32_t) * A->nnz, cudaMemcpyDeviceToHost, st));
    if (vals && A->nnz)
        FV_CUDA_TRY(cudaMemcpyAsync(vals, A->vals, sizeof(double) * A->nnz, cudaMemcpyDeviceToHost, st));
    FV_CUDA_TRY(cudaStreamSynchronize(st));
    return FV_OK;
}

extern "C" fv_status fv_csr_destroy(fv_csr *A) {
    if (!A) return FV_OK;
    if (A->owns_pattern) {
        cudaFree(A->row_ptr);
        cudaFree(A->cols);
    }
    cudaFree(A->vals);
    cudaFree(A->perm);
    cudaFree(A->perm_amap);
    fv_symbolic_free(A->sym);
    delete A;
    return FV_OK;
}

// ------------------------------------------------------------------ kernels
namespace {

constexpr int RB = 256;  // block size of every reduction kernel

// Row dot: y_i = sum_k a_k x_col(k), left to right from 0.0 (dmatrix.rs:138-145).
// The first 8 entries' column, value and x loads are all issued before the
// sum starts (the x gathers of a row are independent), the sum still runs in
// entry order.
__device__ __forceinline__ double row_dot(const int32_t *__restrict__ ptr, const int32_t *__restrict__ col,
                                          const double *__restrict__ val, const double *__restrict__ x, int64_t i) {
    constexpr int E = 8;
    const int k0 = ptr[i], k1 = ptr[i + 1];
    const int len = k1 - k0;
    double av[E], xv[E];
#pragma unroll
    for (int q = 0; q < E; ++q) {
        av[q] = 0.0;
        xv[q] = 0.0;
        if (q < len) {
            av[q] = val[k0 + q];
            xv[q] = __ldg(&x[col[k0 + q]]);
        }
    }
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < E; ++q)
        if (q < len) s += av[q] * xv[q];
    for (int k = k0 + E; k < k1; ++k) s += val[k] * __ldg(&x[col[k]]);
    return s;
}

__global__ void __launch_bounds__(256) k_spmv(int64_t n, const int32_t *__restrict__ ptr,
                                              const int32_t *__restrict__ col, const double *__restrict__ val,
                                              const double *__restrict__ x, double *__restrict__ y) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = row_dot(ptr, col, val, x, i);
}

// Device-resident state of one solve.
struct SolverState {
    double tol, rtol;
    int64_t max_it;
    double bnorm, init_res, error;
    double rho, alpha, omega, beta, rz;
    int64_t iter;
    int done, restart, finish_h, zero_x, breakdown, restarts;
    unsigned ticket;
    double *hist;        // max_it + 2 entries
    double *partial;     // [grid * 4]
};

// Last-block reduction of NV partials per block, then the scalar epilogue.
template <int NV, class Epi>
__device__ __forceinline__ void finish_reduce(double (&v)[NV], SolverState *S, Epi epi) {
    __shared__ double sm[NV * 32];
    __shared__ bool last;
    fv_block_reduce<NV>(v, sm);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) S->partial[blockIdx.x * NV + q] = v[q];
        __threadfence();
        last = (atomicAdd(&S->ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    double t[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) t[q] = 0.0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
        for (int q = 0; q < NV; ++q) t[q] += __ldcg(&S->partial[b * NV + q]);
    fv_block_reduce<NV>(t, sm);
    if (threadIdx.x == 0) {
        S->ticket = 0;
        epi(S, t);
    }
}

__device__ __forceinline__ bool bad(double x) { return !isfinite(x); }

// ---- generic epilogues
struct EpiBnorm {  // bnorm = sqrt(b.b); bnorm < 1e-14 -> x = 0, done
    __device__ void operator()(SolverState *S, const double *t) const {
        S->bnorm = sqrt(t[0]);
        if (S->bnorm < 1e-14) {
            S->init_res = S->bnorm;
            S->error = S->bnorm;
            S->hist[0] = S->bnorm;
            S->iter = 0;
            S->zero_x = 1;
            S->done = 1;
        }
    }
};

// r = -(A x - b); rr = r.r  (conjugate_gradient.rs:89-94; also copies r to rh, p for BiCGStab)
template <bool BICG>
__global__ void __launch_bounds__(RB) k_residual(int64_t n, const int32_t *__restrict__ ptr,
                                                 const int32_t *__restrict__ col, const double *__restrict__ val,
                                                 const double *__restrict__ x, const double *__restrict__ b,
                                                 double *__restrict__ r, double *__restrict__ rh,
                                                 double *__restrict__ p, SolverState *S) {
    if (S->done) return;
    double v[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double ri = row_dot(ptr, col, val, x, i);
        ri -= b[i];
        ri *= -1.0;
        r[i] = ri;
        if (BICG) {
            rh[i] = ri;
            p[i] = ri;
        }
        v[0] += ri * ri;
    }
    finish_reduce<1>(v, S, [] __device__(SolverState * S, const double *t) {
        S->init_res = sqrt(t[0]) / S->bnorm;
        S->error = 1.0;
        if (BICG) {
            if (S->init_res < S->tol) {
                S->error = S->init_res;
                S->hist[0] = S->init_res;
                S->iter = 0;
                S->done = 1;
                return;
            }
            S->rho = t[0];  // rh.r with rh == r
        }
        if (!(S->error > S->tol) || S->iter > S->max_it) S->done = 1;
    });
}

__global__ void __launch_bounds__(RB) k_dot_self(int64_t n, const double *__restrict__ a, SolverState *S) {
    double v[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        v[0] += a[i] * a[i];
    finish_reduce<1>(v, S, EpiBnorm());
}

__global__ void k_zero_if(int64_t n, double *x, const SolverState *S) {
    if (!S->zero_x) return;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = 0.0;
}

__global__ void k_copy_if_active(int64_t n, const double *__restrict__ a, double *__restrict__ b,
                                 const SolverState *S) {
    if (S->done) return;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = a[i];
}

// ---- CG
// p = z, rz = r.z (conjugate_gradient.rs:100-113: set p, then r.z of the first iteration)
__global__ void __launch_bounds__(RB) k_cg_init_p(int64_t n, const double *__restrict__ r,
                                                  const double *__restrict__ z, double *__restrict__ p,
                                                  SolverState *S) {
    if (S->done) return;
    double v[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double zi = z[i];
        p[i] = zi;
        v[0] += r[i] * zi;
    }
    finish_reduce<1>(v, S, [] __device__(SolverState * S, const double *t) { S->rz = t[0]; });
}

// ap = A p; alpha = r.z / p.ap
__global__ void __launch_bounds__(RB) k_cg_spmv(int64_t n, const int32_t *__restrict__ ptr,
                                                const int32_t *__restrict__ col, const double *__restrict__ val,
                                                const double *__restrict__ p, double *__restrict__ ap,
                                                SolverState *S) {
    if (S->done) return;
    double v[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double y = row_dot(ptr, col, val, p, i);
        ap[i] = y;
        v[0] += p[i] * y;
    }
    finish_reduce<1>(v, S, [] __device__(SolverState * S, const double *t) { S->alpha = S->rz / t[0]; });
}

// x += p alpha; r -= ap alpha; error = |r|/|b| and the convergence test (:119-131)
__global__ void __launch_bounds__(RB) k_cg_update(int64_t n, double *__restrict__ x, double *__restrict__ r,
                                                  const double *__restrict__ p, const double *__restrict__ ap,
                                                  SolverState *S) {
    if (S->done) return;
    const double alpha = S->alpha;
    double v[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        x[i] += p[i] * alpha;
        const double ri = r[i] - ap[i] * alpha;
        r[i] = ri;
        v[0] += ri * ri;
    }
    finish_reduce<1>(v, S, [] __device__(SolverState * S, const double *t) {
        S->error = sqrt(t[0]) / S->bnorm;
        if ((S->error < S->tol) || (S->error / S->init_res < S->rtol)) {
            S->hist[S->iter] = S->error;
            S->iter += 1;
            S->done = 1;
        }
        if (bad(S->alpha)) S->breakdown = 1;
    });
}

// beta = r.z_new / r.z; history; loop guard (:136-150)
__global__ void __launch_bounds__(RB) k_cg_rz(int64_t n, const double *__restrict__ r, const double *__restrict__ z,
                                              SolverState *S) {
    if (S->done) return;
    double v[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        v[0] += r[i] * z[i];
    finish_reduce<1>(v, S, [] __device__(SolverState * S, const double *t) {
        S->beta = t[0] / S->rz;
        S->rz = t[0];
        S->hist[S->iter] = S->error;
        S->iter += 1;
        if (!(S->error > S->tol) || S->iter > S->max_it) S->done = 1;
    });
}

__global__ void __launch_bounds__(RB) k_cg_p(int64_t n, const double *__restrict__ z, double *__restrict__ p,
                                             const SolverState *S) {
    if (S->done) return;
    const double beta = S->beta;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = z[i] + p[i] * beta;
}

// ---- BiCGStab
// v = A y; alpha = rho / rh.v
__global__ void __launch_bounds__(RB) k_bi_spmv1(int64_t n, const int32_t *__restrict__ ptr,
                                                 const int32_t *__restrict__ col, const double *__restrict__ val,
                                                 const double *__restrict__ y, double *__restrict__ v_out,
                                                 const double *__restrict__ rh, SolverState *S) {
    if (S->done) return;
    double v[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double vi = row_dot(ptr, col, val, y, i);
        v_out[i] = vi;
        v[0] += rh[i] * vi;
    }
    finish_reduce<1>(v, S, [] __device__(SolverState * S, const double *t) { S->alpha = S->rho / t[0]; });
}

// s = r - v alpha; |s|/|b| test (bi_conjugate_gradient_stab.rs:100-118).  h = x + y alpha is not
// stored: it is recomputed, with the same rounding, where it is used.
__global__ void __launch_bounds__(RB) k_bi_s(int64_t n, const double *__restrict__ r, const double *__restrict__ vv,
                                             double *__restrict__ s, SolverState *S) {
    if (S->done) return;
    const double alpha = S->alpha;
    double v[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double si = r[i] - vv[i] * alpha;
        s[i] = si;
        v[0] += si * si;
    }
    finish_reduce<1>(v, S, [] __device__(SolverState * S, const double *t) {
        const double sn = sqrt(t[0]) / S->bnorm;
        if ((sn < S->tol) || (sn / S->init_res < S->rtol)) {
            S->error = sn;
            S->hist[S->iter] = sn;
            S->finish_h = 1;
            S->iter += 1;
            S->done = 1;
        }
        if (bad(S->alpha)) S->breakdown = 1;
    });
}

// t = A z; omega = t.s / t.t
__global__ void __launch_bounds__(RB) k_bi_spmv2(int64_t n, const int32_t *__restrict__ ptr,
                                                 const int32_t *__restrict__ col, const double *__restrict__ val,
                                                 const double *__restrict__ z, double *__restrict__ t_out,
                                                 const double *__restrict__ s, SolverState *S) {
    if (S->done) return;
    double v[2] = {0.0, 0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double ti = row_dot(ptr, col, val, z, i);
        t_out[i] = ti;
        v[0] += ti * s[i];
        v[1] += ti * ti;
    }
    finish_reduce<2>(v, S, [] __device__(SolverState * S, const double *t) { S->omega = t[0] / t[1]; });
}

// x = (x + y alpha) + z omega; r = s - t omega; rr, rh.r; test; beta, restart (:122-169)
__global__ void __launch_bounds__(RB) k_bi_update(int64_t n, double *__restrict__ x, double *__restrict__ r,
                                                  const double *__restrict__ y, const double *__restrict__ z,
                                                  const double *__restrict__ s, const double *__restrict__ t,
                                                  const double *__restrict__ rh, SolverState *S) {
    if (S->done) return;
    const double alpha = S->alpha, omega = S->omega;
    double v[2] = {0.0, 0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double h = x[i] + y[i] * alpha;
        x[i] = h + z[i] * omega;
        const double ri = s[i] - t[i] * omega;
        r[i] = ri;
        v[0] += ri * ri;
        v[1] += rh[i] * ri;
    }
    finish_reduce<2>(v, S, [] __device__(SolverState * S, const double *t) {
        const double rn = sqrt(t[0]) / S->bnorm;
        if ((rn < S->tol) || (rn / S->init_res < S->rtol)) {
            S->error = rn;
            S->hist[S->iter] = rn;
            S->iter += 1;
            S->done = 1;
            return;
        }
        const double rho_new = t[1];
        S->beta = (rho_new / S->rho) * (S->alpha / S->omega);
        S->rho = rho_new;
        if (fabs(S->rho) > (1e-15 * S->bnorm)) {
            S->restart = 0;
        } else {
            S->restart = 1;
            S->restarts += 1;
            S->rho = t[0];  // rh = r, then rh.r
        }
        if (bad(S->omega) || bad(S->beta)) S->breakdown = 1;
        S->error = rn / S->bnorm;  // the loop guard divides by |b| twice (:171)
        S->hist[S->iter] = S->error;
        S->iter += 1;
        if (!(S->error > S->tol) || S->iter > S->max_it) S->done = 1;
    });
}

// p = r + (p - v omega) beta, or the restart rh = r, p = r
__global__ void __launch_bounds__(RB) k_bi_p(int64_t n, const double *__restrict__ r, const double *__restrict__ vv,
                                             double *__restrict__ p, double *__restrict__ rh, const SolverState *S) {
    if (S->done) return;
    const double omega = S->omega, beta = S->beta;
    if (S->restart) {
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
            rh[i] = r[i];
            p[i] = r[i];
        }
    } else {
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
            p[i] = r[i] + (p[i] - vv[i] * omega) * beta;
    }
}

// x = h = x + y alpha when the |s| test ended the solve
__global__ void k_bi_finish(int64_t n, double *__restrict__ x, const double *__restrict__ y, const SolverState *S) {
    if (!S->finish_h) return;
    const double alpha = S->alpha;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = x[i] + y[i] * alpha;
}

}  // namespace

extern "C" fv_status fv_spmv(const fv_csr *A, const double *x, double *y, void *stream) {
    if (!A || !x || !y || x == y) return FV_ERR_INVALID;
    if (A->nrows == 0) return FV_OK;
    const int G = (int)std::min<int64_t>((A->nrows + 255) / 256, 148 * 16);
    fv_note_launch(), k_spmv<<<G, 256, 0, fv_stream(stream)>>>(A->nrows, A->row_ptr, A->cols, A->vals, x, y);
    FV_CUDA_TRY(cudaGetLastError());
    return FV_OK;
}

extern "C" fv_status fv_spmv_host(const fv_csr *A, const double *x_host, double *y_host, void *stream) {
    if (!A || !x_host || !y_host) return FV_ERR_INVALID;
    cudaStream_t st = fv_stream(stream);
    double *buf = nullptr;
    FV_CUDA_TRY(fv_malloc_async(&buf, sizeof(double) * (A->ncols + A->nrows + 1), st));
    FV_CUDA_TRY(cudaMemcpyAsync(buf, x_host, sizeof(double) * A->ncols, cudaMemcpyHostToDevice, st));
    fv_status s = fv_spmv(A, buf, buf + A->ncols, stream);
    if (s == FV_OK)
        FV_CUDA_TRY(cudaMemcpyAsync(y_host, buf + A->ncols, sizeof(double) * A->nrows, cudaMemcpyDeviceToHost, st));
    cudaFreeAsync(buf, st);
    FV_CUDA_TRY(cudaStreamSynchronize(st));
    return s;
}

// ------------------------------------------------------------------ drivers
namespace {

struct Workspace {
    SolverState *S = nullptr;
    double *vec = nullptr;
    int nvec = 0;
};

fv_status ws_alloc(Workspace &w, int64_t n, int nvec, const fv_solver_options &opt, int grid, cudaStream_t st) {
    const int64_t hist = opt.max_iterations + 3;
    const size_t bytes = sizeof(SolverState) + sizeof(double) * ((size_t)grid * 4 + (size_t)hist + (size_t)n * nvec);
    char *mem = nullptr;
    FV_CUDA_TRY(fv_malloc_async(&mem, bytes, st));
    w.S = (SolverState *)mem;
    double *d = (double *)(mem + sizeof(SolverState));
    SolverState h{};
    h.tol = opt.absolute_tolerance;
    h.rtol = opt.relative_tolerance;
    h.max_it = opt.max_iterations;
    h.error = 1.0;
    h.partial = d;
    h.hist = d + (size_t)grid * 4;
    w.vec = h.hist + hist;
    w.nvec = nvec;
    FV_CUDA_TRY(cudaMemcpyAsync(w.S, &h, sizeof(SolverState), cudaMemcpyHostToDevice, st));
    return FV_OK;
}

fv_status read_state(const Workspace &w, SolverState &h, cudaStream_t st) {
    FV_CUDA_TRY(cudaMemcpyAsync(&h, w.S, sizeof(SolverState), cudaMemcpyDeviceToHost, st));
    FV_CUDA_TRY(cudaStreamSynchronize(st));
    return FV_OK;
}

fv_status fill_info(bool bicg, const SolverState &h, fv_solver_info *info, fv_precond *P, cudaStream_t st) {
    if (!info) return FV_OK;
    info->iterations = h.iter;
    info->initial_residual = h.init_res;
    info->final_residual = h.error;
    info->restarts = h.restarts;
    int64_t hl = h.zero_x ? 1 : h.iter;
    if (bicg && !h.zero_x && h.done && h.iter == 0 && h.init_res < h.tol) hl = 1;  // BiCGStab early return
    info->history_len = hl;
    if (info->history && info->history_cap > 0 && hl > 0) {
        int64_t c = std::min(hl, info->history_cap);
        FV_CUDA_TRY(cudaMemcpyAsync(info->history, h.hist, sizeof(double) * c, cudaMemcpyDeviceToHost, st));
        FV_CUDA_TRY(cudaStreamSynchronize(st));
    }
    fv_status s = FV_OK;
    if (P) s = fv_precond_check_error(P, st);
    if (s == FV_OK && (h.breakdown || !std::isfinite(h.error))) s = FV_ERR_BREAKDOWN;
    info->status = s;
    return s;
}

fv_status apply_or_copy(fv_precond *P, const double *r, double *z, int64_t n, int G, const SolverState *S,
                        cudaStream_t st) {
    if (P) return fv_precond_apply_dev(P, r, z, st, &S->done, nullptr);
    fv_note_launch(), k_copy_if_active<<<G, RB, 0, st>>>(n, r, z, S);  // IdentityPreconditioner
    FV_CUDA_TRY(cudaGetLastError());
    return FV_OK;
}

int batch_size(int64_t n) { return n >= (1 << 20) ? 4 : 8; }

// One pinned int per host thread for the done flag of loop_until_done,
// allocated on first use and kept for the thread's life (freeing pinned
// memory may synchronise the device); nullptr if it cannot be allocated.
int *pinned_flag() {
    struct Holder {
        int *p = nullptr;
        bool tried = false;
        ~Holder() {
            if (p) cudaFreeHost(p);
        }
    };
    thread_local Holder h;
    if (!h.tried) {
        h.tried = true;
        if (cudaHostAlloc((void **)&h.p, sizeof(int), cudaHostAllocDefault) != cudaSuccess) {
            h.p = nullptr;
            cudaGetLastError();
        }
    }
    return h.p;
}

// Runs body(stream) -- one batch of iterations -- until the device state says
// done.  The batch is captured once into a CUDA graph on a private stream (the
// legacy default stream cannot be captured) and replayed, so the GPU runs the
// iterations back to back and the host only reads one state word per replay.
// Falls back to plain launches on the caller's stream when capture fails.
template <class Body>
fv_status loop_until_done(const Workspace &w, cudaStream_t st, Body body, SolverState &h) {
    cudaStream_t cs = nullptr;
    cudaEvent_t ev = nullptr;
    cudaGraphExec_t gx = nullptr;
    long long per_replay = 0;
    bool graph_ok = false;
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) == cudaSuccess &&
        cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess) {
        cudaEventRecord(ev, st);
        cudaStreamWaitEvent(cs, ev, 0);
        const unsigned long long c0 = fv_launches_now();
        if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            const fv_status bs = body(cs);
            cudaGraph_t g = nullptr;
            const cudaError_t e = cudaStreamEndCapture(cs, &g);
            if (bs == FV_OK && e == cudaSuccess && g && cudaGraphInstantiate(&gx, g, 0) == cudaSuccess)
                graph_ok = true;
            if (g) cudaGraphDestroy(g);
        }
        per_replay = (long long)(fv_launches_now() - c0);
        fv_note_launches(-per_replay);  // captured, not run
        cudaGetLastError();
    }
    fv_status s = FV_OK;
    int *done_h = pinned_flag();
    cudaEvent_t evd = nullptr;
    if (graph_ok && done_h && cudaEventCreateWithFlags(&evd, cudaEventDisableTiming) == cudaSuccess) {
        // The next replay is queued before the host waits for the previous
        // replay's done flag (copied into pinned memory behind it), so the GPU
        // does not idle while the host reads, nor while its thread is
        // descheduled.  One replay may run after convergence: its kernels see
        // the done flag and return at once, so the results do not change.
        auto replay = [&]() -> fv_status {
            const cudaError_t e = cudaGraphLaunch(gx, cs);
            if (e != cudaSuccess) {
                fv_internal_set_cuda_error(e, "cudaGraphLaunch");
                return FV_ERR_CUDA;
            }
            fv_note_launches(per_replay);
            return FV_OK;
        };
        auto flag_after = [&]() -> fv_status {
            FV_CUDA_TRY(cudaMemcpyAsync(done_h, &w.S->done, sizeof(int), cudaMemcpyDeviceToHost, cs));
            FV_CUDA_TRY(cudaEventRecord(evd, cs));
            return FV_OK;
        };
        s = replay();
        if (s == FV_OK) s = flag_after();
        while (s == FV_OK) {
            s = replay();
            if (s != FV_OK) break;
            const cudaError_t e = cudaEventSynchronize(evd);
            if (e != cudaSuccess) {
                fv_internal_set_cuda_error(e, "cudaEventSynchronize");
                s = FV_ERR_CUDA;
                break;
            }
            if (*(volatile int *)done_h) break;
            s = flag_after();
        }
        if (s == FV_OK) s = read_state(w, h, cs);
        cudaEventRecord(ev, cs);
        cudaStreamWaitEvent(st, ev, 0);
    } else if (graph_ok) {
        while (true) {
            cudaError_t e = cudaGraphLaunch(gx, cs);
            if (e != cudaSuccess) {
                fv_internal_set_cuda_error(e, "cudaGraphLaunch");
                s = FV_ERR_CUDA;
                break;
            }
            fv_note_launches(per_replay);
            s = read_state(w, h, cs);
            if (s != FV_OK || h.done) break;
        }
        cudaEventRecord(ev, cs);
        cudaStreamWaitEvent(st, ev, 0);
    } else {
        while (true) {
            s = body(st);
            if (s != FV_OK) break;
            s = read_state(w, h, st);
            if (s != FV_OK || h.done) break;
        }
    }
    if (evd) cudaEventDestroy(evd);
    if (gx) cudaGraphExecDestroy(gx);
    if (ev) cudaEventDestroy(ev);
    if (cs) cudaStreamDestroy(cs);
    return s;
}

}  // namespace

extern "C" fv_status fv_cg(const fv_csr *A, fv_precond *P, const double *b, double *x, fv_solver_options opt,
                           fv_solver_info *info, void *stream) {
    if (!A || !b || !x || A->nrows != A->ncols || opt.max_iterations < 0) return FV_ERR_INVALID;
    cudaStream_t st = fv_stream(stream);
    const int64_t n = A->nrows;
    const int G = fv_reduce_grid(n, RB);
    Workspace w;
    FV_TRY(ws_alloc(w, n, 4, opt, G, st));
    double *r = w.vec, *z = w.vec + n, *p = w.vec + 2 * n, *ap = w.vec + 3 * n;
    SolverState *S = w.S;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    fv_note_launch(), k_dot_self<<<G, RB, 0, st>>>(n, b, S);
    fv_note_launch(), k_zero_if<<<G, RB, 0, st>>>(n, x, S);
    fv_note_launch(), k_residual<false><<<G, RB, 0, st>>>(n, A->row_ptr, A->cols, A->vals, x, b, r, nullptr, nullptr, S);
    fv_status s = apply_or_copy(P, r, z, n, G, S, st);
    fv_note_launch(), k_cg_init_p<<<G, RB, 0, st>>>(n, r, z, p, S);
    FV_CUDA_TRY(cudaGetLastError());
    SolverState h{};
    const int B = batch_size(n);
    auto body = [&](cudaStream_t q_st) -> fv_status {
        for (int q = 0; q < B; ++q) {
            fv_note_launch(), k_cg_spmv<<<G, RB, 0, q_st>>>(n, A->row_ptr, A->cols, A->vals, p, ap, S);
            fv_note_launch(), k_cg_update<<<G, RB, 0, q_st>>>(n, x, r, p, ap, S);
            FV_TRY(apply_or_copy(P, r, z, n, G, S, q_st));
            fv_note_launch(), k_cg_rz<<<G, RB, 0, q_st>>>(n, r, z, S);
            fv_note_launch(), k_cg_p<<<G, RB, 0, q_st>>>(n, z, p, S);
        }
        FV_CUDA_TRY(cudaGetLastError());
        return FV_OK;
    };
    if (s == FV_OK) s = loop_until_done(w, st, body, h);
    cudaEventRecord(e1, st);
    if (s == FV_OK) s = read_state(w, h, st);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (info) info->device_ms = ms;
    if (s == FV_OK) s = fill_info(false, h, info, P, st);
    cudaFreeAsync(w.S, st);
    return s;
}

extern "C" fv_status fv_bicgstab(const fv_csr *A, fv_precond *P, const double *b, double *x, fv_solver_options opt,
                                 fv_solver_info *info, void *stream) {
    if (!A || !b || !x || A->nrows != A->ncols || opt.max_iterations < 0) return FV_ERR_INVALID;
    cudaStream_t st = fv_stream(stream);
    const int64_t n = A->nrows;
    const int G = fv_reduce_grid(n, RB);
    Workspace w;
    FV_TRY(ws_alloc(w, n, 8, opt, G, st));
    double *r = w.vec, *rh = r + n, *p = rh + n, *y = p + n, *v = y + n, *s_ = v + n, *z = s_ + n, *t = z + n;
    SolverState *S = w.S;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    fv_note_launch(), k_dot_self<<<G, RB, 0, st>>>(n, b, S);
    fv_note_launch(), k_zero_if<<<G, RB, 0, st>>>(n, x, S);
    fv_note_launch(), k_residual<true><<<G, RB, 0, st>>>(n, A->row_ptr, A->cols, A->vals, x, b, r, rh, p, S);
    FV_CUDA_TRY(cudaGetLastError());
    fv_status s = FV_OK;
    SolverState h{};
    const int B = batch_size(n);
    auto body = [&](cudaStream_t q_st) -> fv_status {
        for (int q = 0; q < B; ++q) {
            FV_TRY(apply_or_copy(P, p, y, n, G, S, q_st));
            fv_note_launch(), k_bi_spmv1<<<G, RB, 0, q_st>>>(n, A->row_ptr, A->cols, A->vals, y, v, rh, S);
            fv_note_launch(), k_bi_s<<<G, RB, 0, q_st>>>(n, r, v, s_, S);
            FV_TRY(apply_or_copy(P, s_, z, n, G, S, q_st));
            fv_note_launch(), k_bi_spmv2<<<G, RB, 0, q_st>>>(n, A->row_ptr, A->cols, A->vals, z, t, s_, S);
            fv_note_launch(), k_bi_update<<<G, RB, 0, q_st>>>(n, x, r, y, z, s_, t, rh, S);
            fv_note_launch(), k_bi_p<<<G, RB, 0, q_st>>>(n, r, v, p, rh, S);
        }
        FV_CUDA_TRY(cudaGetLastError());
        return FV_OK;
    };
    s = loop_until_done(w, st, body, h);
    fv_note_launch(), k_bi_finish<<<G, RB, 0, st>>>(n, x, y, S);
    cudaEventRecord(e1, st);
    if (s == FV_OK) s = read_state(w, h, st);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (info) info->device_ms = ms;
    if (s == FV_OK) s = fill_info(true, h, info, P, st);
    cudaFreeAsync(w.S, st);
    return s;
}

static fv_status solve_host(bool bicg, const fv_csr *A, fv_precond *P, const double *b_host, double *x_host,
                            fv_solver_options opt, fv_solver_info *info, void *stream) {
    if (!A || !b_host || !x_host) return FV_ERR_INVALID;
    cudaStream_t st = fv_stream(stream);
    const int64_t n = A->nrows;
    double *buf = nullptr;
    FV_CUDA_TRY(fv_malloc_async(&buf, sizeof(double) * 2 * n, st));
    FV_CUDA_TRY(cudaMemcpyAsync(buf, b_host, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    FV_CUDA_TRY(cudaMemcpyAsync(buf + n, x_host, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    fv_status s = bicg ? fv_bicgstab(A, P, buf, buf + n, opt, info, stream) : fv_cg(A, P, buf, buf + n, opt, info, stream);
    FV_CUDA_TRY(cudaMemcpyAsync(x_host, buf + n, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    cudaFreeAsync(buf, st);
    FV_CUDA_TRY(cudaStreamSynchronize(st));
    return s;
}

extern "C" fv_status fv_cg_host(const fv_csr *A, fv_precond *P, const double *b_host, double *x_host,
                                fv_solver_options opt, fv_solver_info *info, void *stream) {
    return solve_host(false, A, P, b_host, x_host, opt, info, stream);
}
extern "C" fv_status fv_bicgstab_host(const fv_csr *A, fv_precond *P, const double *b_host, double *x_host,
                                      fv_solver_options opt, fv_solver_info *info, void *stream) {
    return solve_host(true, A, P, b_host, x_host, opt, info, stream);
}

// ------------------------------------------------------------------ fv_cg_noalloc
// Allocation-free conjugate gradient.  fv_cg takes its Krylov workspace from
// cudaMallocAsync on every call; this variant takes it from one statically
// sized device array that is created when this file's CUDA module is loaded on
// a device (under lazy module loading, the CUDA 12 default: at the first
// launch from, or symbol lookup in, this module on that device).  It launches
// the same kernels in the same order as fv_cg, so its results are the same bits.
namespace {
constexpr int64_t kNoAllocMaxRows = FV_NOALLOC_MAX_ROWS;
constexpr int64_t kNoAllocMaxHist = FV_NOALLOC_MAX_ITERATIONS + 3;
constexpr size_t kNoAllocState = (sizeof(SolverState) + 255) / 256 * 256;
constexpr size_t kNoAllocPartial = 1184 * 4 * sizeof(double);  // fv_reduce_grid never exceeds 1184 blocks
constexpr size_t kNoAllocBytes =
    kNoAllocState + kNoAllocPartial + kNoAllocMaxHist * sizeof(double) + 4 * kNoAllocMaxRows * sizeof(double);
}  // namespace

// The workspace: solver state, block partials, residual history, r/z/p/Ap.
// In host code this name is only a handle for cudaGetSymbolAddress, never a
// device address.
static __device__ __align__(256) unsigned char g_cg_noalloc_scratch[kNoAllocBytes];

#include <cuda.h>  // CUcontext / CUresult types only; the driver calls are reached through the runtime

#include <mutex>
static std::mutex g_cg_noalloc_mu;
struct NoAllocSlot {
    void *addr = nullptr;
    unsigned long long ctx_id = 0;  // unique id of the context the address belongs to (0: none yet)
};
static NoAllocSlot g_cg_noalloc_slot[256];

// Unique id of the calling thread's current context (cuCtxGetId, unique over
// the process's life), or 0 when the driver does not provide it.
static unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext *);
    using GetId = CUresult (*)(CUcontext, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = (GetCurrent)f;
        f = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (GetId)f;
        cudaGetLastError();
    });
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

// Device address of the scratch array on the current device.  Set-up runs
// once per device, with that device current: cudaGetSymbolAddress, checked.
// The address is kept together with the id of the context it belongs to and
// looked up again when that context has been replaced (cudaDeviceReset, or a
// primary context released and re-created), so a stale address is never used.
static fv_status cg_noalloc_scratch(void **out) {
    int dev = -1;
    FV_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256) return FV_ERR_INVALID;
    const unsigned long long ctx = current_context_id();  // 0 while no context is current on this thread
    std::lock_guard<std::mutex> lock(g_cg_noalloc_mu);
    NoAllocSlot &slot = g_cg_noalloc_slot[dev];
    if (!slot.addr || ctx == 0 || slot.ctx_id != ctx) {
        void *p = nullptr;
        FV_CUDA_TRY(cudaGetSymbolAddress(&p, g_cg_noalloc_scratch));  // makes the primary context current
        slot.addr = p;
        slot.ctx_id = current_context_id();
    }
    *out = slot.addr;
    return FV_OK;
}

extern "C" fv_status fv_cg_noalloc(const fv_csr *A, fv_precond *P, const double *b, double *x,
                                   fv_solver_options opt, fv_solver_info *info, void *stream) {
    if (!A || !b || !x || A->nrows != A->ncols || opt.max_iterations < 0) return FV_ERR_INVALID;
    const int64_t n = A->nrows;
    if (n > kNoAllocMaxRows) {
        fv_internal_set_error_text("fv_cg_noalloc: the matrix has more than FV_NOALLOC_MAX_ROWS rows");
        return FV_ERR_INVALID;
    }
    if (opt.max_iterations > FV_NOALLOC_MAX_ITERATIONS) {
        fv_internal_set_error_text("fv_cg_noalloc: max_iterations exceeds FV_NOALLOC_MAX_ITERATIONS");
        return FV_ERR_INVALID;
    }
    cudaStream_t st = fv_stream(stream);
    const int G = fv_reduce_grid(n, RB);
    void *base = nullptr;
    FV_TRY(cg_noalloc_scratch(&base));
    unsigned char *mem = (unsigned char *)base;
    Workspace w;
    w.S = (SolverState *)mem;
    double *partial = (double *)(mem + kNoAllocState);
    double *hist = partial + 1184 * 4;
    w.vec = hist + kNoAllocMaxHist;
    w.nvec = 4;
    // The array keeps whatever the previous call left: the state (including
    // the reduction ticket and the done flag) is rewritten in full here, and
    // r, z, p, Ap, the partials and the history are written before they are read.
    SolverState hs{};
    hs.tol = opt.absolute_tolerance;
    hs.rtol = opt.relative_tolerance;
    hs.max_it = opt.max_iterations;
    hs.error = 1.0;
    hs.partial = partial;
    hs.hist = hist;
    FV_CUDA_TRY(cudaMemcpyAsync(w.S, &hs, sizeof(SolverState), cudaMemcpyHostToDevice, st));
    double *r = w.vec, *z = w.vec + n, *p = w.vec + 2 * n, *ap = w.vec + 3 * n;
    SolverState *S = w.S;
    fv_note_launch(), k_dot_self<<<G, RB, 0, st>>>(n, b, S);
    fv_note_launch(), k_zero_if<<<G, RB, 0, st>>>(n, x, S);
    fv_note_launch(), k_residual<false><<<G, RB, 0, st>>>(n, A->row_ptr, A->cols, A->vals, x, b, r, nullptr, nullptr, S);
    fv_status s = apply_or_copy(P, r, z, n, G, S, st);
    fv_note_launch(), k_cg_init_p<<<G, RB, 0, st>>>(n, r, z, p, S);
    FV_CUDA_TRY(cudaGetLastError());
    SolverState h{};
    const int B = batch_size(n);
    for (int64_t it = 0; s == FV_OK;) {
        for (int q = 0; q < B && s == FV_OK; ++q, ++it) {
            fv_note_launch(), k_cg_spmv<<<G, RB, 0, st>>>(n, A->row_ptr, A->cols, A->vals, p, ap, S);
            fv_note_launch(), k_cg_update<<<G, RB, 0, st>>>(n, x, r, p, ap, S);
            s = apply_or_copy(P, r, z, n, G, S, st);
            fv_note_launch(), k_cg_rz<<<G, RB, 0, st>>>(n, r, z, S);
            fv_note_launch(), k_cg_p<<<G, RB, 0, st>>>(n, z, p, S);
        }
        FV_CUDA_TRY(cudaGetLastError());
        if (s != FV_OK) break;
        FV_TRY(read_state(w, h, st));
        if (h.done) break;
    }
    if (s == FV_OK) s = read_state(w, h, st);
    if (info) info->device_ms = 0.0;
    if (s == FV_OK) s = fill_info(false, h, info, P, st);
    return s;
}
