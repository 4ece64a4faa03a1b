// One rank of a problem split over several GPUs: the reference's MPI design.
//
// Reference: the crate runs one MPI rank per partition of the mesh
// (core/mesh/decompose.rs).  Each rank owns a set of rows; its local matrix
// has columns for its own cells followed by ghost columns for the cells of
// other ranks that share a face with its cells (linalg/dmatrix.rs:38-50 over
// the local cell_to_cell).  Before every SpMV the ghost values are refreshed
// with Communicator::collect (core/communicator.rs:226-266); every dot
// product is a local sum followed by Communicator::reduce_add
// (core/communicator.rs:282-290); the preconditioners factorise only the
// square block of owned columns (DistributedMatrix::square_block,
// linalg/dmatrix.rs:214-229; incomplete_cholesky.rs:151,
// incomplete_lower_upper.rs:202), i.e. block Jacobi across ranks.  The Krylov
// loops are conjugate_gradient.rs:12-111 and bi_conjugate_gradient_stab.rs:13-178.
//
// Design: the two communication steps are callbacks (fv_comm), so the same
// library serves an NCCL process group (one process per GPU, buffers on the
// device, operations ordered on the solve's stream), an MPI communicator, or
// an in-process emulation of several ranks.  The scalar recurrences run on the
// host as in the reference: after each reduce_add the few global sums come back
// through one small pinned copy.  Vector work is fused: every update kernel
// also produces the block partial sums of the dots that follow it, so an
// iteration is SpMV + sweeps + 3 (CG) or 4 (BiCGStab) fused vector kernels.
// Local sums use a fixed grid per row count, so a rank's partial sums are
// reproducible; ranks add them in rank order when the communicator does.
#include <cmath>
#include <vector>

#include <cub/device/device_scan.cuh>

#include "fv_internal.cuh"

struct fv_precond;
fv_status fv_precond_apply_dev(fv_precond *P, const double *r, double *z, cudaStream_t st, const int *skip,
                               const fv_row_skip *rskip);
fv_status fv_precond_check_error(fv_precond *P, cudaStream_t st);
int64_t fv_precond_rows(const fv_precond *P);

struct fv_dist {
    const fv_csr *A = nullptr;  // n_own rows, n_own + n_ghost columns
    int64_t n_own = 0, n_ghost = 0, n_send = 0;
    int32_t *send_idx = nullptr;  // owned rows to send, in the plan's order
    double *send = nullptr;       // packed send buffer
    fv_comm comm{};
    double *part = nullptr;  // block partial sums
    double *sums = nullptr;  // reduced sums (device)
    double *host = nullptr;  // pinned copy of sums
};

namespace {

constexpr int DB = 256;
constexpr int kMaxDots = 3;

int dot_grid(int64_t n) { return fv_reduce_grid(n, DB); }

__global__ void __launch_bounds__(DB) kd_gather(int64_t m, const int32_t *__restrict__ idx,
                                                const double *__restrict__ x, double *__restrict__ out) {
    for (int64_t k = (int64_t)blockIdx.x * DB + threadIdx.x; k < m; k += (int64_t)gridDim.x * DB) out[k] = x[idx[k]];
}

// Block partials of K dot products; partial[q * gridDim.x + block].
template <int K>
__device__ __forceinline__ void write_partials(double (&v)[K], double *part) {
    __shared__ double sm[K * 32];
    fv_block_reduce<K>(v, sm);
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < K; ++q) part[q * gridDim.x + blockIdx.x] = v[q];
}

// Sum the G partials of each of K dots in block order (one warp per dot,
// fixed lane assignment and shuffle tree): out[q].
__global__ void kd_finish(int K, int G, const double *__restrict__ part, double *__restrict__ out) {
    const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (q >= K) return;
    double s = 0.0;
    for (int b = lane; b < G; b += 32) s += part[q * G + b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) out[q] = s;
}

// Up to three dots of vector pairs.
struct Pairs {
    const double *a[kMaxDots];
    const double *b[kMaxDots];
};

template <int K>
__global__ void __launch_bounds__(DB) kd_dots(int64_t n, Pairs p, double *__restrict__ part) {
    double v[K];
#pragma unroll
    for (int q = 0; q < K; ++q) v[q] = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * DB + threadIdx.x; i < n; i += (int64_t)gridDim.x * DB)
#pragma unroll
        for (int q = 0; q < K; ++q) v[q] += p.a[q][i] * p.b[q][i];
    write_partials<K>(v, part);
}

// r = -(A x - b) (the reference's r = A x; r -= b; r *= -1); optional copy to rh; dots r.r
__global__ void __launch_bounds__(DB) kd_residual(int64_t n, const double *__restrict__ ax,
                                                  const double *__restrict__ b, double *__restrict__ r,
                                                  double *__restrict__ rh, double *__restrict__ part) {
    double v[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * DB + threadIdx.x; i < n; i += (int64_t)gridDim.x * DB) {
        double t = ax[i];
        t -= b[i];
        t *= -1.0;
        r[i] = t;
        if (rh) rh[i] = t;
        v[0] += t * t;
    }
    write_partials<1>(v, part);
}

// CG: x += p a; r -= ap a; dot r.r
__global__ void __launch_bounds__(DB) kd_cg_xr(int64_t n, double alpha, const double *__restrict__ p,
                                               const double *__restrict__ ap, double *__restrict__ x,
                                               double *__restrict__ r, double *__restrict__ part) {
    double v[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * DB + threadIdx.x; i < n; i += (int64_t)gridDim.x * DB) {
        x[i] += p[i] * alpha;
        const double ri = r[i] - ap[i] * alpha;
        r[i] = ri;
        v[0] += ri * ri;
    }
    write_partials<1>(v, part);
}

// CG: p = z + p b
__global__ void __launch_bounds__(DB) kd_cg_p(int64_t n, double beta, const double *__restrict__ z,
                                              double *__restrict__ p) {
    for (int64_t i = (int64_t)blockIdx.x * DB + threadIdx.x; i < n; i += (int64_t)gridDim.x * DB)
        p[i] = z[i] + p[i] * beta;
}

// BiCGStab: h = x + y a; s = r - v a; dot s.s
__global__ void __launch_bounds__(DB) kd_bi_hs(int64_t n, double alpha, const double *__restrict__ x,
                                               const double *__restrict__ y, const double *__restrict__ r,
                                               const double *__restrict__ vv, double *__restrict__ h,
                                               double *__restrict__ s, double *__restrict__ part) {
    double v[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * DB + threadIdx.x; i < n; i += (int64_t)gridDim.x * DB) {
        h[i] = x[i] + y[i] * alpha;
        const double si = r[i] - vv[i] * alpha;
        s[i] = si;
        v[0] += si * si;
    }
    write_partials<1>(v, part);
}

// BiCGStab: x = h + z w; r = s - t w; dots r.r, rh.r
__global__ void __launch_bounds__(DB) kd_bi_xr(int64_t n, double omega, const double *__restrict__ h,
                                               const double *__restrict__ z, const double *__restrict__ s,
                                               const double *__restrict__ t, const double *__restrict__ rh,
                                               double *__restrict__ x, double *__restrict__ r,
                                               double *__restrict__ part) {
    double v[2] = {0.0, 0.0};
    for (int64_t i = (int64_t)blockIdx.x * DB + threadIdx.x; i < n; i += (int64_t)gridDim.x * DB) {
        x[i] = h[i] + z[i] * omega;
        const double ri = s[i] - t[i] * omega;
        r[i] = ri;
        v[0] += ri * ri;
        v[1] += rh[i] * ri;
    }
    write_partials<2>(v, part);
}

// BiCGStab: p = r + (p - v w) b, or the restart rh = r, p = r (with dot rh.r)
__global__ void __launch_bounds__(DB) kd_bi_p(int64_t n, double beta, double omega, int restart,
                                              const double *__restrict__ r, const double *__restrict__ vv,
                                              double *__restrict__ p, double *__restrict__ rh,
                                              double *__restrict__ part) {
    double v[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * DB + threadIdx.x; i < n; i += (int64_t)gridDim.x * DB) {
        const double ri = r[i];
        if (restart) {
            rh[i] = ri;
            p[i] = ri;
            v[0] += ri * ri;
        } else {
            p[i] = ri + (p[i] - vv[i] * omega) * beta;
        }
    }
    write_partials<1>(v, part);
}

__global__ void __launch_bounds__(DB) kd_square_count(int64_t n, const int32_t *__restrict__ ptr,
                                                      const int32_t *__restrict__ col, int32_t *__restrict__ cnt) {
    for (int64_t i = (int64_t)blockIdx.x * DB + threadIdx.x; i < n; i += (int64_t)gridDim.x * DB) {
        int c = 0;
        for (int k = ptr[i]; k < ptr[i + 1]; ++k) c += col[k] < n ? 1 : 0;
        cnt[i] = c;
    }
}

__global__ void __launch_bounds__(DB) kd_square_fill(int64_t n, const int32_t *__restrict__ ptr,
                                                     const int32_t *__restrict__ col,
                                                     const double *__restrict__ val,
                                                     const int32_t *__restrict__ optr, int32_t *__restrict__ ocol,
                                                     double *__restrict__ oval) {
    for (int64_t i = (int64_t)blockIdx.x * DB + threadIdx.x; i < n; i += (int64_t)gridDim.x * DB) {
        int o = optr[i];
        for (int k = ptr[i]; k < ptr[i + 1]; ++k)
            if (col[k] < n) {
                ocol[o] = col[k];
                oval[o++] = val[k];
            }
    }
}

int vec_grid(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + DB - 1) / DB, 148 * 8)); }

// Sums of the last fused kernel: finish the partials, reduce over ranks, copy to the host.
fv_status reduce(fv_dist *D, int K, int G, cudaStream_t st, double *out) {
    fv_note_launch(), kd_finish<<<1, 32 * K, 0, st>>>(K, G, D->part, D->sums);
    FV_CUDA_TRY(cudaGetLastError());
    if (D->comm.reduce_add && D->comm.reduce_add(D->comm.ctx, D->sums, K, (void *)st) != 0) {
        fv_internal_set_error_text("fv_comm.reduce_add failed");
        return FV_ERR_COMM;
    }
    FV_CUDA_TRY(cudaMemcpyAsync(D->host, D->sums, sizeof(double) * K, cudaMemcpyDeviceToHost, st));
    FV_CUDA_TRY(cudaStreamSynchronize(st));
    for (int q = 0; q < K; ++q) out[q] = D->host[q];
    return FV_OK;
}

fv_status dots(fv_dist *D, int K, const Pairs &p, cudaStream_t st, double *out) {
    const int64_t n = D->n_own;
    const int G = dot_grid(n);
    if (K == 1)
        fv_note_launch(), kd_dots<1><<<G, DB, 0, st>>>(n, p, D->part);
    else if (K == 2)
        fv_note_launch(), kd_dots<2><<<G, DB, 0, st>>>(n, p, D->part);
    else
        fv_note_launch(), kd_dots<3><<<G, DB, 0, st>>>(n, p, D->part);
    FV_CUDA_TRY(cudaGetLastError());
    return reduce(D, K, G, st, out);
}

// y = A x after refreshing the ghost tail x[n_own ..] from the other ranks.
fv_status dist_spmv(fv_dist *D, double *x, double *y, cudaStream_t st) {
    if (D->n_send > 0) {
        fv_note_launch(), kd_gather<<<vec_grid(D->n_send), DB, 0, st>>>(D->n_send, D->send_idx, x, D->send);
        FV_CUDA_TRY(cudaGetLastError());
    }
    if (D->comm.collect && D->comm.collect(D->comm.ctx, D->send, x + D->n_own, (void *)st) != 0) {
        fv_internal_set_error_text("fv_comm.collect failed");
        return FV_ERR_COMM;
    }
    return fv_spmv(D->A, x, y, (void *)st);
}

fv_status precond(fv_precond *P, const double *r, double *z, int64_t n, cudaStream_t st) {
    if (!P) {
        FV_CUDA_TRY(cudaMemcpyAsync(z, r, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        return FV_OK;
    }
    return fv_precond_apply_dev(P, r, z, st, nullptr, nullptr);
}

struct Vecs {
    double *base = nullptr;
    fv_status alloc(int64_t total, cudaStream_t st) {
        FV_CUDA_TRY(fv_malloc_async(&base, sizeof(double) * (total ? total : 1), st));
        FV_CUDA_TRY(cudaMemsetAsync(base, 0, sizeof(double) * (total ? total : 1), st));
        return FV_OK;
    }
    void release(cudaStream_t st) {
        if (base) cudaFreeAsync(base, st);
        base = nullptr;
    }
};

void record(fv_solver_info *info, int64_t k, double e) {
    if (info->history && k < info->history_cap) {
        info->history[k] = e;
        info->history_len = k + 1;
    }
}

fv_status check_args(fv_dist *D, fv_precond *P, const double *b, const double *x, fv_solver_info *info) {
    if (!D || !b || !x || !info) return FV_ERR_INVALID;
    if (P && fv_precond_rows(P) != D->n_own) return FV_ERR_INVALID;
    return FV_OK;
}

}  // namespace

extern "C" fv_status fv_csr_square_block(const fv_csr *A, void *stream, fv_csr **out) {
    if (!A || !out) return FV_ERR_INVALID;
    *out = nullptr;
    cudaStream_t st = fv_stream(stream);
    const int64_t n = A->nrows;
    fv_csr *s = new fv_csr();
    s->nrows = s->ncols = n;
    int32_t *cnt = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    fv_status rc = FV_OK;
    cudaError_t e = cudaMalloc(&s->row_ptr, sizeof(int32_t) * (n + 1));
    if (e == cudaSuccess) e = fv_malloc_async(&cnt, sizeof(int32_t) * (n + 1), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (n + 1), st);
    if (e == cudaSuccess && n > 0) {
        fv_note_launch(), kd_square_count<<<vec_grid(n), DB, 0, st>>>(n, A->row_ptr, A->cols, cnt);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cnt, s->row_ptr, (int)(n + 1), st);
    if (e == cudaSuccess) e = fv_malloc_async(&tmp, tmp_bytes ? tmp_bytes : 1, st);
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, cnt, s->row_ptr, (int)(n + 1), st);
    int32_t nnz = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&nnz, s->row_ptr + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) {
        s->nnz = nnz;
        e = cudaMalloc(&s->cols, sizeof(int32_t) * (nnz ? nnz : 1));
        if (e == cudaSuccess) e = cudaMalloc(&s->vals, sizeof(double) * (nnz ? nnz : 1));
    }
    if (e == cudaSuccess && n > 0) {
        fv_note_launch(), kd_square_fill<<<vec_grid(n), DB, 0, st>>>(n, A->row_ptr, A->cols, A->vals, s->row_ptr,
                                                                      s->cols, s->vals);
        e = cudaGetLastError();
    }
    if (cnt) cudaFreeAsync(cnt, st);
    if (tmp) cudaFreeAsync(tmp, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        fv_internal_set_cuda_error(e, "fv_csr_square_block");
        fv_csr_destroy(s);
        rc = e == cudaErrorMemoryAllocation ? FV_ERR_ALLOC : FV_ERR_CUDA;
        return rc;
    }
    *out = s;
    return FV_OK;
}

extern "C" fv_status fv_dist_create(const fv_csr *A, int64_t n_ghost, const int32_t *send_idx, int64_t n_send,
                                    const fv_comm *comm, fv_dist **out) {
    if (!A || !out || n_ghost < 0 || n_send < 0 || (n_send > 0 && !send_idx)) return FV_ERR_INVALID;
    if (A->ncols != A->nrows + n_ghost) return FV_ERR_INVALID;
    *out = nullptr;
    for (int64_t k = 0; k < n_send; ++k)
        if (send_idx[k] < 0 || send_idx[k] >= A->nrows) return FV_ERR_INVALID;
    fv_dist *D = new fv_dist();
    D->A = A;
    D->n_own = A->nrows;
    D->n_ghost = n_ghost;
    D->n_send = n_send;
    if (comm) D->comm = *comm;
    const int G = dot_grid(D->n_own);
    cudaError_t e = cudaMalloc(&D->send_idx, sizeof(int32_t) * (n_send ? n_send : 1));
    if (e == cudaSuccess) e = cudaMalloc(&D->send, sizeof(double) * (n_send ? n_send : 1));
    if (e == cudaSuccess) e = cudaMalloc(&D->part, sizeof(double) * kMaxDots * G);
    if (e == cudaSuccess) e = cudaMalloc(&D->sums, sizeof(double) * kMaxDots);
    if (e == cudaSuccess) e = cudaMallocHost(&D->host, sizeof(double) * kMaxDots);
    if (e == cudaSuccess && n_send)
        e = cudaMemcpy(D->send_idx, send_idx, sizeof(int32_t) * n_send, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        fv_internal_set_cuda_error(e, "fv_dist_create");
        fv_dist_destroy(D);
        return e == cudaErrorMemoryAllocation ? FV_ERR_ALLOC : FV_ERR_CUDA;
    }
    *out = D;
    return FV_OK;
}

extern "C" fv_status fv_dist_destroy(fv_dist *D) {
    if (!D) return FV_OK;
    cudaFree(D->send_idx);
    cudaFree(D->send);
    cudaFree(D->part);
    cudaFree(D->sums);
    if (D->host) cudaFreeHost(D->host);
    delete D;
    return FV_OK;
}

extern "C" fv_status fv_dist_spmv(fv_dist *D, double *x, double *y, void *stream) {
    if (!D || !x || !y || x == y) return FV_ERR_INVALID;
    return dist_spmv(D, x, y, fv_stream(stream));
}

extern "C" fv_status fv_dist_dot(fv_dist *D, const double *x, const double *y, double *result, void *stream) {
    if (!D || !x || !y || !result) return FV_ERR_INVALID;
    Pairs p{};
    p.a[0] = x;
    p.b[0] = y;
    return dots(D, 1, p, fv_stream(stream), result);
}

// conjugate_gradient.rs:12-111 on this rank's rows.
extern "C" fv_status fv_dist_cg(fv_dist *D, fv_precond *P, const double *b, double *x, fv_solver_options opt,
                                fv_solver_info *info, void *stream) {
    FV_TRY(check_args(D, P, b, x, info));
    cudaStream_t st = fv_stream(stream);
    const int64_t n = D->n_own, ng = D->n_ghost;
    info->iterations = 0;
    info->restarts = 0;
    info->history_len = 0;
    info->status = FV_OK;
    cudaEvent_t e0, e1;
    FV_CUDA_TRY(cudaEventCreate(&e0));
    FV_CUDA_TRY(cudaEventCreate(&e1));
    FV_CUDA_TRY(cudaEventRecord(e0, st));
    Vecs W;
    fv_status rc = W.alloc(5 * n + 2 * ng, st);
    double *r = W.base, *z = r + n, *ap = z + n, *p = ap + n, *xg = p + n + ng;  // p, xg carry ghost tails
    double sum[kMaxDots];
    double bnorm = 0.0, init = 0.0, error = 1.0;
    int64_t iter = 0;
    auto body = [&]() -> fv_status {
        Pairs pb{};
        pb.a[0] = b;
        pb.b[0] = b;
        FV_TRY(dots(D, 1, pb, st, sum));
        bnorm = std::sqrt(sum[0]);
        if (bnorm < 1e-14) {  // conjugate_gradient.rs:31-36
            FV_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(double) * n, st));
            init = error = bnorm;
            return FV_OK;
        }
        FV_CUDA_TRY(cudaMemcpyAsync(xg, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        FV_TRY(dist_spmv(D, xg, ap, st));
        const int G = dot_grid(n);
        fv_note_launch(), kd_residual<<<G, DB, 0, st>>>(n, ap, b, r, nullptr, D->part);
        FV_CUDA_TRY(cudaGetLastError());
        FV_TRY(reduce(D, 1, G, st, sum));
        init = std::sqrt(sum[0]) / bnorm;
        FV_TRY(precond(P, r, z, n, st));
        FV_CUDA_TRY(cudaMemcpyAsync(p, z, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        error = 1.0;
        while (error > opt.absolute_tolerance) {
            if (iter > opt.max_iterations) break;
            FV_TRY(dist_spmv(D, p, ap, st));
            Pairs q{};
            q.a[0] = r;
            q.b[0] = z;
            q.a[1] = p;
            q.b[1] = ap;
            FV_TRY(dots(D, 2, q, st, sum));
            const double rz = sum[0], alpha = rz / sum[1];
            fv_note_launch(), kd_cg_xr<<<G, DB, 0, st>>>(n, alpha, p, ap, x, r, D->part);
            FV_CUDA_TRY(cudaGetLastError());
            FV_TRY(reduce(D, 1, G, st, sum));
            error = std::sqrt(sum[0]) / bnorm;
            if (!std::isfinite(alpha) || !std::isfinite(error)) {
                info->status = FV_ERR_BREAKDOWN;
                record(info, iter, error);
                iter++;
                break;
            }
            if (error < opt.absolute_tolerance || error / init < opt.relative_tolerance) {
                record(info, iter, error);
                iter++;
                break;
            }
            FV_TRY(precond(P, r, z, n, st));
            Pairs q2{};
            q2.a[0] = r;
            q2.b[0] = z;
            FV_TRY(dots(D, 1, q2, st, sum));
            const double beta = sum[0] / rz;
            fv_note_launch(), kd_cg_p<<<vec_grid(n), DB, 0, st>>>(n, beta, z, p);
            FV_CUDA_TRY(cudaGetLastError());
            record(info, iter, error);
            iter++;
        }
        if (P) FV_TRY(fv_precond_check_error(P, st));
        return FV_OK;
    };
    if (rc == FV_OK) rc = body();
    W.release(st);
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    info->device_ms = ms;
    info->iterations = iter;
    info->initial_residual = init;
    info->final_residual = error;
    if (rc != FV_OK && info->status == FV_OK) info->status = rc;
    return rc;
}

// bi_conjugate_gradient_stab.rs:13-178 on this rank's rows (right preconditioned,
// restart when |rho| <= 1e-15 |b|, loop guard divided by |b| twice).
extern "C" fv_status fv_dist_bicgstab(fv_dist *D, fv_precond *P, const double *b, double *x,
                                      fv_solver_options opt, fv_solver_info *info, void *stream) {
    FV_TRY(check_args(D, P, b, x, info));
    cudaStream_t st = fv_stream(stream);
    const int64_t n = D->n_own, ng = D->n_ghost;
    info->iterations = 0;
    info->restarts = 0;
    info->history_len = 0;
    info->status = FV_OK;
    cudaEvent_t e0, e1;
    FV_CUDA_TRY(cudaEventCreate(&e0));
    FV_CUDA_TRY(cudaEventCreate(&e1));
    FV_CUDA_TRY(cudaEventRecord(e0, st));
    Vecs W;
    fv_status rc = W.alloc(10 * n + 3 * ng, st);
    // y, z and xg carry ghost tails (they are SpMV inputs)
    double *p = W.base, *r = p + n, *rh = r + n, *vv = rh + n, *h = vv + n, *s = h + n, *t = s + n;
    double *y = t + n, *z = y + n + ng, *xg = z + n + ng;
    double sum[kMaxDots];
    double bnorm = 0.0, init = 0.0, error = 1.0;
    int64_t iter = 0;
    auto body = [&]() -> fv_status {
        Pairs pb{};
        pb.a[0] = b;
        pb.b[0] = b;
        FV_TRY(dots(D, 1, pb, st, sum));
        bnorm = std::sqrt(sum[0]);
        if (bnorm < 1e-14) {
            FV_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(double) * n, st));
            init = error = bnorm;
            return FV_OK;
        }
        FV_CUDA_TRY(cudaMemcpyAsync(xg, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        FV_TRY(dist_spmv(D, xg, vv, st));
        const int G = dot_grid(n);
        fv_note_launch(), kd_residual<<<G, DB, 0, st>>>(n, vv, b, r, rh, D->part);
        FV_CUDA_TRY(cudaGetLastError());
        FV_TRY(reduce(D, 1, G, st, sum));
        init = std::sqrt(sum[0]) / bnorm;
        error = 1.0;
        if (init < opt.absolute_tolerance) {
            error = init;
            return FV_OK;
        }
        FV_CUDA_TRY(cudaMemcpyAsync(p, r, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        Pairs q0{};
        q0.a[0] = rh;
        q0.b[0] = r;
        FV_TRY(dots(D, 1, q0, st, sum));
        double rho = sum[0];
        while (error > opt.absolute_tolerance) {
            if (iter > opt.max_iterations) break;
            FV_TRY(precond(P, p, y, n, st));
            FV_TRY(dist_spmv(D, y, vv, st));
            Pairs q1{};
            q1.a[0] = rh;
            q1.b[0] = vv;
            FV_TRY(dots(D, 1, q1, st, sum));
            const double alpha = rho / sum[0];
            fv_note_launch(), kd_bi_hs<<<G, DB, 0, st>>>(n, alpha, x, y, r, vv, h, s, D->part);
            FV_CUDA_TRY(cudaGetLastError());
            FV_TRY(reduce(D, 1, G, st, sum));
            const double sn = std::sqrt(sum[0]) / bnorm;
            if (!std::isfinite(sn)) {
                info->status = FV_ERR_BREAKDOWN;
                error = sn;
                record(info, iter, error);
                iter++;
                break;
            }
            if (sn < opt.absolute_tolerance || sn / init < opt.relative_tolerance) {
                error = sn;
                FV_CUDA_TRY(cudaMemcpyAsync(x, h, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
                record(info, iter, error);
                iter++;
                break;
            }
            FV_TRY(precond(P, s, z, n, st));
            FV_TRY(dist_spmv(D, z, t, st));
            Pairs q2{};
            q2.a[0] = t;
            q2.b[0] = s;
            q2.a[1] = t;
            q2.b[1] = t;
            FV_TRY(dots(D, 2, q2, st, sum));
            const double omega = sum[0] / sum[1];
            fv_note_launch(), kd_bi_xr<<<G, DB, 0, st>>>(n, omega, h, z, s, t, rh, x, r, D->part);
            FV_CUDA_TRY(cudaGetLastError());
            FV_TRY(reduce(D, 2, G, st, sum));
            const double rn = std::sqrt(sum[0]) / bnorm;
            if (!std::isfinite(rn)) {
                info->status = FV_ERR_BREAKDOWN;
                error = rn;
                record(info, iter, error);
                iter++;
                break;
            }
            if (rn < opt.absolute_tolerance || rn / init < opt.relative_tolerance) {
                error = rn;
                record(info, iter, error);
                iter++;
                break;
            }
            const double rho_new = sum[1];
            const double beta = (rho_new / rho) * (alpha / omega);
            rho = rho_new;
            const int restart = std::fabs(rho) > 1e-15 * bnorm ? 0 : 1;
            fv_note_launch(), kd_bi_p<<<G, DB, 0, st>>>(n, beta, omega, restart, r, vv, p, rh, D->part);
            FV_CUDA_TRY(cudaGetLastError());
            if (restart) {
                FV_TRY(reduce(D, 1, G, st, sum));
                rho = sum[0];
                info->restarts++;
            }
            error = rn / bnorm;
            record(info, iter, error);
            iter++;
        }
        if (P) FV_TRY(fv_precond_check_error(P, st));
        return FV_OK;
    };
    if (rc == FV_OK) rc = body();
    W.release(st);
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    info->device_ms = ms;
    info->iterations = iter;
    info->initial_residual = init;
    info->final_residual = error;
    if (rc != FV_OK && info->status == FV_OK) info->status = rc;
    return rc;
}
