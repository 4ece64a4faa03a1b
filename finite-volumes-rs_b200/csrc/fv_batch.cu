// Batched Krylov solves over many independent problems packed as one
// block-diagonal system.
//
// Reference: conjugate_gradient (src/linalg/solvers/conjugate_gradient.rs:12-111)
// applied to every problem of the batch, with IC(0) (incomplete_cholesky.rs)
// as preconditioner.
//
// Design.  Independent meshes are concatenated into one mesh whose CSR matrix
// is block diagonal (one block per problem); assembly, the pattern, IC(0) /
// ILU(0) and the sweeps of that union are exactly the per-problem ones, and the
// level-ordered sync-free sweeps run all problems' levels together, so a
// batch fills the GPU where one small problem cannot.  The Krylov scalars are
// per problem: rows are cut into problem-aligned tiles of `tile` rows; each
// tile writes its partial sums to its own slot, and the last tile of a problem
// to finish (a per-problem ticket) reduces that problem's tiles in order and
// runs the problem's scalar update.  A problem's result therefore depends on
// nothing but its own rows: it is the same alone and in any mix.
//
// Precision modes:
//   FV_BATCH_FP64  -- CG in FP64 with the reference's semantics per problem.
//   FV_BATCH_MIXED -- FP64 iterative refinement: r = b - A x in FP64, an
//                     FP32 CG (FP32 SpMV, FP32 IC(0) sweeps, FP32 sums) solves
//                     A d = r to a relative tolerance, x += d in FP64, until
//                     |b - A x| / |b| <= the outer tolerance.
#include <algorithm>
#include <cmath>
#include <vector>

#include "fv_internal.cuh"

struct fv_precond;
fv_status fv_precond_apply_dev(fv_precond *P, const double *r, double *z, cudaStream_t st, const int *skip,
                               const fv_row_skip *rskip);
fv_status fv_precond_apply_dev_f32(fv_precond *P, const float *r, float *z, cudaStream_t st, const int *skip,
                                   const fv_row_skip *rskip);
fv_status fv_precond_make_f32(fv_precond *P, cudaStream_t st);
fv_status fv_precond_check_error(fv_precond *P, cudaStream_t st);

namespace {

struct BProb {
    // inner CG (reference semantics on its right-hand side)
    double bnorm, init_res, error, rz, alpha, beta, tol, rtol;
    int64_t iter, max_it;
    int done, breakdown;
    unsigned ticket;
    int pad;
    // BiCGStab
    double rho, omega;
    int restart, restarts, finish_h, pad2;
    // mixed precision: reliable updates of the FP32 residual from the FP64 one
    double last_rn;   // FP32 residual estimate (relative) at the last replacement
    int replace, n_replace;
    double prev_res64;      // FP64 residual at the previous replacement
    int strikes, stagnated; // replacements without progress; gave up on FP32
    int kry_restart, p_reset;
    int64_t iter_at_rep;    // iteration of the last replacement
    int forced, pad3;       // the pending replacement was forced by the period
    // outer refinement (FP64)
    double bnorm64, res64;
    // stepwise runs: 1 once the retired problem's pending correction is applied
    int fin, pad4;
};

struct BGlobal {
    int active;       // problems whose inner solve is running
    int all_done;     // 1 when active == 0 (skips the sweeps)
    int pad[2];
};

constexpr int TB = 256;  // threads per tile block
constexpr int kMaxTileSums = 3;  // largest NV of finish_tile (kbm_rep2); sizes the partial-sum buffer

template <int NV, class Epi>
__device__ __forceinline__ void finish_tile(double (&v)[NV], int p, int64_t t, const int32_t *__restrict__ ptile,
                                            double *partial, BProb *S, BGlobal *G, Epi epi) {
    static_assert(NV <= kMaxTileSums, "the partial-sum buffer holds kMaxTileSums values per tile");
    __shared__ double sm[NV * 32];
    __shared__ bool last;
    fv_block_reduce<NV>(v, sm);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) partial[t * NV + q] = v[q];
        __threadfence();
        const unsigned nt = (unsigned)(ptile[p + 1] - ptile[p]);
        last = (atomicAdd(&S[p].ticket, 1u) == nt - 1);
    }
    __syncthreads();
    if (!last) return;
    double tot[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) tot[q] = 0.0;
    for (int64_t u = ptile[p] + threadIdx.x; u < ptile[p + 1]; u += blockDim.x)
#pragma unroll
        for (int q = 0; q < NV; ++q) tot[q] += __ldcg(&partial[u * NV + q]);
    fv_block_reduce<NV>(tot, sm);
    if (threadIdx.x == 0) {
        S[p].ticket = 0;
        epi(S[p], tot, G);
    }
    __syncthreads();
}

__device__ __forceinline__ void retire(BProb &s, BGlobal *G) {
    s.done = 1;
    if (atomicSub(&G->active, 1) == 1) G->all_done = 1;
}

// Row dot y_i = sum_k a_k x_col(k), left to right from 0 (dmatrix.rs:138-145).
template <typename T>
__device__ __forceinline__ T row_dot_t(const int32_t *__restrict__ ptr, const int32_t *__restrict__ col,
                                       const T *__restrict__ val, const T *__restrict__ x, int64_t i) {
    T s = T(0);
    const int k1 = ptr[i + 1];
    for (int k = ptr[i]; k < k1; ++k) s += val[k] * __ldg(&x[col[k]]);
    return s;
}

struct Tiles {
    int64_t ntiles;
    const int32_t *prob, *row0, *row1, *ptile;
};

// Mixed precision: the FP32 Krylov run asks for a residual replacement when
// its residual estimate fell by `delta` since the last one or reached the
// target; the replacement recomputes the true residual in FP64.
struct MixedCfg {
    int on;
    double outer_tol, delta;
};
// A replacement is also forced after this many FP32 iterations without one,
// so an FP32 run whose own residual estimate stalls is still checked in FP64.
constexpr int64_t kForcedReplacePeriod = 128;

__device__ __forceinline__ void mixed_trigger(BProb &s, double est, const MixedCfg &mx) {
    if (est <= mx.outer_tol || est <= mx.delta * s.last_rn || !isfinite(est)) {
        s.replace = 1;
        s.forced = 0;
    } else if (s.iter - s.iter_at_rep >= kForcedReplacePeriod) {
        s.replace = 1;
        s.forced = 1;
    }
}

// ---- inner CG kernels (T = double or float)
// r given, d = 0: bnorm = |r|, init_res = 1 (conjugate_gradient.rs:71-94 with x0 = 0)
template <typename T>
__global__ void __launch_bounds__(TB) kb_init(Tiles tl, const T *__restrict__ r, T *__restrict__ d,
                                              double *partial, BProb *S, BGlobal *G) {
    for (int64_t t = blockIdx.x; t < tl.ntiles; t += gridDim.x) {
        const int p = tl.prob[t];
        if (S[p].done) continue;
        T acc = T(0);  // per-thread sums in the inner precision; tile and problem sums in FP64
        for (int64_t i = tl.row0[t] + threadIdx.x; i < tl.row1[t]; i += blockDim.x) {
            const T ri = r[i];
            d[i] = T(0);
            acc += ri * ri;
        }
        double v[1] = {(double)acc};
        finish_tile<1>(v, p, t, tl.ptile, partial, S, G, [] __device__(BProb & s, const double *tot, BGlobal *G) {
            s.bnorm = sqrt(tot[0]);
            s.iter = 0;
            s.error = 1.0;
            s.last_rn = 1.0;
            s.replace = 0;
            s.p_reset = 0;
            s.kry_restart = 0;
            s.iter_at_rep = 0;
            if (s.bnorm < 1e-14) {
                s.init_res = s.bnorm;
                s.error = s.bnorm;
                retire(s, G);
                return;
            }
            s.init_res = sqrt(tot[0]) / s.bnorm;
            if (!(s.error > s.tol) || s.iter > s.max_it) retire(s, G);
        });
    }
}

// p = z; rz = r.z
template <typename T>
__global__ void __launch_bounds__(TB) kb_init_p(Tiles tl, const T *__restrict__ r, const T *__restrict__ z,
                                                T *__restrict__ pv, double *partial, BProb *S, BGlobal *G) {
    for (int64_t t = blockIdx.x; t < tl.ntiles; t += gridDim.x) {
        const int p = tl.prob[t];
        if (S[p].done) continue;
        T acc = T(0);
        for (int64_t i = tl.row0[t] + threadIdx.x; i < tl.row1[t]; i += blockDim.x) {
            const T zi = z[i];
            pv[i] = zi;
            acc += r[i] * zi;
        }
        double v[1] = {(double)acc};
        finish_tile<1>(v, p, t, tl.ptile, partial, S, G,
                       [] __device__(BProb & s, const double *tot, BGlobal *) { s.rz = tot[0]; });
    }
}

// ap = A p; alpha = rz / p.ap
template <typename T>
__global__ void __launch_bounds__(TB) kb_spmv(Tiles tl, const int32_t *__restrict__ ptr,
                                              const int32_t *__restrict__ col, const T *__restrict__ val,
                                              const T *__restrict__ pv, T *__restrict__ ap, double *partial, BProb *S,
                                              BGlobal *G) {
    for (int64_t t = blockIdx.x; t < tl.ntiles; t += gridDim.x) {
        const int p = tl.prob[t];
        if (S[p].done) continue;
        T acc = T(0);
        for (int64_t i = tl.row0[t] + threadIdx.x; i < tl.row1[t]; i += blockDim.x) {
            const T y = row_dot_t(ptr, col, val, pv, i);
            ap[i] = y;
            acc += pv[i] * y;
        }
        double v[1] = {(double)acc};
        finish_tile<1>(v, p, t, tl.ptile, partial, S, G, [] __device__(BProb & s, const double *tot, BGlobal *) {
            s.alpha = s.rz / tot[0];
        });
    }
}

// d += alpha p; r -= alpha ap; convergence test
template <typename T>
__global__ void __launch_bounds__(TB) kb_update(Tiles tl, T *__restrict__ d, T *__restrict__ r,
                                                const T *__restrict__ pv, const T *__restrict__ ap, double *partial,
                                                BProb *S, BGlobal *G, MixedCfg mx) {
    for (int64_t t = blockIdx.x; t < tl.ntiles; t += gridDim.x) {
        const int p = tl.prob[t];
        if (S[p].done) continue;
        const T alpha = (T)S[p].alpha;
        T acc = T(0);
        for (int64_t i = tl.row0[t] + threadIdx.x; i < tl.row1[t]; i += blockDim.x) {
            d[i] += pv[i] * alpha;
            const T ri = r[i] - ap[i] * alpha;
            r[i] = ri;
            acc += ri * ri;
        }
        double v[1] = {(double)acc};
        finish_tile<1>(v, p, t, tl.ptile, partial, S, G, [mx] __device__(BProb & s, const double *tot, BGlobal *G) {
            s.error = sqrt(tot[0]) / s.bnorm;
            if (!isfinite(s.alpha)) s.breakdown = 1;
            if (mx.on) {
                mixed_trigger(s, s.error, mx);
            } else if ((s.error < s.tol) || (s.error / s.init_res < s.rtol)) {
                s.iter += 1;
                retire(s, G);
            }
        });
    }
}

// beta = r.z_new / r.z; loop guard
template <typename T>
__global__ void __launch_bounds__(TB) kb_rz(Tiles tl, const T *__restrict__ r, const T *__restrict__ z,
                                            double *partial, BProb *S, BGlobal *G) {
    for (int64_t t = blockIdx.x; t < tl.ntiles; t += gridDim.x) {
        const int p = tl.prob[t];
        if (S[p].done) continue;
        T acc = T(0);
        for (int64_t i = tl.row0[t] + threadIdx.x; i < tl.row1[t]; i += blockDim.x) acc += r[i] * z[i];
        double v[1] = {(double)acc};
        finish_tile<1>(v, p, t, tl.ptile, partial, S, G, [] __device__(BProb & s, const double *tot, BGlobal *G) {
            s.p_reset = s.kry_restart;  // a fresh Krylov start: p = z
            s.kry_restart = 0;
            s.beta = s.p_reset ? 0.0 : tot[0] / s.rz;
            s.rz = tot[0];
            s.iter += 1;
            if (!(s.error > s.tol) || s.iter > s.max_it) retire(s, G);
        });
    }
}

template <typename T>
__global__ void __launch_bounds__(TB) kb_p(Tiles tl, const T *__restrict__ z, T *__restrict__ pv, const BProb *S) {
    for (int64_t t = blockIdx.x; t < tl.ntiles; t += gridDim.x) {
        const int p = tl.prob[t];
        if (S[p].done) continue;
        const T beta = (T)S[p].beta;
        if (S[p].p_reset) {
            for (int64_t i = tl.row0[t] + threadIdx.x; i < tl.row1[t]; i += blockDim.x) pv[i] = z[i];
        } else {
            for (int64_t i = tl.row0[t] + threadIdx.x; i < tl.row1[t]; i += blockDim.x) pv[i] = z[i] + pv[i] * beta;
        }
    }
}

// ---- inner BiCGStab kernels (bi_conjugate_gradient_stab.rs:13-178 per problem, x0 = 0)
// r given, d = 0, rh = r, p = r; bnorm = |r|, init_res = 1, rho = rh.r
template <typename T>
__global__ void __launch_bounds__(TB) kbb_init(Tiles tl, const T *__restrict__ r, T *__restrict__ d,
                                               T *__restrict__ rh, T *__restrict__ pv, double *partial, BProb *S,
                                               BGlobal *G) {
    for (int64_t t = blockIdx.x; t < tl.ntiles; t += gridDim.x) {
        const int p = tl.prob[t];
        if (S[p].done) continue;
        T acc = T(0);
        for (int64_t i = tl.row0[t] + threadIdx.x; i < tl.row1[t]; i += blockDim.x) {
            const T ri = r[i];
            d[i] = T(0);
            rh[i] = ri;
            pv[i] = ri;
            acc += ri * ri;
        }
        double v[1] = {(double)acc};
        finish_tile<1>(v, p, t, tl.ptile, partial, S, G, [] __device__(BProb & s, const double *tot, BGlobal *G) {
            s.bnorm = sqrt(tot[0]);
            s.iter = 0;
            s.restart = 0;
            s.finish_h = 0;
            s.last_rn = 1.0;
            s.replace = 0;
            s.iter_at_rep = 0;
            s.p_reset = 0;
            s.kry_restart = 0;
            s.iter_at_rep = 0;
            if (s.bnorm < 1e-14) {
                s.init_res = s.bnorm;
                s.error = s.bnorm;
                retire(s, G);
                return;
            }
            s.init_res = sqrt(tot[0]) / s.bnorm;
            if (s.init_res < s.tol) {
                s.error = s.init_res;
                retire(s, G);
                return;
            }
            s.rho = tot[0];
            s.error = 1.0;
            if (!(s.error > s.tol) || s.iter > s.max_it) retire(s, G);
        });
    }
}

// v = A y; alpha = rho / rh.v
template <typename T>
__global__ void __launch_bounds__(TB) kbb_spmv1(Tiles tl, const int32_t *__restrict__ ptr,
                                                const int32_t *__restrict__ col, const T *__restrict__ val,
                                                const T *__restrict__ y, T *__restrict__ vv, const T *__restrict__ rh,
                                                double *partial, BProb *S, BGlobal *G) {
    for (int64_t t = blockIdx.x; t < tl.ntiles; t += gridDim.x) {
        const int p = tl.prob[t];
        if (S[p].done) continue;
        T acc = T(0);
        for (int64_t i = tl.row0[t] + threadIdx.x; i < tl.row1[t]; i += blockDim.x) {
            const T vi = row_dot_t(ptr, col, val, y, i);
            vv[i] = vi;
            acc += rh[i] * vi;
        }
        double v[1] = {(double)acc};
        finish_tile<1>(v, p, t, tl.ptile, partial, S, G,
                       [] __device__(BProb & s, const double *tot, BGlobal *) { s.alpha = s.rho / tot[0]; });
    }
}

// s = r - v alpha; |s| test.  h = d + y alpha is not stored: it is recomputed,
// with the same rounding, where it is used (kbb_update, kbb_finish).
template <typename T>
__global__ void __launch_bounds__(TB) kbb_s(Tiles tl, const T *__restrict__ r, const T *__restrict__ vv,
                                            T *__restrict__ sv, double *partial, BProb *S, BGlobal *G, MixedCfg mx) {
    for (int64_t t = blockIdx.x; t < tl.ntiles; t += gridDim.x) {
        const int p = tl.prob[t];
        if (S[p].done) continue;
        const T alpha = (T)S[p].alpha;
        T acc = T(0);
        for (int64_t i = tl.row0[t] + threadIdx.x; i < tl.row1[t]; i += blockDim.x) {
            const T si = r[i] - vv[i] * alpha;
            sv[i] = si;
            acc += si * si;
        }
        double v[1] = {(double)acc};
        finish_tile<1>(v, p, t, tl.ptile, partial, S, G, [mx] __device__(BProb & s, const double *tot, BGlobal *G) {
            const double sn = sqrt(tot[0]) / s.bnorm;
            if (!isfinite(s.alpha)) s.breakdown = 1;
            if (mx.on) return;  // mixed: convergence is decided on the FP64 residual only
            if ((sn < s.tol) || (sn / s.init_res < s.rtol)) {
                s.error = sn;
                s.finish_h = 1;
                s.iter += 1;
                retire(s, G);
            }
        });
    }
}

// t = A z; omega = t.s / t.t
template <typename T>
__global__ void __launch_bounds__(TB) kbb_spmv2(Tiles tl, const int32_t *__restrict__ ptr,
                                                const int32_t *__restrict__ col, const T *__restrict__ val,
                                                const T *__restrict__ z, T *__restrict__ tv, const T *__restrict__ sv,
                                                double *partial, BProb *S, BGlobal *G) {
    for (int64_t t = blockIdx.x; t < tl.ntiles; t += gridDim.x) {
        const int p = tl.prob[t];
        if (S[p].done) continue;
        T a0 = T(0), a1 = T(0);
        for (int64_t i = tl.row0[t] + threadIdx.x; i < tl.row1[t]; i += blockDim.x) {
            const T ti = row_dot_t(ptr, col, val, z, i);
            tv[i] = ti;
            a0 += ti * sv[i];
            a1 += ti * ti;
        }
        double v[2] = {(double)a0, (double)a1};
        finish_tile<2>(v, p, t, tl.ptile, partial, S, G,
                       [] __device__(BProb & s, const double *tot, BGlobal *) { s.omega = tot[0] / tot[1]; });
    }
}

// d = h + z omega with h = d + y alpha; r = s - t omega; |r| test; beta and the restart (:122-171)
template <typename T>
__global__ void __launch_bounds__(TB) kbb_update(Tiles tl, T *__restrict__ d, T *__restrict__ r,
                                                 const T *__restrict__ y, const T *__restrict__ z,
                                                 const T *__restrict__ sv, const T *__restrict__ tv,
                                                 const T *__restrict__ rh, double *partial, BProb *S, BGlobal *G,
                                                 MixedCfg mx) {
    for (int64_t t = blockIdx.x; t < tl.ntiles; t += gridDim.x) {
        const int p = tl.prob[t];
        if (S[p].done) continue;
        const T alpha = (T)S[p].alpha, omega = (T)S[p].omega;
        T a0 = T(0), a1 = T(0);
        for (int64_t i = tl.row0[t] + threadIdx.x; i < tl.row1[t]; i += blockDim.x) {
            const T hi = d[i] + y[i] * alpha;
            d[i] = hi + z[i] * omega;
            const T ri = sv[i] - tv[i] * omega;
            r[i] = ri;
            a0 += ri * ri;
            a1 += rh[i] * ri;
        }
        double v[2] = {(double)a0, (double)a1};
        finish_tile<2>(v, p, t, tl.ptile, partial, S, G, [mx] __device__(BProb & s, const double *tot, BGlobal *G) {
            const double rn = sqrt(tot[0]) / s.bnorm;
            if (!mx.on && ((rn < s.tol) || (rn / s.init_res < s.rtol))) {
                s.error = rn;
                s.iter += 1;
                retire(s, G);
                return;
            }
            if (mx.on) {
                mixed_trigger(s, rn, mx);
                if (s.replace) {
                    s.error = rn;  // beta and the restart decision wait for the replaced residual
                    s.iter += 1;
                    return;
                }
            }
            const double rho_new = tot[1];
            s.beta = (rho_new / s.rho) * (s.alpha / s.omega);
            s.rho = rho_new;
            if (fabs(s.rho) > (1e-15 * s.bnorm)) {
                s.restart = 0;
            } else {
                s.restart = 1;
                s.restarts += 1;
                s.rho = tot[0];
            }
            if (!isfinite(s.omega) || !isfinite(s.beta)) s.breakdown = 1;
            s.error = rn / s.bnorm;
            s.iter += 1;
            if (!(s.error > s.tol) || s.iter > s.max_it) retire(s, G);
        });
    }
}

template <typename T>
__global__ void __launch_bounds__(TB) kbb_p(Tiles tl, const T *__restrict__ r, const T *__restrict__ vv,
                                            T *__restrict__ pv, T *__restrict__ rh, const BProb *S) {
    for (int64_t t = blockIdx.x; t < tl.ntiles; t += gridDim.x) {
        const int p = tl.prob[t];
        if (S[p].done) continue;
        const T omega = (T)S[p].omega, beta = (T)S[p].beta;
        if (S[p].restart) {
            for (int64_t i = tl.row0[t] + threadIdx.x; i < tl.row1[t]; i += blockDim.x) {
                rh[i] = r[i];
                pv[i] = r[i];
            }
        } else {
            for (int64_t i = tl.row0[t] + threadIdx.x; i < tl.row1[t]; i += blockDim.x)
                pv[i] = r[i] + (pv[i] - vv[i] * omega) * beta;
        }
    }
}

// d = h = d + y alpha for problems whose |s| test ended the solve
template <typename T>
__global__ void kbb_finish(Tiles tl, T *__restrict__ d, const T *__restrict__ y, BProb *S) {
    for (int64_t t = blockIdx.x; t < tl.ntiles; t += gridDim.x) {
        const int p = tl.prob[t];
        if (S[p].finish_h != 1) continue;
        const T alpha = (T)S[p].alpha;
        for (int64_t i = tl.row0[t] + threadIdx.x; i < tl.row1[t]; i += blockDim.x) d[i] = d[i] + y[i] * alpha;
    }
}

// ---- mixed precision with reliable updates
// x = 0, r32 = (float) b, |b| in FP64
__global__ void __launch_bounds__(TB) kbm_init(Tiles tl, const double *__restrict__ b, double *__restrict__ x,
                                               float *__restrict__ r32, double *partial, BProb *S, BGlobal *G) {
    for (int64_t t = blockIdx.x; t < tl.ntiles; t += gridDim.x) {
        const int p = tl.prob[t];
        if (S[p].done) continue;  // a problem carried over from another batch keeps its state
        double v[1] = {0.0};
        for (int64_t i = tl.row0[t] + threadIdx.x; i < tl.row1[t]; i += blockDim.x) {
            const double bi = b[i];
            x[i] = 0.0;
            r32[i] = (float)bi;
            v[0] += bi * bi;
        }
        finish_tile<1>(v, p, t, tl.ptile, partial, S, G, [] __device__(BProb & s, const double *tot, BGlobal *) {
            s.bnorm64 = sqrt(tot[0]);
            s.res64 = 1.0;
            s.n_replace = 0;
        });
    }
}

// x64 += d; d = 0 for the problems that asked for a replacement
template <typename T>
__global__ void __launch_bounds__(TB) kbm_rep1(Tiles tl, double *__restrict__ x, T *__restrict__ d, const BProb *S) {
    for (int64_t t = blockIdx.x; t < tl.ntiles; t += gridDim.x) {
        const int p = tl.prob[t];
        if (S[p].done || !S[p].replace) continue;
        for (int64_t i = tl.row0[t] + threadIdx.x; i < tl.row1[t]; i += blockDim.x) {
            x[i] += (double)d[i];
            d[i] = T(0);
        }
    }
}

// r64 = b - A x64 (FP64), r = (T) r64; the FP64 norm decides convergence.
// BiCGStab also finishes the deferred beta / restart with the replaced r.
template <typename T, bool BICG>
__global__ void __launch_bounds__(TB) kbm_rep2(Tiles tl, const int32_t *__restrict__ ptr,
                                               const int32_t *__restrict__ col, const double *__restrict__ val,
                                               const double *__restrict__ x, const double *__restrict__ b,
                                               T *__restrict__ r, const T *__restrict__ rh, double *partial, BProb *S,
                                               BGlobal *G, double outer_tol) {
    for (int64_t t = blockIdx.x; t < tl.ntiles; t += gridDim.x) {
        const int p = tl.prob[t];
        if (S[p].done || !S[p].replace) continue;
        double a0 = 0.0;
        T a1 = T(0), a2 = T(0);
        for (int64_t i = tl.row0[t] + threadIdx.x; i < tl.row1[t]; i += blockDim.x) {
            const double ri = b[i] - row_dot_t(ptr, col, val, x, i);
            const T rt = (T)ri;
            r[i] = rt;
            a0 += ri * ri;
            if (BICG) {
                a1 += rh[i] * rt;
                a2 += rt * rt;
            }
        }
        double v[3] = {a0, (double)a1, (double)a2};
        finish_tile<3>(v, p, t, tl.ptile, partial, S, G, [outer_tol] __device__(BProb & s, const double *tot,
                                                                                BGlobal *G) {
            s.res64 = s.bnorm64 > 0.0 ? sqrt(tot[0]) / s.bnorm64 : 0.0;
            s.replace = 0;
            s.n_replace += 1;
            if (s.res64 <= outer_tol) {
                retire(s, G);
                return;
            }
            // No progress since the previous replacement (or a non-finite
            // residual): the FP32 run cannot resolve this problem.  The first
            // time, restart the Krylov space from the true residual; the
            // second time, give up on FP32 (an FP64 pass finishes it).
            // Progress expected: a replacement triggered by a 1/delta drop of the
            // FP32 estimate must at least halve the FP64 residual; a forced one
            // (128 iterations without a trigger) must cut it by 10%.
            // A progress-triggered replacement also fails when the true
            // residual is far above the FP32 estimate that triggered it: the
            // FP32 recursion has decoupled from the FP64 residual.
            bool fresh = false;
            const double need = s.forced ? 0.9 : 0.5;
            const bool gap = !s.forced && s.res64 * s.bnorm64 > 100.0 * s.error * s.bnorm;
            s.iter_at_rep = s.iter;
            if (!isfinite(s.res64) || gap || (s.n_replace > 1 && s.res64 > need * s.prev_res64)) {
                s.strikes += 1;
                if (s.strikes >= 2 || !isfinite(s.res64)) {
                    s.stagnated = 1;
                    retire(s, G);
                    return;
                }
                fresh = true;
            }
            s.prev_res64 = s.res64;
            s.last_rn = sqrt(tot[0]) / s.bnorm;  // the replaced residual in the units of the FP32 estimate
            if (!BICG) {
                if (fresh) s.kry_restart = 1;
            } else {
                const double rho_new = tot[1];
                s.beta = (rho_new / s.rho) * (s.alpha / s.omega);
                s.rho = rho_new;
                if (!fresh && fabs(s.rho) > (1e-15 * s.bnorm)) {
                    s.restart = 0;
                } else {
                    s.restart = 1;
                    s.restarts += 1;
                    s.rho = tot[2];
                }
                if (!isfinite(s.omega) || !isfinite(s.beta)) s.breakdown = 1;
                if (s.iter > s.max_it) retire(s, G);
            }
        });
    }
}

// x64 += d for every problem: the correction pending when a problem stopped on max_iterations
template <typename T>
__global__ void kbm_flush(Tiles tl, double *__restrict__ x, T *__restrict__ d) {
    for (int64_t t = blockIdx.x; t < tl.ntiles; t += gridDim.x)
        for (int64_t i = tl.row0[t] + threadIdx.x; i < tl.row1[t]; i += blockDim.x) {
            x[i] += (double)d[i];
            d[i] = T(0);
        }
}

// ---- stepwise runs
// The result of every problem that retired since the last call: d = h = d +
// y alpha where BiCGStab's |s| test ended the solve (y non-null), x64 += d
// (mixed, x64 non-null).  Per problem these are the operations kbb_finish and
// kbm_flush apply at the end of a whole-batch solve.
template <typename T>
__global__ void kb_finalize(Tiles tl, T *__restrict__ d, const T *__restrict__ y, double *__restrict__ x64,
                            const BProb *S) {
    for (int64_t t = blockIdx.x; t < tl.ntiles; t += gridDim.x) {
        const int p = tl.prob[t];
        if (!S[p].done || S[p].fin) continue;
        const bool take_h = y && S[p].finish_h == 1;
        const T alpha = (T)S[p].alpha;
        for (int64_t i = tl.row0[t] + threadIdx.x; i < tl.row1[t]; i += blockDim.x) {
            if (take_h) d[i] = d[i] + y[i] * alpha;
            if (x64) {
                x64[i] += (double)d[i];
                d[i] = T(0);
            }
        }
    }
}

__global__ void kb_mark_fin(int np, BProb *S) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x)
        if (S[p].done) S[p].fin = 1;
}

// Copy the rows of the problems carried over from another batch:
// seg[3 s .. 3 s + 2] = (source row, destination row, rows) of segment s.
template <typename T>
__global__ void kb_adopt(const int64_t *__restrict__ seg, int nseg, const T *__restrict__ src, T *__restrict__ dst) {
    for (int s = blockIdx.y; s < nseg; s += gridDim.y) {
        const int64_t a = seg[3 * s], b = seg[3 * s + 1], len = seg[3 * s + 2];
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x)
            dst[b + i] = src[a + i];
    }
}

// The carried-over problems, held as done while the new problems were
// initialised, run again.
__global__ void kb_resume(const int32_t *__restrict__ list, int cnt, BProb *S, BGlobal *G) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += gridDim.x * blockDim.x) S[list[k]].done = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0 && cnt > 0) {
        atomicAdd(&G->active, cnt);
        G->all_done = 0;
    }
}

__global__ void k_to_f32b(int64_t n, const double *__restrict__ a, float *__restrict__ b) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

}  // namespace

struct fv_batch {
    const fv_csr *A = nullptr;
    int np = 0;
    int64_t n = 0;
    int tile = 0;
    int64_t ntiles = 0;
    std::vector<int64_t> off;
    int32_t *tile_prob = nullptr, *tile_row0 = nullptr, *tile_row1 = nullptr, *ptile = nullptr;
    int32_t *row_prob = nullptr;  // problem of every row (sweeps skip converged problems)
    BProb *S = nullptr;
    BGlobal *G = nullptr;
    double *partial = nullptr;
    float *a32 = nullptr;
    void *vec = nullptr;
    size_t vec_bytes = 0;
    void *vec64 = nullptr;  // FP64 fallback workspace (allocated on first need)
    size_t vec64_bytes = 0;
    // the run begun by fv_batch_begin (or a whole-batch solve)
    bool run = false, bicg = false, mixed = false;
    fv_precond *P = nullptr;
    const double *b = nullptr;
    double *x = nullptr;
    fv_batch_options opt{};
    int64_t launched = 0;        // iterations enqueued for the whole batch
    std::vector<BProb> hs;       // the problems' state as of the end of the last begin / advance
    int64_t *seg = nullptr;      // carried-over segments (kb_adopt)
    int32_t *resume = nullptr;   // carried-over problems (kb_resume)
};

extern "C" fv_status fv_batch_destroy(fv_batch *B) {
    if (!B) return FV_OK;
    cudaFree(B->tile_prob);
    cudaFree(B->row_prob);
    cudaFree(B->tile_row0);
    cudaFree(B->tile_row1);
    cudaFree(B->ptile);
    cudaFree(B->S);
    cudaFree(B->G);
    cudaFree(B->partial);
    cudaFree(B->a32);
    cudaFree(B->vec);
    cudaFree(B->vec64);
    cudaFree(B->seg);
    cudaFree(B->resume);
    delete B;
    return FV_OK;
}

static fv_status batch_create_impl(const fv_csr *A, int32_t n_problems, const int64_t *row_offsets,
                                   int32_t tile_rows, void *stream, fv_batch **out) {
    if (!A || !out || n_problems <= 0 || !row_offsets || A->nrows != A->ncols) return FV_ERR_INVALID;
    if (row_offsets[0] != 0 || row_offsets[n_problems] != A->nrows) return FV_ERR_INVALID;
    if (tile_rows <= 0) tile_rows = 1024;
    if (tile_rows % 32) return FV_ERR_INVALID;
    *out = nullptr;
    cudaStream_t st = fv_stream(stream);
    fv_batch *B = new fv_batch();
    B->A = A;
    B->np = n_problems;
    B->n = A->nrows;
    B->tile = tile_rows;
    B->off.assign(row_offsets, row_offsets + n_problems + 1);
    std::vector<int32_t> tp, r0, r1, pt(n_problems + 1);
    for (int p = 0; p < n_problems; ++p) {
        pt[p] = (int32_t)tp.size();
        if (row_offsets[p + 1] < row_offsets[p]) {
            delete B;
            return FV_ERR_INVALID;
        }
        for (int64_t a = row_offsets[p]; a < row_offsets[p + 1]; a += tile_rows) {
            tp.push_back(p);
            r0.push_back((int32_t)a);
            r1.push_back((int32_t)std::min<int64_t>(a + tile_rows, row_offsets[p + 1]));
        }
        if (row_offsets[p + 1] == row_offsets[p]) {  // empty problem: one empty tile keeps the tickets simple
            tp.push_back(p);
            r0.push_back((int32_t)row_offsets[p]);
            r1.push_back((int32_t)row_offsets[p]);
        }
    }
    pt[n_problems] = (int32_t)tp.size();
    B->ntiles = (int64_t)tp.size();
    std::vector<int32_t> rp((size_t)B->n);
    for (int p = 0; p < n_problems; ++p)
        for (int64_t i = row_offsets[p]; i < row_offsets[p + 1]; ++i) rp[i] = p;
    cudaError_t e = cudaSuccess;
    auto up = [&](int32_t **d, const std::vector<int32_t> &h) {
        if (e != cudaSuccess) return;
        e = cudaMalloc(d, sizeof(int32_t) * h.size());
        if (e == cudaSuccess) e = cudaMemcpyAsync(*d, h.data(), sizeof(int32_t) * h.size(), cudaMemcpyHostToDevice, st);
    };
    up(&B->tile_prob, tp);
    up(&B->tile_row0, r0);
    up(&B->tile_row1, r1);
    up(&B->ptile, pt);
    up(&B->row_prob, rp);
    if (e == cudaSuccess) e = cudaMalloc(&B->S, sizeof(BProb) * n_problems);
    if (e == cudaSuccess) e = cudaMalloc(&B->G, sizeof(BGlobal));
    if (e == cudaSuccess) e = cudaMalloc(&B->partial, sizeof(double) * B->ntiles * kMaxTileSums);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        fv_internal_set_cuda_error(e, "fv_batch_create");
        fv_batch_destroy(B);
        return e == cudaErrorMemoryAllocation ? FV_ERR_ALLOC : FV_ERR_CUDA;
    }
    *out = B;
    return FV_OK;
}

extern "C" fv_status fv_batch_create(const fv_csr *A, int32_t n_problems, const int64_t *row_offsets,
                                     int32_t tile_rows, void *stream, fv_batch **out) {
    return fv_host_guard([&] { return batch_create_impl(A, n_problems, row_offsets, tile_rows, stream, out); });
}

namespace {

template <typename T>
struct InnerVecs {
    T *r, *z, *p, *ap, *d;       // CG: residual, M^-1 r, direction, A p, solution
    T *rh, *y, *v, *s, *t;       // BiCGStab (p, r, z, d shared)
};

fv_row_skip row_skip(fv_batch *B);

template <typename T>
fv_status precond(fv_batch *B, fv_precond *P, const T *r, T *z, cudaStream_t st, const int *skip) {
    const fv_row_skip rs = row_skip(B);
    if constexpr (sizeof(T) == 8)
        return fv_precond_apply_dev(P, (const double *)r, (double *)z, st, skip, &rs);
    else
        return fv_precond_apply_dev_f32(P, (const float *)r, (float *)z, st, skip, &rs);
}

fv_status wait_all_done(fv_batch *B, cudaStream_t st, bool &done);

// Mixed mode adds the reliable-update step after the x/r update of every
// iteration (x64 and b64 are the FP64 solution and right-hand side).
struct MixedArgs {
    MixedCfg cfg;
    double *x64;
    const double *b64;
};

constexpr int kGroupCG = 8;    // CG iterations enqueued between two host checks
constexpr int kGroupBiCG = 4;  // BiCGStab iterations enqueued between two host checks

// The start of an inner solve for the problems not done: CG (r given; d = 0,
// z = M^-1 r, p = z) or BiCGStab (r given; d = 0, rh = p = r).
template <typename T>
fv_status inner_start(bool bicg, fv_batch *B, fv_precond *P, InnerVecs<T> v, int G, const Tiles &tl,
                      cudaStream_t st) {
    const int *skip = &B->G->all_done;
    if (!bicg) {
        fv_note_launch(), kb_init<T><<<G, TB, 0, st>>>(tl, v.r, v.d, B->partial, B->S, B->G);
        FV_TRY(precond<T>(B, P, v.r, v.z, st, skip));
        fv_note_launch(), kb_init_p<T><<<G, TB, 0, st>>>(tl, v.r, v.z, v.p, B->partial, B->S, B->G);
    } else {
        fv_note_launch(), kbb_init<T><<<G, TB, 0, st>>>(tl, v.r, v.d, v.rh, v.p, B->partial, B->S, B->G);
    }
    FV_CUDA_TRY(cudaGetLastError());
    return FV_OK;
}

// One group of iterations for the problems not done.  Between two groups
// every problem is at an iteration boundary: CG's state is (d, r, p, rz),
// BiCGStab's (d, r, rh, p, rho, alpha, omega), plus x64 in mixed mode.
template <typename T>
fv_status inner_group(bool bicg, fv_batch *B, fv_precond *P, const T *vals, InnerVecs<T> v, int G, const Tiles &tl,
                      cudaStream_t st, int64_t &launched_iters, const MixedArgs &mx) {
    const fv_csr *A = B->A;
    const int *skip = &B->G->all_done;
    if (!bicg) {
        for (int q = 0; q < kGroupCG; ++q) {
            fv_note_launch(), kb_spmv<T><<<G, TB, 0, st>>>(tl, A->row_ptr, A->cols, vals, v.p, v.ap, B->partial, B->S,
                                                          B->G);
            fv_note_launch(), kb_update<T><<<G, TB, 0, st>>>(tl, v.d, v.r, v.p, v.ap, B->partial, B->S, B->G, mx.cfg);
            if (mx.cfg.on) {
                fv_note_launch(), kbm_rep1<T><<<G, TB, 0, st>>>(tl, mx.x64, v.d, B->S);
                fv_note_launch(), kbm_rep2<T, false><<<G, TB, 0, st>>>(tl, A->row_ptr, A->cols, A->vals, mx.x64,
                                                                      mx.b64, v.r, v.rh, B->partial, B->S, B->G,
                                                                      mx.cfg.outer_tol);
            }
            FV_TRY(precond<T>(B, P, v.r, v.z, st, skip));
            fv_note_launch(), kb_rz<T><<<G, TB, 0, st>>>(tl, v.r, v.z, B->partial, B->S, B->G);
            fv_note_launch(), kb_p<T><<<G, TB, 0, st>>>(tl, v.z, v.p, B->S);
            ++launched_iters;
        }
    } else {
        for (int q = 0; q < kGroupBiCG; ++q) {
            FV_TRY(precond<T>(B, P, v.p, v.y, st, skip));
            fv_note_launch(), kbb_spmv1<T><<<G, TB, 0, st>>>(tl, A->row_ptr, A->cols, vals, v.y, v.v, v.rh,
                                                            B->partial, B->S, B->G);
            fv_note_launch(), kbb_s<T><<<G, TB, 0, st>>>(tl, v.r, v.v, v.s, B->partial, B->S, B->G, mx.cfg);
            FV_TRY(precond<T>(B, P, v.s, v.z, st, skip));
            fv_note_launch(), kbb_spmv2<T><<<G, TB, 0, st>>>(tl, A->row_ptr, A->cols, vals, v.z, v.t, v.s,
                                                            B->partial, B->S, B->G);
            fv_note_launch(), kbb_update<T><<<G, TB, 0, st>>>(tl, v.d, v.r, v.y, v.z, v.s, v.t, v.rh, B->partial,
                                                             B->S, B->G, mx.cfg);
            if (mx.cfg.on) {
                fv_note_launch(), kbm_rep1<T><<<G, TB, 0, st>>>(tl, mx.x64, v.d, B->S);
                fv_note_launch(), kbm_rep2<T, true><<<G, TB, 0, st>>>(tl, A->row_ptr, A->cols, A->vals, mx.x64,
                                                                     mx.b64, v.r, v.rh, B->partial, B->S, B->G,
                                                                     mx.cfg.outer_tol);
            }
            fv_note_launch(), kbb_p<T><<<G, TB, 0, st>>>(tl, v.r, v.v, v.p, v.rh, B->S);
            ++launched_iters;
        }
    }
    FV_CUDA_TRY(cudaGetLastError());
    return FV_OK;
}

// A whole inner solve of the problems not done (the FP64 pass over the
// problems a mixed run could not finish).
template <typename T>
fv_status inner_solve(bool bicg, fv_batch *B, fv_precond *P, const T *vals, InnerVecs<T> v, int G, const Tiles &tl,
                      cudaStream_t st, int64_t &launched_iters, const MixedArgs &mx) {
    FV_TRY(inner_start<T>(bicg, B, P, v, G, tl, st));
    for (bool done = false; !done;) {
        FV_TRY(inner_group<T>(bicg, B, P, vals, v, G, tl, st, launched_iters, mx));
        FV_TRY(wait_all_done(B, st, done));
    }
    if (bicg) fv_note_launch(), kbb_finish<T><<<G, TB, 0, st>>>(tl, v.d, v.y, B->S);
    if (mx.cfg.on) fv_note_launch(), kbm_flush<T><<<G, TB, 0, st>>>(tl, mx.x64, v.d);
    FV_CUDA_TRY(cudaGetLastError());
    return FV_OK;
}

fv_row_skip row_skip(fv_batch *B) {
    static_assert(sizeof(BProb) % sizeof(int) == 0, "BProb stride");
    return fv_row_skip{B->row_prob, &B->S[0].done, (int)(sizeof(BProb) / sizeof(int))};
}

fv_status wait_all_done(fv_batch *B, cudaStream_t st, bool &done) {
    FV_CUDA_TRY(cudaGetLastError());
    BGlobal h{};
    FV_CUDA_TRY(cudaMemcpyAsync(&h, B->G, sizeof(BGlobal), cudaMemcpyDeviceToHost, st));
    FV_CUDA_TRY(cudaStreamSynchronize(st));
    done = h.all_done != 0;
    return FV_OK;
}

template <typename T>
InnerVecs<T> carve(void *mem, int64_t n, T *d) {
    T *a = (T *)mem;
    InnerVecs<T> v;
    v.r = a;
    v.z = a + n;
    v.p = a + 2 * n;
    v.ap = a + 3 * n;
    v.rh = a + 4 * n;
    v.y = a + 5 * n;
    v.v = a + 6 * n;
    v.s = a + 7 * n;
    v.t = a + 8 * n;
    v.d = d ? d : a + 9 * n;
    return v;
}

// Blocks of the tile kernels: at most 8 per SM, and the tiles spread evenly
// over them (a block takes every G-th tile), so the last round is not a tail.
int grid_of(const fv_batch *B) {
    const int64_t cap = 148 * 8;
    const int64_t rounds = (B->ntiles + cap - 1) / cap;
    return (int)std::max<int64_t>(1, (B->ntiles + rounds - 1) / rounds);
}

Tiles tiles_of(const fv_batch *B) { return Tiles{B->ntiles, B->tile_prob, B->tile_row0, B->tile_row1, B->ptile}; }

fv_status ensure_bytes(void *&p, size_t &have, size_t need) {
    if (have >= need) return FV_OK;
    cudaFree(p);
    p = nullptr;
    have = 0;
    FV_CUDA_TRY(cudaMalloc(&p, need));
    have = need;
    return FV_OK;
}

fv_status download_state(fv_batch *B, cudaStream_t st) {
    B->hs.resize(B->np);
    FV_CUDA_TRY(cudaMemcpyAsync(B->hs.data(), B->S, sizeof(BProb) * B->np, cudaMemcpyDeviceToHost, st));
    FV_CUDA_TRY(cudaStreamSynchronize(st));
    return FV_OK;
}

// Start a run: every problem from x0 = 0, except those that from_problem maps
// to a running problem of `from`, whose state (the Krylov vectors' rows, x's
// rows and the per-problem scalars) is carried over unchanged.  Those are held
// as done while the new problems are initialised, then run again.
fv_status run_begin(fv_batch *B, fv_precond *P, bool bicg, const double *b, double *x, const fv_batch_options *opt,
                    const fv_batch *from, const int32_t *from_problem, cudaStream_t st) {
    if (!B || !P || !b || !x || !opt || opt->max_iterations < 0) return FV_ERR_INVALID;
    if (opt->precision != FV_BATCH_FP64 && opt->precision != FV_BATCH_MIXED) return FV_ERR_INVALID;
    const int64_t n = B->n;
    const int np = B->np;
    const bool mixed = opt->precision == FV_BATCH_MIXED;
    std::vector<int32_t> list;
    std::vector<int64_t> seg;
    std::vector<BProb> hs(np);
    for (int p = 0; p < np; ++p) {
        BProb q{};
        // mixed: the FP32 run never stops on its own estimate (tol = rtol = 0);
        // it stops when the FP64 residual reaches the outer tolerance
        q.tol = mixed ? 0.0 : opt->absolute_tolerance;
        q.rtol = mixed ? 0.0 : opt->relative_tolerance;
        q.max_it = opt->max_iterations;
        hs[p] = q;
    }
    if (from_problem) {
        // the carried-over problems must run the same iteration in the new batch:
        // same method, precision, mixed-precision settings and tile partition
        if (!from || from == B || !from->run || from->bicg != bicg || from->mixed != mixed || from->tile != B->tile ||
            (int)from->hs.size() != from->np)
            return FV_ERR_INVALID;
        if (mixed && (from->opt.outer_tolerance != opt->outer_tolerance ||
                      from->opt.inner_relative_tolerance != opt->inner_relative_tolerance))
            return FV_ERR_INVALID;
        std::vector<char> used((size_t)from->np, 0);
        for (int p = 0; p < np; ++p) {
            const int32_t sp = from_problem[p];
            if (sp < 0) continue;
            if (sp >= from->np || used[sp] || from->hs[sp].done) return FV_ERR_INVALID;
            const int64_t len = B->off[p + 1] - B->off[p];
            if (from->off[sp + 1] - from->off[sp] != len) return FV_ERR_INVALID;
            used[sp] = 1;
            list.push_back(p);
            seg.insert(seg.end(), {from->off[sp], B->off[p], len});
            hs[p] = from->hs[sp];
            hs[p].done = 1;  // held while the new problems start
            hs[p].ticket = 0;
        }
    }
    const int nfresh = np - (int)list.size();
    B->run = false;
    FV_TRY(ensure_bytes(B->vec, B->vec_bytes, mixed ? sizeof(float) * 10 * (size_t)n : sizeof(double) * 9 * (size_t)n));
    FV_CUDA_TRY(cudaMemcpyAsync(B->S, hs.data(), sizeof(BProb) * np, cudaMemcpyHostToDevice, st));
    BGlobal g0{nfresh, nfresh == 0 ? 1 : 0, {0, 0}};
    FV_CUDA_TRY(cudaMemcpyAsync(B->G, &g0, sizeof(BGlobal), cudaMemcpyHostToDevice, st));
    if (!list.empty()) {
        cudaFree(B->seg);
        cudaFree(B->resume);
        B->seg = nullptr;
        B->resume = nullptr;
        FV_CUDA_TRY(cudaMalloc(&B->seg, sizeof(int64_t) * seg.size()));
        FV_CUDA_TRY(cudaMalloc(&B->resume, sizeof(int32_t) * list.size()));
        FV_CUDA_TRY(cudaMemcpyAsync(B->seg, seg.data(), sizeof(int64_t) * seg.size(), cudaMemcpyHostToDevice, st));
        FV_CUDA_TRY(
            cudaMemcpyAsync(B->resume, list.data(), sizeof(int32_t) * list.size(), cudaMemcpyHostToDevice, st));
    }
    const int nseg = (int)list.size();
    const dim3 ag(32, (unsigned)std::min(nseg, 65535));
    const int G = grid_of(B);
    const Tiles tl = tiles_of(B);
    if (!mixed) {
        InnerVecs<double> v = carve<double>(B->vec, n, x);
        FV_CUDA_TRY(cudaMemcpyAsync(v.r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        if (nseg) {
            const InnerVecs<double> u = carve<double>(from->vec, from->n, from->x);
            fv_note_launch(), kb_adopt<double><<<ag, 256, 0, st>>>(B->seg, nseg, u.r, v.r);
            fv_note_launch(), kb_adopt<double><<<ag, 256, 0, st>>>(B->seg, nseg, u.p, v.p);
            fv_note_launch(), kb_adopt<double><<<ag, 256, 0, st>>>(B->seg, nseg, u.d, v.d);
            if (bicg) fv_note_launch(), kb_adopt<double><<<ag, 256, 0, st>>>(B->seg, nseg, u.rh, v.rh);
        }
        FV_TRY(inner_start<double>(bicg, B, P, v, G, tl, st));
    } else {
        if (!B->a32) FV_CUDA_TRY(cudaMalloc(&B->a32, sizeof(float) * (B->A->nnz ? B->A->nnz : 1)));
        fv_note_launch(), k_to_f32b<<<148 * 8, 256, 0, st>>>(B->A->nnz, B->A->vals, B->a32);
        FV_TRY(fv_precond_make_f32(P, st));
        InnerVecs<float> v = carve<float>(B->vec, n, nullptr);
        if (nseg) {
            const InnerVecs<float> u = carve<float>(from->vec, from->n, nullptr);
            fv_note_launch(), kb_adopt<float><<<ag, 256, 0, st>>>(B->seg, nseg, u.r, v.r);
            fv_note_launch(), kb_adopt<float><<<ag, 256, 0, st>>>(B->seg, nseg, u.p, v.p);
            fv_note_launch(), kb_adopt<float><<<ag, 256, 0, st>>>(B->seg, nseg, u.d, v.d);
            if (bicg) fv_note_launch(), kb_adopt<float><<<ag, 256, 0, st>>>(B->seg, nseg, u.rh, v.rh);
            fv_note_launch(), kb_adopt<double><<<ag, 256, 0, st>>>(B->seg, nseg, from->x, x);
        }
        fv_note_launch(), kbm_init<<<G, TB, 0, st>>>(tl, b, x, v.r, B->partial, B->S, B->G);
        FV_TRY(inner_start<float>(bicg, B, P, v, G, tl, st));
    }
    if (nseg) fv_note_launch(), kb_resume<<<(nseg + 255) / 256, 256, 0, st>>>(B->resume, nseg, B->S, B->G);
    FV_CUDA_TRY(cudaGetLastError());
    FV_TRY(download_state(B, st));
    B->run = true;
    B->bicg = bicg;
    B->mixed = mixed;
    B->P = P;
    B->b = b;
    B->x = x;
    B->opt = *opt;
    B->launched = 0;
    return FV_OK;
}

// Up to max_iterations more iterations (whole groups) until every problem is
// done; the problems that retired get their result, and the state is read back.
fv_status run_advance(fv_batch *B, int64_t max_iterations, cudaStream_t st) {
    if (!B || !B->run || max_iterations < 0) return FV_ERR_INVALID;
    const int64_t n = B->n;
    const int G = grid_of(B);
    const Tiles tl = tiles_of(B);
    bool done = true;
    for (const BProb &q : B->hs) done = done && q.done;
    const int group = B->bicg ? kGroupBiCG : kGroupCG;
    int64_t it = 0;
    if (B->mixed) {
        InnerVecs<float> v = carve<float>(B->vec, n, nullptr);
        const MixedArgs mx{MixedCfg{1, B->opt.outer_tolerance, B->opt.inner_relative_tolerance}, B->x, B->b};
        for (; !done && it < max_iterations; it += group) {
            FV_TRY(inner_group<float>(B->bicg, B, B->P, B->a32, v, G, tl, st, B->launched, mx));
            FV_TRY(wait_all_done(B, st, done));
        }
        fv_note_launch(), kb_finalize<float><<<G, TB, 0, st>>>(tl, v.d, nullptr, B->x, B->S);
    } else {
        InnerVecs<double> v = carve<double>(B->vec, n, B->x);
        const MixedArgs none{MixedCfg{0, 0.0, 0.0}, nullptr, nullptr};
        for (; !done && it < max_iterations; it += group) {
            FV_TRY(inner_group<double>(B->bicg, B, B->P, B->A->vals, v, G, tl, st, B->launched, none));
            FV_TRY(wait_all_done(B, st, done));
        }
        fv_note_launch(), kb_finalize<double><<<G, TB, 0, st>>>(tl, v.d, B->bicg ? v.y : nullptr, nullptr, B->S);
    }
    fv_note_launch(), kb_mark_fin<<<(B->np + 255) / 256, 256, 0, st>>>(B->np, B->S);
    FV_CUDA_TRY(cudaGetLastError());
    return download_state(B, st);
}

// Per-problem results from the host copy of the state.  fallback[p]: the
// problem was finished by the FP64 pass (whole-batch solves) -- or, for a
// stepwise run, the FP32 run stagnated and left it unfinished.
void fill_info(const fv_batch *B, fv_batch_info *info, const std::vector<int> &fallback) {
    if (!info) return;
    info->launched_iterations = B->launched;
    const bool mixed = B->mixed;
    for (int p = 0; p < B->np; ++p) {
        const BProb &q = B->hs[p];
        if (info->iterations) info->iterations[p] = q.iter;
        if (info->outer_steps) info->outer_steps[p] = mixed ? q.n_replace : 0;
        if (info->final_residual) info->final_residual[p] = mixed ? q.res64 : q.error;
        if (info->status)
            info->status[p] = (q.breakdown || !std::isfinite(mixed ? q.res64 : q.error)) ? FV_ERR_BREAKDOWN : FV_OK;
        if (info->fp64_fallback) info->fp64_fallback[p] = fallback.empty() ? 0 : fallback[p];
    }
}

fv_status batch_solve(bool bicg, fv_batch *B, fv_precond *P, const double *b, double *x, const fv_batch_options *opt,
                      fv_batch_info *info, cudaStream_t st) {
    if (!B || !P || !b || !x || !opt || opt->max_iterations < 0) return FV_ERR_INVALID;
    const int64_t n = B->n;
    const int np = B->np;
    const int G = grid_of(B);
    const Tiles tl = tiles_of(B);
    const bool mixed = opt->precision == FV_BATCH_MIXED;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    fv_status s = run_begin(B, P, bicg, b, x, opt, nullptr, nullptr, st);
    if (s == FV_OK) s = run_advance(B, INT64_MAX, st);
    std::vector<int> fallback;
    std::vector<BProb> &hs = B->hs;
    // FP64 pass for the problems the FP32 run could not finish (from x0 = 0)
    if (s == FV_OK && mixed) {
        fallback.assign(np, 0);
        int nfail = 0;
        for (int p = 0; p < np; ++p)
            if (hs[p].stagnated || !(hs[p].res64 <= opt->outer_tolerance)) {
                fallback[p] = 1;
                ++nfail;
            }
        if (nfail) {
            std::vector<BProb> fs(np);
            for (int p = 0; p < np; ++p) {
                BProb q{};
                q.tol = opt->outer_tolerance;
                q.rtol = opt->outer_tolerance;
                q.max_it = opt->max_iterations;
                q.done = fallback[p] ? 0 : 1;
                q.bnorm64 = hs[p].bnorm64;
                fs[p] = q;
            }
            FV_CUDA_TRY(cudaMemcpyAsync(B->S, fs.data(), sizeof(BProb) * np, cudaMemcpyHostToDevice, st));
            BGlobal g1{nfail, 0, {0, 0}};
            FV_CUDA_TRY(cudaMemcpyAsync(B->G, &g1, sizeof(BGlobal), cudaMemcpyHostToDevice, st));
            FV_TRY(ensure_bytes(B->vec64, B->vec64_bytes, sizeof(double) * 9 * (size_t)n));
            InnerVecs<double> w = carve<double>(B->vec64, n, x);
            FV_CUDA_TRY(cudaMemcpyAsync(w.r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
            const MixedArgs none{MixedCfg{0, 0.0, 0.0}, nullptr, nullptr};
            s = inner_solve<double>(bicg, B, P, B->A->vals, w, G, tl, st, B->launched, none);
            if (s == FV_OK) {
                std::vector<BProb> f2(np);
                FV_CUDA_TRY(cudaMemcpyAsync(f2.data(), B->S, sizeof(BProb) * np, cudaMemcpyDeviceToHost, st));
                FV_CUDA_TRY(cudaStreamSynchronize(st));
                for (int p = 0; p < np; ++p)
                    if (fallback[p]) {
                        hs[p].iter += f2[p].iter;
                        hs[p].res64 = f2[p].error;  // |r|/|b| of the FP64 CG/BiCGStab
                        hs[p].breakdown = f2[p].breakdown;
                    }
                FV_CUDA_TRY(cudaMemcpyAsync(B->S, hs.data(), sizeof(BProb) * np, cudaMemcpyHostToDevice, st));
            }
        }
    }
    cudaEventRecord(e1, st);
    FV_CUDA_TRY(cudaStreamSynchronize(st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    B->run = false;  // the state was overwritten by the FP64 pass: nothing to carry over
    if (s == FV_OK) s = fv_precond_check_error(P, st);
    if (s == FV_OK && info) {
        fill_info(B, info, fallback);
        info->device_ms = ms;
    }
    return s;
}

}  // namespace

extern "C" fv_status fv_batch_cg(fv_batch *B, fv_precond *P, const double *b, double *x,
                                 const fv_batch_options *opt, fv_batch_info *info, void *stream) {
    return fv_host_guard([&] { return batch_solve(false, B, P, b, x, opt, info, fv_stream(stream)); });
}

extern "C" fv_status fv_batch_bicgstab(fv_batch *B, fv_precond *P, const double *b, double *x,
                                       const fv_batch_options *opt, fv_batch_info *info, void *stream) {
    return fv_host_guard([&] { return batch_solve(true, B, P, b, x, opt, info, fv_stream(stream)); });
}

extern "C" fv_status fv_batch_begin(fv_batch *B, fv_precond *P, int32_t method, const double *b, double *x,
                                    const fv_batch_options *opt, const fv_batch *from, const int32_t *from_problem,
                                    void *stream) {
    if (method != FV_BATCH_CG && method != FV_BATCH_BICGSTAB) return FV_ERR_INVALID;
    return fv_host_guard([&] {
        return run_begin(B, P, method == FV_BATCH_BICGSTAB, b, x, opt, from, from_problem, fv_stream(stream));
    });
}

extern "C" fv_status fv_batch_advance(fv_batch *B, int64_t max_iterations, int32_t *n_running, int32_t *done,
                                      void *stream) {
    return fv_host_guard([&] {
        FV_TRY(run_advance(B, max_iterations, fv_stream(stream)));
        int32_t running = 0;
        for (int p = 0; p < B->np; ++p) {
            running += B->hs[p].done ? 0 : 1;
            if (done) done[p] = B->hs[p].done ? 1 : 0;
        }
        if (n_running) *n_running = running;
        return FV_OK;
    });
}

extern "C" fv_status fv_batch_report(const fv_batch *B, fv_batch_info *info) {
    if (!B || !B->run || !info) return FV_ERR_INVALID;
    return fv_host_guard([&] {
        std::vector<int> stalled(B->np, 0);
        for (int p = 0; p < B->np; ++p) stalled[p] = B->mixed && B->hs[p].stagnated;
        fill_info(B, info, stalled);
        info->device_ms = 0.0;
        return FV_OK;
    });
}
