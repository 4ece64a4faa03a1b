/*
 * CPU oracle, MPI semantics -- TEST AND CPU-BASELINE INFRASTRUCTURE ONLY.
 *
 * Restates what the finite-volumes crate computes when it runs on P MPI
 * ranks, with one OpenMP thread standing for one rank:
 *   - the rows are split into P contiguous partitions (the reference uses a
 *     METIS part_recursive split, core/mesh/decompose.rs:32; METIS is not
 *     available here, so partitions are contiguous ranges of the natural order);
 *   - every rank factorises only its square diagonal block
 *     (DistributedMatrix::square_block, src/linalg/dmatrix.rs:214-229, used by
 *     incomplete_cholesky.rs:151 and incomplete_lower_upper.rs:202):
 *     a block-Jacobi IC(0) / ILU(0);
 *   - SpMV reads ghost values after the halo `collect`
 *     (core/communicator.rs:226-266): with shared memory the halo is the
 *     global vector itself;
 *   - every dot product is a per-rank serial sum followed by reduce_add
 *     (core/communicator.rs:282-290), summed here in rank order;
 *   - CG / BiCGStab otherwise follow conjugate_gradient.rs / bi_conjugate_gradient_stab.rs.
 * With P = 1 this is the single-rank oracle of oracle.c.
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct or_precond or_precond;
or_precond *or_ic0_create(int64_t n, const int32_t *ptr, const int32_t *col, const double *val, int *status);
or_precond *or_ilu0_create(int64_t n, const int32_t *ptr, const int32_t *col, const double *val, int *status);
void or_precond_apply(const or_precond *p, const double *rhs, double *sol);
void or_precond_free(or_precond *p);

typedef struct {
    int P;
    int64_t n;
    int64_t *lo; /* P+1 partition bounds */
    or_precond **blk;
} or_bj;

void or_bj_free(or_bj *b) {
    if (!b) return;
    for (int t = 0; t < b->P; ++t) or_precond_free(b->blk[t]);
    free(b->blk);
    free(b->lo);
    free(b);
}

/* kind 1 = IC(0), 2 = ILU(0) on each rank's square block */
or_bj *or_bj_create(int kind, int64_t n, const int32_t *ptr, const int32_t *col, const double *val, int P,
                    int *status) {
    or_bj *b = (or_bj *)calloc(1, sizeof(or_bj));
    b->P = P;
    b->n = n;
    b->lo = (int64_t *)malloc(sizeof(int64_t) * (P + 1));
    b->blk = (or_precond **)calloc((size_t)P, sizeof(or_precond *));
    for (int t = 0; t <= P; ++t) b->lo[t] = n * t / P;
    int bad = 0;
#pragma omp parallel for num_threads(P) schedule(static, 1) reduction(| : bad)
    for (int t = 0; t < P; ++t) {
        const int64_t lo = b->lo[t], hi = b->lo[t + 1], m = hi - lo;
        int64_t nz = 0;
        for (int64_t i = lo; i < hi; ++i)
            for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k)
                if (col[k] >= lo && col[k] < hi) ++nz;
        int32_t *bp = (int32_t *)malloc(sizeof(int32_t) * (m + 1));
        int32_t *bc = (int32_t *)malloc(sizeof(int32_t) * (nz ? nz : 1));
        double *bv = (double *)malloc(sizeof(double) * (nz ? nz : 1));
        int64_t o = 0;
        for (int64_t i = lo; i < hi; ++i) {
            bp[i - lo] = (int32_t)o;
            for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k)
                if (col[k] >= lo && col[k] < hi) {
                    bc[o] = (int32_t)(col[k] - lo);
                    bv[o++] = val[k];
                }
        }
        bp[m] = (int32_t)o;
        int st = 0;
        b->blk[t] = kind == 1 ? or_ic0_create(m, bp, bc, bv, &st) : or_ilu0_create(m, bp, bc, bv, &st);
        if (!b->blk[t] || st) bad |= (st ? st : 1);
        free(bp);
        free(bc);
        free(bv);
    }
    *status = bad;
    if (bad) {
        or_bj_free(b);
        return NULL;
    }
    return b;
}

static void bj_apply(const or_bj *b, const double *r, double *z) {
#pragma omp parallel for num_threads(b->P) schedule(static, 1)
    for (int t = 0; t < b->P; ++t) or_precond_apply(b->blk[t], r + b->lo[t], z + b->lo[t]);
}

static void spmv_par(const or_bj *b, const int32_t *ptr, const int32_t *col, const double *val, const double *x,
                     double *y) {
#pragma omp parallel for num_threads(b->P) schedule(static, 1)
    for (int t = 0; t < b->P; ++t)
        for (int64_t i = b->lo[t]; i < b->lo[t + 1]; ++i) {
            double s = 0.0;
            for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k) s += val[k] * x[col[k]];
            y[i] = s;
        }
}

static double dot_par(const or_bj *b, const double *x, const double *y, double *part) {
#pragma omp parallel for num_threads(b->P) schedule(static, 1)
    for (int t = 0; t < b->P; ++t) {
        double s = 0.0;
        for (int64_t i = b->lo[t]; i < b->lo[t + 1]; ++i) s += x[i] * y[i];
        part[t] = s;
    }
    double s = 0.0;
    for (int t = 0; t < b->P; ++t) s += part[t];
    return s;
}

typedef struct {
    int64_t iterations;
    double initial_residual;
    double final_residual;
    int64_t history_len;
    int32_t restarts;
} or_info;

#define PAR_FOR(b) _Pragma("omp parallel for num_threads(b->P) schedule(static, 1)") for (int t = 0; t < b->P; ++t)
#define ROWS(b) for (int64_t i = b->lo[t]; i < b->lo[t + 1]; ++i)

int or_bj_cg(int64_t n, const int32_t *ptr, const int32_t *col, const double *val, const or_bj *b,
             const double *rhs, double *x, double rtol, double atol, int64_t max_iter, or_info *info) {
    memset(info, 0, sizeof(*info));
    double *part = (double *)calloc((size_t)b->P, sizeof(double));
    const double bnorm = sqrt(dot_par(b, rhs, rhs, part));
    if (bnorm < 1e-14) {
        memset(x, 0, sizeof(double) * n);
        info->initial_residual = info->final_residual = bnorm;
        info->history_len = 1;
        free(part);
        return 0;
    }
    double *p = (double *)calloc((size_t)n, sizeof(double)), *r = (double *)calloc((size_t)n, sizeof(double));
    double *z = (double *)calloc((size_t)n, sizeof(double)), *ap = (double *)calloc((size_t)n, sizeof(double));
    spmv_par(b, ptr, col, val, x, r);
    PAR_FOR(b) ROWS(b) {
        r[i] -= rhs[i];
        r[i] *= -1.0;
    }
    const double init = sqrt(dot_par(b, r, r, part)) / bnorm;
    bj_apply(b, r, z);
    memcpy(p, z, sizeof(double) * n);
    double error = 1.0;
    int64_t iter = 0;
    while (error > atol) {
        if (iter > max_iter) break;
        spmv_par(b, ptr, col, val, p, ap);
        const double rz = dot_par(b, r, z, part), pap = dot_par(b, p, ap, part);
        const double alpha = rz / pap;
        PAR_FOR(b) ROWS(b) {
            x[i] += p[i] * alpha;
            r[i] -= ap[i] * alpha;
        }
        error = sqrt(dot_par(b, r, r, part)) / bnorm;
        if (error < atol || error / init < rtol) {
            iter++;
            break;
        }
        bj_apply(b, r, z);
        const double beta = dot_par(b, r, z, part) / rz;
        PAR_FOR(b) ROWS(b) p[i] = z[i] + p[i] * beta;
        iter++;
    }
    info->iterations = iter;
    info->initial_residual = init;
    info->final_residual = error;
    info->history_len = iter;
    free(p);
    free(r);
    free(z);
    free(ap);
    free(part);
    return 0;
}

int or_bj_bicgstab(int64_t n, const int32_t *ptr, const int32_t *col, const double *val, const or_bj *b,
                   const double *rhs, double *x, double rtol, double atol, int64_t max_iter, or_info *info) {
    memset(info, 0, sizeof(*info));
    double *part = (double *)calloc((size_t)b->P, sizeof(double));
    const double bnorm = sqrt(dot_par(b, rhs, rhs, part));
    if (bnorm < 1e-14) {
        memset(x, 0, sizeof(double) * n);
        info->initial_residual = info->final_residual = bnorm;
        info->history_len = 1;
        free(part);
        return 0;
    }
    double *v[9];
    for (int k = 0; k < 9; ++k) v[k] = (double *)calloc((size_t)n, sizeof(double));
    double *p = v[0], *r = v[1], *rh = v[2], *z = v[3], *y = v[4], *vv = v[5], *h = v[6], *s = v[7], *tt = v[8];
    spmv_par(b, ptr, col, val, x, r);
    PAR_FOR(b) ROWS(b) {
        r[i] -= rhs[i];
        r[i] *= -1.0;
        rh[i] = r[i];
    }
    const double init = sqrt(dot_par(b, r, r, part)) / bnorm;
    double error = 1.0;
    int64_t iter = 0;
    if (init < atol) {
        info->initial_residual = info->final_residual = init;
        info->history_len = 1;
        goto done;
    }
    memcpy(p, r, sizeof(double) * n);
    double rho = dot_par(b, rh, r, part);
    while (error > atol) {
        if (iter > max_iter) break;
        bj_apply(b, p, y);
        spmv_par(b, ptr, col, val, y, vv);
        const double alpha = rho / dot_par(b, rh, vv, part);
        PAR_FOR(b) ROWS(b) {
            h[i] = x[i] + y[i] * alpha;
            s[i] = r[i] - vv[i] * alpha;
        }
        const double sn = sqrt(dot_par(b, s, s, part)) / bnorm;
        if (sn < atol || sn / init < rtol) {
            error = sn;
            memcpy(x, h, sizeof(double) * n);
            iter++;
            break;
        }
        bj_apply(b, s, z);
        spmv_par(b, ptr, col, val, z, tt);
        const double omega = dot_par(b, tt, s, part) / dot_par(b, tt, tt, part);
        PAR_FOR(b) ROWS(b) {
            x[i] = h[i] + z[i] * omega;
            r[i] = s[i] - tt[i] * omega;
        }
        const double rn = sqrt(dot_par(b, r, r, part)) / bnorm;
        if (rn < atol || rn / init < rtol) {
            error = rn;
            iter++;
            break;
        }
        const double rho_new = dot_par(b, rh, r, part);
        const double beta = (rho_new / rho) * (alpha / omega);
        rho = rho_new;
        if (fabs(rho) > 1e-15 * bnorm) {
            PAR_FOR(b) ROWS(b) p[i] = r[i] + (p[i] - vv[i] * omega) * beta;
        } else {
            PAR_FOR(b) ROWS(b) {
                rh[i] = r[i];
                p[i] = r[i];
            }
            rho = dot_par(b, rh, r, part);
            info->restarts++;
        }
        error = rn / bnorm;
        iter++;
    }
    info->iterations = iter;
    info->initial_residual = init;
    info->final_residual = error;
    info->history_len = iter;
done:
    for (int k = 0; k < 9; ++k) free(v[k]);
    free(part);
    return 0;
}

/* ------------------------------------------------------------ assembly per rank
 * What each rank does in assemble (fvm/assembly.rs:11-78) for its own cells:
 * rank t owns the rows [lo_t, hi_t) (contiguous partitions, as above), builds
 * their sorted cell_to_cell rows (dmatrix.rs:38-50) and adds every face
 * contribution that lands in them, in ascending face order.  A row therefore
 * receives the same additions in the same order as in the single-rank oracle
 * (or_pattern + or_assemble), and every value equals it bit for bit.  Terms:
 * c_conv*convection(Upwind(F), F) + c_lap*laplacian(Orthogonal, kappa)
 * + c_src*source(f), boundary closure (bndi, bnde). */
static int cmp_i32_mpi(const void *a, const void *b) {
    const int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
    return (x > y) - (x < y);
}

static int row_pattern(int64_t c, const int32_t *cell_face_ptr, const int32_t *cell_faces, const int32_t *owner,
                       const int32_t *neighbor, int32_t *tmp) {
    int len = 0;
    tmp[len++] = (int32_t)c;
    for (int32_t k = cell_face_ptr[c]; k < cell_face_ptr[c + 1]; ++k) {
        const int32_t f = cell_faces[k], nb = neighbor[f];
        if (nb < 0) continue;
        const int32_t other = (nb == (int32_t)c) ? owner[f] : nb;
        int dup = 0;
        for (int q = 1; q < len; ++q)
            if (tmp[q] == other) dup = 1;
        if (!dup) {
            if (len >= 64) return -1;
            tmp[len++] = other;
        }
    }
    qsort(tmp, (size_t)len, sizeof(int32_t), cmp_i32_mpi);
    return len;
}

/* Pattern on P threads: cols == NULL only counts (returns nnz in *nnz_out). */
int or_pattern_par(int64_t n_cells, const int32_t *cell_face_ptr, const int32_t *cell_faces, const int32_t *owner,
                   const int32_t *neighbor, int P, int32_t *row_ptr, int32_t *cols, int64_t *nnz_out) {
    int bad = 0;
    if (!cols) {
#pragma omp parallel for num_threads(P) schedule(static) reduction(| : bad)
        for (int64_t c = 0; c < n_cells; ++c) {
            int32_t tmp[64];
            const int len = row_pattern(c, cell_face_ptr, cell_faces, owner, neighbor, tmp);
            if (len < 0) bad = 1;
            row_ptr[c + 1] = len < 0 ? 0 : len;
        }
        if (bad) return 2;
        row_ptr[0] = 0;
        for (int64_t c = 0; c < n_cells; ++c) row_ptr[c + 1] += row_ptr[c];
        *nnz_out = row_ptr[n_cells];
        return 0;
    }
#pragma omp parallel for num_threads(P) schedule(static)
    for (int64_t c = 0; c < n_cells; ++c) {
        int32_t tmp[64];
        const int len = row_pattern(c, cell_face_ptr, cell_faces, owner, neighbor, tmp);
        for (int q = 0; q < len; ++q) cols[row_ptr[c] + q] = tmp[q];
    }
    *nnz_out = row_ptr[n_cells];
    return 0;
}

static int64_t find_mpi(const int32_t *ptr, const int32_t *col, int64_t i, int32_t j) {
    int64_t lo = ptr[i], hi = ptr[i + 1];
    while (lo < hi) {
        const int64_t mid = (lo + hi) / 2;
        if (col[mid] < j)
            lo = mid + 1;
        else
            hi = mid;
    }
    return (lo < ptr[i + 1] && col[lo] == j) ? lo : -1;
}

int or_assemble_par(int32_t dim, int64_t n_cells, int64_t n_faces, int64_t n_bfaces, const int32_t *owner,
                    const int32_t *neighbor, const double *area, const double *face_center,
                    const double *cell_center, const double *volume, double c_lap, double c_conv, double c_src,
                    const double *kappa, const double *flux, const double *source, const double *bndi,
                    const double *bnde, const int32_t *row_ptr, const int32_t *cols, int P, double *vals,
                    double *rhs) {
    const int64_t fb0 = n_faces - n_bfaces;
    int bad = 0;
#pragma omp parallel num_threads(P) reduction(| : bad)
    {
        const int t = omp_get_thread_num(), nt = omp_get_num_threads();
        const int64_t lo = n_cells * t / nt, hi = n_cells * (t + 1) / nt;
        for (int64_t k = row_ptr[lo]; k < row_ptr[hi]; ++k) vals[k] = 0.0;
        /* cell loop (assembly.rs:26-32) */
        for (int64_t c = lo; c < hi; ++c) {
            const double l = 0.0;
            const double r = c_src != 0.0 ? c_src * (-source[c]) : 0.0;
            const int64_t kd = find_mpi(row_ptr, cols, c, (int32_t)c);
            if (kd < 0) {
                bad = 1;
                continue;
            }
            vals[kd] = l * volume[c];
            rhs[c] = r * volume[c];
        }
        /* face loop (assembly.rs:35-75), contributions to own rows only */
        for (int64_t f = 0; f < n_faces && !bad; ++f) {
            const int64_t i = owner[f], j = neighbor[f];
            const int own_i = i >= lo && i < hi, own_j = j >= lo && j < hi;
            if (!own_i && !own_j) continue;
            const double *ci = cell_center + i * dim;
            const double *cj = j >= 0 ? cell_center + j * dim : face_center + f * dim;
            double dvec[3], dd = 0.0;
            for (int d = 0; d < dim; ++d) dvec[d] = cj[d] - ci[d];
            for (int d = 0; d < dim; ++d) dd += dvec[d] * dvec[d];
            const double tt = 1.0 / sqrt(dd); /* Orthogonal (orthogonal.rs:26-46) */
            double lap0 = 0.0, lap1 = 0.0, conv0 = 0.0, conv1 = 0.0;
            if (c_lap != 0.0) {
                lap0 = kappa[f] * (-tt);
                lap1 = kappa[f] * tt;
            }
            if (c_conv != 0.0) { /* Upwind (upwind.rs:26-33) */
                const double F = flux[f];
                if (F > 0.0) {
                    conv0 = 1.0 * F;
                    conv1 = 0.0 * F;
                } else {
                    conv0 = 0.0 * F;
                    conv1 = 1.0 * F;
                }
            }
            double li, lj;
            if (c_conv != 0.0 && c_lap != 0.0) {
                li = c_conv * conv0 + c_lap * lap0;
                lj = c_conv * conv1 + c_lap * lap1;
            } else if (c_lap != 0.0) {
                li = c_lap * lap0;
                lj = c_lap * lap1;
            } else {
                li = c_conv * conv0;
                lj = c_conv * conv1;
            }
            const double r = 0.0;
            li = li * area[f];
            lj = lj * area[f];
            const double ra = r * area[f];
            if (j >= 0) {
                if (own_i) {
                    const int64_t kii = find_mpi(row_ptr, cols, i, (int32_t)i);
                    const int64_t kij = find_mpi(row_ptr, cols, i, (int32_t)j);
                    if (kii < 0 || kij < 0) {
                        bad = 1;
                        continue;
                    }
                    vals[kii] += li;
                    vals[kij] += lj;
                    rhs[i] += ra;
                }
                if (own_j) {
                    const int64_t kji = find_mpi(row_ptr, cols, j, (int32_t)i);
                    const int64_t kjj = find_mpi(row_ptr, cols, j, (int32_t)j);
                    if (kji < 0 || kjj < 0) {
                        bad = 1;
                        continue;
                    }
                    vals[kji] -= li;
                    vals[kjj] -= lj;
                    rhs[j] -= ra;
                }
            } else {
                if (f < fb0) {
                    bad = 1;
                    continue;
                }
                const double bi = bndi[f - fb0], be = bnde[f - fb0];
                const int64_t kii = find_mpi(row_ptr, cols, i, (int32_t)i);
                if (kii < 0) {
                    bad = 1;
                    continue;
                }
                vals[kii] += li;
                vals[kii] += lj * bi;
                rhs[i] += ra - lj * be;
            }
        }
    }
    return bad ? 2 : 0;
}
