/*
 * CPU oracle -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, single-threaded FP64 restatement of the finite-volumes crate's
 * assembly + Krylov path, with the reference's loop structure, indexing
 * (binary search into sorted CSR rows) and floating-point operation order.
 * Built with -ffp-contract=off so no a*b+c is fused, as in the Rust build.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it,
 * and only as the checker / the timed CPU baseline.  The product library
 * (libfvb200.so) never links or calls it.
 *
 * Pinning: the reference ships no assembly / factorisation / solver tests and
 * cannot be built here (Rust toolchain and MPI absent), so these functions
 * are parity-unpinned against the reference itself; they are cross-checked
 * against SciPy (direct solves, factor residuals) and against hand-derived
 * two-point-flux coefficients in tests/.  The mesh geometry they consume is
 * pinned by the reference's own square.su2 known-answer test.
 *
 * Reference files followed (paths inside the reference crate):
 *   assemble ............ src/fvm/assembly.rs:11-78
 *   terms ............... src/fvm/terms/{laplacian.rs:35-45,convection.rs:36-45,
 *                          source.rs:34-40,operations.rs:86-199}
 *   schemes ............. src/fvm/schemes/facengrad/orthogonal.rs:26-46,
 *                          src/fvm/schemes/facengrad/corrected.rs:36-67,
 *                          src/fvm/schemes/faceinterp/upwind.rs:26-33
 *   transient terms ..... src/fvm/terms/time.rs:19-35, src/fvm/schemes/time/{euler.rs,backward.rs},
 *                          src/fvm/terms/source.rs:61-79 (linear_source),
 *                          src/fvm/terms/divergence.rs:22-43
 *   gradients ........... src/core/mesh/compute.rs:155-203 (coefficients),
 *                          src/core/matrix.rs:320-380 (Matrix::inv),
 *                          src/fvm/tools/gradients.rs:48-86 (compute_gradients)
 *   CSR ................. src/linalg/dmatrix.rs:38-50 (pattern), 136-146 (imul),
 *                          262-286 (Index by binary search), 76-88 (is_symmetric)
 *   dot ................. src/linalg/dvector.rs:63-79
 *   IC(k) ............... src/linalg/preconditioners/incomplete_cholesky.rs:87-255
 *   ILU(k) .............. src/linalg/preconditioners/incomplete_lower_upper.rs:200-329,
 *                          src/linalg/sparse_array.rs:48-50 (drop rule)
 *   CG .................. src/linalg/solvers/conjugate_gradient.rs:12-111
 *   BiCGStab ............ src/linalg/solvers/bi_conjugate_gradient_stab.rs:13-178
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum { OR_OK = 0, OR_ERR_ALLOC = 1, OR_ERR_INVALID = 2, OR_ERR_SINGULAR = 3, OR_ERR_NOT_SYMMETRIC = 6 };

/* ---------------------------------------------------------------- CSR */
typedef struct {
    int64_t n;
    int32_t *ptr; /* n+1 */
    int32_t *col;
    double *val;
} csr_t;

/* binary search of column j in row i; -1 when absent (dmatrix.rs:262-286) */
static int64_t csr_find(const int32_t *ptr, const int32_t *col, int64_t i, int32_t j) {
    int64_t lo = ptr[i], hi = ptr[i + 1];
    while (lo < hi) {
        int64_t mid = lo + (hi - lo) / 2;
        if (col[mid] < j)
            lo = mid + 1;
        else if (col[mid] > j)
            hi = mid;
        else
            return mid;
    }
    return -1;
}

static int cmp_i32(const void *a, const void *b) {
    int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
    return (x > y) - (x < y);
}

/* ------------------------------------------------------------- assemble */
/*
 * Pattern: cell_to_cell (own cell + the other cell of every interior face,
 * duplicates removed; compute.rs:135-152), rows sorted (dmatrix.rs:38-50).
 * Returns nnz in *nnz_out; when cols == NULL only the count is produced.
 */
int or_pattern(int64_t n_cells, const int32_t *cell_face_ptr, const int32_t *cell_faces, const int32_t *owner,
               const int32_t *neighbor, int32_t *row_ptr, int32_t *cols, int64_t *nnz_out) {
    int64_t nnz = 0;
    int32_t tmp[64];
    for (int64_t c = 0; c < n_cells; ++c) {
        int len = 0;
        tmp[len++] = (int32_t)c;
        for (int32_t k = cell_face_ptr[c]; k < cell_face_ptr[c + 1]; ++k) {
            int32_t f = cell_faces[k];
            int32_t nb = neighbor[f];
            if (nb < 0) continue;
            int32_t other = (nb == (int32_t)c) ? owner[f] : nb;
            int dup = 0;
            for (int q = 1; q < len; ++q)
                if (tmp[q] == other) dup = 1;
            if (!dup) {
                if (len >= 64) return OR_ERR_INVALID;
                tmp[len++] = other;
            }
        }
        qsort(tmp, (size_t)len, sizeof(int32_t), cmp_i32);
        if (row_ptr) row_ptr[c] = (int32_t)nnz;
        if (cols)
            for (int q = 0; q < len; ++q) cols[nnz + q] = tmp[q];
        nnz += len;
    }
    if (row_ptr) row_ptr[n_cells] = (int32_t)nnz;
    *nnz_out = nnz;
    return OR_OK;
}

/*
 * assemble(c_conv*convection(Upwind(F),F) + c_lap*laplacian(Orthogonal,kappa)
 *          + c_src*source(f), bc, mesh)             (assembly.rs:11-78)
 *
 * Term values (operations.rs evaluates the expression tree term by term):
 *   Orthogonal (orthogonal.rs:26-46): t = 1/|c_j - c_i| (boundary: 1/|x_f - c_i|),
 *      (lhs0, lhs1) = (-t, t); Laplacian multiplies by kappa_f.
 *   Upwind (upwind.rs:26-33): F>0 -> (1,0), else (0,1); Convection multiplies by F.
 *   Source (source.rs:34-40): cell rhs -f_c.
 * A face value is conv*c_conv + lap*c_lap; with c in {-1,0,1} this is the one
 * rounding the reference performs for `conv - lap`, `-lap`, etc.
 */
/* Face-normal gradient scheme of the laplacian for face f with owner centre
 * ci and other point cj (neighbour centre, or face centre on the boundary):
 * Orthogonal (facengrad/orthogonal.rs:26-46): t = 1/|cj - ci|, no rhs;
 * Corrected (facengrad/corrected.rs:36-67): t = 1/(n.d), rhs = explicit
 * correction gf.(n - t d) * reduction, gf interpolated with
 * w = (x_f - ci).n / (d.n) on interior faces, the owner's gradient on
 * boundary faces. */
static double dotv(int dim, const double *a, const double *b) {
    double x = 0.0;
    for (int d = 0; d < dim; ++d) x += a[d] * b[d];
    return x;
}

static void scheme_terms(int32_t dim, int scheme, int64_t f, int64_t i, int64_t j, const double *ci,
                         const double *cj, const double *face_center, const double *face_normal,
                         const double *grad, double red, double *t_out, double *rsch_out) {
    double dvec[3];
    for (int d = 0; d < dim; ++d) dvec[d] = cj[d] - ci[d];
    if (scheme == 0) {
        *t_out = 1.0 / sqrt(dotv(dim, dvec, dvec));
        *rsch_out = 0.0;
        return;
    }
    const double *n = face_normal + f * dim;
    const double c_corr = 1.0 / dotv(dim, n, dvec);
    double v[3], gf[3];
    for (int d = 0; d < dim; ++d) v[d] = n[d] - c_corr * dvec[d];
    if (j >= 0) {
        double e[3];
        const double *xf = face_center + f * dim;
        for (int d = 0; d < dim; ++d) e[d] = xf[d] - ci[d];
        const double w = dotv(dim, e, n) / dotv(dim, dvec, n);
        for (int d = 0; d < dim; ++d) gf[d] = grad[i * dim + d] * (1.0 - w) + grad[j * dim + d] * w;
    } else {
        for (int d = 0; d < dim; ++d) gf[d] = grad[i * dim + d];
    }
    *t_out = c_corr;
    *rsch_out = dotv(dim, gf, v) * red;
}

int or_assemble_scheme(int32_t dim, int64_t n_cells, int64_t n_faces, int64_t n_bfaces, const int32_t *owner,
                       const int32_t *neighbor, const double *area, const double *face_center,
                       const double *cell_center, const double *volume, double c_lap, double c_conv, double c_src,
                       const double *kappa, const double *flux, const double *source, const double *bndi,
                       const double *bnde, const int32_t *row_ptr, const int32_t *cols, double *vals, double *rhs,
                       int scheme, const double *face_normal, const double *grad, double red);

/* Extra terms of an expression: time(Euler | Backward) (terms/time.rs,
 * schemes/time/euler.rs, backward.rs), linear_source (terms/source.rs:61-79),
 * divergence (terms/divergence.rs:22-43).  coef = {c_time, c_lin, c_div},
 * time_scheme 1 Euler / 2 Backward; dens* may be NULL (density 1). */
typedef struct {
    double c_time, c_lin, c_div;
    int time_scheme;
    double dt, dt_2;
    const double *prev, *prev2, *dens, *densp, *densp2, *lin, *divflux;
} or_extra;

int or_assemble_full(int32_t dim, int64_t n_cells, int64_t n_faces, int64_t n_bfaces, const int32_t *owner,
                     const int32_t *neighbor, const double *area, const double *face_center,
                     const double *cell_center, const double *volume, double c_lap, double c_conv, double c_src,
                     const double *kappa, const double *flux, const double *source, const double *bndi,
                     const double *bnde, const int32_t *row_ptr, const int32_t *cols, double *vals, double *rhs,
                     int scheme, const double *face_normal, const double *grad, double red, const or_extra *ex);

int or_assemble(int32_t dim, int64_t n_cells, int64_t n_faces, int64_t n_bfaces, const int32_t *owner,
                const int32_t *neighbor, const double *area, const double *face_center,
                const double *cell_center, const double *volume, double c_lap, double c_conv, double c_src,
                const double *kappa, const double *flux, const double *source, const double *bndi,
                const double *bnde, const int32_t *row_ptr, const int32_t *cols, double *vals, double *rhs) {
    return or_assemble_full(dim, n_cells, n_faces, n_bfaces, owner, neighbor, area, face_center, cell_center,
                            volume, c_lap, c_conv, c_src, kappa, flux, source, bndi, bnde, row_ptr, cols, vals,
                            rhs, 0, NULL, NULL, 0.0, NULL);
}

int or_assemble_scheme(int32_t dim, int64_t n_cells, int64_t n_faces, int64_t n_bfaces, const int32_t *owner,
                       const int32_t *neighbor, const double *area, const double *face_center,
                       const double *cell_center, const double *volume, double c_lap, double c_conv, double c_src,
                       const double *kappa, const double *flux, const double *source, const double *bndi,
                       const double *bnde, const int32_t *row_ptr, const int32_t *cols, double *vals, double *rhs,
                       int scheme, const double *face_normal, const double *grad, double red) {
    return or_assemble_full(dim, n_cells, n_faces, n_bfaces, owner, neighbor, area, face_center, cell_center,
                            volume, c_lap, c_conv, c_src, kappa, flux, source, bndi, bnde, row_ptr, cols, vals,
                            rhs, scheme, face_normal, grad, red, NULL);
}

/* the cell terms of the time schemes (euler.rs:37-47, backward.rs:44-66) */
static void time_cell(const or_extra *ex, int64_t c, double *tl, double *tr) {
    if (ex->time_scheme == 1) {
        const double r0 = ex->dens ? ex->dens[c] : 1.0, r1 = ex->dens ? ex->densp[c] : 1.0;
        *tl = 1.0 * (1.0 / ex->dt) * r0;
        *tr = ex->prev[c] / ex->dt * r1;
    } else {
        const double wn = ex->dt / ex->dt_2;
        const double a_next = (1.0 + 2.0 * wn) / (1.0 + wn);
        const double a_last = ((1.0 + wn) * (1.0 + wn)) / (1.0 + wn);
        const double a_last_2 = (wn * wn) / (1.0 + wn);
        const double r0 = ex->dens ? ex->dens[c] : 1.0, r1 = ex->dens ? ex->densp[c] : 1.0,
                     r2 = ex->dens ? ex->densp2[c] : 1.0;
        *tl = 1.0 * (a_next / ex->dt) * r0;
        *tr = (ex->prev[c] * a_last * r1 - ex->prev2[c] * a_last_2 * r2) / ex->dt;
    }
}

int or_assemble_full(int32_t dim, int64_t n_cells, int64_t n_faces, int64_t n_bfaces, const int32_t *owner,
                     const int32_t *neighbor, const double *area, const double *face_center,
                     const double *cell_center, const double *volume, double c_lap, double c_conv, double c_src,
                     const double *kappa, const double *flux, const double *source, const double *bndi,
                     const double *bnde, const int32_t *row_ptr, const int32_t *cols, double *vals, double *rhs,
                     int scheme, const double *face_normal, const double *grad, double red, const or_extra *ex) {
    const or_extra none = {0};
    if (!ex) ex = &none;
    const int64_t nnz = row_ptr[n_cells];
    const int64_t fb0 = n_faces - n_bfaces;
    for (int64_t k = 0; k < nnz; ++k) vals[k] = 0.0;
    /* cell loop (assembly.rs:26-32); at most two nonzero terms per side, so
     * the signed sum equals the term tree's value in any order */
    for (int64_t c = 0; c < n_cells; ++c) {
        double tl = 0.0, tr = 0.0;
        if (ex->c_time != 0.0) time_cell(ex, c, &tl, &tr);
        double l = 0.0;
        if (ex->c_time != 0.0 && ex->c_lin != 0.0)
            l = ex->c_time * tl + ex->c_lin * ex->lin[c];
        else if (ex->c_time != 0.0)
            l = ex->c_time * tl;
        else if (ex->c_lin != 0.0)
            l = ex->c_lin * ex->lin[c];
        double r = 0.0;
        if (ex->c_time != 0.0 && c_src != 0.0)
            r = ex->c_time * tr + c_src * (-source[c]);
        else if (ex->c_time != 0.0)
            r = ex->c_time * tr;
        else if (c_src != 0.0)
            r = c_src * (-source[c]);
        int64_t kd = csr_find(row_ptr, cols, c, (int32_t)c);
        if (kd < 0) return OR_ERR_INVALID;
        vals[kd] = l * volume[c];
        rhs[c] = r * volume[c];
    }
    /* face loop (assembly.rs:35-75) */
    for (int64_t f = 0; f < n_faces; ++f) {
        const int64_t i = owner[f];
        const int64_t j = neighbor[f];
        const double *ci = cell_center + i * dim;
        const double *cj = j >= 0 ? cell_center + j * dim : face_center + f * dim;
        double t, rsch;
        scheme_terms(dim, c_lap != 0.0 ? scheme : 0, f, i, j, ci, cj, face_center, face_normal, grad, red, &t, &rsch);
        double lap0 = 0.0, lap1 = 0.0, lap_r = 0.0, conv0 = 0.0, conv1 = 0.0;
        if (c_lap != 0.0) {
            lap0 = kappa[f] * (-t);
            lap1 = kappa[f] * t;
            lap_r = -(kappa[f] * rsch); /* laplacian.rs:35-45 */
        }
        if (c_conv != 0.0) {
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
        /* face rhs: the Corrected laplacian's and the divergence's (-F); combined as li/lj */
        double r = 0.0;
        const int corr = scheme == 1 && c_lap != 0.0;
        if (corr && ex->c_div != 0.0)
            r = c_lap * lap_r + ex->c_div * (-ex->divflux[f]);
        else if (corr)
            r = c_conv != 0.0 ? c_conv * 0.0 + c_lap * lap_r : c_lap * lap_r;
        else if (ex->c_div != 0.0)
            r = ex->c_div * (-ex->divflux[f]);
        li = li * area[f];
        lj = lj * area[f];
        const double ra = r * area[f];
        if (j >= 0) {
            int64_t kii = csr_find(row_ptr, cols, i, (int32_t)i);
            int64_t kij = csr_find(row_ptr, cols, i, (int32_t)j);
            int64_t kji = csr_find(row_ptr, cols, j, (int32_t)i);
            int64_t kjj = csr_find(row_ptr, cols, j, (int32_t)j);
            if (kii < 0 || kij < 0 || kji < 0 || kjj < 0) return OR_ERR_INVALID;
            vals[kii] += li;
            vals[kij] += lj;
            rhs[i] += ra;
            vals[kji] -= li;
            vals[kjj] -= lj;
            rhs[j] -= ra;
        } else {
            if (f < fb0) return OR_ERR_INVALID;
            const double bi = bndi[f - fb0], be = bnde[f - fb0];
            int64_t kii = csr_find(row_ptr, cols, i, (int32_t)i);
            if (kii < 0) return OR_ERR_INVALID;
            vals[kii] += li;
            vals[kii] += lj * bi;
            rhs[i] += ra - lj * be;
        }
    }
    return OR_OK;
}

/* ------------------------------------------------------------ gradients */
/* Matrix::inv (core/matrix.rs:320-380): Gauss-Jordan; a pivot below 1e-14
 * is swapped with the row given by the largest entry of the pivot row. */
static int mat_inv(int n, double a[3][3], double out[3][3]) {
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) out[i][j] = i == j ? 1.0 : 0.0;
    for (int k = 0; k < n - 1; ++k) {
        double piv = a[k][k];
        if (fabs(piv) < 1e-14) {
            int maxi = k;
            double maxp = fabs(piv);
            for (int j = k + 1; j < n; ++j) {
                double pj = fabs(a[k][j]);
                if (pj > maxp) {
                    maxi = j;
                    maxp = pj;
                }
            }
            if (maxi == k) return OR_ERR_INVALID;
            for (int j = 0; j < n; ++j) {
                double t = a[k][j];
                a[k][j] = a[maxi][j];
                a[maxi][j] = t;
                t = out[k][j];
                out[k][j] = out[maxi][j];
                out[maxi][j] = t;
            }
        }
        piv = a[k][k];
        for (int i = k + 1; i < n; ++i) {
            const double f = (-a[i][k]) / piv;
            for (int j = 0; j < n; ++j) {
                a[i][j] += a[k][j] * f;
                out[i][j] += out[k][j] * f;
            }
        }
    }
    for (int k = 0; k < n; ++k) {
        const double piv = a[k][k];
        if (fabs(piv) < 1e-14) return OR_ERR_INVALID;
        for (int j = 0; j < n; ++j) {
            a[k][j] /= piv;
            out[k][j] /= piv;
        }
    }
    for (int k = n - 1; k >= 1; --k) {
        const double piv = a[k][k];
        for (int i = 0; i < k; ++i) {
            const double f = (-a[i][k]) / piv;
            for (int j = 0; j < n; ++j) {
                a[i][j] += a[k][j] * f;
                out[i][j] += out[k][j] * f;
            }
        }
    }
    return OR_OK;
}

static void grad_dgc(int dim, int64_t c, int32_t f, const int32_t *owner, const int32_t *neighbor,
                     const double *face_center, const double *cell_center, double *dgc) {
    const double *p;
    if (neighbor[f] < 0) {
        p = face_center + (int64_t)f * dim;
    } else {
        const int64_t co = neighbor[f] == c ? owner[f] : neighbor[f];
        p = cell_center + co * dim;
    }
    for (int d = 0; d < dim; ++d) dgc[d] = p[d] - cell_center[c * dim + d];
}

/* Gradient coefficients of Mesh::compute (core/mesh/compute.rs:155-203):
 * G = sum_k dgc_k dgc_k^T over the cell's faces in mesh order, g_k = G^-1 dgc_k,
 * own = -sum_k g_k. */
int or_grad_coeffs(int32_t dim, int64_t n_cells, const int32_t *owner, const int32_t *neighbor,
                   const double *face_center, const double *cell_center, const int32_t *cf_ptr,
                   const int32_t *cf, double *gcoef, double *gdiag) {
    for (int64_t c = 0; c < n_cells; ++c) {
        double g[3][3] = {{0}}, gi[3][3], dgc[3];
        for (int32_t k = cf_ptr[c]; k < cf_ptr[c + 1]; ++k) {
            grad_dgc(dim, c, cf[k], owner, neighbor, face_center, cell_center, dgc);
            for (int i = 0; i < dim; ++i)
                for (int j = 0; j < dim; ++j) g[i][j] += dgc[i] * dgc[j];
        }
        if (mat_inv(dim, g, gi) != OR_OK) return OR_ERR_INVALID;
        double own[3] = {0.0, 0.0, 0.0};
        for (int32_t k = cf_ptr[c]; k < cf_ptr[c + 1]; ++k) {
            grad_dgc(dim, c, cf[k], owner, neighbor, face_center, cell_center, dgc);
            for (int i = 0; i < dim; ++i) {
                double x = 0.0;
                for (int j = 0; j < dim; ++j) x += gi[i][j] * dgc[j];
                gcoef[(int64_t)k * dim + i] = x;
                own[i] -= x;
            }
        }
        for (int i = 0; i < dim; ++i) gdiag[c * dim + i] = own[i];
    }
    return OR_OK;
}

/* compute_gradients (fvm/tools/gradients.rs:48-86) of a scalar cell field. */
void or_gradients(int32_t dim, int64_t n_cells, int64_t n_faces, int64_t n_bfaces, const int32_t *owner,
                  const int32_t *neighbor, const int32_t *cf_ptr, const int32_t *cf, const double *gcoef,
                  const double *gdiag, const double *values, const double *bndi, const double *bnde,
                  double *grad) {
    const int64_t fb0 = n_faces - n_bfaces;
    for (int64_t c = 0; c < n_cells; ++c) {
        double g[3];
        for (int d = 0; d < dim; ++d) g[d] = values[c] * gdiag[c * dim + d];
        for (int32_t k = cf_ptr[c]; k < cf_ptr[c + 1]; ++k) {
            const int32_t f = cf[k];
            double w;
            if (neighbor[f] >= 0)
                w = values[neighbor[f] == c ? owner[f] : neighbor[f]];
            else
                w = bndi[f - fb0] * values[c] + bnde[f - fb0];
            for (int d = 0; d < dim; ++d) g[d] += w * gcoef[(int64_t)k * dim + d];
        }
        for (int d = 0; d < dim; ++d) grad[c * dim + d] = g[d];
    }
}

/* -------------------------------------------------------- level-k patterns */
/* The depth-first walks of the reference's level-k patterns: a stack (last
 * pushed first), a visited mark per walk, a path length per pushed node.
 *   mode 0: row_i_u_sparsity (incomplete_lower_upper.rs:30-83)
 *   mode 1: row_i_l_sparsity (incomplete_lower_upper.rs:86-137)
 *   mode 2: row_i_sparsity_edit (incomplete_cholesky.rs:35-85)
 * Appends the nodes the walk collects to out (unsorted), returns their count. */
static int64_t level_walk(int mode, int64_t i, int level, const int32_t *ptr, const int32_t *col, int64_t *mark,
                          int64_t tag, int32_t *dist, int32_t *stack, int32_t *out) {
    int64_t top = 0, cnt = 0;
    stack[top++] = (int32_t)i;
    mark[i] = tag;
    dist[i] = 0;
    while (top > 0) {
        int32_t k = stack[--top];
        int32_t lk = dist[k];
        for (int32_t t = ptr[k]; t < ptr[k + 1]; ++t) {
            int32_t j = col[t];
            if (j == k || mark[j] == tag) continue;
            mark[j] = tag;
            if (mode == 2) {
                if (lk < level) {
                    stack[top++] = j;
                    dist[j] = lk + 1;
                    out[cnt++] = j;
                }
            } else if (mode == 0) {
                if (j < i && lk < level) {
                    stack[top++] = j;
                    dist[j] = lk + 1;
                } else if (j > i) {
                    out[cnt++] = j;
                }
            } else {
                if (j > i && lk < level) {
                    stack[top++] = j;
                    dist[j] = lk + 1;
                } else if (j < i) {
                    out[cnt++] = j;
                }
            }
        }
    }
    return cnt;
}

/* Sorted pattern of the level-k factor (kind 1 = IC, 2 = ILU) of the
 * pattern (ptr, col): two calls, the first with fptr/fcol/fill NULL returns
 * the entry count.  fill[k] = 1 for entries not in the input pattern. */
int64_t or_fill_pattern(int kind, int level, int64_t n, const int32_t *ptr, const int32_t *col, int32_t *fptr,
                        int32_t *fcol, unsigned char *fill) {
    int64_t *mark = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n ? n : 1));
    int32_t *dist = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n ? n : 1));
    int32_t *stack = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n ? n : 1));
    int32_t *row = (int32_t *)malloc(sizeof(int32_t) * (size_t)(2 * n + 2));
    for (int64_t i = 0; i < n; ++i) mark[i] = -1;
    int64_t total = 0;
    if (fptr) fptr[0] = 0;
    for (int64_t i = 0; i < n; ++i) {
        int64_t m = 0;
        if (kind == 2) {
            m += level_walk(1, i, level, ptr, col, mark, 2 * i, dist, stack, row + m);
            row[m++] = (int32_t)i;
            m += level_walk(0, i, level, ptr, col, mark, 2 * i + 1, dist, stack, row + m);
        } else {
            m += level_walk(2, i, level, ptr, col, mark, 2 * i, dist, stack, row + m);
            for (int32_t t = ptr[i]; t < ptr[i + 1]; ++t) row[m++] = col[t];
        }
        qsort(row, (size_t)m, sizeof(int32_t), cmp_i32);
        int64_t u = 0;
        for (int64_t q = 0; q < m; ++q)
            if (q == 0 || row[q] != row[q - 1]) row[u++] = row[q];
        if (fcol) {
            for (int64_t q = 0; q < u; ++q) {
                fcol[total + q] = row[q];
                int in_a = 0;
                for (int32_t t = ptr[i]; t < ptr[i + 1]; ++t) in_a |= col[t] == row[q];
                fill[total + q] = (unsigned char)!in_a;
            }
            fptr[i + 1] = (int32_t)(total + u);
        }
        total += u;
    }
    free(mark);
    free(dist);
    free(stack);
    free(row);
    return total;
}

/* ------------------------------------------------------------- SpMV / dot */
void or_spmv(int64_t n, const int32_t *ptr, const int32_t *col, const double *val, const double *x, double *y) {
    for (int64_t i = 0; i < n; ++i) {
        double s = 0.0;
        for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k) s += val[k] * x[col[k]];
        y[i] = s;
    }
}

double or_dot(int64_t n, const double *a, const double *b) {
    double out = 0.0;
    for (int64_t i = 0; i < n; ++i) out += a[i] * b[i];
    return out;
}

/* ---------------------------------------------------------- preconditioners */
typedef struct or_precond_s {
    int kind;    /* 1 = IC, 2 = ILU, 3 = diagonal, 4 = reordered (wraps `inner`) */
    int64_t n;
    /* reordered: inner is the preconditioner of B = Q A Q^T, perm[i] = the row
     * of A that is row i of B; wr / wz are work vectors in B's numbering */
    int32_t *perm;
    struct or_precond_s *inner;
    double *wr, *wz;
    /* IC: l (lower incl. diag), sp_t (upper pattern), l_vt, inv_diag */
    csr_t l;
    int32_t *spt_ptr, *spt_col;
    double *l_vt, *inv_diag;
    /* ILU: lu (single CSR, unit L implicit) */
    csr_t lu;
    int64_t n_dropped;
} or_precond;

static void csr_free(csr_t *a) {
    free(a->ptr);
    free(a->col);
    free(a->val);
    memset(a, 0, sizeof(*a));
}

void or_precond_free(or_precond *p) {
    if (!p) return;
    if (p->kind == 4) {
        or_precond_free(p->inner);
        free(p->perm);
        free(p->wr);
        free(p->wz);
        free(p);
        return;
    }
    csr_free(&p->l);
    csr_free(&p->lu);
    free(p->spt_ptr);
    free(p->spt_col);
    free(p->l_vt);
    free(p->inv_diag);
    free(p);
}

/* is_symmetric (dmatrix.rs:76-88) with cmp_approx |a-b| < 1e-14 (linalg/mod.rs) */
static int is_symmetric(int64_t n, const int32_t *ptr, const int32_t *col, const double *val) {
    for (int64_t i = 0; i < n; ++i)
        for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k) {
            int32_t j = col[k];
            if (j < n) {
                int64_t kt = csr_find(ptr, col, j, (int32_t)i);
                if (kt < 0) return 0; /* reference panics on the missing index */
                if (!(fabs(val[k] - val[kt]) < 1e-14)) return 0;
            }
        }
    return 1;
}

/* IncompleteCholesky::from_matrix(A, 0): build (incomplete_cholesky.rs:148-202)
 * and compute (:87-145).  Level 0 adds no fill. */
or_precond *or_ic_create_fill(int64_t n, const int32_t *ptr, const int32_t *col, const double *val,
                              const unsigned char *fill, int *status);
or_precond *or_ic0_create(int64_t n, const int32_t *ptr, const int32_t *col, const double *val, int *status) {
    return or_ic_create_fill(n, ptr, col, val, NULL, status);
}

/* IncompleteCholesky::build + compute on a (possibly filled) sorted pattern.
 * fill[k] = 1 marks entries that are fill (zeros, not entries of the
 * matrix): sp_t lists a row's matrix entries first and its fill after them
 * (incomplete_cholesky.rs:167-192), which is the order the backward sweep sums in. */
or_precond *or_ic_create_fill(int64_t n, const int32_t *ptr, const int32_t *col, const double *val,
                              const unsigned char *fill, int *status) {
    *status = OR_OK;
    if (!is_symmetric(n, ptr, col, val)) {
        *status = OR_ERR_NOT_SYMMETRIC;
        return NULL;
    }
    or_precond *p = (or_precond *)calloc(1, sizeof(or_precond));
    p->kind = 1;
    p->n = n;
    int64_t nl = 0, nu = 0;
    for (int64_t i = 0; i < n; ++i)
        for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k) {
            if (col[k] <= i) ++nl;
            if (col[k] >= i) ++nu;
        }
    p->l.n = n;
    p->l.ptr = (int32_t *)malloc(sizeof(int32_t) * (n + 1));
    p->l.col = (int32_t *)malloc(sizeof(int32_t) * (nl ? nl : 1));
    p->l.val = (double *)malloc(sizeof(double) * (nl ? nl : 1));
    p->spt_ptr = (int32_t *)malloc(sizeof(int32_t) * (n + 1));
    p->spt_col = (int32_t *)malloc(sizeof(int32_t) * (nu ? nu : 1));
    p->l_vt = (double *)calloc((size_t)(nl ? nl : 1), sizeof(double));
    p->inv_diag = (double *)calloc((size_t)n, sizeof(double));
    int64_t a = 0, b = 0;
    for (int64_t i = 0; i < n; ++i) {
        p->l.ptr[i] = (int32_t)a;
        p->spt_ptr[i] = (int32_t)b;
        for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k) {
            int32_t j = col[k];
            if (j <= i) {
                p->l.col[a] = j;
                p->l.val[a++] = val[k];
            }
            if (j >= i && !(fill && fill[k])) p->spt_col[b++] = j;
        }
        if (fill)
            for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k)
                if (col[k] >= i && fill[k]) p->spt_col[b++] = col[k];
    }
    p->l.ptr[n] = (int32_t)a;
    p->spt_ptr[n] = (int32_t)b;
    /* compute (right-looking, incomplete_cholesky.rs:87-135) */
    int32_t *lp = p->l.ptr, *lc = p->l.col;
    double *lv = p->l.val;
    for (int64_t k = 0; k < n; ++k) {
        int64_t kk = csr_find(lp, lc, k, (int32_t)k);
        if (kk < 0) {
            *status = OR_ERR_INVALID;
            or_precond_free(p);
            return NULL;
        }
        double lkk = sqrt(lv[kk]);
        double lkkinv = 1.0 / lkk;
        p->inv_diag[k] = lkkinv;
        lv[kk] = lkk;
        for (int32_t q = p->spt_ptr[k]; q < p->spt_ptr[k + 1]; ++q) {
            int32_t i = p->spt_col[q];
            if (i <= k) continue;
            int64_t ki = csr_find(lp, lc, i, (int32_t)k);
            if (ki >= 0) lv[ki] = lkkinv * lv[ki];
        }
        for (int32_t qj = p->spt_ptr[k]; qj < p->spt_ptr[k + 1]; ++qj)
            for (int32_t qi = p->spt_ptr[k]; qi < p->spt_ptr[k + 1]; ++qi) {
                int32_t i = p->spt_col[qi], j = p->spt_col[qj];
                if (i < j) continue;
                if (j <= k) continue;
                int64_t a_ik = csr_find(lp, lc, i, (int32_t)k);
                int64_t a_jk = csr_find(lp, lc, j, (int32_t)k);
                double lik = a_ik >= 0 ? lv[a_ik] : 0.0;
                double ljk = a_jk >= 0 ? lv[a_jk] : 0.0;
                int64_t a_ij = csr_find(lp, lc, i, j);
                if (a_ij >= 0) lv[a_ij] -= lik * ljk;
            }
    }
    /* l_vt: values of l in the transposed (sp_t) order (:138-143) */
    for (int64_t row = 0; row < n; ++row)
        for (int32_t q = lp[row]; q < lp[row + 1]; ++q) {
            int32_t c = lc[q];
            int64_t kt = -1;
            for (int32_t s = p->spt_ptr[c]; s < p->spt_ptr[c + 1]; ++s)
                if (p->spt_col[s] == row) {
                    kt = s;
                    break;
                }
            if (kt < 0) {
                *status = OR_ERR_INVALID;
                or_precond_free(p);
                return NULL;
            }
            p->l_vt[kt] = lv[q];
        }
    return p;
}

/* IncompleteLowerUpper::from_matrix(A, 0): build_and_compute_row_by_row
 * (incomplete_lower_upper.rs:200-261).  For level 0 the L / U sets of row i
 * (row_i_l_sparsity / row_i_u_sparsity, :30-137) are the columns of A's row i
 * below / above the diagonal.  The SparseArray row is held in dense scratch
 * indexed by column; `present` plays the role of contains(). */
or_precond *or_ilu0_create(int64_t n, const int32_t *ptr, const int32_t *col, const double *val, int *status) {
    *status = OR_OK;
    or_precond *p = (or_precond *)calloc(1, sizeof(or_precond));
    p->kind = 2;
    p->n = n;
    const int64_t nnz = ptr[n];
    p->lu.n = n;
    p->lu.ptr = (int32_t *)malloc(sizeof(int32_t) * (n + 1));
    p->lu.col = (int32_t *)malloc(sizeof(int32_t) * (nnz ? nnz : 1));
    p->lu.val = (double *)malloc(sizeof(double) * (nnz ? nnz : 1));
    double *row = (double *)calloc((size_t)n, sizeof(double));
    char *present = (char *)calloc((size_t)n, 1);
    int64_t out = 0;
    p->lu.ptr[0] = 0;
    for (int64_t i = 0; i < n; ++i) {
        for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k) {
            if (col[k] >= n) continue; /* square_block */
            row[col[k]] = val[k];
            present[col[k]] = 1;
        }
        if (!present[i]) { /* lu_row.push(i, matrix.get(i,i)) with a missing diagonal = 0 */
            row[i] = 0.0;
            present[i] = 1;
        }
        for (int32_t q = ptr[i]; q < ptr[i + 1]; ++q) {
            int32_t k = col[q];
            if (k >= i) break;
            int64_t kk = csr_find(p->lu.ptr, p->lu.col, k, k);
            double lukk = kk >= 0 ? p->lu.val[kk] : 0.0;
            if (fabs(lukk) < 1e-16) {
                *status = OR_ERR_SINGULAR;
                free(row);
                free(present);
                or_precond_free(p);
                return NULL;
            }
            double lukkinv = 1.0 / lukk;
            row[k] = lukkinv * row[k];
            double lik = row[k];
            for (int32_t s = p->lu.ptr[k]; s < p->lu.ptr[k + 1]; ++s) {
                int32_t j = p->lu.col[s];
                if (j <= k) continue;
                double term = lik * p->lu.val[s];
                if (!present[j]) continue;
                row[j] -= term;
            }
        }
        /* sparsify_btreeset(|u_ii|*1e-6, {i}) then push_row (sorted) */
        double tol = fabs(row[i]) * 1e-6;
        for (int32_t q = ptr[i]; q < ptr[i + 1]; ++q) {
            int32_t j = col[q];
            if (j >= n || !present[j]) continue;
            if (j == i || fabs(row[j]) > tol) {
                p->lu.col[out] = j;
                p->lu.val[out++] = row[j];
            } else {
                p->n_dropped++;
            }
            present[j] = 0;
            row[j] = 0.0;
        }
        if (present[i]) { /* diagonal absent from A's pattern */
            present[i] = 0;
            row[i] = 0.0;
        }
        p->lu.ptr[i + 1] = (int32_t)out;
    }
    free(row);
    free(present);
    return p;
}

/* DiagonalPreconditioner::from_matrix (preconditioners/mod.rs:44-60):
 * diagonal[i] = matrix[[i, i]].inverse() = 1.0 / a_ii (linalg/mod.rs:48-52);
 * NULL with *status = 1 when a row has no diagonal (the reference panics). */
or_precond *or_diag_create(int64_t n, const int32_t *ptr, const int32_t *col, const double *val, int *status) {
    *status = 0;
    or_precond *p = (or_precond *)calloc(1, sizeof(or_precond));
    p->kind = 3;
    p->n = n;
    p->inv_diag = (double *)malloc(sizeof(double) * (n ? n : 1));
    for (int64_t i = 0; i < n; ++i) {
        const int64_t k = csr_find(ptr, col, i, (int32_t)i);
        if (k < 0) {
            *status = 1;
            or_precond_free(p);
            return NULL;
        }
        p->inv_diag[i] = 1.0 / val[k];
    }
    return p;
}

/* Preconditioner::precondition: IC (incomplete_cholesky.rs:217-255),
 * ILU (incomplete_lower_upper.rs:287-329), diagonal (preconditioners/mod.rs:63-67). */
void or_precond_apply(const or_precond *p, const double *rhs, double *sol) {
    const int64_t n = p->n;
    if (p->kind == 4) { /* z = Q^T M_B^{-1} Q r */
        for (int64_t i = 0; i < n; ++i) p->wr[i] = rhs[p->perm[i]];
        or_precond_apply(p->inner, p->wr, p->wz);
        for (int64_t i = 0; i < n; ++i) sol[p->perm[i]] = p->wz[i];
        return;
    }
    if (p->kind == 3) {
        for (int64_t i = 0; i < n; ++i) sol[i] = p->inv_diag[i] * rhs[i];
        return;
    }
    if (p->kind == 1) {
        for (int64_t i = 0; i < n; ++i) {
            double si = rhs[i];
            for (int32_t k = p->l.ptr[i]; k < p->l.ptr[i + 1]; ++k) {
                int32_t j = p->l.col[k];
                if (i != j) si -= p->l.val[k] * sol[j];
            }
            sol[i] = p->inv_diag[i] * si;
        }
        for (int64_t i = n - 1; i >= 0; --i) {
            double si = sol[i];
            for (int32_t k = p->spt_ptr[i]; k < p->spt_ptr[i + 1]; ++k) {
                int32_t j = p->spt_col[k];
                if (i != j) si -= p->l_vt[k] * sol[j];
            }
            sol[i] = p->inv_diag[i] * si;
        }
    } else {
        for (int64_t i = 0; i < n; ++i) {
            double si = rhs[i];
            for (int32_t k = p->lu.ptr[i]; k < p->lu.ptr[i + 1]; ++k) {
                int32_t j = p->lu.col[k];
                if (j < i) si -= p->lu.val[k] * sol[j];
            }
            sol[i] = si;
        }
        for (int64_t i = n - 1; i >= 0; --i) {
            double si = sol[i];
            for (int32_t k = p->lu.ptr[i]; k < p->lu.ptr[i + 1]; ++k) {
                int32_t j = p->lu.col[k];
                if (j > i) si -= p->lu.val[k] * sol[j];
            }
            int64_t kd = csr_find(p->lu.ptr, p->lu.col, i, (int32_t)i);
            sol[i] = (1.0 / p->lu.val[kd]) * si;
        }
    }
}

/* The reordered preconditioner of the product's perf mode (no counterpart in
 * the reference): `inner` (built on B = Q A Q^T, owned from here on) applied
 * in A's numbering.  perm[i] = the row of A that is row i of B. */
or_precond *or_perm_create(int64_t n, const int32_t *perm, or_precond *inner) {
    if (!inner || inner->n != n) return NULL;
    or_precond *p = (or_precond *)calloc(1, sizeof(or_precond));
    if (!p) return NULL;
    p->kind = 4;
    p->n = n;
    p->inner = inner;
    p->perm = (int32_t *)malloc(sizeof(int32_t) * (n ? n : 1));
    p->wr = (double *)malloc(sizeof(double) * (n ? n : 1));
    p->wz = (double *)malloc(sizeof(double) * (n ? n : 1));
    if (!p->perm || !p->wr || !p->wz) {
        p->inner = NULL;
        or_precond_free(p);
        return NULL;
    }
    memcpy(p->perm, perm, sizeof(int32_t) * n);
    return p;
}

/* Factor export.  IC: l (lower incl. diagonal) and inv_diag.  ILU: lu.
 * Reordered: the factors of B. */
int64_t or_precond_nnz(const or_precond *p) {
    if (p->kind == 4) p = p->inner;
    return p->kind == 1 ? p->l.ptr[p->n] : p->lu.ptr[p->n];
}
int64_t or_precond_ndropped(const or_precond *p) { return p->kind == 4 ? p->inner->n_dropped : p->n_dropped; }
void or_precond_export(const or_precond *p, int32_t *ptr, int32_t *col, double *val, double *inv_diag) {
    if (p->kind == 4) p = p->inner;
    const csr_t *a = p->kind == 1 ? &p->l : &p->lu;
    memcpy(ptr, a->ptr, sizeof(int32_t) * (p->n + 1));
    memcpy(col, a->col, sizeof(int32_t) * a->ptr[p->n]);
    memcpy(val, a->val, sizeof(double) * a->ptr[p->n]);
    if (inv_diag && p->kind == 1) memcpy(inv_diag, p->inv_diag, sizeof(double) * p->n);
}

/* Level schedule of the lower (forward) and upper (backward) triangular DAGs
 * of a pattern: level[i] = 0 when row i has no dependency, else
 * 1 + max(level[j]) over its dependencies (j<i forward, j>i backward). */
int32_t or_levels(int64_t n, const int32_t *ptr, const int32_t *col, int32_t upper, int32_t *level) {
    int32_t nlev = 0;
    if (!upper) {
        for (int64_t i = 0; i < n; ++i) {
            int32_t l = 0;
            for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k)
                if (col[k] < i && level[col[k]] + 1 > l) l = level[col[k]] + 1;
            level[i] = l;
            if (l + 1 > nlev) nlev = l + 1;
        }
    } else {
        for (int64_t i = n - 1; i >= 0; --i) {
            int32_t l = 0;
            for (int32_t k = ptr[i]; k < ptr[i + 1]; ++k)
                if (col[k] > i && col[k] < n && level[col[k]] + 1 > l) l = level[col[k]] + 1;
            level[i] = l;
            if (l + 1 > nlev) nlev = l + 1;
        }
    }
    return nlev;
}

/* ------------------------------------------------------------- Krylov */
typedef struct {
    int64_t iterations;
    double initial_residual;
    double final_residual;
    int64_t history_len;
    int32_t restarts;
} or_info;

static void precond_or_copy(const or_precond *p, int64_t n, const double *r, double *z) {
    if (p)
        or_precond_apply(p, r, z);
    else
        memcpy(z, r, sizeof(double) * n); /* IdentityPreconditioner (preconditioners/mod.rs:22-34) */
}

/* conjugate_gradient (conjugate_gradient.rs:12-111) */
int or_cg(int64_t n, const int32_t *ptr, const int32_t *col, const double *val, const or_precond *p,
          const double *rhs, double *x, double rtol, double atol, int64_t max_iter, double *history,
          int64_t history_cap, or_info *info) {
    memset(info, 0, sizeof(*info));
    const double tolerance = atol, relative_tolerance = rtol;
    const double bnorm = sqrt(or_dot(n, rhs, rhs));
    if (bnorm < 1e-14) {
        for (int64_t i = 0; i < n; ++i) x[i] = 0.0;
        info->initial_residual = bnorm;
        info->final_residual = bnorm;
        if (history_cap > 0) history[0] = bnorm;
        info->history_len = 1;
        return OR_OK;
    }
    double *pv = (double *)calloc((size_t)n, sizeof(double));
    double *r = (double *)calloc((size_t)n, sizeof(double));
    double *z = (double *)calloc((size_t)n, sizeof(double));
    double *ap = (double *)calloc((size_t)n, sizeof(double));
    or_spmv(n, ptr, col, val, x, r);
    for (int64_t i = 0; i < n; ++i) r[i] -= rhs[i];
    for (int64_t i = 0; i < n; ++i) r[i] *= -1.0;
    const double initial_residual = sqrt(or_dot(n, r, r)) / bnorm;
    precond_or_copy(p, n, r, z);
    memcpy(pv, z, sizeof(double) * n);
    double error = 1.0;
    int64_t iter = 0, hl = 0;
    while (error > tolerance) {
        if (iter > max_iter) break;
        or_spmv(n, ptr, col, val, pv, ap);
        const double r_dot_z = or_dot(n, r, z);
        const double p_dot_ap = or_dot(n, pv, ap);
        const double alpha = r_dot_z / p_dot_ap;
        for (int64_t i = 0; i < n; ++i) {
            x[i] += pv[i] * alpha;
            r[i] -= ap[i] * alpha;
        }
        const double r_dot_r = or_dot(n, r, r);
        error = sqrt(r_dot_r) / bnorm;
        if ((error < tolerance) || (error / initial_residual < relative_tolerance)) {
            if (hl < history_cap) history[hl] = error;
            hl++;
            iter++;
            break;
        }
        precond_or_copy(p, n, r, z);
        const double r_dot_z_new = or_dot(n, r, z);
        const double beta = r_dot_z_new / r_dot_z;
        for (int64_t i = 0; i < n; ++i) pv[i] = z[i] + pv[i] * beta;
        if (hl < history_cap) history[hl] = error;
        hl++;
        iter++;
    }
    info->iterations = iter;
    info->initial_residual = initial_residual;
    info->final_residual = error;
    info->history_len = hl;
    free(pv);
    free(r);
    free(z);
    free(ap);
    return OR_OK;
}

/* bi_conjugate_gradient_stab (bi_conjugate_gradient_stab.rs:13-178),
 * right preconditioned, restart when |rho| <= 1e-15*bnorm. */
int or_bicgstab(int64_t n, const int32_t *ptr, const int32_t *col, const double *val, const or_precond *pc,
                const double *rhs, double *x, double rtol, double atol, int64_t max_iter, double *history,
                int64_t history_cap, or_info *info) {
    memset(info, 0, sizeof(*info));
    const double tolerance = atol, relative_tolerance = rtol;
    const double bnorm = sqrt(or_dot(n, rhs, rhs));
    if (bnorm < 1e-14) {
        for (int64_t i = 0; i < n; ++i) x[i] = 0.0;
        info->initial_residual = bnorm;
        info->final_residual = bnorm;
        if (history_cap > 0) history[0] = bnorm;
        info->history_len = 1;
        return OR_OK;
    }
    const size_t sz = sizeof(double) * (size_t)n;
    double *p = (double *)calloc((size_t)n, sizeof(double));
    double *r = (double *)calloc((size_t)n, sizeof(double));
    double *rh = (double *)calloc((size_t)n, sizeof(double));
    double *z = (double *)calloc((size_t)n, sizeof(double));
    double *y = (double *)calloc((size_t)n, sizeof(double));
    double *v = (double *)calloc((size_t)n, sizeof(double));
    double *h = (double *)calloc((size_t)n, sizeof(double));
    double *s = (double *)calloc((size_t)n, sizeof(double));
    double *t = (double *)calloc((size_t)n, sizeof(double));
    or_spmv(n, ptr, col, val, x, r);
    for (int64_t i = 0; i < n; ++i) r[i] -= rhs[i];
    for (int64_t i = 0; i < n; ++i) r[i] *= -1.0;
    memcpy(rh, r, sz);
    const double initial_residual = sqrt(or_dot(n, r, r)) / bnorm;
    int64_t iter = 0, hl = 0;
    double error = 1.0;
    if (initial_residual < tolerance) {
        info->initial_residual = initial_residual;
        info->final_residual = initial_residual;
        if (history_cap > 0) history[0] = initial_residual;
        info->history_len = 1;
        goto done;
    }
    memcpy(p, r, sz);
    double rho = or_dot(n, rh, r);
    while (error > tolerance) {
        if (iter > max_iter) break;
        precond_or_copy(pc, n, p, y);
        or_spmv(n, ptr, col, val, y, v);
        const double rh_dot_v = or_dot(n, rh, v);
        const double alpha = rho / rh_dot_v;
        for (int64_t i = 0; i < n; ++i) {
            h[i] = x[i] + y[i] * alpha;
            s[i] = r[i] - v[i] * alpha;
        }
        const double s_norm = sqrt(or_dot(n, s, s)) / bnorm;
        if ((s_norm < tolerance) || (s_norm / initial_residual < relative_tolerance)) {
            error = s_norm;
            if (hl < history_cap) history[hl] = error;
            hl++;
            memcpy(x, h, sz);
            iter++;
            break;
        }
        precond_or_copy(pc, n, s, z);
        or_spmv(n, ptr, col, val, z, t);
        const double t_dot_s = or_dot(n, t, s);
        const double t_dot_t = or_dot(n, t, t);
        const double omega = t_dot_s / t_dot_t;
        for (int64_t i = 0; i < n; ++i) {
            x[i] = h[i] + z[i] * omega;
            r[i] = s[i] - t[i] * omega;
        }
        const double r_norm = sqrt(or_dot(n, r, r)) / bnorm;
        if ((r_norm < tolerance) || (r_norm / initial_residual < relative_tolerance)) {
            error = r_norm;
            if (hl < history_cap) history[hl] = error;
            hl++;
            iter++;
            break;
        }
        const double rho_new = or_dot(n, rh, r);
        const double beta = (rho_new / rho) * (alpha / omega);
        rho = rho_new;
        if (fabs(rho) > (1e-15 * bnorm)) {
            for (int64_t i = 0; i < n; ++i) p[i] = r[i] + (p[i] - v[i] * omega) * beta;
        } else {
            for (int64_t i = 0; i < n; ++i) {
                rh[i] = r[i];
                p[i] = r[i];
            }
            rho = or_dot(n, rh, r);
            info->restarts++;
        }
        /* the loop guard divides by |b| a second time (:171) */
        error = r_norm / bnorm;
        if (hl < history_cap) history[hl] = error;
        hl++;
        iter++;
    }
    info->iterations = iter;
    info->initial_residual = initial_residual;
    info->final_residual = error;
    info->history_len = hl;
done:
    free(p);
    free(r);
    free(rh);
    free(z);
    free(y);
    free(v);
    free(h);
    free(s);
    free(t);
    return OR_OK;
}
