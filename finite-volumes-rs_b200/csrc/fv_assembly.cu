// Mesh upload, CSR pattern and matrix assembly on the device.
//
// Reference: fvm::assembly::assemble (src/fvm/assembly.rs:11-78), the pattern
// of DistributedMatrix::from_cut_sparsity over Mesh::cell_to_cell
// (src/linalg/dmatrix.rs:38-50, src/core/mesh/compute.rs:135-152), the terms
// laplacian/convection/source (src/fvm/terms/*.rs) with the Orthogonal and
// Upwind schemes (src/fvm/schemes/facengrad/orthogonal.rs:26-46,
// src/fvm/schemes/faceinterp/upwind.rs:26-33).
//
// Design: one thread per cell assembles its whole CSR row.  The cell's faces
// are visited in ascending face id -- the order in which the reference's face
// loop touches that row -- so the diagonal, the off-diagonals and the rhs get
// exactly the reference's sequence of additions, with no atomics and no
// face->nnz map.  A face's coefficients are recomputed by both of its cells
// (identical arithmetic, identical bits); the second read of its data hits L2
// because face ids follow element order.
#include <algorithm>
#include <cub/device/device_scan.cuh>
#include <vector>

#include "fv_internal.cuh"

namespace {

template <int MAXF>
__device__ __forceinline__ int row_pattern(int i, int s, int e, const int32_t *__restrict__ cf_other,
                                           int (&c)[MAXF + 1]) {
    int n = 0;
    c[n++] = i;
    for (int k = s; k < e; ++k) {
        int j = cf_other[k];
        if (j < 0) continue;
        bool dup = false;
        for (int q = 1; q < n; ++q) dup |= (c[q] == j);
        if (!dup && n < MAXF + 1) c[n++] = j;
    }
    for (int a = 1; a < n; ++a) {  // insertion sort, n <= MAXF+1
        int v = c[a];
        int b = a - 1;
        while (b >= 0 && c[b] > v) {
            c[b + 1] = c[b];
            --b;
        }
        c[b + 1] = v;
    }
    return n;
}

template <int MAXF>
__global__ void k_row_count(int64_t n, const int32_t *__restrict__ cf_ptr, const int32_t *__restrict__ cf_other,
                            int32_t *__restrict__ len) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c[MAXF + 1];
    len[i] = row_pattern<MAXF>((int)i, cf_ptr[i], cf_ptr[i + 1], cf_other, c);
}

template <int MAXF>
__global__ void k_row_fill(int64_t n, const int32_t *__restrict__ cf_ptr, const int32_t *__restrict__ cf_other,
                           const int32_t *__restrict__ row_ptr, int32_t *__restrict__ cols) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c[MAXF + 1];
    int m = row_pattern<MAXF>((int)i, cf_ptr[i], cf_ptr[i + 1], cf_other, c);
    int32_t *out = cols + row_ptr[i];
    for (int q = 0; q < m; ++q) out[q] = c[q];
}

struct AssembleArgs {
    int64_t n, fb0;
    const int32_t *cf_ptr, *cf_face, *cf_other;
    const int2 *cf_pad;
    const double4 *cell, *bfc;
    const double *area, *kappa, *flux, *src, *bndi, *bnde;
    double c_lap, c_conv, c_src;
    const int32_t *row_ptr;
    double *vals, *rhs;
    // Corrected scheme
    const double4 *fnorm, *fcen;
    const double *grad;
    double red;
    // time derivative, linear source, divergence
    double c_time, dt, a_next, a_last, a_last_2;
    int time_scheme;
    const double *prev, *prev2, *dens, *densp, *densp2;
    double c_lin, c_div;
    const double *lin, *divflux;
    // Orthogonal scheme with the mesh's cached geometry: (area, 1/|d|) per face, volume per cell
    const double2 *geo;
    const double *vol;
};

// Cell terms of the expression (assembly.rs:26-32): lhs and rhs per unit
// volume.  At most two terms carry a nonzero cell value on each side, so the
// coefficient form equals the term tree's evaluation in any order.
__device__ __forceinline__ void cell_terms(const AssembleArgs &a, int64_t i, double srci, double &l, double &r) {
    double tl = 0.0, tr = 0.0;
    if (a.c_time != 0.0) {
        if (a.time_scheme == FV_TIME_EULER) {  // schemes/time/euler.rs
            const double r0 = a.dens ? a.dens[i] : 1.0, r1 = a.dens ? a.densp[i] : 1.0;
            tl = 1.0 * (1.0 / a.dt) * r0;
            tr = a.prev[i] / a.dt * r1;
        } else {  // schemes/time/backward.rs
            const double r0 = a.dens ? a.dens[i] : 1.0, r1 = a.dens ? a.densp[i] : 1.0,
                         r2 = a.dens ? a.densp2[i] : 1.0;
            tl = 1.0 * (a.a_next / a.dt) * r0;
            tr = (a.prev[i] * a.a_last * r1 - a.prev2[i] * a.a_last_2 * r2) / a.dt;
        }
    }
    const double ll = a.c_lin != 0.0 ? a.lin[i] : 0.0;
    if (a.c_time != 0.0 && a.c_lin != 0.0)
        l = a.c_time * tl + a.c_lin * ll;
    else if (a.c_time != 0.0)
        l = a.c_time * tl;
    else if (a.c_lin != 0.0)
        l = a.c_lin * ll;
    else
        l = 0.0;
    const double sr = -srci;  // Source::cell_terms rhs
    if (a.c_time != 0.0 && a.c_src != 0.0)
        r = a.c_time * tr + a.c_src * sr;
    else if (a.c_time != 0.0)
        r = a.c_time * tr;
    else if (a.c_src != 0.0)
        r = a.c_src * sr;
    else
        r = 0.0;
}

// Face rhs of the expression: the Corrected laplacian's -(kappa * explicit)
// (lap_r) and the divergence's -F, combined like li / lj.
__device__ __forceinline__ double face_rhs(const AssembleArgs &a, bool corr, double lap_r, int f) {
    const bool has_div = a.c_div != 0.0;
    if (corr && has_div) return a.c_lap * lap_r + a.c_div * (-a.divflux[f]);
    if (corr) return (a.c_conv != 0.0) ? a.c_conv * 0.0 + a.c_lap * lap_r : a.c_lap * lap_r;
    if (has_div) return a.c_div * (-a.divflux[f]);
    return 0.0;
}

// Face coefficients (li, lj) before the area factor, exactly as the
// reference's term tree evaluates them.
__device__ __forceinline__ void face_terms(double t, double kappa, double F, double c_lap, double c_conv,
                                           double &li, double &lj) {
    double lap0 = 0.0, lap1 = 0.0, conv0 = 0.0, conv1 = 0.0;
    if (c_lap != 0.0) {
        lap0 = kappa * (-t);
        lap1 = kappa * t;
    }
    if (c_conv != 0.0) {
        if (F > 0.0) {
            conv0 = 1.0 * F;
            conv1 = 0.0 * F;
        } else {
            conv0 = 0.0 * F;
            conv1 = 1.0 * F;
        }
    }
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
}

// ------------------------------------------------------------ gradients
// Vector of the face from cell c to the other cell (or to the boundary face
// centre), as Mesh::compute forms it (compute.rs:165-177).
template <int DIM>
__device__ __forceinline__ void grad_dgc(int c, int f, const double4 *__restrict__ cell, const int2 *__restrict__ fc,
                                         const double4 *__restrict__ fcen, double xc[3], double dgc[3]) {
    const int2 on = fc[f];
    double4 p;
    if (on.y < 0) {
        p = fcen[f];
    } else {
        const int co = on.y == c ? on.x : on.y;
        p = cell[co];
    }
    dgc[0] = p.x - xc[0];
    dgc[1] = p.y - xc[1];
    dgc[2] = DIM == 3 ? p.z - xc[2] : 0.0;
}

// Matrix::inv (core/matrix.rs:320-380): Gauss-Jordan with the reference's
// pivot rule (a pivot below 1e-14 is swapped with the row whose entry in the
// pivot row is largest).  Returns false for a singular matrix.
template <int N>
__device__ __forceinline__ bool mat_inv(double (&a)[N][N], double (&out)[N][N]) {
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) out[i][j] = i == j ? 1.0 : 0.0;
#pragma unroll
    for (int k = 0; k < N - 1; ++k) {
        double piv = a[k][k];
        if (fabs(piv) < 1e-14) {
            int maxi = k;
            double maxp = fabs(piv);
#pragma unroll
            for (int j = k + 1; j < N; ++j) {
                const double pj = fabs(a[k][j]);
                if (pj > maxp) {
                    maxi = j;
                    maxp = pj;
                }
            }
            if (maxi == k) return false;
#pragma unroll
            for (int r = k + 1; r < N; ++r)
                if (r == maxi)
#pragma unroll
                    for (int j = 0; j < N; ++j) {
                        double t = a[k][j];
                        a[k][j] = a[r][j];
                        a[r][j] = t;
                        t = out[k][j];
                        out[k][j] = out[r][j];
                        out[r][j] = t;
                    }
        }
        piv = a[k][k];
#pragma unroll
        for (int i = k + 1; i < N; ++i) {
            const double f = (-a[i][k]) / piv;
#pragma unroll
            for (int j = 0; j < N; ++j) {
                a[i][j] += a[k][j] * f;
                out[i][j] += out[k][j] * f;
            }
        }
    }
#pragma unroll
    for (int k = 0; k < N; ++k) {
        const double piv = a[k][k];
        if (fabs(piv) < 1e-14) return false;
#pragma unroll
        for (int j = 0; j < N; ++j) {
            a[k][j] /= piv;
            out[k][j] /= piv;
        }
    }
#pragma unroll
    for (int k = N - 1; k >= 1; --k) {
        const double piv = a[k][k];
#pragma unroll
        for (int i = 0; i < k; ++i) {
            const double f = (-a[i][k]) / piv;
#pragma unroll
            for (int j = 0; j < N; ++j) {
                a[i][j] += a[k][j] * f;
                out[i][j] += out[k][j] * f;
            }
        }
    }
    return true;
}

// Gradient coefficients of Mesh::compute (compute.rs:155-203), one cell per thread.
template <int DIM>
__global__ void k_grad_coeffs(int64_t n, const double4 *__restrict__ cell, const int2 *__restrict__ fc,
                              const double4 *__restrict__ fcen, const int32_t *__restrict__ gptr,
                              const int32_t *__restrict__ gface, double4 *__restrict__ gcoef,
                              double4 *__restrict__ gdiag, int *bad) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const double4 x4 = cell[c];
    double xc[3] = {x4.x, x4.y, x4.z};
    double g[DIM][DIM];
#pragma unroll
    for (int i = 0; i < DIM; ++i)
#pragma unroll
        for (int j = 0; j < DIM; ++j) g[i][j] = 0.0;
    const int s = gptr[c], e = gptr[c + 1];
    for (int k = s; k < e; ++k) {
        double d[3];
        grad_dgc<DIM>((int)c, gface[k], cell, fc, fcen, xc, d);
#pragma unroll
        for (int i = 0; i < DIM; ++i)
#pragma unroll
            for (int j = 0; j < DIM; ++j) g[i][j] += d[i] * d[j];
    }
    double gi[DIM][DIM];
    if (!mat_inv<DIM>(g, gi)) {
        atomicOr(bad, 1);
        return;
    }
    double own[3] = {0.0, 0.0, 0.0};
    for (int k = s; k < e; ++k) {
        double d[3], v[3] = {0.0, 0.0, 0.0};
        grad_dgc<DIM>((int)c, gface[k], cell, fc, fcen, xc, d);
#pragma unroll
        for (int i = 0; i < DIM; ++i) {
            double x = 0.0;
#pragma unroll
            for (int j = 0; j < DIM; ++j) x += gi[i][j] * d[j];
            v[i] = x;
            own[i] -= x;
        }
        gcoef[k] = make_double4(v[0], v[1], v[2], 0.0);
    }
    gdiag[c] = make_double4(own[0], own[1], own[2], 0.0);
}

// compute_gradients (gradients.rs:48-86) for a scalar field, one cell per thread.
template <int DIM>
__global__ void k_gradients(int64_t n, int64_t fb0, const double *__restrict__ val, const int2 *__restrict__ fc,
                            const int32_t *__restrict__ gptr, const int32_t *__restrict__ gface,
                            const double4 *__restrict__ gcoef, const double4 *__restrict__ gdiag,
                            const double *__restrict__ bndi, const double *__restrict__ bnde,
                            double *__restrict__ grad) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const double vc = val[c];
    const double4 o = gdiag[c];
    double g[3] = {vc * o.x, vc * o.y, DIM == 3 ? vc * o.z : 0.0};
    for (int k = gptr[c]; k < gptr[c + 1]; ++k) {
        const int f = gface[k];
        const int2 on = fc[f];
        double w;
        if (on.y >= 0) {
            w = val[on.y == (int)c ? on.x : on.y];
        } else {
            w = bndi[f - fb0] * vc + bnde[f - fb0];
        }
        const double4 q = gcoef[k];
        g[0] += w * q.x;
        g[1] += w * q.y;
        if (DIM == 3) g[2] += w * q.z;
    }
#pragma unroll
    for (int d = 0; d < DIM; ++d) grad[c * DIM + d] = g[d];
}

template <int DIM, int MAXF>
__global__ void __launch_bounds__(128) k_assemble(AssembleArgs a) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int s = a.cf_ptr[i], e = a.cf_ptr[i + 1];
    int c[MAXF + 1];
    const int m = row_pattern<MAXF>((int)i, s, e, a.cf_other, c);
    double v[MAXF + 1];
#pragma unroll
    for (int q = 0; q < MAXF + 1; ++q) v[q] = 0.0;
    int pd = 0;
    for (int q = 0; q < m; ++q)
        if (c[q] == (int)i) pd = q;
    const double4 ci4 = a.cell[i];
    const double V = ci4.w;
    double lcell, rcell;  // cell loop (assembly.rs:26-32)
    cell_terms(a, i, a.c_src != 0.0 ? a.src[i] : 0.0, lcell, rcell);
    double diag = lcell * V;
    double rhs = rcell * V;
    for (int k = s; k < e; ++k) {
        const int32_t fe = a.cf_face[k];
        const bool is_nb = fe < 0;
        const int f = fe & 0x7fffffff;
        const int j = a.cf_other[k];
        double3 pi, pj;  // owner centre, neighbour centre (or boundary face centre)
        if (j >= 0) {
            const double4 o4 = a.cell[j];
            if (is_nb) {
                pi = make_double3(o4.x, o4.y, o4.z);
                pj = make_double3(ci4.x, ci4.y, ci4.z);
            } else {
                pi = make_double3(ci4.x, ci4.y, ci4.z);
                pj = make_double3(o4.x, o4.y, o4.z);
            }
        } else {
            const double4 b4 = a.bfc[f - a.fb0];
            pi = make_double3(ci4.x, ci4.y, ci4.z);
            pj = make_double3(b4.x, b4.y, b4.z);
        }
        double d2 = 0.0;
        {
            double dd = pj.x - pi.x;
            d2 += dd * dd;
            dd = pj.y - pi.y;
            d2 += dd * dd;
            if (DIM == 3) {
                dd = pj.z - pi.z;
                d2 += dd * dd;
            }
        }
        const double t = 1.0 / sqrt(d2);
        double li, lj;
        face_terms(t, a.c_lap != 0.0 ? a.kappa[f] : 0.0, a.c_conv != 0.0 ? a.flux[f] : 0.0, a.c_lap, a.c_conv,
                   li, lj);
        const double A = a.area[f];
        li = li * A;
        lj = lj * A;
        const double ra = face_rhs(a, false, 0.0, f) * A;
        if (j < 0) {
            const double bi = a.bndi[f - a.fb0], be = a.bnde[f - a.fb0];
            diag += li;
            diag += lj * bi;
            rhs += ra - lj * be;
        } else {
            int pj_slot = 0;
            for (int q = 0; q < m; ++q)
                if (c[q] == j) pj_slot = q;
            if (!is_nb) {  // this cell owns the face: lhs[[i,i]] += li; lhs[[i,j]] += lj; rhs[i] += r
                diag += li;
                for (int q = 0; q < MAXF + 1; ++q)
                    if (q == pj_slot) v[q] += lj;
                rhs += ra;
            } else {  // neighbour side: lhs[[j,i]] -= li; lhs[[j,j]] -= lj; rhs[j] -= r
                for (int q = 0; q < MAXF + 1; ++q)
                    if (q == pj_slot) v[q] -= li;
                diag -= lj;
                rhs -= ra;
            }
        }
    }
    double *out = a.vals + a.row_ptr[i];
    for (int q = 0; q < m; ++q) out[q] = (q == pd) ? diag : v[q];
    a.rhs[i] = rhs;
}

// The same row arithmetic with every per-face quantity in registers (MAXF is
// small: 4 for triangles and tetrahedra, 8 up to hexahedra).  All gathers of a
// cell (incidences, face data, the other cells' centres) are issued before any
// of them is used, the slot of each neighbour in the sorted row is a count of
// smaller distinct neighbours instead of a sort, and the block's rows are
// staged in shared memory so the stores of the values are coalesced.  Each
// output value receives the same additions in the same order as in k_assemble.
constexpr int kAsmBlock = 128;

// The cell's incidences, padded to MAXF slots (jj = -2 marks a pad): the
// degree, and pads turned into jj = -1.
template <int MAXF>
__device__ __forceinline__ int unpad(int (&jj)[MAXF]) {
    int deg = 0;
#pragma unroll
    for (int k = 0; k < MAXF; ++k) deg += jj[k] != -2 ? 1 : 0;
#pragma unroll
    for (int k = 0; k < MAXF; ++k)
        if (jj[k] == -2) jj[k] = -1;
    return deg;
}

// The values of row i (one cell): every gather of the cell is issued before
// any of them is used, the slot of each neighbour in the sorted row is a count
// of smaller distinct neighbours instead of a sort, and the row is written to
// the block's staging area (stage[row_ptr[i] - base ...]) so the stores of the
// values are coalesced.  fe / jj: the cell's incidences (face id with the
// neighbour-side bit, the other cell or -1), deg of them.
//
// GEO (Orthogonal scheme only): 1/|d| of every face comes from the mesh's
// cached a.geo (k_face_invd: the same expression, evaluated once per face) and
// the cell's volume is V, so no cell centre is gathered.
template <int DIM, int MAXF, bool CORR, bool GEO = false>
__device__ __forceinline__ void row_values(const AssembleArgs &a, int64_t i, bool live, const int (&fe)[MAXF],
                                           const int (&jj)[MAXF], int deg, const double4 &ci4, double srci,
                                           double *stage, int base, double Vgeo = 0.0) {
    static_assert(!(GEO && CORR), "cached geometry serves the Orthogonal scheme");
    double3 oc[MAXF];
    double ar[MAXF], kp[MAXF], fl[MAXF], tv[MAXF];
#pragma unroll
    for (int k = 0; k < MAXF; ++k) {
        oc[k] = make_double3(0.0, 0.0, 0.0);
        ar[k] = kp[k] = fl[k] = tv[k] = 0.0;
        if (k < deg) {
            const int f = fe[k] & 0x7fffffff;
            if (GEO) {
                const double2 g = a.geo[f];  // area and 1/|d| in one load
                ar[k] = g.x;
                tv[k] = g.y;
            } else {
                ar[k] = a.area[f];
            }
            if (a.c_lap != 0.0) kp[k] = a.kappa[f];
            if (a.c_conv != 0.0) fl[k] = a.flux[f];
            if (!GEO) {
                const double4 o = jj[k] >= 0 ? a.cell[jj[k]] : a.bfc[f - a.fb0];
                oc[k] = make_double3(o.x, o.y, o.z);
            }
        }
    }
    // distinct neighbours: the first incidence of each other cell carries its slot
    bool first[MAXF];
    int ndist = 0, pd = 0;
#pragma unroll
    for (int k = 0; k < MAXF; ++k) {
        bool f1 = jj[k] >= 0;
#pragma unroll
        for (int q = 0; q < k; ++q) f1 = f1 && (jj[q] != jj[k]);
        first[k] = f1;
        ndist += f1 ? 1 : 0;
        pd += (f1 && jj[k] < (int)i) ? 1 : 0;
    }
    const double V = GEO ? Vgeo : ci4.w;
    double lcell = 0.0, rcell = 0.0;  // cell loop (assembly.rs:26-32)
    if (live) cell_terms(a, i, srci, lcell, rcell);
    double diag = lcell * V;
    double rhs = rcell * V;
    double acc[MAXF];
#pragma unroll
    for (int k = 0; k < MAXF; ++k) acc[k] = 0.0;
#pragma unroll
    for (int k = 0; k < MAXF; ++k) {
        if (k < deg) {
            const bool is_nb = fe[k] < 0;
            double3 pi, pj;
            if (jj[k] >= 0 && is_nb) {
                pi = make_double3(oc[k].x, oc[k].y, oc[k].z);
                pj = make_double3(ci4.x, ci4.y, ci4.z);
            } else {
                pi = make_double3(ci4.x, ci4.y, ci4.z);
                pj = make_double3(oc[k].x, oc[k].y, oc[k].z);
            }
            double t, rsch = 0.0;
            if (GEO) {
                t = tv[k];
            } else if (!CORR) {  // Orthogonal (orthogonal.rs:26-46): 1/|d|
                double d2 = 0.0;
                double dd = pj.x - pi.x;
                d2 += dd * dd;
                dd = pj.y - pi.y;
                d2 += dd * dd;
                if (DIM == 3) {
                    dd = pj.z - pi.z;
                    d2 += dd * dd;
                }
                t = 1.0 / sqrt(d2);
            } else {  // Corrected (corrected.rs:36-67): 1/(n.d) and the explicit correction
                const int f = fe[k] & 0x7fffffff;
                const double4 n4 = a.fnorm[f];
                const double d0 = pj.x - pi.x, d1 = pj.y - pi.y, d2 = DIM == 3 ? pj.z - pi.z : 0.0;
                double nd = 0.0;
                nd += n4.x * d0;
                nd += n4.y * d1;
                if (DIM == 3) nd += n4.z * d2;
                const double cc = 1.0 / nd;
                const double v0 = n4.x - cc * d0, v1 = n4.y - cc * d1, v2 = DIM == 3 ? n4.z - cc * d2 : 0.0;
                const int own = (jj[k] >= 0 && is_nb) ? jj[k] : (int)i;
                double g0, g1, g2 = 0.0;
                if (jj[k] >= 0) {
                    const int nbr = is_nb ? (int)i : jj[k];
                    const double4 c4 = a.fcen[f];
                    const double e0 = c4.x - pi.x, e1 = c4.y - pi.y, e2 = DIM == 3 ? c4.z - pi.z : 0.0;
                    double en = 0.0, dn = 0.0;
                    en += e0 * n4.x;
                    en += e1 * n4.y;
                    if (DIM == 3) en += e2 * n4.z;
                    dn += d0 * n4.x;
                    dn += d1 * n4.y;
                    if (DIM == 3) dn += d2 * n4.z;
                    const double w = en / dn;
                    g0 = a.grad[(int64_t)own * DIM] * (1.0 - w) + a.grad[(int64_t)nbr * DIM] * w;
                    g1 = a.grad[(int64_t)own * DIM + 1] * (1.0 - w) + a.grad[(int64_t)nbr * DIM + 1] * w;
                    if (DIM == 3) g2 = a.grad[(int64_t)own * DIM + 2] * (1.0 - w) + a.grad[(int64_t)nbr * DIM + 2] * w;
                } else {
                    g0 = a.grad[(int64_t)own * DIM];
                    g1 = a.grad[(int64_t)own * DIM + 1];
                    if (DIM == 3) g2 = a.grad[(int64_t)own * DIM + 2];
                }
                double ex = 0.0;
                ex += g0 * v0;
                ex += g1 * v1;
                if (DIM == 3) ex += g2 * v2;
                t = cc;
                rsch = ex * a.red;
            }
            double li, lj;
            face_terms(t, kp[k], fl[k], a.c_lap, a.c_conv, li, lj);
            const double A = ar[k];
            li = li * A;
            lj = lj * A;
            // face rhs: the Corrected laplacian's -(kappa * explicit), the divergence's -F
            const double r = face_rhs(a, CORR, CORR ? -(kp[k] * rsch) : 0.0, fe[k] & 0x7fffffff);
            const double ra = r * A;
            if (jj[k] < 0) {
                const int fb = (fe[k] & 0x7fffffff) - (int)a.fb0;
                const double bi = a.bndi[fb], be = a.bnde[fb];
                diag += li;
                diag += lj * bi;
                rhs += ra - lj * be;
            } else {
                // the value of this neighbour's slot sits in acc[] of its first incidence
#pragma unroll
                for (int q = 0; q <= k; ++q) {
                    if (first[q] && jj[q] == jj[k]) {
                        if (!is_nb)
                            acc[q] += lj;
                        else
                            acc[q] -= li;
                    }
                }
                if (!is_nb) {
                    diag += li;
                    rhs += ra;
                } else {
                    diag -= lj;
                    rhs -= ra;
                }
            }
        }
    }
    if (live) {
        const int r0 = a.row_ptr[i] - base;
        stage[r0 + pd] = diag;
#pragma unroll
        for (int k = 0; k < MAXF; ++k) {
            if (first[k]) {
                int pos = jj[k] > (int)i ? 1 : 0;
#pragma unroll
                for (int q = 0; q < MAXF; ++q) pos += (first[q] && jj[q] < jj[k]) ? 1 : 0;
                stage[r0 + pos] = acc[k];
            }
        }
        a.rhs[i] = rhs;
    }
    (void)ndist;
}

// One row per thread, each output value receiving the same additions in the
// same order as in k_assemble (MAXF is small: 4 for triangles and
// tetrahedra, 8 up to hexahedra).
template <int DIM, int MAXF, bool CORR>
__global__ void __launch_bounds__(kAsmBlock, MAXF <= 4 ? 6 : 3) k_assemble_reg(AssembleArgs a) {
    extern __shared__ double stage[];  // kAsmBlock * (MAXF + 1) values
    const int64_t b0 = (int64_t)blockIdx.x * kAsmBlock;
    const int64_t i = b0 + threadIdx.x;
    const int64_t bend = min(b0 + (int64_t)kAsmBlock, a.n);
    const int base = a.row_ptr[b0];
    const int top = a.row_ptr[bend];
    const bool live = i < a.n;
    // the cell's incidences, padded to MAXF slots: no dependent load of cf_ptr
    int fe[MAXF], jj[MAXF];
#pragma unroll
    for (int k = 0; k < MAXF; k += 2) {
        int4 q = make_int4(0, -2, 0, -2);
        if (live) q = *reinterpret_cast<const int4 *>(&a.cf_pad[i * MAXF + k]);
        fe[k] = q.x;
        jj[k] = q.y;
        fe[k + 1] = q.z;
        jj[k + 1] = q.w;
    }
    const int deg = unpad<MAXF>(jj);
    double4 ci4 = make_double4(0.0, 0.0, 0.0, 0.0);
    double srci = 0.0;
    if (live) {
        ci4 = a.cell[i];
        if (a.c_src != 0.0) srci = a.src[i];
    }
    row_values<DIM, MAXF, CORR>(a, i, live, fe, jj, deg, ci4, srci, stage, base);
    __syncthreads();
    double *out = a.vals + base;
    for (int q = threadIdx.x; q < top - base; q += kAsmBlock) out[q] = stage[q];
}

__device__ __forceinline__ void asm_cp16(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void asm_cp8(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void asm_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void asm_cp_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Per-thread prefetch slot of one cell: incidences, source, volume.
template <int MAXF>
struct AsmSlot {
    int2 cf[MAXF];
    double src;
    double vol;
};

// The Orthogonal scheme's rows with the mesh's cached geometry, a block
// walking tiles of kAsmBlock cells: while a tile's rows are computed, the
// next tile's incidences, sources and volumes are already on their way into
// shared memory (cp.async, one slot per thread, read back only by the thread
// that copied it), so only the face gathers (area, kappa, flux, 1/|d|) remain
// between a row's start and its values; no cell centre is read and no
// square root is taken.
template <int DIM, int MAXF, int MINB>
__global__ void __launch_bounds__(kAsmBlock, MINB) k_assemble_pipe(AssembleArgs a, int64_t ntiles) {
    extern __shared__ __align__(32) double smem[];
    double *stage = smem;  // kAsmBlock * (MAXF + 1) values
    AsmSlot<MAXF> *slot = reinterpret_cast<AsmSlot<MAXF> *>(smem + kAsmBlock * (MAXF + 1));  // [2][kAsmBlock]
    const bool use_src = a.c_src != 0.0;
    auto prefetch = [&](int64_t tile, int buf) {
        const int64_t c = tile * kAsmBlock + threadIdx.x;
        if (tile < ntiles && c < a.n) {
            AsmSlot<MAXF> &q = slot[buf * kAsmBlock + threadIdx.x];
#pragma unroll
            for (int k = 0; k < MAXF; k += 2) asm_cp16(&q.cf[k], &a.cf_pad[c * MAXF + k]);
            asm_cp8(&q.vol, &a.vol[c]);
            if (use_src) asm_cp8(&q.src, &a.src[c]);
        }
        asm_cp_commit();
    };
    int buf = 0;
    prefetch(blockIdx.x, 0);
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        prefetch(tile + gridDim.x, buf ^ 1);
        asm_cp_wait1();  // this thread's copies of `tile` have landed
        const int64_t b0 = tile * kAsmBlock;
        const int64_t i = b0 + threadIdx.x;
        const int64_t bend = min(b0 + (int64_t)kAsmBlock, a.n);
        const int base = a.row_ptr[b0];
        const int top = a.row_ptr[bend];
        const bool live = i < a.n;
        int fe[MAXF], jj[MAXF];
        const double4 none = make_double4(0.0, 0.0, 0.0, 0.0);
        double srci = 0.0, vol = 0.0;
        const AsmSlot<MAXF> &q = slot[buf * kAsmBlock + threadIdx.x];
#pragma unroll
        for (int k = 0; k < MAXF; ++k) {
            fe[k] = live ? q.cf[k].x : 0;
            jj[k] = live ? q.cf[k].y : -2;
        }
        if (live) {
            vol = q.vol;
            if (use_src) srci = q.src;
        }
        const int deg = unpad<MAXF>(jj);
        row_values<DIM, MAXF, false, true>(a, i, live, fe, jj, deg, none, srci, stage, base, vol);
        __syncthreads();
        double *out = a.vals + base;
        for (int r = threadIdx.x; r < top - base; r += kAsmBlock) out[r] = stage[r];
        __syncthreads();  // the stage is rewritten by the next tile
        buf ^= 1;
    }
}

// 1/|d| of every face with the expression of the assembly kernels (pi the
// owner's centre, pj the neighbour's or the boundary face's), and the cells'
// volumes: the Orthogonal scheme's geometry, cached on the mesh.
template <int DIM>
__global__ void k_face_invd(int64_t nf, int64_t fb0, const int2 *__restrict__ fc, const double4 *__restrict__ cell,
                            const double4 *__restrict__ bfc, const double *__restrict__ area,
                            double2 *__restrict__ geo) {
    for (int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += (int64_t)gridDim.x * blockDim.x) {
        const int2 oc = fc[f];
        const double4 o = cell[oc.x];
        const double4 q = oc.y >= 0 ? cell[oc.y] : bfc[f - fb0];
        const double3 pi = make_double3(o.x, o.y, o.z), pj = make_double3(q.x, q.y, q.z);
        double d2 = 0.0;
        double dd = pj.x - pi.x;
        d2 += dd * dd;
        dd = pj.y - pi.y;
        d2 += dd * dd;
        if (DIM == 3) {
            dd = pj.z - pi.z;
            d2 += dd * dd;
        }
        geo[f] = make_double2(area[f], 1.0 / sqrt(d2));
    }
}

__global__ void k_cell_vol(int64_t n, const double4 *__restrict__ cell, double *__restrict__ vol) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        vol[i] = cell[i].w;
}

template <int DIM, int MAXF, int MINB>
void launch_pipe(const AssembleArgs &a, unsigned G, size_t smem, cudaStream_t st) {
    const size_t smem_p = smem + 2 * kAsmBlock * sizeof(AsmSlot<MAXF>);
    static int per_sm = 0;  // resident blocks per SM (launch bounds, registers, shared memory)
    if (!per_sm) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_assemble_pipe<DIM, MAXF, MINB>, kAsmBlock, smem_p);
        if (per_sm < 1) per_sm = 1;
    }
    int sms = 148, dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned Gp = (unsigned)std::min<int64_t>(G, (int64_t)sms * per_sm);
    fv_note_launch(), k_assemble_pipe<DIM, MAXF, MINB><<<Gp, kAsmBlock, smem_p, st>>>(a, (int64_t)G);
}

template <int DIM, int MAXF>
void launch_assemble(const AssembleArgs &a, cudaStream_t st) {
    if (a.n <= 0) return;  // no rows: nothing to launch
    const int B = kAsmBlock;
    const unsigned G = (unsigned)((a.n + B - 1) / B);
    if constexpr (MAXF <= 8) {
        const size_t smem = sizeof(double) * B * (MAXF + 1);
        if (a.grad) {
            fv_note_launch(), k_assemble_reg<DIM, MAXF, true><<<G, B, smem, st>>>(a);
        } else if (a.cf_pad && a.geo) {
            // 6 blocks/SM at 80 registers measured fastest for tets (8 at 64 spills and is 23 % slower)
            launch_pipe<DIM, MAXF, MAXF <= 4 ? 6 : 3>(a, G, smem, st);
        } else if (a.cf_pad) {
            fv_note_launch(), k_assemble_reg<DIM, MAXF, false><<<G, B, smem, st>>>(a);
        } else {
            fv_note_launch(), k_assemble<DIM, MAXF><<<G, B, 0, st>>>(a);
        }
    } else {
        fv_note_launch(), k_assemble<DIM, MAXF><<<G, B, 0, st>>>(a);
    }
}

}  // namespace

cudaError_t fv_mesh_launch_grad_coeffs(fv_mesh *m, int *dbad, cudaStream_t st) {
    const unsigned G = (unsigned)((m->n_cells + 127) / 128);
    if (m->dim == 2)
        fv_note_launch(), k_grad_coeffs<2><<<G, 128, 0, st>>>(m->n_cells, m->cell, m->face_cells, m->face_center,
                                                               m->gcf_ptr, m->gcf_face, m->gcoef, m->gdiag, dbad);
    else
        fv_note_launch(), k_grad_coeffs<3><<<G, 128, 0, st>>>(m->n_cells, m->cell, m->face_cells, m->face_center,
                                                               m->gcf_ptr, m->gcf_face, m->gcoef, m->gdiag, dbad);
    return cudaGetLastError();
}

#include <atomic>
#include <mutex>
static std::atomic<unsigned long long> g_launches{0};

cudaError_t fv_malloc_async_raw(void **p, size_t bytes, cudaStream_t st) {
    static std::atomic<bool> configured[64];
    static std::mutex mu;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < 64 && !configured[dev].load()) {
        std::lock_guard<std::mutex> g(mu);
        if (!configured[dev].load()) {
            cudaMemPool_t pool;
            if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
                uint64_t keep = UINT64_MAX;
                cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
            }
            configured[dev].store(true);
        }
    }
    return cudaMallocAsync(p, bytes, st);
}
void fv_note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void fv_note_launches(long long delta) { g_launches.fetch_add((unsigned long long)delta, std::memory_order_relaxed); }
unsigned long long fv_launches_now() { return g_launches.load(std::memory_order_relaxed); }
extern "C" uint64_t fv_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

static thread_local char g_last_error[256];
void fv_internal_set_cuda_error(cudaError_t e, const char *what) {
    snprintf(g_last_error, sizeof(g_last_error), "%s: %s", what, cudaGetErrorString(e));
}

void fv_internal_set_error_text(const char *what) { snprintf(g_last_error, sizeof(g_last_error), "%s", what); }

extern "C" const char *fv_last_error(void) { return g_last_error; }

extern "C" const char *fv_status_string(fv_status s) {
    switch (s) {
    case FV_OK: return "FV_OK";
    case FV_ERR_ALLOC: return "FV_ERR_ALLOC";
    case FV_ERR_INVALID: return "FV_ERR_INVALID";
    case FV_ERR_SINGULAR_PIVOT: return "FV_ERR_SINGULAR_PIVOT";
    case FV_ERR_BREAKDOWN: return "FV_ERR_BREAKDOWN";
    case FV_ERR_TIMEOUT: return "FV_ERR_TIMEOUT";
    case FV_ERR_NOT_SYMMETRIC: return "FV_ERR_NOT_SYMMETRIC";
    case FV_ERR_CUDA: return "FV_ERR_CUDA";
    case FV_ERR_UNSUPPORTED: return "FV_ERR_UNSUPPORTED";
    case FV_ERR_COMM: return "FV_ERR_COMM";
    }
    return "FV_ERR_UNKNOWN";
}

extern "C" fv_status fv_mesh_destroy(fv_mesh *m) {
    if (!m) return FV_OK;
    cudaFree(m->face_cells);
    cudaFree(m->face_area);
    cudaFree(m->bface_center);
    cudaFree(m->cell);
    cudaFree(m->cf_ptr);
    cudaFree(m->cf_face);
    cudaFree(m->cf_other);
    cudaFree(m->cf_pad);
    cudaFree(m->face_normal);
    cudaFree(m->face_center);
    cudaFree(m->gcf_ptr);
    cudaFree(m->gcf_face);
    cudaFree(m->gcoef);
    cudaFree(m->gdiag);
    cudaFree(m->face_geo);
    cudaFree(m->cell_vol);
    cudaFree(m->row_ptr);
    cudaFree(m->cols);
    delete m;
    return FV_OK;
}

static fv_status mesh_upload_impl(const fv_mesh_desc *d, void *stream, fv_mesh **out) {
    if (!d || !out || (d->dim != 2 && d->dim != 3) || d->n_cells <= 0 || d->n_faces <= 0 || d->n_boundary_faces < 0 ||
        d->n_boundary_faces > d->n_faces || !d->face_owner || !d->face_neighbor || !d->face_area ||
        !d->cell_center || !d->cell_volume || (d->n_boundary_faces > 0 && !d->face_center) ||
        d->n_cells >= 0x7fffffffLL || d->n_faces >= 0x7fffffffLL)
        return FV_ERR_INVALID;
    *out = nullptr;
    const int dim = d->dim;
    const int64_t N = d->n_cells, F = d->n_faces, Fb = d->n_boundary_faces, fb0 = F - Fb;
    // validate connectivity; boundary faces must be the tail of the face list
    std::vector<int32_t> cnt((size_t)N + 1, 0);
    for (int64_t f = 0; f < F; ++f) {
        int32_t o = d->face_owner[f], nb = d->face_neighbor[f];
        if (o < 0 || o >= N || nb < -1 || nb >= N || nb == o) return FV_ERR_INVALID;
        if ((nb < 0) != (f >= fb0)) return FV_ERR_INVALID;
        cnt[o + 1]++;
        if (nb >= 0) cnt[nb + 1]++;
    }
    for (int64_t c = 0; c < N; ++c) cnt[c + 1] += cnt[c];
    const int64_t ncf = cnt[N];
    std::vector<int32_t> cff((size_t)ncf), cfo((size_t)ncf), fill(cnt.begin(), cnt.end() - 1);
    for (int64_t f = 0; f < F; ++f) {  // ascending face id per cell by construction
        int32_t o = d->face_owner[f], nb = d->face_neighbor[f];
        int32_t k = fill[o]++;
        cff[k] = (int32_t)f;
        cfo[k] = nb;
        if (nb >= 0) {
            k = fill[nb]++;
            cff[k] = (int32_t)f | (int32_t)0x80000000;
            cfo[k] = o;
        }
    }
    int maxf = 0;
    for (int64_t c = 0; c < N; ++c) maxf = std::max(maxf, cnt[c + 1] - cnt[c]);
    if (maxf > 16) return FV_ERR_UNSUPPORTED;
    // optional gradient data: every listed face must touch its cell
    const bool grad_ok = d->face_normal && d->cell_face_ptr && d->cell_faces && d->face_center;
    if (grad_ok) {
        if (d->cell_face_ptr[0] != 0) return FV_ERR_INVALID;
        for (int64_t c = 0; c < N; ++c) {
            if (d->cell_face_ptr[c + 1] < d->cell_face_ptr[c]) return FV_ERR_INVALID;
            for (int32_t k = d->cell_face_ptr[c]; k < d->cell_face_ptr[c + 1]; ++k) {
                const int32_t f = d->cell_faces[k];
                if (f < 0 || f >= F || (d->face_owner[f] != c && d->face_neighbor[f] != c)) return FV_ERR_INVALID;
            }
        }
    }
    const int padf = maxf <= 4 ? 4 : (maxf <= 8 ? 8 : 0);
    std::vector<int2> pad((size_t)(padf ? N * padf : 1), make_int2(0, -2));
    if (padf)
        for (int64_t c = 0; c < N; ++c)
            for (int32_t k = cnt[c]; k < cnt[c + 1]; ++k) pad[(size_t)(c * padf + (k - cnt[c]))] = make_int2(cff[k], cfo[k]);
    std::vector<double4> cell((size_t)N);
    for (int64_t c = 0; c < N; ++c) {
        const double *p = d->cell_center + c * dim;
        cell[c] = make_double4(p[0], p[1], dim == 3 ? p[2] : 0.0, d->cell_volume[c]);
    }
    std::vector<double4> bfc((size_t)(Fb > 0 ? Fb : 1));
    for (int64_t b = 0; b < Fb; ++b) {
        const double *p = d->face_center + (fb0 + b) * dim;
        bfc[b] = make_double4(p[0], p[1], dim == 3 ? p[2] : 0.0, 0.0);
    }
    std::vector<int2> fc((size_t)F);
    for (int64_t f = 0; f < F; ++f) fc[f] = make_int2(d->face_owner[f], d->face_neighbor[f]);

    fv_mesh *m = new fv_mesh();
    m->dim = dim;
    m->n_cells = N;
    m->n_faces = F;
    m->n_bfaces = Fb;
    m->maxf = maxf;
    m->padf = padf;
    m->ncf = ncf;
    cudaStream_t st = fv_stream(stream);
    cudaError_t e = cudaSuccess;
    e = cudaMalloc(&m->face_cells, sizeof(int2) * F);
    if (e == cudaSuccess) e = cudaMalloc(&m->face_area, sizeof(double) * F);
    if (e == cudaSuccess) e = cudaMalloc(&m->bface_center, sizeof(double4) * bfc.size());
    if (e == cudaSuccess) e = cudaMalloc(&m->cell, sizeof(double4) * N);
    if (e == cudaSuccess) e = cudaMalloc(&m->cf_ptr, sizeof(int32_t) * (N + 1));
    if (e == cudaSuccess) e = cudaMalloc(&m->cf_face, sizeof(int32_t) * (ncf ? ncf : 1));
    if (e == cudaSuccess) e = cudaMalloc(&m->cf_other, sizeof(int32_t) * (ncf ? ncf : 1));
    if (e == cudaSuccess) e = cudaMemcpyAsync(m->face_cells, fc.data(), sizeof(int2) * F, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(m->face_area, d->face_area, sizeof(double) * F, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(m->bface_center, bfc.data(), sizeof(double4) * bfc.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(m->cell, cell.data(), sizeof(double4) * N, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(m->cf_ptr, cnt.data(), sizeof(int32_t) * (N + 1), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && ncf)
        e = cudaMemcpyAsync(m->cf_face, cff.data(), sizeof(int32_t) * ncf, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && ncf)
        e = cudaMemcpyAsync(m->cf_other, cfo.data(), sizeof(int32_t) * ncf, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && padf) e = cudaMalloc(&m->cf_pad, sizeof(int2) * N * padf);
    if (e == cudaSuccess && padf)
        e = cudaMemcpyAsync(m->cf_pad, pad.data(), sizeof(int2) * N * padf, cudaMemcpyHostToDevice, st);
    // normals, all face centres and the mesh-order cell faces: gradient
    // coefficients (compute.rs:155-203) for the Corrected scheme
    std::vector<double4> fn4, fc4;
    int gbad = 0;
    int *dbad = nullptr;
    if (e == cudaSuccess && grad_ok) {
        fn4.resize((size_t)F);
        fc4.resize((size_t)F);
        for (int64_t f = 0; f < F; ++f) {
            const double *q = d->face_normal + f * dim, *p = d->face_center + f * dim;
            fn4[f] = make_double4(q[0], q[1], dim == 3 ? q[2] : 0.0, 0.0);
            fc4[f] = make_double4(p[0], p[1], dim == 3 ? p[2] : 0.0, 0.0);
        }
        const int64_t ng = d->cell_face_ptr[N];
        e = cudaMalloc(&m->face_normal, sizeof(double4) * F);
        if (e == cudaSuccess) e = cudaMalloc(&m->face_center, sizeof(double4) * F);
        if (e == cudaSuccess) e = cudaMalloc(&m->gcf_ptr, sizeof(int32_t) * (N + 1));
        if (e == cudaSuccess) e = cudaMalloc(&m->gcf_face, sizeof(int32_t) * (ng ? ng : 1));
        if (e == cudaSuccess) e = cudaMalloc(&m->gcoef, sizeof(double4) * (ng ? ng : 1));
        if (e == cudaSuccess) e = cudaMalloc(&m->gdiag, sizeof(double4) * N);
        if (e == cudaSuccess) e = cudaMalloc(&dbad, sizeof(int));
        if (e == cudaSuccess) e = cudaMemsetAsync(dbad, 0, sizeof(int), st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(m->face_normal, fn4.data(), sizeof(double4) * F, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(m->face_center, fc4.data(), sizeof(double4) * F, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(m->gcf_ptr, d->cell_face_ptr, sizeof(int32_t) * (N + 1), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess && ng)
            e = cudaMemcpyAsync(m->gcf_face, d->cell_faces, sizeof(int32_t) * ng, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = fv_mesh_launch_grad_coeffs(m, dbad, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&gbad, dbad, sizeof(int), cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // host staging vectors go out of scope
    if (dbad) cudaFree(dbad);
    if (e != cudaSuccess) {
        fv_internal_set_cuda_error(e, "fv_mesh_upload");
        fv_mesh_destroy(m);
        return e == cudaErrorMemoryAllocation ? FV_ERR_ALLOC : FV_ERR_CUDA;
    }
    if (gbad) {  // Mesh::compute returns Error::SingularMatrix
        fv_internal_set_error_text("fv_mesh_upload: singular gradient matrix of a cell");
        fv_mesh_destroy(m);
        return FV_ERR_INVALID;
    }
    *out = m;
    return FV_OK;
}

extern "C" fv_status fv_mesh_upload(const fv_mesh_desc *d, void *stream, fv_mesh **out) {
    return fv_host_guard([&] { return mesh_upload_impl(d, stream, out); });
}

extern "C" fv_status fv_compute_gradients(fv_mesh *m, const double *values, const fv_bc_desc *bc, double *grad,
                                          void *stream) {
    if (!m || !values || !grad) return FV_ERR_INVALID;
    if (!m->gcoef) return FV_ERR_UNSUPPORTED;
    if (m->n_bfaces > 0 && (!bc || !bc->bndi || !bc->bnde)) return FV_ERR_INVALID;
    cudaStream_t st = fv_stream(stream);
    const int64_t N = m->n_cells;
    const unsigned G = (unsigned)((N + 127) / 128);
    const double *bi = bc ? bc->bndi : nullptr, *be = bc ? bc->bnde : nullptr;
    if (m->dim == 2)
        fv_note_launch(), k_gradients<2><<<G, 128, 0, st>>>(N, m->n_faces - m->n_bfaces, values, m->face_cells,
                                                             m->gcf_ptr, m->gcf_face, m->gcoef, m->gdiag, bi, be, grad);
    else
        fv_note_launch(), k_gradients<3><<<G, 128, 0, st>>>(N, m->n_faces - m->n_bfaces, values, m->face_cells,
                                                             m->gcf_ptr, m->gcf_face, m->gcoef, m->gdiag, bi, be, grad);
    FV_CUDA_TRY(cudaGetLastError());
    return FV_OK;
}

// CSR pattern of cell_to_cell, rows sorted (DistributedMatrix::from_cut_sparsity).
static fv_status build_pattern(fv_mesh *m, cudaStream_t st) {
    const int64_t N = m->n_cells;
    const int B = 256;
    const unsigned G = (unsigned)((N + B - 1) / B);
    int32_t *len = nullptr;
    FV_CUDA_TRY(cudaMalloc(&m->row_ptr, sizeof(int32_t) * (N + 1)));
    FV_CUDA_TRY(fv_malloc_async(&len, sizeof(int32_t) * (N + 1), st));
    FV_CUDA_TRY(cudaMemsetAsync(len + N, 0, sizeof(int32_t), st));
    const int mf = m->maxf;
    if (mf <= 4)
        fv_note_launch(), k_row_count<4><<<G, B, 0, st>>>(N, m->cf_ptr, m->cf_other, len);
    else if (mf <= 8)
        fv_note_launch(), k_row_count<8><<<G, B, 0, st>>>(N, m->cf_ptr, m->cf_other, len);
    else
        fv_note_launch(), k_row_count<16><<<G, B, 0, st>>>(N, m->cf_ptr, m->cf_other, len);
    FV_CUDA_TRY(cudaGetLastError());
    size_t tmp_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, len, m->row_ptr, (int)(N + 1), st);
    void *tmp = nullptr;
    FV_CUDA_TRY(fv_malloc_async(&tmp, tmp_bytes, st));
    FV_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, len, m->row_ptr, (int)(N + 1), st));
    int32_t nnz = 0;
    FV_CUDA_TRY(cudaMemcpyAsync(&nnz, m->row_ptr + N, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    FV_CUDA_TRY(cudaStreamSynchronize(st));
    cudaFreeAsync(tmp, st);
    cudaFreeAsync(len, st);
    m->nnz = nnz;
    FV_CUDA_TRY(cudaMalloc(&m->cols, sizeof(int32_t) * (nnz ? nnz : 1)));
    if (mf <= 4)
        fv_note_launch(), k_row_fill<4><<<G, B, 0, st>>>(N, m->cf_ptr, m->cf_other, m->row_ptr, m->cols);
    else if (mf <= 8)
        fv_note_launch(), k_row_fill<8><<<G, B, 0, st>>>(N, m->cf_ptr, m->cf_other, m->row_ptr, m->cols);
    else
        fv_note_launch(), k_row_fill<16><<<G, B, 0, st>>>(N, m->cf_ptr, m->cf_other, m->row_ptr, m->cols);
    FV_CUDA_TRY(cudaGetLastError());
    return FV_OK;
}

// The Orthogonal scheme's cached geometry of a mesh (1/|d| per face, volume per
// cell), built on first use.  Meshes are shared by host threads (a server's
// mesh cache), so the build holds a lock and the pointers are published only
// after the kernels have finished.
static fv_status ensure_orth_geometry(fv_mesh *m, cudaStream_t st) {
    static std::mutex lock;
    std::lock_guard<std::mutex> g(lock);
    if (m->face_geo && m->cell_vol) return FV_OK;
    double2 *geo = nullptr;
    double *vol = nullptr;
    cudaError_t e = cudaMalloc(&geo, sizeof(double2) * (m->n_faces ? m->n_faces : 1));
    if (e == cudaSuccess) e = cudaMalloc(&vol, sizeof(double) * (m->n_cells ? m->n_cells : 1));
    if (e == cudaSuccess && m->n_faces) {
        const unsigned G = (unsigned)std::min<int64_t>((m->n_faces + 255) / 256, 148 * 16);
        if (m->dim == 2)
            fv_note_launch(), k_face_invd<2><<<G, 256, 0, st>>>(m->n_faces, m->n_faces - m->n_bfaces, m->face_cells,
                                                                 m->cell, m->bface_center, m->face_area, geo);
        else
            fv_note_launch(), k_face_invd<3><<<G, 256, 0, st>>>(m->n_faces, m->n_faces - m->n_bfaces, m->face_cells,
                                                                 m->cell, m->bface_center, m->face_area, geo);
    }
    if (e == cudaSuccess && m->n_cells) {
        const unsigned G = (unsigned)std::min<int64_t>((m->n_cells + 255) / 256, 148 * 16);
        fv_note_launch(), k_cell_vol<<<G, 256, 0, st>>>(m->n_cells, m->cell, vol);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cudaFree(geo);
        cudaFree(vol);
        fv_internal_set_cuda_error(e, "fv_assemble geometry");
        return e == cudaErrorMemoryAllocation ? FV_ERR_ALLOC : FV_ERR_CUDA;
    }
    m->face_geo = geo;
    m->cell_vol = vol;
    return FV_OK;
}

extern "C" fv_status fv_assemble(fv_mesh *m, const fv_terms_desc *terms, const fv_bc_desc *bc, fv_csr **A,
                                 double *b, void *stream) {
    if (!m || !terms || !A || !b) return FV_ERR_INVALID;
    auto okc = [](double c) { return c == -1.0 || c == 0.0 || c == 1.0; };
    if (!okc(terms->laplacian_coef) || !okc(terms->convection_coef) || !okc(terms->source_coef))
        return FV_ERR_UNSUPPORTED;
    if ((terms->laplacian_coef != 0.0 && !terms->diffusivity) || (terms->convection_coef != 0.0 && !terms->flux) ||
        (terms->source_coef != 0.0 && !terms->source))
        return FV_ERR_INVALID;
    if (m->n_bfaces > 0 && (!bc || !bc->bndi || !bc->bnde)) return FV_ERR_INVALID;
    cudaStream_t st = fv_stream(stream);
    if (m->nnz < 0) FV_TRY(build_pattern(m, st));
    fv_csr *a = *A;
    if (!a) {
        a = new fv_csr();
        a->nrows = a->ncols = m->n_cells;
        a->nnz = m->nnz;
        a->row_ptr = m->row_ptr;
        a->cols = m->cols;
        a->owns_pattern = false;
        a->mesh = m;
        cudaError_t e = cudaMalloc(&a->vals, sizeof(double) * (a->nnz ? a->nnz : 1));
        if (e != cudaSuccess) {
            delete a;
            fv_internal_set_cuda_error(e, "fv_assemble vals");
            return FV_ERR_ALLOC;
        }
        *A = a;
    } else if (a->mesh != m) {
        return FV_ERR_INVALID;
    }
    AssembleArgs args;
    args.n = m->n_cells;
    args.fb0 = m->n_faces - m->n_bfaces;
    args.cf_ptr = m->cf_ptr;
    args.cf_face = m->cf_face;
    args.cf_other = m->cf_other;
    args.cf_pad = m->cf_pad;
    args.cell = m->cell;
    args.bfc = m->bface_center;
    args.area = m->face_area;
    args.kappa = terms->diffusivity;
    args.flux = terms->flux;
    args.src = terms->source;
    args.bndi = bc ? bc->bndi : nullptr;
    args.bnde = bc ? bc->bnde : nullptr;
    args.c_lap = terms->laplacian_coef;
    args.c_conv = terms->convection_coef;
    args.c_src = terms->source_coef;
    args.row_ptr = m->row_ptr;
    args.vals = a->vals;
    args.rhs = b;
    args.fnorm = m->face_normal;
    args.fcen = m->face_center;
    args.grad = nullptr;
    args.red = terms->corrector_reduction;
    args.c_time = terms->time_coef;
    args.time_scheme = terms->time_scheme;
    args.dt = terms->dt;
    args.prev = terms->previous;
    args.prev2 = terms->previous_2;
    args.dens = terms->density;
    args.densp = terms->density_previous;
    args.densp2 = terms->density_previous_2;
    args.c_lin = terms->linear_source_coef;
    args.lin = terms->linear_source;
    args.c_div = terms->divergence_coef;
    args.divflux = terms->divergence_flux;
    args.a_next = args.a_last = args.a_last_2 = 0.0;
    if (args.c_time != 0.0) {
        if ((args.time_scheme != FV_TIME_EULER && args.time_scheme != FV_TIME_BACKWARD) || !args.prev ||
            !(args.dt != 0.0) || (args.time_scheme == FV_TIME_BACKWARD && (!args.prev2 || !(terms->dt_2 != 0.0))) ||
            (args.dens && (!args.densp || (args.time_scheme == FV_TIME_BACKWARD && !args.densp2))))
            return FV_ERR_INVALID;
        if (args.time_scheme == FV_TIME_BACKWARD) {  // Backward::new (backward.rs:23-28); powi(2) is x*x
            const double wn = terms->dt / terms->dt_2;
            args.a_next = (1.0 + 2.0 * wn) / (1.0 + wn);
            args.a_last = ((1.0 + wn) * (1.0 + wn)) / (1.0 + wn);
            args.a_last_2 = (wn * wn) / (1.0 + wn);
        }
    }
    if ((args.c_lin != 0.0 && !args.lin) || (args.c_div != 0.0 && !args.divflux)) return FV_ERR_INVALID;
    if (terms->scheme == FV_SCHEME_CORRECTED && terms->laplacian_coef != 0.0) {
        if (!m->face_normal || !m->cf_pad) return FV_ERR_UNSUPPORTED;
        if (!terms->gradients) return FV_ERR_INVALID;
        args.grad = terms->gradients;
    } else if (terms->scheme != FV_SCHEME_ORTHOGONAL && terms->scheme != FV_SCHEME_CORRECTED) {
        return FV_ERR_INVALID;
    }
    args.geo = nullptr;
    args.vol = nullptr;
    if (!args.grad && m->cf_pad) {
        FV_TRY(ensure_orth_geometry(m, st));
        args.geo = m->face_geo;
        args.vol = m->cell_vol;
    }
    const int mf = m->maxf;
    if (m->dim == 2) {
        if (mf <= 4)
            launch_assemble<2, 4>(args, st);
        else if (mf <= 8)
            launch_assemble<2, 8>(args, st);
        else
            launch_assemble<2, 16>(args, st);
    } else {
        if (mf <= 4)
            launch_assemble<3, 4>(args, st);
        else if (mf <= 8)
            launch_assemble<3, 8>(args, st);
        else
            launch_assemble<3, 16>(args, st);
    }
    FV_CUDA_TRY(cudaGetLastError());
    return FV_OK;
}

extern "C" fv_status fv_assemble_host(fv_mesh *m, const fv_terms_desc *terms, const fv_bc_desc *bc, fv_csr **A,
                                      double *b_host, void *stream) {
    if (!m || !terms || !A || !b_host) return FV_ERR_INVALID;
    cudaStream_t st = fv_stream(stream);
    const int64_t N = m->n_cells, F = m->n_faces, Fb = m->n_bfaces;
    double *buf = nullptr;
    const size_t tot = (size_t)(3 * F + 8 * N + 2 * Fb + N * m->dim);
    FV_CUDA_TRY(fv_malloc_async(&buf, sizeof(double) * tot, st));
    double *dk = buf, *dfl = buf + F, *ds = buf + 2 * F, *db = buf + 2 * F + N, *dbi = buf + 2 * F + 2 * N,
           *dbe = dbi + Fb, *dg = dbe + Fb, *dx = dg + N * m->dim;
    fv_terms_desc t = *terms;
    if (terms->gradients) {
        FV_CUDA_TRY(cudaMemcpyAsync(dg, terms->gradients, sizeof(double) * N * m->dim, cudaMemcpyHostToDevice, st));
        t.gradients = dg;
    }
    // per-cell fields of the time / linear-source terms and the divergence flux
    const double **cellf[6] = {&t.previous, &t.previous_2, &t.density, &t.density_previous,
                               &t.density_previous_2, &t.linear_source};
    for (int q = 0; q < 6; ++q)
        if (*cellf[q]) {
            FV_CUDA_TRY(cudaMemcpyAsync(dx + q * N, *cellf[q], sizeof(double) * N, cudaMemcpyHostToDevice, st));
            *cellf[q] = dx + q * N;
        }
    if (terms->divergence_flux) {
        FV_CUDA_TRY(cudaMemcpyAsync(dx + 6 * N, terms->divergence_flux, sizeof(double) * F, cudaMemcpyHostToDevice,
                                    st));
        t.divergence_flux = dx + 6 * N;
    }
    if (terms->diffusivity) {
        FV_CUDA_TRY(cudaMemcpyAsync(dk, terms->diffusivity, sizeof(double) * F, cudaMemcpyHostToDevice, st));
        t.diffusivity = dk;
    }
    if (terms->flux) {
        FV_CUDA_TRY(cudaMemcpyAsync(dfl, terms->flux, sizeof(double) * F, cudaMemcpyHostToDevice, st));
        t.flux = dfl;
    }
    if (terms->source) {
        FV_CUDA_TRY(cudaMemcpyAsync(ds, terms->source, sizeof(double) * N, cudaMemcpyHostToDevice, st));
        t.source = ds;
    }
    fv_bc_desc bd = {nullptr, nullptr};
    if (bc && Fb > 0) {
        FV_CUDA_TRY(cudaMemcpyAsync(dbi, bc->bndi, sizeof(double) * Fb, cudaMemcpyHostToDevice, st));
        FV_CUDA_TRY(cudaMemcpyAsync(dbe, bc->bnde, sizeof(double) * Fb, cudaMemcpyHostToDevice, st));
        bd.bndi = dbi;
        bd.bnde = dbe;
    }
    fv_status s = fv_assemble(m, &t, bc ? &bd : nullptr, A, db, stream);
    if (s == FV_OK) {
        FV_CUDA_TRY(cudaMemcpyAsync(b_host, db, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
    }
    cudaFreeAsync(buf, st);
    FV_CUDA_TRY(cudaStreamSynchronize(st));
    return s;
}
