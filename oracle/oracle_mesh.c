/*
 * oracle_mesh.c -- TEST AND CPU-BASELINE INFRASTRUCTURE ONLY.
 *
 * The oracle's own input generator: the seeded synthetic meshes of the
 * benchmark configurations (unit square of n x n squares split into two
 * triangles each, unit cube of n^3 hexes split into six Kuhn tetrahedra each,
 * interior nodes jittered) and their seeded fields, built without the product
 * library so that the CPU reference arm never loads it.  The mesh is numbered
 * and measured as the reference does when it reads such an element list:
 *
 *   compute_vtk_faces ..... core/mesh/io.rs:364-486  (faces in discovery order,
 *                           interior first, then boundary faces by sorted marker)
 *   VTK face tables ....... core/mesh/vtk.rs:56-125  (tri kind 5, tet kind 10)
 *   add_face / add_cell ... core/mesh/mod.rs:451-529 (owner = first cell to
 *                           claim a face, neighbour = the second)
 *   calc_face_data ........ core/mesh/compute.rs:267-321 (incl. the 3D normal
 *                           of the last sub-triangle divided by the area)
 *   calc_cell_data ........ core/mesh/compute.rs:325-375
 *   orientation ........... core/mesh/compute.rs:97-131
 *   face diffusivity ...... fvm/schemes/faceinterp/linear.rs:40 weights
 *
 * It restates the same steps as oracle/mesh_ref.py (pure Python, small meshes)
 * in C for benchmark sizes; the CPU suite checks both against the library's
 * host builder bit for bit.  Compiled with -ffp-contract=off: every product
 * and sum is rounded on its own, in the reference's order.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ RNG */
/* splitmix64-seeded xoshiro256**, uniform in [0,1) from the top 53 bits,
 * normal by Box-Muller (cosine branch): the generator the benchmark inputs
 * are specified with. */
typedef struct {
    uint64_t s[4];
} or_rng;

static uint64_t splitmix(uint64_t *x) {
    uint64_t z = (*x += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
static void rng_init(or_rng *r, uint64_t seed) {
    uint64_t x = seed;
    for (int i = 0; i < 4; ++i) r->s[i] = splitmix(&x);
}
static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
static uint64_t rng_next(or_rng *r) {
    uint64_t *s = r->s;
    const uint64_t res = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return res;
}
static double rng_uniform(or_rng *r) { return (double)(rng_next(r) >> 11) * 0x1.0p-53; }
static double rng_normal(or_rng *r) {
    const double u1 = 1.0 - rng_uniform(r);
    const double u2 = rng_uniform(r);
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

/* ------------------------------------------------------------------ mesh */
typedef struct or_mesh {
    int32_t dim;
    int64_t n_nodes, n_cells, n_faces, n_bfaces;
    double *nodes;                         /* n_nodes x dim */
    int32_t *cell_face_ptr, *cell_faces;   /* per cell, the faces in VTK local order */
    int32_t *face_owner, *face_neighbor;   /* -1: boundary */
    double *face_area, *face_normal, *face_center; /* F, F x dim, F x dim */
    double *cell_center, *cell_volume;     /* N x dim, N */
} or_mesh;

void or_mesh_free(or_mesh *m) {
    if (!m) return;
    free(m->nodes);
    free(m->cell_face_ptr);
    free(m->cell_faces);
    free(m->face_owner);
    free(m->face_neighbor);
    free(m->face_area);
    free(m->face_normal);
    free(m->face_center);
    free(m->cell_center);
    free(m->cell_volume);
    free(m);
}

/* VTK local faces (core/mesh/vtk.rs): triangle edges (0,1) (1,2) (2,0);
 * tetrahedron faces (0,2,1) (0,1,3) (1,2,3) (0,3,2). */
static const int TRI_FACES[3][2] = {{0, 1}, {1, 2}, {2, 0}};
static const int TET_FACES[4][3] = {{0, 2, 1}, {0, 1, 3}, {1, 2, 3}, {0, 3, 2}};

/* Open-addressing table from a face's sorted node ids to its discovery id. */
typedef struct {
    uint64_t *k0, *k1;
    int32_t *val;
    uint64_t mask;
} face_table;

static int table_init(face_table *t, int64_t expected) {
    uint64_t cap = 1;
    while (cap < (uint64_t)expected * 2) cap <<= 1;
    t->mask = cap - 1;
    t->k0 = (uint64_t *)malloc(cap * sizeof(uint64_t));
    t->k1 = (uint64_t *)malloc(cap * sizeof(uint64_t));
    t->val = (int32_t *)malloc(cap * sizeof(int32_t));
    if (!t->k0 || !t->k1 || !t->val) return -1;
    for (uint64_t i = 0; i < cap; ++i) t->val[i] = -1;
    return 0;
}
static void table_free(face_table *t) {
    free(t->k0);
    free(t->k1);
    free(t->val);
}
/* Returns the id stored for the key, or stores `fresh` and returns -1. */
static int32_t table_find_or_add(face_table *t, uint64_t k0, uint64_t k1, int32_t fresh) {
    uint64_t h = (k0 * 0x9e3779b97f4a7c15ULL) ^ (k1 * 0xc2b2ae3d27d4eb4fULL);
    h ^= h >> 29;
    for (uint64_t i = h & t->mask;; i = (i + 1) & t->mask) {
        if (t->val[i] < 0) {
            t->k0[i] = k0;
            t->k1[i] = k1;
            t->val[i] = fresh;
            return -1;
        }
        if (t->k0[i] == k0 && t->k1[i] == k1) return t->val[i];
    }
}

static double dotd(const double *a, const double *b, int d) {
    double x = 0.0;
    for (int i = 0; i < d; ++i) x += a[i] * b[i];
    return x;
}

/* Element lists of the two generators (the library's synthetic inputs). */
static int gen_elements(int dim, int n, double jitter, uint64_t seed, or_mesh *m, int32_t **en_out,
                        int *npe_out) {
    const int64_t n1 = n + 1;
    const double h = 1.0 / n;
    or_rng rng;
    rng_init(&rng, seed);
    if (dim == 2) {
        m->n_nodes = n1 * n1;
        m->nodes = (double *)malloc(sizeof(double) * m->n_nodes * 2);
        if (!m->nodes) return -1;
        for (int j = 0; j <= n; ++j)
            for (int i = 0; i <= n; ++i) {
                const int64_t p = (int64_t)j * n1 + i;
                double x = (double)i / n, y = (double)j / n;
                if (i > 0 && i < n && j > 0 && j < n) {
                    x += (2.0 * rng_uniform(&rng) - 1.0) * jitter * h;
                    y += (2.0 * rng_uniform(&rng) - 1.0) * jitter * h;
                }
                m->nodes[p * 2] = x;
                m->nodes[p * 2 + 1] = y;
            }
        const int64_t ne = 2LL * n * n;
        int32_t *en = (int32_t *)malloc(sizeof(int32_t) * ne * 3);
        if (!en) return -1;
        int64_t e = 0;
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const int32_t a = j * (n + 1) + i, b = a + 1, c = a + n + 2, d = a + n + 1;
                const int32_t t[6] = {a, b, c, a, c, d};
                for (int q = 0; q < 6; ++q) en[e * 3 + q] = t[q];
                e += 2;
            }
        m->n_cells = ne;
        *en_out = en;
        *npe_out = 3;
        return 0;
    }
    m->n_nodes = n1 * n1 * n1;
    m->nodes = (double *)malloc(sizeof(double) * m->n_nodes * 3);
    if (!m->nodes) return -1;
    for (int k = 0; k <= n; ++k)
        for (int j = 0; j <= n; ++j)
            for (int i = 0; i <= n; ++i) {
                const int64_t p = ((int64_t)k * n1 + j) * n1 + i;
                double x = (double)i / n, y = (double)j / n, z = (double)k / n;
                if (i > 0 && i < n && j > 0 && j < n && k > 0 && k < n) {
                    x += (2.0 * rng_uniform(&rng) - 1.0) * jitter * h;
                    y += (2.0 * rng_uniform(&rng) - 1.0) * jitter * h;
                    z += (2.0 * rng_uniform(&rng) - 1.0) * jitter * h;
                }
                m->nodes[p * 3] = x;
                m->nodes[p * 3 + 1] = y;
                m->nodes[p * 3 + 2] = z;
            }
    const int64_t ne = 6LL * n * n * n;
    int32_t *en = (int32_t *)malloc(sizeof(int32_t) * ne * 4);
    if (!en) return -1;
    /* Kuhn split: the six monotone corner paths from (0,0,0) to (1,1,1) */
    static const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    const int64_t stride[3] = {1, n1, n1 * n1};
    int64_t e = 0;
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const int64_t base = ((int64_t)k * n1 + j) * n1 + i;
                for (int t = 0; t < 6; ++t) {
                    int64_t v = base;
                    en[e * 4] = (int32_t)v;
                    for (int s = 0; s < 3; ++s) {
                        v += stride[perm[t][s]];
                        en[e * 4 + 1 + s] = (int32_t)v;
                    }
                    ++e;
                }
            }
    m->n_cells = ne;
    *en_out = en;
    *npe_out = 4;
    return 0;
}

/* Which sides of the unit square / cube a generator node lies on (bit mask):
 * a face is a boundary face (marker 0) when all its nodes share a side. */
static unsigned side_mask(int dim, int n, int32_t p) {
    const int64_t n1 = n + 1;
    const int64_t i = p % n1, j = (p / n1) % n1, k = dim == 3 ? p / (n1 * n1) : -1;
    unsigned m = 0;
    if (i == 0) m |= 1u;
    if (i == n) m |= 2u;
    if (j == 0) m |= 4u;
    if (j == n) m |= 8u;
    if (k == 0) m |= 16u;
    if (k == n) m |= 32u;
    return m;
}

static void sort_small(int32_t *a, int k) {
    for (int i = 1; i < k; ++i)
        for (int j = i; j > 0 && a[j - 1] > a[j]; --j) {
            const int32_t t = a[j];
            a[j] = a[j - 1];
            a[j - 1] = t;
        }
}

int or_mesh_generate(int dim, int n, double jitter, uint64_t seed, or_mesh **out) {
    *out = NULL;
    if ((dim != 2 && dim != 3) || n < 1 || (dim == 2 && n > 8192) || (dim == 3 && n > 1000)) return 2;
    or_mesh *m = (or_mesh *)calloc(1, sizeof(or_mesh));
    if (!m) return 1;
    m->dim = dim;
    int32_t *en = NULL;
    int npe = 0;
    if (gen_elements(dim, n, jitter, seed, m, &en, &npe)) {
        free(en);
        or_mesh_free(m);
        return 1;
    }
    const int nlf = dim == 2 ? 3 : 4;   /* faces per element */
    const int fsz = dim == 2 ? 2 : 3;   /* nodes per face */
    const int64_t N = m->n_cells;
    const int64_t bound = N * nlf;      /* upper bound of the face count */
    face_table tab;
    int32_t *disc_nodes = (int32_t *)malloc(sizeof(int32_t) * bound * fsz); /* nodes of face (discovery id) */
    char *is_bnd = (char *)malloc((size_t)bound);
    int32_t *ef = (int32_t *)malloc(sizeof(int32_t) * N * nlf);
    if (!disc_nodes || !is_bnd || !ef || table_init(&tab, bound / 2 + 16)) {
        free(en), free(disc_nodes), free(is_bnd), free(ef);
        table_free(&tab);
        or_mesh_free(m);
        return 1;
    }
    /* compute_vtk_faces: walk the elements in order, a face gets the next id
     * when first met, with its nodes in the discovering element's local order */
    int64_t nf = 0, nb = 0;
    for (int64_t c = 0; c < N; ++c) {
        const int32_t *v = en + c * npe;
        for (int l = 0; l < nlf; ++l) {
            int32_t fn[3], key[3];
            for (int q = 0; q < fsz; ++q) fn[q] = v[dim == 2 ? TRI_FACES[l][q] : TET_FACES[l][q]];
            memcpy(key, fn, sizeof(int32_t) * fsz);
            sort_small(key, fsz);
            const uint64_t k0 = ((uint64_t)(uint32_t)key[0] << 32) | (uint32_t)key[1];
            const uint64_t k1 = fsz == 3 ? (uint64_t)(uint32_t)key[2] : 0;
            int32_t id = table_find_or_add(&tab, k0, k1, (int32_t)nf);
            if (id < 0) {
                id = (int32_t)nf++;
                memcpy(disc_nodes + (int64_t)id * fsz, fn, sizeof(int32_t) * fsz);
                unsigned sm = ~0u;
                for (int q = 0; q < fsz; ++q) sm &= side_mask(dim, n, fn[q]);
                is_bnd[id] = sm != 0;
                nb += is_bnd[id];
            }
            ef[c * nlf + l] = id;
        }
    }
    table_free(&tab);
    free(en);
    /* final numbering: interior faces in discovery order, then the boundary
     * faces of the one marker (0) in discovery order */
    int32_t *u2f = (int32_t *)malloc(sizeof(int32_t) * (nf ? nf : 1));
    if (!u2f) {
        free(disc_nodes), free(is_bnd), free(ef);
        or_mesh_free(m);
        return 1;
    }
    {
        int64_t ni = 0, bi = nf - nb;
        for (int64_t f = 0; f < nf; ++f) u2f[f] = (int32_t)(is_bnd[f] ? bi++ : ni++);
    }
    m->n_faces = nf;
    m->n_bfaces = nb;
    const int64_t F = nf;
    int32_t *face_nodes = (int32_t *)malloc(sizeof(int32_t) * F * fsz);
    m->cell_face_ptr = (int32_t *)malloc(sizeof(int32_t) * (N + 1));
    m->cell_faces = (int32_t *)malloc(sizeof(int32_t) * N * nlf);
    m->face_owner = (int32_t *)malloc(sizeof(int32_t) * F);
    m->face_neighbor = (int32_t *)malloc(sizeof(int32_t) * F);
    m->face_area = (double *)malloc(sizeof(double) * F);
    m->face_normal = (double *)malloc(sizeof(double) * F * dim);
    m->face_center = (double *)malloc(sizeof(double) * F * dim);
    m->cell_center = (double *)malloc(sizeof(double) * N * dim);
    m->cell_volume = (double *)malloc(sizeof(double) * N);
    if (!face_nodes || !m->cell_face_ptr || !m->cell_faces || !m->face_owner || !m->face_neighbor ||
        !m->face_area || !m->face_normal || !m->face_center || !m->cell_center || !m->cell_volume) {
        free(face_nodes), free(u2f), free(disc_nodes), free(is_bnd), free(ef);
        or_mesh_free(m);
        return 1;
    }
    for (int64_t f = 0; f < F; ++f) memcpy(face_nodes + (int64_t)u2f[f] * fsz, disc_nodes + f * fsz, sizeof(int32_t) * fsz);
    free(disc_nodes);
    char *bnd = (char *)malloc((size_t)(F ? F : 1));
    if (!bnd) {
        free(face_nodes), free(u2f), free(is_bnd), free(ef);
        or_mesh_free(m);
        return 1;
    }
    for (int64_t f = 0; f < F; ++f) bnd[u2f[f]] = is_bnd[f];
    free(is_bnd);
    for (int64_t c = 0; c <= N; ++c) m->cell_face_ptr[c] = (int32_t)(c * nlf);
    for (int64_t k = 0; k < N * nlf; ++k) m->cell_faces[k] = u2f[ef[k]];
    free(ef);
    free(u2f);
    /* add_cell: owner = the first cell listing the face, neighbour = the
     * second one unless the face is a boundary face */
    for (int64_t f = 0; f < F; ++f) m->face_owner[f] = m->face_neighbor[f] = -1;
    for (int64_t c = 0; c < N; ++c)
        for (int l = 0; l < nlf; ++l) {
            const int32_t f = m->cell_faces[c * nlf + l];
            if (m->face_owner[f] < 0)
                m->face_owner[f] = (int32_t)c;
            else if (!bnd[f] && m->face_neighbor[f] < 0)
                m->face_neighbor[f] = (int32_t)c;
        }
    free(bnd);
    /* calc_face_data */
    const double *X = m->nodes;
    for (int64_t f = 0; f < F; ++f) {
        const int32_t *fn = face_nodes + f * fsz;
        double c[3] = {0.0, 0.0, 0.0};
        for (int q = 0; q < fsz; ++q)
            for (int d = 0; d < dim; ++d) c[d] += X[(int64_t)fn[q] * dim + d];
        for (int d = 0; d < dim; ++d) c[d] = c[d] / (double)fsz;
        double *nrm = m->face_normal + f * dim, *ctr = m->face_center + f * dim;
        if (dim == 2) {
            const double *n0 = X + (int64_t)fn[0] * 2, *n1 = X + (int64_t)fn[1] * 2;
            const double dn[2] = {n1[0] - n0[0], n1[1] - n0[1]};
            const double dsn[2] = {-dn[1], dn[0]};
            const double area = sqrt(dotd(dsn, dsn, 2));
            m->face_area[f] = area;
            nrm[0] = dsn[0] / area;
            nrm[1] = dsn[1] / area;
            ctr[0] = (n0[0] + n1[0]) * 0.5;
            ctr[1] = (n0[1] + n1[1]) * 0.5;
            continue;
        }
        double center[3] = {0.0, 0.0, 0.0}, normal[3] = {0.0, 0.0, 0.0}, area = 0.0;
        for (int i = 0; i < fsz; ++i) {
            const double *n0 = X + (int64_t)fn[i] * 3;
            const double *n1 = X + (int64_t)fn[i == fsz - 1 ? 0 : i + 1] * 3;
            double d0[3], d1[3], dsn[3];
            for (int k = 0; k < 3; ++k) d0[k] = n0[k] - c[k];
            for (int k = 0; k < 3; ++k) d1[k] = n1[k] - c[k];
            dsn[0] = d0[1] * d1[2] - d0[2] * d1[1];
            dsn[1] = d0[2] * d1[0] - d0[0] * d1[2];
            dsn[2] = d0[0] * d1[1] - d0[1] * d1[0];
            for (int k = 0; k < 3; ++k) dsn[k] = dsn[k] * 0.5;
            const double ai = sqrt(dotd(dsn, dsn, 3));
            area += ai;
            for (int k = 0; k < 3; ++k) normal[k] = dsn[k]; /* overwritten, not summed (Q1) */
            for (int k = 0; k < 3; ++k) center[k] += ((((n0[k] + n1[k]) + c[k]) * 1.0) / 3.0) * ai;
        }
        m->face_area[f] = area;
        for (int k = 0; k < 3; ++k) nrm[k] = normal[k] / area;
        for (int k = 0; k < 3; ++k) ctr[k] = center[k] / area;
    }
    free(face_nodes);
    /* calc_cell_data */
    const double vdiv = dim == 2 ? 2.0 : 3.0, cmul = dim == 2 ? 2.0 : 3.0, cdiv = dim == 2 ? 3.0 : 4.0;
    for (int64_t c = 0; c < N; ++c) {
        const int32_t *cf = m->cell_faces + c * nlf;
        double ave[3] = {0.0, 0.0, 0.0}, ctr[3] = {0.0, 0.0, 0.0}, vol = 0.0;
        for (int l = 0; l < nlf; ++l)
            for (int d = 0; d < dim; ++d) ave[d] += m->face_center[(int64_t)cf[l] * dim + d];
        for (int d = 0; d < dim; ++d) ave[d] = ave[d] / (double)nlf;
        for (int l = 0; l < nlf; ++l) {
            const int64_t f = cf[l];
            double dfc[3];
            for (int d = 0; d < dim; ++d) dfc[d] = m->face_center[f * dim + d] - ave[d];
            const double h = fabs(dotd(dfc, m->face_normal + f * dim, dim));
            const double vi = h * m->face_area[f] / vdiv;
            for (int d = 0; d < dim; ++d) ctr[d] += ((m->face_center[f * dim + d] * cmul + ave[d]) / cdiv) * vi;
            vol += vi;
        }
        m->cell_volume[c] = vol;
        for (int d = 0; d < dim; ++d) m->cell_center[c * dim + d] = ctr[d] / vol;
    }
    /* orientation: normals point from the owner outwards */
    for (int64_t f = 0; f < F; ++f) {
        const double *ip = m->cell_center + (int64_t)m->face_owner[f] * dim;
        double *nrm = m->face_normal + f * dim;
        double dd[3];
        for (int d = 0; d < dim; ++d) dd[d] = m->face_center[f * dim + d] - ip[d];
        if (dotd(nrm, dd, dim) < 0.0)
            for (int d = 0; d < dim; ++d) nrm[d] = nrm[d] * -1.0;
    }
    *out = m;
    return 0;
}

void or_mesh_sizes(const or_mesh *m, int64_t *sizes) {
    sizes[0] = m->dim;
    sizes[1] = m->n_nodes;
    sizes[2] = m->n_cells;
    sizes[3] = m->n_faces;
    sizes[4] = m->n_bfaces;
    sizes[5] = m->cell_face_ptr[m->n_cells];
}

/* Copies the arrays out (any pointer may be NULL). */
void or_mesh_arrays(const or_mesh *m, double *nodes, int32_t *cell_face_ptr, int32_t *cell_faces, int32_t *owner,
                    int32_t *neighbor, double *area, double *normal, double *fcenter, double *ccenter,
                    double *volume) {
    const int64_t d = m->dim, N = m->n_cells, F = m->n_faces;
    if (nodes) memcpy(nodes, m->nodes, sizeof(double) * m->n_nodes * d);
    if (cell_face_ptr) memcpy(cell_face_ptr, m->cell_face_ptr, sizeof(int32_t) * (N + 1));
    if (cell_faces) memcpy(cell_faces, m->cell_faces, sizeof(int32_t) * m->cell_face_ptr[N]);
    if (owner) memcpy(owner, m->face_owner, sizeof(int32_t) * F);
    if (neighbor) memcpy(neighbor, m->face_neighbor, sizeof(int32_t) * F);
    if (area) memcpy(area, m->face_area, sizeof(double) * F);
    if (normal) memcpy(normal, m->face_normal, sizeof(double) * F * d);
    if (fcenter) memcpy(fcenter, m->face_center, sizeof(double) * F * d);
    if (ccenter) memcpy(ccenter, m->cell_center, sizeof(double) * N * d);
    if (volume) memcpy(volume, m->cell_volume, sizeof(double) * N);
}

/* Seeded fields of the benchmark inputs: cell diffusivity kappa0 *
 * exp(sigma * N(0,1)) interpolated to the faces with the Linear weights
 * (linear.rs:40, clamped to [0,1]; a boundary face takes its owner's value),
 * face flux v . n (the mesh's normal), cell source (constant, or U(0,1)). */
int or_fields_generate(const or_mesh *m, uint64_t seed, double kappa0, double sigma, const double *velocity,
                       double source_const, int source_uniform, double *kappa_face, double *flux_face,
                       double *source_cell) {
    const int dim = m->dim;
    if (kappa_face) {
        double *kc = (double *)malloc(sizeof(double) * (m->n_cells ? m->n_cells : 1));
        if (!kc) return 1;
        or_rng rk;
        rng_init(&rk, seed ^ 0x6b617070615f6365ULL);
        for (int64_t c = 0; c < m->n_cells; ++c) kc[c] = kappa0 * exp(sigma * rng_normal(&rk));
        for (int64_t f = 0; f < m->n_faces; ++f) {
            const int32_t o = m->face_owner[f], nb = m->face_neighbor[f];
            if (nb < 0) {
                kappa_face[f] = kc[o];
                continue;
            }
            const double *nv = m->face_normal + f * dim, *fc = m->face_center + f * dim;
            const double *cc = m->cell_center + (int64_t)o * dim, *nc = m->cell_center + (int64_t)nb * dim;
            double num = 0.0, den = 0.0;
            for (int d = 0; d < dim; ++d) num += nv[d] * (nc[d] - fc[d]);
            for (int d = 0; d < dim; ++d) den += nv[d] * (nc[d] - cc[d]);
            double w = num / (den < 1e-14 ? 1e-14 : den);
            w = 0.0 < w ? w : 0.0;
            w = w < 1.0 ? w : 1.0;
            kappa_face[f] = w * kc[o] + (1.0 - w) * kc[nb];
        }
        free(kc);
    }
    if (flux_face)
        for (int64_t f = 0; f < m->n_faces; ++f) {
            double s = 0.0;
            for (int d = 0; d < dim; ++d) s += velocity[d] * m->face_normal[f * dim + d];
            flux_face[f] = s;
        }
    if (source_cell) {
        or_rng rs;
        rng_init(&rs, seed ^ 0x736f757263655f63ULL);
        for (int64_t c = 0; c < m->n_cells; ++c) source_cell[c] = source_uniform ? rng_uniform(&rs) : source_const;
    }
    return 0;
}
