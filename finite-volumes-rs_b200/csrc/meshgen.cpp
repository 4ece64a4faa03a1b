// Host-side mesh construction and synthetic inputs.
//
// This file stands in for the reference's Mesh<DIM> (the caller of the hot
// path): it builds the face/cell numbering exactly as Mesh::read_su2 does and
// computes the geometry exactly as Mesh::compute does, so that the arrays it
// produces are the arrays the reference would hand to assemble().
//
//   compute_vtk_faces ............ core/mesh/io.rs:364-486
//   VTK element face tables ...... core/mesh/vtk.rs:56-125
//   add_face / add_cell owner/nb . core/mesh/mod.rs:451-529
//   face + cell geometry ......... core/mesh/compute.rs:34-69, 267-375
//   normal orientation ........... core/mesh/compute.rs:97-131
//   Normal (half cross product) .. core/vector.rs:302-329
//
// All floating-point expressions keep the reference's operation order and are
// compiled without FP contraction (-ffp-contract=off), so the doubles match
// the Rust build bit for bit.
#include "fv_b200.h"

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <string>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

void fv_internal_set_error_text(const char *what);  // fv_assembly.cu

#define FV_RETURN_IF(expr)            \
    do {                              \
        const fv_status _s = (expr);  \
        if (_s != FV_OK) return _s;   \
    } while (0)

namespace {

// ---------------------------------------------------------------- RNG
// splitmix64-seeded xoshiro256**; uniform doubles from the top 53 bits.
struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed) {
        uint64_t x = seed;
        for (int i = 0; i < 4; ++i) s[i] = splitmix(x);
    }
    static uint64_t splitmix(uint64_t &x) {
        uint64_t z = (x += 0x9e3779b97f4a7c15ULL);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        return z ^ (z >> 31);
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        uint64_t r = rotl(s[1] * 5, 7) * 9;
        uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    double uniform() { return (double)(next() >> 11) * 0x1.0p-53; }
    // Box-Muller, cosine branch only.
    double normal() {
        double u1 = 1.0 - uniform();
        double u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

// ---------------------------------------------------------------- VTK faces
// Local face node tables of core/mesh/vtk.rs:56-125 (same node order).
static int vtk_faces(int kind, const int32_t *n, int32_t *fn, int *fstart) {
    switch (kind) {
    case 5: {  // triangle
        const int t[6] = {n[0], n[1], n[1], n[2], n[2], n[0]};
        for (int i = 0; i < 6; ++i) fn[i] = t[i];
        for (int i = 0; i <= 3; ++i) fstart[i] = 2 * i;
        return 3;
    }
    case 9: {  // quad
        const int t[8] = {n[0], n[1], n[1], n[2], n[2], n[3], n[3], n[0]};
        for (int i = 0; i < 8; ++i) fn[i] = t[i];
        for (int i = 0; i <= 4; ++i) fstart[i] = 2 * i;
        return 4;
    }
    case 10: {  // tetrahedron
        const int t[12] = {n[0], n[2], n[1], n[0], n[1], n[3], n[1], n[2], n[3], n[0], n[3], n[2]};
        for (int i = 0; i < 12; ++i) fn[i] = t[i];
        for (int i = 0; i <= 4; ++i) fstart[i] = 3 * i;
        return 4;
    }
    case 12: {  // hexahedron
        const int t[24] = {n[0], n[3], n[2], n[1], n[4], n[5], n[6], n[7], n[0], n[1], n[5], n[4],
                           n[1], n[2], n[6], n[5], n[2], n[3], n[7], n[6], n[3], n[0], n[4], n[7]};
        for (int i = 0; i < 24; ++i) fn[i] = t[i];
        for (int i = 0; i <= 6; ++i) fstart[i] = 4 * i;
        return 6;
    }
    default:
        return -1;
    }
}

static int vtk_nnodes(int kind) {
    switch (kind) {
    case 5: return 3;
    case 9: return 4;
    case 10: return 4;
    case 12: return 8;
    default: return -1;
    }
}

// ---------------------------------------------------------------- face hash
// Open addressing on the sorted node tuple (up to 4 node ids).
struct FaceKey {
    uint64_t a, b;
    bool operator==(const FaceKey &o) const { return a == o.a && b == o.b; }
};

static FaceKey make_key(const int32_t *nodes, int len) {
    uint32_t s[4] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu};
    for (int i = 0; i < len; ++i) s[i] = (uint32_t)nodes[i];
    std::sort(s, s + len);
    FaceKey k;
    k.a = ((uint64_t)s[0] << 32) | s[1];
    k.b = ((uint64_t)s[2] << 32) | s[3];
    return k;
}

struct FaceTable {
    std::vector<FaceKey> keys;
    std::vector<int32_t> vals;
    uint64_t mask = 0;
    explicit FaceTable(size_t expected) {
        size_t cap = 16;
        while (cap < 2 * expected + 16) cap <<= 1;
        keys.assign(cap, FaceKey{~0ULL, ~0ULL});
        vals.assign(cap, -1);
        mask = cap - 1;
    }
    static uint64_t hash(const FaceKey &k) {
        uint64_t h = k.a * 0x9e3779b97f4a7c15ULL ^ (k.b + 0x632be59bd9b4e019ULL) * 0xc2b2ae3d27d4eb4fULL;
        h ^= h >> 29;
        h *= 0xbf58476d1ce4e5b9ULL;
        h ^= h >> 32;
        return h;
    }
    // Returns the existing value, or inserts v and returns -1.
    int32_t find_or_insert(const FaceKey &k, int32_t v) {
        uint64_t i = hash(k) & mask;
        while (true) {
            if (vals[i] < 0) {
                keys[i] = k;
                vals[i] = v;
                return -1;
            }
            if (keys[i] == k) return vals[i];
            i = (i + 1) & mask;
        }
    }
    int32_t find(const FaceKey &k) const {
        uint64_t i = hash(k) & mask;
        while (true) {
            if (vals[i] < 0) return -1;
            if (keys[i] == k) return vals[i];
            i = (i + 1) & mask;
        }
    }
};

template <class T>
static T *dup_vec(const std::vector<T> &v) {
    T *p = (T *)std::malloc(sizeof(T) * (v.size() ? v.size() : 1));
    if (p && !v.empty()) std::memcpy(p, v.data(), sizeof(T) * v.size());
    return p;
}

// ---------------------------------------------------------------- geometry
// calc_face_data (compute.rs:267-321).
static void face_geometry(int dim, const double *nodes, const int32_t *fn, int len, double *area,
                          double *normal, double *center) {
    double c[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < len; ++i)
        for (int d = 0; d < dim; ++d) c[d] += nodes[(int64_t)fn[i] * dim + d];
    for (int d = 0; d < dim; ++d) c[d] /= (double)len;

    if (dim == 2) {
        const double *n0 = nodes + (int64_t)fn[0] * 2;
        const double *n1 = nodes + (int64_t)fn[1] * 2;
        double dn[2] = {n1[0] - n0[0], n1[1] - n0[1]};
        double dsn[2] = {-dn[1], dn[0]};
        double dd = 0.0;
        dd += dsn[0] * dsn[0];
        dd += dsn[1] * dsn[1];
        double a = std::sqrt(dd);
        *area = a;
        normal[0] = dsn[0] / a;
        normal[1] = dsn[1] / a;
        center[0] = (n0[0] + n1[0]) * 0.5;
        center[1] = (n0[1] + n1[1]) * 0.5;
        return;
    }
    double ctr[3] = {0.0, 0.0, 0.0};
    double nrm[3] = {0.0, 0.0, 0.0};
    double a = 0.0;
    for (int i = 0; i < len; ++i) {
        const double *n0 = nodes + (int64_t)fn[i] * 3;
        const double *n1 = nodes + (int64_t)fn[i == len - 1 ? 0 : i + 1] * 3;
        double d0[3] = {n0[0] - c[0], n0[1] - c[1], n0[2] - c[2]};
        double d1[3] = {n1[0] - c[0], n1[1] - c[1], n1[2] - c[2]};
        double dsn[3];
        dsn[0] = d0[1] * d1[2] - d0[2] * d1[1];
        dsn[1] = d0[2] * d1[0] - d0[0] * d1[2];
        dsn[2] = d0[0] * d1[1] - d0[1] * d1[0];
        for (int d = 0; d < 3; ++d) dsn[d] *= 0.5;
        double dd = 0.0;
        for (int d = 0; d < 3; ++d) dd += dsn[d] * dsn[d];
        double ai = std::sqrt(dd);
        a += ai;
        for (int d = 0; d < 3; ++d) nrm[d] = dsn[d];  // overwritten, not accumulated (compute.rs:305)
        for (int d = 0; d < 3; ++d) {
            double t = n0[d] + n1[d];
            t = t + c[d];
            t = t * 1.0;
            t = t / 3.0;
            t = t * ai;
            ctr[d] += t;
        }
    }
    for (int d = 0; d < 3; ++d) nrm[d] /= a;
    for (int d = 0; d < 3; ++d) ctr[d] /= a;
    *area = a;
    for (int d = 0; d < 3; ++d) {
        normal[d] = nrm[d];
        center[d] = ctr[d];
    }
}

// calc_cell_data (compute.rs:325-375); facec_ave = mean of face centres in cell_faces order.
static void cell_geometry(int dim, const int32_t *cf, int len, const double *farea, const double *fnormal,
                          const double *fcenter, double *center, double *volume) {
    double ave[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < len; ++i)
        for (int d = 0; d < dim; ++d) ave[d] += fcenter[(int64_t)cf[i] * dim + d];
    for (int d = 0; d < dim; ++d) ave[d] /= (double)len;
    const double vdiv = dim == 2 ? 2.0 : 3.0;
    const double cmul = dim == 2 ? 2.0 : 3.0;
    const double cdiv = dim == 2 ? 3.0 : 4.0;
    double ctr[3] = {0.0, 0.0, 0.0};
    double vol = 0.0;
    for (int i = 0; i < len; ++i) {
        const int64_t f = cf[i];
        const double *fc = fcenter + f * dim;
        const double *fnv = fnormal + f * dim;
        double dfc[3];
        for (int d = 0; d < dim; ++d) dfc[d] = fc[d] - ave[d];
        double h = 0.0;
        for (int d = 0; d < dim; ++d) h += dfc[d] * fnv[d];
        h = std::fabs(h);
        double vi = h * farea[f] / vdiv;
        for (int d = 0; d < dim; ++d) {
            double ci = (fc[d] * cmul + ave[d]) / cdiv;
            ctr[d] += ci * vi;
        }
        vol += vi;
    }
    *volume = vol;
    for (int d = 0; d < dim; ++d) center[d] = ctr[d] / vol;
}

// Mesh::compute (compute.rs:12-131) on a host mesh whose topology is set:
// face data, then cell data, then orientation.
void compute_geometry(fv_host_mesh *m) {
    const int dim = m->dim;
    const int64_t F = m->n_faces, N = m->n_cells;
#pragma omp parallel for schedule(static)
    for (int64_t f = 0; f < F; ++f)
        face_geometry(dim, m->nodes, m->face_nodes + m->face_node_ptr[f], m->face_node_ptr[f + 1] - m->face_node_ptr[f],
                      m->face_area + f, m->face_normal + f * dim, m->face_center + f * dim);
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < N; ++c)
        cell_geometry(dim, m->cell_faces + m->cell_face_ptr[c], m->cell_face_ptr[c + 1] - m->cell_face_ptr[c],
                      m->face_area, m->face_normal, m->face_center, m->cell_center + c * dim, m->cell_volume + c);
#pragma omp parallel for schedule(static)
    for (int64_t f = 0; f < F; ++f) {
        const double *ip = m->cell_center + (int64_t)m->face_owner[f] * dim;
        double *nv = m->face_normal + f * dim;
        const double *fc = m->face_center + f * dim;
        double s = 0.0;
        for (int d = 0; d < dim; ++d) s += nv[d] * (fc[d] - ip[d]);
        if (s < 0.0)
            for (int d = 0; d < dim; ++d) nv[d] *= -1.0;
    }
}

}  // namespace

extern "C" void fv_host_mesh_free(fv_host_mesh *m) {
    if (!m) return;
    std::free(m->nodes);
    std::free(m->face_node_ptr);
    std::free(m->face_nodes);
    std::free(m->face_patch);
    std::free(m->cell_face_ptr);
    std::free(m->cell_faces);
    std::free(m->face_owner);
    std::free(m->face_neighbor);
    std::free(m->face_area);
    std::free(m->face_normal);
    std::free(m->face_center);
    std::free(m->cell_center);
    std::free(m->cell_volume);
    std::free(m);
}

extern "C" fv_status fv_host_mesh_from_elements(int32_t dim, int64_t n_nodes, const double *nodes,
                                                int64_t n_elems, const int32_t *elem_kind,
                                                const int32_t *elem_node_ptr, const int32_t *elem_nodes,
                                                int64_t n_bfaces, const int32_t *bface_node_ptr,
                                                const int32_t *bface_nodes, const int32_t *bface_marker,
                                                fv_host_mesh **out) {
    if (!out || (dim != 2 && dim != 3) || n_nodes <= 0 || n_elems <= 0 || !nodes || !elem_kind ||
        !elem_node_ptr || !elem_nodes || n_nodes >= 0x7fffffffLL)
        return FV_ERR_INVALID;
    *out = nullptr;
    try {
        // Boundary face keys -> marker (read_su2_boundaries).
        FaceTable bnd((size_t)(n_bfaces > 0 ? n_bfaces : 1));
        for (int64_t b = 0; b < n_bfaces; ++b) {
            int len = bface_node_ptr[b + 1] - bface_node_ptr[b];
            if (len < 2 || len > 4 || bface_marker[b] < 0) return FV_ERR_INVALID;
            for (int q = 0; q < len; ++q)
                if (bface_nodes[bface_node_ptr[b] + q] < 0 || bface_nodes[bface_node_ptr[b] + q] >= n_nodes)
                    return FV_ERR_INVALID;
            FaceKey k = make_key(bface_nodes + bface_node_ptr[b], len);
            bnd.find_or_insert(k, bface_marker[b]);
        }
        int64_t total_local = 0;
        for (int64_t e = 0; e < n_elems; ++e) {
            int k = elem_kind[e];
            int nn = vtk_nnodes(k);
            if (nn < 0 || elem_node_ptr[e + 1] - elem_node_ptr[e] != nn) return FV_ERR_INVALID;
            if ((dim == 2) != (k == 5 || k == 9)) return FV_ERR_INVALID;
            for (int q = 0; q < nn; ++q) {
                const int32_t id = elem_nodes[elem_node_ptr[e] + q];
                if (id < 0 || id >= n_nodes) return FV_ERR_INVALID;
            }
            total_local += (k == 5 ? 3 : (k == 12 ? 6 : 4));
        }
        if (total_local >= 0x7fffffffLL) return FV_ERR_INVALID;

        // compute_vtk_faces: unique faces in discovery order.
        FaceTable faces((size_t)(total_local / 2 + n_bfaces + 16));
        std::vector<int32_t> elem_face_ptr(n_elems + 1);
        std::vector<int32_t> elem_faces((size_t)total_local);
        std::vector<int64_t> uface_src;    // (element*8 + local face) of the discovering element
        std::vector<int32_t> uface_bnd;    // marker or -1
        uface_src.reserve((size_t)(total_local / 2 + n_bfaces + 16));
        uface_bnd.reserve(uface_src.capacity());
        int32_t fn[24];
        int fs[8];
        int64_t pos = 0;
        for (int64_t e = 0; e < n_elems; ++e) {
            elem_face_ptr[e] = (int32_t)pos;
            int nf = vtk_faces(elem_kind[e], elem_nodes + elem_node_ptr[e], fn, fs);
            for (int l = 0; l < nf; ++l) {
                const int32_t *fi = fn + fs[l];
                int len = fs[l + 1] - fs[l];
                FaceKey k = make_key(fi, len);
                int32_t id = (int32_t)uface_src.size();
                int32_t got = faces.find_or_insert(k, id);
                if (got < 0) {
                    uface_src.push_back(e * 8 + l);
                    uface_bnd.push_back(n_bfaces > 0 ? bnd.find(k) : -1);
                    got = id;
                }
                elem_faces[pos++] = got;
            }
        }
        elem_face_ptr[n_elems] = (int32_t)pos;
        const int64_t n_unique = (int64_t)uface_src.size();

        // Final ids: interior faces in discovery order, then boundary faces
        // grouped by ascending marker id, discovery order within a marker.
        std::vector<int32_t> u2f((size_t)n_unique);
        int64_t n_int = 0;
        std::vector<int32_t> markers;
        for (int64_t i = 0; i < n_unique; ++i) {
            if (uface_bnd[i] < 0)
                u2f[i] = (int32_t)n_int++;
            else
                markers.push_back(uface_bnd[i]);
        }
        std::sort(markers.begin(), markers.end());
        markers.erase(std::unique(markers.begin(), markers.end()), markers.end());
        int64_t running = n_int;
        for (int32_t mk : markers)
            for (int64_t i = 0; i < n_unique; ++i)
                if (uface_bnd[i] == mk) u2f[i] = (int32_t)running++;
        const int64_t F = n_unique;

        fv_host_mesh *m = (fv_host_mesh *)std::calloc(1, sizeof(fv_host_mesh));
        if (!m) return FV_ERR_ALLOC;
        m->dim = dim;
        m->n_nodes = n_nodes;
        m->n_faces = F;
        m->n_cells = n_elems;
        m->n_boundary_faces = F - n_int;
        m->nodes = (double *)std::malloc(sizeof(double) * n_nodes * dim);
        m->face_node_ptr = (int32_t *)std::malloc(sizeof(int32_t) * (F + 1));
        m->face_patch = (int32_t *)std::malloc(sizeof(int32_t) * F);
        m->face_owner = (int32_t *)std::malloc(sizeof(int32_t) * F);
        m->face_neighbor = (int32_t *)std::malloc(sizeof(int32_t) * F);
        m->face_area = (double *)std::malloc(sizeof(double) * F);
        m->face_normal = (double *)std::malloc(sizeof(double) * F * dim);
        m->face_center = (double *)std::malloc(sizeof(double) * F * dim);
        m->cell_face_ptr = (int32_t *)std::malloc(sizeof(int32_t) * (n_elems + 1));
        m->cell_faces = (int32_t *)std::malloc(sizeof(int32_t) * (pos ? pos : 1));
        m->cell_center = (double *)std::malloc(sizeof(double) * n_elems * dim);
        m->cell_volume = (double *)std::malloc(sizeof(double) * n_elems);
        if (!m->nodes || !m->face_node_ptr || !m->face_patch || !m->face_owner || !m->face_neighbor ||
            !m->face_area || !m->face_normal || !m->face_center || !m->cell_face_ptr || !m->cell_faces ||
            !m->cell_center || !m->cell_volume) {
            fv_host_mesh_free(m);
            return FV_ERR_ALLOC;
        }
        std::memcpy(m->nodes, nodes, sizeof(double) * n_nodes * dim);

        // face node lists in final order (first discoverer's local order)
        std::vector<int32_t> f2u((size_t)F);
        for (int64_t i = 0; i < n_unique; ++i) f2u[u2f[i]] = (int32_t)i;
        int64_t fnn = 0;
        m->face_node_ptr[0] = 0;
        for (int64_t f = 0; f < F; ++f) {
            int64_t src = uface_src[f2u[f]];
            int64_t e = src / 8;
            int l = (int)(src % 8);
            vtk_faces(elem_kind[e], elem_nodes + elem_node_ptr[e], fn, fs);
            fnn += fs[l + 1] - fs[l];
            m->face_node_ptr[f + 1] = (int32_t)fnn;
        }
        m->face_nodes = (int32_t *)std::malloc(sizeof(int32_t) * (fnn ? fnn : 1));
        if (!m->face_nodes) {
            fv_host_mesh_free(m);
            return FV_ERR_ALLOC;
        }
        for (int64_t f = 0; f < F; ++f) {
            int64_t src = uface_src[f2u[f]];
            int64_t e = src / 8;
            int l = (int)(src % 8);
            vtk_faces(elem_kind[e], elem_nodes + elem_node_ptr[e], fn, fs);
            std::memcpy(m->face_nodes + m->face_node_ptr[f], fn + fs[l], sizeof(int32_t) * (fs[l + 1] - fs[l]));
            m->face_patch[f] = uface_bnd[f2u[f]];
        }
        // add_cell: owner = first cell listing the face, neighbour = second.
        for (int64_t f = 0; f < F; ++f) {
            m->face_owner[f] = -1;
            m->face_neighbor[f] = -1;
        }
        for (int64_t e = 0; e <= n_elems; ++e) m->cell_face_ptr[e] = elem_face_ptr[e];
        for (int64_t e = 0; e < n_elems; ++e) {
            for (int32_t k = elem_face_ptr[e]; k < elem_face_ptr[e + 1]; ++k) {
                int32_t f = u2f[elem_faces[k]];
                m->cell_faces[k] = f;
                if (m->face_owner[f] < 0)
                    m->face_owner[f] = (int32_t)e;
                else if (m->face_patch[f] < 0 && m->face_neighbor[f] < 0)
                    m->face_neighbor[f] = (int32_t)e;
            }
        }
        for (int64_t f = 0; f < n_int; ++f)
            if (m->face_neighbor[f] < 0) {  // interior face seen by one cell only: unmarked boundary
                fv_host_mesh_free(m);
                return FV_ERR_INVALID;
            }

        compute_geometry(m);
        *out = m;
        return FV_OK;
    } catch (const std::bad_alloc &) {
        return FV_ERR_ALLOC;
    }
}

// An element list as fv_host_mesh_from_elements / fv_mesh_build_elements take it.
namespace {
struct Elements {
    int32_t dim = 0;
    std::vector<double> nodes;
    std::vector<int32_t> kind, ptr, en, bptr, bn, bm;
};

fv_status to_host(const Elements &el, fv_host_mesh **out) {
    return fv_host_mesh_from_elements(el.dim, (int64_t)(el.nodes.size() / el.dim), el.nodes.data(),
                                      (int64_t)el.kind.size(), el.kind.data(), el.ptr.data(), el.en.data(),
                                      (int64_t)el.bm.size(), el.bptr.data(), el.bn.data(), el.bm.data(), out);
}

fv_status to_device(const Elements &el, void *stream, fv_mesh **out, fv_host_mesh **host_out) {
    return fv_mesh_build_elements(el.dim, (int64_t)(el.nodes.size() / el.dim), el.nodes.data(),
                                  (int64_t)el.kind.size(), el.kind.data(), el.ptr.data(), el.en.data(),
                                  (int64_t)el.bm.size(), el.bptr.data(), el.bn.data(), el.bm.data(), stream, out,
                                  host_out);
}

fv_status square_elements(int32_t n, double jitter, uint64_t seed, Elements &el) {
    if (n < 1 || n > 8192) return FV_ERR_INVALID;
    try {
        const int64_t np = (int64_t)(n + 1) * (n + 1);
        const double h = 1.0 / n;
        el.dim = 2;
        std::vector<double> &nodes = el.nodes;
        nodes.assign((size_t)np * 2, 0.0);
        Rng rng(seed);
        for (int j = 0; j <= n; ++j)
            for (int i = 0; i <= n; ++i) {
                int64_t p = (int64_t)j * (n + 1) + i;
                double x = (double)i / n, y = (double)j / n;
                if (i > 0 && i < n && j > 0 && j < n) {
                    x += (2.0 * rng.uniform() - 1.0) * jitter * h;
                    y += (2.0 * rng.uniform() - 1.0) * jitter * h;
                }
                nodes[p * 2] = x;
                nodes[p * 2 + 1] = y;
            }
        const int64_t ne = 2LL * n * n;
        el.kind.assign((size_t)ne, 5);
        el.ptr.assign((size_t)ne + 1, 0);
        el.en.assign((size_t)ne * 3, 0);
        std::vector<int32_t> &ptr = el.ptr, &en = el.en;
        int64_t e = 0;
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                int32_t a = j * (n + 1) + i, b = a + 1, c = a + n + 2, d = a + n + 1;
                const int32_t t[6] = {a, b, c, a, c, d};
                for (int q = 0; q < 6; ++q) en[e * 3 + q] = t[q];
                e += 2;
            }
        for (int64_t q = 0; q <= ne; ++q) ptr[q] = (int32_t)(3 * q);
        // one boundary marker (id 0) holding every boundary edge
        std::vector<int32_t> &bptr = el.bptr, &bn = el.bn, &bm = el.bm;
        bptr.push_back(0);
        auto add_edge = [&](int32_t u, int32_t v) {
            bn.push_back(u);
            bn.push_back(v);
            bptr.push_back((int32_t)bn.size());
            bm.push_back(0);
        };
        for (int i = 0; i < n; ++i) {
            add_edge(i, i + 1);
            add_edge(n * (n + 1) + i, n * (n + 1) + i + 1);
            add_edge(i * (n + 1), (i + 1) * (n + 1));
            add_edge(i * (n + 1) + n, (i + 1) * (n + 1) + n);
        }
        return FV_OK;
    } catch (const std::bad_alloc &) {
        return FV_ERR_ALLOC;
    }
}

fv_status cube_elements(int32_t n, double jitter, uint64_t seed, Elements &el) {
    if (n < 1 || n > 1000) return FV_ERR_INVALID;
    try {
        const int64_t n1 = n + 1;
        const int64_t np = n1 * n1 * n1;
        const double h = 1.0 / n;
        el.dim = 3;
        std::vector<double> &nodes = el.nodes;
        nodes.assign((size_t)np * 3, 0.0);
        Rng rng(seed);
        for (int k = 0; k <= n; ++k)
            for (int j = 0; j <= n; ++j)
                for (int i = 0; i <= n; ++i) {
                    int64_t p = ((int64_t)k * n1 + j) * n1 + i;
                    double x = (double)i / n, y = (double)j / n, z = (double)k / n;
                    if (i > 0 && i < n && j > 0 && j < n && k > 0 && k < n) {
                        x += (2.0 * rng.uniform() - 1.0) * jitter * h;
                        y += (2.0 * rng.uniform() - 1.0) * jitter * h;
                        z += (2.0 * rng.uniform() - 1.0) * jitter * h;
                    }
                    nodes[p * 3] = x;
                    nodes[p * 3 + 1] = y;
                    nodes[p * 3 + 2] = z;
                }
        const int64_t ne = 6LL * n * n * n;
        el.kind.assign((size_t)ne, 10);
        el.ptr.assign((size_t)ne + 1, 0);
        el.en.assign((size_t)ne * 4, 0);
        std::vector<int32_t> &ptr = el.ptr, &en = el.en;
        // Kuhn split: the 6 monotone paths from corner (0,0,0) to (1,1,1).
        const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
        const int64_t stride[3] = {1, n1, n1 * n1};
        int64_t e = 0;
        for (int k = 0; k < n; ++k)
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i) {
                    int64_t base = ((int64_t)k * n1 + j) * n1 + i;
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
        for (int64_t q = 0; q <= ne; ++q) ptr[q] = (int32_t)(4 * q);
        // Boundary triangles: tet faces whose three nodes lie on one cube side.
        auto side_mask = [&](int32_t p) -> unsigned {
            int64_t i = p % n1, j = (p / n1) % n1, k = p / (n1 * n1);
            unsigned m = 0;
            if (i == 0) m |= 1u;
            if (i == n) m |= 2u;
            if (j == 0) m |= 4u;
            if (j == n) m |= 8u;
            if (k == 0) m |= 16u;
            if (k == n) m |= 32u;
            return m;
        };
        std::vector<int32_t> &bptr = el.bptr, &bn = el.bn, &bm = el.bm;
        bptr.push_back(0);
        int32_t fn[24];
        int fs[8];
        for (int64_t q = 0; q < ne; ++q) {
            const int64_t hex = q / 6;  // only hexes touching a side hold boundary faces
            const int64_t hi = hex % n, hj = (hex / n) % n, hk = hex / ((int64_t)n * n);
            if (hi > 0 && hi < n - 1 && hj > 0 && hj < n - 1 && hk > 0 && hk < n - 1) {
                q += 5;
                continue;
            }
            vtk_faces(10, en.data() + q * 4, fn, fs);
            for (int l = 0; l < 4; ++l) {
                const int32_t *f = fn + fs[l];
                if (side_mask(f[0]) & side_mask(f[1]) & side_mask(f[2])) {
                    bn.push_back(f[0]);
                    bn.push_back(f[1]);
                    bn.push_back(f[2]);
                    bptr.push_back((int32_t)bn.size());
                    bm.push_back(0);
                }
            }
        }
        return FV_OK;
    } catch (const std::bad_alloc &) {
        return FV_ERR_ALLOC;
    }
}
}  // namespace

extern "C" fv_status fv_host_mesh_generate_square(int32_t n, double jitter, uint64_t seed, fv_host_mesh **out) {
    if (!out) return FV_ERR_INVALID;
    Elements el;
    FV_RETURN_IF(square_elements(n, jitter, seed, el));
    return to_host(el, out);
}

extern "C" fv_status fv_host_mesh_generate_cube(int32_t n, double jitter, uint64_t seed, fv_host_mesh **out) {
    if (!out) return FV_ERR_INVALID;
    Elements el;
    FV_RETURN_IF(cube_elements(n, jitter, seed, el));
    return to_host(el, out);
}

extern "C" fv_status fv_mesh_build_square(int32_t n, double jitter, uint64_t seed, void *stream, fv_mesh **out,
                                          fv_host_mesh **host_out) {
    if (!out) return FV_ERR_INVALID;
    Elements el;
    FV_RETURN_IF(square_elements(n, jitter, seed, el));
    return to_device(el, stream, out, host_out);
}

extern "C" fv_status fv_mesh_build_cube(int32_t n, double jitter, uint64_t seed, void *stream, fv_mesh **out,
                                        fv_host_mesh **host_out) {
    if (!out) return FV_ERR_INVALID;
    Elements el;
    FV_RETURN_IF(cube_elements(n, jitter, seed, el));
    return to_device(el, stream, out, host_out);
}

extern "C" fv_status fv_host_fields_generate(const fv_host_mesh *m, uint64_t seed, double kappa0, double sigma,
                                             const double *velocity, double source_const, int32_t source_uniform,
                                             double *kappa_face, double *flux_face, double *source_cell) {
    if (!m) return FV_ERR_INVALID;
    const int dim = m->dim;
    try {
        if (kappa_face) {
            std::vector<double> kc((size_t)m->n_cells);
            Rng rk(seed ^ 0x6b617070615f6365ULL);
            for (int64_t c = 0; c < m->n_cells; ++c) kc[c] = kappa0 * std::exp(sigma * rk.normal());
            for (int64_t f = 0; f < m->n_faces; ++f) {
                const int32_t o = m->face_owner[f], nb = m->face_neighbor[f];
                if (nb < 0) {
                    kappa_face[f] = kc[o];
                    continue;
                }
                const double *nv = m->face_normal + f * dim;
                const double *fc = m->face_center + f * dim;
                const double *cc = m->cell_center + (int64_t)o * dim;
                const double *nc = m->cell_center + (int64_t)nb * dim;
                double num = 0.0, den = 0.0;
                for (int d = 0; d < dim; ++d) num += nv[d] * (nc[d] - fc[d]);
                for (int d = 0; d < dim; ++d) den += nv[d] * (nc[d] - cc[d]);
                double w = num / std::max(den, 1e-14);
                w = std::min(1.0, std::max(0.0, w));
                kappa_face[f] = w * kc[o] + (1.0 - w) * kc[nb];
            }
        }
        if (flux_face) {
            for (int64_t f = 0; f < m->n_faces; ++f) {
                double s = 0.0;
                for (int d = 0; d < dim; ++d) s += velocity[d] * m->face_normal[f * dim + d];
                flux_face[f] = s;
            }
        }
        if (source_cell) {
            Rng rs(seed ^ 0x736f757263655f63ULL);
            for (int64_t c = 0; c < m->n_cells; ++c) source_cell[c] = source_uniform ? rs.uniform() : source_const;
        }
        return FV_OK;
    } catch (const std::bad_alloc &) {
        return FV_ERR_ALLOC;
    }
}

// Mesh::read_su2 (core/mesh/io.rs:228-533): NPOIN node lines (the first dim
// values), NELEM element lines (VTK kind then its nodes; trailing indices
// ignored), MARKER_TAG / MARKER_ELEMS boundary lines (markers numbered 0, 1,
// ... in file order, a face's key = its sorted nodes), then the same face
// numbering and geometry as fv_host_mesh_from_elements.
namespace {
fv_status su2_elements(const char *path, int32_t dim, Elements &el) {
    if (!path) return FV_ERR_INVALID;
    FILE *fp = fopen(path, "r");
    if (!fp) return FV_ERR_INVALID;
    std::vector<std::string> lines;
    {
        char buf[4096];
        std::string cur;
        while (fgets(buf, sizeof(buf), fp)) {
            cur += buf;
            if (!cur.empty() && cur.back() == '\n') {
                cur.pop_back();
                if (!cur.empty() && cur.back() == '\r') cur.pop_back();
                lines.push_back(cur);
                cur.clear();
            }
        }
        if (!cur.empty()) lines.push_back(cur);
        fclose(fp);
    }
    auto value_after = [](const std::string &l, const char *key, long long &v) -> bool {
        size_t p = l.find(key);
        if (p == std::string::npos) return false;
        v = atoll(l.c_str() + p + strlen(key));
        return true;
    };
    auto tokens = [](const std::string &l) {
        std::vector<std::string> t;
        size_t i = 0;
        while (i < l.size()) {
            while (i < l.size() && isspace((unsigned char)l[i])) ++i;
            size_t j = i;
            while (j < l.size() && !isspace((unsigned char)l[j])) ++j;
            if (j > i) t.push_back(l.substr(i, j - i));
            i = j;
        }
        return t;
    };
    try {
        long long ndime = 0;
        for (const auto &l : lines)
            if (value_after(l, "NDIME=", ndime)) break;
        const int d = dim > 0 ? dim : (int)ndime;
        if (d != 2 && d != 3) return FV_ERR_INVALID;
        el.dim = d;
        std::vector<double> &nodes = el.nodes;
        std::vector<int32_t> &kind = el.kind, &eptr = el.ptr, &enodes = el.en, &bptr = el.bptr, &bnodes = el.bn,
                             &bmark = el.bm;
        eptr.assign(1, 0);
        bptr.assign(1, 0);
        int marker = -1;
        for (size_t li = 0; li < lines.size(); ++li) {
            long long cnt = 0;
            if (value_after(lines[li], "NPOIN=", cnt)) {
                for (long long q = 0; q < cnt; ++q) {
                    if (li + 1 + q >= lines.size()) return FV_ERR_INVALID;
                    auto t = tokens(lines[li + 1 + q]);
                    if ((int)t.size() < d) return FV_ERR_INVALID;
                    for (int c = 0; c < d; ++c) nodes.push_back(strtod(t[c].c_str(), nullptr));
                }
                li += (size_t)cnt;
            } else if (value_after(lines[li], "NELEM=", cnt)) {
                for (long long q = 0; q < cnt; ++q) {
                    if (li + 1 + q >= lines.size()) return FV_ERR_INVALID;
                    auto t = tokens(lines[li + 1 + q]);
                    if (t.empty()) return FV_ERR_INVALID;
                    const int k = atoi(t[0].c_str());
                    const int nn = vtk_nnodes(k);
                    if (nn < 0 || (int)t.size() < 1 + nn) return FV_ERR_INVALID;
                    kind.push_back(k);
                    for (int c = 0; c < nn; ++c) enodes.push_back(atoi(t[1 + c].c_str()));
                    eptr.push_back((int32_t)enodes.size());
                }
                li += (size_t)cnt;
            } else if (lines[li].find("MARKER_TAG=") != std::string::npos) {
                ++marker;
            } else if (value_after(lines[li], "MARKER_ELEMS=", cnt)) {
                if (marker < 0) return FV_ERR_INVALID;
                for (long long q = 0; q < cnt; ++q) {
                    if (li + 1 + q >= lines.size()) return FV_ERR_INVALID;
                    auto t = tokens(lines[li + 1 + q]);
                    if (t.size() < 3) return FV_ERR_INVALID;
                    for (size_t c = 1; c < t.size(); ++c) bnodes.push_back(atoi(t[c].c_str()));
                    bptr.push_back((int32_t)bnodes.size());
                    bmark.push_back(marker);
                }
                li += (size_t)cnt;
            }
        }
        if (kind.empty() || nodes.empty()) return FV_ERR_INVALID;
        return FV_OK;
    } catch (const std::bad_alloc &) {
        return FV_ERR_ALLOC;
    }
}
}  // namespace

extern "C" fv_status fv_host_mesh_read_su2(const char *path, int32_t dim, fv_host_mesh **out) {
    if (!path || !out) return FV_ERR_INVALID;
    *out = nullptr;
    Elements el;
    FV_RETURN_IF(su2_elements(path, dim, el));
    return to_host(el, out);
}

extern "C" fv_status fv_mesh_build_su2(const char *path, int32_t dim, void *stream, fv_mesh **out,
                                       fv_host_mesh **host_out) {
    if (!path || !out) return FV_ERR_INVALID;
    *out = nullptr;
    Elements el;
    FV_RETURN_IF(su2_elements(path, dim, el));
    return to_device(el, stream, out, host_out);
}

// ---------------------------------------------------------------- explicit faces
// add_face / add_cell (mod.rs:451-529) for explicit face and cell lists: the
// first cell listing a face owns it, the second becomes its neighbour unless
// the face carries a boundary tag; then Mesh::compute.  The tagged faces must
// be the tail of the face list (the layout every mesh read from SU2 has).
extern "C" fv_status fv_host_mesh_from_faces(int32_t dim, int64_t n_nodes, const double *nodes, int64_t n_faces,
                                             const int32_t *face_node_ptr, const int32_t *face_nodes,
                                             const int32_t *face_patch, int64_t n_cells,
                                             const int32_t *cell_face_ptr, const int32_t *cell_faces,
                                             fv_host_mesh **out) {
    if (!out || (dim != 2 && dim != 3) || n_nodes <= 0 || n_faces <= 0 || n_cells <= 0 || !nodes ||
        !face_node_ptr || !face_nodes || !face_patch || !cell_face_ptr || !cell_faces || n_nodes >= 0x7fffffffLL ||
        n_faces >= 0x7fffffffLL || n_cells >= 0x7fffffffLL || face_node_ptr[0] != 0 || cell_face_ptr[0] != 0)
        return FV_ERR_INVALID;
    *out = nullptr;
    int64_t n_tagged = 0;
    for (int64_t f = 0; f < n_faces; ++f) {
        const int len = face_node_ptr[f + 1] - face_node_ptr[f];
        if (len < 2 || len > 64 || (dim == 2 && len != 2)) return FV_ERR_INVALID;
        for (int q = 0; q < len; ++q) {
            const int32_t id = face_nodes[face_node_ptr[f] + q];
            if (id < 0 || id >= n_nodes) return FV_ERR_INVALID;
        }
        if (face_patch[f] >= 0) {
            ++n_tagged;
        } else if (n_tagged) {
            fv_internal_set_error_text("fv_host_mesh_from_faces: tagged faces must be the tail of the face list");
            return FV_ERR_UNSUPPORTED;
        }
    }
    for (int64_t c = 0; c < n_cells; ++c) {
        const int len = cell_face_ptr[c + 1] - cell_face_ptr[c];
        if (len < 2 || len > 64) return FV_ERR_INVALID;
        for (int q = 0; q < len; ++q) {
            const int32_t f = cell_faces[cell_face_ptr[c] + q];
            if (f < 0 || f >= n_faces) return FV_ERR_INVALID;
        }
    }
    try {
        fv_host_mesh *m = (fv_host_mesh *)std::calloc(1, sizeof(fv_host_mesh));
        if (!m) return FV_ERR_ALLOC;
        const int64_t F = n_faces, N = n_cells, fnn = face_node_ptr[F], ncf = cell_face_ptr[N];
        m->dim = dim;
        m->n_nodes = n_nodes;
        m->n_faces = F;
        m->n_cells = N;
        m->n_boundary_faces = n_tagged;
        m->nodes = (double *)std::malloc(sizeof(double) * n_nodes * dim);
        m->face_node_ptr = (int32_t *)std::malloc(sizeof(int32_t) * (F + 1));
        m->face_nodes = (int32_t *)std::malloc(sizeof(int32_t) * fnn);
        m->face_patch = (int32_t *)std::malloc(sizeof(int32_t) * F);
        m->cell_face_ptr = (int32_t *)std::malloc(sizeof(int32_t) * (N + 1));
        m->cell_faces = (int32_t *)std::malloc(sizeof(int32_t) * ncf);
        m->face_owner = (int32_t *)std::malloc(sizeof(int32_t) * F);
        m->face_neighbor = (int32_t *)std::malloc(sizeof(int32_t) * F);
        m->face_area = (double *)std::malloc(sizeof(double) * F);
        m->face_normal = (double *)std::malloc(sizeof(double) * F * dim);
        m->face_center = (double *)std::malloc(sizeof(double) * F * dim);
        m->cell_center = (double *)std::malloc(sizeof(double) * N * dim);
        m->cell_volume = (double *)std::malloc(sizeof(double) * N);
        if (!m->nodes || !m->face_node_ptr || !m->face_nodes || !m->face_patch || !m->cell_face_ptr ||
            !m->cell_faces || !m->face_owner || !m->face_neighbor || !m->face_area || !m->face_normal ||
            !m->face_center || !m->cell_center || !m->cell_volume) {
            fv_host_mesh_free(m);
            return FV_ERR_ALLOC;
        }
        std::memcpy(m->nodes, nodes, sizeof(double) * n_nodes * dim);
        std::memcpy(m->face_node_ptr, face_node_ptr, sizeof(int32_t) * (F + 1));
        std::memcpy(m->face_nodes, face_nodes, sizeof(int32_t) * fnn);
        std::memcpy(m->face_patch, face_patch, sizeof(int32_t) * F);
        std::memcpy(m->cell_face_ptr, cell_face_ptr, sizeof(int32_t) * (N + 1));
        std::memcpy(m->cell_faces, cell_faces, sizeof(int32_t) * ncf);
        for (int64_t f = 0; f < F; ++f) m->face_owner[f] = m->face_neighbor[f] = -1;
        for (int64_t c = 0; c < N; ++c)
            for (int32_t k = cell_face_ptr[c]; k < cell_face_ptr[c + 1]; ++k) {
                const int32_t f = cell_faces[k];
                if (m->face_owner[f] < 0)
                    m->face_owner[f] = (int32_t)c;
                else if (m->face_patch[f] < 0 && m->face_neighbor[f] < 0)
                    m->face_neighbor[f] = (int32_t)c;
            }
        for (int64_t f = 0; f < F; ++f)
            if (m->face_owner[f] < 0 || (m->face_patch[f] < 0 && m->face_neighbor[f] < 0) ||
                m->face_neighbor[f] == m->face_owner[f]) {
                fv_internal_set_error_text(
                    "fv_host_mesh_from_faces: a face no cell lists, an untagged face with one cell, or a cell listing "
                    "a face twice");
                fv_host_mesh_free(m);
                return FV_ERR_INVALID;
            }
        compute_geometry(m);
        *out = m;
        return FV_OK;
    } catch (const std::bad_alloc &) {
        return FV_ERR_ALLOC;
    }
}

// ---------------------------------------------------------------- .msh
// The crate's own mesh format, Mesh::write / Mesh::read (io.rs:10-225):
//   NDIME=<dim>
//   NPATCH=<k>, then "<name> <id> <first face> <faces>" per patch
//   NNODES=<n>, then the coordinates, separated by one space
//   NFACES=<n>, then "<len> <nodes...> <tag|-> <global id> <-|owner rank>"
//   NCELLS=<n>, then "<len> <faces...> <global id> <-|owner rank>"
// Numbers print as Rust's Display does: integers in decimal, doubles as the
// shortest digits that read back to the same value, never in exponent form.
namespace {

struct Topology {
    int32_t dim = 0;
    std::vector<double> nodes;
    std::vector<int32_t> fptr{0}, fnodes, fpatch, cptr{0}, cfaces;
};

// Rust's `{}` for f64: shortest round-trip digits, positional notation.
std::string rust_f64(double v) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v < 0 ? "-inf" : "inf";
    if (v == 0.0) return std::signbit(v) ? "-0" : "0";
    char buf[64];
    int p = 1;
    for (; p <= 17; ++p) {
        snprintf(buf, sizeof(buf), "%.*e", p - 1, v);
        if (strtod(buf, nullptr) == v) break;
    }
    // buf = [-]d[.ddd]e[+-]xx
    std::string s(buf), digits;
    const bool neg = s[0] == '-';
    size_t i = neg ? 1 : 0;
    for (; i < s.size() && s[i] != 'e'; ++i)
        if (s[i] != '.') digits += s[i];
    const int e10 = atoi(s.c_str() + i + 1);
    while (digits.size() > 1 && digits.back() == '0') digits.pop_back();
    const int nd = (int)digits.size();
    std::string out = neg ? "-" : "";
    if (e10 < 0) {
        out += "0.";
        out.append((size_t)(-e10 - 1), '0');
        out += digits;
    } else if (e10 >= nd - 1) {
        out += digits;
        out.append((size_t)(e10 - (nd - 1)), '0');
    } else {
        out += digits.substr(0, (size_t)e10 + 1);
        out += ".";
        out += digits.substr((size_t)e10 + 1);
    }
    return out;
}

bool parse_i64(const std::string &t, long long &v) {
    if (t.empty()) return false;
    char *end = nullptr;
    errno = 0;
    v = strtoll(t.c_str(), &end, 10);
    return errno == 0 && end && *end == '\0' && !isspace((unsigned char)t[0]);
}

std::vector<std::string> split_spaces(const std::string &l) {  // str::split(" "): empty pieces kept
    std::vector<std::string> t;
    size_t a = 0;
    while (true) {
        const size_t b = l.find(' ', a);
        t.push_back(l.substr(a, b == std::string::npos ? std::string::npos : b - a));
        if (b == std::string::npos) break;
        a = b + 1;
    }
    return t;
}

std::string trim(const std::string &l) {
    size_t a = 0, b = l.size();
    while (a < b && isspace((unsigned char)l[a])) ++a;
    while (b > a && isspace((unsigned char)l[b - 1])) --b;
    return l.substr(a, b - a);
}

fv_status msh_parse(const char *path, int32_t dim, Topology &t) {
    if (!path) return FV_ERR_INVALID;
    FILE *fp = fopen(path, "r");
    if (!fp) {
        fv_internal_set_error_text("read_msh: cannot open the file");
        return FV_ERR_INVALID;
    }
    auto bad = [&](long long line, const char *what) {
        char msg[160];
        snprintf(msg, sizeof(msg), "read_msh: line %lld: %s", line, what);
        fv_internal_set_error_text(msg);
        return FV_ERR_INVALID;
    };
    std::string section = "none", line;
    long long nodes_left = 0, faces_left = 0, cells_left = 0, patches_left = 0, line_id = 0;
    int d = dim;
    fv_status st = FV_OK;
    char buf[1 << 16];
    std::string cur;
    bool eof = false;
    while (st == FV_OK && !eof) {
        cur.clear();
        while (true) {
            if (!fgets(buf, sizeof(buf), fp)) {
                eof = true;
                break;
            }
            cur += buf;
            if (!cur.empty() && cur.back() == '\n') break;
        }
        if (eof && cur.empty()) break;
        ++line_id;
        const std::string ls = trim(cur);
        if (ls.empty()) continue;
        if (ls[0] == 'N') {
            const size_t eq = ls.find('=');
            if (eq == std::string::npos) {
                st = bad(line_id, "section header without '='");
                break;
            }
            section = ls.substr(0, eq);
            std::string rest = ls.substr(eq + 1);
            const size_t eq2 = rest.find('=');
            if (eq2 != std::string::npos) rest = rest.substr(0, eq2);
            long long val = 0;
            if (!parse_i64(rest, val) || val < 0) {
                st = bad(line_id, "section size is not a number");
                break;
            }
            if (section == "NDIME") {
                if (d == 0) d = (int)val;
                if (val != d || (d != 2 && d != 3)) {
                    fv_internal_set_error_text("read_msh: NDIME differs from the requested dimension");
                    st = FV_ERR_INVALID;
                    break;
                }
                t.dim = d;
            } else if (section == "NNODES") {
                nodes_left = val;
            } else if (section == "NFACES") {
                faces_left = val;
            } else if (section == "NCELLS") {
                cells_left = val;
            } else if (section == "NPATCH") {
                patches_left = val;
            }
            continue;
        }
        if (section == "none") continue;
        if (section == "NNODES") {
            if (nodes_left == 0) continue;
            if (t.dim == 0) {
                st = bad(line_id, "nodes before NDIME");
                break;
            }
            double x[3] = {0.0, 0.0, 0.0};
            const auto tok = split_spaces(ls);
            for (size_t i = 0; i < tok.size() && (int)i < t.dim; ++i) {
                const std::string v = trim(tok[i]);
                char *end = nullptr;
                x[i] = strtod(v.c_str(), &end);
                if (v.empty() || !end || *end != '\0') {
                    st = bad(line_id, "bad coordinate");
                    break;
                }
            }
            for (int i = 0; i < t.dim; ++i) t.nodes.push_back(x[i]);
            --nodes_left;
        } else if (section == "NFACES" || section == "NCELLS") {
            const bool faces = section == "NFACES";
            if ((faces ? faces_left : cells_left) == 0) continue;
            const auto tok = split_spaces(ls);
            long long size = 0;
            if (tok.empty() || !parse_i64(tok[0], size) || size < 0 || size > 64 ||
                (long long)tok.size() < 1 + size + (faces ? 3 : 2)) {
                st = bad(line_id, faces ? "bad face line" : "bad cell line");
                break;
            }
            for (long long i = 0; i < size; ++i) {
                long long v = 0;
                if (!parse_i64(tok[1 + i], v) || v < 0 || v > 0x7fffffffLL) {
                    st = bad(line_id, "bad index");
                    break;
                }
                (faces ? t.fnodes : t.cfaces).push_back((int32_t)v);
            }
            if (st != FV_OK) break;
            size_t k = (size_t)(1 + size);
            if (faces) {
                long long tag = -1;
                if (tok[k] != "-" && (!parse_i64(tok[k], tag) || tag < 0 || tag > 65535)) {
                    st = bad(line_id, "bad boundary tag");
                    break;
                }
                t.fpatch.push_back((int32_t)tag);
                ++k;
            }
            long long gid = 0;
            if (!parse_i64(tok[k], gid) || gid < 0 || gid > 0xffffffffLL) {
                st = bad(line_id, "bad global id");
                break;
            }
            if (tok[k + 1] != "-") {  // Ownership::Remote: a ghost of a decomposed mesh
                fv_internal_set_error_text("read_msh: remote (ghost) faces or cells are not supported");
                st = FV_ERR_UNSUPPORTED;
                break;
            }
            if (faces) {
                t.fptr.push_back((int32_t)t.fnodes.size());
                --faces_left;
            } else {
                t.cptr.push_back((int32_t)t.cfaces.size());
                --cells_left;
            }
        } else if (section == "NPATCH") {
            if (patches_left == 0) continue;
            const auto tok = split_spaces(ls);
            long long bid = 0, fstart = 0, len = 0;
            if (tok.size() < 4 || !parse_i64(tok[1], bid) || !parse_i64(tok[2], fstart) || !parse_i64(tok[3], len)) {
                st = bad(line_id, "bad patch line");
                break;
            }
            --patches_left;
        }
    }
    fclose(fp);
    if (st != FV_OK) return st;
    if (t.dim == 0 || t.nodes.empty() || t.fpatch.empty() || t.cptr.size() < 2) {
        fv_internal_set_error_text("read_msh: missing NDIME, nodes, faces or cells");
        return FV_ERR_INVALID;
    }
    return FV_OK;
}

fv_status topology_to_host(const Topology &t, fv_host_mesh **out) {
    return fv_host_mesh_from_faces(t.dim, (int64_t)(t.nodes.size() / t.dim), t.nodes.data(), (int64_t)t.fpatch.size(),
                                   t.fptr.data(), t.fnodes.data(), t.fpatch.data(), (int64_t)t.cptr.size() - 1,
                                   t.cptr.data(), t.cfaces.data(), out);
}

}  // namespace

extern "C" fv_status fv_host_mesh_read_msh(const char *path, int32_t dim, fv_host_mesh **out) {
    if (!path || !out) return FV_ERR_INVALID;
    *out = nullptr;
    try {
        Topology t;
        FV_RETURN_IF(msh_parse(path, dim, t));
        return topology_to_host(t, out);
    } catch (const std::bad_alloc &) {
        return FV_ERR_ALLOC;
    }
}

extern "C" fv_status fv_mesh_build_msh(const char *path, int32_t dim, void *stream, fv_mesh **out,
                                       fv_host_mesh **host_out) {
    if (!path || !out) return FV_ERR_INVALID;
    *out = nullptr;
    try {
        Topology t;
        FV_RETURN_IF(msh_parse(path, dim, t));
        return fv_mesh_build_faces(t.dim, (int64_t)(t.nodes.size() / t.dim), t.nodes.data(), (int64_t)t.fpatch.size(),
                                   t.fptr.data(), t.fnodes.data(), t.fpatch.data(), (int64_t)t.cptr.size() - 1,
                                   t.cptr.data(), t.cfaces.data(), stream, out, host_out);
    } catch (const std::bad_alloc &) {
        return FV_ERR_ALLOC;
    }
}

extern "C" fv_status fv_host_mesh_write_msh(const fv_host_mesh *m, const char *path, const char *const *patch_names,
                                            int32_t n_patch_names) {
    if (!m || !path) return FV_ERR_INVALID;
    FILE *fp = fopen(path, "w");
    if (!fp) return FV_ERR_INVALID;
    try {
        const int dim = m->dim;
        // patches: the tagged faces grouped by tag, in face order
        std::vector<int32_t> ids;
        std::vector<int64_t> first, count;
        for (int64_t f = 0; f < m->n_faces; ++f) {
            const int32_t p = m->face_patch[f];
            if (p < 0) continue;
            if (ids.empty() || ids.back() != p) {
                ids.push_back(p);
                first.push_back(f);
                count.push_back(0);
            }
            ++count.back();
        }
        std::string out;
        out.reserve(1 << 20);
        auto flush = [&]() {
            fwrite(out.data(), 1, out.size(), fp);
            out.clear();
        };
        out += "NDIME=" + std::to_string(dim) + "\n";
        out += "NPATCH=" + std::to_string(ids.size()) + "\n";
        for (size_t i = 0; i < ids.size(); ++i) {
            std::string name = (patch_names && ids[i] < n_patch_names && patch_names[ids[i]])
                                   ? std::string(patch_names[ids[i]])
                                   : "patch_" + std::to_string(ids[i]);
            out += name + " " + std::to_string(ids[i]) + " " + std::to_string(first[i]) + " " +
                   std::to_string(count[i]) + "\n";
        }
        out += "NNODES=" + std::to_string(m->n_nodes) + "\n";
        for (int64_t n = 0; n < m->n_nodes; ++n) {
            for (int d = 0; d < dim; ++d) {
                if (d) out += ' ';
                out += rust_f64(m->nodes[n * dim + d]);
            }
            out += '\n';
            if (out.size() > (1 << 20)) flush();
        }
        out += "NFACES=" + std::to_string(m->n_faces) + "\n";
        for (int64_t f = 0; f < m->n_faces; ++f) {
            out += std::to_string(m->face_node_ptr[f + 1] - m->face_node_ptr[f]);
            for (int32_t k = m->face_node_ptr[f]; k < m->face_node_ptr[f + 1]; ++k)
                out += " " + std::to_string(m->face_nodes[k]);
            out += m->face_patch[f] >= 0 ? " " + std::to_string(m->face_patch[f]) : std::string(" -");
            out += " " + std::to_string(f) + " -\n";
            if (out.size() > (1 << 20)) flush();
        }
        out += "NCELLS=" + std::to_string(m->n_cells) + "\n";
        for (int64_t c = 0; c < m->n_cells; ++c) {
            out += std::to_string(m->cell_face_ptr[c + 1] - m->cell_face_ptr[c]);
            for (int32_t k = m->cell_face_ptr[c]; k < m->cell_face_ptr[c + 1]; ++k)
                out += " " + std::to_string(m->cell_faces[k]);
            out += " " + std::to_string(c) + " -\n";
            if (out.size() > (1 << 20)) flush();
        }
        flush();
        const bool ok = fclose(fp) == 0;
        return ok ? FV_OK : FV_ERR_INVALID;
    } catch (const std::bad_alloc &) {
        fclose(fp);
        return FV_ERR_ALLOC;
    }
}
