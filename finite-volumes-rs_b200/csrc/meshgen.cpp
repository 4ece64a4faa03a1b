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
#include <cmath>
#include <cstdio>
#include <string>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

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

struct Builder {
    int dim = 0;
    int64_t n_nodes = 0;
    const double *nodes = nullptr;
};

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

        // Mesh::compute: face data, then cell data, then orientation.
#pragma omp parallel for schedule(static)
        for (int64_t f = 0; f < F; ++f)
            face_geometry(dim, m->nodes, m->face_nodes + m->face_node_ptr[f],
                          m->face_node_ptr[f + 1] - m->face_node_ptr[f], m->face_area + f,
                          m->face_normal + f * dim, m->face_center + f * dim);
#pragma omp parallel for schedule(static)
        for (int64_t c = 0; c < n_elems; ++c)
            cell_geometry(dim, m->cell_faces + m->cell_face_ptr[c], m->cell_face_ptr[c + 1] - m->cell_face_ptr[c],
                          m->face_area, m->face_normal, m->face_center, m->cell_center + c * dim,
                          m->cell_volume + c);
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
