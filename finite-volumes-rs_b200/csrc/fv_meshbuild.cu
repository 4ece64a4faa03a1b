// Device mesh builder: the face numbering of Mesh::read_su2 and the geometry
// of Mesh::compute, run on the GPU from an element list.
//
//   compute_vtk_faces ............ core/mesh/io.rs:364-486
//   VTK element face tables ...... core/mesh/vtk.rs:56-125
//   add_face / add_cell owner/nb . core/mesh/mod.rs:451-529
//   face + cell geometry ......... core/mesh/compute.rs:34-69, 267-375
//   normal orientation ........... core/mesh/compute.rs:97-131
//   gradient coefficients ........ core/mesh/compute.rs:155-203
//
// The host builder (meshgen.cpp) finds unique faces with a hash table while
// it walks the elements in order.  Here every (element, local face)
// incidence is a record keyed by its sorted node ids (padded with n_nodes,
// which is no node id), followed by one record per boundary face of the
// input.  A stable LSD radix sort over the key words groups equal faces and
// keeps each group's records in input order, so the first element record of
// a group is the element that discovered the face (its owner), the second is
// the neighbour, and the first boundary record gives the marker: the answers
// of the sequential loop.  One more sort on (class, discoverer), class 0 for
// interior faces and marker + 1 for boundary faces, numbers the faces:
// interior faces in discovery order, then boundary faces by ascending marker,
// discovery order within a marker.  The geometry kernels repeat the host
// expressions operation for operation (the library is built without FP
// contraction), so every array equals the host builder's bit for bit.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "fv_internal.cuh"

namespace {

constexpr int kB = 256;
enum : int {
    kBadElement = 1,     // unknown kind, wrong node count or pointer range, kind of the other dimension
    kBadNode = 2,        // node id outside [0, n_nodes)
    kBadOpenFace = 4,    // unmarked face listed by one element only
    kBadSelf = 8,        // an element lists the same face twice
    kBadForeign = 16,    // a marked face listed by a second element (neither owner nor neighbour)
    kHasQuadFace = 32,   // a hexahedron: faces of four nodes
};

// Local faces of the VTK kinds (vtk.rs:56-125): node slots within the element.
// Kinds in index order: triangle (5), quad (9), tetrahedron (10), hexahedron (12).
__constant__ int8_t c_slot[4][6][4] = {
    {{0, 1}, {1, 2}, {2, 0}},
    {{0, 1}, {1, 2}, {2, 3}, {3, 0}},
    {{0, 2, 1}, {0, 1, 3}, {1, 2, 3}, {0, 3, 2}},
    {{0, 3, 2, 1}, {4, 5, 6, 7}, {0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {3, 0, 4, 7}},
};
__constant__ int8_t c_nf[4] = {3, 4, 4, 6};
__constant__ int8_t c_nn[4] = {3, 4, 4, 8};
__constant__ int8_t c_flen[4] = {2, 2, 3, 4};

__device__ __forceinline__ int kind_index(int k) {
    return k == 5 ? 0 : (k == 9 ? 1 : (k == 10 ? 2 : (k == 12 ? 3 : -1)));
}

__global__ void k_elem_count(int64_t ne, int dim, const int32_t *__restrict__ kind,
                             const int32_t *__restrict__ eptr, int64_t en_len, int32_t *__restrict__ nf,
                             int *flags) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int bad = 0, hex = 0;
    if (e < ne) {
        const int ki = kind_index(kind[e]);
        const int64_t p0 = eptr[e], p1 = eptr[e + 1];
        const bool ok = ki >= 0 && ((dim == 2) == (ki <= 1)) && p0 >= 0 && p1 <= en_len && p1 - p0 == c_nn[ki];
        nf[e] = ok ? c_nf[ki] : 0;
        bad = ok ? 0 : kBadElement;
        hex = ok && ki == 3;
    }
    const unsigned any_bad = __ballot_sync(0xffffffffu, bad != 0), any_hex = __ballot_sync(0xffffffffu, hex != 0);
    if ((threadIdx.x & 31) == 0 && (any_bad | any_hex))
        atomicOr(flags, (any_bad ? kBadElement : 0) | (any_hex ? kHasQuadFace : 0));
}

// One element per thread: its faces' sorted node keys, word w of record r at key[w * M + r].
__global__ void k_incidences(int64_t ne, const int32_t *__restrict__ kind, const int32_t *__restrict__ eptr,
                             const int32_t *__restrict__ en, const int32_t *__restrict__ efp, int64_t n_nodes,
                             int W, int64_t M, uint32_t *__restrict__ key, int32_t *__restrict__ rec_elem,
                             int *flags) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    const int ki = kind_index(kind[e]);
    const int32_t *v = en + eptr[e];
    const int64_t base = efp[e];
    const uint32_t pad = (uint32_t)n_nodes;
    int bad = 0;
    for (int l = 0; l < c_nf[ki]; ++l) {
        uint32_t s[4] = {pad, pad, pad, pad};
        for (int q = 0; q < c_flen[ki]; ++q) {
            const int32_t id = v[c_slot[ki][l][q]];
            if (id < 0 || (int64_t)id >= n_nodes)
                bad = kBadNode;
            else
                s[q] = (uint32_t)id;
        }
        for (int a = 1; a < 4; ++a)  // insertion sort of four words
            for (int b = a; b > 0 && s[b - 1] > s[b]; --b) {
                const uint32_t t = s[b];
                s[b] = s[b - 1];
                s[b - 1] = t;
            }
        for (int w = 0; w < W; ++w) key[w * M + base + l] = s[w];
        rec_elem[base + l] = (int32_t)e;
    }
    if (bad) atomicOr(flags, bad);
}

// Boundary faces of the input (already checked on the host), records L .. L + nb - 1.
__global__ void k_bface_keys(int64_t nb, const int32_t *__restrict__ bptr, const int32_t *__restrict__ bn,
                             int64_t n_nodes, int W, int64_t M, int64_t L, uint32_t *__restrict__ key) {
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const uint32_t pad = (uint32_t)n_nodes;
    uint32_t s[4] = {pad, pad, pad, pad};
    for (int q = 0; q < bptr[b + 1] - bptr[b]; ++q) s[q] = (uint32_t)bn[bptr[b] + q];
    for (int a = 1; a < 4; ++a)
        for (int c = a; c > 0 && s[c - 1] > s[c]; --c) {
            const uint32_t t = s[c];
            s[c] = s[c - 1];
            s[c - 1] = t;
        }
    for (int w = 0; w < W; ++w) key[w * M + L + b] = s[w];
}

__global__ void k_iota(int64_t n, int32_t *__restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (int32_t)i;
}

__global__ void k_gather_key(int64_t M, const uint32_t *__restrict__ kw, const int32_t *__restrict__ perm,
                             uint32_t *__restrict__ out) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < M) out[j] = kw[perm[j]];
}

__global__ void k_heads(int64_t M, int W, const uint32_t *__restrict__ key, const int32_t *__restrict__ perm,
                        int32_t *__restrict__ head) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= M) return;
    int h = 1;
    if (j > 0) {
        const int64_t r = perm[j], p = perm[j - 1];
        h = 0;
        for (int w = 0; w < W; ++w) h |= key[w * M + r] != key[w * M + p];
    }
    head[j] = h;
}

__global__ void k_group_start(int64_t M, const int32_t *__restrict__ head, const int32_t *__restrict__ gid1,
                              int32_t *__restrict__ gstart) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= M) return;
    if (head[j]) gstart[gid1[j] - 1] = (int32_t)j;
    if (j == M - 1) gstart[gid1[j]] = (int32_t)M;
}

// One group (a distinct face key) per thread: discoverer, neighbour, marker.
__global__ void k_groups(int64_t G, int64_t L, const int32_t *__restrict__ gstart, const int32_t *__restrict__ perm,
                         const int32_t *__restrict__ rec_elem, const int32_t *__restrict__ bmark,
                         uint64_t *__restrict__ gkey, int32_t *__restrict__ gidx, int2 *__restrict__ gcells,
                         int32_t *__restrict__ gmarker, int32_t *__restrict__ gfirst,
                         unsigned long long *__restrict__ counts, int *flags) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int valid = 0, interior = 0, bad = 0;
    if (g < G) {
        int first = -1, second = -1, marker = -1;
        for (int32_t j = gstart[g]; j < gstart[g + 1]; ++j) {
            const int32_t r = perm[j];
            if (r < L) {
                if (first < 0)
                    first = r;
                else if (second < 0)
                    second = r;
            } else if (marker < 0) {
                marker = bmark[r - L];
            }
        }
        gidx[g] = (int32_t)g;
        if (first < 0) {  // a boundary face of the input that no element has
            gkey[g] = ~0ULL;
        } else {
            valid = 1;
            interior = marker < 0;
            const int32_t owner = rec_elem[first];
            int32_t nb = -1;
            if (second >= 0) {
                const int32_t other = rec_elem[second];
                if (other == owner) bad |= kBadSelf;
                if (marker < 0)
                    nb = other;
                else
                    bad |= kBadForeign;
            }
            if (marker < 0 && nb < 0) bad |= kBadOpenFace;
            const uint64_t cls = marker < 0 ? 0u : (uint64_t)marker + 1u;
            gkey[g] = (cls << 32) | (uint32_t)first;
            gcells[g] = make_int2(owner, nb);
            gmarker[g] = marker;
            gfirst[g] = first;
        }
    }
    const unsigned vm = __ballot_sync(0xffffffffu, valid), im = __ballot_sync(0xffffffffu, interior);
    const unsigned bm = __ballot_sync(0xffffffffu, bad != 0);
    if ((threadIdx.x & 31) == 0) {
        if (vm) atomicAdd(&counts[0], (unsigned long long)__popc(vm));
        if (im) atomicAdd(&counts[1], (unsigned long long)__popc(im));
    }
    if (bm && bad) atomicOr(flags, bad);
}

// Faces in final order: cells, patch, node count; group -> face id.
__global__ void k_faces(int64_t F, const int32_t *__restrict__ gorder, const int2 *__restrict__ gcells,
                        const int32_t *__restrict__ gmarker, const int32_t *__restrict__ gfirst,
                        const int32_t *__restrict__ rec_elem, const int32_t *__restrict__ efp,
                        const int32_t *__restrict__ kind, int32_t *__restrict__ fid, int2 *__restrict__ face_cells,
                        int32_t *__restrict__ face_patch, int32_t *__restrict__ face_src,
                        int32_t *__restrict__ face_len) {
    const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) return;
    const int32_t g = gorder[f];
    fid[g] = (int32_t)f;
    face_cells[f] = gcells[g];
    face_patch[f] = gmarker[g];
    const int32_t r = gfirst[g];
    face_src[f] = r;
    face_len[f] = c_flen[kind_index(kind[rec_elem[r]])];
}

// calc_face_data (compute.rs:267-321) of face f from its node ids (any count).
template <int DIM>
__device__ __forceinline__ void face_geom(int64_t f, const int32_t *fn, int len, const double *__restrict__ nodes,
                                          double *__restrict__ area, double4 *__restrict__ normal4,
                                          double4 *__restrict__ center4) {
    double c[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < len; ++i)
#pragma unroll
        for (int d = 0; d < DIM; ++d) c[d] += nodes[(int64_t)fn[i] * DIM + d];
#pragma unroll
    for (int d = 0; d < DIM; ++d) c[d] /= (double)len;
    if (DIM == 2) {
        const double *n0 = nodes + (int64_t)fn[0] * 2;
        const double *n1 = nodes + (int64_t)fn[1] * 2;
        const double dn[2] = {n1[0] - n0[0], n1[1] - n0[1]};
        const double dsn[2] = {-dn[1], dn[0]};
        double dd = 0.0;
        dd += dsn[0] * dsn[0];
        dd += dsn[1] * dsn[1];
        const double a = sqrt(dd);
        area[f] = a;
        normal4[f] = make_double4(dsn[0] / a, dsn[1] / a, 0.0, 0.0);
        center4[f] = make_double4((n0[0] + n1[0]) * 0.5, (n0[1] + n1[1]) * 0.5, 0.0, 0.0);
        return;
    }
    double ctr[3] = {0.0, 0.0, 0.0}, nrm[3] = {0.0, 0.0, 0.0};
    double a = 0.0;
    for (int i = 0; i < len; ++i) {
        const double *n0 = nodes + (int64_t)fn[i] * 3;
        const double *n1 = nodes + (int64_t)fn[i == len - 1 ? 0 : i + 1] * 3;
        const double d0[3] = {n0[0] - c[0], n0[1] - c[1], n0[2] - c[2]};
        const double d1[3] = {n1[0] - c[0], n1[1] - c[1], n1[2] - c[2]};
        double dsn[3];
        dsn[0] = d0[1] * d1[2] - d0[2] * d1[1];
        dsn[1] = d0[2] * d1[0] - d0[0] * d1[2];
        dsn[2] = d0[0] * d1[1] - d0[1] * d1[0];
#pragma unroll
        for (int d = 0; d < 3; ++d) dsn[d] *= 0.5;
        double dd = 0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) dd += dsn[d] * dsn[d];
        const double ai = sqrt(dd);
        a += ai;
#pragma unroll
        for (int d = 0; d < 3; ++d) nrm[d] = dsn[d];  // the last triangle's normal (compute.rs:305)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double t = n0[d] + n1[d];
            t = t + c[d];
            t = t * 1.0;
            t = t / 3.0;
            t = t * ai;
            ctr[d] += t;
        }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        nrm[d] /= a;
        ctr[d] /= a;
    }
    area[f] = a;
    normal4[f] = make_double4(nrm[0], nrm[1], nrm[2], 0.0);
    center4[f] = make_double4(ctr[0], ctr[1], ctr[2], 0.0);
}

// Face f of the element build, its nodes in the discoverer's local order.
template <int DIM>
__global__ void k_face_geom(int64_t F, const int32_t *__restrict__ face_src, const int32_t *__restrict__ rec_elem,
                            const int32_t *__restrict__ efp, const int32_t *__restrict__ kind,
                            const int32_t *__restrict__ eptr, const int32_t *__restrict__ en,
                            const double *__restrict__ nodes, const int32_t *__restrict__ fnp,
                            int32_t *__restrict__ face_nodes, double *__restrict__ area,
                            double4 *__restrict__ normal4, double4 *__restrict__ center4) {
    const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) return;
    const int32_t r = face_src[f];
    const int32_t e = rec_elem[r];
    const int ki = kind_index(kind[e]);
    const int l = r - efp[e];
    const int len = c_flen[ki];
    int32_t fn[4];
    for (int q = 0; q < len; ++q) {
        fn[q] = en[eptr[e] + c_slot[ki][l][q]];
        face_nodes[fnp[f] + q] = fn[q];
    }
    face_geom<DIM>(f, fn, len, nodes, area, normal4, center4);
}

// Faces given as node lists (fv_mesh_build_faces).
template <int DIM>
__global__ void k_face_geom_list(int64_t F, const int32_t *__restrict__ fnp, const int32_t *__restrict__ fnodes,
                                 const double *__restrict__ nodes, double *__restrict__ area,
                                 double4 *__restrict__ normal4, double4 *__restrict__ center4) {
    const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) return;
    face_geom<DIM>(f, fnodes + fnp[f], fnp[f + 1] - fnp[f], nodes, area, normal4, center4);
}

__global__ void k_cell_faces(int64_t M, int64_t L, const int32_t *__restrict__ perm, const int32_t *__restrict__ gid1,
                             const int32_t *__restrict__ fid, int32_t *__restrict__ cell_faces) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= M) return;
    const int32_t r = perm[j];
    if (r < L) cell_faces[r] = fid[gid1[j] - 1];
}

// calc_cell_data (compute.rs:325-375), the face centres averaged in cell_faces order.
template <int DIM>
__global__ void k_cell_geom(int64_t N, const int32_t *__restrict__ cptr, const int32_t *__restrict__ cfaces,
                            const double *__restrict__ area, const double4 *__restrict__ normal4,
                            const double4 *__restrict__ center4, double4 *__restrict__ cell) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    const int s = cptr[c], len = cptr[c + 1] - s;
    double ave[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < len; ++i) {
        const double4 q = center4[cfaces[s + i]];
        const double fc[3] = {q.x, q.y, q.z};
#pragma unroll
        for (int d = 0; d < DIM; ++d) ave[d] += fc[d];
    }
#pragma unroll
    for (int d = 0; d < DIM; ++d) ave[d] /= (double)len;
    const double vdiv = DIM == 2 ? 2.0 : 3.0, cmul = DIM == 2 ? 2.0 : 3.0, cdiv = DIM == 2 ? 3.0 : 4.0;
    double ctr[3] = {0.0, 0.0, 0.0};
    double vol = 0.0;
    for (int i = 0; i < len; ++i) {
        const int32_t f = cfaces[s + i];
        const double4 q = center4[f], n = normal4[f];
        const double fc[3] = {q.x, q.y, q.z}, fnv[3] = {n.x, n.y, n.z};
        double dfc[3];
#pragma unroll
        for (int d = 0; d < DIM; ++d) dfc[d] = fc[d] - ave[d];
        double h = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) h += dfc[d] * fnv[d];
        h = fabs(h);
        const double vi = h * area[f] / vdiv;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const double ci = (fc[d] * cmul + ave[d]) / cdiv;
            ctr[d] += ci * vi;
        }
        vol += vi;
    }
    double out[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int d = 0; d < DIM; ++d) out[d] = ctr[d] / vol;
    cell[c] = make_double4(out[0], out[1], out[2], vol);
}

// Orientation (compute.rs:97-131): the normal points away from the owner.
template <int DIM>
__global__ void k_orient(int64_t F, const int2 *__restrict__ fc, const double4 *__restrict__ cell,
                         const double4 *__restrict__ center4, double4 *__restrict__ normal4) {
    const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) return;
    const double4 ip4 = cell[fc[f].x], c4 = center4[f], n4 = normal4[f];
    const double ip[3] = {ip4.x, ip4.y, ip4.z}, fcv[3] = {c4.x, c4.y, c4.z};
    double nv[3] = {n4.x, n4.y, n4.z};
    double s = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) s += nv[d] * (fcv[d] - ip[d]);
    if (s < 0.0) {
#pragma unroll
        for (int d = 0; d < DIM; ++d) nv[d] *= -1.0;
        normal4[f] = make_double4(nv[0], nv[1], nv[2], 0.0);
    }
}

// Cell -> faces where the cell is owner or neighbour, ascending face id (the
// layout fv_mesh_upload builds): counts, then the lists.
__global__ void k_cf_count(int64_t N, const int32_t *__restrict__ cptr, const int32_t *__restrict__ cfaces,
                           const int2 *__restrict__ fc, int32_t *__restrict__ cnt, int *maxf, int *flags) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int n = 0, bad = 0;
    if (c < N) {
        for (int k = cptr[c]; k < cptr[c + 1]; ++k) {
            const int2 on = fc[cfaces[k]];
            if (on.x == (int)c || on.y == (int)c)
                ++n;
            else
                bad = kBadForeign;
        }
        cnt[c] = n;
    }
    const int wmax = __reduce_max_sync(0xffffffffu, n);
    const unsigned bm = __ballot_sync(0xffffffffu, bad != 0);
    if ((threadIdx.x & 31) == 0) {
        atomicMax(maxf, wmax);
        if (bm) atomicOr(flags, kBadForeign);
    }
}

__global__ void k_cf_fill(int64_t N, const int32_t *__restrict__ cptr, const int32_t *__restrict__ cfaces,
                          const int2 *__restrict__ fc, const int32_t *__restrict__ cf_ptr,
                          int32_t *__restrict__ cf_face, int32_t *__restrict__ cf_other, int padf,
                          int2 *__restrict__ cf_pad) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    int32_t face[16], other[16];
    int n = 0;
    for (int k = cptr[c]; k < cptr[c + 1] && n < 16; ++k) {
        const int32_t f = cfaces[k];
        const int2 on = fc[f];
        if (on.x == (int)c) {
            face[n] = f;
            other[n++] = on.y;
        } else if (on.y == (int)c) {
            face[n] = f | (int32_t)0x80000000;
            other[n++] = on.x;
        }
    }
    for (int a = 1; a < n; ++a)  // ascending face id
        for (int b = a; b > 0 && (face[b - 1] & 0x7fffffff) > (face[b] & 0x7fffffff); --b) {
            const int32_t tf = face[b], to = other[b];
            face[b] = face[b - 1];
            other[b] = other[b - 1];
            face[b - 1] = tf;
            other[b - 1] = to;
        }
    const int32_t o = cf_ptr[c];
    for (int k = 0; k < n; ++k) {
        cf_face[o + k] = face[k];
        cf_other[o + k] = other[k];
    }
    if (padf)
        for (int k = 0; k < padf; ++k)
            cf_pad[c * padf + k] = k < n ? make_int2(face[k], other[k]) : make_int2(0, -2);
}

// add_cell (mod.rs:489-529) for explicit cell lists: with k the position of a
// (cell, face) entry in cell_faces (k grows with the cell), the face's owner
// is the cell of its smallest k and its neighbour the cell of the second
// smallest, unless the face is tagged.
__global__ void k_first_listing(int64_t N, const int32_t *__restrict__ cptr, const int32_t *__restrict__ cfaces,
                                int32_t *__restrict__ rec_cell, int32_t *__restrict__ first) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    for (int32_t k = cptr[c]; k < cptr[c + 1]; ++k) {
        rec_cell[k] = (int32_t)c;
        atomicMin(&first[cfaces[k]], k);
    }
}

__global__ void k_second_listing(int64_t L, const int32_t *__restrict__ cfaces, const int32_t *__restrict__ first,
                                 int32_t *__restrict__ second) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= L) return;
    const int32_t f = cfaces[k];
    if (first[f] != (int32_t)k) atomicMin(&second[f], (int32_t)k);
}

__global__ void k_listed_cells(int64_t F, const int32_t *__restrict__ first, const int32_t *__restrict__ second,
                               const int32_t *__restrict__ rec_cell, const int32_t *__restrict__ patch,
                               int2 *__restrict__ face_cells, int *flags) {
    const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int bad = 0;
    if (f < F) {
        const int32_t k1 = first[f], k2 = second[f];
        if (k1 == INT32_MAX) {
            bad = kBadOpenFace;
            face_cells[f] = make_int2(0, -1);
        } else {
            const int32_t owner = rec_cell[k1];
            int32_t nb = -1;
            if (k2 != INT32_MAX && patch[f] < 0) nb = rec_cell[k2];
            if (nb == owner) bad |= kBadSelf;
            if (patch[f] < 0 && nb < 0) bad |= kBadOpenFace;
            face_cells[f] = make_int2(owner, nb);
        }
    }
    const unsigned bm = __ballot_sync(0xffffffffu, bad != 0);
    if (bm && bad) atomicOr(flags, bad);
}

__global__ void k_fill_i32(int64_t n, int32_t v, int32_t *__restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = v;
}

int bitlen(uint64_t x) { return x ? 64 - __builtin_clzll(x) : 0; }

inline unsigned blocks(int64_t n) { return (unsigned)((n + kB - 1) / kB); }

// Scratch memory from the stream-ordered pool, released when the build returns.
struct Scratch {
    cudaStream_t st;
    std::vector<void *> ptrs;
    cudaError_t err = cudaSuccess;
    explicit Scratch(cudaStream_t s) : st(s) {}
    ~Scratch() {
        for (void *p : ptrs) cudaFreeAsync(p, st);
    }
    template <typename T>
    T *get(size_t count) {
        T *p = nullptr;
        if (err != cudaSuccess) return nullptr;
        err = fv_malloc_async(&p, sizeof(T) * (count ? count : 1), st);
        if (err == cudaSuccess) ptrs.push_back(p);
        return p;
    }
};

fv_status fail(cudaError_t e, const char *what) {
    fv_internal_set_cuda_error(e, what);
    return e == cudaErrorMemoryAllocation ? FV_ERR_ALLOC : FV_ERR_CUDA;
}

fv_status flag_status(int flags) {
    if (flags & kBadElement) fv_internal_set_error_text("fv_mesh_build: invalid element (kind, node count or dimension)");
    else if (flags & kBadNode) fv_internal_set_error_text("fv_mesh_build: element node id out of range");
    else if (flags & kBadOpenFace) fv_internal_set_error_text("fv_mesh_build: unmarked face with one cell (missing boundary marker)");
    else if (flags & kBadSelf) fv_internal_set_error_text("fv_mesh_build: an element lists one face twice");
    else if (flags & kBadForeign) fv_internal_set_error_text("fv_mesh_build: a marked face is shared by two elements");
    else return FV_OK;
    return FV_ERR_INVALID;
}

template <typename T>
cudaError_t sort_pairs(Scratch &sc, const T *kin, T *kout, const int32_t *vin, int32_t *vout, int64_t n, int end_bit) {
    size_t bytes = 0;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, bytes, kin, kout, vin, vout, (int)n, 0, end_bit, sc.st);
    if (e != cudaSuccess) return e;
    void *tmp = sc.get<uint8_t>(bytes);
    if (sc.err != cudaSuccess) return sc.err;
    return cub::DeviceRadixSort::SortPairs(tmp, bytes, kin, kout, vin, vout, (int)n, 0, end_bit, sc.st);
}

template <typename T>
cudaError_t scan(Scratch &sc, const T *in, T *out, int64_t n, bool inclusive) {
    size_t bytes = 0;
    cudaError_t e = inclusive ? cub::DeviceScan::InclusiveSum(nullptr, bytes, in, out, (int)n, sc.st)
                              : cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, (int)n, sc.st);
    if (e != cudaSuccess) return e;
    void *tmp = sc.get<uint8_t>(bytes);
    if (sc.err != cudaSuccess) return sc.err;
    return inclusive ? cub::DeviceScan::InclusiveSum(tmp, bytes, in, out, (int)n, sc.st)
                     : cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, (int)n, sc.st);
}

template <typename T>
cudaError_t to_device(Scratch &sc, T *&dst, const T *src, size_t count) {
    dst = sc.get<T>(count);
    if (sc.err != cudaSuccess) return sc.err;
    return count ? cudaMemcpyAsync(dst, src, sizeof(T) * count, cudaMemcpyHostToDevice, sc.st) : cudaSuccess;
}

// The host mirror of the built mesh (the arrays fv_host_mesh_from_elements returns).
fv_status read_back(const fv_mesh *m, int dim, int64_t n_nodes, const double *nodes, const int32_t *fnp,
                    const int32_t *fnodes, const int32_t *fpatch, const int32_t *cptr, const int32_t *cfaces,
                    cudaStream_t st, fv_host_mesh **host_out) {
    const int64_t F = m->n_faces, N = m->n_cells;
    fv_host_mesh *h = (fv_host_mesh *)std::calloc(1, sizeof(fv_host_mesh));
    if (!h) return FV_ERR_ALLOC;
    h->dim = dim;
    h->n_nodes = n_nodes;
    h->n_faces = F;
    h->n_cells = N;
    h->n_boundary_faces = m->n_bfaces;
    h->nodes = (double *)std::malloc(sizeof(double) * n_nodes * dim);
    h->face_node_ptr = (int32_t *)std::malloc(sizeof(int32_t) * (F + 1));
    h->face_patch = (int32_t *)std::malloc(sizeof(int32_t) * F);
    h->face_owner = (int32_t *)std::malloc(sizeof(int32_t) * F);
    h->face_neighbor = (int32_t *)std::malloc(sizeof(int32_t) * F);
    h->face_area = (double *)std::malloc(sizeof(double) * F);
    h->face_normal = (double *)std::malloc(sizeof(double) * F * dim);
    h->face_center = (double *)std::malloc(sizeof(double) * F * dim);
    h->cell_face_ptr = (int32_t *)std::malloc(sizeof(int32_t) * (N + 1));
    h->cell_center = (double *)std::malloc(sizeof(double) * N * dim);
    h->cell_volume = (double *)std::malloc(sizeof(double) * N);
    std::vector<int2> fc;
    std::vector<double4> fn4, fc4, cell;
    try {
        fc.resize((size_t)F);
        fn4.resize((size_t)F);
        fc4.resize((size_t)F);
        cell.resize((size_t)N);
    } catch (const std::bad_alloc &) {
        fv_host_mesh_free(h);
        return FV_ERR_ALLOC;
    }
    if (!h->nodes || !h->face_node_ptr || !h->face_patch || !h->face_owner || !h->face_neighbor || !h->face_area ||
        !h->face_normal || !h->face_center || !h->cell_face_ptr || !h->cell_center || !h->cell_volume) {
        fv_host_mesh_free(h);
        return FV_ERR_ALLOC;
    }
    std::memcpy(h->nodes, nodes, sizeof(double) * n_nodes * dim);
    cudaError_t e = cudaMemcpyAsync(h->face_node_ptr, fnp, sizeof(int32_t) * (F + 1), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->cell_face_ptr, cptr, sizeof(int32_t) * (N + 1), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) {
        h->face_nodes = (int32_t *)std::malloc(sizeof(int32_t) * (h->face_node_ptr[F] ? h->face_node_ptr[F] : 1));
        h->cell_faces = (int32_t *)std::malloc(sizeof(int32_t) * (h->cell_face_ptr[N] ? h->cell_face_ptr[N] : 1));
        if (!h->face_nodes || !h->cell_faces) {
            fv_host_mesh_free(h);
            return FV_ERR_ALLOC;
        }
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h->face_nodes, fnodes, sizeof(int32_t) * h->face_node_ptr[F], cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h->cell_faces, cfaces, sizeof(int32_t) * h->cell_face_ptr[N], cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->face_patch, fpatch, sizeof(int32_t) * F, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->face_area, m->face_area, sizeof(double) * F, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(fc.data(), m->face_cells, sizeof(int2) * F, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(fn4.data(), m->face_normal, sizeof(double4) * F, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(fc4.data(), m->face_center, sizeof(double4) * F, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(cell.data(), m->cell, sizeof(double4) * N, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        fv_host_mesh_free(h);
        return fail(e, "fv_mesh_build_elements (read back)");
    }
#pragma omp parallel for schedule(static)
    for (int64_t f = 0; f < F; ++f) {
        h->face_owner[f] = fc[f].x;
        h->face_neighbor[f] = fc[f].y;
        const double n[3] = {fn4[f].x, fn4[f].y, fn4[f].z}, c[3] = {fc4[f].x, fc4[f].y, fc4[f].z};
        for (int d = 0; d < dim; ++d) {
            h->face_normal[f * dim + d] = n[d];
            h->face_center[f * dim + d] = c[d];
        }
    }
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < N; ++c) {
        const double x[3] = {cell[c].x, cell[c].y, cell[c].z};
        for (int d = 0; d < dim; ++d) h->cell_center[c * dim + d] = x[d];
        h->cell_volume[c] = cell[c].w;
    }
    *host_out = h;
    return FV_OK;
}


// Everything after the faces exist (cells listed, face_cells, unoriented face
// geometry): cell geometry, orientation, the cell -> face lists of the
// assembly kernels, gradient coefficients and the optional host copy.
// m->gcf_ptr / m->gcf_face hold the cells' faces in mesh order (L entries).
fv_status finish(Scratch &sc, fv_mesh *m, int64_t L, int *d_flags, int64_t n_nodes, const double *nodes,
                 const int32_t *fnp, const int32_t *fnodes, const int32_t *face_patch, fv_host_mesh **host_out) {
    cudaStream_t st = sc.st;
    const int dim = m->dim;
    const int64_t N = m->n_cells, F = m->n_faces, n_int = F - m->n_bfaces;
    cudaError_t e = cudaSuccess;
    fv_note_launch();
    if (dim == 2)
        k_cell_geom<2><<<blocks(N), kB, 0, st>>>(N, m->gcf_ptr, m->gcf_face, m->face_area, m->face_normal,
                                                 m->face_center, m->cell);
    else
        k_cell_geom<3><<<blocks(N), kB, 0, st>>>(N, m->gcf_ptr, m->gcf_face, m->face_area, m->face_normal,
                                                 m->face_center, m->cell);
    fv_note_launch();
    if (dim == 2)
        k_orient<2><<<blocks(F), kB, 0, st>>>(F, m->face_cells, m->cell, m->face_center, m->face_normal);
    else
        k_orient<3><<<blocks(F), kB, 0, st>>>(F, m->face_cells, m->cell, m->face_center, m->face_normal);
    e = cudaGetLastError();
    if (e == cudaSuccess && F > n_int)
        e = cudaMemcpyAsync(m->bface_center, m->face_center + n_int, sizeof(double4) * (F - n_int),
                            cudaMemcpyDeviceToDevice, st);

    // cell -> faces lists of the assembly kernels
    int32_t *cnt = sc.get<int32_t>((size_t)N + 1);
    int *d_maxf = d_flags + 1;
    if (e == cudaSuccess) e = sc.err;
    if (e == cudaSuccess) e = cudaMalloc(&m->cf_ptr, sizeof(int32_t) * (N + 1));
    if (e == cudaSuccess) e = cudaMemsetAsync(cnt + N, 0, sizeof(int32_t), st);
    if (e == cudaSuccess) {
        fv_note_launch();
        k_cf_count<<<blocks(N), kB, 0, st>>>(N, m->gcf_ptr, m->gcf_face, m->face_cells, cnt, d_maxf, d_flags);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = scan(sc, cnt, m->cf_ptr, N + 1, false);
    int32_t ncf = 0;
    int h_flags[4] = {0, 0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(&ncf, m->cf_ptr + N, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_flags, d_flags, sizeof(int) * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(e, "fv_mesh_build (geometry)");
    if (flag_status(h_flags[0]) != FV_OK) return FV_ERR_INVALID;
    const int maxf = h_flags[1];
    if (maxf > 16) {
        fv_internal_set_error_text("fv_mesh_build: a cell with more than 16 faces");
        return FV_ERR_UNSUPPORTED;
    }
    m->maxf = maxf;
    m->ncf = ncf;
    m->padf = maxf <= 4 ? 4 : (maxf <= 8 ? 8 : 0);
    e = cudaMalloc(&m->cf_face, sizeof(int32_t) * (ncf ? ncf : 1));
    if (e == cudaSuccess) e = cudaMalloc(&m->cf_other, sizeof(int32_t) * (ncf ? ncf : 1));
    if (e == cudaSuccess && m->padf) e = cudaMalloc(&m->cf_pad, sizeof(int2) * N * m->padf);
    if (e == cudaSuccess) {
        fv_note_launch();
        k_cf_fill<<<blocks(N), kB, 0, st>>>(N, m->gcf_ptr, m->gcf_face, m->face_cells, m->cf_ptr, m->cf_face,
                                            m->cf_other, m->padf, m->cf_pad);
        e = cudaGetLastError();
    }

    // gradient coefficients (compute.rs:155-203) over the mesh-order cell faces
    int *d_gbad = d_flags + 2;
    if (e == cudaSuccess) e = cudaMalloc(&m->gcoef, sizeof(double4) * (L ? L : 1));
    if (e == cudaSuccess) e = cudaMalloc(&m->gdiag, sizeof(double4) * N);
    if (e == cudaSuccess) e = fv_mesh_launch_grad_coeffs(m, d_gbad, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_flags, d_flags, sizeof(int) * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(e, "fv_mesh_build (cell faces)");
    if (h_flags[2]) {  // Mesh::compute returns Error::SingularMatrix
        fv_internal_set_error_text("fv_mesh_build: singular gradient matrix of a cell");
        return FV_ERR_INVALID;
    }
    if (host_out)
        return read_back(m, dim, n_nodes, nodes, fnp, fnodes, face_patch, m->gcf_ptr, m->gcf_face, st, host_out);
    return FV_OK;
}

}  // namespace

extern "C" fv_status fv_mesh_build_elements(int32_t dim, int64_t n_nodes, const double *nodes, int64_t n_elems,
                                            const int32_t *elem_kind, const int32_t *elem_node_ptr,
                                            const int32_t *elem_nodes, int64_t n_bfaces,
                                            const int32_t *bface_node_ptr, const int32_t *bface_nodes,
                                            const int32_t *bface_marker, void *stream, fv_mesh **out,
                                            fv_host_mesh **host_out) {
    if (!out || (dim != 2 && dim != 3) || n_nodes <= 0 || n_elems <= 0 || !nodes || !elem_kind || !elem_node_ptr ||
        !elem_nodes || n_bfaces < 0 || n_nodes >= 0x7fffffffLL || n_elems >= (0x7fffffffLL / 8))
        return FV_ERR_INVALID;
    if (n_bfaces > 0 && (!bface_node_ptr || !bface_nodes || !bface_marker)) return FV_ERR_INVALID;
    *out = nullptr;
    if (host_out) *host_out = nullptr;
    // boundary faces: checked here (few), as fv_host_mesh_from_elements does
    int bmax_len = 0, max_marker = -1;
    if (n_bfaces > 0) {
        if (bface_node_ptr[0] != 0) return FV_ERR_INVALID;
        for (int64_t b = 0; b < n_bfaces; ++b) {
            const int len = bface_node_ptr[b + 1] - bface_node_ptr[b];
            if (len < 2 || len > 4 || bface_marker[b] < 0) return FV_ERR_INVALID;
            for (int q = 0; q < len; ++q) {
                const int32_t id = bface_nodes[bface_node_ptr[b] + q];
                if (id < 0 || id >= n_nodes) return FV_ERR_INVALID;
            }
            bmax_len = std::max(bmax_len, len);
            max_marker = std::max(max_marker, bface_marker[b]);
        }
    }
    const int64_t en_len = elem_node_ptr[n_elems];
    if (en_len <= 0) return FV_ERR_INVALID;
    cudaStream_t st = fv_stream(stream);
    Scratch sc(st);
    cudaError_t e = cudaSuccess;
    double *d_nodes = nullptr;
    int32_t *d_kind = nullptr, *d_eptr = nullptr, *d_en = nullptr, *d_bptr = nullptr, *d_bn = nullptr, *d_bm = nullptr;
    e = to_device(sc, d_nodes, nodes, (size_t)(n_nodes * dim));
    if (e == cudaSuccess) e = to_device(sc, d_kind, elem_kind, (size_t)n_elems);
    if (e == cudaSuccess) e = to_device(sc, d_eptr, elem_node_ptr, (size_t)n_elems + 1);
    if (e == cudaSuccess) e = to_device(sc, d_en, elem_nodes, (size_t)en_len);
    if (e == cudaSuccess && n_bfaces > 0) e = to_device(sc, d_bptr, bface_node_ptr, (size_t)n_bfaces + 1);
    if (e == cudaSuccess && n_bfaces > 0) e = to_device(sc, d_bn, bface_nodes, (size_t)bface_node_ptr[n_bfaces]);
    if (e == cudaSuccess && n_bfaces > 0) e = to_device(sc, d_bm, bface_marker, (size_t)n_bfaces);
    int32_t *efp = nullptr;  // element -> first record; becomes the mesh's cell_face_ptr
    int *d_flags = sc.get<int>(4);
    unsigned long long *d_counts = sc.get<unsigned long long>(2);
    int32_t *nf = sc.get<int32_t>((size_t)n_elems + 1);
    if (e == cudaSuccess) e = sc.err;
    if (e == cudaSuccess) e = cudaMalloc(&efp, sizeof(int32_t) * (n_elems + 1));
    fv_mesh *m = new fv_mesh();
    m->gcf_ptr = efp;
    auto give_up = [&](fv_status s) {
        fv_mesh_destroy(m);
        return s;
    };
    if (e == cudaSuccess) e = cudaMemsetAsync(d_flags, 0, sizeof(int) * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_counts, 0, sizeof(unsigned long long) * 2, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(nf + n_elems, 0, sizeof(int32_t), st);
    if (e == cudaSuccess) {
        fv_note_launch();
        k_elem_count<<<blocks(n_elems), kB, 0, st>>>(n_elems, dim, d_kind, d_eptr, en_len, nf, d_flags);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = scan(sc, nf, efp, n_elems + 1, false);
    int h_flags[4] = {0, 0, 0, 0};
    int32_t L32 = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_flags, d_flags, sizeof(int) * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&L32, efp + n_elems, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return give_up(fail(e, "fv_mesh_build_elements (elements)"));
    if (flag_status(h_flags[0]) != FV_OK) return give_up(FV_ERR_INVALID);
    const int64_t L = L32, M = L + n_bfaces;
    if (M >= 0x7fffffffLL) return give_up(FV_ERR_UNSUPPORTED);
    const int W = std::max(dim == 2 ? 2 : ((h_flags[0] & kHasQuadFace) ? 4 : 3), bmax_len);
    const int bits = bitlen((uint64_t)n_nodes);

    // records, then the stable LSD sort over the key words (last word first)
    uint32_t *key = sc.get<uint32_t>((size_t)(W * M));
    uint32_t *tk = sc.get<uint32_t>((size_t)M), *tk2 = sc.get<uint32_t>((size_t)M);
    int32_t *rec_elem = sc.get<int32_t>((size_t)L);
    int32_t *perm = sc.get<int32_t>((size_t)M), *perm2 = sc.get<int32_t>((size_t)M);
    if (sc.err != cudaSuccess) return give_up(fail(sc.err, "fv_mesh_build_elements (records)"));
    fv_note_launch();
    k_incidences<<<blocks(n_elems), kB, 0, st>>>(n_elems, d_kind, d_eptr, d_en, efp, n_nodes, W, M, key, rec_elem,
                                                 d_flags);
    if (n_bfaces > 0)
        fv_note_launch(), k_bface_keys<<<blocks(n_bfaces), kB, 0, st>>>(n_bfaces, d_bptr, d_bn, n_nodes, W, M, L, key);
    fv_note_launch();
    k_iota<<<blocks(M), kB, 0, st>>>(M, perm);
    e = cudaGetLastError();
    for (int w = W - 1; w >= 0 && e == cudaSuccess; --w) {
        const uint32_t *kin = key + (size_t)w * M;
        if (w != W - 1) {
            fv_note_launch();
            k_gather_key<<<blocks(M), kB, 0, st>>>(M, kin, perm, tk);
            kin = tk;
        }
        e = sort_pairs(sc, kin, tk2, perm, perm2, M, bits);
        std::swap(perm, perm2);
    }
    int32_t *head = perm2, *gid1 = sc.get<int32_t>((size_t)M);  // perm2 is free after the last pass
    int32_t *gstart = sc.get<int32_t>((size_t)M + 1);
    if (e == cudaSuccess) e = sc.err;
    if (e == cudaSuccess) {
        fv_note_launch();
        k_heads<<<blocks(M), kB, 0, st>>>(M, W, key, perm, head);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = scan(sc, head, gid1, M, true);
    if (e == cudaSuccess) {
        fv_note_launch();
        k_group_start<<<blocks(M), kB, 0, st>>>(M, head, gid1, gstart);
        e = cudaGetLastError();
    }
    int32_t G32 = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&G32, gid1 + (M - 1), sizeof(int32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_flags, d_flags, sizeof(int) * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return give_up(fail(e, "fv_mesh_build_elements (face keys)"));
    if (flag_status(h_flags[0]) != FV_OK) return give_up(FV_ERR_INVALID);
    const int64_t G = G32;

    // one entry per distinct key, then the face numbering sort
    uint64_t *gkey = sc.get<uint64_t>((size_t)G), *gkey2 = sc.get<uint64_t>((size_t)G);
    int32_t *gidx = sc.get<int32_t>((size_t)G), *gorder = sc.get<int32_t>((size_t)G);
    int2 *gcells = sc.get<int2>((size_t)G);
    int32_t *gmarker = sc.get<int32_t>((size_t)G), *gfirst = sc.get<int32_t>((size_t)G);
    if (sc.err != cudaSuccess) return give_up(fail(sc.err, "fv_mesh_build_elements (groups)"));
    fv_note_launch();
    k_groups<<<blocks(G), kB, 0, st>>>(G, L, gstart, perm, rec_elem, d_bm, gkey, gidx, gcells, gmarker, gfirst,
                                       d_counts, d_flags);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = sort_pairs(sc, gkey, gkey2, gidx, gorder, G, 32 + bitlen((uint64_t)(max_marker + 1)) + 1);
    unsigned long long h_counts[2] = {0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_counts, d_counts, sizeof(h_counts), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_flags, d_flags, sizeof(int) * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return give_up(fail(e, "fv_mesh_build_elements (numbering)"));
    if (flag_status(h_flags[0]) != FV_OK) return give_up(FV_ERR_INVALID);
    const int64_t F = (int64_t)h_counts[0], n_int = (int64_t)h_counts[1];
    m->dim = dim;
    m->n_cells = n_elems;
    m->n_faces = F;
    m->n_bfaces = F - n_int;

    // faces: cells, patch, node lists and geometry
    int32_t *fid = sc.get<int32_t>((size_t)G), *face_patch = sc.get<int32_t>((size_t)F);
    int32_t *face_src = sc.get<int32_t>((size_t)F), *face_len = sc.get<int32_t>((size_t)F + 1);
    int32_t *fnp = sc.get<int32_t>((size_t)F + 1), *fnodes = sc.get<int32_t>((size_t)F * W);
    if (sc.err != cudaSuccess) return give_up(fail(sc.err, "fv_mesh_build_elements (faces)"));
    e = cudaMalloc(&m->face_cells, sizeof(int2) * F);
    if (e == cudaSuccess) e = cudaMalloc(&m->face_area, sizeof(double) * F);
    if (e == cudaSuccess) e = cudaMalloc(&m->face_normal, sizeof(double4) * F);
    if (e == cudaSuccess) e = cudaMalloc(&m->face_center, sizeof(double4) * F);
    if (e == cudaSuccess) e = cudaMalloc(&m->cell, sizeof(double4) * n_elems);
    if (e == cudaSuccess) e = cudaMalloc(&m->gcf_face, sizeof(int32_t) * L);
    if (e == cudaSuccess) e = cudaMalloc(&m->bface_center, sizeof(double4) * (F - n_int > 0 ? F - n_int : 1));
    if (e == cudaSuccess) e = cudaMemsetAsync(face_len + F, 0, sizeof(int32_t), st);
    if (e == cudaSuccess) {
        fv_note_launch();
        k_faces<<<blocks(F), kB, 0, st>>>(F, gorder, gcells, gmarker, gfirst, rec_elem, efp, d_kind, fid,
                                          m->face_cells, face_patch, face_src, face_len);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = scan(sc, face_len, fnp, F + 1, false);
    if (e == cudaSuccess) {
        fv_note_launch();
        if (dim == 2)
            k_face_geom<2><<<blocks(F), kB, 0, st>>>(F, face_src, rec_elem, efp, d_kind, d_eptr, d_en, d_nodes, fnp,
                                                     fnodes, m->face_area, m->face_normal, m->face_center);
        else
            k_face_geom<3><<<blocks(F), kB, 0, st>>>(F, face_src, rec_elem, efp, d_kind, d_eptr, d_en, d_nodes, fnp,
                                                     fnodes, m->face_area, m->face_normal, m->face_center);
        fv_note_launch();
        k_cell_faces<<<blocks(M), kB, 0, st>>>(M, L, perm, gid1, fid, m->gcf_face);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return give_up(fail(e, "fv_mesh_build_elements (faces)"));
    const fv_status fs = finish(sc, m, L, d_flags, n_nodes, nodes, fnp, fnodes, face_patch, host_out);
    if (fs != FV_OK) return give_up(fs);
    *out = m;
    return FV_OK;
}

// Mesh::compute on the device for explicit faces and cells (the layout of the
// crate's own mesh files): owner / neighbour as add_cell assigns them, then
// the same geometry, orientation, cell-face lists and gradient coefficients.
extern "C" fv_status fv_mesh_build_faces(int32_t dim, int64_t n_nodes, const double *nodes, int64_t n_faces,
                                         const int32_t *face_node_ptr, const int32_t *face_nodes,
                                         const int32_t *face_patch, int64_t n_cells, const int32_t *cell_face_ptr,
                                         const int32_t *cell_faces, void *stream, fv_mesh **out,
                                         fv_host_mesh **host_out) {
    if (!out || (dim != 2 && dim != 3) || n_nodes <= 0 || n_faces <= 0 || n_cells <= 0 || !nodes ||
        !face_node_ptr || !face_nodes || !face_patch || !cell_face_ptr || !cell_faces || n_nodes >= 0x7fffffffLL ||
        n_faces >= 0x7fffffffLL || n_cells >= 0x7fffffffLL || face_node_ptr[0] != 0 || cell_face_ptr[0] != 0)
        return FV_ERR_INVALID;
    *out = nullptr;
    if (host_out) *host_out = nullptr;
    // index ranges are checked here: the kernels below index with them
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
            fv_internal_set_error_text("fv_mesh_build_faces: tagged faces must be the tail of the face list");
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
    const int64_t F = n_faces, N = n_cells, fnn = face_node_ptr[F], L = cell_face_ptr[N];
    cudaStream_t st = fv_stream(stream);
    Scratch sc(st);
    double *d_nodes = nullptr;
    int32_t *fnp = nullptr, *fnodes = nullptr, *patch = nullptr;
    cudaError_t e = to_device(sc, d_nodes, nodes, (size_t)(n_nodes * dim));
    if (e == cudaSuccess) e = to_device(sc, fnp, face_node_ptr, (size_t)F + 1);
    if (e == cudaSuccess) e = to_device(sc, fnodes, face_nodes, (size_t)fnn);
    if (e == cudaSuccess) e = to_device(sc, patch, face_patch, (size_t)F);
    int32_t *first = sc.get<int32_t>((size_t)F), *second = sc.get<int32_t>((size_t)F);
    int32_t *rec_cell = sc.get<int32_t>((size_t)L);
    int *d_flags = sc.get<int>(4);
    if (e == cudaSuccess) e = sc.err;
    fv_mesh *m = new fv_mesh();
    auto give_up = [&](fv_status s) {
        fv_mesh_destroy(m);
        return s;
    };
    m->dim = dim;
    m->n_cells = N;
    m->n_faces = F;
    m->n_bfaces = n_tagged;
    if (e == cudaSuccess) e = cudaMalloc(&m->gcf_ptr, sizeof(int32_t) * (N + 1));
    if (e == cudaSuccess) e = cudaMalloc(&m->gcf_face, sizeof(int32_t) * (L ? L : 1));
    if (e == cudaSuccess) e = cudaMalloc(&m->face_cells, sizeof(int2) * F);
    if (e == cudaSuccess) e = cudaMalloc(&m->face_area, sizeof(double) * F);
    if (e == cudaSuccess) e = cudaMalloc(&m->face_normal, sizeof(double4) * F);
    if (e == cudaSuccess) e = cudaMalloc(&m->face_center, sizeof(double4) * F);
    if (e == cudaSuccess) e = cudaMalloc(&m->cell, sizeof(double4) * N);
    if (e == cudaSuccess) e = cudaMalloc(&m->bface_center, sizeof(double4) * (n_tagged ? n_tagged : 1));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(m->gcf_ptr, cell_face_ptr, sizeof(int32_t) * (N + 1), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && L)
        e = cudaMemcpyAsync(m->gcf_face, cell_faces, sizeof(int32_t) * L, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_flags, 0, sizeof(int) * 4, st);
    if (e == cudaSuccess) {
        fv_note_launch();
        k_fill_i32<<<blocks(F), kB, 0, st>>>(F, INT32_MAX, first);
        fv_note_launch();
        k_fill_i32<<<blocks(F), kB, 0, st>>>(F, INT32_MAX, second);
        fv_note_launch();
        k_first_listing<<<blocks(N), kB, 0, st>>>(N, m->gcf_ptr, m->gcf_face, rec_cell, first);
        fv_note_launch();
        k_second_listing<<<blocks(L), kB, 0, st>>>(L, m->gcf_face, first, second);
        fv_note_launch();
        k_listed_cells<<<blocks(F), kB, 0, st>>>(F, first, second, rec_cell, patch, m->face_cells, d_flags);
        fv_note_launch();
        if (dim == 2)
            k_face_geom_list<2><<<blocks(F), kB, 0, st>>>(F, fnp, fnodes, d_nodes, m->face_area, m->face_normal,
                                                          m->face_center);
        else
            k_face_geom_list<3><<<blocks(F), kB, 0, st>>>(F, fnp, fnodes, d_nodes, m->face_area, m->face_normal,
                                                          m->face_center);
        e = cudaGetLastError();
    }
    int h_flags[4] = {0, 0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_flags, d_flags, sizeof(int) * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return give_up(fail(e, "fv_mesh_build_faces"));
    if (flag_status(h_flags[0]) != FV_OK) return give_up(FV_ERR_INVALID);
    const fv_status fs = finish(sc, m, L, d_flags, n_nodes, nodes, fnp, fnodes, patch, host_out);
    if (fs != FV_OK) return give_up(fs);
    *out = m;
    return FV_OK;
}

// ---------------------------------------------------------------- union of meshes
// One mesh from several resident meshes, laid out as a batch of independent
// problems: the interior faces of every part first (in part order), then the
// boundary faces of every part; cells in part order.  Each part keeps its
// faces' relative order, and interior faces stay ahead of boundary faces, so
// every cell's ascending face list maps to an ascending list: assembly and
// factorisation of the union give each part's own system on the diagonal,
// exactly as the same union uploaded from host arrays.  Gradient data is not
// carried over (the union has none, like a host upload without normals).
namespace {

struct CatPtrs {
    const int2 *const *face_cells;
    const double *const *face_area;
    const double4 *const *bface_center;
    const double4 *const *cell;
    const int32_t *const *cf_ptr;
    const int32_t *const *cf_face;
    const int32_t *const *cf_other;
    const int64_t *co, *io, *bo, *cfo, *fi;  // cell / interior-face / boundary-face / cf-entry offsets, interior faces
};

__device__ __forceinline__ int part_of(const int64_t *off, int P, int64_t x) {  // largest p with off[p] <= x
    int lo = 0, hi = P - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= x)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int32_t union_face(const CatPtrs &q, int64_t TI, int p, int32_t f) {
    return (int32_t)(f < q.fi[p] ? q.io[p] + f : TI + q.bo[p] + (f - q.fi[p]));
}

__global__ void k_cat_faces(int64_t F, int64_t TI, int P, CatPtrs q, int2 *__restrict__ fc, double *__restrict__ area,
                            double4 *__restrict__ bfc) {
    const int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= F) return;
    int p;
    int64_t f;
    if (u < TI) {
        p = part_of(q.io, P, u);
        f = u - q.io[p];
    } else {
        p = part_of(q.bo, P, u - TI);
        f = q.fi[p] + (u - TI - q.bo[p]);
    }
    const int2 on = q.face_cells[p][f];
    fc[u] = make_int2(on.x + (int32_t)q.co[p], on.y >= 0 ? on.y + (int32_t)q.co[p] : on.y);
    area[u] = q.face_area[p][f];
    if (u >= TI) bfc[u - TI] = q.bface_center[p][f - q.fi[p]];
}

__global__ void k_cat_cells(int64_t N, int64_t TI, int P, CatPtrs q, int padf, double4 *__restrict__ cell,
                            int32_t *__restrict__ cf_ptr, int32_t *__restrict__ cf_face,
                            int32_t *__restrict__ cf_other, int2 *__restrict__ cf_pad) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    const int p = part_of(q.co, P, c);
    const int64_t cl = c - q.co[p];
    cell[c] = q.cell[p][cl];
    const int32_t k0 = q.cf_ptr[p][cl], k1 = q.cf_ptr[p][cl + 1];
    const int64_t base = q.cfo[p];
    cf_ptr[c] = (int32_t)(base + k0);
    if (c == N - 1) cf_ptr[N] = (int32_t)q.cfo[P];
    for (int32_t k = k0; k < k1; ++k) {
        const int32_t raw = q.cf_face[p][k];
        const int32_t f = union_face(q, TI, p, raw & 0x7fffffff) | (raw & (int32_t)0x80000000);
        const int32_t o = q.cf_other[p][k];
        const int32_t other = o >= 0 ? o + (int32_t)q.co[p] : o;
        cf_face[base + k] = f;
        cf_other[base + k] = other;
        if (padf && k - k0 < padf) cf_pad[c * padf + (k - k0)] = make_int2(f, other);
    }
    for (int s = k1 - k0; s < padf; ++s) cf_pad[c * padf + s] = make_int2(0, -2);
}

}  // namespace

static fv_status mesh_concat_impl(const fv_mesh *const *parts, int32_t n_parts, void *stream, fv_mesh **out) {
    if (!parts || n_parts <= 0 || !out) return FV_ERR_INVALID;
    *out = nullptr;
    const int P = n_parts;
    const int dim = parts[0] ? parts[0]->dim : 0;
    std::vector<int64_t> co(P + 1, 0), io(P + 1, 0), bo(P + 1, 0), cfo(P + 1, 0), fi(P, 0);
    int maxf = 0;
    for (int p = 0; p < P; ++p) {
        const fv_mesh *m = parts[p];
        if (!m || m->dim != dim || !m->cf_ptr || m->n_cells <= 0) return FV_ERR_INVALID;
        fi[p] = m->n_faces - m->n_bfaces;
        co[p + 1] = co[p] + m->n_cells;
        io[p + 1] = io[p] + fi[p];
        bo[p + 1] = bo[p] + m->n_bfaces;
        cfo[p + 1] = cfo[p] + m->ncf;
        maxf = std::max(maxf, m->maxf);
    }
    const int64_t N = co[P], TI = io[P], TB = bo[P], F = TI + TB, NCF = cfo[P];
    if (N >= 0x7fffffffLL || F >= 0x7fffffffLL || NCF >= 0x7fffffffLL) return FV_ERR_UNSUPPORTED;
    cudaStream_t st = fv_stream(stream);
    std::vector<const void *> ptrs((size_t)7 * P);
    for (int p = 0; p < P; ++p) {
        ptrs[0 * P + p] = parts[p]->face_cells;
        ptrs[1 * P + p] = parts[p]->face_area;
        ptrs[2 * P + p] = parts[p]->bface_center;
        ptrs[3 * P + p] = parts[p]->cell;
        ptrs[4 * P + p] = parts[p]->cf_ptr;
        ptrs[5 * P + p] = parts[p]->cf_face;
        ptrs[6 * P + p] = parts[p]->cf_other;
    }
    std::vector<int64_t> offs;
    offs.reserve((size_t)5 * (P + 1));
    for (auto *v : {&co, &io, &bo, &cfo}) offs.insert(offs.end(), v->begin(), v->end());
    offs.insert(offs.end(), fi.begin(), fi.end());
    Scratch sc(st);
    const void **d_ptrs = nullptr;
    int64_t *d_offs = nullptr;
    cudaError_t e = to_device(sc, d_ptrs, ptrs.data(), ptrs.size());
    if (e == cudaSuccess) e = to_device(sc, d_offs, offs.data(), offs.size());
    fv_mesh *m = new fv_mesh();
    m->dim = dim;
    m->n_cells = N;
    m->n_faces = F;
    m->n_bfaces = TB;
    m->maxf = maxf;
    m->padf = maxf <= 4 ? 4 : (maxf <= 8 ? 8 : 0);
    m->ncf = NCF;
    if (e == cudaSuccess) e = cudaMalloc(&m->face_cells, sizeof(int2) * F);
    if (e == cudaSuccess) e = cudaMalloc(&m->face_area, sizeof(double) * F);
    if (e == cudaSuccess) e = cudaMalloc(&m->bface_center, sizeof(double4) * (TB ? TB : 1));
    if (e == cudaSuccess) e = cudaMalloc(&m->cell, sizeof(double4) * N);
    if (e == cudaSuccess) e = cudaMalloc(&m->cf_ptr, sizeof(int32_t) * (N + 1));
    if (e == cudaSuccess) e = cudaMalloc(&m->cf_face, sizeof(int32_t) * (NCF ? NCF : 1));
    if (e == cudaSuccess) e = cudaMalloc(&m->cf_other, sizeof(int32_t) * (NCF ? NCF : 1));
    if (e == cudaSuccess && m->padf) e = cudaMalloc(&m->cf_pad, sizeof(int2) * N * m->padf);
    if (e == cudaSuccess) {
        CatPtrs q;
        q.face_cells = reinterpret_cast<const int2 *const *>(d_ptrs + 0 * P);
        q.face_area = reinterpret_cast<const double *const *>(d_ptrs + 1 * P);
        q.bface_center = reinterpret_cast<const double4 *const *>(d_ptrs + 2 * P);
        q.cell = reinterpret_cast<const double4 *const *>(d_ptrs + 3 * P);
        q.cf_ptr = reinterpret_cast<const int32_t *const *>(d_ptrs + 4 * P);
        q.cf_face = reinterpret_cast<const int32_t *const *>(d_ptrs + 5 * P);
        q.cf_other = reinterpret_cast<const int32_t *const *>(d_ptrs + 6 * P);
        q.co = d_offs;
        q.io = d_offs + (P + 1);
        q.bo = d_offs + 2 * (P + 1);
        q.cfo = d_offs + 3 * (P + 1);
        q.fi = d_offs + 4 * (P + 1);
        fv_note_launch();
        k_cat_faces<<<blocks(F), kB, 0, st>>>(F, TI, P, q, m->face_cells, m->face_area, m->bface_center);
        fv_note_launch();
        k_cat_cells<<<blocks(N), kB, 0, st>>>(N, TI, P, q, m->padf, m->cell, m->cf_ptr, m->cf_face, m->cf_other,
                                              m->cf_pad);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // host staging vectors go out of scope
    if (e != cudaSuccess) {
        fv_mesh_destroy(m);
        return fail(e, "fv_mesh_concat");
    }
    *out = m;
    return FV_OK;
}

extern "C" fv_status fv_mesh_concat(const fv_mesh *const *parts, int32_t n_parts, void *stream, fv_mesh **out) {
    return fv_host_guard([&] { return mesh_concat_impl(parts, n_parts, stream, out); });
}
