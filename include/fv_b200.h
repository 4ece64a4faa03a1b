/*
 * fv_b200.h -- C ABI of the B200 assembly + sparse Krylov path.
 *
 * This library replaces, behind a plain C boundary, the hot path of the
 * finite-volumes crate (x318aVkl/finite-volumes-rs):
 *
 *   fvm::assembly::assemble                      src/fvm/assembly.rs:11-78
 *   DistributedMatrix::imul (CSR SpMV)           src/linalg/dmatrix.rs:136-146
 *   IncompleteCholesky::from_matrix (IC(0))      src/linalg/preconditioners/incomplete_cholesky.rs:205
 *   IncompleteLowerUpper::from_matrix (ILU(0))   src/linalg/preconditioners/incomplete_lower_upper.rs:266
 *   Preconditioner::precondition                 src/linalg/preconditioners/mod.rs:13-17
 *   solvers::conjugate_gradient                  src/linalg/solvers/conjugate_gradient.rs:12-111
 *   solvers::bi_conjugate_gradient_stab          src/linalg/solvers/bi_conjugate_gradient_stab.rs:13-178
 *
 * Conventions
 *   - Every call returns an fv_status; nothing aborts the process.  Invariant
 *     violations that the reference turns into a panic (missing matrix entry,
 *     ILU pivot below 1e-16, IC on a non-symmetric matrix) are returned as
 *     FV_ERR_INVALID / FV_ERR_SINGULAR_PIVOT / FV_ERR_NOT_SYMMETRIC.
 *   - Non-convergence is not an error (as in the reference): check
 *     fv_solver_info.iterations / final_residual.
 *   - Handles are opaque, single-stream and not thread-safe (the reference is
 *     single-threaded per MPI rank).  `stream` is a cudaStream_t passed as
 *     void*; 0 means the legacy default stream.
 *   - Device pointers are used for vectors unless the function name ends in
 *     _host, in which case host memory is read/written and the copies happen
 *     inside the call.
 *   - Scalars are FP64 and indices int32, cells/faces numbered as in the
 *     reference's Mesh.  Arithmetic follows the reference's operation order
 *     without fused multiply-add, so assembly, SpMV, factorisation and the
 *     triangular sweeps reproduce the reference bit for bit; only reductions
 *     (dot products) are summed in a different (fixed, deterministic) order.
 */
#ifndef FV_B200_H
#define FV_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  Mirrors the panics / Result of the reference (core/error.rs:4-21). */
typedef enum fv_status {
    FV_OK = 0,
    FV_ERR_ALLOC = 1,          /* device or host allocation failed */
    FV_ERR_INVALID = 2,        /* bad argument, corrupted CSR, missing matrix entry */
    FV_ERR_SINGULAR_PIVOT = 3, /* ILU |u_kk| < 1e-16 (incomplete_lower_upper.rs:234-235) */
    FV_ERR_BREAKDOWN = 4,      /* Krylov breakdown: NaN/Inf scalar detected on the device */
    FV_ERR_TIMEOUT = 5,        /* a bounded device-side wait gave up */
    FV_ERR_NOT_SYMMETRIC = 6,  /* IC on a matrix failing |a_ij-a_ji|<1e-14 (incomplete_cholesky.rs:153) */
    FV_ERR_CUDA = 7,           /* a CUDA runtime call failed */
    FV_ERR_UNSUPPORTED = 8,    /* feature outside the implemented scope (e.g. level>0) */
    FV_ERR_COMM = 9            /* a communicator callback (fv_comm) reported failure */
} fv_status;

/* ------------------------------------------------------------------------ */
/* Host-side mesh (the stand-in for the reference's Mesh<DIM> after
 * Mesh::compute).  Produced by the generators below or built from an element
 * list; numbering and geometry follow core/mesh/io.rs:364-486
 * (compute_vtk_faces), core/mesh/mod.rs:451-529 (add_face/add_cell) and
 * core/mesh/compute.rs:12-375 (face/cell geometry, orientation).            */
typedef struct fv_host_mesh {
    int32_t dim;              /* 2 or 3 */
    int64_t n_nodes;
    int64_t n_faces;          /* interior faces first, boundary faces last */
    int64_t n_cells;
    int64_t n_boundary_faces; /* boundary faces are [n_faces-n_boundary_faces, n_faces) */
    double  *nodes;           /* n_nodes*dim */
    int32_t *face_node_ptr;   /* n_faces+1 */
    int32_t *face_nodes;
    int32_t *face_patch;      /* n_faces; -1 for interior faces, else marker id */
    int32_t *cell_face_ptr;   /* n_cells+1 */
    int32_t *cell_faces;      /* faces of each cell in element-local order */
    int32_t *face_owner;      /* n_faces */
    int32_t *face_neighbor;   /* n_faces; -1 for boundary faces */
    double  *face_area;       /* n_faces */
    double  *face_normal;     /* n_faces*dim (3D: |n| = 1/3 for triangles, as the reference) */
    double  *face_center;     /* n_faces*dim */
    double  *cell_center;     /* n_cells*dim */
    double  *cell_volume;     /* n_cells */
} fv_host_mesh;

/* Build from an element list, as Mesh::read_su2 does (io.rs:489-533).
 * elem_kind uses VTK ids: 5 triangle, 9 quad, 10 tetrahedron, 12 hexahedron.
 * Boundary faces are given as node lists with a marker id (SU2 MARKER_ELEMS). */
/* Mesh::read_su2 (io.rs:228-533): an SU2 file (NDIME, NPOIN, NELEM, MARKER_TAG
 * / MARKER_ELEMS) into the same host mesh as fv_host_mesh_from_elements.
 * dim 0 takes NDIME from the file. */
fv_status fv_host_mesh_read_su2(const char *path, int32_t dim, fv_host_mesh **out);
fv_status fv_host_mesh_from_elements(int32_t dim, int64_t n_nodes, const double *nodes,
                                     int64_t n_elems, const int32_t *elem_kind,
                                     const int32_t *elem_node_ptr, const int32_t *elem_nodes,
                                     int64_t n_bfaces, const int32_t *bface_node_ptr,
                                     const int32_t *bface_nodes, const int32_t *bface_marker,
                                     fv_host_mesh **out);

/* Unit square, n x n squares each split into 2 triangles along the (i,j)-(i+1,j+1)
 * diagonal, interior nodes jittered by U(-jitter*h, jitter*h) per coordinate. */
fv_status fv_host_mesh_generate_square(int32_t n, double jitter, uint64_t seed, fv_host_mesh **out);

/* Unit cube, n^3 hexes each split into 6 Kuhn tetrahedra (same orientation in
 * every hex), interior nodes jittered by U(-jitter*h, jitter*h). */
fv_status fv_host_mesh_generate_cube(int32_t n, double jitter, uint64_t seed, fv_host_mesh **out);

void fv_host_mesh_free(fv_host_mesh *m);

/* add_face / add_cell + Mesh::compute on the host for explicit faces and cells
 * (see fv_mesh_build_faces). */
fv_status fv_host_mesh_from_faces(int32_t dim, int64_t n_nodes, const double *nodes, int64_t n_faces,
                                  const int32_t *face_node_ptr, const int32_t *face_nodes,
                                  const int32_t *face_patch, int64_t n_cells, const int32_t *cell_face_ptr,
                                  const int32_t *cell_faces, fv_host_mesh **out);
/* Mesh::read / Mesh::write (io.rs:10-225), the crate's own ".msh" format:
 *   NDIME=<dim>, NPATCH=<k> + "<name> <id> <first face> <faces>",
 *   NNODES=<n> + coordinates, NFACES=<n> + "<len> <nodes> <tag|-> <gid> -",
 *   NCELLS=<n> + "<len> <faces> <gid> -".
 * The writer prints doubles as Rust's Display does (shortest digits that read
 * back exactly, positional) and names patch p patch_names[p] (NULL or short:
 * "patch_<p>"). */
fv_status fv_host_mesh_read_msh(const char *path, int32_t dim, fv_host_mesh **out);
fv_status fv_host_mesh_write_msh(const fv_host_mesh *m, const char *path, const char *const *patch_names,
                                 int32_t n_patch_names);

/* Seeded synthetic fields on a host mesh.
 *   cell diffusivity kappa_c = kappa0 * exp(sigma * z), z ~ N(0,1)
 *   face diffusivity: linear interpolation weights of faceinterp/linear.rs:25-42
 *     (w clamped to [0,1]); boundary faces take the owner value
 *   flux_f = velocity . normal_f (reference normal)
 *   source_c = source_const if source_uniform==0, else U(0,1)
 * Any output pointer may be NULL. */
fv_status fv_host_fields_generate(const fv_host_mesh *m, uint64_t seed, double kappa0, double sigma,
                                  const double *velocity, double source_const, int32_t source_uniform,
                                  double *kappa_face, double *flux_face, double *source_cell);

/* ------------------------------------------------------------------------ */
/* Device objects                                                            */
typedef struct fv_mesh fv_mesh;       /* device-resident geometry + cell->face table */
typedef struct fv_csr fv_csr;         /* device CSR matrix, FP64 values, int32 indices */
typedef struct fv_precond fv_precond; /* IC(0) / ILU(0) factors + level schedules */

typedef struct fv_mesh_desc {
    int32_t dim;
    int64_t n_cells;
    int64_t n_faces;
    int64_t n_boundary_faces;     /* boundary faces are the tail of the face list */
    const int32_t *face_owner;    /* host pointers; copied by fv_mesh_upload */
    const int32_t *face_neighbor; /* -1 = boundary */
    const double  *face_area;
    const double  *face_center;   /* n_faces*dim */
    const double  *cell_center;   /* n_cells*dim */
    const double  *cell_volume;
    /* Optional, for the Corrected scheme and compute_gradients (NULL when not
     * needed): the face normals (n_faces*dim) and every cell's faces in the
     * mesh's own order (Mesh::cell_faces, cell_face_ptr[n_cells+1]), which is
     * the order the gradient coefficients are summed in (compute.rs:155-203). */
    const double  *face_normal;
    const int32_t *cell_face_ptr;
    const int32_t *cell_faces;
} fv_mesh_desc;

/* The term expression c_conv*convection(Upwind(F),F) + c_lap*laplacian(S,kappa)
 * + c_src*source(f) of fvm/terms (laplacian.rs:35-45, convection.rs:36-45,
 * source.rs:34-40, operations.rs:86-199).  Coefficients must be -1, 0 or +1
 * (the reference's term algebra has +, - and unary - only).  The face-normal
 * gradient scheme S is Orthogonal (orthogonal.rs:26-46) or Corrected
 * (corrected.rs:36-67: coefficient 1/(n.d) and the explicit non-orthogonal
 * correction kappa * grad_f.(n - d/(n.d)) * corrector_reduction on the rhs,
 * grad_f interpolated from the cell gradients). */
#define FV_SCHEME_ORTHOGONAL 0
#define FV_SCHEME_CORRECTED 1
typedef struct fv_terms_desc {
    double laplacian_coef;
    double convection_coef;
    double source_coef;
    const double *diffusivity; /* n_faces, device (fv_assemble) or host (_host) */
    const double *flux;        /* n_faces */
    const double *source;      /* n_cells */
    int32_t scheme;            /* FV_SCHEME_ORTHOGONAL or FV_SCHEME_CORRECTED */
    double corrector_reduction;/* Corrected: 0 = no correction ... 1 = full */
    const double *gradients;   /* Corrected: n_cells*dim cell gradients (fv_compute_gradients) */
    /* Transient and further terms, each with a coefficient -1, 0 or +1 in the
     * same expression:
     *   time(Euler(previous, dt)) (terms/time.rs:19-35, schemes/time/euler.rs):
     *     cell lhs (1/dt)*rho, cell rhs previous/dt*rho_prev;
     *   time(Backward(previous, previous_2, dt, dt_2)) (schemes/time/backward.rs):
     *     cell lhs (a_next/dt)*rho, rhs (previous*a_last*rho_prev
     *     - previous_2*a_last_2*rho_prev_2)/dt with the reference's a_* of dt/dt_2;
     *   linear_source(c) (terms/source.rs:61-79): cell lhs c;
     *   divergence(F) (terms/divergence.rs:22-43): face rhs -F.
     * Densities are optional (NULL: 1). */
    double time_coef;
    int32_t time_scheme;       /* FV_TIME_EULER or FV_TIME_BACKWARD */
    double dt, dt_2;
    const double *previous;    /* n_cells */
    const double *previous_2;  /* n_cells (Backward) */
    const double *density;     /* n_cells, optional */
    const double *density_previous;
    const double *density_previous_2;
    double linear_source_coef;
    const double *linear_source;   /* n_cells */
    double divergence_coef;
    const double *divergence_flux; /* n_faces */
} fv_terms_desc;
#define FV_TIME_EULER 1
#define FV_TIME_BACKWARD 2

/* Boundary closure value_b = bndi*value_i + bnde per boundary face
 * (assembly.rs:64-73, bcs/mod.rs:33).  Dirichlet g: (0,g); zero gradient: (1,0). */
typedef struct fv_bc_desc {
    const double *bndi; /* n_boundary_faces */
    const double *bnde; /* n_boundary_faces */
} fv_bc_desc;

/* LinearSolverOptions (solvers/mod.rs:22-35). */
typedef struct fv_solver_options {
    double relative_tolerance;
    double absolute_tolerance;
    int64_t max_iterations;
} fv_solver_options;

/* LinearSolverInfo (solvers/mod.rs:11-17) plus device-side status. */
typedef struct fv_solver_info {
    int64_t iterations;
    double initial_residual;
    double final_residual;
    int32_t status;        /* fv_status of the solve (BREAKDOWN, TIMEOUT, ...) */
    int32_t restarts;      /* BiCGStab restarts (bi_conjugate_gradient_stab.rs:155-169) */
    double *history;       /* optional caller buffer for the per-iteration residual */
    int64_t history_cap;   /* capacity of history (0 = do not record) */
    int64_t history_len;   /* entries written */
    double device_ms;      /* device time of the solve, CUDA events */
} fv_solver_info;

fv_status fv_mesh_upload(const fv_mesh_desc *desc, void *stream, fv_mesh **out);
fv_status fv_mesh_destroy(fv_mesh *m);

/* Mesh::read_su2's face numbering (io.rs:364-533, mod.rs:451-529) and
 * Mesh::compute (compute.rs:12-375) on the device: from the element list of
 * fv_host_mesh_from_elements (host pointers) to a resident fv_mesh, gradient
 * coefficients included, with no host pass over faces or cells.  The arrays
 * equal fv_host_mesh_from_elements' bit for bit; host_out (optional, NULL to
 * skip) receives them as an fv_host_mesh (free with fv_host_mesh_free).
 * Replaces the caller-side Mesh::read_su2 + Mesh::compute before assemble. */
fv_status fv_mesh_build_elements(int32_t dim, int64_t n_nodes, const double *nodes,
                                 int64_t n_elems, const int32_t *elem_kind,
                                 const int32_t *elem_node_ptr, const int32_t *elem_nodes,
                                 int64_t n_bfaces, const int32_t *bface_node_ptr,
                                 const int32_t *bface_nodes, const int32_t *bface_marker,
                                 void *stream, fv_mesh **out, fv_host_mesh **host_out);
/* Mesh::compute on the device for explicit faces and cells (add_face /
 * add_cell, mod.rs:451-529: the first cell listing a face owns it, the second
 * is its neighbour unless the face is tagged).  face_patch: tag per face, -1
 * untagged; tagged faces must be the tail of the face list.  Same outputs as
 * fv_host_mesh_from_faces. */
fv_status fv_mesh_build_faces(int32_t dim, int64_t n_nodes, const double *nodes, int64_t n_faces,
                              const int32_t *face_node_ptr, const int32_t *face_nodes,
                              const int32_t *face_patch, int64_t n_cells, const int32_t *cell_face_ptr,
                              const int32_t *cell_faces, void *stream, fv_mesh **out,
                              fv_host_mesh **host_out);
/* The crate's own mesh file (Mesh::read, io.rs:68-225; ".msh"): on the device,
 * or on the host (fv_host_mesh_read_msh).  dim 0 takes NDIME from the file.
 * Remote (ghost) faces or cells of a decomposed mesh: FV_ERR_UNSUPPORTED. */
fv_status fv_mesh_build_msh(const char *path, int32_t dim, void *stream, fv_mesh **out,
                            fv_host_mesh **host_out);
/* One resident mesh from n_parts resident meshes, laid out as a batch of
 * independent problems (batched and served solves): the interior faces of every part in part order,
 * then the boundary faces of every part; cells in part order.  Equal to
 * fv_mesh_upload of the same union built on the host, without its host
 * pass; no gradient data.  The parts stay owned by the caller. */
fv_status fv_mesh_concat(const fv_mesh *const *parts, int32_t n_parts, void *stream, fv_mesh **out);
/* The same from an SU2 file (the parser of fv_host_mesh_read_su2) and from the
 * synthetic generators (fv_host_mesh_generate_square / _cube). */
fv_status fv_mesh_build_su2(const char *path, int32_t dim, void *stream, fv_mesh **out,
                            fv_host_mesh **host_out);
fv_status fv_mesh_build_square(int32_t n, double jitter, uint64_t seed, void *stream, fv_mesh **out,
                               fv_host_mesh **host_out);
fv_status fv_mesh_build_cube(int32_t n, double jitter, uint64_t seed, void *stream, fv_mesh **out,
                             fv_host_mesh **host_out);

/* compute_gradients (fvm/tools/gradients.rs:48-86): least-squares cell
 * gradients of a cell field, grad[c] = values[c] * own_c + sum over the
 * cell's faces (mesh order) of value_other * g_k, a boundary face taking
 * bndi*values[c] + bnde.  The coefficients own_c and g_k are those of
 * Mesh::compute (compute.rs:155-203), computed at upload; the mesh must have
 * been uploaded with cell_face_ptr / cell_faces (else FV_ERR_UNSUPPORTED).
 * values: n_cells, grad: n_cells*dim (device). */
fv_status fv_compute_gradients(fv_mesh *m, const double *values, const fv_bc_desc *bc, double *grad,
                               void *stream);

/* assemble(): builds the CSR pattern of cell_to_cell (dmatrix.rs:38-50) on the
 * first call (*A == NULL) and refills values into the existing pattern when
 * *A is a matrix returned by an earlier call on the same mesh.
 * terms/bc pointers are device pointers; b is a device vector of n_cells. */
fv_status fv_assemble(fv_mesh *m, const fv_terms_desc *terms, const fv_bc_desc *bc,
                      fv_csr **A, double *b, void *stream);
fv_status fv_assemble_host(fv_mesh *m, const fv_terms_desc *terms, const fv_bc_desc *bc,
                           fv_csr **A, double *b_host, void *stream);

/* Generic CSR from host arrays (sorted columns per row required). */
fv_status fv_csr_create_host(int64_t nrows, int64_t ncols, const int32_t *row_ptr,
                             const int32_t *cols, const double *vals, void *stream, fv_csr **out);
fv_status fv_csr_info(const fv_csr *A, int64_t *nrows, int64_t *ncols, int64_t *nnz);
fv_status fv_csr_download(const fv_csr *A, int32_t *row_ptr, int32_t *cols, double *vals, void *stream);
fv_status fv_csr_destroy(fv_csr *A);

/* y = A x (DistributedMatrix::imul, dmatrix.rs:136-146); bit-exact per row. */
fv_status fv_spmv(const fv_csr *A, const double *x, double *y, void *stream);
fv_status fv_spmv_host(const fv_csr *A, const double *x_host, double *y_host, void *stream);

/* DistributedVector operations (linalg/dvector.rs:46-160) on device vectors.
 * fv_vec_dot: dot / dot_smaller (the caller passes the shorter length);
 * fv_vec_sum: sum.  Both write the result to host *out after their stream
 * finished; the sum order is fixed by n (strided per thread, a fixed tree,
 * block partials in order), not the reference's serial order: results agree
 * to rounding.  fv_vec_update, elementwise and exact: op 0 y += x, 1 y -= x,
 * 2 y *= a, 3 y = 1/y (inv), 4 y = x (set / set_smaller with the shorter n). */
fv_status fv_vec_dot(int64_t n, const double *x, const double *y, void *stream, double *out);
fv_status fv_vec_sum(int64_t n, const double *x, void *stream, double *out);
fv_status fv_vec_update(int64_t n, double *y, const double *x, double a, int32_t op, void *stream);

/* IncompleteCholesky::from_matrix(A, 0) / IncompleteLowerUpper::from_matrix(A, 0). */
fv_status fv_ic0_factor(const fv_csr *A, void *stream, fv_precond **out);
fv_status fv_ilu0_factor(const fv_csr *A, void *stream, fv_precond **out);
/* DiagonalPreconditioner::from_matrix(A) (preconditioners/mod.rs:38-68):
 * z_i = (1 / a_ii) r_i.  A row without its diagonal: FV_ERR_INVALID (the
 * reference panics).  Usable wherever an fv_precond is taken (solvers,
 * batched and distributed solves, fv_precond_apply / _refactor / _export);
 * fv_precond_levels answers FV_ERR_UNSUPPORTED (no sweeps). */
fv_status fv_diag_factor(const fv_csr *A, void *stream, fv_precond **out);
/* IncompleteCholesky / IncompleteLowerUpper ::from_matrix(A, level) for any
 * level (incomplete_cholesky.rs:35-85,148-205; incomplete_lower_upper.rs:
 * 30-137,200-266): the reference's level-k patterns (depth-first walks over
 * the matrix graph, restated in their visiting order), then the level-0
 * numerics on that pattern with zeros at fill positions.  IC(1) has the
 * pattern of A (the reference's walk adds no node for level 1). */
fv_status fv_ic_factor(const fv_csr *A, int32_t level, void *stream, fv_precond **out);
fv_status fv_ilu_factor(const fv_csr *A, int32_t level, void *stream, fv_precond **out);
/* Value-only refactorisation of P after the values of the matrix it was built
 * from changed (same pattern, same fv_csr object); reuses the symbolic
 * analysis (triangular split, level schedules) and the factor storage. */
fv_status fv_precond_refactor(fv_precond *P, void *stream);
/* z = M^-1 r (Preconditioner::precondition).  r and z must not alias. */
fv_status fv_precond_apply(fv_precond *P, const double *r, double *z, void *stream);
fv_status fv_precond_apply_host(fv_precond *P, const double *r_host, double *z_host, void *stream);
/* Export of the stored factors (ILU: dropped entries removed).  Pass NULL
 * arrays to query sizes (nnz_lower, nnz_upper).  IC: lower = L incl. diagonal
 * as the reference's `l`; ILU: lower = strict L, upper = U incl. diagonal,
 * merged per row exactly as the reference's single `lu` CSR when merged=1. */
fv_status fv_precond_export(const fv_precond *P, int64_t *nnz, int32_t *row_ptr, int32_t *cols,
                            double *vals, int32_t *n_dropped, void *stream);
/* Level schedules: level of every row in the forward (lower) and backward (upper) DAG. */
fv_status fv_precond_levels(const fv_precond *P, int32_t *fwd_level, int32_t *bwd_level,
                            int32_t *n_fwd_levels, int32_t *n_bwd_levels, void *stream);
/* Sweep schedule of P.  request: -1 query only; 0 or 1 level chunks (the
 * default for rows not sorted by level); 2 box tiles, available when the
 * matrix was assembled on a mesh whose box order exists (FV_ERR_UNSUPPORTED
 * otherwise); 3 level chunks with each warp loading its next chunk's rows
 * before waiting on the current one; 4 consecutive rows in index order, block
 * tickets (the default when the factorised matrix's rows are already sorted
 * by forward level, e.g. a matrix permuted by fv_order_boxes' order; any
 * level-0 factorisation accepts it, FV_ERR_UNSUPPORTED for reordered or fill
 * factorisations).  *active receives 1, 2, 3 or 4.  stats (optional, 6 doubles): box edge
 * in mean cell sizes, number of boxes, lane use of the forward / backward
 * steps, share of dependencies read from shared memory forward / backward
 * (zeros without a tiling).  Both schedules give the same bits. */
fv_status fv_precond_schedule(fv_precond *P, int32_t request, int32_t *active, double *stats);
/* Sweep launch shape: blocks of 256 threads per sweep launch (1..4736; 0 =
 * the default: 2 per SM for natural-order sweeps, up to 8 per SM for the
 * reordered ones) and rows per thread of the reordered sweeps (1, 2, 4 or 8;
 * 0 = 1).  A tuning knob: every shape gives the same results. */
fv_status fv_precond_set_grid(fv_precond *P, int32_t blocks, int32_t rows_per_thread);
fv_status fv_precond_destroy(fv_precond *P);
/* The box-tile plan fv_ic0_factor / fv_ilu0_factor make for a matrix
 * assembled on a mesh, computed from host arrays (cell: n x 4 doubles, the
 * centre in the first dim entries): direction 0 = forward over the strict
 * lower part, 1 = backward over the strict upper part.  sizes receives
 * (boxes, steps, swept-side entries); pass NULL arrays to query sizes.
 * box_step: boxes+1 entries; sptr: steps+1; trow: n; dsrc: swept-side
 * entries in row order (column j, or -(ring slot + 1)); stats (4 doubles):
 * box edge in mean cell sizes, lane use, share of ring reads, estimated
 * critical path of both sweeps relative to the level schedule.  FV_ERR_UNSUPPORTED when
 * no box order exists (the sweeps then use level chunks). */
fv_status fv_tile_plan_host(int64_t n, int32_t dim, const double *cell, const int32_t *row_ptr,
                            const int32_t *cols, int32_t direction, int64_t *sizes, int32_t *box_step,
                            int32_t *sptr, int32_t *trow, int32_t *dsrc, double *stats);
/* The level-k factor pattern fv_ic_factor (kind 1) / fv_ilu_factor (kind 2)
 * build, computed from a host CSR pattern (n rows, sorted columns): the
 * depth-first walks of IncompleteCholesky's row_i_sparsity_edit
 * (incomplete_cholesky.rs:35-85) and IncompleteLowerUpper's row_i_l_sparsity /
 * row_i_u_sparsity (incomplete_lower_upper.rs:30-137), rows sorted.  Call
 * with fcol == NULL to receive *nnz only; then fptr (n + 1), fcol (*nnz) and,
 * optionally, amap (row_ptr[n]: position of every entry of A in the pattern)
 * and fill (*nnz, kind 1 only: 1 for entries that are not entries of A). */
fv_status fv_fill_pattern_host(int32_t kind, int32_t level, int64_t n, const int32_t *row_ptr, const int32_t *cols,
                               int64_t *nnz, int32_t *fptr, int32_t *fcol, int32_t *amap, uint8_t *fill);

/* conjugate_gradient / bi_conjugate_gradient_stab.  x is the initial guess on
 * input and the solution on output (device vectors).  P may be NULL (identity). */
fv_status fv_cg(const fv_csr *A, fv_precond *P, const double *b, double *x,
                fv_solver_options opt, fv_solver_info *info, void *stream);
fv_status fv_bicgstab(const fv_csr *A, fv_precond *P, const double *b, double *x,
                      fv_solver_options opt, fv_solver_info *info, void *stream);
fv_status fv_cg_host(const fv_csr *A, fv_precond *P, const double *b_host, double *x_host,
                     fv_solver_options opt, fv_solver_info *info, void *stream);
fv_status fv_bicgstab_host(const fv_csr *A, fv_precond *P, const double *b_host, double *x_host,
                           fv_solver_options opt, fv_solver_info *info, void *stream);

/* ------------------------------------------------------------------------ */
/* Batched solves (no single counterpart in the reference: every problem is
 * solved as conjugate_gradient.rs:12-111 would solve it alone).  A is the
 * block-diagonal union of independent problems (e.g. assembled on a mesh made
 * by concatenating meshes); row_offsets[p]..row_offsets[p+1] are problem p's
 * rows.  Per-problem reductions never mix problems, so each result is the same
 * whether the problem is solved alone or in any batch. */
typedef struct fv_batch fv_batch;

#define FV_BATCH_FP64 0  /* Krylov in FP64, reference semantics per problem */
#define FV_BATCH_MIXED 1 /* FP32 Krylov + FP32 factors with FP64 reliable updates: whenever the
                            FP32 residual estimate fell by inner_relative_tolerance (or reached the
                            target), x64 += d32 and the residual is recomputed as b - A x64 in FP64
                            and replaces the FP32 one; the solve stops when that FP64 residual
                            |b - A x| / |b| <= outer_tolerance. */

typedef struct fv_batch_options {
    int32_t precision;               /* FV_BATCH_FP64 or FV_BATCH_MIXED */
    double relative_tolerance;       /* FP64 mode: the CG rtol / atol of LinearSolverOptions */
    double absolute_tolerance;
    int64_t max_iterations;          /* per inner solve */
    double inner_relative_tolerance; /* mixed: residual reduction that triggers a replacement (e.g. 1e-2) */
    double outer_tolerance;          /* mixed: stop when |b - A x| / |b| <= this (FP64) */
    int32_t max_outer;               /* unused (kept for ABI stability) */
} fv_batch_options;

typedef struct fv_batch_info {
    double device_ms;
    int64_t launched_iterations;     /* CG iterations enqueued for the whole batch */
    int64_t *iterations;             /* per problem (optional): Krylov iterations */
    int32_t *outer_steps;            /* per problem (optional): FP64 residual replacements (mixed) */
    double *final_residual;          /* per problem (optional): FP64 mode |r|/|b| as LinearSolverInfo;
                                        mixed: the true FP64 |b - A x| / |b| */
    int32_t *status;                 /* per problem (optional) */
    int32_t *fp64_fallback;          /* per problem (optional, mixed): 1 when the FP32 run stagnated
                                        (no FP64 progress over two replacements; kappa * eps32 >> 1) and
                                        an FP64 batched pass over the stagnated problems finished it */
} fv_batch_info;

fv_status fv_batch_create(const fv_csr *A, int32_t n_problems, const int64_t *row_offsets, int32_t tile_rows,
                          void *stream, fv_batch **out);
/* x0 = 0 for every problem; P is the IC(0) (CG) or ILU(0) (BiCGStab) of A. */
fv_status fv_batch_cg(fv_batch *B, fv_precond *P, const double *b, double *x, const fv_batch_options *opt,
                      fv_batch_info *info, void *stream);
fv_status fv_batch_bicgstab(fv_batch *B, fv_precond *P, const double *b, double *x, const fv_batch_options *opt,
                            fv_batch_info *info, void *stream);
fv_status fv_batch_destroy(fv_batch *B);

/* Stepwise runs (continuous batching): the iterations of fv_batch_cg /
 * fv_batch_bicgstab, split at iteration boundaries so a caller can take the
 * finished problems out and carry the running ones into another batch (built
 * over the running problems plus newly admitted ones) without changing any
 * bit of their iterations.
 *
 * fv_batch_begin starts a run of `method` (FV_BATCH_CG / FV_BATCH_BICGSTAB).
 * Problem p starts from x0 = 0 unless from_problem (optional, np entries) maps
 * it to a running problem from_problem[p] >= 0 of the batch `from`: that
 * problem's state (the rows of x and of the Krylov vectors, its iteration
 * count and scalars) is copied and it continues where it stopped.  Its matrix,
 * right-hand side and preconditioner rows must be the same bits in both
 * batches (the same request assembled again), and both runs must use the same
 * method, precision, mixed-precision settings and tile_rows; otherwise, or
 * when a mapped problem is not running or has another size, FV_ERR_INVALID.
 * `from` (and its b, x) must stay alive until fv_batch_begin returns; it does
 * not change.  b, x and P must stay alive for the whole run.
 *
 * fv_batch_advance runs up to max_iterations more iterations (whole groups of
 * 8 CG / 4 BiCGStab iterations; fewer when every problem finished), applies
 * the pending result of every problem that finished (x final in its rows) and
 * returns the number of running problems and per problem done[p] (optional).
 * fv_batch_report fills the per-problem fields of info for the state after the
 * last begin / advance (device_ms = 0).  A stepwise mixed run does not run the
 * FP64 pass: fp64_fallback[p] = 1 marks a problem whose FP32 run stagnated
 * (done, unconverged); its caller solves it again in FP64.
 * A problem gives the same bits through any sequence of stepwise batches as
 * alone in fv_batch_cg / fv_batch_bicgstab (mixed: when it does not stagnate). */
#define FV_BATCH_CG 0
#define FV_BATCH_BICGSTAB 1
fv_status fv_batch_begin(fv_batch *B, fv_precond *P, int32_t method, const double *b, double *x,
                         const fv_batch_options *opt, const fv_batch *from, const int32_t *from_problem,
                         void *stream);
fv_status fv_batch_advance(fv_batch *B, int64_t max_iterations, int32_t *n_running, int32_t *done, void *stream);
fv_status fv_batch_report(const fv_batch *B, fv_batch_info *info);

/* ------------------------------------------------------------------------ */
/* Reordered factorisations (the perf mode of the triangular sweeps).
 *
 * No counterpart in the reference, which factorises in the natural row order
 * (incomplete_lower_upper.rs:200-261, incomplete_cholesky.rs:87-145, applied
 * by the sweeps of incomplete_lower_upper.rs:287-329 and
 * incomplete_cholesky.rs:217-255).  In that order a 3D mesh's sweeps have a
 * level count proportional to the mesh's extent, and every level is a
 * dependency handoff between SMs.  These calls factorise B = Q A Q^T instead,
 * for a permutation Q of the caller's choice (perm[i] = the row of A that
 * becomes row i of B; host memory), and apply it in A's numbering:
 * z = Q^T M_B^{-1} Q r.  The factors are the reference's algorithm run on B
 * (bit for bit: fv_precond_export returns B's factors), so the preconditioner
 * is a different one from A's natural-order factorisation and the Krylov
 * iteration counts differ.  fv_precond_refactor moves A's new values into B
 * (same pattern).  Errors: FV_ERR_INVALID when perm is not a permutation of
 * 0..n-1, else as fv_ic0_factor / fv_ilu0_factor. */
fv_status fv_ic0_factor_perm(const fv_csr *A, const int32_t *perm, void *stream, fv_precond **out);
fv_status fv_ilu0_factor_perm(const fv_csr *A, const int32_t *perm, void *stream, fv_precond **out);
/* The permutation of a reordered preconditioner (n entries; FV_ERR_INVALID otherwise). */
fv_status fv_precond_perm(const fv_precond *P, int32_t *perm, void *stream);

/* Box-colour ordering for fv_*_factor_perm.  The cells are grouped into
 * boxes of their centres (about rows_per_box rows each, a grid over the
 * domain box lo..hi shaped like the domain), the boxes coloured greedily so
 * that no two coupled boxes share a colour, and the rows numbered colour by
 * colour, box by box, in natural order inside a box; the rows are then sorted
 * (stably) by their level in that ordering's forward dependency graph, which
 * keeps the graph and makes every level a contiguous range of rows.  The
 * sweeps then have about (colours) x (levels inside a box) levels, each
 * spanning all boxes of a colour.  On meshes whose boxes align with the
 * element grid two colours suffice.  O(n + nnz) on the host. */
typedef struct fv_order_info {
    int64_t n_boxes;            /* occupied boxes */
    int32_t boxes_per_axis[3];  /* grid (1 on unused axes; the first problem's for a batch) */
    int32_t n_colours;
    int32_t n_levels;           /* levels of the forward sweep in the new order */
} fv_order_info;
/* cell_center: n points of `dim` coordinates, point i at cell_center + i * center_stride;
 * lo / hi: the domain box (NULL: the centres' bounding box); row_ptr / cols: the
 * CSR pattern of A (host).  perm (out): n entries.  rows_per_box <= 0 takes the
 * default: 32 rows in 2D, 384 in 3D (4 x 4 squares of 2 triangles, 4^3 hexes of
 * 6 tetrahedra). */
fv_status fv_order_boxes_host(int64_t n, int32_t dim, const double *cell_center, int64_t center_stride,
                              const double *lo, const double *hi, const int32_t *row_ptr, const int32_t *cols,
                              int32_t rows_per_box, int32_t *perm, fv_order_info *info);
/* A block-diagonal union of independent problems (problem p = rows
 * offsets[p]..offsets[p+1]-1, coupled to nothing else): each problem ordered
 * as above within its own domain box (lo / hi: dim values per problem, or
 * NULL), then all rows sorted stably by (level, problem): the union has the
 * largest problem's level count. */
fv_status fv_order_boxes_batch_host(int32_t n_problems, const int64_t *offsets, int32_t dim,
                                    const double *cell_center, int64_t center_stride, const double *lo,
                                    const double *hi, const int32_t *row_ptr, const int32_t *cols,
                                    int32_t rows_per_box, int32_t *perm, fv_order_info *info);
/* The same for a matrix assembled on a device mesh: centres from the mesh, the
 * domain box(es) from its boundary faces (FV_ERR_INVALID for a matrix without
 * mesh).  n_problems <= 1: one problem; else offsets as above. */
fv_status fv_order_boxes(const fv_csr *A, int32_t n_problems, const int64_t *offsets, int32_t rows_per_box,
                         int32_t *perm, fv_order_info *info, void *stream);
/* One problem's ordering plus level[i], the level of row i of the reordered
 * matrix (non-decreasing in i): a caller that keeps each mesh's order can
 * merge several meshes' orders into the order fv_order_boxes gives their
 * union -- for each level, every problem's rows of that level in problem
 * order, offset by the problem's first row. */
fv_status fv_order_boxes_host_levels(int64_t n, int32_t dim, const double *cell_center, int64_t center_stride,
                                     const double *lo, const double *hi, const int32_t *row_ptr,
                                     const int32_t *cols, int32_t rows_per_box, int32_t *perm, int32_t *level,
                                     fv_order_info *info);
fv_status fv_order_boxes_levels(const fv_csr *A, int32_t rows_per_box, int32_t *perm, int32_t *level,
                                fv_order_info *info, void *stream);

/* A permuted copy B = Q A Q^T of a square matrix: B's row i is A's row
 * perm[i] (host array of n entries, a permutation; FV_ERR_INVALID otherwise;
 * rows of more than 32 entries: FV_ERR_UNSUPPORTED), columns renumbered the
 * same way and sorted.  With perm from fv_order_boxes,
 * B's rows are sorted by level and its IC(0)/ILU(0) (fv_ic0_factor /
 * fv_ilu0_factor on B) sweeps consecutive rows (schedule 4) with no gather or
 * scatter: solving B y = Q b and x = Q^T y is the reordered perf mode without
 * the permutation inside every preconditioner apply.  No counterpart in the
 * reference.  B keeps a pointer to A (A must outlive B);
 * fv_csr_permute_values copies A's current values into B (after A is
 * re-assembled), fv_vec_permute maps vectors: back = 0: y[i] = x[perm[i]];
 * back = 1: y[perm[i]] = x[i] (x and y distinct device vectors of n). */
fv_status fv_csr_permute(const fv_csr *A, const int32_t *perm, void *stream, fv_csr **B);
fv_status fv_csr_permute_values(fv_csr *B, void *stream);
fv_status fv_vec_permute(const fv_csr *B, const double *x, double *y, int32_t back, void *stream);

/* Allocation-free conjugate gradient.  No counterpart in the reference crate.
 *
 * Same contract and same results as fv_cg, for callers that must not allocate
 * device memory inside the solve: fv_cg obtains its Krylov workspace with
 * cudaMallocAsync on every call, which an application cannot allow when
 * another runtime owns the device memory budget (all memory reserved up front,
 * a fixed-size pool, a memory-capped process) or when the solve runs in a
 * phase where allocation is forbidden.  This entry point takes the workspace
 * from a statically sized device array instead and calls no cudaMalloc,
 * cudaMallocAsync, cudaFree or allocating library routine.
 *
 * Limits: at most FV_NOALLOC_MAX_ROWS rows and FV_NOALLOC_MAX_ITERATIONS
 * iterations; larger requests return FV_ERR_INVALID (fv_last_error() names
 * the limit).  The array (about 8.6 MB) belongs to the solvers' CUDA module
 * and is held until the process exits on every GPU where that module is
 * loaded.  Under lazy module loading (the CUDA 12 default,
 * CUDA_MODULE_LOADING=LAZY) the module, and with it the array, is created on
 * a device at the first solver call there (fv_cg, fv_bicgstab or this one),
 * so that first call does take device memory: make one call on each device
 * before the phase in which nothing may be allocated (with
 * CUDA_MODULE_LOADING=EAGER the array is created when the library's kernels
 * are loaded).
 * The first call on each device looks up the array's device address with
 * cudaGetSymbolAddress (that device must be current); make that first call
 * before any stream capture.  The address is looked up again when the
 * device's context has been replaced (cudaDeviceReset), so a reset never
 * leaves a stale address behind; every handle made before the reset (A, P)
 * is invalid after it, as for the rest of this library.  All calls share the one array: calls that
 * overlap on the GPU (other streams, other host threads) race and must be
 * serialised by the caller.  info->device_ms is left at 0.  A and P are
 * created beforehand by the allocating calls (fv_assemble / fv_csr_create_host,
 * fv_ic0_factor). */
#define FV_NOALLOC_MAX_ROWS 262144
#define FV_NOALLOC_MAX_ITERATIONS 4093
fv_status fv_cg_noalloc(const fv_csr *A, fv_precond *P, const double *b, double *x,
                        fv_solver_options opt, fv_solver_info *info, void *stream);

/* ------------------------------------------------------------------------ */
/* One rank of a problem split over several GPUs (the reference's MPI design,
 * core/communicator.rs, core/mesh/decompose.rs).  The rank's matrix A has
 * n_own rows (its cells) and n_own + n_ghost columns: its own cells first,
 * then the ghost cells owned by other ranks (dmatrix.rs:38-50 over the local
 * cell_to_cell).  The two communication steps are supplied by the caller. */
typedef struct fv_comm {
    void *ctx;
    /* Communicator::collect (core/communicator.rs:226-266): send[0..n_send)
     * holds this rank's values that other ranks need, packed in the order of
     * the send_idx given to fv_dist_create; fill ghost[0..n_ghost) with the
     * ghost values in ghost-column order.  Device pointers; order the transfer
     * on `stream` (or finish it before returning).  Return 0 on success.
     * NULL means a single rank with no ghosts. */
    int (*collect)(void *ctx, const double *send, double *ghost, void *stream);
    /* Communicator::reduce_add (core/communicator.rs:282-290): replace
     * buf[0..count) (device) by its sum over all ranks, ordered on `stream`.
     * Return 0 on success.  NULL means a single rank. */
    int (*reduce_add)(void *ctx, double *buf, int count, void *stream);
} fv_comm;

typedef struct fv_dist fv_dist;

/* DistributedMatrix::square_block (dmatrix.rs:214-229): the rows of A with
 * the columns >= nrows (ghost columns) dropped. */
fv_status fv_csr_square_block(const fv_csr *A, void *stream, fv_csr **out);
/* A: this rank's matrix (n_own rows, n_own + n_ghost columns; kept, not
 * copied).  send_idx (host, n_send entries): the owned rows whose values the
 * other ranks need, in the order collect() expects them.  comm is copied. */
fv_status fv_dist_create(const fv_csr *A, int64_t n_ghost, const int32_t *send_idx, int64_t n_send,
                         const fv_comm *comm, fv_dist **out);
fv_status fv_dist_destroy(fv_dist *D);
/* y[0..n_own) = A x after collect() refreshed x[n_own .. n_own + n_ghost). */
fv_status fv_dist_spmv(fv_dist *D, double *x, double *y, void *stream);
/* Global dot product (local sum + reduce_add), returned on the host. */
fv_status fv_dist_dot(fv_dist *D, const double *x, const double *y, double *result, void *stream);
/* conjugate_gradient / bi_conjugate_gradient_stab on every rank together
 * (each rank calls with its own D, P, b and x; all ranks take the same number
 * of iterations).  P: this rank's preconditioner built on fv_csr_square_block(A)
 * (block Jacobi across ranks), or NULL.  b, x: n_own entries (device). */
fv_status fv_dist_cg(fv_dist *D, fv_precond *P, const double *b, double *x,
                     fv_solver_options opt, fv_solver_info *info, void *stream);
fv_status fv_dist_bicgstab(fv_dist *D, fv_precond *P, const double *b, double *x,
                           fv_solver_options opt, fv_solver_info *info, void *stream);

/* Human-readable name of a status. */
const char *fv_status_string(fv_status s);
/* Text of the last CUDA error recorded by this thread (after FV_ERR_CUDA). */
const char *fv_last_error(void);
/* Number of kernels this library has launched in this process (diagnostics). */
uint64_t fv_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* FV_B200_H */
