/* tptfem.h -- C ABI of the B200 (sm_100a) finite-element hot path.
 *
 * Drop-in boundary for tpt-fem's assemble -> CSR -> SPD-solve path.  The
 * reference is a Rust workspace with no FFI of its own; each entry point below
 * names the Rust function it replaces (path:line inside the tpt-fem project),
 * so a Rust crate can bind it 1:1 through a `-sys` crate of extern "C"
 * declarations that mirror this header.
 *
 * Conventions
 *  - Every function returns tptfem_status; on failure the context keeps a
 *    message readable with tptfem_last_error().
 *  - Pointers named `*_host` or documented as host arrays are plain host
 *    memory owned by the caller; the library copies what it needs.
 *  - Index arrays at the ABI are int64 (the reference's usize); the device
 *    uses int32 and every conversion is range-checked (TPTFEM_ERR_INVALID_ARG
 *    or TPTFEM_ERR_CREATION before any kernel launch).
 *  - A context owns one CUDA stream on one device.  Calls on one context are
 *    serialised by the caller; distinct contexts may be used from distinct
 *    threads.  Handles (meshes, matrices, systems) belong to the context that
 *    created them.
 *  - The library never falls back to the CPU: without a usable CUDA device,
 *    tptfem_create() fails with TPTFEM_ERR_DEVICE.
 */
#ifndef TPTFEM_H
#define TPTFEM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  CREATION/SYMBOLIC/NUMERIC mirror SparseError
 * (crates/tpt-fem-sparse/src/lib.rs:67-74); MODEL_DIM_MISMATCH mirrors
 * ElasticityError::ModelDimMismatch (crates/tpt-fem-elasticity/src/lib.rs:28-35). */
typedef enum tptfem_status {
  TPTFEM_OK = 0,
  TPTFEM_ERR_CREATION = 1,
  TPTFEM_ERR_SYMBOLIC = 2,
  TPTFEM_ERR_NUMERIC = 3,
  TPTFEM_ERR_MODEL_DIM_MISMATCH = 4,
  TPTFEM_ERR_NOT_CONVERGED = 5,
  TPTFEM_ERR_BREAKDOWN = 6,
  TPTFEM_ERR_DEVICE = 7,
  TPTFEM_ERR_TIMEOUT = 8,
  TPTFEM_ERR_INVALID_ARG = 9,
  TPTFEM_ERR_OUT_OF_MEMORY = 10
} tptfem_status;

/* Cell types (crates/tpt-fem-mesh CellType, numbered from Line = 1; the linear
   cells of the device path: Tri3 and Quad4 in 2-D, Tet4 in 3-D). */
enum { TPTFEM_CELL_TRI3 = 2, TPTFEM_CELL_QUAD4 = 3, TPTFEM_CELL_TET4 = 4 };

/* ElasticModel (crates/tpt-fem-elasticity/src/lib.rs:56-66). */
enum {
  TPTFEM_MODEL_BAR_AXIAL = 0,
  TPTFEM_MODEL_PLANE_STRESS = 1,
  TPTFEM_MODEL_PLANE_STRAIN = 2,
  TPTFEM_MODEL_CONTINUUM_3D = 3
};

/* Solvers for the reduced SPD system. */
enum {
  /* FP64 Jacobi-preconditioned CG: the plain method and the fallback. */
  TPTFEM_SOLVER_JACOBI_PCG = 0,
  /* Mixed precision: FP32 matrix, vectors and Jacobi preconditioner inside
   * FP64 reliable updates (true residual b - A x and solution in FP64). */
  TPTFEM_SOLVER_MP_PCG = 1,
  /* FP64 Krylov (operator, vectors, reliable updates) preconditioned by the
   * factorised sparse approximate inverse M^-1 = G^T G, G = diag(s)(I + L) on
   * the lower node-block pattern of the reduced matrix, classic FSAI values,
   * the factor stored and applied in reduced precision (s^2 FP32, L FP16). */
  TPTFEM_SOLVER_FSAI_MP_PCG = 2,
  /* As FSAI_MP_PCG with the factor's values emitted by the learned network
   * attached with tptfem_system_attach_lfsai (same pattern, same FP16/FP32
   * storage).  Falls back to FP64 Jacobi-PCG (stats.fell_back = 1) when the
   * factor is invalid or the preconditioned iteration breaks down or does not
   * converge. */
  TPTFEM_SOLVER_LEARNED_FSAI_PCG = 3
};

typedef struct tptfem_context tptfem_context;
typedef struct tptfem_mesh tptfem_mesh;
typedef struct tptfem_matrix tptfem_matrix;
typedef struct tptfem_system tptfem_system;
typedef struct tptfem_dist tptfem_dist;

typedef struct tptfem_solver_opts {
  int32_t solver;        /* TPTFEM_SOLVER_* */
  int32_t max_outer;     /* unused, kept 0 */
  double rel_tol;        /* stop at ||b - A x||_2 / ||b||_2 <= rel_tol, FP64 (0 -> 1e-10) */
  double inner_rel_tol;  /* reliable-update trigger: FP64 residual replacement once the
                            recursive residual fell by this factor (0 -> 1e-6 FP64, 5e-2 FP32) */
  int64_t max_iter;      /* cap on total PCG iterations (0 -> 100000) */
  int32_t batch;         /* PCG iterations per CUDA-graph launch (0 -> auto) */
  int32_t flags;         /* TPTFEM_SOLVE_* bits */
  int32_t coarse_aggregates;  /* TPTFEM_SOLVE_COARSE: target number of aggregates
                                 (0 -> node groups / 2800 for vector problems, / 700
                                 for scalar ones, between 8 and 3000) */
  int32_t reserved;
} tptfem_solver_opts;

/* Recompute the preconditioner's values inside this solve (they are otherwise
 * kept on the system from its first solve); its sparsity pattern is kept. */
#define TPTFEM_SOLVE_FRESH_SETUP 1
/* Keep the scalar CSR operator and factor even where the node-block layout
 * applies (for A/B measurements).  For Jacobi-PCG it selects a separate
 * CSR-only engine; for the FSAI solvers it must be given on the first solve. */
#define TPTFEM_SOLVE_CSR_ONLY 2
/* Node-block operator: use the full block storage of K instead of the default
 * symmetric half storage (lower blocks + diagonal, the upper half applied as
 * the transposes of the lower blocks; K is symmetric up to the FP64 rounding
 * of its element matrices, and the FP64 true residual always uses K itself). */
#define TPTFEM_SOLVE_FULL_OPERATOR 4
/* FSAI / learned-FSAI solvers: add an aggregation coarse correction,
 * M^-1 = G^T G + P A_c^-1 P^T, with P the rigid-body modes (translations and
 * rotations; constants for one dof per node) of the free nodes binned by
 * coordinates into about coarse_aggregates boxes, A_c = P^T A P factorised in
 * FP64 and applied as an FP32 inverse.  Needs full node groups and the mesh
 * geometry (systems from tptfem_reduce_system); otherwise the solve runs
 * without it (stats.coarse_size = 0). */
#define TPTFEM_SOLVE_COARSE 8

typedef struct tptfem_solve_stats {
  int64_t iterations;    /* total PCG iterations (inner iterations for MP) */
  int32_t outer_steps;   /* FP64 true-residual (reliable) updates performed */
  int32_t solver_used;   /* TPTFEM_SOLVER_* actually run (after any fallback) */
  double rel_residual;   /* final TRUE residual ||b - A x||_2/||b||_2 in FP64 */
  double setup_ms;       /* preconditioner set-up, device time (first solve of a system) */
  double solve_ms;       /* iterations + residual checks, device time */
  int32_t fell_back;     /* 1 if the requested method fell back to FP64 Jacobi-PCG */
  int32_t coarse_size;   /* dimension of the coarse space used (0: none) */
} tptfem_solve_stats;

/* ---- context ---------------------------------------------------------------- */
const char* tptfem_version(void);
tptfem_status tptfem_create(int device, tptfem_context** out);
void tptfem_destroy(tptfem_context* ctx);
/* Copies the last error message (NUL-terminated, truncated to len); returns its full length. */
size_t tptfem_last_error(const tptfem_context* ctx, char* buf, size_t len);
tptfem_status tptfem_synchronize(tptfem_context* ctx);

/* ---- meshes (crates/tpt-fem-mesh/src/lib.rs:115-148) -------------------------- */
/* Upload coords (n_nodes x coord_dim, row-major) and conn (n_elems x nodes per
   cell: 3 for Tri3, 4 for Quad4 and Tet4), as MeshBuilder::add_node/add_element
   would hold them (crates/tpt-fem-mesh/src/lib.rs:115-148). */
tptfem_status tptfem_mesh_upload(tptfem_context* ctx, int cell_type, int coord_dim, const double* coords,
                                 int64_t n_nodes, const int64_t* conn, int64_t n_elems, tptfem_mesh** out);
/* box_mesh(min, max, n) generated on the device (crates/tpt-fem-mesh-gen/src/lib.rs:422-495). */
tptfem_status tptfem_mesh_box(tptfem_context* ctx, const double min[3], const double max[3], const int64_t n[3],
                              tptfem_mesh** out);
tptfem_status tptfem_mesh_sizes(const tptfem_mesh* mesh, int64_t* n_nodes, int64_t* n_elems, int* cell_type,
                                int* coord_dim);
tptfem_status tptfem_mesh_download(tptfem_context* ctx, const tptfem_mesh* mesh, double* coords, int64_t* conn);
/* write_vtk / write_vtk_with_data (crates/tpt-fem-io-vtk/src/lib.rs:117-196): the mesh
 * as a legacy BINARY unstructured-grid .vtk file (version 4.1, big-endian, points padded
 * to 3-D) with n_fields per-node scalar fields (names[f]; values[f]: n_nodes doubles in
 * host memory), byte for byte the reference writer's layout.  title NULL -> "tpt-fem mesh",
 * the reference's title. */
tptfem_status tptfem_mesh_write_vtk(tptfem_context* ctx, const tptfem_mesh* mesh, const char* path, const char* title,
                                    int n_fields, const char* const* names, const double* const* values);
/* write_exodus (crates/tpt-fem-io-exodus/src/lib.rs:384-563): the mesh as an Exodus II
 * file in NetCDF-3 classic (CDF-1) form, one element block, coordinates in single
 * precision, with the reference writer's dimensions, variables and byte layout. */
tptfem_status tptfem_mesh_write_exodus(tptfem_context* ctx, const tptfem_mesh* mesh, const char* path);
void tptfem_mesh_free(tptfem_mesh* mesh);

/* ---- assembly ------------------------------------------------------------------
 * Global stiffness in CSR, equal to Coo::to_csr(assemble(...)) of the reference:
 * the pattern holds (row, col) iff at least one element contributed a non-zero
 * value (zero-skip of crates/tpt-fem-assembly/src/lib.rs:469-472), and each value
 * is the sum of element contributions in ascending element order
 * (crates/tpt-fem-sparse/src/lib.rs:144-163), computed in the reference's FP64
 * operation order without FMA contraction.
 *
 * `coef` is per element (per_element = 1, n_elems values) or one constant. */

/* assemble(mesh, 1, poisson_element_matrix) -- crates/tpt-fem-thermal/src/lib.rs:132-160,
 * crates/tpt-fem-assembly/src/lib.rs:458-480. */
tptfem_status tptfem_assemble_poisson(tptfem_context* ctx, tptfem_mesh* mesh, const double* conductivity,
                                      int per_element, int quad_order, tptfem_matrix** out);
/* assemble(mesh, 1, poisson_element_matrix) followed by apply_robin(mesh, 1, h, coo)
 * (crates/tpt-fem-thermal/src/lib.rs:218-237, crates/tpt-fem-assembly/src/lib.rs:674-753):
 * the Robin coefficient is robin_h on the boundary faces whose outward unit normal n
 * has robin_sign * n[robin_axis] > 0.5 and zero on the others; robin_axis < 0 puts
 * robin_h on every boundary face.  As in the reference, every pair of nodes of a
 * boundary face gets a matrix entry (the Robin pushes are not zero-skipped) and the
 * Robin terms are summed after the element terms.  Reassembly keeps the term. */
tptfem_status tptfem_assemble_poisson_robin(tptfem_context* ctx, tptfem_mesh* mesh, const double* conductivity,
                                            int per_element, int quad_order, int robin_axis, double robin_sign,
                                            double robin_h, tptfem_matrix** out);
/* try_assemble(mesh, dim, elasticity_element_matrix) -- crates/tpt-fem-elasticity/src/lib.rs:262-309,
 * crates/tpt-fem-assembly/src/lib.rs:428-450. */
tptfem_status tptfem_assemble_elasticity(tptfem_context* ctx, tptfem_mesh* mesh, int model, const double* young,
                                         int per_element, double poisson, int quad_order, tptfem_matrix** out);
/* Recompute the values of `mat` for new coefficients, reusing its pattern.  If
 * the new coefficients change which entries are non-zero, the pattern is rebuilt
 * (the result still equals a fresh assemble). */
tptfem_status tptfem_reassemble(tptfem_context* ctx, tptfem_matrix* mat, const double* coef, int per_element);
/* Diagnostic (no reference counterpart): average device time in ms of `reps`
 * numeric re-assemblies of `mat` (values only, pattern fixed, coefficients
 * already on the device), timed with CUDA events; the values are rewritten
 * unchanged. */
tptfem_status tptfem_matrix_profile_assembly(tptfem_context* ctx, tptfem_matrix* mat, int reps, double* ms);
/* Csr::nrows / ncols / nnz (crates/tpt-fem-sparse/src/lib.rs:51-63, 122-143). */
tptfem_status tptfem_matrix_sizes(const tptfem_matrix* mat, int64_t* nrows, int64_t* ncols, int64_t* nnz);
tptfem_status tptfem_matrix_download(tptfem_context* ctx, const tptfem_matrix* mat, int64_t* row_ptrs,
                                     int64_t* col_ind, double* values);
void tptfem_matrix_free(tptfem_matrix* mat);
/* Csr::matvec (crates/tpt-fem-sparse/src/lib.rs:195-205): y has max(nrows, xlen) entries. */
tptfem_status tptfem_csr_matvec(tptfem_context* ctx, const tptfem_matrix* mat, const double* x, int64_t xlen,
                                double* y);

/* ---- loads (host rhs arrays, overwritten / accumulated as documented) ---------- */
/* rhs[n_nodes] = Poisson load loop of solve_poisson (crates/tpt-fem-thermal/src/lib.rs:224-230)
 * for a constant source. */
tptfem_status tptfem_load_poisson_source(tptfem_context* ctx, tptfem_mesh* mesh, double source, int quad_order,
                                         double* rhs);
/* rhs[n_nodes*dim] = body-force loop of solve_elasticity (crates/tpt-fem-elasticity/src/lib.rs:371-379). */
tptfem_status tptfem_load_body(tptfem_context* ctx, tptfem_mesh* mesh, const double* body, int quad_order,
                               double* rhs);
/* rhs += apply_neumann (crates/tpt-fem-assembly/src/lib.rs:591-667) with the scalar flux
 * g = traction[c] on boundary faces whose outward unit normal n has sign*n[axis] > 0.5
 * (0 elsewhere), applied to component c of each of the dofs_per_node components. */
tptfem_status tptfem_apply_traction(tptfem_context* ctx, tptfem_mesh* mesh, int dofs_per_node, int axis,
                                    double sign, const double* traction, double* rhs);

/* ---- caller-evaluated sources and fluxes (the reference's closures) --------------
 * The reference takes the volumetric source, the body force, the Neumann flux and the
 * Robin coefficient as Rust closures of the physical point (and of the outward unit
 * normal on the boundary): solve_poisson (crates/tpt-fem-thermal/src/lib.rs:206-240),
 * solve_elasticity (crates/tpt-fem-elasticity/src/lib.rs:355-381), apply_neumann and
 * apply_robin (crates/tpt-fem-assembly/src/lib.rs:591-753).  Across this ABI a closure
 * becomes its values at the points where the reference would call it: query the points,
 * evaluate on the host, pass the values; or pass a C function and let the library do so.
 *
 * Element points: n_elems * nq points, point q of element e at index e * nq + q, with
 * x = sum_k N_k(xi_q) X_k over every stored coordinate (coord_dim values), as
 * poisson_source_vector / elasticity_body_vector form it (thermal:163-196,
 * elasticity:312-348).  *nq is written always; points (n_elems * nq * coord_dim
 * doubles) only when non-NULL. */
tptfem_status tptfem_mesh_quadrature_points(tptfem_context* ctx, tptfem_mesh* mesh, int quad_order, int32_t* nq,
                                            double* points);
/* Boundary points: every boundary face (boundary_faces order, assembly:563-583: by element,
 * then by the cell's face index) and its face-rule points (assembly:336-358), with the
 * outward unit normal of the face (assembly:394-420, 617-653).  *n_points is written
 * always; x and normal (n_points * dim doubles each, dim = 3 for Tet4, 2 for Tri3/Quad4)
 * when non-NULL.  Needs coord_dim == dim (TPTFEM_ERR_INVALID_ARG otherwise). */
tptfem_status tptfem_mesh_boundary_points(tptfem_context* ctx, tptfem_mesh* mesh, int64_t* n_points, double* x,
                                          double* normal);
/* rhs[n_nodes] = the Poisson load loop (thermal:224-230) with the source given at every
 * element point (n_elems * nq values). */
tptfem_status tptfem_load_poisson_source_points(tptfem_context* ctx, tptfem_mesh* mesh, const double* source,
                                                int quad_order, double* rhs);
/* rhs[n_nodes*dim] = the body-force loop (elasticity:371-379) with the body force given at
 * every element point (n_elems * nq * dim values, component-fastest). */
tptfem_status tptfem_load_body_points(tptfem_context* ctx, tptfem_mesh* mesh, const double* body, int quad_order,
                                      double* rhs);
/* rhs += apply_neumann (assembly:591-667) with g given at every boundary point; as in the
 * reference the scalar g is applied to each of the dofs_per_node components, here those
 * whose bit is set in comp_mask (all: 0xFFFFFFFF). */
tptfem_status tptfem_apply_neumann_points(tptfem_context* ctx, tptfem_mesh* mesh, int dofs_per_node, const double* g,
                                          uint32_t comp_mask, double* rhs);
/* assemble(mesh, 1, poisson_element_matrix) followed by apply_robin(mesh, 1, h, coo)
 * (assembly:684-753) with h given at every boundary point. */
tptfem_status tptfem_assemble_poisson_robin_points(tptfem_context* ctx, tptfem_mesh* mesh, const double* conductivity,
                                                   int per_element, int quad_order, const double* h,
                                                   tptfem_matrix** out);
/* The closures as C functions.  `x` holds coord_dim values, `normal` dim values; a body
 * force writes dim values to `out`.  The library calls them on the calling thread, once per
 * point, in point order; values must be finite. */
typedef double (*tptfem_source_fn)(const double* x, int dim, void* user);
typedef double (*tptfem_flux_fn)(const double* x, const double* normal, int dim, void* user);
typedef void (*tptfem_body_fn)(const double* x, int dim, double* out, void* user);
/* solve_poisson (thermal:206-240) with its closures: source(x), optional Neumann flux
 * g(x, n) and Robin coefficient h(x, n) (NULL: none).  u has n_nodes entries. */
tptfem_status tptfem_solve_poisson_fn(tptfem_context* ctx, tptfem_mesh* mesh, double conductivity, int quad_order,
                                      tptfem_source_fn source, void* source_user, const int64_t* bc_dof,
                                      const double* bc_val, int64_t nbc, tptfem_flux_fn neumann,
                                      void* neumann_user, tptfem_flux_fn robin, void* robin_user,
                                      const tptfem_solver_opts* opts, double* u, tptfem_solve_stats* stats);
/* solve_elasticity (elasticity:355-381) with the body force as a closure of x. */
tptfem_status tptfem_solve_elasticity_fn(tptfem_context* ctx, tptfem_mesh* mesh, int model, double young,
                                         double poisson, int quad_order, tptfem_body_fn body, void* body_user,
                                         const int64_t* bc_dof, const double* bc_val, int64_t nbc,
                                         const tptfem_solver_opts* opts, double* u, tptfem_solve_stats* stats);

/* ---- row-partitioned solve over several GPUs ---------------------------------------
 * No counterpart in the reference (its solve is single-threaded).  The reduced system is
 * split into contiguous row ranges row_starts[k] .. row_starts[k+1] (node-aligned: the
 * x-slabs of a box mesh); rank k, on its own GPU, creates its part from the whole reduced
 * system and runs FP64 PCG (Jacobi unless tptfem_dist_set_precond, below) with the caller
 * doing the communication each iteration:
 *   tptfem_dist_start                           -> local r.r, r.z        (sum over ranks)
 *   loop: tptfem_dist_pack; exchange (send_buf segment for rank q goes to q's ghost segment
 *         for this rank, counts from tptfem_dist_counts); tptfem_dist_spmv_dot -> local p.q
 *         (sum); alpha = r.z / p.q; tptfem_dist_update(alpha) -> local r.r, r.z (sum);
 *         beta = r.z_new / r.z; tptfem_dist_direction(beta)
 * Partial sums are reproducible; add the ranks' values in rank order for bitwise-equal runs. */
tptfem_status tptfem_dist_create(tptfem_context* ctx, tptfem_system* sys, int rank, int size,
                                 const int64_t* row_starts, tptfem_dist** out);
/* owned rows, ghost entries, and per peer rank the send / receive counts (size entries each) */
tptfem_status tptfem_dist_counts(const tptfem_dist* d, int64_t* n_owned, int64_t* n_ghost, int64_t* send_counts,
                                 int64_t* recv_counts);
/* device pointers: the packed send buffer (peers in rank order) and the ghost part of p
 * (peers in rank order), for a device-side exchange such as NCCL send/recv */
tptfem_status tptfem_dist_buffers(const tptfem_dist* d, double** send_buf, double** ghost_buf);
tptfem_status tptfem_dist_start(tptfem_context* ctx, tptfem_dist* d, double out_rr_rz[2]);
tptfem_status tptfem_dist_pack(tptfem_context* ctx, tptfem_dist* d);
tptfem_status tptfem_dist_spmv_dot(tptfem_context* ctx, tptfem_dist* d, double* out_pq);
tptfem_status tptfem_dist_update(tptfem_context* ctx, tptfem_dist* d, double alpha, double out_rr_rz[2]);
tptfem_status tptfem_dist_direction(tptfem_context* ctx, tptfem_dist* d, double beta);
/* the owned part of the reduced solution (n_owned doubles, host) */
tptfem_status tptfem_dist_solution(tptfem_context* ctx, const tptfem_dist* d, double* x_owned);
void tptfem_dist_free(tptfem_dist* d);

/* Two-level preconditioner in partitioned form, instead of Jacobi:
 *   M^-1 = blockdiag_k(G_k^T G_k) + P A_c^-1 P^T
 * G_k: the FSAI factor of rank k's owned diagonal block -- classic values
 * (TPTFEM_DIST_PC_FSAI) or the network attached to the system
 * (TPTFEM_DIST_PC_LEARNED, tptfem_system_attach_lfsai); it needs no exchange.
 * With coarse_aggregates >= 0 (0: the one-GPU solver's default count) also the
 * aggregation coarse space of the whole system (full node groups and the mesh
 * geometry needed, row ranges node-aligned; *coarse_size 0 when it does not
 * apply).  sys is the system the rank was created from and must outlive it.
 * Set-up, per rank: tptfem_dist_set_precond leaves this rank's part of A_c
 * (nc x nc doubles) in coarse_matrix (tptfem_dist_coarse_buffers); sum it over
 * the ranks in place, then tptfem_dist_coarse_factor.
 * Iterations: tptfem_dist_start and tptfem_dist_update then return the local
 * r.r in out[0] and 0 in out[1] and leave this rank's part of P^T r (nc doubles)
 * in coarse_vector: sum it over the ranks in place (when nc > 0), then
 * tptfem_dist_precondition -> local r.z (sum); after the start,
 * tptfem_dist_direction(0) sets p = z. */
enum { TPTFEM_DIST_PC_FSAI = 1, TPTFEM_DIST_PC_LEARNED = 2 };
tptfem_status tptfem_dist_set_precond(tptfem_context* ctx, tptfem_dist* d, tptfem_system* sys, int kind,
                                      int coarse_aggregates, int64_t* coarse_size);
/* device pointers (NULL without a coarse space) for the caller's in-place sums */
tptfem_status tptfem_dist_coarse_buffers(const tptfem_dist* d, double** coarse_matrix, double** coarse_vector);
tptfem_status tptfem_dist_coarse_factor(tptfem_context* ctx, tptfem_dist* d);
tptfem_status tptfem_dist_precondition(tptfem_context* ctx, tptfem_dist* d, double* out_rz);
/* Reliable update (the true residual replaces the recursive one; the search
 * direction is kept).  When the summed r.r of a tptfem_dist_update has dropped
 * by 1e-12 since the last replacement, or below the target, skip that step's
 * direction update and: tptfem_dist_residual_begin (x takes the place of p's
 * owned part); pack and exchange as usual; tptfem_dist_residual_end computes
 * r = b - A x (compensated sums) and returns the local r.r, r.z as
 * tptfem_dist_update does (with a block preconditioner: r.r and 0, the
 * restriction's part in coarse_vector, then tptfem_dist_precondition).  Stop
 * if the true r.r meets the target; otherwise beta = r.z (true) / the r.z of
 * the last step length, and tptfem_dist_direction(beta). */
tptfem_status tptfem_dist_residual_begin(tptfem_context* ctx, tptfem_dist* d);
tptfem_status tptfem_dist_residual_end(tptfem_context* ctx, tptfem_dist* d, double out_rr_rz[2]);
/* nranks ranks on this context's GPU in lock step, the exchange done by device copies:
 * the same arithmetic as nranks GPUs (Jacobi, with the reliable updates above);
 * x (n_free doubles, host), *relres the true relative residual at exit.  For testing
 * the partitioned path on one device. */
tptfem_status tptfem_dist_solve_local(tptfem_context* ctx, tptfem_system* sys, int nranks, double rel_tol,
                                      int64_t max_iter, double* x, int64_t* iterations, double* relres);
/* The same with the two-level preconditioner in partitioned form (kind and
 * coarse_aggregates as tptfem_dist_set_precond): every rank's set-up, the
 * partial coarse matrices and restrictions summed in rank order. */
tptfem_status tptfem_dist_solve_local_precond(tptfem_context* ctx, tptfem_system* sys, int nranks, int kind,
                                              int coarse_aggregates, double rel_tol, int64_t max_iter, double* x,
                                              int64_t* iterations, double* relres);

/* ---- eigenvalues (crates/tpt-fem-eigen/src/lib.rs) ---------------------------------- */
enum { TPTFEM_EIG_SMALLEST = 0, TPTFEM_EIG_LARGEST = 1 };  /* EigWhich (eigen:122-129) */
/* lanczos_eigs (eigen:223-262): Lanczos from e_0 with full re-orthogonalisation and
 * lanczos_dim vectors on the device matrix, Ritz pairs of the tridiagonal from the cyclic
 * Jacobi method.  Writes *found = min(num, basis size) eigenvalues (ascending for
 * SMALLEST, descending for LARGEST) and, when vectors != NULL, the unit Ritz vectors
 * (found x nrows, row-major). */
tptfem_status tptfem_lanczos_eigs(tptfem_context* ctx, const tptfem_matrix* mat, int num, int which,
                                  int lanczos_dim, double* values, double* vectors, int* found);
/* power_iteration (eigen:62-88): dominant eigenpair from x_i = i + 1, stopping when the
 * Rayleigh quotient changes by less than tol * max(|lambda|, 1).  x (nrows) may be NULL. */
tptfem_status tptfem_power_iteration(tptfem_context* ctx, const tptfem_matrix* mat, int max_iter, double tol,
                                     double* lambda, double* x, int* iterations);

/* ---- Dirichlet reduction and solve ----------------------------------------------- */
/* reduce_system (crates/tpt-fem-assembly/src/lib.rs:504-535) into a device-resident system. */
tptfem_status tptfem_reduce_system(tptfem_context* ctx, const tptfem_matrix* mat, const double* rhs, int64_t n,
                                   const int64_t* bc_dof, const double* bc_val, int64_t nbc, tptfem_system** out);
/* New values for an existing reduced system: `mat` assembled on the same mesh
 * with new coefficients (same sparsity pattern) and a new rhs; the Dirichlet
 * set and every structure built for the system (node-block layout, factor
 * patterns, coarse geometry, captured graphs) are kept, and each method sets
 * its preconditioner up afresh on its next solve.  This is the reference's
 * reduce_system (crates/tpt-fem-assembly/src/lib.rs:504-535) applied to new
 * values without rebuilding the pattern, as in a loop over coefficient fields
 * on one mesh.  TPTFEM_ERR_INVALID_ARG if the reduced pattern differs. */
tptfem_status tptfem_system_refresh(tptfem_context* ctx, tptfem_system* sys, const tptfem_matrix* mat,
                                    const double* rhs, int64_t n);
tptfem_status tptfem_system_sizes(const tptfem_system* sys, int64_t* n_free, int64_t* nnz);
/* Reduced CSR, fred and the free map, for inspection. */
tptfem_status tptfem_system_download(tptfem_context* ctx, const tptfem_system* sys, int64_t* row_ptrs,
                                     int64_t* col_ind, double* values, double* fred, int64_t* free_dofs);
/* Solve the reduced system on the device; the solution stays resident. */
tptfem_status tptfem_system_solve(tptfem_context* ctx, tptfem_system* sys, const tptfem_solver_opts* opts,
                                  tptfem_solve_stats* stats);
/* Full-length solution as solve_with_dirichlet returns it (crates/tpt-fem-assembly/src/lib.rs:549-558). */
tptfem_status tptfem_system_solution(tptfem_context* ctx, const tptfem_system* sys, double* u);
void tptfem_system_free(tptfem_system* sys);
/* FSAI factor of the reduced system (no reference counterpart): builds the
 * classic factor once (kept on the system) and returns nnz of L.  The
 * download gives L (CSR, strictly lower, values widened from FP16) and
 * sigma^2 (n_free values, widened from FP32); M^-1 = G^T G with
 * G = diag(sigma)(I + L). */
tptfem_status tptfem_system_fsai(tptfem_context* ctx, tptfem_system* sys, int64_t* nnz_l);
tptfem_status tptfem_system_fsai_download(tptfem_context* ctx, const tptfem_system* sys, int64_t* l_row_ptrs,
                                          int64_t* l_col_ind, double* l_values, double* sigma2);
/* Diagnostic (no reference counterpart): average device time in ms of the
 * solver's SpMV kernels on this system -- FP64 CSR, FP32 CSR, FP64 node-block
 * sliced-ELL with full storage and with symmetric half storage (-1 when the
 * system has partial node groups; *nb_bytes / *nbs_bytes = the bytes those
 * layouts must move per launch) -- `reps` launches each, timed with CUDA
 * events on the context's stream.  Used for roofline reports. */
tptfem_status tptfem_system_profile_spmv(tptfem_context* ctx, tptfem_system* sys, int reps, double* ms_f64,
                                         double* ms_f32, double* ms_nb_f64, double* nb_bytes, double* ms_nbs_f64,
                                         double* nbs_bytes);

/* Diagnostic (no reference counterpart): the aggregation coarse space of the
 * system's last TPTFEM_SOLVE_COARSE solve -- number of aggregates, modes per
 * aggregate, bins per axis and, when ainv is non-NULL, the FP32 inverse of
 * A_c = P^T A P widened to FP64 ((na*nm)^2 values, row-major).  *na = 0 when
 * no coarse space was built. */
tptfem_status tptfem_system_coarse(tptfem_context* ctx, const tptfem_system* sys, int32_t* na, int32_t* nm,
                                   int32_t* bins, double* ainv);

/* Allocation-free check of a solution (no counterpart in the reference):
 * relative residual ||b - A x||_2 / ||b||_2 of an n x n CSR system whose arrays
 * (int32 row_ptrs[n+1] and col_ind, FP64 values, x[n], b[n]) are DEVICE memory
 * owned by the caller, computed with compensated FP64 accumulation like the
 * solver's own stopping test.  The result is written to the host double
 * *rel_residual (||r||_2 itself when ||b||_2 = 0).
 * For callers that must not let a library allocate device memory -- e.g. an
 * application holding the whole GPU under a fixed memory budget, or a time-step
 * loop that cannot absorb the device-wide synchronisation of cudaMalloc/cudaFree
 * on every call.  It calls no cudaMalloc, cudaFree or allocating routine: its
 * only scratch is a static 16,448-byte device array (2048 partial sums plus
 * counters), resident on every GPU that loads the library until exit.
 * Limits: 1 <= n <= 2147483646.  Preconditions: row_ptrs holds n+1 entries,
 * col_ind and values hold row_ptrs[n] entries each.  Checked on the device
 * (TPTFEM_ERR_INVALID_ARG, offending rows and entries skipped, never read
 * outside those row_ptrs[n] entries): every row range 0 <= row_ptrs[i] <=
 * row_ptrs[i+1] <= row_ptrs[n], and every column index in [0, n).  `stream`
 * is a cudaStream_t (NULL: the default stream); the call synchronises it
 * before returning.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) and should come before any stream capture;
 * a call that fails with TPTFEM_ERR_DEVICE forgets that address, so the next
 * call looks it up again.  Every call shares the array: calls whose kernels
 * overlap on the GPU race and must be serialised by the caller.
 * `err` (may be NULL) receives a message of at most err_len bytes. */
tptfem_status tptfem_rel_residual_noalloc(int device, void* stream, int64_t n, const int32_t* row_ptrs,
                                          const int32_t* col_ind, const double* values, const double* x,
                                          const double* b, double* rel_residual, char* err, size_t err_len);

/* solve_with_dirichlet (crates/tpt-fem-assembly/src/lib.rs:543-559): reduce, solve, scatter. */
tptfem_status tptfem_solve_with_dirichlet(tptfem_context* ctx, const tptfem_matrix* mat, const double* rhs,
                                          int64_t n, const int64_t* bc_dof, const double* bc_val, int64_t nbc,
                                          const tptfem_solver_opts* opts, double* u, tptfem_solve_stats* stats);

/* solve_poisson with a constant source and no Neumann/Robin term
 * (crates/tpt-fem-thermal/src/lib.rs:206-240).  u has n_nodes entries. */
tptfem_status tptfem_solve_poisson(tptfem_context* ctx, tptfem_mesh* mesh, double conductivity, int quad_order,
                                   double source, const int64_t* bc_dof, const double* bc_val, int64_t nbc,
                                   const tptfem_solver_opts* opts, double* u, tptfem_solve_stats* stats);
/* solve_elasticity with a constant body force (crates/tpt-fem-elasticity/src/lib.rs:355-381).
 * u has n_nodes*dim entries. */
tptfem_status tptfem_solve_elasticity(tptfem_context* ctx, tptfem_mesh* mesh, int model, double young,
                                      double poisson, int quad_order, const double* body, const int64_t* bc_dof,
                                      const double* bc_val, int64_t nbc, const tptfem_solver_opts* opts, double* u,
                                      tptfem_solve_stats* stats);

/* ---- learned FSAI preconditioner (no counterpart in the reference) ----------
 * A small message-passing network over the graph of the reduced matrix that
 * emits the off-diagonal values L of the FSAI factor G = diag(s)(I + L) on the
 * node-block lower pattern; s_i = q_i^-1/2 with q_i = (e_i + L_i) A^ (e_i + L_i)^T
 * (A^ = D^-1/2 A D^-1/2), so M^-1 = G^T G is SPD for any weights.  Trained on
 * the device by the library's own forward/backward kernels on Kaporin's
 * condition number of G^ A^ G^T: loss = (1/n) sum_i log q_i. */
typedef struct tptfem_lfsai tptfem_lfsai;
/* Number of FP32 parameters of the network. */
int64_t tptfem_lfsai_param_count(void);
/* New model on ctx's device, initialised from `seed` (starts as I - tril(A^)). */
tptfem_status tptfem_lfsai_create(tptfem_context* ctx, uint64_t seed, tptfem_lfsai** out);
void tptfem_lfsai_free(tptfem_lfsai* model);
tptfem_status tptfem_lfsai_get_params(tptfem_context* ctx, const tptfem_lfsai* model, float* params);
tptfem_status tptfem_lfsai_set_params(tptfem_context* ctx, tptfem_lfsai* model, const float* params);
/* Loss on `sys`.  with_grad: ADD d loss/d params to the model's gradient
 * buffer (and copy the accumulated gradient to `grad` when it is non-NULL). */
tptfem_status tptfem_lfsai_loss(tptfem_context* ctx, tptfem_lfsai* model, tptfem_system* sys, int32_t with_grad,
                                double* loss, float* grad);
/* Adam step with the accumulated gradient (clipped to +-clip), then zero it. */
tptfem_status tptfem_lfsai_adam(tptfem_context* ctx, tptfem_lfsai* model, double lr, double clip);
/* Use `model` for TPTFEM_SOLVER_LEARNED_FSAI_PCG solves of `sys` (NULL detaches). */
tptfem_status tptfem_system_attach_lfsai(tptfem_context* ctx, tptfem_system* sys, tptfem_lfsai* model);

/* ---- batched 2-D SIMP topology optimisation --------------------------------
 * Replaces topopt_simp (crates/tpt-fem-topopt/src/lib.rs:342-385) for many
 * independent instances: each instance is TopOptParams with a grid of
 * nelx x nely unit-size elements (Grid::new(nelx + 1, nely + 1, h),
 * topopt:89-116), its load vector and its Dirichlet list.  Per iteration the
 * displacement solve is a banded FP64 Cholesky factorisation of K_FF (the
 * reference uses a dense LU), refined to relative residual opts.rel_tol, or
 * FP64 PCG on the matrix-free Q1 operator for grids too wide for the band
 * kernel (see tptfem_topopt_opts.pcg_only).
 * density_filter = 0 follows the reference exactly (E_min = emin, set it to
 * 1e-3 * e0 as topopt:54 does; sensitivity filter topopt:259-279; OC
 * topopt:284-331); density_filter = 1 uses the density filter and OC loop of
 * the published 88-line SIMP code (not in the reference). */
typedef struct tptfem_topopt_instance {
  int32_t nelx, nely;      /* elements along x and y */
  int32_t max_iter;        /* OC iterations (history has max_iter + 1 values) */
  int32_t density_filter;  /* 0: reference sensitivity filter, 1: density filter */
  double h, e0, nu, vol_frac, penal, filter_radius, move_limit, emin;
  /* Loads: f (2 (nelx+1)(nely+1) values, node j*(nelx+1)+i, dofs interleaved)
   * or, when f is NULL, one point load load_value at load_dof. */
  const double* f;
  int64_t load_dof;
  double load_value;
  /* Dirichlet (dof, value) pairs; NULL bc_dof clamps the whole left edge as
   * cantilever_load (topopt:398-415) does.  NULL bc_val means all zero. */
  const int64_t* bc_dof;
  const double* bc_val;
  int64_t nbc;
} tptfem_topopt_instance;

typedef struct tptfem_topopt_opts {
  double rel_tol;         /* displacement solve tolerance (0: 1e-10) */
  int32_t max_pcg_iter;   /* per solve (0: 50000) */
  int32_t block_threads;  /* threads per instance: 256, 512, 1024, or 0 = autotune */
  int32_t use_graph;      /* capture all iterations in one CUDA graph */
  int32_t plain_jacobi;   /* 1: Jacobi-PCG only; 0: Jacobi + per-instance coarse space of plane
                             rigid modes on about 48 node-box aggregates (the default) */
  int32_t pcg_only;       /* 1: every instance by PCG; 0: instances whose grid is at most 110
                             nodes across (half-bandwidth 2 min(nx, ny) + 3 <= 224) are solved
                             by a banded Cholesky factor with iterative refinement to rel_tol,
                             the others (and any factorisation that breaks down) by PCG */
} tptfem_topopt_opts;

typedef struct tptfem_topopt_stats {
  double total_ms;         /* device time of all iterations (CUDA events) */
  double tune_ms;          /* autotuner time (0 when the shape was cached) */
  int64_t pcg_iterations;  /* summed over instances and iterations */
  int32_t block_threads;   /* threads per instance used */
  int32_t not_converged;   /* instances with a solve that hit max_pcg_iter or broke down */
  int64_t refinement_steps; /* iterative-refinement steps of the direct solves, summed */
  int32_t direct_instances; /* instances solved by the banded Cholesky factor */
} tptfem_topopt_stats;

/* Runs n instances.  compliance: sum over instances of (max_iter + 1) values,
 * instance after instance (TopOptResult.compliance); densities: sum of
 * nelx * nely values (TopOptResult.densities; the physical densities in
 * density-filter mode).  Returns TPTFEM_ERR_NOT_CONVERGED (outputs still
 * written) when a solve did not reach rel_tol. */
tptfem_status tptfem_topopt_batch(tptfem_context* ctx, const tptfem_topopt_instance* instances, int32_t n,
                                  const tptfem_topopt_opts* opts, double* compliance, double* densities,
                                  tptfem_topopt_stats* stats);
/* element_stiffness_unit (topopt:166-217): the 8x8 unit-modulus Q1 plane-stress matrix. */
tptfem_status tptfem_topopt_element_stiffness(double nu, double h, double* ke);

/* ---- synthetic input generator (no counterpart in the reference) ---------
 * Gaussian random field by random Fourier features at n host points
 * (n x 3, row-major): out[p] = scale * sum_{m=0}^{M-1} cos(w_m . x_p + phi_m),
 * w host 3 x M row-major (row d = component d of every frequency), phi host
 * M, M = n_features in 1..2048.  The sum runs in ascending m and the dot
 * product as ((x w_0 + y w_1) + z w_2) + phi without contraction, so the
 * same inputs give the same bits on every GPU.  The heterogeneous-Poisson
 * benchmark's conductivity is k = exp(g) at the element centroids. */
tptfem_status tptfem_grf_eval(tptfem_context* ctx, const double* points, int64_t n, const double* w,
                              const double* phi, int32_t n_features, double scale, double* out);

#ifdef __cplusplus
}
#endif
#endif /* TPTFEM_H */
