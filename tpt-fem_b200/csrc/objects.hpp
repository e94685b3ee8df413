// objects.hpp -- the structs behind the opaque C-ABI handles and the internal
// entry points the C ABI (api.cu) dispatches to.
#pragma once
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"

struct tptfem_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  void* cusolver = nullptr;  // cusolverDnHandle_t, created on first use
  void* cublas = nullptr;    // cublasHandle_t, created on first use
  int* d_flag = nullptr;  // device error/validation flag scratch (one int)
  int* h_pinned = nullptr;  // pinned staging (64 bytes)
  void* h_stage = nullptr;  // pinned staging of large user arrays (staging.cu), grown on demand
  size_t h_stage_bytes = 0;
  std::map<uint64_t, int> topo_tuned;  // topopt autotuner: batch shape -> threads per instance
};

namespace tptfem {

// TPTFEM_DEBUG=1: one line per reliable update and per set-up phase on stderr.
inline bool debug_trace() {
  static int v = -1;
  if (v < 0) {
    const char* e = std::getenv("TPTFEM_DEBUG");
    v = (e && e[0] == '1') ? 1 : 0;
  }
  return v == 1;
}

// TPTFEM_DEBUG=1: stream-synchronised wall time of a set-up phase on stderr.
struct PhaseTimer {
  cudaStream_t s;
  const char* name;
  double t0 = 0.0;
  PhaseTimer(cudaStream_t stream, const char* n) : s(stream), name(n) {
    if (debug_trace()) { cudaStreamSynchronize(s); t0 = now_ms(); }
  }
  ~PhaseTimer() {
    if (debug_trace()) {
      cudaStreamSynchronize(s);
      std::fprintf(stderr, "[tptfem] %-28s %9.3f ms\n", name, now_ms() - t0);
    }
  }
  static double now_ms() {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
  }
};

// Device-resident mesh plus lazily built node->element adjacency.
struct MeshData {
  tptfem_context* ctx = nullptr;
  int cell = TPTFEM_CELL_TET4;
  int cdim = 3;   // coordinates stored per node
  int npe = 4;    // nodes per element
  int64_t n_nodes = 0, n_elems = 0;
  DevBuf<double> coords;  // n_nodes x cdim (row-major)
  DevBuf<int> conn;       // n_elems x npe
  // node -> incident elements, sorted by element id: entries (eid << 2) | local_index
  bool adj = false;
  DevBuf<int> ne_ptr, ne;
  // node -> sorted neighbour nodes (including itself)
  DevBuf<int> nb_ptr, nb;
  // per ne entry: position of each of the element's nodes in the node's neighbour list
  DevBuf<uchar4> slot;
  int max_nb = 0;   // largest neighbour count
  int max_deg = 0;  // largest incident-element count
  // per element bitmask of boundary faces (lazy)
  bool bfaces = false;
  DevBuf<unsigned char> bface;
  // boundary faces numbered in (element, face) order: face_off[e] = faces of
  // the elements before e (lazy, with n_bfaces)
  bool foffs = false;
  DevBuf<int> face_off;
  int64_t n_bfaces = 0;
  // per incidence the chain positions of its four blocks, per neighbour entry
  // the start of that slot's chain (lazy, Tet4 chain assembly)
  bool tchains = false;
  DevBuf<uchar4> cpos;
  DevBuf<unsigned char> coff;
};

struct MatrixData {
  tptfem_context* ctx = nullptr;
  std::shared_ptr<MeshData> mesh;
  int physics = 0;  // 0 Poisson, 1 elasticity
  int model = TPTFEM_MODEL_CONTINUUM_3D;
  double nu = 0.0;
  int quad_order = 2;
  int dpn = 1;
  int64_t nrows = 0, nnz = 0;
  int64_t ref_nrows = 0, ref_ncols = 0;  // what Coo::to_csr would report
  DevBuf<int> row_ptr, col;
  DevBuf<double> val;
  DevBuf<double> coef;  // n_elems or 1
  int per_element = 0;
  // apply_robin term added after the element contributions (Poisson): h on the
  // boundary faces whose outward normal n has sign * n[axis] > 0.5 (axis < 0:
  // every boundary face)
  int robin = 0, robin_axis = -1;
  double robin_sign = 1.0, robin_h = 0.0;
  // per-point Robin coefficient h(x, n) at every boundary-face quadrature
  // point (replaces the face selector when not empty)
  DevBuf<double> robin_pts;
  // Tet4 chain assembly: per neighbour entry of every node (nb order), the
  // DPN x DPN mask of its non-zero entries in the current pattern
  DevBuf<unsigned short> nzmask;
};

struct SolverWork;  // solver.cu
struct LfModel;     // lfsai.hpp

// FSAI factor G = diag(sigma) (I + L): sigma^2 (FP32, one per row) and the
// strictly lower L (FP16, CSR) with its explicit transpose (CSR, FP16);
// perm[k_t] = index in L of transposed entry k_t.
struct FsaiFactor {
  int64_t n = 0, nnz = 0;
  bool ready_pattern = false;
  bool overflow = false;  // some pattern row exceeded the device limit
  bool transposed = false;  // trp/tci/perm/tva built (only the row-wise CSR apply needs them)
  bool values_set = false;
  DevBuf<int> rp, ci, trp, tci, perm;
  DevBuf<float> sigma2;
  DevBuf<__half> va, tva;
};

// Node-block sliced-ELL copies of the operator and of the FSAI factor (nbsell.cu).
struct NbSell {
  int state = 0;  // 0 not tried, 1 built, 2 not applicable (partial node groups)
  int dpn = 0, ngroups = 0, nchunks = 0;
  int64_t k_slots = 0, l_slots = 0, u_slots = 0;
  DevBuf<int> gptr, glist;  // group -> sorted neighbour groups
  DevBuf<int> k_cptr, k_col;
  DevBuf<double> k_val;
  DevBuf<int> l_cptr, l_col, u_cptr, u_col, u_pos, nlow;
  DevBuf<uint4> l_pack, u_pack;  // 8 FP16 block values per slot and lane
  DevBuf<__half> l_tail, u_tail, l_diag;
  bool factor_checked = false, factor_ok = false;
  // symmetric half storage of K: lower blocks in the L slots, diagonal blocks
  // per chunk, and for each L^T slot the base index of the transposed block
  bool sym_built = false;
  DevBuf<double> ks_lval, ks_diag;
  DevBuf<int> ku_base;
  bool fresh_fill = false;  // values filled from the CSR since the last solve's set-up
  bool full_stale = false;  // full-storage values predate the last value refresh
};

// Aggregation coarse space of a node-block system (coarse.cu): free mesh
// nodes binned by coordinates into boxes (aggregates); per aggregate the
// rigid-body modes (DPN 3: 3 translations + 3 rotations; DPN 2: 2 + 1;
// DPN 1: the constant), orthonormalised; P = block diagonal of those modes;
// A_c = P^T A P and its inverse (FP32) for the additive correction
// z += P A_c^-1 P^T r.
struct CoarseSpace {
  int state = 0;  // 0 not tried, 1 geometry built, 2 not applicable
  int target = 0;               // requested aggregate count the geometry was built for
  int generation = 0;           // incremented by every (re)build: engines refresh their pointers
  int na = 0, nm = 0, nc = 0;   // aggregates, modes per aggregate, coarse size
  int ld = 0;                   // row stride of Ainv (nc rounded up to a multiple of 4)
  int nseg = 0;                 // segments of aggregate group lists (restriction work items)
  DevBuf<int> sbeg, send;       // per segment: range in alist
  DevBuf<int> aseg;             // aggregate -> its segments (na + 1)
  DevBuf<double> smom;          // per segment: raw mode moments (nseg x nm)
  int bins[3] = {1, 1, 1};
  DevBuf<int> agg;              // per group: aggregate
  DevBuf<int> aptr, alist;      // aggregate -> its groups, ascending
  DevBuf<int> abin;             // per aggregate: bin coordinates (x, y, z)
  DevBuf<int> bin2agg;          // per bin: aggregate or -1
  DevBuf<float> y;              // per group: node position minus the aggregate centroid
  DevBuf<double> T;             // per aggregate: nm x nm mode transform (columns orthonormal modes)
  DevBuf<double> Ac;            // nc x nc, then its Cholesky factor / inverse (FP64)
  DevBuf<int> info;             // status of the last Cholesky (0: positive definite)
  DevBuf<float> Ainv;           // nc x nc inverse (FP32, symmetric, row-major, stride ld)
  DevBuf<double> yc, uc;        // coarse vectors
  DevBuf<double> cm;            // per aggregate: raw-mode coefficients of the prolongation, T uc
  DevBuf<double> Pfull;         // P itself: per dof its nm orthonormal-mode values (geometry only)
  DevBuf<unsigned char> gcolour;  // per group: colour of its aggregate
  DevBuf<unsigned> gmask;       // per group: bit c set iff a neighbour group (or itself) has colour c
  DevBuf<unsigned> cmask;       // per chunk of 32 groups: OR of its groups' gmask
  bool ready = false;           // Ainv holds the inverse for the current values
};

struct SystemData {
  tptfem_context* ctx = nullptr;
  NbSell nb;
  CoarseSpace coarse;
  std::shared_ptr<MeshData> mesh;  // geometry of the matrix the system was reduced from
  int64_t n = 0, n_free = 0, nnz = 0;
  int dpn = 1;            // dofs per mesh node of the full system
  DevBuf<int> free_map;   // reduced -> full
  DevBuf<int> red_map;    // full -> reduced, -1 for fixed dofs
  DevBuf<int> row_ptr, col;
  DevBuf<double> val;
  DevBuf<float> val32;    // lazily converted FP32 copy for mixed precision
  DevBuf<double> fred, x;
  DevBuf<double> u_fixed;  // full-length vector holding the prescribed values
  // kept for tptfem_system_refresh: first bcs index per dof (INT_MAX: free),
  // bcs values, rank of each free dof
  DevBuf<int> bc_first, red_rank;
  DevBuf<double> bc_vals;
  int value_gen = 0;       // incremented when the values are refreshed
  std::shared_ptr<SolverWork> work;
  std::shared_ptr<LfModel> lmodel;  // network used by the learned-FSAI solver
  ~SystemData();
};

// mesh.cu
void mesh_box(MeshData& m, const double mn[3], const double mx[3], const int64_t n[3]);
void mesh_build_adjacency(MeshData& m);
void mesh_build_boundary_faces(MeshData& m);

// assemble.cu
void assemble_matrix(MatrixData& A);             // symbolic + numeric
bool reassemble_values(MatrixData& A);           // numeric; false if the pattern changed
// d_pts (optional): the source / body force at every quadrature point
// (mesh_quad_points order, 1 or dim values per point) instead of the constant.
void load_poisson_source(MeshData& m, double s, int quad_order, double* d_rhs, const double* d_pts = nullptr);
void load_body(MeshData& m, const double* body, int quad_order, double* d_rhs, const double* d_pts = nullptr);
int cell_point_count(int cell, int quad_order);  // quadrature points per element
int face_point_count(int cell);                  // quadrature points per boundary face
void mesh_quad_points(MeshData& m, int quad_order, double* d_out);  // n_elems * nq * cdim
void mesh_build_face_offsets(MeshData& m);
void mesh_face_points(MeshData& m, double* d_x, double* d_n);  // n_bfaces * nqf * sd each
// apply_neumann_order with g given at every boundary-face point, onto the components in comp_mask
void apply_neumann_points(MeshData& m, int dpn, const double* d_g, unsigned comp_mask, double* d_rhs);
void apply_traction(MeshData& m, int dpn, int axis, double sign, const double* t, double* d_rhs);
void csr_matvec_f64(tptfem_context* ctx, int64_t nrows, const int* rp, const int* ci, const double* va,
                    const double* x, double* y);

// reduce.cu
// New values for an existing system (same matrix pattern, same Dirichlet set):
// false if the matrix's reduced pattern differs from the system's.
bool system_refresh(SystemData& S, const MatrixData& A, const double* d_rhs);
std::unique_ptr<SystemData> reduce_system(tptfem_context* ctx, const MatrixData& A, const double* d_rhs,
                                          const int64_t* bc_dof, const double* bc_val, int64_t nbc);
void system_solution(const SystemData& S, double* d_u);

// fsai.cu
struct SystemData;
void fsai_build_pattern(const SystemData& S, FsaiFactor& F);
bool fsai_classic(const SystemData& S, FsaiFactor& F);
// Install FP64 device values (sigma^2 per row, L per pattern entry); false if
// a value is not finite / positive or outside the FP16 range.
bool fsai_set_values(const SystemData& S, FsaiFactor& F, const double* d_sig2, const double* d_lva);

// nbsell.cu
bool nb_build_operator(SystemData& S);  // false when the system has partial node groups
void fsai_build_transpose(const SystemData& S, FsaiFactor& F);  // explicit L^T for the CSR apply (idempotent)
bool nb_fill_factor(SystemData& S, const FsaiFactor& F);  // false: factor rows not node-block shaped
bool nb_factor_shape_ok(SystemData& S, const FsaiFactor& F);  // factor rows = dpn * (lower neighbours) + a
// io_vtk.cu: write_vtk_with_data's legacy binary bytes for a device-resident mesh
std::string vtk_legacy_binary(const MeshData& m, const std::string& title, const std::vector<std::string>& names,
                              const std::vector<const double*>& values);
void write_file(const char* path, const std::string& bytes);
// eigen.cu: lanczos_eigs / power_iteration on a device matrix (returns pairs found / iterations)
int lanczos_eigs(tptfem_context* ctx, const MatrixData& M, int num, int largest, int dim, double* values,
                 double* vectors);
int power_iteration(tptfem_context* ctx, const MatrixData& M, int max_iter, double tol, double* lambda, double* x_out);
// staging.cu: large host arrays through the context's pinned buffer (host threads + one DMA);
// the _ids / _finite variants narrow / check on the way and return false on a bad value.
void host_to_device(tptfem_context* ctx, void* dst, const void* src, size_t bytes);
void device_to_host(tptfem_context* ctx, void* dst, const void* src, size_t bytes);
bool host_to_device_ids(tptfem_context* ctx, int* dst, const int64_t* src, size_t count, int64_t limit);
bool host_to_device_finite(tptfem_context* ctx, double* dst, const double* src, size_t count);
// The groups [g0, g1) of a row-partitioned system (one rank's rows): their
// part of every aggregate's group list, in segments like the whole system's.
struct CoarseLocal {
  int64_t g0 = 0, g1 = 0;
  int nseg = 0;
  DevBuf<int> sbeg, send, alist, aseg;  // aseg: na + 1 entries, empty for aggregates without local groups
  DevBuf<double> smom;                  // restriction moments (nseg x nm)
};
// dist.cu: one rank of the row-partitioned FP64 PCG (see the file's header)
struct DistData {
  tptfem_context* ctx = nullptr;
  int rank = 0, size = 1;
  int64_t r0 = 0, r1 = 0, nloc = 0, nghost = 0;
  DevBuf<int> rp, ci, send_idx;
  DevBuf<double> va, dinv, b, x, xl, r, z, p, q, send_buf, part;  // x + xl: the solution
  std::vector<int64_t> send_off, recv_off;  // per peer rank: ranges in send_buf / in the ghost part of p
  std::vector<int> ghost_cols;              // global reduced index of every ghost column, ascending
  std::vector<double> hpart;
  int blocks_spmv = 1, blocks_vec = 1;
  // block preconditioner (dist_set_precond); pc 0: Jacobi
  int pc = 0;
  SystemData* sys = nullptr;             // the whole reduced system (coarse geometry); the caller keeps it
  std::unique_ptr<SystemData> blk;       // the owned diagonal block as a system of its own
  const FsaiFactor* fac = nullptr;       // its factor (owned by blk)
  int nc = 0, ld = 0;                    // coarse size (0: none) and row stride of ainv
  int cgen = -1;                         // generation of the system's coarse geometry it was built on
  bool coarse_ready = false;
  CoarseLocal cl;
  DevBuf<int> gcol;                      // local column -> global reduced index
  DevBuf<double> t, ac, yc, uc, cm;      // FSAI intermediate; partial / summed A_c; coarse vectors
  DevBuf<double> pbak;                   // owned part of p while x takes its place (true residual)
  DevBuf<float> ainv;
  double sum_parts(int nb, int stride, int which);
};
std::unique_ptr<DistData> dist_create(tptfem_context* ctx, SystemData& S, int rank, int size,
                                      const int64_t* row_starts);
void dist_start(DistData& D, double* out);
void dist_pack(DistData& D);
double dist_spmv_dot(DistData& D);
void dist_update(DistData& D, double alpha, double* out);
void dist_direction(DistData& D, double beta);
// block FSAI (kind 1 classic, 2 learned) of the owned rows, and with aggregates >= 0
// the rank's partial coarse matrix; returns the coarse size (0: none)
int dist_set_precond(DistData& D, SystemData& S, int kind, int aggregates);
void dist_coarse_factor(DistData& D);  // after the caller summed the partial A_c over ranks
double dist_precondition(DistData& D);  // z = M r once the restriction is summed; local r.z
void dist_accumulate(DistData& D);       // x += xl, xl = 0
void dist_residual_begin(DistData& D);   // x in place of p's owned part, for the caller's exchange
void dist_residual_end(DistData& D, double* out);  // r = b - A x; out as dist_update's
// kind 0: Jacobi; 1 / 2 with aggregates as dist_set_precond
int64_t dist_solve_local(tptfem_context* ctx, SystemData& S, int nranks, double tol, int64_t max_iter,
                         double* u_red, double* relres, int kind = 0, int aggregates = -1);
// io_exodus.cu: write_exodus's NetCDF-3 classic bytes for a device-resident mesh
std::string exodus_bytes(const MeshData& m);
void nb_build_sym(SystemData& S);  // after nb_build_operator succeeded
void nb_refill_values(SystemData& S, bool sym);  // operator values again from the CSR (symmetric or full storage)
void nb_refresh_values(SystemData& S);  // refill the node-block values from S.val

// coarse.cu
bool coarse_build(SystemData& S, int target_aggregates);  // geometry (once); false: not applicable
bool coarse_assemble(SystemData& S);                      // A_c and its inverse for the current values
// the same enqueued on stream s with no host wait (false: no coarse geometry),
// then, once s's work is complete or ordered before stream s2, its status
bool coarse_assemble_async(SystemData& S, cudaStream_t s);
bool coarse_finish(SystemData& S, cudaStream_t s2);
// uc = A_c^-1 P^T r and cm = T uc; every kernel returns at once while *done != 0
// (a PCG iteration of a captured batch that the converged solve does not need)
void coarse_restrict_solve(const SystemData& S, const double* r, cudaStream_t s, const int* done);
void coarse_download(const SystemData& S, int* na, int* nm, double* Ainv_or_null);  // FP32 inverse, widened
int coarse_default_aggregates(const SystemData& S);  // about one aggregate per 2000 (vector) / 700 (scalar) groups
// Cholesky and FP32 explicit inverse of an SPD nc x nc matrix (Ac is overwritten;
// zero rows / columns of dropped modes get a unit diagonal); false if not SPD.
bool coarse_factor(tptfem_context* ctx, int nc, int ld, double* Ac, float* Ainv);
// the same enqueued on stream s; the Cholesky's status (0: SPD) goes to d_info
void coarse_factor_async(tptfem_context* ctx, cudaStream_t s, int nc, int ld, double* Ac, float* Ainv, int* d_info);
// partitioned coarse space, the rows of the groups [g0, g1) only (dist.cu)
void coarse_local_build(const SystemData& S, int64_t g0, int64_t g1, CoarseLocal& L);
// this rank's part of A_c = P^T A P (nc x nc, written whole): its rows of A (local CSR,
// gcol: local column -> global reduced index)
void coarse_local_matrix(const SystemData& S, const CoarseLocal& L, int64_t nloc, const int* rp, const int* ci,
                         const double* va, const int* gcol, double* Acp);
void coarse_local_restrict(const SystemData& S, CoarseLocal& L, const double* r_loc, double* yc, cudaStream_t s);
// uc = A_c^-1 yc and cm = T uc (raw-mode coefficients of the prolongation)
void coarse_local_solve(const SystemData& S, int ld, const float* Ainv, const double* yc, double* uc, double* cm,
                        cudaStream_t s);
// solver.cu: y = A x with the system's node-block operator (no reduction)
void nb_operator_apply(SystemData& S, const double* x, double* y);
// Y = A X for the rigid_modes(dpn) interleaved vectors of X (symmetric half
// storage); with gcol, only groups of colour `colour` contribute
void nb_operator_apply_modes(SystemData& S, const double* X, double* Y, const unsigned char* gcol, int colour,
                             const unsigned* cmask, cudaStream_t s);

// solver.cu
int64_t system_fsai_classic(SystemData& S);  // builds (once) the classic factor; -1 on failure
// factor of a whole system for an explicit apply (with its transpose): classic or the
// attached network's values; nullptr when it cannot be built
const FsaiFactor* system_block_factor(SystemData& S, bool learned);
void system_fsai_download(const SystemData& S, int64_t* rp, int64_t* ci, double* lva, double* sig2);
// average device time in ms of `reps` numeric re-assemblies (values only,
// pattern fixed, coefficients resident), timed with CUDA events
double profile_numeric_assembly(MatrixData& M, int reps);
void system_profile_spmv(SystemData& S, int reps, double* ms_f64, double* ms_f32, double* ms_nb, double* nb_bytes,
                         double* ms_nbs, double* nbs_bytes);
void system_solve(SystemData& S, const tptfem_solver_opts& o, tptfem_solve_stats& st);
void system_values_changed(SystemData& S);  // after the values of S.val / S.fred were replaced

// topopt.cu
void topopt_batch(tptfem_context* ctx, const tptfem_topopt_instance* in, int n, const tptfem_topopt_opts* opts,
                  double* compliance, double* densities, tptfem_topopt_stats* stats);
void topopt_element_stiffness(double nu, double h, double* ke);

// grf.cu: random-Fourier-feature field scale * sum_m cos(w_m . x + phi_m) at n
// host points (n x 3), w host 3 x M row-major, phi host M; result to host out.
constexpr int GRF_MAX_FEATURES = 2048;
void grf_eval(tptfem_context* ctx, const double* h_points, int64_t n, const double* h_w, const double* h_phi, int M,
              double scale, double* h_out);

}  // namespace tptfem

struct tptfem_mesh {
  std::shared_ptr<tptfem::MeshData> d;
};
struct tptfem_matrix {
  std::unique_ptr<tptfem::MatrixData> d;
};
struct tptfem_dist {
  std::unique_ptr<tptfem::DistData> d;
};
struct tptfem_system {
  std::unique_ptr<tptfem::SystemData> d;
};
