// api.cu -- the extern "C" boundary declared in include/tptfem.h.
//
// Every entry point validates its arguments on the host before any launch,
// converts int64 indices to the device's int32 with range checks, and maps
// internal errors to tptfem_status plus a message kept in the context.
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <cmath>
#include <cstring>
#include <new>

#include "lfsai.hpp"
#include "objects.hpp"

using namespace tptfem;

namespace {

// Csr::matvec (crates/tpt-fem-sparse/src/lib.rs:195-205): one thread per row,
// sequential s += v * x[c] with explicit round-to-nearest (no FMA), so the
// result matches the reference bit for bit.
__global__ void matvec_exact(int64_t nrows, const int* __restrict__ rp, const int* __restrict__ ci,
                             const double* __restrict__ va, const double* __restrict__ x, double* __restrict__ y) {
  int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrows) return;
  double s = 0.0;
  for (int k = rp[r]; k < rp[r + 1]; ++k) s = __dadd_rn(s, __dmul_rn(va[k], x[ci[k]]));
  y[r] = s;
}

// conn64 -> conn32 with 0 <= c < n_nodes (bit 0 of *flag otherwise); finite coords (bit 1).
tptfem_status fail(tptfem_context* ctx, tptfem_status st, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return st;
}

void set_device(tptfem_context* ctx) { TPT_CUDA(cudaSetDevice(ctx->device)); }

#define API_TRY try {
#define API_CATCH(ctx)                                                         \
  }                                                                            \
  catch (const Error& e) {                                                     \
    return fail((ctx), e.status, e.msg);                                       \
  }                                                                            \
  catch (const std::bad_alloc&) {                                              \
    return fail((ctx), TPTFEM_ERR_OUT_OF_MEMORY, "host allocation failed");    \
  }                                                                            \
  catch (...) {                                                                \
    return fail((ctx), TPTFEM_ERR_DEVICE, "unexpected internal error");        \
  }                                                                            \
  return TPTFEM_OK;

tptfem_solver_opts default_opts(const tptfem_solver_opts* o) {
  tptfem_solver_opts d{};
  d.solver = TPTFEM_SOLVER_JACOBI_PCG;
  d.rel_tol = 1e-10;
  if (o) d = *o;
  return d;
}

void check_coef(const double* coef, int64_t count, const char* what) {
  TPT_REQUIRE(coef != nullptr, TPTFEM_ERR_INVALID_ARG, std::string(what) + " is NULL");
  for (int64_t i = 0; i < count; ++i)
    TPT_REQUIRE(std::isfinite(coef[i]), TPTFEM_ERR_INVALID_ARG, std::string(what) + " holds a non-finite value");
}

struct RobinSpec {
  int on = 0, axis = -1;
  double sign = 1.0, h = 0.0;
  const double* pts = nullptr;  // host h(x, n) per boundary-face point (replaces the selector)
};

std::unique_ptr<MatrixData> new_matrix(tptfem_context* ctx, tptfem_mesh* mesh, int physics, int model,
                                       const double* coef, int per_element, double nu, int quad_order,
                                       RobinSpec robin = RobinSpec{}) {
  TPT_REQUIRE(mesh && mesh->d, TPTFEM_ERR_INVALID_ARG, "mesh is NULL");
  MeshData& m = *mesh->d;
  TPT_REQUIRE(m.ctx == ctx, TPTFEM_ERR_INVALID_ARG, "mesh belongs to another context");
  if (m.cell == TPTFEM_CELL_QUAD4)  // Tet4 and Tri3 use one fixed rule and ignore quad_order
    TPT_REQUIRE(quad_order >= 1 && quad_order <= 5, TPTFEM_ERR_INVALID_ARG, "quad_order must be in 1..=5");
  const int64_t count = per_element ? m.n_elems : 1;
  TPT_REQUIRE(coef != nullptr, TPTFEM_ERR_INVALID_ARG, std::string(physics ? "young" : "conductivity") + " is NULL");
  TPT_REQUIRE(std::isfinite(nu), TPTFEM_ERR_INVALID_ARG, "poisson ratio is not finite");
  auto M = std::make_unique<MatrixData>();
  M->ctx = ctx;
  M->mesh = mesh->d;
  M->physics = physics;
  M->model = model;
  M->nu = nu;
  M->quad_order = quad_order;
  M->per_element = per_element ? 1 : 0;
  M->coef.alloc(count, ctx->stream);
  TPT_REQUIRE(host_to_device_finite(ctx, M->coef.p, coef, (size_t)count), TPTFEM_ERR_INVALID_ARG,
              std::string(physics ? "young" : "conductivity") + " holds a non-finite value");
  M->robin = robin.on;
  M->robin_axis = robin.axis;
  M->robin_sign = robin.sign;
  M->robin_h = robin.h;
  if (robin.on && robin.pts) {
    mesh_build_face_offsets(m);
    const size_t np = (size_t)m.n_bfaces * face_point_count(m.cell);
    M->robin_pts.alloc(std::max<size_t>(np, 1), ctx->stream);
    TPT_REQUIRE(host_to_device_finite(ctx, M->robin_pts.p, robin.pts, np), TPTFEM_ERR_INVALID_ARG,
                "robin coefficient holds a non-finite value");
  }
  assemble_matrix(*M);
  return M;
}

void check_quad_order(const MeshData& m, int quad_order) {
  if (m.cell == TPTFEM_CELL_QUAD4)  // Tet4 and Tri3 use one fixed rule and ignore quad_order
    TPT_REQUIRE(quad_order >= 1 && quad_order <= 5, TPTFEM_ERR_INVALID_ARG, "quad_order must be in 1..=5");
}

int mesh_sd(const MeshData& m) { return m.cell == TPTFEM_CELL_TET4 ? 3 : 2; }

// Element quadrature points on the host (n_elems * nq * cdim).
std::vector<double> host_quad_points(tptfem_context* ctx, MeshData& m, int quad_order, int& nq) {
  nq = cell_point_count(m.cell, quad_order);
  const size_t n = (size_t)m.n_elems * nq * m.cdim;
  std::vector<double> h(n);
  DevBuf<double> d;
  d.alloc(std::max<size_t>(n, 1), ctx->stream);
  mesh_quad_points(m, quad_order, d.p);
  device_to_host(ctx, h.data(), d.p, n * sizeof(double));
  return h;
}

// Boundary-face points and normals on the host (n_points * sd each).
void host_face_points(tptfem_context* ctx, MeshData& m, std::vector<double>& x, std::vector<double>& nrm) {
  TPT_REQUIRE(m.cdim == mesh_sd(m), TPTFEM_ERR_INVALID_ARG,
              "boundary points need as many stored coordinates as the cell's dimension");
  mesh_build_face_offsets(m);
  const size_t n = (size_t)m.n_bfaces * face_point_count(m.cell) * mesh_sd(m);
  x.resize(n);
  nrm.resize(n);
  DevBuf<double> dx, dn;
  dx.alloc(std::max<size_t>(n, 1), ctx->stream);
  dn.alloc(std::max<size_t>(n, 1), ctx->stream);
  mesh_face_points(m, dx.p, dn.p);
  device_to_host(ctx, x.data(), dx.p, n * sizeof(double));
  device_to_host(ctx, nrm.data(), dn.p, n * sizeof(double));
}

// A caller's flux g(x, n) at every boundary-face point, called in point order.
std::vector<double> eval_flux(tptfem_context* ctx, MeshData& m, tptfem_flux_fn fn, void* user) {
  std::vector<double> x, nrm;
  host_face_points(ctx, m, x, nrm);
  const int sd = mesh_sd(m);
  std::vector<double> g(x.size() / sd);
  for (size_t p = 0; p < g.size(); ++p) g[p] = fn(&x[p * sd], &nrm[p * sd], sd, user);
  return g;
}

// rhs (host, in/out) += the per-point Neumann term of g on the components in comp_mask.
void neumann_points_host(tptfem_context* ctx, MeshData& m, int dpn, const double* g, unsigned comp_mask,
                         double* rhs) {
  TPT_REQUIRE(dpn >= 1 && dpn <= 3, TPTFEM_ERR_INVALID_ARG, "dofs_per_node must be 1..3");
  TPT_REQUIRE(m.cdim == mesh_sd(m), TPTFEM_ERR_INVALID_ARG,
              "boundary points need as many stored coordinates as the cell's dimension");
  mesh_build_face_offsets(m);
  const size_t np = (size_t)m.n_bfaces * face_point_count(m.cell);
  const int64_t n = m.n_nodes * dpn;
  DevBuf<double> dg, d;
  dg.alloc(std::max<size_t>(np, 1), ctx->stream);
  TPT_REQUIRE(host_to_device_finite(ctx, dg.p, g, np), TPTFEM_ERR_INVALID_ARG, "flux holds a non-finite value");
  d.alloc(n, ctx->stream);
  host_to_device(ctx, d.p, rhs, n * sizeof(double));
  apply_neumann_points(m, dpn, dg.p, comp_mask, d.p);
  device_to_host(ctx, rhs, d.p, n * sizeof(double));
}

}  // namespace

extern "C" {

const char* tptfem_version(void) { return "tptfem-b200 0.1.0 (sm_100a)"; }

tptfem_status tptfem_create(int device, tptfem_context** out) {
  if (!out) return TPTFEM_ERR_INVALID_ARG;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return TPTFEM_ERR_DEVICE;
  if (device < 0 || device >= count) return TPTFEM_ERR_INVALID_ARG;
  tptfem_context* ctx = new (std::nothrow) tptfem_context;
  if (!ctx) return TPTFEM_ERR_OUT_OF_MEMORY;
  ctx->device = device;
  try {
    TPT_CUDA(cudaSetDevice(device));
    int major = 0;
    TPT_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
    TPT_REQUIRE(major == 10, TPTFEM_ERR_DEVICE, "this build targets sm_100a (B200)");
    TPT_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    for (auto& e : ctx->ev) TPT_CUDA(cudaEventCreate(&e));
    TPT_CUDA(cudaMalloc(&ctx->d_flag, 64));
    TPT_CUDA(cudaMallocHost(&ctx->h_pinned, 64));
    // Stream-ordered allocations (every temporary of the solver and the
    // learned factor) come from the device's default pool; keep freed blocks
    // in it instead of unmapping them at each synchronisation, so repeated
    // solves reuse memory without remapping.  tptfem_destroy trims the pool.
    cudaMemPool_t pool;
    TPT_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t keep = UINT64_MAX;
    TPT_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    // the dense-library handles of the coarse-space set-up, created with the
    // context (their creation takes milliseconds) rather than inside a solve
    cusolverDnHandle_t hs = nullptr;
    TPT_REQUIRE(cusolverDnCreate(&hs) == CUSOLVER_STATUS_SUCCESS, TPTFEM_ERR_DEVICE, "cusolverDnCreate failed");
    ctx->cusolver = hs;
    cublasHandle_t hb = nullptr;
    TPT_REQUIRE(cublasCreate(&hb) == CUBLAS_STATUS_SUCCESS, TPTFEM_ERR_DEVICE, "cublasCreate failed");
    ctx->cublas = hb;
  } catch (const Error& e) {
    tptfem_destroy(ctx);
    return e.status;
  }
  *out = ctx;
  return TPTFEM_OK;
}

void tptfem_destroy(tptfem_context* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto& e : ctx->ev)
    if (e) cudaEventDestroy(e);
  if (ctx->d_flag) cudaFree(ctx->d_flag);
  if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
  if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
  if (ctx->cusolver) cusolverDnDestroy((cusolverDnHandle_t)ctx->cusolver);
  if (ctx->cublas) cublasDestroy((cublasHandle_t)ctx->cublas);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, ctx->device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
  delete ctx;
}

size_t tptfem_last_error(const tptfem_context* ctx, char* buf, size_t len) {
  if (!ctx) return 0;
  const std::string& m = ctx->err;
  if (buf && len) {
    size_t n = m.size() < len - 1 ? m.size() : len - 1;
    std::memcpy(buf, m.data(), n);
    buf[n] = 0;
  }
  return m.size();
}

tptfem_status tptfem_synchronize(tptfem_context* ctx) {
  if (!ctx) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  TPT_CUDA(cudaStreamSynchronize(ctx->stream));
  API_CATCH(ctx)
}

// ---- meshes -------------------------------------------------------------------

tptfem_status tptfem_mesh_upload(tptfem_context* ctx, int cell_type, int coord_dim, const double* coords,
                                 int64_t n_nodes, const int64_t* conn, int64_t n_elems, tptfem_mesh** out) {
  if (!ctx || !out) return TPTFEM_ERR_INVALID_ARG;
  *out = nullptr;
  API_TRY
  set_device(ctx);
  TPT_REQUIRE(cell_type == TPTFEM_CELL_TET4 || cell_type == TPTFEM_CELL_QUAD4 || cell_type == TPTFEM_CELL_TRI3,
              TPTFEM_ERR_INVALID_ARG, "cell_type must be TPTFEM_CELL_TET4, TPTFEM_CELL_QUAD4 or TPTFEM_CELL_TRI3");
  TPT_REQUIRE(cell_type == TPTFEM_CELL_TET4 ? coord_dim == 3 : (coord_dim == 2 || coord_dim == 3),
              TPTFEM_ERR_INVALID_ARG, "coord_dim must be 3 for Tet4 and 2 or 3 for Quad4 and Tri3");
  const int npe = cell_type == TPTFEM_CELL_TRI3 ? 3 : 4;
  TPT_REQUIRE(coords && conn, TPTFEM_ERR_INVALID_ARG, "coords/conn is NULL");
  TPT_REQUIRE(n_nodes > 0 && n_nodes < (1LL << 31), TPTFEM_ERR_INVALID_ARG, "n_nodes out of range");
  TPT_REQUIRE(n_elems > 0 && n_elems < (1LL << 29), TPTFEM_ERR_INVALID_ARG, "n_elems out of range");
  auto m = std::make_shared<MeshData>();
  m->ctx = ctx;
  m->cell = cell_type;
  m->cdim = coord_dim;
  m->npe = npe;
  m->n_nodes = n_nodes;
  m->n_elems = n_elems;
  m->coords.alloc(n_nodes * coord_dim, ctx->stream);
  m->conn.alloc(n_elems * npe, ctx->stream);
  // int64 connectivity narrowed to int32 and range-checked, coordinates checked
  // for finiteness, both on the host threads that stage the copies
  TPT_REQUIRE(host_to_device_finite(ctx, m->coords.p, coords, (size_t)(n_nodes * coord_dim)),
              TPTFEM_ERR_INVALID_ARG, "coords hold a non-finite value");
  TPT_REQUIRE(host_to_device_ids(ctx, m->conn.p, conn, (size_t)(n_elems * npe), n_nodes), TPTFEM_ERR_INVALID_ARG,
              "connectivity entry out of range");
  *out = new tptfem_mesh{m};
  API_CATCH(ctx)
}

tptfem_status tptfem_mesh_box(tptfem_context* ctx, const double min[3], const double max[3], const int64_t n[3],
                              tptfem_mesh** out) {
  if (!ctx || !out || !min || !max || !n) return TPTFEM_ERR_INVALID_ARG;
  *out = nullptr;
  API_TRY
  set_device(ctx);
  auto m = std::make_shared<MeshData>();
  m->ctx = ctx;
  mesh_box(*m, min, max, n);
  TPT_CUDA(cudaStreamSynchronize(ctx->stream));
  *out = new tptfem_mesh{m};
  API_CATCH(ctx)
}

tptfem_status tptfem_mesh_sizes(const tptfem_mesh* mesh, int64_t* n_nodes, int64_t* n_elems, int* cell_type,
                                int* coord_dim) {
  if (!mesh || !mesh->d) return TPTFEM_ERR_INVALID_ARG;
  if (n_nodes) *n_nodes = mesh->d->n_nodes;
  if (n_elems) *n_elems = mesh->d->n_elems;
  if (cell_type) *cell_type = mesh->d->cell;
  if (coord_dim) *coord_dim = mesh->d->cdim;
  return TPTFEM_OK;
}

tptfem_status tptfem_mesh_download(tptfem_context* ctx, const tptfem_mesh* mesh, double* coords, int64_t* conn) {
  if (!ctx || !mesh || !mesh->d) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  const MeshData& m = *mesh->d;
  if (coords) m.coords.download(coords, m.n_nodes * m.cdim);
  std::vector<int> c32;
  if (conn) {
    c32.resize(m.n_elems * m.npe);
    m.conn.download(c32.data(), c32.size());
  }
  TPT_CUDA(cudaStreamSynchronize(ctx->stream));
  for (size_t i = 0; i < c32.size(); ++i) conn[i] = c32[i];
  API_CATCH(ctx)
}

tptfem_status tptfem_mesh_write_vtk(tptfem_context* ctx, const tptfem_mesh* mesh, const char* path, const char* title,
                                    int n_fields, const char* const* names, const double* const* values) {
  if (!ctx || !mesh || !mesh->d || !path || n_fields < 0 || (n_fields > 0 && (!names || !values)))
    return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  std::vector<std::string> nm;
  std::vector<const double*> va;
  for (int f = 0; f < n_fields; ++f) {
    TPT_REQUIRE(names[f] && values[f], TPTFEM_ERR_INVALID_ARG, "field name or values is NULL");
    nm.emplace_back(names[f]);
    va.push_back(values[f]);
  }
  write_file(path, vtk_legacy_binary(*mesh->d, title ? title : "tpt-fem mesh", nm, va));
  API_CATCH(ctx)
}

tptfem_status tptfem_mesh_write_exodus(tptfem_context* ctx, const tptfem_mesh* mesh, const char* path) {
  if (!ctx || !mesh || !mesh->d || !path) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  write_file(path, exodus_bytes(*mesh->d));
  API_CATCH(ctx)
}

tptfem_status tptfem_lanczos_eigs(tptfem_context* ctx, const tptfem_matrix* mat, int num, int which,
                                  int lanczos_dim, double* values, double* vectors, int* found) {
  if (!ctx || !mat || !mat->d || (num > 0 && !values) || !found) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  TPT_REQUIRE(which == TPTFEM_EIG_SMALLEST || which == TPTFEM_EIG_LARGEST, TPTFEM_ERR_INVALID_ARG,
              "which must be TPTFEM_EIG_SMALLEST or TPTFEM_EIG_LARGEST");
  *found = lanczos_eigs(ctx, *mat->d, num, which == TPTFEM_EIG_LARGEST, lanczos_dim, values, vectors);
  API_CATCH(ctx)
}

tptfem_status tptfem_power_iteration(tptfem_context* ctx, const tptfem_matrix* mat, int max_iter, double tol,
                                     double* lambda, double* x, int* iterations) {
  if (!ctx || !mat || !mat->d || !lambda || max_iter < 0) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  const int it = power_iteration(ctx, *mat->d, max_iter, tol, lambda, x);
  if (iterations) *iterations = it;
  API_CATCH(ctx)
}

tptfem_status tptfem_dist_create(tptfem_context* ctx, tptfem_system* sys, int rank, int size,
                                 const int64_t* row_starts, tptfem_dist** out) {
  if (!ctx || !sys || !sys->d || !row_starts || !out) return TPTFEM_ERR_INVALID_ARG;
  *out = nullptr;
  API_TRY
  set_device(ctx);
  *out = new tptfem_dist{dist_create(ctx, *sys->d, rank, size, row_starts)};
  API_CATCH(ctx)
}

tptfem_status tptfem_dist_counts(const tptfem_dist* d, int64_t* n_owned, int64_t* n_ghost, int64_t* send_counts,
                                 int64_t* recv_counts) {
  if (!d || !d->d) return TPTFEM_ERR_INVALID_ARG;
  const DistData& D = *d->d;
  if (n_owned) *n_owned = D.nloc;
  if (n_ghost) *n_ghost = D.nghost;
  for (int k = 0; k < D.size; ++k) {
    if (send_counts) send_counts[k] = D.send_off[k + 1] - D.send_off[k];
    if (recv_counts) recv_counts[k] = D.recv_off[k + 1] - D.recv_off[k];
  }
  return TPTFEM_OK;
}

tptfem_status tptfem_dist_buffers(const tptfem_dist* d, double** send_buf, double** ghost_buf) {
  if (!d || !d->d || !send_buf || !ghost_buf) return TPTFEM_ERR_INVALID_ARG;
  *send_buf = d->d->send_buf.p;
  *ghost_buf = d->d->p.p + d->d->nloc;
  return TPTFEM_OK;
}

#define TPT_DIST_CALL(body)                        \
  if (!ctx || !d || !d->d) return TPTFEM_ERR_INVALID_ARG; \
  API_TRY                                          \
  set_device(ctx);                                 \
  body;                                            \
  API_CATCH(ctx)

tptfem_status tptfem_dist_start(tptfem_context* ctx, tptfem_dist* d, double out_rr_rz[2]) {
  TPT_DIST_CALL(dist_start(*d->d, out_rr_rz))
}
tptfem_status tptfem_dist_pack(tptfem_context* ctx, tptfem_dist* d) { TPT_DIST_CALL(dist_pack(*d->d)) }
tptfem_status tptfem_dist_spmv_dot(tptfem_context* ctx, tptfem_dist* d, double* out_pq) {
  TPT_DIST_CALL(*out_pq = dist_spmv_dot(*d->d))
}
tptfem_status tptfem_dist_update(tptfem_context* ctx, tptfem_dist* d, double alpha, double out_rr_rz[2]) {
  TPT_DIST_CALL(dist_update(*d->d, alpha, out_rr_rz))
}
tptfem_status tptfem_dist_direction(tptfem_context* ctx, tptfem_dist* d, double beta) {
  TPT_DIST_CALL(dist_direction(*d->d, beta))
}
tptfem_status tptfem_dist_precondition(tptfem_context* ctx, tptfem_dist* d, double* out_rz) {
  TPT_DIST_CALL({
    TPT_REQUIRE(out_rz, TPTFEM_ERR_INVALID_ARG, "out_rz is NULL");
    *out_rz = dist_precondition(*d->d);
  })
}
tptfem_status tptfem_dist_residual_begin(tptfem_context* ctx, tptfem_dist* d) {
  TPT_DIST_CALL(dist_residual_begin(*d->d))
}
tptfem_status tptfem_dist_residual_end(tptfem_context* ctx, tptfem_dist* d, double out_rr_rz[2]) {
  TPT_DIST_CALL({
    TPT_REQUIRE(out_rr_rz, TPTFEM_ERR_INVALID_ARG, "out_rr_rz is NULL");
    dist_residual_end(*d->d, out_rr_rz);
  })
}
tptfem_status tptfem_dist_coarse_factor(tptfem_context* ctx, tptfem_dist* d) {
  TPT_DIST_CALL(dist_coarse_factor(*d->d))
}
tptfem_status tptfem_dist_solution(tptfem_context* ctx, const tptfem_dist* d, double* x_owned) {
  TPT_DIST_CALL({
    dist_accumulate(*d->d);
    if (d->d->nloc) device_to_host(ctx, x_owned, d->d->x.p, d->d->nloc * sizeof(double));
  })
}
#undef TPT_DIST_CALL

tptfem_status tptfem_dist_set_precond(tptfem_context* ctx, tptfem_dist* d, tptfem_system* sys, int kind,
                                      int coarse_aggregates, int64_t* coarse_size) {
  if (!ctx || !d || !d->d || !sys || !sys->d) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  const int nc = dist_set_precond(*d->d, *sys->d, kind, coarse_aggregates);
  if (coarse_size) *coarse_size = nc;
  API_CATCH(ctx)
}

tptfem_status tptfem_dist_coarse_buffers(const tptfem_dist* d, double** coarse_matrix, double** coarse_vector) {
  if (!d || !d->d || !coarse_matrix || !coarse_vector) return TPTFEM_ERR_INVALID_ARG;
  *coarse_matrix = d->d->nc ? d->d->ac.p : nullptr;
  *coarse_vector = d->d->nc ? d->d->yc.p : nullptr;
  return TPTFEM_OK;
}

void tptfem_dist_free(tptfem_dist* d) { delete d; }

tptfem_status tptfem_dist_solve_local(tptfem_context* ctx, tptfem_system* sys, int nranks, double rel_tol,
                                      int64_t max_iter, double* x, int64_t* iterations, double* relres) {
  if (!ctx || !sys || !sys->d || !x || !iterations || !relres) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  *iterations = dist_solve_local(ctx, *sys->d, nranks, rel_tol > 0 ? rel_tol : 1e-10, max_iter > 0 ? max_iter : 100000,
                                 x, relres);
  API_CATCH(ctx)
}

tptfem_status tptfem_dist_solve_local_precond(tptfem_context* ctx, tptfem_system* sys, int nranks, int kind,
                                              int coarse_aggregates, double rel_tol, int64_t max_iter, double* x,
                                              int64_t* iterations, double* relres) {
  if (!ctx || !sys || !sys->d || !x || !iterations || !relres) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  TPT_REQUIRE(kind == TPTFEM_DIST_PC_FSAI || kind == TPTFEM_DIST_PC_LEARNED, TPTFEM_ERR_INVALID_ARG,
              "kind must be TPTFEM_DIST_PC_FSAI or TPTFEM_DIST_PC_LEARNED");
  *iterations = dist_solve_local(ctx, *sys->d, nranks, rel_tol > 0 ? rel_tol : 1e-10, max_iter > 0 ? max_iter : 100000,
                                 x, relres, kind, coarse_aggregates);
  API_CATCH(ctx)
}

void tptfem_mesh_free(tptfem_mesh* mesh) { delete mesh; }

// ---- assembly -----------------------------------------------------------------

tptfem_status tptfem_assemble_poisson(tptfem_context* ctx, tptfem_mesh* mesh, const double* conductivity,
                                      int per_element, int quad_order, tptfem_matrix** out) {
  if (!ctx || !out) return TPTFEM_ERR_INVALID_ARG;
  *out = nullptr;
  API_TRY
  set_device(ctx);
  auto M = new_matrix(ctx, mesh, 0, 0, conductivity, per_element, 0.0, quad_order);
  *out = new tptfem_matrix{std::move(M)};
  API_CATCH(ctx)
}

tptfem_status tptfem_assemble_poisson_robin(tptfem_context* ctx, tptfem_mesh* mesh, const double* conductivity,
                                            int per_element, int quad_order, int robin_axis, double robin_sign,
                                            double robin_h, tptfem_matrix** out) {
  if (!ctx || !out) return TPTFEM_ERR_INVALID_ARG;
  *out = nullptr;
  API_TRY
  set_device(ctx);
  TPT_REQUIRE(std::isfinite(robin_h) && std::isfinite(robin_sign), TPTFEM_ERR_INVALID_ARG,
              "robin coefficient or sign is not finite");
  RobinSpec r;
  r.on = 1;
  r.axis = robin_axis < 0 ? -1 : robin_axis;
  r.sign = robin_sign;
  r.h = robin_h;
  auto M = new_matrix(ctx, mesh, 0, 0, conductivity, per_element, 0.0, quad_order, r);
  *out = new tptfem_matrix{std::move(M)};
  API_CATCH(ctx)
}

tptfem_status tptfem_assemble_elasticity(tptfem_context* ctx, tptfem_mesh* mesh, int model, const double* young,
                                         int per_element, double poisson, int quad_order, tptfem_matrix** out) {
  if (!ctx || !out) return TPTFEM_ERR_INVALID_ARG;
  *out = nullptr;
  API_TRY
  set_device(ctx);
  TPT_REQUIRE(model >= TPTFEM_MODEL_BAR_AXIAL && model <= TPTFEM_MODEL_CONTINUUM_3D, TPTFEM_ERR_INVALID_ARG,
              "unknown elasticity model");
  auto M = new_matrix(ctx, mesh, 1, model, young, per_element, poisson, quad_order);
  *out = new tptfem_matrix{std::move(M)};
  API_CATCH(ctx)
}

tptfem_status tptfem_reassemble(tptfem_context* ctx, tptfem_matrix* mat, const double* coef, int per_element) {
  if (!ctx || !mat || !mat->d) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  MatrixData& M = *mat->d;
  const int64_t count = per_element ? M.mesh->n_elems : 1;
  TPT_REQUIRE(coef != nullptr, TPTFEM_ERR_INVALID_ARG, "coefficient is NULL");
  if (M.coef.n != (size_t)count) M.coef.alloc(count, ctx->stream);
  TPT_REQUIRE(host_to_device_finite(ctx, M.coef.p, coef, (size_t)count), TPTFEM_ERR_INVALID_ARG,
              "coefficient holds a non-finite value");
  M.per_element = per_element ? 1 : 0;
  if (!reassemble_values(M)) assemble_matrix(M);  // pattern changed: rebuild it
  API_CATCH(ctx)
}

tptfem_status tptfem_matrix_profile_assembly(tptfem_context* ctx, tptfem_matrix* mat, int reps, double* ms) {
  if (!ctx || !mat || !mat->d || !ms || reps < 1) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  *ms = profile_numeric_assembly(*mat->d, reps);
  API_CATCH(ctx)
}

tptfem_status tptfem_matrix_sizes(const tptfem_matrix* mat, int64_t* nrows, int64_t* ncols, int64_t* nnz) {
  if (!mat || !mat->d) return TPTFEM_ERR_INVALID_ARG;
  if (nrows) *nrows = mat->d->ref_nrows;
  if (ncols) *ncols = mat->d->ref_ncols;
  if (nnz) *nnz = mat->d->nnz;
  return TPTFEM_OK;
}

tptfem_status tptfem_matrix_download(tptfem_context* ctx, const tptfem_matrix* mat, int64_t* row_ptrs,
                                     int64_t* col_ind, double* values) {
  if (!ctx || !mat || !mat->d) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  const MatrixData& M = *mat->d;
  std::vector<int> rp(M.ref_nrows + 1), ci(M.nnz);
  M.row_ptr.download(rp.data(), rp.size());
  M.col.download(ci.data(), ci.size());
  if (values) M.val.download(values, M.nnz);
  TPT_CUDA(cudaStreamSynchronize(ctx->stream));
  if (row_ptrs)
    for (size_t i = 0; i < rp.size(); ++i) row_ptrs[i] = rp[i];
  if (col_ind)
    for (size_t i = 0; i < ci.size(); ++i) col_ind[i] = ci[i];
  API_CATCH(ctx)
}

void tptfem_matrix_free(tptfem_matrix* mat) { delete mat; }

tptfem_status tptfem_csr_matvec(tptfem_context* ctx, const tptfem_matrix* mat, const double* x, int64_t xlen,
                                double* y) {
  if (!ctx || !mat || !mat->d || !x || !y) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  const MatrixData& M = *mat->d;
  TPT_REQUIRE(xlen >= M.ref_ncols, TPTFEM_ERR_INVALID_ARG, "x is shorter than the matrix's column count");
  cudaStream_t s = ctx->stream;
  const int64_t ylen = std::max<int64_t>(M.ref_nrows, xlen);
  DevBuf<double> dx, dy;
  dx.alloc(std::max<int64_t>(xlen, M.nrows), s);
  dx.zero();
  dx.upload(x, xlen);
  dy.alloc(std::max<int64_t>(ylen, M.nrows), s);
  dy.zero();
  matvec_exact<<<ceil_div(M.ref_nrows, 256), 256, 0, s>>>(M.ref_nrows, M.row_ptr.p, M.col.p, M.val.p, dx.p, dy.p);
  TPT_CHECK_LAUNCH();
  dy.download(y, ylen);
  TPT_CUDA(cudaStreamSynchronize(s));
  API_CATCH(ctx)
}

// ---- loads ----------------------------------------------------------------------

tptfem_status tptfem_load_poisson_source(tptfem_context* ctx, tptfem_mesh* mesh, double source, int quad_order,
                                         double* rhs) {
  if (!ctx || !mesh || !mesh->d || !rhs) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  MeshData& m = *mesh->d;
  if (m.cell == TPTFEM_CELL_QUAD4)  // Tet4 and Tri3 use one fixed rule and ignore quad_order
    TPT_REQUIRE(quad_order >= 1 && quad_order <= 5, TPTFEM_ERR_INVALID_ARG, "quad_order must be in 1..=5");
  TPT_REQUIRE(std::isfinite(source), TPTFEM_ERR_INVALID_ARG, "source is not finite");
  DevBuf<double> d;
  d.alloc(m.n_nodes, ctx->stream);
  load_poisson_source(m, source, quad_order, d.p);
  d.download(rhs, m.n_nodes);
  TPT_CUDA(cudaStreamSynchronize(ctx->stream));
  API_CATCH(ctx)
}

tptfem_status tptfem_load_body(tptfem_context* ctx, tptfem_mesh* mesh, const double* body, int quad_order,
                               double* rhs) {
  if (!ctx || !mesh || !mesh->d || !rhs || !body) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  MeshData& m = *mesh->d;
  if (m.cell == TPTFEM_CELL_QUAD4)  // Tet4 and Tri3 use one fixed rule and ignore quad_order
    TPT_REQUIRE(quad_order >= 1 && quad_order <= 5, TPTFEM_ERR_INVALID_ARG, "quad_order must be in 1..=5");
  const int dim = m.cell == TPTFEM_CELL_TET4 ? 3 : 2;
  check_coef(body, dim, "body force");
  DevBuf<double> d;
  d.alloc(m.n_nodes * dim, ctx->stream);
  load_body(m, body, quad_order, d.p);
  d.download(rhs, m.n_nodes * dim);
  TPT_CUDA(cudaStreamSynchronize(ctx->stream));
  API_CATCH(ctx)
}

tptfem_status tptfem_apply_traction(tptfem_context* ctx, tptfem_mesh* mesh, int dofs_per_node, int axis,
                                    double sign, const double* traction, double* rhs) {
  if (!ctx || !mesh || !mesh->d || !rhs || !traction) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  MeshData& m = *mesh->d;
  TPT_REQUIRE(dofs_per_node >= 1 && dofs_per_node <= 3, TPTFEM_ERR_INVALID_ARG, "dofs_per_node must be 1..3");
  check_coef(traction, dofs_per_node, "traction");
  const int64_t n = m.n_nodes * dofs_per_node;
  DevBuf<double> d;
  d.alloc(n, ctx->stream);
  host_to_device(ctx, d.p, rhs, n * sizeof(double));
  apply_traction(m, dofs_per_node, axis, sign, traction, d.p);
  device_to_host(ctx, rhs, d.p, n * sizeof(double));
  API_CATCH(ctx)
}

// ---- reduction and solve ------------------------------------------------------------

tptfem_status tptfem_reduce_system(tptfem_context* ctx, const tptfem_matrix* mat, const double* rhs, int64_t n,
                                   const int64_t* bc_dof, const double* bc_val, int64_t nbc, tptfem_system** out) {
  if (!ctx || !mat || !mat->d || !rhs || !out || (nbc > 0 && (!bc_dof || !bc_val))) return TPTFEM_ERR_INVALID_ARG;
  *out = nullptr;
  API_TRY
  set_device(ctx);
  const MatrixData& M = *mat->d;
  TPT_REQUIRE(n == M.nrows, TPTFEM_ERR_INVALID_ARG, "rhs length does not match the matrix dimension");
  DevBuf<double> d;
  d.alloc(n, ctx->stream);
  host_to_device(ctx, d.p, rhs, n * sizeof(double));
  auto S = reduce_system(ctx, M, d.p, bc_dof, bc_val, nbc);
  *out = new tptfem_system{std::move(S)};
  API_CATCH(ctx)
}

tptfem_status tptfem_system_refresh(tptfem_context* ctx, tptfem_system* sys, const tptfem_matrix* mat,
                                    const double* rhs, int64_t n) {
  if (!ctx || !sys || !sys->d || !mat || !mat->d || !rhs) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  SystemData& S = *sys->d;
  TPT_REQUIRE(n == S.n, TPTFEM_ERR_INVALID_ARG, "rhs length does not match the system");
  DevBuf<double> d;
  d.alloc(n, ctx->stream);
  host_to_device(ctx, d.p, rhs, n * sizeof(double));
  const bool ok = system_refresh(S, *mat->d, d.p);
  system_values_changed(S);  // values were (partly) overwritten either way
  TPT_REQUIRE(ok, TPTFEM_ERR_INVALID_ARG,
              "refresh: the matrix's pattern differs from the system's (reduce the system again)");
  API_CATCH(ctx)
}

tptfem_status tptfem_system_sizes(const tptfem_system* sys, int64_t* n_free, int64_t* nnz) {
  if (!sys || !sys->d) return TPTFEM_ERR_INVALID_ARG;
  if (n_free) *n_free = sys->d->n_free;
  if (nnz) *nnz = sys->d->nnz;
  return TPTFEM_OK;
}

tptfem_status tptfem_system_download(tptfem_context* ctx, const tptfem_system* sys, int64_t* row_ptrs,
                                     int64_t* col_ind, double* values, double* fred, int64_t* free_dofs) {
  if (!ctx || !sys || !sys->d) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  const SystemData& S = *sys->d;
  std::vector<int> rp(S.n_free + 1), ci(S.nnz), fm(S.n_free);
  S.row_ptr.download(rp.data(), rp.size());
  S.col.download(ci.data(), ci.size());
  S.free_map.download(fm.data(), fm.size());
  if (values) S.val.download(values, S.nnz);
  if (fred) S.fred.download(fred, S.n_free);
  TPT_CUDA(cudaStreamSynchronize(ctx->stream));
  if (row_ptrs)
    for (size_t i = 0; i < rp.size(); ++i) row_ptrs[i] = rp[i];
  if (col_ind)
    for (size_t i = 0; i < ci.size(); ++i) col_ind[i] = ci[i];
  if (free_dofs)
    for (size_t i = 0; i < fm.size(); ++i) free_dofs[i] = fm[i];
  API_CATCH(ctx)
}

tptfem_status tptfem_system_solve(tptfem_context* ctx, tptfem_system* sys, const tptfem_solver_opts* opts,
                                  tptfem_solve_stats* stats) {
  if (!ctx || !sys || !sys->d) return TPTFEM_ERR_INVALID_ARG;
  tptfem_solve_stats st{};
  tptfem_status rc = TPTFEM_OK;
  try {
    set_device(ctx);
    system_solve(*sys->d, default_opts(opts), st);
  } catch (const Error& e) {
    rc = fail(ctx, e.status, e.msg);
  } catch (...) {
    rc = fail(ctx, TPTFEM_ERR_DEVICE, "unexpected internal error");
  }
  if (stats) *stats = st;
  return rc;
}

tptfem_status tptfem_system_solution(tptfem_context* ctx, const tptfem_system* sys, double* u) {
  if (!ctx || !sys || !sys->d || !u) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  const SystemData& S = *sys->d;
  DevBuf<double> d;
  d.alloc(S.n, ctx->stream);
  system_solution(S, d.p);
  device_to_host(ctx, u, d.p, S.n * sizeof(double));
  API_CATCH(ctx)
}

void tptfem_system_free(tptfem_system* sys) { delete sys; }

tptfem_status tptfem_system_fsai(tptfem_context* ctx, tptfem_system* sys, int64_t* nnz_l) {
  if (!ctx || !sys || !sys->d || !nnz_l) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  const int64_t nnz = system_fsai_classic(*sys->d);
  TPT_REQUIRE(nnz >= 0, TPTFEM_ERR_NUMERIC, "FSAI factor failed (a principal block is not SPD or a row is too long)");
  *nnz_l = nnz;
  API_CATCH(ctx)
}

tptfem_status tptfem_system_fsai_download(tptfem_context* ctx, const tptfem_system* sys, int64_t* l_row_ptrs,
                                          int64_t* l_col_ind, double* l_values, double* sigma2) {
  if (!ctx || !sys || !sys->d) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  system_fsai_download(*sys->d, l_row_ptrs, l_col_ind, l_values, sigma2);
  API_CATCH(ctx)
}

tptfem_status tptfem_system_profile_spmv(tptfem_context* ctx, tptfem_system* sys, int reps, double* ms_f64,
                                         double* ms_f32, double* ms_nb_f64, double* nb_bytes, double* ms_nbs_f64,
                                         double* nbs_bytes) {
  if (!ctx || !sys || !sys->d || !ms_f64 || !ms_f32 || !ms_nb_f64 || !nb_bytes || !ms_nbs_f64 || !nbs_bytes ||
      reps < 1)
    return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  *nb_bytes = 0.0;
  *nbs_bytes = 0.0;
  *ms_nbs_f64 = -1.0;
  system_profile_spmv(*sys->d, reps, ms_f64, ms_f32, ms_nb_f64, nb_bytes, ms_nbs_f64, nbs_bytes);
  API_CATCH(ctx)
}

tptfem_status tptfem_system_coarse(tptfem_context* ctx, const tptfem_system* sys, int32_t* na, int32_t* nm,
                                   int32_t* bins, double* ainv) {
  if (!ctx || !sys || !sys->d || !na || !nm) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  const SystemData& S = *sys->d;
  *na = 0;
  *nm = 0;
  if (S.coarse.state == 1) {
    int a = 0, m = 0;
    coarse_download(S, &a, &m, S.coarse.ready ? ainv : nullptr);
    *na = a;
    *nm = m;
    if (bins)
      for (int d = 0; d < 3; ++d) bins[d] = S.coarse.bins[d];
  }
  API_CATCH(ctx)
}

tptfem_status tptfem_solve_with_dirichlet(tptfem_context* ctx, const tptfem_matrix* mat, const double* rhs,
                                          int64_t n, const int64_t* bc_dof, const double* bc_val, int64_t nbc,
                                          const tptfem_solver_opts* opts, double* u, tptfem_solve_stats* stats) {
  if (!u) return TPTFEM_ERR_INVALID_ARG;
  tptfem_system* sys = nullptr;
  tptfem_status rc = tptfem_reduce_system(ctx, mat, rhs, n, bc_dof, bc_val, nbc, &sys);
  if (rc != TPTFEM_OK) return rc;
  rc = tptfem_system_solve(ctx, sys, opts, stats);
  if (rc == TPTFEM_OK) rc = tptfem_system_solution(ctx, sys, u);
  tptfem_system_free(sys);
  return rc;
}

tptfem_status tptfem_solve_poisson(tptfem_context* ctx, tptfem_mesh* mesh, double conductivity, int quad_order,
                                   double source, const int64_t* bc_dof, const double* bc_val, int64_t nbc,
                                   const tptfem_solver_opts* opts, double* u, tptfem_solve_stats* stats) {
  if (!ctx || !mesh || !mesh->d || !u) return TPTFEM_ERR_INVALID_ARG;
  tptfem_matrix* K = nullptr;
  tptfem_status rc = tptfem_assemble_poisson(ctx, mesh, &conductivity, 0, quad_order, &K);
  if (rc != TPTFEM_OK) return rc;
  std::vector<double> rhs(mesh->d->n_nodes);
  rc = tptfem_load_poisson_source(ctx, mesh, source, quad_order, rhs.data());
  if (rc == TPTFEM_OK)
    rc = tptfem_solve_with_dirichlet(ctx, K, rhs.data(), (int64_t)rhs.size(), bc_dof, bc_val, nbc, opts, u, stats);
  tptfem_matrix_free(K);
  return rc;
}

tptfem_status tptfem_solve_elasticity(tptfem_context* ctx, tptfem_mesh* mesh, int model, double young,
                                      double poisson, int quad_order, const double* body, const int64_t* bc_dof,
                                      const double* bc_val, int64_t nbc, const tptfem_solver_opts* opts, double* u,
                                      tptfem_solve_stats* stats) {
  if (!ctx || !mesh || !mesh->d || !u || !body) return TPTFEM_ERR_INVALID_ARG;
  tptfem_matrix* K = nullptr;
  tptfem_status rc = tptfem_assemble_elasticity(ctx, mesh, model, &young, 0, poisson, quad_order, &K);
  if (rc != TPTFEM_OK) return rc;
  const int dim = mesh->d->cell == TPTFEM_CELL_TET4 ? 3 : 2;
  std::vector<double> rhs(mesh->d->n_nodes * dim);
  rc = tptfem_load_body(ctx, mesh, body, quad_order, rhs.data());
  if (rc == TPTFEM_OK)
    rc = tptfem_solve_with_dirichlet(ctx, K, rhs.data(), (int64_t)rhs.size(), bc_dof, bc_val, nbc, opts, u, stats);
  tptfem_matrix_free(K);
  return rc;
}

// ---- learned FSAI -----------------------------------------------------------------

int64_t tptfem_lfsai_param_count(void) { return lf_param_count(); }

tptfem_status tptfem_lfsai_create(tptfem_context* ctx, uint64_t seed, tptfem_lfsai** out) {
  if (!ctx || !out) return TPTFEM_ERR_INVALID_ARG;
  *out = nullptr;
  API_TRY
  set_device(ctx);
  auto M = std::make_shared<LfModel>();
  M->ctx = ctx;
  const int np = lf_param_count();
  std::vector<float> h(np);
  lf_init_params(seed, h.data());
  M->prm.alloc(np, ctx->stream);
  M->prm.upload(h.data(), np);
  M->grad.alloc(np, ctx->stream);
  M->grad.zero();
  M->m1.alloc(np, ctx->stream);
  M->m1.zero();
  M->m2.alloc(np, ctx->stream);
  M->m2.zero();
  TPT_CUDA(cudaStreamSynchronize(ctx->stream));
  *out = new tptfem_lfsai{M};
  API_CATCH(ctx)
}

void tptfem_lfsai_free(tptfem_lfsai* model) { delete model; }

tptfem_status tptfem_lfsai_get_params(tptfem_context* ctx, const tptfem_lfsai* model, float* params) {
  if (!ctx || !model || !model->d || !params) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  model->d->prm.download(params, model->d->prm.n);
  TPT_CUDA(cudaStreamSynchronize(ctx->stream));
  API_CATCH(ctx)
}

tptfem_status tptfem_lfsai_set_params(tptfem_context* ctx, tptfem_lfsai* model, const float* params) {
  if (!ctx || !model || !model->d || !params) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  for (size_t i = 0; i < model->d->prm.n; ++i)
    TPT_REQUIRE(std::isfinite(params[i]), TPTFEM_ERR_INVALID_ARG, "parameters hold a non-finite value");
  model->d->prm.upload(params, model->d->prm.n);
  TPT_CUDA(cudaStreamSynchronize(ctx->stream));
  API_CATCH(ctx)
}

tptfem_status tptfem_lfsai_loss(tptfem_context* ctx, tptfem_lfsai* model, tptfem_system* sys, int32_t with_grad,
                                double* loss, float* grad) {
  if (!ctx || !model || !model->d || !sys || !sys->d || !loss) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  SystemData& S = *sys->d;
  TPT_REQUIRE(S.n_free > 0, TPTFEM_ERR_INVALID_ARG, "empty system");
  FsaiFactor* F = nullptr;
  LfGraph& G = system_lf_graph(S, &F);
  LfModel& M = *model->d;
  *loss = lf_loss_grad(S, *F, G, M.prm.p, with_grad ? M.grad.p : nullptr);
  if (with_grad && grad) {
    M.grad.download(grad, M.grad.n);
    TPT_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  API_CATCH(ctx)
}

tptfem_status tptfem_lfsai_adam(tptfem_context* ctx, tptfem_lfsai* model, double lr, double clip) {
  if (!ctx || !model || !model->d || !(lr > 0) || !(clip > 0)) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  LfModel& M = *model->d;
  M.step += 1;
  lf_adam_step(ctx->stream, (int)M.prm.n, M.prm.p, M.grad.p, M.m1.p, M.m2.p, M.step, (float)lr, (float)clip);
  M.grad.zero();
  TPT_CUDA(cudaStreamSynchronize(ctx->stream));
  API_CATCH(ctx)
}

tptfem_status tptfem_system_attach_lfsai(tptfem_context* ctx, tptfem_system* sys, tptfem_lfsai* model) {
  if (!ctx || !sys || !sys->d) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  sys->d->lmodel = model ? model->d : nullptr;
  API_CATCH(ctx)
}

tptfem_status tptfem_topopt_batch(tptfem_context* ctx, const tptfem_topopt_instance* instances, int32_t n,
                                  const tptfem_topopt_opts* opts, double* compliance, double* densities,
                                  tptfem_topopt_stats* stats) {
  if (!ctx || !instances || n < 1 || !compliance || !densities) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  topopt_batch(ctx, instances, n, opts, compliance, densities, stats);
  API_CATCH(ctx)
}

tptfem_status tptfem_topopt_element_stiffness(double nu, double h, double* ke) {
  if (!ke || !(h > 0) || !(nu > -1.0 && nu < 0.5)) return TPTFEM_ERR_INVALID_ARG;
  topopt_element_stiffness(nu, h, ke);
  return TPTFEM_OK;
}

// ---- caller-evaluated sources and fluxes ---------------------------------------

tptfem_status tptfem_mesh_quadrature_points(tptfem_context* ctx, tptfem_mesh* mesh, int quad_order, int32_t* nq,
                                            double* points) {
  if (!ctx || !mesh || !mesh->d || !nq) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  MeshData& m = *mesh->d;
  check_quad_order(m, quad_order);
  *nq = cell_point_count(m.cell, quad_order);
  if (points) {
    int q = 0;
    std::vector<double> h = host_quad_points(ctx, m, quad_order, q);
    std::memcpy(points, h.data(), h.size() * sizeof(double));
  }
  API_CATCH(ctx)
}

tptfem_status tptfem_mesh_boundary_points(tptfem_context* ctx, tptfem_mesh* mesh, int64_t* n_points, double* x,
                                          double* normal) {
  if (!ctx || !mesh || !mesh->d || !n_points) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  MeshData& m = *mesh->d;
  mesh_build_face_offsets(m);
  *n_points = m.n_bfaces * face_point_count(m.cell);
  if (x || normal) {
    std::vector<double> hx, hn;
    host_face_points(ctx, m, hx, hn);
    if (x) std::memcpy(x, hx.data(), hx.size() * sizeof(double));
    if (normal) std::memcpy(normal, hn.data(), hn.size() * sizeof(double));
  }
  API_CATCH(ctx)
}

tptfem_status tptfem_load_poisson_source_points(tptfem_context* ctx, tptfem_mesh* mesh, const double* source,
                                                int quad_order, double* rhs) {
  if (!ctx || !mesh || !mesh->d || !rhs || !source) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  MeshData& m = *mesh->d;
  check_quad_order(m, quad_order);
  const size_t np = (size_t)m.n_elems * cell_point_count(m.cell, quad_order);
  DevBuf<double> dv, d;
  dv.alloc(std::max<size_t>(np, 1), ctx->stream);
  TPT_REQUIRE(host_to_device_finite(ctx, dv.p, source, np), TPTFEM_ERR_INVALID_ARG,
              "source holds a non-finite value");
  d.alloc(m.n_nodes, ctx->stream);
  load_poisson_source(m, 0.0, quad_order, d.p, dv.p);
  device_to_host(ctx, rhs, d.p, m.n_nodes * sizeof(double));
  API_CATCH(ctx)
}

tptfem_status tptfem_load_body_points(tptfem_context* ctx, tptfem_mesh* mesh, const double* body, int quad_order,
                                      double* rhs) {
  if (!ctx || !mesh || !mesh->d || !rhs || !body) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  MeshData& m = *mesh->d;
  check_quad_order(m, quad_order);
  const int dim = mesh_sd(m);
  const size_t np = (size_t)m.n_elems * cell_point_count(m.cell, quad_order) * dim;
  DevBuf<double> dv, d;
  dv.alloc(std::max<size_t>(np, 1), ctx->stream);
  TPT_REQUIRE(host_to_device_finite(ctx, dv.p, body, np), TPTFEM_ERR_INVALID_ARG,
              "body force holds a non-finite value");
  d.alloc(m.n_nodes * dim, ctx->stream);
  load_body(m, nullptr, quad_order, d.p, dv.p);
  device_to_host(ctx, rhs, d.p, m.n_nodes * dim * sizeof(double));
  API_CATCH(ctx)
}

tptfem_status tptfem_apply_neumann_points(tptfem_context* ctx, tptfem_mesh* mesh, int dofs_per_node, const double* g,
                                          uint32_t comp_mask, double* rhs) {
  if (!ctx || !mesh || !mesh->d || !rhs || !g) return TPTFEM_ERR_INVALID_ARG;
  API_TRY
  set_device(ctx);
  neumann_points_host(ctx, *mesh->d, dofs_per_node, g, comp_mask, rhs);
  API_CATCH(ctx)
}

tptfem_status tptfem_assemble_poisson_robin_points(tptfem_context* ctx, tptfem_mesh* mesh, const double* conductivity,
                                                   int per_element, int quad_order, const double* h,
                                                   tptfem_matrix** out) {
  if (!ctx || !out || !h) return TPTFEM_ERR_INVALID_ARG;
  *out = nullptr;
  API_TRY
  set_device(ctx);
  TPT_REQUIRE(mesh && mesh->d, TPTFEM_ERR_INVALID_ARG, "mesh is NULL");
  TPT_REQUIRE(mesh->d->cdim == mesh_sd(*mesh->d), TPTFEM_ERR_INVALID_ARG,
              "boundary points need as many stored coordinates as the cell's dimension");
  RobinSpec r;
  r.on = 1;
  r.pts = h;
  auto M = new_matrix(ctx, mesh, 0, 0, conductivity, per_element, 0.0, quad_order, r);
  *out = new tptfem_matrix{std::move(M)};
  API_CATCH(ctx)
}

tptfem_status tptfem_solve_poisson_fn(tptfem_context* ctx, tptfem_mesh* mesh, double conductivity, int quad_order,
                                      tptfem_source_fn source, void* source_user, const int64_t* bc_dof,
                                      const double* bc_val, int64_t nbc, tptfem_flux_fn neumann,
                                      void* neumann_user, tptfem_flux_fn robin, void* robin_user,
                                      const tptfem_solver_opts* opts, double* u, tptfem_solve_stats* stats) {
  if (!ctx || !mesh || !mesh->d || !u || !source) return TPTFEM_ERR_INVALID_ARG;
  tptfem_matrix* K = nullptr;
  std::vector<double> rhs;
  tptfem_status rc = TPTFEM_OK;
  try {
    set_device(ctx);
    MeshData& m = *mesh->d;
    check_quad_order(m, quad_order);
    // the source closure at every element quadrature point, in element order
    int nq = 0;
    std::vector<double> x = host_quad_points(ctx, m, quad_order, nq);
    std::vector<double> sv((size_t)m.n_elems * nq);
    for (size_t p = 0; p < sv.size(); ++p) sv[p] = source(&x[p * m.cdim], m.cdim, source_user);
    std::vector<double> hv;
    if (robin) hv = eval_flux(ctx, m, robin, robin_user);
    rc = robin ? tptfem_assemble_poisson_robin_points(ctx, mesh, &conductivity, 0, quad_order, hv.data(), &K)
               : tptfem_assemble_poisson(ctx, mesh, &conductivity, 0, quad_order, &K);
    if (rc != TPTFEM_OK) return rc;
    rhs.resize(m.n_nodes);
    rc = tptfem_load_poisson_source_points(ctx, mesh, sv.data(), quad_order, rhs.data());
    if (rc == TPTFEM_OK && neumann) {
      std::vector<double> g = eval_flux(ctx, m, neumann, neumann_user);
      neumann_points_host(ctx, m, 1, g.data(), 1u, rhs.data());
    }
  } catch (const Error& e) {
    if (K) tptfem_matrix_free(K);
    return fail(ctx, e.status, e.msg);
  } catch (const std::bad_alloc&) {
    if (K) tptfem_matrix_free(K);
    return fail(ctx, TPTFEM_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
  if (rc == TPTFEM_OK)
    rc = tptfem_solve_with_dirichlet(ctx, K, rhs.data(), (int64_t)rhs.size(), bc_dof, bc_val, nbc, opts, u, stats);
  tptfem_matrix_free(K);
  return rc;
}

tptfem_status tptfem_solve_elasticity_fn(tptfem_context* ctx, tptfem_mesh* mesh, int model, double young,
                                         double poisson, int quad_order, tptfem_body_fn body, void* body_user,
                                         const int64_t* bc_dof, const double* bc_val, int64_t nbc,
                                         const tptfem_solver_opts* opts, double* u, tptfem_solve_stats* stats) {
  if (!ctx || !mesh || !mesh->d || !u || !body) return TPTFEM_ERR_INVALID_ARG;
  std::vector<double> rhs, bv;
  try {
    set_device(ctx);
    MeshData& m = *mesh->d;
    check_quad_order(m, quad_order);
    int nq = 0;
    std::vector<double> x = host_quad_points(ctx, m, quad_order, nq);
    const int dim = mesh_sd(m);
    bv.assign((size_t)m.n_elems * nq * dim, 0.0);
    for (size_t p = 0; p < (size_t)m.n_elems * nq; ++p) body(&x[p * m.cdim], m.cdim, &bv[p * dim], body_user);
    rhs.resize(m.n_nodes * dim);
  } catch (const Error& e) {
    return fail(ctx, e.status, e.msg);
  } catch (const std::bad_alloc&) {
    return fail(ctx, TPTFEM_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
  tptfem_matrix* K = nullptr;
  tptfem_status rc = tptfem_assemble_elasticity(ctx, mesh, model, &young, 0, poisson, quad_order, &K);
  if (rc != TPTFEM_OK) return rc;
  rc = tptfem_load_body_points(ctx, mesh, bv.data(), quad_order, rhs.data());
  if (rc == TPTFEM_OK)
    rc = tptfem_solve_with_dirichlet(ctx, K, rhs.data(), (int64_t)rhs.size(), bc_dof, bc_val, nbc, opts, u, stats);
  tptfem_matrix_free(K);
  return rc;
}

tptfem_status tptfem_grf_eval(tptfem_context* ctx, const double* points, int64_t n, const double* w,
                              const double* phi, int32_t n_features, double scale, double* out) {
  if (!ctx || n < 0 || (n > 0 && (!points || !out)) || !w || !phi) return TPTFEM_ERR_INVALID_ARG;
  if (n_features < 1 || n_features > GRF_MAX_FEATURES)
    return fail(ctx, TPTFEM_ERR_INVALID_ARG, "n_features must be in 1..2048");
  if (n == 0) return TPTFEM_OK;
  API_TRY
  set_device(ctx);
  grf_eval(ctx, points, n, w, phi, n_features, scale, out);
  API_CATCH(ctx)
}

}  // extern "C"
