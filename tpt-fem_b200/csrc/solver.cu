// solver.cu -- CSR SpMV and the PCG solvers for the reduced SPD system.
//
// The reference solves with a dense partial-pivot LU
// (crates/tpt-fem-sparse/src/lib.rs:244-278), infeasible beyond a few thousand
// dofs; the device path replaces it with preconditioned CG:
//   * TPTFEM_SOLVER_JACOBI_PCG: FP64 values, vectors and reductions; the plain
//     method and the fallback.
//   * TPTFEM_SOLVER_MP_PCG: FP32 matrix/vectors inside FP64 iterative
//     refinement: the outer loop forms r = b - A x with the FP64 matrix and
//     accumulates x in FP64, each inner solve reduces the FP32 residual by
//     inner_rel_tol.
//
// Kernel structure per PCG iteration (three launches, captured in a CUDA
// graph in batches so the host only checks convergence once per batch):
//   K1 spmv_dot : q = A p, pq = p.q
//   K2 update   : alpha = rz/pq; x += alpha p; r -= alpha q; rz' = r.(D^-1 r), rr = r.r
//   K3 direction: beta = rz'/rz; p = D^-1 r + beta p
// Every dot product is reduced deterministically: per-block partials, then
// the last block to finish (atomic ticket) sums them in a fixed order and
// writes the scalar into the solver state.  Results are bitwise reproducible
// for a fixed launch configuration.  No kernel spins or waits on another.
#include <algorithm>
#include <cmath>

#include "objects.hpp"

namespace tptfem {

namespace {

constexpr int VEC_THREADS = 256;
constexpr int SPMV_THREADS = 256;

struct PcgState {
  double rz[2];   // r.z by iteration parity
  double pq;
  double rr;
  double stop2;   // stop when rr <= stop2
  int done;       // 0 running, 1 converged, 2 breakdown, 3 iteration cap
  int iters;
  int max_iters;
  int pad;
  unsigned ticket[4];
};

// Block-wide sum of up to two doubles in a fixed order.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV]) {
  __shared__ double sh[NV][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_down_sync(0xffffffffu, v[i], o);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int i = 0; i < NV; ++i) sh[i][wid] = v[i];
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      double t = lane < nw ? sh[i][lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
      v[i] = t;
    }
  }
}

// Per-block partials then a fixed-order sum by the last block to arrive.
// Returns true in thread 0 of the last block, with the totals in v.
template <int NV>
__device__ __forceinline__ bool grid_sum(double (&v)[NV], double* partials, unsigned* ticket) {
  block_sum<NV>(v);
  __shared__ bool last;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) partials[i * gridDim.x + blockIdx.x] = v[i];
    __threadfence();
    unsigned t = atomicAdd(ticket, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double acc[NV];
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    acc[i] = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) acc[i] += __ldcg(partials + i * gridDim.x + b);
  }
  block_sum<NV>(acc);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) v[i] = acc[i];
    *ticket = 0;
  }
  return threadIdx.x == 0;
}

// y = A x with LANES threads per row; all lanes of a warp run the same number
// of loop trips so the segment shuffles are always converged.
template <typename T, int LANES>
__device__ __forceinline__ T row_dot(const int* __restrict__ rp, const int* __restrict__ ci,
                                     const T* __restrict__ va, const T* __restrict__ x, int row, bool valid) {
  T s = T(0);
  if (valid) {
    const int b = rp[row], e = rp[row + 1];
    for (int k = b + (threadIdx.x & (LANES - 1)); k < e; k += LANES) s += va[k] * __ldg(x + ci[k]);
  }
#pragma unroll
  for (int o = LANES / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, LANES);
  return s;
}

template <typename T, int LANES, bool DOT>
__global__ void __launch_bounds__(SPMV_THREADS) spmv_kernel(int n, const int* __restrict__ rp,
                                                            const int* __restrict__ ci, const T* __restrict__ va,
                                                            const T* __restrict__ x, T* __restrict__ y,
                                                            PcgState* st, double* partials) {
  if (DOT && st->done) return;
  constexpr int RPW = 32 / LANES;  // rows per warp per trip
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int sub = (threadIdx.x & 31) / LANES;
  const bool head = (threadIdx.x & (LANES - 1)) == 0;
  double d[1] = {0.0};
  for (int base = warp * RPW; base < n; base += nwarps * RPW) {
    const int row = base + sub;
    const bool valid = row < n;
    T s = row_dot<T, LANES>(rp, ci, va, x, row, valid);
    if (valid && head) {
      y[row] = s;
      if (DOT) d[0] += (double)x[row] * (double)s;
    }
  }
  if (DOT) {
    if (grid_sum<1>(d, partials, &st->ticket[0])) {
      st->pq = d[0];
      if (!(d[0] > 0.0)) st->done = 2;  // p.Ap <= 0 or NaN: not SPD / breakdown
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(VEC_THREADS) pcg_update(int n, int par, T* __restrict__ x, T* __restrict__ r,
                                                          const T* __restrict__ p, const T* __restrict__ q,
                                                          const T* __restrict__ dinv, PcgState* st,
                                                          double* partials) {
  if (st->done) return;
  const double alpha = st->rz[par] / st->pq;
  const T a = (T)alpha;
  double v[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] += a * p[i];
    T ri = r[i] - a * q[i];
    r[i] = ri;
    v[0] += (double)ri * (double)(dinv[i] * ri);
    v[1] += (double)ri * (double)ri;
  }
  if (grid_sum<2>(v, partials, &st->ticket[1])) {
    st->rz[par ^ 1] = v[0];
    st->rr = v[1];
    st->iters += 1;
    if (!(v[1] == v[1]) || !(v[0] == v[0])) st->done = 2;
    else if (v[1] <= st->stop2) st->done = 1;
    else if (st->iters >= st->max_iters) st->done = 3;
  }
}

template <typename T>
__global__ void __launch_bounds__(VEC_THREADS) pcg_direction(int n, int par, const T* __restrict__ r,
                                                             T* __restrict__ p, const T* __restrict__ dinv,
                                                             const PcgState* st) {
  if (st->done) return;
  const T beta = (T)(st->rz[par ^ 1] / st->rz[par]);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = dinv[i] * r[i] + beta * p[i];
}

// x = 0, r = b, p = D^-1 b; rz[0] = r.z, rr = r.r; stop2 = (tol^2) * rr.
template <typename T>
__global__ void pcg_init(int n, const T* __restrict__ b, T* __restrict__ x, T* __restrict__ r, T* __restrict__ p,
                         const T* __restrict__ dinv, PcgState* st, double* partials, double tol2, int max_iters) {
  double v[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    T bi = b[i];
    x[i] = T(0);
    r[i] = bi;
    p[i] = dinv[i] * bi;
    v[0] += (double)bi * (double)(dinv[i] * bi);
    v[1] += (double)bi * (double)bi;
  }
  if (grid_sum<2>(v, partials, &st->ticket[2])) {
    st->rz[0] = v[0];
    st->rr = v[1];
    st->stop2 = tol2 * v[1];
    st->iters = 0;
    st->max_iters = max_iters;
    st->pq = 0.0;
    st->done = (v[1] == 0.0) ? 1 : 0;
  }
}

// dinv = 1 / diag(A); flags rows whose diagonal is missing or not positive.
template <typename T>
__global__ void jacobi_diag(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                            const double* __restrict__ va, T* __restrict__ dinv, int* flag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double d = 0.0;
  for (int k = rp[i]; k < rp[i + 1]; ++k)
    if (ci[k] == i) d = va[k];
  if (!(d > 0.0)) atomicOr(flag, 1);
  dinv[i] = (T)(1.0 / d);
}

// FP64 true residual r = b - A x and ||r||^2 (into st->rr via the ticket).
template <int LANES>
__global__ void __launch_bounds__(SPMV_THREADS) residual_f64(int n, const int* __restrict__ rp,
                                                             const int* __restrict__ ci,
                                                             const double* __restrict__ va,
                                                             const double* __restrict__ x,
                                                             const double* __restrict__ b, double* __restrict__ r,
                                                             double* out2, unsigned* ticket, double* partials) {
  constexpr int RPW = 32 / LANES;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int sub = (threadIdx.x & 31) / LANES;
  const bool head = (threadIdx.x & (LANES - 1)) == 0;
  double d[1] = {0.0};
  for (int base = warp * RPW; base < n; base += nwarps * RPW) {
    const int row = base + sub;
    const bool valid = row < n;
    double s = row_dot<double, LANES>(rp, ci, va, x, row, valid);
    if (valid && head) {
      double ri = b[row] - s;
      r[row] = ri;
      d[0] += ri * ri;
    }
  }
  if (grid_sum<1>(d, partials, ticket)) *out2 = d[0];
}

__global__ void to_f32(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}

__global__ void add_f32_to_f64(int n, const float* __restrict__ d, double* __restrict__ x) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] += (double)d[i];
}

__global__ void sumsq_kernel(int n, const double* __restrict__ b, double* out, unsigned* ticket, double* partials) {
  double v[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[0] += b[i] * b[i];
  if (grid_sum<1>(v, partials, ticket)) *out = v[0];
}

// ---- host side -------------------------------------------------------------------

int pick_lanes(int64_t nrows, int64_t nnz) {
  double avg = nrows ? (double)nnz / (double)nrows : 1.0;
  if (avg <= 3) return 2;
  if (avg <= 12) return 4;
  if (avg <= 40) return 8;
  if (avg <= 96) return 16;
  return 32;
}

template <typename T, bool DOT>
void launch_spmv(int lanes, int grid, cudaStream_t s, int n, const int* rp, const int* ci, const T* va, const T* x,
                 T* y, PcgState* st, double* partials) {
  switch (lanes) {
    case 2: spmv_kernel<T, 2, DOT><<<grid, SPMV_THREADS, 0, s>>>(n, rp, ci, va, x, y, st, partials); break;
    case 4: spmv_kernel<T, 4, DOT><<<grid, SPMV_THREADS, 0, s>>>(n, rp, ci, va, x, y, st, partials); break;
    case 8: spmv_kernel<T, 8, DOT><<<grid, SPMV_THREADS, 0, s>>>(n, rp, ci, va, x, y, st, partials); break;
    case 16: spmv_kernel<T, 16, DOT><<<grid, SPMV_THREADS, 0, s>>>(n, rp, ci, va, x, y, st, partials); break;
    default: spmv_kernel<T, 32, DOT><<<grid, SPMV_THREADS, 0, s>>>(n, rp, ci, va, x, y, st, partials); break;
  }
  TPT_CHECK_LAUNCH();
}

void launch_residual(int lanes, int grid, cudaStream_t s, int n, const int* rp, const int* ci, const double* va,
                     const double* x, const double* b, double* r, double* out2, unsigned* ticket,
                     double* partials) {
  switch (lanes) {
    case 2: residual_f64<2><<<grid, SPMV_THREADS, 0, s>>>(n, rp, ci, va, x, b, r, out2, ticket, partials); break;
    case 4: residual_f64<4><<<grid, SPMV_THREADS, 0, s>>>(n, rp, ci, va, x, b, r, out2, ticket, partials); break;
    case 8: residual_f64<8><<<grid, SPMV_THREADS, 0, s>>>(n, rp, ci, va, x, b, r, out2, ticket, partials); break;
    case 16: residual_f64<16><<<grid, SPMV_THREADS, 0, s>>>(n, rp, ci, va, x, b, r, out2, ticket, partials); break;
    default: residual_f64<32><<<grid, SPMV_THREADS, 0, s>>>(n, rp, ci, va, x, b, r, out2, ticket, partials); break;
  }
  TPT_CHECK_LAUNCH();
}

}  // namespace

// Per-precision PCG engine: vectors, state and the captured iteration graph.
template <typename T>
struct Pcg {
  int n = 0;
  int lanes = 8, spmv_grid = 0, vec_grid = 0, batch = 32;
  const int* rp = nullptr;
  const int* ci = nullptr;
  const T* va = nullptr;
  DevBuf<T> x, r, p, q, dinv, b;
  DevBuf<double> partials;
  DevBuf<PcgState> st;
  cudaGraphExec_t exec = nullptr;
  ~Pcg() {
    if (exec) cudaGraphExecDestroy(exec);
  }
  void setup(int n_, const int* rp_, const int* ci_, const T* va_, int64_t nnz, cudaStream_t s, int batch_) {
    n = n_;
    rp = rp_; ci = ci_; va = va_;
    lanes = pick_lanes(n, nnz);
    const int sms = sm_count();
    int per_sm = 0;
    TPT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, spmv_kernel<T, 8, true>, SPMV_THREADS, 0));
    spmv_grid = std::max(1, std::min(sms * std::max(per_sm, 1), ceil_div((int64_t)n * lanes, SPMV_THREADS)));
    vec_grid = std::max(1, std::min(sms * 4, ceil_div(n, VEC_THREADS)));
    batch = batch_ > 0 ? batch_ : 32;
    x.alloc(n, s); r.alloc(n, s); p.alloc(n, s); q.alloc(n, s); dinv.alloc(n, s); b.alloc(n, s);
    partials.alloc(2 * (size_t)std::max(spmv_grid, vec_grid) + 2, s);
    st.alloc(1, s);
    st.zero();
  }
  void capture(cudaStream_t s) {
    if (exec) return;
    cudaGraph_t g;
    TPT_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int it = 0; it < batch; ++it) {
      const int par = it & 1;
      launch_spmv<T, true>(lanes, spmv_grid, s, n, rp, ci, va, p.p, q.p, st.p, partials.p);
      pcg_update<T><<<vec_grid, VEC_THREADS, 0, s>>>(n, par, x.p, r.p, p.p, q.p, dinv.p, st.p, partials.p);
      pcg_direction<T><<<vec_grid, VEC_THREADS, 0, s>>>(n, par, r.p, p.p, dinv.p, st.p);
    }
    TPT_CUDA(cudaStreamEndCapture(s, &g));
    cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    TPT_CUDA(e);
  }
  // Run PCG on the current b from x = 0.  Returns the final state.
  PcgState run(double rel_tol, int max_iters, cudaStream_t s, PcgState* h_state) {
    pcg_init<T><<<vec_grid, VEC_THREADS, 0, s>>>(n, b.p, x.p, r.p, p.p, dinv.p, st.p, partials.p,
                                                 rel_tol * rel_tol, max_iters);
    TPT_CHECK_LAUNCH();
    capture(s);
    // The batch graph always starts at parity 0: keep batches even-sized so the
    // parity of rz matches the iteration count.
    for (;;) {
      TPT_CUDA(cudaMemcpyAsync(h_state, st.p, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
      TPT_CUDA(cudaStreamSynchronize(s));
      if (h_state->done) break;
      TPT_CUDA(cudaGraphLaunch(exec, s));
    }
    return *h_state;
  }
};

struct SolverWork {
  Pcg<double> f64;
  Pcg<float> f32;
  bool f64_ready = false, f32_ready = false;
  DevBuf<double> res;   // FP64 residual / scratch
  DevBuf<double> sc;    // scalars
  DevBuf<unsigned> tk;  // tickets for standalone reductions
  DevBuf<double> partials;
  PcgState* h_state = nullptr;
  ~SolverWork() {
    if (h_state) cudaFreeHost(h_state);
  }
};

SystemData::~SystemData() = default;

namespace {

void ensure_work(SystemData& S) {
  cudaStream_t s = S.ctx->stream;
  if (!S.work) {
    S.work = std::make_shared<SolverWork>();
    TPT_CUDA(cudaMallocHost(&S.work->h_state, sizeof(PcgState)));
    S.work->res.alloc(std::max<int64_t>(S.n_free, 1), s);
    S.work->sc.alloc(8, s);
    S.work->tk.alloc(8, s);
    S.work->tk.zero();
    S.work->partials.alloc(4096, s);
  }
}

void diag_check(tptfem_context* ctx) {
  TPT_CUDA(cudaMemcpyAsync(ctx->h_pinned, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  TPT_CUDA(cudaStreamSynchronize(ctx->stream));
  TPT_REQUIRE(ctx->h_pinned[0] == 0, TPTFEM_ERR_NUMERIC,
              "reduced matrix has a missing or non-positive diagonal entry (not SPD)");
}

void prepare_f64(SystemData& S, int batch) {
  SolverWork& W = *S.work;
  if (W.f64_ready) return;
  cudaStream_t s = S.ctx->stream;
  W.f64.setup((int)S.n_free, S.row_ptr.p, S.col.p, S.val.p, S.nnz, s, batch);
  TPT_CUDA(cudaMemsetAsync(S.ctx->d_flag, 0, sizeof(int), s));
  jacobi_diag<double><<<ceil_div(S.n_free, 256), 256, 0, s>>>((int)S.n_free, S.row_ptr.p, S.col.p, S.val.p,
                                                              W.f64.dinv.p, S.ctx->d_flag);
  TPT_CHECK_LAUNCH();
  diag_check(S.ctx);
  W.f64_ready = true;
}

void prepare_f32(SystemData& S, int batch) {
  SolverWork& W = *S.work;
  if (W.f32_ready) return;
  cudaStream_t s = S.ctx->stream;
  if (!S.val32.p) {
    S.val32.alloc(S.nnz, s);
    to_f32<<<ceil_div(S.nnz, 256), 256, 0, s>>>(S.nnz, S.val.p, S.val32.p);
    TPT_CHECK_LAUNCH();
  }
  W.f32.setup((int)S.n_free, S.row_ptr.p, S.col.p, S.val32.p, S.nnz, s, batch);
  TPT_CUDA(cudaMemsetAsync(S.ctx->d_flag, 0, sizeof(int), s));
  jacobi_diag<float><<<ceil_div(S.n_free, 256), 256, 0, s>>>((int)S.n_free, S.row_ptr.p, S.col.p, S.val.p,
                                                             W.f32.dinv.p, S.ctx->d_flag);
  TPT_CHECK_LAUNCH();
  diag_check(S.ctx);
  W.f32_ready = true;
}

// ||b - A x||^2 in FP64 into W.sc[1]; r into W.res.  Returns the value.
double true_residual2(SystemData& S, const double* x) {
  SolverWork& W = *S.work;
  cudaStream_t s = S.ctx->stream;
  int lanes = pick_lanes(S.n_free, S.nnz);
  int grid = std::max(1, std::min(sm_count() * 8, ceil_div(S.n_free * lanes, SPMV_THREADS)));
  launch_residual(lanes, grid, s, (int)S.n_free, S.row_ptr.p, S.col.p, S.val.p, x, S.fred.p, W.res.p, W.sc.p + 1,
                  W.tk.p + 1, W.partials.p);
  double h;
  TPT_CUDA(cudaMemcpyAsync(&h, W.sc.p + 1, sizeof(double), cudaMemcpyDeviceToHost, s));
  TPT_CUDA(cudaStreamSynchronize(s));
  return h;
}

double norm2_b(SystemData& S) {
  SolverWork& W = *S.work;
  cudaStream_t s = S.ctx->stream;
  int grid = std::max(1, std::min(sm_count() * 4, ceil_div(S.n_free, VEC_THREADS)));
  sumsq_kernel<<<grid, VEC_THREADS, 0, s>>>((int)S.n_free, S.fred.p, W.sc.p, W.tk.p, W.partials.p);
  TPT_CHECK_LAUNCH();
  double h;
  TPT_CUDA(cudaMemcpyAsync(&h, W.sc.p, sizeof(double), cudaMemcpyDeviceToHost, s));
  TPT_CUDA(cudaStreamSynchronize(s));
  return h;
}

__global__ void axpy_f64(int n, const double* __restrict__ d, double* __restrict__ x) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] += d[i];
}

}  // namespace

void system_solve(SystemData& S, const tptfem_solver_opts& o, tptfem_solve_stats& st) {
  tptfem_context* ctx = S.ctx;
  cudaStream_t s = ctx->stream;
  const double tol = o.rel_tol > 0 ? o.rel_tol : 1e-10;
  const int64_t max_it = o.max_iter > 0 ? o.max_iter : 100000;
  const int max_outer = o.max_outer > 0 ? o.max_outer : 50;
  const double inner_tol = o.inner_rel_tol > 0 ? o.inner_rel_tol : 1e-4;
  int batch = o.batch > 0 ? o.batch : 32;
  batch += batch & 1;
  st = tptfem_solve_stats{};
  st.solver_used = o.solver;
  TPT_REQUIRE(o.solver == TPTFEM_SOLVER_JACOBI_PCG || o.solver == TPTFEM_SOLVER_MP_PCG, TPTFEM_ERR_INVALID_ARG,
              "unknown solver");
  if (S.n_free == 0) {
    st.rel_residual = 0.0;
    return;
  }
  ensure_work(S);
  SolverWork& W = *S.work;
  TPT_CUDA(cudaEventRecord(ctx->ev[0], s));
  if (o.solver == TPTFEM_SOLVER_JACOBI_PCG) prepare_f64(S, batch);
  else prepare_f32(S, batch);
  TPT_CUDA(cudaEventRecord(ctx->ev[1], s));
  const double bb = norm2_b(S);
  const double bnorm = std::sqrt(bb);
  S.x.zero();
  if (bb == 0.0) {
    st.rel_residual = 0.0;
    TPT_CUDA(cudaEventRecord(ctx->ev[2], s));
  } else if (o.solver == TPTFEM_SOLVER_JACOBI_PCG) {
    // FP64 PCG; if the recursive residual drifted from the true one, restart
    // from the current iterate on the true residual.
    Pcg<double>& P = W.f64;
    int64_t total = 0;
    double rel = 1.0;
    for (int restart = 0; restart < max_outer; ++restart) {
      double r2 = true_residual2(S, S.x.p);
      rel = std::sqrt(r2) / bnorm;
      if (rel <= tol || total >= max_it) break;
      TPT_CUDA(cudaMemcpyAsync(P.b.p, W.res.p, S.n_free * sizeof(double), cudaMemcpyDeviceToDevice, s));
      // stop the inner run a little below the target so the true residual passes
      double inner = std::min(0.5, 0.5 * tol / rel);
      PcgState fin = P.run(inner, (int)std::min<int64_t>(max_it - total, 1 << 30), s, W.h_state);
      total += fin.iters;
      axpy_f64<<<ceil_div(S.n_free, 256), 256, 0, s>>>((int)S.n_free, P.x.p, S.x.p);
      TPT_CHECK_LAUNCH();
      st.outer_steps += 1;
      if (fin.done == 2) {
        st.iterations = total;
        TPT_REQUIRE(false, TPTFEM_ERR_BREAKDOWN, "PCG breakdown: p.Ap <= 0 or NaN (matrix not SPD?)");
      }
    }
    rel = std::sqrt(true_residual2(S, S.x.p)) / bnorm;
    st.iterations = total;
    st.rel_residual = rel;
    TPT_CUDA(cudaEventRecord(ctx->ev[2], s));
    TPT_REQUIRE(rel <= tol, TPTFEM_ERR_NOT_CONVERGED, "PCG did not reach the requested residual");
  } else {
    // Mixed precision: FP32 Jacobi-PCG inner solves, FP64 refinement.
    Pcg<float>& P = W.f32;
    int64_t total = 0;
    double rel = 1.0;
    for (int outer = 0; outer < max_outer; ++outer) {
      double r2 = true_residual2(S, S.x.p);
      rel = std::sqrt(r2) / bnorm;
      if (rel <= tol || total >= max_it) break;
      to_f32<<<ceil_div(S.n_free, 256), 256, 0, s>>>(S.n_free, W.res.p, P.b.p);
      TPT_CHECK_LAUNCH();
      double inner = std::max(inner_tol, 0.5 * tol / rel);
      PcgState fin = P.run(inner, (int)std::min<int64_t>(max_it - total, 1 << 30), s, W.h_state);
      total += fin.iters;
      add_f32_to_f64<<<ceil_div(S.n_free, 256), 256, 0, s>>>((int)S.n_free, P.x.p, S.x.p);
      TPT_CHECK_LAUNCH();
      st.outer_steps += 1;
      if (fin.done == 2) {
        st.iterations = total;
        TPT_REQUIRE(false, TPTFEM_ERR_BREAKDOWN, "inner PCG breakdown: p.Ap <= 0 or NaN");
      }
    }
    rel = std::sqrt(true_residual2(S, S.x.p)) / bnorm;
    st.iterations = total;
    st.rel_residual = rel;
    TPT_CUDA(cudaEventRecord(ctx->ev[2], s));
    TPT_REQUIRE(rel <= tol, TPTFEM_ERR_NOT_CONVERGED, "mixed-precision PCG did not reach the requested residual");
  }
  TPT_CUDA(cudaEventSynchronize(ctx->ev[2]));
  float ms0 = 0.f, ms1 = 0.f;
  TPT_CUDA(cudaEventElapsedTime(&ms0, ctx->ev[0], ctx->ev[1]));
  TPT_CUDA(cudaEventElapsedTime(&ms1, ctx->ev[1], ctx->ev[2]));
  st.setup_ms = ms0;
  st.solve_ms = ms1;
}

void csr_matvec_f64(tptfem_context* ctx, int64_t nrows, const int* rp, const int* ci, const double* va,
                    const double* x, double* y) {
  if (nrows == 0) return;
  int64_t nnz_guess = nrows * 8;
  int lanes = pick_lanes(nrows, nnz_guess);
  int grid = std::max(1, std::min(sm_count() * 8, ceil_div(nrows * lanes, SPMV_THREADS)));
  launch_spmv<double, false>(lanes, grid, ctx->stream, (int)nrows, rp, ci, va, x, y, nullptr, nullptr);
}

}  // namespace tptfem
