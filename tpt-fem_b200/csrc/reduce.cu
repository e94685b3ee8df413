// reduce.cu -- Dirichlet condensation on the device.
//
// Restates reduce_system / solve_with_dirichlet
// (crates/tpt-fem-assembly/src/lib.rs:504-559):
//   * free dofs ascending; reduced index = rank among free dofs;
//   * kred keeps the free x free entries of each free row in column order
//     (the reference re-sorts them with a second to_csr, which leaves that
//     order unchanged);
//   * fred[i] = rhs[f] - sum over fixed columns (in column order) of v * val,
//     where val is the FIRST bcs entry naming that column (assembly:525);
//   * the returned solution overwrites fixed dofs with the LAST bcs entry
//     (assembly:555-557).
// fred uses explicit round-to-nearest multiply and subtract so no FMA is
// contracted, matching the reference bit for bit.
#include <climits>

#include "objects.hpp"

namespace tptfem {

namespace {

__global__ void init_first_last(int64_t n, int* __restrict__ first, int* __restrict__ last) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    first[i] = INT_MAX;
    last[i] = -1;
  }
}

__global__ void bc_first_last(const int* __restrict__ dof, int64_t nbc, int* __restrict__ first,
                              int* __restrict__ last) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nbc) return;
  atomicMin(&first[dof[i]], (int)i);
  atomicMax(&last[dof[i]], (int)i);
}

__global__ void free_flags(const int* __restrict__ first, int64_t n, int* __restrict__ is_free) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) is_free[i] = first[i] == INT_MAX;
}

__global__ void free_lists(const int* __restrict__ first, const int* __restrict__ red, int64_t n,
                           int* __restrict__ free_map) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && first[i] == INT_MAX) free_map[red[i]] = (int)i;
}

__global__ void reduced_counts(const int* __restrict__ rp, const int* __restrict__ ci,
                               const int* __restrict__ first, const int* __restrict__ free_map, int64_t n_free,
                               int* __restrict__ cnt) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_free) return;
  int f = free_map[i], c = 0;
  for (int k = rp[f]; k < rp[f + 1]; ++k) c += first[ci[k]] == INT_MAX;
  cnt[i] = c;
}

// One warp per free row: lanes take 32 consecutive entries at a time; kept
// (free-column) entries are placed by a ballot prefix count, and the lifting
// terms of fixed columns are subtracted one by one in column order, as the
// reference's loop does.
__global__ void reduced_fill(const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ va,
                             const int* __restrict__ first, const int* __restrict__ red,
                             const int* __restrict__ free_map, const double* __restrict__ bc_val,
                             const double* __restrict__ rhs, int64_t n_free, const int* __restrict__ rrp,
                             int* __restrict__ rci, double* __restrict__ rva, double* __restrict__ fred) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= n_free) return;  // whole warps leave together
  const int f = free_map[i];
  double r = rhs[f];
  int o = rrp[i];
  const int k1 = rp[f + 1];
  for (int k0 = rp[f]; k0 < k1; k0 += 32) {
    const int k = k0 + lane;
    const bool in = k < k1;
    const int col = in ? ci[k] : 0;
    const double v = in ? va[k] : 0.0;
    const int fb = in ? first[col] : INT_MAX;
    const bool fixed = in && fb != INT_MAX, kept = in && fb == INT_MAX;
    const unsigned km = __ballot_sync(0xffffffffu, kept);
    if (kept) {
      const int pos = o + __popc(km & ((1u << lane) - 1u));
      rci[pos] = red[col];
      rva[pos] = v;
    }
    o += __popc(km);
    unsigned fm = __ballot_sync(0xffffffffu, fixed);
    const double prod = fixed ? __dmul_rn(v, bc_val[fb]) : 0.0;
    while (fm) {
      const int src = __ffs(fm) - 1;
      r = __dsub_rn(r, __shfl_sync(0xffffffffu, prod, src));
      fm &= fm - 1;
    }
  }
  if (lane == 0) fred[i] = r;
}

// Values of an existing reduced system from a matrix with the same pattern:
// flags any column that differs from the system's.
__global__ void reduced_refill(const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ va,
                               const int* __restrict__ first, const int* __restrict__ red,
                               const int* __restrict__ free_map, const double* __restrict__ bc_val,
                               const double* __restrict__ rhs, int64_t n_free, const int* __restrict__ rrp,
                               const int* __restrict__ rci, double* __restrict__ rva, double* __restrict__ fred,
                               int* __restrict__ flag) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_free) return;
  int f = free_map[i];
  double r = rhs[f];
  int o = rrp[i];
  const int oe = rrp[i + 1];
  for (int k = rp[f]; k < rp[f + 1]; ++k) {
    int col = ci[k];
    double v = va[k];
    int fb = first[col];
    if (fb != INT_MAX) {
      r = __dsub_rn(r, __dmul_rn(v, bc_val[fb]));
    } else {
      if (o >= oe || rci[o] != red[col]) { atomicOr(flag, 1); return; }
      rva[o] = v;
      ++o;
    }
  }
  if (o != oe) atomicOr(flag, 1);
  fred[i] = r;
}

__global__ void reduced_index(const int* __restrict__ first, const int* __restrict__ red, int64_t n,
                              int* __restrict__ red_map) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) red_map[i] = first[i] == INT_MAX ? red[i] : -1;
}

__global__ void fixed_values(const int* __restrict__ last, const double* __restrict__ bc_val, int64_t n,
                             double* __restrict__ u_fixed) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) u_fixed[i] = last[i] >= 0 ? bc_val[last[i]] : 0.0;
}

__global__ void scatter_solution(const double* __restrict__ x, const int* __restrict__ free_map, int64_t n_free,
                                 double* __restrict__ u) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_free) u[free_map[i]] = x[i];
}

}  // namespace

std::unique_ptr<SystemData> reduce_system(tptfem_context* ctx, const MatrixData& A, const double* d_rhs,
                                          const int64_t* bc_dof, const double* bc_val, int64_t nbc) {
  cudaStream_t s = ctx->stream;
  const int64_t n = A.nrows;
  TPT_REQUIRE(nbc >= 0 && nbc < (1LL << 31), TPTFEM_ERR_INVALID_ARG, "bad number of boundary conditions");
  std::vector<int> hdof(nbc);
  for (int64_t i = 0; i < nbc; ++i) {
    TPT_REQUIRE(bc_dof[i] >= 0 && bc_dof[i] < n, TPTFEM_ERR_INVALID_ARG, "boundary-condition dof out of range");
    hdof[i] = (int)bc_dof[i];
  }
  auto S = std::make_unique<SystemData>();
  S->ctx = ctx;
  S->n = n;
  S->dpn = A.dpn;
  S->mesh = A.mesh;
  DevBuf<int> dof, first, last, red, cnt;
  DevBuf<double> val;
  dof.alloc(nbc, s);
  dof.upload(hdof.data(), nbc);
  val.alloc(nbc, s);
  val.upload(bc_val, nbc);
  first.alloc(n, s);
  last.alloc(n, s);
  init_first_last<<<ceil_div(n, 256), 256, 0, s>>>(n, first.p, last.p);
  TPT_CHECK_LAUNCH();
  if (nbc) {
    bc_first_last<<<ceil_div(nbc, 256), 256, 0, s>>>(dof.p, nbc, first.p, last.p);
    TPT_CHECK_LAUNCH();
  }
  red.alloc(n + 1, s);
  cnt.alloc(n, s);
  free_flags<<<ceil_div(n, 256), 256, 0, s>>>(first.p, n, cnt.p);
  TPT_CHECK_LAUNCH();
  S->n_free = exclusive_scan_i32(cnt.p, red.p, n, s);
  S->free_map.alloc(S->n_free, s);
  free_lists<<<ceil_div(n, 256), 256, 0, s>>>(first.p, red.p, n, S->free_map.p);
  TPT_CHECK_LAUNCH();
  S->red_map.alloc(n, s);
  reduced_index<<<ceil_div(n, 256), 256, 0, s>>>(first.p, red.p, n, S->red_map.p);
  TPT_CHECK_LAUNCH();
  DevBuf<int> rcnt;
  rcnt.alloc(S->n_free + 1, s);
  S->row_ptr.alloc(S->n_free + 1, s);
  if (S->n_free) {
    reduced_counts<<<ceil_div(S->n_free, 256), 256, 0, s>>>(A.row_ptr.p, A.col.p, first.p, S->free_map.p,
                                                            S->n_free, rcnt.p);
    TPT_CHECK_LAUNCH();
  }
  S->nnz = exclusive_scan_i32(rcnt.p, S->row_ptr.p, S->n_free, s);
  S->col.alloc(S->nnz, s);
  S->val.alloc(S->nnz, s);
  S->fred.alloc(S->n_free, s);
  if (S->n_free) {
    reduced_fill<<<ceil_div(S->n_free * 32, 256), 256, 0, s>>>(A.row_ptr.p, A.col.p, A.val.p, first.p, red.p,
                                                          S->free_map.p, val.p, d_rhs, S->n_free, S->row_ptr.p,
                                                          S->col.p, S->val.p, S->fred.p);
    TPT_CHECK_LAUNCH();
  }
  S->u_fixed.alloc(n, s);
  fixed_values<<<ceil_div(n, 256), 256, 0, s>>>(last.p, val.p, n, S->u_fixed.p);
  TPT_CHECK_LAUNCH();
  S->x.alloc(S->n_free, s);
  S->x.zero();
  S->bc_first = std::move(first);
  S->red_rank = std::move(red);
  S->bc_vals = std::move(val);
  TPT_CUDA(cudaStreamSynchronize(s));
  return S;
}

bool system_refresh(SystemData& S, const MatrixData& A, const double* d_rhs) {
  cudaStream_t s = S.ctx->stream;
  TPT_REQUIRE(A.nrows == S.n && A.dpn == S.dpn, TPTFEM_ERR_INVALID_ARG,
              "refresh: the matrix does not match the system's size");
  TPT_CUDA(cudaMemsetAsync(S.ctx->d_flag, 0, sizeof(int), s));
  if (S.n_free) {
    reduced_refill<<<ceil_div(S.n_free, 256), 256, 0, s>>>(A.row_ptr.p, A.col.p, A.val.p, S.bc_first.p,
                                                           S.red_rank.p, S.free_map.p, S.bc_vals.p, d_rhs, S.n_free,
                                                           S.row_ptr.p, S.col.p, S.val.p, S.fred.p, S.ctx->d_flag);
    TPT_CHECK_LAUNCH();
  }
  int flag = 0;
  TPT_CUDA(cudaMemcpyAsync(&flag, S.ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
  TPT_CUDA(cudaStreamSynchronize(s));
  return flag == 0;
}

void system_solution(const SystemData& S, double* d_u) {
  cudaStream_t s = S.ctx->stream;
  TPT_CUDA(cudaMemcpyAsync(d_u, S.u_fixed.p, S.n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  if (S.n_free) {
    scatter_solution<<<ceil_div(S.n_free, 256), 256, 0, s>>>(S.x.p, S.free_map.p, S.n_free, d_u);
    TPT_CHECK_LAUNCH();
  }
}

}  // namespace tptfem
