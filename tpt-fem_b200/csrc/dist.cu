// dist.cu -- row-partitioned FP64 PCG over several ranks (one per GPU).
//
// The reduced system is split into contiguous, node-aligned row ranges (the
// x-slabs of a box mesh, whose nodes are numbered x-major).  Rank k keeps its
// rows with the columns renumbered: owned columns first (0..nloc), then the
// ghost columns it reads from other ranks, sorted by global index, so the
// ghosts of each peer form one contiguous run.  One PCG iteration needs one
// exchange of p's ghost values and two all-reduces:
//   pack p -> send | exchange | q = A_loc p, p.q | sum | x, r, z update, r.r, r.z | sum | p = z + beta p
// This file does each rank's device work (C ABI tptfem_dist_*); the exchange
// and the sums belong to the caller (NCCL over torch.distributed for ranks on
// different GPUs), or to tptfem_dist_solve_local, which runs several ranks on
// one device in lock step with device copies as the exchange.  Partial sums
// are per-block values added in a fixed order, so results are reproducible.
//
// Preconditioners: Jacobi (the plain method), or, after dist_set_precond, the
// two-level method of the one-GPU solver in partitioned form:
//   M^-1 = blockdiag_k(G_k^T G_k) + P A_c^-1 P^T
// G_k is the FSAI factor (classic, or the attached network's values) of rank
// k's owned diagonal block, so applying it needs no exchange.  P is the
// aggregation coarse space of the whole system (every rank builds the same
// aggregates from the mesh geometry); rank k forms P_k^T A_k P from its own
// rows, the caller sums these partial coarse matrices over the ranks once
// (an all-reduce of nc x nc values) and every rank factors the sum.  Each
// iteration then adds one all-reduce of the nc restriction values P_k^T r_k:
//   ... | x, r update, r.r, P_k^T r_k | sum r.r; sum P^T r | z = M r, r.z | sum | p = z + beta p
//
// Reliable updates, as in the one-GPU solver: the steps accumulate in xl,
// apart from x, and whenever the recursive r.r has dropped by 1e-12 since the
// last replacement (and before the solve may stop) x += xl and the true
// residual b - A x, summed with compensation, replaces the recursive one; x's
// ghost values travel through the same pack + exchange as p's.
#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include <cuda_fp16.h>

#include "modes.cuh"
#include "objects.hpp"

namespace tptfem {

namespace {

constexpr int DT_THREADS = 256, DT_LPR = 8;
// reliable updates: the true residual replaces the recursive one whenever the
// latter has dropped by this factor, and before the solve may stop
constexpr double DIST_DELTA = 1e-6;

// q = A_loc p on the owned rows (DT_LPR lanes per row), per-block p.q partials.
__global__ void __launch_bounds__(DT_THREADS) dist_spmv_dot(int64_t nloc, const int* __restrict__ rp,
                                                            const int* __restrict__ ci,
                                                            const double* __restrict__ va,
                                                            const double* __restrict__ p, double* __restrict__ q,
                                                            double* __restrict__ part) {
  __shared__ double sh[DT_THREADS / DT_LPR];
  const int64_t t = (int64_t)blockIdx.x * DT_THREADS + threadIdx.x;
  const int64_t i = t / DT_LPR;
  const int l = (int)(t % DT_LPR);
  double s = 0.0;
  if (i < nloc)
    for (int k = rp[i] + l; k < rp[i + 1]; k += DT_LPR) s += va[k] * p[ci[k]];
  const unsigned m = 0xffffffffu;
  for (int o = DT_LPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(m, s, o, DT_LPR);
  double d = 0.0;
  if (i < nloc && l == 0) {
    q[i] = s;
    d = p[i] * s;
  }
  if (l == 0) sh[threadIdx.x / DT_LPR] = d;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0;
    for (int w = 0; w < DT_THREADS / DT_LPR; ++w) a += sh[w];
    part[blockIdx.x] = a;
  }
}

// x += a p, r -= a q, with Jacobi z = dinv r; per-block partials of r.r and r.z
// (r.z 0 without Jacobi: the block preconditioner forms z afterwards).
__global__ void __launch_bounds__(DT_THREADS) dist_update(int64_t nloc, double a, double* __restrict__ x,
                                                          double* __restrict__ r, double* __restrict__ z,
                                                          const double* __restrict__ p,
                                                          const double* __restrict__ q,
                                                          const double* __restrict__ dinv,
                                                          double* __restrict__ part, bool jacobi) {
  __shared__ double s1[DT_THREADS], s2[DT_THREADS];
  const int64_t i = (int64_t)blockIdx.x * DT_THREADS + threadIdx.x;
  double rr = 0.0, rz = 0.0;
  if (i < nloc) {
    x[i] += a * p[i];
    const double ri = r[i] - a * q[i];
    r[i] = ri;
    rr = ri * ri;
    if (jacobi) {
      const double zi = dinv[i] * ri;
      z[i] = zi;
      rz = ri * zi;
    }
  }
  s1[threadIdx.x] = rr;
  s2[threadIdx.x] = rz;
  __syncthreads();
  for (int o = DT_THREADS / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      s1[threadIdx.x] += s1[threadIdx.x + o];
      s2[threadIdx.x] += s2[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = s1[0];
    part[2 * blockIdx.x + 1] = s2[0];
  }
}

// r = b - A x with compensated (double-double) accumulation, so that r is the
// residual of the FP64 x rather than a sum whose cancellation noise can exceed
// a 1e-10 target; with Jacobi z = dinv r.  Per-block partials of r.r and r.z.
__global__ void __launch_bounds__(DT_THREADS) dist_true_residual(int64_t nloc, const int* __restrict__ rp,
                                                                 const int* __restrict__ ci,
                                                                 const double* __restrict__ va,
                                                                 const double* __restrict__ x,
                                                                 const double* __restrict__ b,
                                                                 double* __restrict__ r, double* __restrict__ z,
                                                                 const double* __restrict__ dinv,
                                                                 double* __restrict__ part, bool jacobi) {
  __shared__ double s1[DT_THREADS / DT_LPR], s2[DT_THREADS / DT_LPR];
  const int64_t t = (int64_t)blockIdx.x * DT_THREADS + threadIdx.x;
  const int64_t i = t / DT_LPR;
  const int l = (int)(t % DT_LPR);
  double hi = 0.0, lo = 0.0;
  if (i < nloc)
    for (int k = rp[i] + l; k < rp[i + 1]; k += DT_LPR) {
      double p, pe, s, se;
      two_prod(va[k], x[ci[k]], p, pe);
      two_sum(hi, p, s, se);
      hi = s;
      lo += pe + se;
    }
  for (int o = DT_LPR / 2; o > 0; o >>= 1) {
    const double oh = __shfl_xor_sync(0xffffffffu, hi, o, DT_LPR);
    const double ol = __shfl_xor_sync(0xffffffffu, lo, o, DT_LPR);
    double s, se;
    two_sum(hi, oh, s, se);
    hi = s;
    lo += ol + se;
  }
  double rr = 0.0, rz = 0.0;
  if (i < nloc && l == 0) {
    double r1, e1;
    two_sum(b[i], -hi, r1, e1);
    const double ri = r1 + (e1 - lo);
    r[i] = ri;
    rr = ri * ri;
    if (jacobi) {
      const double zi = dinv[i] * ri;
      z[i] = zi;
      rz = ri * zi;
    }
  }
  if (l == 0) {
    s1[threadIdx.x / DT_LPR] = rr;
    s2[threadIdx.x / DT_LPR] = rz;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a1 = 0.0, a2 = 0.0;
    for (int w = 0; w < DT_THREADS / DT_LPR; ++w) {
      a1 += s1[w];
      a2 += s2[w];
    }
    part[2 * blockIdx.x] = a1;
    part[2 * blockIdx.x + 1] = a2;
  }
}

// Block FSAI, first half: t = sigma^2 (r + L r) (DT_LPR lanes per row).
__global__ void __launch_bounds__(DT_THREADS) dist_fsai_lower(int64_t n, const int* __restrict__ rp,
                                                              const int* __restrict__ ci,
                                                              const __half* __restrict__ va,
                                                              const float* __restrict__ sig2,
                                                              const double* __restrict__ r, double* __restrict__ t) {
  const int64_t tid = (int64_t)blockIdx.x * DT_THREADS + threadIdx.x;
  const int64_t i = tid / DT_LPR;
  const int l = (int)(tid % DT_LPR);
  double s = 0.0;
  if (i < n)
    for (int k = rp[i] + l; k < rp[i + 1]; k += DT_LPR) s += (double)__half2float(va[k]) * r[ci[k]];
  for (int o = DT_LPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, DT_LPR);
  if (i < n && l == 0) t[i] = (double)sig2[i] * (r[i] + s);
}

// Second half: z = t + L^T t, plus the coarse correction P (A_c^-1 P^T r) on
// the owned groups when cm is given (raw-mode coefficients per aggregate);
// per-block partials of r.z.
template <int DPN>
__global__ void __launch_bounds__(DT_THREADS) dist_fsai_upper(int64_t n, const int* __restrict__ trp,
                                                              const int* __restrict__ tci,
                                                              const __half* __restrict__ tva,
                                                              const double* __restrict__ t,
                                                              const double* __restrict__ r, double* __restrict__ z,
                                                              int64_t r0, const int* __restrict__ agg,
                                                              const float* __restrict__ y,
                                                              const double* __restrict__ cm,
                                                              double* __restrict__ part) {
  constexpr int NM = rigid_modes(DPN);
  __shared__ double sh[DT_THREADS / DT_LPR];
  const int64_t tid = (int64_t)blockIdx.x * DT_THREADS + threadIdx.x;
  const int64_t i = tid / DT_LPR;
  const int l = (int)(tid % DT_LPR);
  double s = 0.0;
  if (i < n)
    for (int k = trp[i] + l; k < trp[i + 1]; k += DT_LPR) s += (double)__half2float(tva[k]) * t[tci[k]];
  for (int o = DT_LPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, DT_LPR);
  double d = 0.0;
  if (i < n && l == 0) {
    double zi = t[i] + s;
    if (cm) {
      const int64_t gi = r0 + i, g = gi / DPN;
      const int a = (int)(gi - g * DPN);
      double R[DPN][NM];
      mode_rows<DPN>(y + 3 * g, R);
      const double* c = cm + (int64_t)agg[g] * NM;
      double pc = 0.0;
#pragma unroll
      for (int k = 0; k < NM; ++k) pc += R[a][k] * c[k];
      zi += pc;
    }
    z[i] = zi;
    d = r[i] * zi;
  }
  if (l == 0) sh[threadIdx.x / DT_LPR] = d;
  __syncthreads();
  if (threadIdx.x == 0) {
    double acc = 0.0;
    for (int w = 0; w < DT_THREADS / DT_LPR; ++w) acc += sh[w];
    part[blockIdx.x] = acc;
  }
}

// The owned diagonal block of the local rows: per row the count of owned
// columns (< nloc), then those entries in row order.
__global__ void dist_block_count(int64_t nloc, const int* __restrict__ rp, const int* __restrict__ ci,
                                 int* __restrict__ cnt) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nloc) return;
  int c = 0;
  for (int k = rp[i]; k < rp[i + 1]; ++k) c += ci[k] < nloc;
  cnt[i] = c;
}

__global__ void dist_block_fill(int64_t nloc, const int* __restrict__ rp, const int* __restrict__ ci,
                                const double* __restrict__ va, const int* __restrict__ brp, int* __restrict__ bci,
                                double* __restrict__ bva) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nloc) return;
  int o = brp[i];
  for (int k = rp[i]; k < rp[i + 1]; ++k)
    if (ci[k] < nloc) {
      bci[o] = ci[k];
      bva[o] = va[k];
      ++o;
    }
}

// full dof -> block row (-1 outside the owned range [r0, r1) of reduced rows)
__global__ void dist_block_red_map(int64_t n, const int* __restrict__ red, int64_t r0, int64_t r1,
                                   int* __restrict__ out) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int v = red[j];
  out[j] = (v >= r0 && v < r1) ? (int)(v - r0) : -1;
}

__global__ void dist_add(int64_t n, const double* __restrict__ a, double* __restrict__ acc) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) acc[i] += a[i];
}

__global__ void dist_add_clear(int64_t nloc, double* __restrict__ xl, double* __restrict__ x) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nloc) {
    x[i] += xl[i];
    xl[i] = 0.0;
  }
}

__global__ void dist_direction(int64_t nloc, double beta, const double* __restrict__ z, double* __restrict__ p) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nloc) p[i] = z[i] + beta * p[i];
}

__global__ void dist_pack(int64_t ns, const int* __restrict__ idx, const double* __restrict__ p,
                          double* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ns) out[i] = p[idx[i]];
}

__global__ void dist_diag(int64_t nloc, const int* __restrict__ rp, const int* __restrict__ ci,
                          const double* __restrict__ va, double* __restrict__ dinv, int* __restrict__ flag) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nloc) return;
  double d = 0.0;
  for (int k = rp[i]; k < rp[i + 1]; ++k)
    if (ci[k] == i) d = va[k];
  if (!(d > 0.0)) atomicOr(flag, 1);
  dinv[i] = d > 0.0 ? 1.0 / d : 0.0;
}

}  // namespace

double DistData::sum_parts(int nb, int stride, int which) {
  TPT_CUDA(cudaMemcpyAsync(hpart.data(), part.p, (size_t)nb * stride * sizeof(double), cudaMemcpyDeviceToHost,
                           ctx->stream));
  TPT_CUDA(cudaStreamSynchronize(ctx->stream));
  double s = 0.0;
  for (int b = 0; b < nb; ++b) s += hpart[(size_t)b * stride + which];
  return s;
}

std::unique_ptr<DistData> dist_create(tptfem_context* ctx, SystemData& S, int rank, int size,
                                      const int64_t* row_starts) {
  TPT_REQUIRE(size >= 1 && rank >= 0 && rank < size, TPTFEM_ERR_INVALID_ARG, "bad rank / size");
  TPT_REQUIRE(row_starts[0] == 0 && row_starts[size] == S.n_free, TPTFEM_ERR_INVALID_ARG,
              "row_starts must run from 0 to the number of free dofs");
  for (int k = 0; k < size; ++k)
    TPT_REQUIRE(row_starts[k] <= row_starts[k + 1], TPTFEM_ERR_INVALID_ARG, "row_starts must be ascending");
  cudaStream_t s = ctx->stream;
  auto D = std::make_unique<DistData>();
  D->ctx = ctx;
  D->rank = rank;
  D->size = size;
  D->r0 = row_starts[rank];
  D->r1 = row_starts[rank + 1];
  D->nloc = D->r1 - D->r0;
  const int64_t n = S.n_free;
  // structure on the host, once: the whole pattern (every rank needs its
  // peers' ghost lists to know what to send)
  std::vector<int> hrp(n + 1), hci(S.nnz);
  S.row_ptr.download(hrp.data(), n + 1);
  S.col.download(hci.data(), S.nnz);
  TPT_CUDA(cudaStreamSynchronize(s));
  auto owner = [&](int64_t c) {
    return (int)(std::upper_bound(row_starts, row_starts + size + 1, c) - row_starts - 1);
  };
  // ghosts of this rank: columns of its rows outside [r0, r1), sorted unique
  std::vector<int> ghosts;
  for (int64_t row = D->r0; row < D->r1; ++row)
    for (int k = hrp[row]; k < hrp[row + 1]; ++k)
      if (hci[k] < D->r0 || hci[k] >= D->r1) ghosts.push_back(hci[k]);
  std::sort(ghosts.begin(), ghosts.end());
  ghosts.erase(std::unique(ghosts.begin(), ghosts.end()), ghosts.end());
  D->nghost = (int64_t)ghosts.size();
  D->sys = &S;
  D->recv_off.assign(size + 1, 0);
  for (int g : ghosts) D->recv_off[owner(g) + 1]++;
  for (int k = 0; k < size; ++k) D->recv_off[k + 1] += D->recv_off[k];
  // local CSR with renumbered columns
  const int64_t k0 = hrp[D->r0], k1 = hrp[D->r1], nnzl = k1 - k0;
  std::vector<int> lrp(D->nloc + 1), lci(nnzl);
  for (int64_t row = D->r0; row <= D->r1; ++row) lrp[row - D->r0] = (int)(hrp[row] - k0);
  for (int64_t k = k0; k < k1; ++k) {
    const int c = hci[k];
    lci[k - k0] = (c >= D->r0 && c < D->r1)
                      ? (int)(c - D->r0)
                      : (int)(D->nloc + (std::lower_bound(ghosts.begin(), ghosts.end(), c) - ghosts.begin()));
  }
  // send lists: for each peer q, the owned rows q reads, ascending (q's ghost order)
  std::vector<int> sidx;
  D->send_off.assign(size + 1, 0);
  for (int qr = 0; qr < size; ++qr) {
    std::vector<int> need;
    if (qr != rank)
      for (int64_t row = row_starts[qr]; row < row_starts[qr + 1]; ++row)
        for (int k = hrp[row]; k < hrp[row + 1]; ++k)
          if (hci[k] >= D->r0 && hci[k] < D->r1) need.push_back(hci[k]);
    std::sort(need.begin(), need.end());
    need.erase(std::unique(need.begin(), need.end()), need.end());
    for (int c : need) sidx.push_back((int)(c - D->r0));
    D->send_off[qr + 1] = D->send_off[qr] + (int64_t)need.size();
  }
  D->ghost_cols = std::move(ghosts);
  D->rp.alloc(D->nloc + 1, s);
  D->rp.upload(lrp.data(), lrp.size());
  D->ci.alloc(std::max<int64_t>(nnzl, 1), s);
  D->ci.upload(lci.data(), nnzl);
  D->va.alloc(std::max<int64_t>(nnzl, 1), s);
  if (nnzl) TPT_CUDA(cudaMemcpyAsync(D->va.p, S.val.p + k0, nnzl * sizeof(double), cudaMemcpyDeviceToDevice, s));
  D->send_idx.alloc(std::max<size_t>(sidx.size(), 1), s);
  D->send_idx.upload(sidx.data(), sidx.size());
  D->send_buf.alloc(std::max<size_t>(sidx.size(), 1), s);
  const int64_t nl = std::max<int64_t>(D->nloc, 1);
  D->b.alloc(nl, s);
  if (D->nloc)
    TPT_CUDA(cudaMemcpyAsync(D->b.p, S.fred.p + D->r0, D->nloc * sizeof(double), cudaMemcpyDeviceToDevice, s));
  D->dinv.alloc(nl, s);
  D->x.alloc(nl, s);
  D->xl.alloc(nl, s);
  D->r.alloc(nl, s);
  D->z.alloc(nl, s);
  D->q.alloc(nl, s);
  D->p.alloc(D->nloc + D->nghost + 1, s);
  D->blocks_spmv = std::max(1, ceil_div(D->nloc * DT_LPR, DT_THREADS));
  D->blocks_vec = std::max(1, ceil_div(D->nloc, DT_THREADS));
  D->part.alloc(2 * (size_t)std::max(D->blocks_spmv, D->blocks_vec), s);
  D->hpart.resize(2 * (size_t)std::max(D->blocks_spmv, D->blocks_vec));
  TPT_CUDA(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), s));
  if (D->nloc) {
    dist_diag<<<ceil_div(D->nloc, 256), 256, 0, s>>>(D->nloc, D->rp.p, D->ci.p, D->va.p, D->dinv.p, ctx->d_flag);
    TPT_CHECK_LAUNCH();
  }
  int flag = 0;
  TPT_CUDA(cudaMemcpyAsync(&flag, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
  TPT_CUDA(cudaStreamSynchronize(s));
  TPT_REQUIRE(flag == 0, TPTFEM_ERR_NUMERIC, "a diagonal entry is not positive");
  return D;
}

// x = 0, r = b; Jacobi: z = dinv r, p = z; partial r.r and r.z into out[0..1].
// With a block preconditioner: partial r.r and 0, the coarse restriction's
// partial in yc, p = 0 (the caller sets p = z after tptfem_dist_precondition).
void dist_start(DistData& D, double* out) {
  cudaStream_t s = D.ctx->stream;
  if (D.nloc) {
    TPT_CUDA(cudaMemsetAsync(D.x.p, 0, D.nloc * sizeof(double), s));
    TPT_CUDA(cudaMemsetAsync(D.xl.p, 0, D.nloc * sizeof(double), s));
    TPT_CUDA(cudaMemcpyAsync(D.r.p, D.b.p, D.nloc * sizeof(double), cudaMemcpyDeviceToDevice, s));
    TPT_CUDA(cudaMemsetAsync(D.q.p, 0, D.nloc * sizeof(double), s));
    TPT_CUDA(cudaMemsetAsync(D.p.p, 0, D.nloc * sizeof(double), s));
  }
  dist_update(D, 0.0, out);
  if (!D.pc) {
    dist_direction<<<D.blocks_vec, DT_THREADS, 0, s>>>(D.nloc, 0.0, D.z.p, D.p.p);
    TPT_CHECK_LAUNCH();
  }
}

void dist_pack(DistData& D) {
  const int64_t ns = D.send_off[D.size];
  if (ns) {
    dist_pack<<<ceil_div(ns, 256), 256, 0, D.ctx->stream>>>(ns, D.send_idx.p, D.p.p, D.send_buf.p);
    TPT_CHECK_LAUNCH();
  }
  TPT_CUDA(cudaStreamSynchronize(D.ctx->stream));  // the caller's exchange reads send_buf
}

double dist_spmv_dot(DistData& D) {
  dist_spmv_dot<<<D.blocks_spmv, DT_THREADS, 0, D.ctx->stream>>>(D.nloc, D.rp.p, D.ci.p, D.va.p, D.p.p, D.q.p,
                                                                 D.part.p);
  TPT_CHECK_LAUNCH();
  return D.sum_parts(D.blocks_spmv, 1, 0);
}

// The rank's coarse data index the whole system's aggregates: refuse to go on
// if that geometry was rebuilt (another aggregate count) since the set-up.
static void check_coarse(const DistData& D) {
  if (!D.nc) return;
  const CoarseSpace& C = D.sys->coarse;
  TPT_REQUIRE(C.state == 1 && C.generation == D.cgen && C.nc == D.nc, TPTFEM_ERR_INVALID_ARG,
              "the system's coarse space was rebuilt after tptfem_dist_set_precond");
}

void dist_update(DistData& D, double alpha, double* out) {
  check_coarse(D);
  cudaStream_t s = D.ctx->stream;
  dist_update<<<D.blocks_vec, DT_THREADS, 0, s>>>(D.nloc, alpha, D.xl.p, D.r.p, D.z.p, D.p.p, D.q.p, D.dinv.p,
                                                  D.part.p, D.pc == 0);
  TPT_CHECK_LAUNCH();
  if (D.nc) coarse_local_restrict(*D.sys, D.cl, D.r.p, D.yc.p, s);  // this rank's part of P^T r
  out[0] = D.sum_parts(D.blocks_vec, 2, 0);  // (synchronises: yc is ready for the caller's sum)
  out[1] = D.sum_parts(D.blocks_vec, 2, 1);
}

int dist_set_precond(DistData& D, SystemData& S, int kind, int aggregates) {
  TPT_REQUIRE(kind == 1 || kind == 2, TPTFEM_ERR_INVALID_ARG, "kind must be TPTFEM_DIST_PC_FSAI or _LEARNED");
  TPT_REQUIRE(D.sys == &S, TPTFEM_ERR_INVALID_ARG, "not the system this rank was created from");
  TPT_REQUIRE(D.pc == 0, TPTFEM_ERR_INVALID_ARG, "the rank's preconditioner is already set");
  cudaStream_t s = D.ctx->stream;
  const int64_t nl = std::max<int64_t>(D.nloc, 1);
  // the owned diagonal block as a system of its own: the local rows' entries
  // in owned columns (ascending in every row, as the global columns are)
  auto B = std::make_unique<SystemData>();
  B->ctx = D.ctx;
  B->mesh = S.mesh;
  B->lmodel = S.lmodel;
  B->n = S.n;
  B->n_free = D.nloc;
  B->dpn = S.dpn;
  B->free_map.alloc(nl, s);
  if (D.nloc)
    TPT_CUDA(cudaMemcpyAsync(B->free_map.p, S.free_map.p + D.r0, D.nloc * sizeof(int), cudaMemcpyDeviceToDevice, s));
  B->red_map.alloc(std::max<int64_t>(S.n, 1), s);
  dist_block_red_map<<<ceil_div(std::max<int64_t>(S.n, 1), 256), 256, 0, s>>>(S.n, S.red_map.p, D.r0, D.r1,
                                                                              B->red_map.p);
  TPT_CHECK_LAUNCH();
  DevBuf<int> cnt;
  cnt.alloc(nl + 1, s);
  B->row_ptr.alloc(D.nloc + 1, s);
  if (D.nloc) {
    dist_block_count<<<ceil_div(D.nloc, 256), 256, 0, s>>>(D.nloc, D.rp.p, D.ci.p, cnt.p);
    TPT_CHECK_LAUNCH();
  }
  B->nnz = exclusive_scan_i32(cnt.p, B->row_ptr.p, D.nloc, s);
  B->col.alloc(std::max<int64_t>(B->nnz, 1), s);
  B->val.alloc(std::max<int64_t>(B->nnz, 1), s);
  if (D.nloc) {
    dist_block_fill<<<ceil_div(D.nloc, 256), 256, 0, s>>>(D.nloc, D.rp.p, D.ci.p, D.va.p, B->row_ptr.p, B->col.p,
                                                           B->val.p);
    TPT_CHECK_LAUNCH();
  }
  if (D.nloc) {
    D.fac = system_block_factor(*B, kind == 2);
    TPT_REQUIRE(D.fac, TPTFEM_ERR_NUMERIC,
                "the block's FSAI factor could not be built (a pattern row too long or a non-positive pivot)");
  }
  D.blk = std::move(B);
  D.t.alloc(nl, s);
  D.pc = kind;
  D.nc = 0;
  D.coarse_ready = false;
  // the coarse space of the whole system (geometry on every rank), this rank's part of A_c
  if (aggregates >= 0 && nb_build_operator(S) &&
      coarse_build(S, aggregates > 0 ? aggregates : coarse_default_aggregates(S))) {
    const int dpn = S.dpn;
    TPT_REQUIRE(D.r0 % dpn == 0 && D.r1 % dpn == 0, TPTFEM_ERR_INVALID_ARG,
                "row ranges must hold whole node groups for the coarse space");
    coarse_local_build(S, D.r0 / dpn, D.r1 / dpn, D.cl);
    std::vector<int> gc(D.nloc + D.nghost);
    for (int64_t i = 0; i < D.nloc; ++i) gc[i] = (int)(D.r0 + i);
    for (int64_t k = 0; k < D.nghost; ++k) gc[D.nloc + k] = D.ghost_cols[k];
    D.gcol.alloc(std::max<size_t>(gc.size(), 1), s);
    D.gcol.upload(gc.data(), gc.size());
    const int nc = S.coarse.nc;
    D.ld = (nc + 3) & ~3;
    D.ac.alloc((size_t)nc * nc, s);
    D.yc.alloc(nc, s);
    D.uc.alloc(nc, s);
    D.cm.alloc(nc, s);
    D.ainv.alloc((size_t)nc * D.ld, s);
    coarse_local_matrix(S, D.cl, D.nloc, D.rp.p, D.ci.p, D.va.p, D.gcol.p, D.ac.p);
    D.nc = nc;
    D.cgen = S.coarse.generation;
  }
  TPT_CUDA(cudaStreamSynchronize(s));  // ac is ready for the caller's sum; host vectors are released
  return D.nc;
}

void dist_coarse_factor(DistData& D) {
  TPT_REQUIRE(D.nc > 0, TPTFEM_ERR_INVALID_ARG, "the rank has no coarse space");
  TPT_REQUIRE(!D.coarse_ready, TPTFEM_ERR_INVALID_ARG, "the coarse matrix is already factored");
  const bool ok = coarse_factor(D.ctx, D.nc, D.ld, D.ac.p, D.ainv.p);
  TPT_REQUIRE(ok, TPTFEM_ERR_NUMERIC, "the summed coarse matrix is not positive definite");
  TPT_CUDA(cudaStreamSynchronize(D.ctx->stream));
  D.coarse_ready = true;
}

double dist_precondition(DistData& D) {
  TPT_REQUIRE(D.pc != 0, TPTFEM_ERR_INVALID_ARG, "no block preconditioner set (Jacobi forms z in the update)");
  TPT_REQUIRE(!D.nc || D.coarse_ready, TPTFEM_ERR_INVALID_ARG,
              "the coarse matrix is not factored: sum it over the ranks, then call tptfem_dist_coarse_factor");
  check_coarse(D);
  cudaStream_t s = D.ctx->stream;
  const SystemData& S = *D.sys;
  if (D.nc) coarse_local_solve(S, D.ld, D.ainv.p, D.yc.p, D.uc.p, D.cm.p, s);
  const int64_t n = D.nloc;
  const bool coarse = D.nc > 0;
  if (n) {
    const FsaiFactor& F = *D.fac;
    dist_fsai_lower<<<D.blocks_spmv, DT_THREADS, 0, s>>>(n, F.rp.p, F.ci.p, F.va.p, F.sigma2.p, D.r.p, D.t.p);
    TPT_CHECK_LAUNCH();
  }
#define TPT_DIST_UP(DP)                                                                                             \
  dist_fsai_upper<DP><<<D.blocks_spmv, DT_THREADS, 0, s>>>(                                                        \
      n, n ? D.fac->trp.p : nullptr, n ? D.fac->tci.p : nullptr, n ? D.fac->tva.p : nullptr, D.t.p, D.r.p, D.z.p, \
      D.r0, coarse ? S.coarse.agg.p : nullptr, coarse ? S.coarse.y.p : nullptr, coarse ? D.cm.p : nullptr, D.part.p);
  if (coarse && S.dpn == 3) { TPT_DIST_UP(3) }
  else if (coarse && S.dpn == 2) { TPT_DIST_UP(2) }
  else { TPT_DIST_UP(1) }
#undef TPT_DIST_UP
  TPT_CHECK_LAUNCH();
  return D.sum_parts(D.blocks_spmv, 1, 0);
}

void dist_direction(DistData& D, double beta) {
  dist_direction<<<D.blocks_vec, DT_THREADS, 0, D.ctx->stream>>>(D.nloc, beta, D.z.p, D.p.p);
  TPT_CHECK_LAUNCH();
}

// x += xl, xl = 0: the steps since the last reliable update are kept apart
// from x (a correction far smaller than x), so their rounding does not set a
// floor under the true residual.
void dist_accumulate(DistData& D) {
  if (!D.nloc) return;
  dist_add_clear<<<D.blocks_vec, DT_THREADS, 0, D.ctx->stream>>>(D.nloc, D.xl.p, D.x.p);
  TPT_CHECK_LAUNCH();
}

// True residual, part 1: the owned part of p is saved and replaced by x, so
// that the caller's usual pack + exchange brings x's ghost values.
void dist_residual_begin(DistData& D) {
  cudaStream_t s = D.ctx->stream;
  if (!D.nloc) return;
  dist_accumulate(D);
  if (!D.pbak.p) D.pbak.alloc(D.nloc, s);
  TPT_CUDA(cudaMemcpyAsync(D.pbak.p, D.p.p, D.nloc * sizeof(double), cudaMemcpyDeviceToDevice, s));
  TPT_CUDA(cudaMemcpyAsync(D.p.p, D.x.p, D.nloc * sizeof(double), cudaMemcpyDeviceToDevice, s));
}

// Part 2 (after the exchange): r = b - A x replaces the recursive residual;
// out as dist_update's (with a block preconditioner: the coarse restriction's
// partial in yc); the search direction is restored.
void dist_residual_end(DistData& D, double* out) {
  check_coarse(D);
  cudaStream_t s = D.ctx->stream;
  dist_true_residual<<<D.blocks_spmv, DT_THREADS, 0, s>>>(D.nloc, D.rp.p, D.ci.p, D.va.p, D.p.p, D.b.p, D.r.p, D.z.p,
                                                          D.dinv.p, D.part.p, D.pc == 0);
  TPT_CHECK_LAUNCH();
  if (D.nloc)
    TPT_CUDA(cudaMemcpyAsync(D.p.p, D.pbak.p, D.nloc * sizeof(double), cudaMemcpyDeviceToDevice, s));
  if (D.nc) coarse_local_restrict(*D.sys, D.cl, D.r.p, D.yc.p, s);
  out[0] = D.sum_parts(D.blocks_spmv, 2, 0);
  out[1] = D.sum_parts(D.blocks_spmv, 2, 1);
}

// Several ranks on one device in lock step, the exchange done by device copies.
int64_t dist_solve_local(tptfem_context* ctx, SystemData& S, int nranks, double tol, int64_t max_iter, double* u_red,
                         double* relres, int kind, int aggregates) {
  TPT_REQUIRE(nranks >= 1, TPTFEM_ERR_INVALID_ARG, "nranks must be >= 1");
  const int64_t groups = S.n_free / std::max(1, S.dpn);
  std::vector<int64_t> starts(nranks + 1);
  for (int k = 0; k <= nranks; ++k)
    starts[k] = (S.n_free % S.dpn == 0) ? groups * k / nranks * S.dpn : S.n_free * k / nranks;
  starts[nranks] = S.n_free;
  std::vector<std::unique_ptr<DistData>> R;
  for (int k = 0; k < nranks; ++k) R.push_back(dist_create(ctx, S, k, nranks, starts.data()));
  cudaStream_t s = ctx->stream;
  auto exchange = [&]() {
    for (auto& d : R) dist_pack(*d);
    for (int k = 0; k < nranks; ++k)
      for (int q = 0; q < nranks; ++q) {
        const int64_t cnt = R[q]->send_off[k + 1] - R[q]->send_off[k];
        if (q == k || !cnt) continue;
        TPT_CUDA(cudaMemcpyAsync(R[k]->p.p + R[k]->nloc + R[k]->recv_off[q], R[q]->send_buf.p + R[q]->send_off[k],
                                 cnt * sizeof(double), cudaMemcpyDeviceToDevice, s));
      }
  };
  // block preconditioner: every rank's set-up, the partial coarse matrices
  // summed in rank order into each rank's copy, each copy factored
  int nc = 0;
  DevBuf<double> csum;
  auto sum_into_all = [&](auto get, size_t n) {
    if (R.size() > 1) {
      TPT_CUDA(cudaMemcpyAsync(csum.p, get(*R[0]), n * sizeof(double), cudaMemcpyDeviceToDevice, s));
      for (size_t k = 1; k < R.size(); ++k) {
        dist_add<<<ceil_div((int64_t)n, 256), 256, 0, s>>>((int64_t)n, get(*R[k]), csum.p);
        TPT_CHECK_LAUNCH();
      }
      for (auto& d : R)
        TPT_CUDA(cudaMemcpyAsync(get(*d), csum.p, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
    TPT_CUDA(cudaStreamSynchronize(s));
  };
  if (kind) {
    for (auto& d : R) nc = dist_set_precond(*d, S, kind, aggregates);
    if (nc) {
      csum.alloc((size_t)nc * nc, s);
      sum_into_all([](DistData& d) { return d.ac.p; }, (size_t)nc * nc);
      for (auto& d : R) dist_coarse_factor(*d);
    }
  }
  auto precondition = [&]() {  // z = M r on every rank, the summed r.z
    if (nc) sum_into_all([](DistData& d) { return d.yc.p; }, (size_t)nc);
    double v = 0.0;
    for (auto& d : R) v += dist_precondition(*d);
    return v;
  };
  double rr = 0.0, rz = 0.0, bb = 0.0;
  for (auto& d : R) {
    double o[2];
    dist_start(*d, o);
    rr += o[0];
    rz += o[1];
  }
  if (kind) {
    rz = precondition();
    for (auto& d : R) dist_direction(*d, 0.0);
  }
  bb = rr;
  int64_t it = 0;
  const double target = tol * tol * bb;
  double rr_upd = bb;  // true r.r at the last replacement
  while (bb > 0.0) {
    // iterate until the recursive residual has dropped by DIST_DELTA since the
    // last replacement, or (a little below) the target; the iteration that
    // gets there stops after the x, r update (no new direction)
    const double until = std::max(0.25 * target, DIST_DELTA * DIST_DELTA * rr_upd);
    while (it < max_iter) {
      exchange();
      double pq = 0.0;
      for (auto& d : R) pq += dist_spmv_dot(*d);
      TPT_REQUIRE(pq > 0.0, TPTFEM_ERR_BREAKDOWN, "PCG breakdown: p.Ap <= 0");
      const double alpha = rz / pq;
      double nrr = 0.0, nrz = 0.0;
      for (auto& d : R) {
        double o[2];
        dist_update(*d, alpha, o);
        nrr += o[0];
        nrz += o[1];
      }
      ++it;
      rr = nrr;
      if (rr <= until) break;
      if (kind) nrz = precondition();
      const double beta = nrz / rz;
      rz = nrz;
      for (auto& d : R) dist_direction(*d, beta);
    }
    // reliable update: the true residual replaces the recursive one, and the
    // direction continues from the last one with beta = r.z (true) / the r.z
    // of the last step length
    for (auto& d : R) dist_residual_begin(*d);
    exchange();
    double trr = 0.0, trz = 0.0;
    for (auto& d : R) {
      double o[2];
      dist_residual_end(*d, o);
      trr += o[0];
      trz += o[1];
    }
    rr = trr;
    if (rr <= target || it >= max_iter) break;
    if (kind) trz = precondition();
    const double beta = trz / rz;
    rz = trz;
    rr_upd = rr;
    for (auto& d : R) dist_direction(*d, beta);
  }
  for (auto& d : R) {
    dist_accumulate(*d);
    if (d->nloc) d->x.download(u_red + d->r0, d->nloc);
  }
  TPT_CUDA(cudaStreamSynchronize(s));
  *relres = bb > 0.0 ? std::sqrt(rr / bb) : 0.0;  // true residual
  return it;
}

}  // namespace tptfem
