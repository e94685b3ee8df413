// fsai.cu -- factorised sparse approximate inverse M^-1 = G^T G of the reduced
// SPD matrix A (Kolotilina-Yeremin FSAI), in the scaled form
//     G = diag(sigma) (I + L),   L strictly lower triangular,
// which is SPD by construction for any sigma > 0 and any L.  sigma^2 is kept in
// FP32 and L in FP16: the preconditioner is the low-precision part of the
// mixed-precision solver (the Krylov recurrences and the operator stay FP64).
//
// Pattern: the lower triangle of the NODE-BLOCK pattern of A -- row i may use
// every free dof j < i of every mesh node coupled to i's node in A (for
// scalar problems, one dof per node, this is tril(A) itself).  The same
// pattern carries the learned factor's values.
//
// Classic values: one thread per row i gathers A[P,P] for P = pattern(i) + {i}
// by merging sorted CSR rows, factors it by Cholesky (packed, local memory)
// and solves A[P,P] y = e_i; then sigma_i^2 = y_i and L_ij = y_j / y_i.
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>

#include <climits>

#include "objects.hpp"

namespace tptfem {

namespace {

constexpr int FSAI_MAXM = 48;  // longest pattern row (incl. the diagonal) handled

// Strictly-lower node-block pattern of reduced row i (sorted), COUNT or FILL.
template <bool FILL>
__global__ void nb_lower_pattern(int n, int dpn, const int* __restrict__ rp, const int* __restrict__ ci,
                                 const int* __restrict__ free_map, const int* __restrict__ red_map,
                                 int* __restrict__ cnt, const int* __restrict__ lrp, int* __restrict__ lci,
                                 int* __restrict__ flag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int node = free_map[i] / dpn;
  int g0 = i, g1 = i + 1;  // rows of the same node are consecutive
  while (g0 > 0 && free_map[g0 - 1] / dpn == node) --g0;
  while (g1 < n && free_map[g1] / dpn == node) ++g1;
  int list[FSAI_MAXM];
  int len = 0;
  bool over = false;
  for (int g = g0; g < g1 && !over; ++g)
    for (int k = rp[g]; k < rp[g + 1] && !over; ++k) {
      const int m = free_map[ci[k]] / dpn;
      for (int c = 0; c < dpn; ++c) {
        const int j = red_map[m * dpn + c];
        if (j < 0 || j >= i) continue;
        int lo = 0, hi = len;
        while (lo < hi) { int mid = (lo + hi) >> 1; if (list[mid] < j) lo = mid + 1; else hi = mid; }
        if (lo < len && list[lo] == j) continue;
        if (len == FSAI_MAXM - 1) { over = true; break; }
        for (int t = len; t > lo; --t) list[t] = list[t - 1];
        list[lo] = j;
        ++len;
      }
    }
  if (over) { atomicOr(flag, 1); len = 0; }
  if (!FILL) {
    cnt[i] = len;
  } else {
    const int o = lrp[i];
    for (int t = 0; t < len; ++t) lci[o + t] = list[t];
  }
}

// The same pattern from the node-group adjacency (sorted neighbour groups of
// each group, the union over its dofs' rows), valid when every free node has
// all its dofs free, so that reduced dof = group * dpn + component: row
// i = g dpn + a holds every component of the neighbour groups J < g, then the
// node's own components c < a.  Same rows, order and overflow rule as
// nb_lower_pattern.
template <bool FILL>
__global__ void nb_lower_from_groups(int n, int dpn, const int* __restrict__ gptr, const int* __restrict__ glist,
                                     int* __restrict__ cnt, const int* __restrict__ lrp, int* __restrict__ lci,
                                     int* __restrict__ flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int g = i / dpn, a = i - g * dpn;
  int nlow = 0;
  for (int k = gptr[g]; k < gptr[g + 1] && glist[k] < g; ++k) ++nlow;
  const int len = nlow * dpn + a;
  if (len >= FSAI_MAXM) {
    atomicOr(flag, 1);
    if (!FILL) cnt[i] = 0;
    return;
  }
  if (!FILL) {
    cnt[i] = len;
  } else {
    int* out = lci + lrp[i];
    for (int k = gptr[g]; k < gptr[g] + nlow; ++k)
      for (int c = 0; c < dpn; ++c) *out++ = glist[k] * dpn + c;
    for (int c = 0; c < a; ++c) *out++ = g * dpn + c;
  }
}

__global__ void col_counts(int64_t nnz, const int* __restrict__ gci, int* __restrict__ cnt) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nnz) atomicAdd(&cnt[gci[k]], 1);
}

// Scatter L's entries into the rows of L^T (unordered), recording L's index.
__global__ void transpose_fill(int n, const int* __restrict__ grp, const int* __restrict__ gci,
                               const int* __restrict__ trp, int* __restrict__ cursor, int* __restrict__ tci,
                               int* __restrict__ perm) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int k = grp[i]; k < grp[i + 1]; ++k) {
    int j = gci[k];
    int pos = trp[j] + atomicAdd(&cursor[j], 1);
    tci[pos] = i;
    perm[pos] = k;
  }
}

// Sort each L^T row by column -> deterministic.  One warp per row: rows of up
// to 64 entries are bitonic-sorted in registers (2 keys per lane); longer rows
// fall back to an insertion sort by one lane.
__global__ void transpose_sort(int n, const int* __restrict__ trp, int* __restrict__ tci, int* __restrict__ perm) {
  const int lane = threadIdx.x & 31;
  const int j = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (j >= n) return;
  const int b = trp[j], e = trp[j + 1], len = e - b;
  if (len <= 1) return;
  if (len > 64) {
    if (lane == 0)
      for (int a = b + 1; a < e; ++a) {
        int c = tci[a], p = perm[a];
        int q = a - 1;
        while (q >= b && tci[q] > c) { tci[q + 1] = tci[q]; perm[q + 1] = perm[q]; --q; }
        tci[q + 1] = c;
        perm[q + 1] = p;
      }
    return;
  }
  int key[2], val[2];
  for (int h = 0; h < 2; ++h) {
    const int t = 2 * lane + h;
    key[h] = t < len ? tci[b + t] : INT_MAX;
    val[h] = t < len ? perm[b + t] : 0;
  }
  for (int k = 2; k <= 64; k <<= 1)
    for (int d = k >> 1; d >= 1; d >>= 1) {
      if (d == 1) {
        const bool asc = ((2 * lane) & k) == 0;
        if (asc ? key[0] > key[1] : key[0] < key[1]) {
          int t = key[0]; key[0] = key[1]; key[1] = t;
          t = val[0]; val[0] = val[1]; val[1] = t;
        }
      } else {
        for (int h = 0; h < 2; ++h) {
          const int el = 2 * lane + h, pe = el ^ d;
          const int pk = __shfl_xor_sync(0xffffffffu, key[h], d >> 1);
          const int pv = __shfl_xor_sync(0xffffffffu, val[h], d >> 1);
          const bool asc = (el & k) == 0;
          const bool take_min = (el < pe) == asc;
          const bool swap = take_min ? pk < key[h] : pk > key[h];
          if (swap) { key[h] = pk; val[h] = pv; }
        }
      }
    }
  for (int h = 0; h < 2; ++h) {
    const int t = 2 * lane + h;
    if (t < len) { tci[b + t] = key[h]; perm[b + t] = val[h]; }
  }
}

// Classic FSAI row i: B = A[P,P] with P = (L pattern of i, i), Cholesky, y = B^-1 e_m.
__global__ void fsai_rows(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ va,
                          const int* __restrict__ lrp, const int* __restrict__ lci, double* __restrict__ sig2,
                          double* __restrict__ lva, int* __restrict__ flag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int l0 = lrp[i], m = lrp[i + 1] - l0 + 1;
  double B[FSAI_MAXM * (FSAI_MAXM + 1) / 2];  // packed lower triangle, row-major
  int P[FSAI_MAXM];
  for (int a = 0; a < m - 1; ++a) P[a] = lci[l0 + a];
  P[m - 1] = i;
  for (int a = 0; a < m; ++a) {
    const int r = P[a];
    int k = rp[r], b = 0;
    const int ke = rp[r + 1];
    double* row = B + a * (a + 1) / 2;
    for (int t = 0; t <= a; ++t) row[t] = 0.0;
    while (k < ke && b <= a) {
      const int c = ci[k];
      if (c == P[b]) { row[b] = va[k]; ++k; ++b; }
      else if (c < P[b]) ++k;
      else ++b;
    }
  }
  for (int a = 0; a < m; ++a) {
    double* ra = B + a * (a + 1) / 2;
    for (int b = 0; b <= a; ++b) {
      const double* rb = B + b * (b + 1) / 2;
      double s = ra[b];
      for (int t = 0; t < b; ++t) s -= ra[t] * rb[t];
      if (b == a) {
        if (!(s > 0.0)) { atomicOr(flag, 2); return; }
        ra[a] = sqrt(s);
      } else {
        ra[b] = s / rb[b];
      }
    }
  }
  double y[FSAI_MAXM];
  for (int a = 0; a < m; ++a) y[a] = 0.0;
  y[m - 1] = 1.0 / B[(m - 1) * m / 2 + (m - 1)];
  for (int a = m - 1; a >= 0; --a) {
    double s = y[a];
    for (int t = a + 1; t < m; ++t) s -= B[t * (t + 1) / 2 + a] * y[t];
    y[a] = s / B[a * (a + 1) / 2 + a];
  }
  const double d = y[m - 1];
  if (!(d > 0.0) || !isfinite(d)) { atomicOr(flag, 2); return; }
  sig2[i] = d;
  for (int a = 0; a < m - 1; ++a) lva[l0 + a] = y[a] / d;
}

__global__ void factor_to_lowp(int n, int64_t nnz, const double* __restrict__ sig2, const double* __restrict__ lva,
                               const int* __restrict__ perm, float* __restrict__ s32, __half* __restrict__ va16,
                               __half* __restrict__ tva16, int* __restrict__ flag) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) {
    const double s = sig2[k];
    if (!(s > 0.0) || !isfinite(s)) atomicOr(flag, 4);
    s32[k] = (float)s;
  }
  if (k < nnz) {
    const double v = lva[k];
    if (!isfinite(v) || fabs(v) > 6.0e4) atomicOr(flag, 4);  // outside FP16 range
    va16[k] = __double2half(v);
    if (perm) tva16[k] = __double2half(lva[perm[k]]);
  }
}

// Values of the explicit transpose from the FP16 factor: tva[k] = va[perm[k]].
__global__ void transpose_values(int64_t nnz, const int* __restrict__ perm, const __half* __restrict__ va,
                                 __half* __restrict__ tva) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nnz) tva[k] = va[perm[k]];
}

}  // namespace

void fsai_build_pattern(const SystemData& S, FsaiFactor& F) {
  if (F.ready_pattern) return;
  cudaStream_t s = S.ctx->stream;
  const int n = (int)S.n_free;
  F.n = n;
  DevBuf<int> cnt;
  cnt.alloc(n + 1, s);
  TPT_CUDA(cudaMemsetAsync(S.ctx->d_flag, 0, sizeof(int), s));
  // from the node-group adjacency when the node-block operator exists (one pass
  // over each group's neighbour list instead of a sorted union per row)
  const bool groups = S.nb.state == 1 && S.nb.dpn == S.dpn;
  if (groups)
    nb_lower_from_groups<false><<<ceil_div(n, 256), 256, 0, s>>>(n, S.dpn, S.nb.gptr.p, S.nb.glist.p, cnt.p, nullptr,
                                                                 nullptr, S.ctx->d_flag);
  else
    nb_lower_pattern<false><<<ceil_div(n, 128), 128, 0, s>>>(n, S.dpn, S.row_ptr.p, S.col.p, S.free_map.p,
                                                              S.red_map.p, cnt.p, nullptr, nullptr, S.ctx->d_flag);
  TPT_CHECK_LAUNCH();
  F.rp.alloc(n + 1, s);
  F.nnz = exclusive_scan_i32(cnt.p, F.rp.p, n, s);
  int flag = 0;
  TPT_CUDA(cudaMemcpyAsync(&flag, S.ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
  TPT_CUDA(cudaStreamSynchronize(s));
  F.overflow = flag != 0;
  F.ci.alloc(F.nnz, s);
  if (groups)
    nb_lower_from_groups<true><<<ceil_div(n, 256), 256, 0, s>>>(n, S.dpn, S.nb.gptr.p, S.nb.glist.p, nullptr, F.rp.p,
                                                                F.ci.p, S.ctx->d_flag);
  else
    nb_lower_pattern<true><<<ceil_div(n, 128), 128, 0, s>>>(n, S.dpn, S.row_ptr.p, S.col.p, S.free_map.p,
                                                             S.red_map.p, nullptr, F.rp.p, F.ci.p, S.ctx->d_flag);
  TPT_CHECK_LAUNCH();
  F.sigma2.alloc(n, s);
  F.va.alloc(F.nnz, s);
  F.ready_pattern = true;
}

void fsai_build_transpose(const SystemData& S, FsaiFactor& F) {
  if (F.transposed || !F.ready_pattern) return;
  cudaStream_t s = S.ctx->stream;
  const int n = (int)F.n;
  DevBuf<int> cnt;
  cnt.alloc(n + 1, s);
  cnt.zero();
  col_counts<<<ceil_div(std::max<int64_t>(F.nnz, 1), 256), 256, 0, s>>>(F.nnz, F.ci.p, cnt.p);
  TPT_CHECK_LAUNCH();
  F.trp.alloc(n + 1, s);
  exclusive_scan_i32(cnt.p, F.trp.p, n, s);
  F.tci.alloc(F.nnz, s);
  F.perm.alloc(F.nnz, s);
  cnt.zero();
  transpose_fill<<<ceil_div(n, 256), 256, 0, s>>>(n, F.rp.p, F.ci.p, F.trp.p, cnt.p, F.tci.p, F.perm.p);
  TPT_CHECK_LAUNCH();
  transpose_sort<<<ceil_div((int64_t)n * 32, 256), 256, 0, s>>>(n, F.trp.p, F.tci.p, F.perm.p);
  TPT_CHECK_LAUNCH();
  F.tva.alloc(F.nnz, s);
  if (F.values_set && F.nnz) {
    transpose_values<<<ceil_div(F.nnz, 256), 256, 0, s>>>(F.nnz, F.perm.p, F.va.p, F.tva.p);
    TPT_CHECK_LAUNCH();
  }
  F.transposed = true;
}

bool fsai_set_values(const SystemData& S, FsaiFactor& F, const double* d_sig2, const double* d_lva) {
  cudaStream_t s = S.ctx->stream;
  TPT_CUDA(cudaMemsetAsync(S.ctx->d_flag, 0, sizeof(int), s));
  const int64_t m = std::max<int64_t>(F.n, F.nnz);
  factor_to_lowp<<<ceil_div(std::max<int64_t>(m, 1), 256), 256, 0, s>>>(
      (int)F.n, F.nnz, d_sig2, d_lva, F.transposed ? F.perm.p : nullptr, F.sigma2.p, F.va.p,
      F.transposed ? F.tva.p : nullptr, S.ctx->d_flag);
  TPT_CHECK_LAUNCH();
  F.values_set = true;
  int flag = 0;
  TPT_CUDA(cudaMemcpyAsync(&flag, S.ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
  TPT_CUDA(cudaStreamSynchronize(s));
  return flag == 0;
}

bool fsai_classic(const SystemData& S, FsaiFactor& F) {
  fsai_build_pattern(S, F);
  if (F.overflow) return false;
  cudaStream_t s = S.ctx->stream;
  DevBuf<double> sig2, lva;
  sig2.alloc(F.n, s);
  lva.alloc(std::max<int64_t>(F.nnz, 1), s);
  TPT_CUDA(cudaMemsetAsync(S.ctx->d_flag, 0, sizeof(int), s));
  fsai_rows<<<ceil_div(F.n, 128), 128, 0, s>>>((int)F.n, S.row_ptr.p, S.col.p, S.val.p, F.rp.p, F.ci.p, sig2.p,
                                               lva.p, S.ctx->d_flag);
  TPT_CHECK_LAUNCH();
  int flag = 0;
  TPT_CUDA(cudaMemcpyAsync(&flag, S.ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
  TPT_CUDA(cudaStreamSynchronize(s));
  if (flag) return false;
  return fsai_set_values(S, F, sig2.p, lva.p);
}

}  // namespace tptfem
