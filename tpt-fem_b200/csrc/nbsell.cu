// nbsell.cu -- node-block sliced-ELL ("NB-SELL") storage of the reduced
// operator K and of the FSAI factor, for systems whose free dofs come in full
// node groups of DPN consecutive dofs (every mesh node has all or none of its
// dofs fixed; true for clamped boundaries).
//
// Layout: groups (mesh nodes with free dofs) are taken 32 at a time (one warp,
// one thread per group).  Chunk c stores `slots[c]` block slots; for slot k the
// 32 block columns are contiguous (int32), so every column load of a warp is
// one coalesced transaction.
//   K   : all neighbour blocks, FP64; each of the DPN*DPN values is a
//         contiguous run of 32 (one 256-byte warp load per value).
//   L   : strictly-lower neighbour blocks (J < I), FP16, each lane's block
//         packed in a 16-byte word (8 values) + a 2-byte tail (the 9th; for
//         one dof per node the tail alone holds the value),
//         + the strictly-lower part of the diagonal block;
//   L^T : strictly-upper neighbour blocks (J > I) holding transposed blocks of
//         L, same packing; it reuses L's diagonal part, transposed.
// A group with fewer neighbours than its chunk's slot count is padded with its
// own column and zero values.
//
// The factor's CSR rows have a fixed shape on the node-block pattern: row
// DPN*I + a holds the DPN columns of each lower neighbour group in ascending
// order, then a entries of its own group.  The build step records, for every
// L^T slot, the position of I in the neighbour's lower list, so refilling the
// blocks after new factor values (classic or learned) is a pure gather.
#include <cuda_fp16.h>

#include <algorithm>

#include "objects.hpp"

namespace tptfem {

namespace {

constexpr int NB_MAX = 96;  // neighbour groups per group handled

// Groups are full iff free_map[g*dpn + c] = node_g*dpn + c for every c.
__global__ void check_groups(int ngroups, int dpn, const int* __restrict__ free_map, int* __restrict__ flag) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngroups) return;
  const int base = free_map[g * dpn];
  if (base % dpn != 0) { atomicOr(flag, 1); return; }
  for (int c = 1; c < dpn; ++c)
    if (free_map[g * dpn + c] != base + c) atomicOr(flag, 1);
}

// Sorted neighbour groups of group g (union over its dpn rows); COUNT / FILL.
template <bool FILL>
__global__ void group_neighbours(int ngroups, int dpn, const int* __restrict__ rp, const int* __restrict__ ci,
                                 int* __restrict__ cnt, const int* __restrict__ gptr, int* __restrict__ glist,
                                 int* __restrict__ flag) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngroups) return;
  int list[NB_MAX];
  int len = 0;
  for (int a = 0; a < dpn; ++a) {
    const int row = g * dpn + a;
    for (int k = rp[row]; k < rp[row + 1]; ++k) {
      const int J = ci[k] / dpn;
      int lo = 0, hi = len;
      while (lo < hi) { int mid = (lo + hi) >> 1; if (list[mid] < J) lo = mid + 1; else hi = mid; }
      if (lo < len && list[lo] == J) continue;
      if (len == NB_MAX) { atomicOr(flag, 2); return; }
      for (int t = len; t > lo; --t) list[t] = list[t - 1];
      list[lo] = J;
      ++len;
    }
  }
  if (!FILL) {
    cnt[g] = len;
  } else {
    const int o = gptr[g];
    for (int t = 0; t < len; ++t) glist[o + t] = list[t];
  }
}

// Slots of chunk c = max over its groups of the selected neighbour count.
// which: 0 all, 1 lower (J < g), 2 upper (J > g).
__global__ void chunk_slots(int ngroups, const int* __restrict__ gptr, const int* __restrict__ glist, int which,
                            int* __restrict__ slots) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  int m = 0;
  if (g < ngroups) {
    for (int k = gptr[g]; k < gptr[g + 1]; ++k) {
      const int J = glist[k];
      m += which == 0 || (which == 1 && J < g) || (which == 2 && J > g);
    }
  }
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, o));
  if (lane == 0 && (g >> 5) < (ngroups + 31) / 32) slots[g >> 5] = m;
}

// Value of row `row`, column `col` of a CSR matrix (binary search; 0 if absent).
__device__ __forceinline__ double csr_at(const int* __restrict__ rp, const int* __restrict__ ci,
                                         const double* __restrict__ va, int row, int col) {
  int lo = rp[row], hi = rp[row + 1];
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (ci[mid] < col) lo = mid + 1;
    else hi = mid;
  }
  return (lo < rp[row + 1] && ci[lo] == col) ? va[lo] : 0.0;
}

// Fill K's NB-SELL blocks (FP64) from the reduced CSR.
__global__ void fill_k(int ngroups, int dpn, const int* __restrict__ rp, const int* __restrict__ ci,
                       const double* __restrict__ va, const int* __restrict__ gptr, const int* __restrict__ glist,
                       const int* __restrict__ cptr, int* __restrict__ bcol, double* __restrict__ bval) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngroups) return;
  const int c = g >> 5, lane = g & 31;
  const int nslot = cptr[c + 1] - cptr[c];
  const int nb = gptr[g + 1] - gptr[g];
  const int d2 = dpn * dpn;
  for (int k = 0; k < nslot; ++k) {
    const int64_t s = (int64_t)(cptr[c] + k);
    const int J = k < nb ? glist[gptr[g] + k] : g;
    bcol[s * 32 + lane] = J;
    for (int a = 0; a < dpn; ++a)
      for (int b = 0; b < dpn; ++b)
        bval[(s * d2 + a * dpn + b) * 32 + lane] = k < nb ? csr_at(rp, ci, va, g * dpn + a, J * dpn + b) : 0.0;
  }
}

// Columns of the L (lower) and L^T (upper) slots, the lower count per group,
// and for each L^T slot the position of g in the neighbour's lower list.
__global__ void factor_columns(int ngroups, const int* __restrict__ gptr, const int* __restrict__ glist,
                               const int* __restrict__ lcptr, const int* __restrict__ ucptr, int* __restrict__ lcol,
                               int* __restrict__ ucol, int* __restrict__ upos, int* __restrict__ nlow) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngroups) return;
  const int c = g >> 5, lane = g & 31;
  int kl = 0, ku = 0;
  for (int t = gptr[g]; t < gptr[g + 1]; ++t) {
    const int J = glist[t];
    if (J < g) {
      lcol[((int64_t)lcptr[c] + kl++) * 32 + lane] = J;
    } else if (J > g) {
      // position of g among J's neighbours below J
      int p = 0;
      for (int u = gptr[J]; u < gptr[J + 1] && glist[u] < g; ++u) ++p;
      const int64_t s = ((int64_t)ucptr[c] + ku++) * 32 + lane;
      ucol[s] = J;
      upos[s] = p;
    }
  }
  nlow[g] = kl;
  for (; kl < lcptr[c + 1] - lcptr[c]; ++kl) lcol[((int64_t)lcptr[c] + kl) * 32 + lane] = g;
  for (; ku < ucptr[c + 1] - ucptr[c]; ++ku) {
    const int64_t s = ((int64_t)ucptr[c] + ku) * 32 + lane;
    ucol[s] = g;
    upos[s] = -1;
  }
}

// Every factor row must have the node-block shape the fill relies on.
__global__ void check_factor_shape(int ngroups, int dpn, const int* __restrict__ lrp, const int* __restrict__ nlow,
                                   int* __restrict__ flag) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngroups) return;
  for (int a = 0; a < dpn; ++a) {
    const int row = g * dpn + a;
    if (lrp[row + 1] - lrp[row] != dpn * nlow[g] + a) atomicOr(flag, 1);
  }
}

__device__ __forceinline__ void store_block(uint4* pack, __half* tail, int64_t idx, const float* v, int d2) {
  if (d2 == 1) {  // a single value: the 2-byte array holds it, the word stays unused
    tail[idx] = __float2half(v[0]);
    return;
  }
  __half h[8];
  for (int q = 0; q < 8; ++q) h[q] = __float2half(q < d2 ? v[q] : 0.f);
  uint4 w;
  __half2* hw = reinterpret_cast<__half2*>(&w);
  for (int i = 0; i < 4; ++i) hw[i] = __halves2half2(h[2 * i], h[2 * i + 1]);
  pack[idx] = w;
  tail[idx] = __float2half(d2 == 9 ? v[8] : 0.f);
}

// Gather the L / L^T blocks and L's diagonal part from the factor's CSR values.
__global__ void fill_factor(int ngroups, int dpn, const int* __restrict__ lrp, const __half* __restrict__ lva,
                            const int* __restrict__ nlow, const int* __restrict__ lcptr, const int* __restrict__ lcol,
                            const int* __restrict__ ucptr, const int* __restrict__ ucol,
                            const int* __restrict__ upos, uint4* __restrict__ lpack, __half* __restrict__ ltail,
                            uint4* __restrict__ upack, __half* __restrict__ utail, __half* __restrict__ ldiag) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngroups) return;
  const int c = g >> 5, lane = g & 31;
  const int d2 = dpn * dpn;
  const int nl = nlow[g];
  float v[9];
  for (int k = 0; k < lcptr[c + 1] - lcptr[c]; ++k) {
    const int64_t idx = ((int64_t)lcptr[c] + k) * 32 + lane;
    for (int a = 0; a < dpn; ++a)
      for (int b = 0; b < dpn; ++b)
        v[a * dpn + b] = k < nl ? __half2float(lva[lrp[g * dpn + a] + dpn * k + b]) : 0.f;
    store_block(lpack, ltail, idx, v, d2);
  }
  for (int k = 0; k < ucptr[c + 1] - ucptr[c]; ++k) {
    const int64_t idx = ((int64_t)ucptr[c] + k) * 32 + lane;
    const int J = ucol[idx], p = upos[idx];
    // L^T block (g, J)[a][b] = L[J*dpn + b][g*dpn + a]
    for (int a = 0; a < dpn; ++a)
      for (int b = 0; b < dpn; ++b)
        v[a * dpn + b] = p >= 0 ? __half2float(lva[lrp[J * dpn + b] + dpn * p + a]) : 0.f;
    store_block(upack, utail, idx, v, d2);
  }
  int q = 0;
  for (int a = 1; a < dpn; ++a)
    for (int b = 0; b < a; ++b, ++q) ldiag[((int64_t)c * 3 + q) * 32 + lane] = lva[lrp[g * dpn + a] + dpn * nl + b];
}

// Symmetric half storage of K: the strictly-lower blocks in the L slot
// structure, the diagonal blocks per chunk, and for each L^T slot (g, J > g)
// the index of block (J, g) in the lower storage (its transpose is K_gJ).
// One block of 32 threads per chunk; lanes past the last group are skipped.
__global__ void upper_bases(int ngroups, int dpn, const int* __restrict__ lcptr, const int* __restrict__ ucptr,
                            const int* __restrict__ ucol, const int* __restrict__ upos, int* __restrict__ ubase) {
  const int c = blockIdx.x, lane = threadIdx.x;
  if (c * 32 + lane >= ngroups) return;
  for (int64_t s = ucptr[c]; s < ucptr[c + 1]; ++s) {
    const int64_t idx = s * 32 + lane;
    const int J = ucol[idx], p = upos[idx];
    ubase[idx] = p < 0 ? -1 : (int)(((int64_t)lcptr[J >> 5] + p) * dpn * dpn * 32 + (J & 31));
  }
}

// Values of the symmetric half storage from the CSR, structure kept: thread
// (a, g) merges CSR row g*dpn+a with group g's lower slots (ascending block
// columns, all below the diagonal block) and then the diagonal block.  Writes
// for one (slot, a, b) are coalesced over the chunk's 32 lanes.
__global__ void refill_ksym(int ngroups, int dpn, const int* __restrict__ rp, const int* __restrict__ ci,
                            const double* __restrict__ va, const int* __restrict__ lcptr,
                            const int* __restrict__ lcol, const int* __restrict__ nlow, double* __restrict__ lval,
                            double* __restrict__ dval) {
  const int lane = threadIdx.x & 31, a = threadIdx.x >> 5;  // blockDim = 32 * dpn
  const int c = blockIdx.x, g = c * 32 + lane;
  if (g >= ngroups || a >= dpn) return;
  const int d2 = dpn * dpn, nl = nlow[g];
  const int row = g * dpn + a;
  int k = rp[row];
  const int ke = rp[row + 1];
  const int64_t s0 = lcptr[c], ns = lcptr[c + 1] - s0;
  for (int64_t sl = 0; sl < ns; ++sl) {
    const int64_t s = s0 + sl;
    const int J = sl < nl ? lcol[s * 32 + lane] : -1;
    for (int b = 0; b < dpn; ++b) {
      double v = 0.0;
      if (J >= 0) {
        const int col = J * dpn + b;
        while (k < ke && ci[k] < col) ++k;
        if (k < ke && ci[k] == col) v = va[k];
      }
      lval[(s * d2 + a * dpn + b) * 32 + lane] = v;
    }
  }
  for (int b = 0; b < dpn; ++b) {
    const int col = g * dpn + b;
    while (k < ke && ci[k] < col) ++k;
    dval[((int64_t)c * d2 + a * dpn + b) * 32 + lane] = (k < ke && ci[k] == col) ? va[k] : 0.0;
  }
}

}  // namespace

void nb_build_sym(SystemData& S) {
  NbSell& N = S.nb;
  if (N.sym_built) return;
  TPT_REQUIRE(N.state == 1, TPTFEM_ERR_INVALID_ARG, "symmetric operator needs the node-block layout");
  cudaStream_t s = S.ctx->stream;
  const int d2 = N.dpn * N.dpn;
  TPT_REQUIRE(std::max<int64_t>(N.l_slots, 1) * 32 * d2 < (1LL << 31), TPTFEM_ERR_INVALID_ARG,
              "symmetric operator: lower storage exceeds int32 indexing");
  N.ks_lval.alloc(std::max<int64_t>(N.l_slots, 1) * 32 * d2, s);
  N.ks_diag.alloc((int64_t)N.nchunks * 32 * d2, s);
  N.ku_base.alloc(std::max<int64_t>(N.u_slots, 1) * 32, s);
  N.ks_diag.zero();
  upper_bases<<<N.nchunks, 32, 0, s>>>(N.ngroups, N.dpn, N.l_cptr.p, N.u_cptr.p, N.u_col.p, N.u_pos.p, N.ku_base.p);
  TPT_CHECK_LAUNCH();
  refill_ksym<<<N.nchunks, 32 * N.dpn, 0, s>>>(N.ngroups, N.dpn, S.row_ptr.p, S.col.p, S.val.p, N.l_cptr.p,
                                               N.l_col.p, N.nlow.p, N.ks_lval.p, N.ks_diag.p);
  TPT_CHECK_LAUNCH();
  N.sym_built = true;
  N.fresh_fill = true;
}

void nb_refill_values(SystemData& S, bool sym) {
  NbSell& N = S.nb;
  if (N.state != 1) return;
  cudaStream_t s = S.ctx->stream;
  if (sym && N.sym_built) {
    refill_ksym<<<N.nchunks, 32 * N.dpn, 0, s>>>(N.ngroups, N.dpn, S.row_ptr.p, S.col.p, S.val.p, N.l_cptr.p,
                                                 N.l_col.p, N.nlow.p, N.ks_lval.p, N.ks_diag.p);
  } else {
    if (!N.k_val.p) {
      N.k_col.alloc(std::max<int64_t>(N.k_slots, 1) * 32, s);
      N.k_val.alloc(std::max<int64_t>(N.k_slots, 1) * 32 * N.dpn * N.dpn, s);
    }
    fill_k<<<ceil_div(N.ngroups, 128), 128, 0, s>>>(N.ngroups, N.dpn, S.row_ptr.p, S.col.p, S.val.p, N.gptr.p,
                                                    N.glist.p, N.k_cptr.p, N.k_col.p, N.k_val.p);
    N.full_stale = false;
  }
  TPT_CHECK_LAUNCH();
  N.fresh_fill = true;
}

void nb_refresh_values(SystemData& S) {
  NbSell& N = S.nb;
  if (N.state != 1) return;
  if (N.sym_built) nb_refill_values(S, true);
  N.full_stale = true;  // the full storage is refilled when a solve asks for it
}

bool nb_build_operator(SystemData& S) {
  if (S.nb.state != 0) return S.nb.state == 1;
  cudaStream_t s = S.ctx->stream;
  const int dpn = S.dpn;
  S.nb.state = 2;
  if (dpn < 1 || dpn > 3 || S.n_free % dpn != 0 || S.n_free == 0) return false;
  const int ng = (int)(S.n_free / dpn);
  TPT_CUDA(cudaMemsetAsync(S.ctx->d_flag, 0, sizeof(int), s));
  check_groups<<<ceil_div(ng, 256), 256, 0, s>>>(ng, dpn, S.free_map.p, S.ctx->d_flag);
  TPT_CHECK_LAUNCH();
  DevBuf<int> cnt;
  cnt.alloc(ng + 1, s);
  group_neighbours<false><<<ceil_div(ng, 128), 128, 0, s>>>(ng, dpn, S.row_ptr.p, S.col.p, cnt.p, nullptr, nullptr,
                                                             S.ctx->d_flag);
  TPT_CHECK_LAUNCH();
  int flag = 0;
  TPT_CUDA(cudaMemcpyAsync(&flag, S.ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
  TPT_CUDA(cudaStreamSynchronize(s));
  if (flag) return false;
  NbSell& N = S.nb;
  N.dpn = dpn;
  N.ngroups = ng;
  N.nchunks = ceil_div(ng, 32);
  N.gptr.alloc(ng + 1, s);
  const int64_t tot = exclusive_scan_i32(cnt.p, N.gptr.p, ng, s);
  N.glist.alloc(std::max<int64_t>(tot, 1), s);
  group_neighbours<true><<<ceil_div(ng, 128), 128, 0, s>>>(ng, dpn, S.row_ptr.p, S.col.p, nullptr, N.gptr.p,
                                                            N.glist.p, S.ctx->d_flag);
  TPT_CHECK_LAUNCH();
  const int cgrid = ceil_div((int64_t)N.nchunks * 32, 256);
  // operator K
  DevBuf<int> slots;
  slots.alloc(N.nchunks + 1, s);
  chunk_slots<<<cgrid, 256, 0, s>>>(ng, N.gptr.p, N.glist.p, 0, slots.p);
  TPT_CHECK_LAUNCH();
  N.k_cptr.alloc(N.nchunks + 1, s);
  N.k_slots = exclusive_scan_i32(slots.p, N.k_cptr.p, N.nchunks, s);
  N.full_stale = true;  // the full storage (1.7x the symmetric one) is filled when a solve asks for it
  // slot structure of L (lower) and L^T (upper)
  chunk_slots<<<cgrid, 256, 0, s>>>(ng, N.gptr.p, N.glist.p, 1, slots.p);
  TPT_CHECK_LAUNCH();
  N.l_cptr.alloc(N.nchunks + 1, s);
  N.l_slots = exclusive_scan_i32(slots.p, N.l_cptr.p, N.nchunks, s);
  chunk_slots<<<cgrid, 256, 0, s>>>(ng, N.gptr.p, N.glist.p, 2, slots.p);
  TPT_CHECK_LAUNCH();
  N.u_cptr.alloc(N.nchunks + 1, s);
  N.u_slots = exclusive_scan_i32(slots.p, N.u_cptr.p, N.nchunks, s);
  const int64_t ls = std::max<int64_t>(N.l_slots, 1) * 32, us = std::max<int64_t>(N.u_slots, 1) * 32;
  N.l_col.alloc(ls, s);
  N.u_col.alloc(us, s);
  N.u_pos.alloc(us, s);
  N.nlow.alloc(ng, s);
  N.l_pack.alloc(ls, s);
  N.l_tail.alloc(ls, s);
  N.u_pack.alloc(us, s);
  N.u_tail.alloc(us, s);
  N.l_diag.alloc((int64_t)N.nchunks * 3 * 32, s);
  N.l_diag.zero();
  factor_columns<<<ceil_div(ng, 128), 128, 0, s>>>(ng, N.gptr.p, N.glist.p, N.l_cptr.p, N.u_cptr.p, N.l_col.p,
                                                   N.u_col.p, N.u_pos.p, N.nlow.p);
  TPT_CHECK_LAUNCH();
  TPT_CUDA(cudaStreamSynchronize(s));
  N.state = 1;
  return true;
}

bool nb_factor_shape_ok(SystemData& S, const FsaiFactor& F) {
  NbSell& N = S.nb;
  cudaStream_t s = S.ctx->stream;
  if (N.state != 1) return false;
  if (!N.factor_checked) {
    TPT_CUDA(cudaMemsetAsync(S.ctx->d_flag, 0, sizeof(int), s));
    check_factor_shape<<<ceil_div(N.ngroups, 256), 256, 0, s>>>(N.ngroups, N.dpn, F.rp.p, N.nlow.p, S.ctx->d_flag);
    TPT_CHECK_LAUNCH();
    int flag = 0;
    TPT_CUDA(cudaMemcpyAsync(&flag, S.ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    TPT_CUDA(cudaStreamSynchronize(s));
    N.factor_checked = true;
    N.factor_ok = flag == 0;
  }
  return N.factor_ok;
}

bool nb_fill_factor(SystemData& S, const FsaiFactor& F) {
  NbSell& N = S.nb;
  cudaStream_t s = S.ctx->stream;
  if (!nb_factor_shape_ok(S, F)) return false;
  fill_factor<<<ceil_div(N.ngroups, 128), 128, 0, s>>>(N.ngroups, N.dpn, F.rp.p, F.va.p, N.nlow.p, N.l_cptr.p,
                                                       N.l_col.p, N.u_cptr.p, N.u_col.p, N.u_pos.p, N.l_pack.p,
                                                       N.l_tail.p, N.u_pack.p, N.u_tail.p, N.l_diag.p);
  TPT_CHECK_LAUNCH();
  return true;
}

}  // namespace tptfem
