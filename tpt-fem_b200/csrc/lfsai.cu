// lfsai.cu -- learned factorised sparse approximate inverse.
//
// A small message-passing network over the graph of the reduced matrix emits
// the FSAI factor's values on the node-block lower pattern (fsai.cu):
//   A^ = D^-1/2 A D^-1/2                       (unit diagonal, scale free)
//   h0_i  = [1, sum|a^_ij|, sum a^_ij, sum a^_ij^2, onehot(dof component), deg/40]
//   h_l+1 = tanh(Ws h_l + Wa (|A^_off| h_l) + Wb (A^_off h_l) + b)   (2 layers, width 16)
//   edge (i, j) of the pattern, j < i:
//       z_ij = tanh(U h_i + V h_j + ue a^_ij + ce),  L^_ij = we . z_ij + w0 a^_ij
//   g_i = e_i + L^_i,  q_i = g_i A^ g_i^T,  sigma^_i = q_i^-1/2
//   G^ = diag(sigma^) (I + L^)  -> SPD G^T G for any parameters, diag(G^ A^ G^T) = 1;
//   G = G^ D^-1/2, i.e. sigma_i^2 = sigma^_i^2 / d_i, L_ij = L^_ij sqrt(d_i / d_j).
// With we = 0, w0 = -1 the network starts as the first-order approximate
// inverse factor I - tril(A^).
//
// Training minimises Kaporin's condition number of G^ A^ G^T,
//   K = (tr(G^ A^ G^T) / n) / det(G^ A^ G^T)^(1/n),
// which with the diagonal scaling above is  log K = (1/n) sum_i log q_i - log det(A^) / n.
// The constant drops out: loss = (1/n) sum_i log q_i, d loss / d L^_ij = 2 (g_i A^)_j / (n q_i).
// On a fixed pattern its minimiser is the classic FSAI factor (each row's dense
// solve in fsai.cu); the network amortises those solves into a forward pass.
// Forward and backward are hand-written kernels, Adam runs on the device.
// Everything is FP32 except q (FP64 accumulation) and the final conversion of
// the factor for the solver.  Weight gradients are summed with block
// reductions and atomics (training is not bitwise reproducible; inference is).
// The matrix is taken as symmetric: the backward of A^ h uses A^ itself.
#include <cmath>
#include <cstring>

#include "lfsai.hpp"

namespace tptfem {

namespace {

constexpr int D0 = LF_D0, H = LF_H;
constexpr int LF_THREADS = 128;
static_assert(D0 % 4 == 0 && H % 4 == 0, "feature widths are read four channels at a time");
constexpr int LF_MAXM = 48;  // longest pattern row incl. the diagonal (the FSAI pattern's bound)

struct Off {  // parameter offsets (floats)
  int ws[LF_LAYERS], wa[LF_LAYERS], wb[LF_LAYERS], b[LF_LAYERS], din[LF_LAYERS];
  int U, V, ue, ce, we, w0, total;
};

Off offsets() {
  Off o;
  int p = 0;
  for (int l = 0; l < LF_LAYERS; ++l) {
    const int din = l == 0 ? D0 : H;
    o.din[l] = din;
    o.ws[l] = p; p += H * din;
    o.wa[l] = p; p += H * din;
    o.wb[l] = p; p += H * din;
    o.b[l] = p; p += H;
  }
  o.U = p; p += H * H;
  o.V = p; p += H * H;
  o.ue = p; p += H;
  o.ce = p; p += H;
  o.we = p; p += H;
  o.w0 = p; p += 1;
  o.total = p;
  return o;
}

// ---- preparation ----------------------------------------------------------------

// d^-1/2
__global__ void lf_prep(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ va,
                        double* __restrict__ dis) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double di = 1.0;
  for (int k = rp[i]; k < rp[i + 1]; ++k)
    if (ci[k] == i) di = va[k];
  dis[i] = 1.0 / sqrt(di);
}

// Sub-warp of LF_LPR lanes per row: lanes stride over the row's entries, so
// consecutive lanes read consecutive CSR entries.
constexpr int LF_LPR = 8;

__device__ __forceinline__ unsigned subwarp_mask(int width) {
  const int base = (threadIdx.x & 31) & ~(width - 1);
  return (width == 32 ? 0xffffffffu : ((1u << width) - 1u)) << base;
}

// A^ values and node features.
__global__ void lf_prep2(int n, int dpn, const int* __restrict__ rp, const int* __restrict__ ci,
                         const double* __restrict__ va, const int* __restrict__ free_map,
                         const double* __restrict__ dis, float* __restrict__ ahat, float* __restrict__ x0) {
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int i = (int)(tid / LF_LPR), l = (int)(tid % LF_LPR);
  if (i >= n) return;  // whole sub-warps leave together
  const double di = dis[i];
  float sa = 0.f, ss = 0.f, sq = 0.f;
  int deg = 0;
  for (int k = rp[i] + l; k < rp[i + 1]; k += LF_LPR) {
    const int j = ci[k];
    const float a = (float)(va[k] * di * dis[j]);
    ahat[k] = a;
    if (j != i) { sa += fabsf(a); ss += a; sq += a * a; ++deg; }
  }
  const unsigned m = subwarp_mask(LF_LPR);
  for (int o = LF_LPR / 2; o > 0; o >>= 1) {
    sa += __shfl_xor_sync(m, sa, o, LF_LPR);
    ss += __shfl_xor_sync(m, ss, o, LF_LPR);
    sq += __shfl_xor_sync(m, sq, o, LF_LPR);
    deg += __shfl_xor_sync(m, deg, o, LF_LPR);
  }
  if (l != 0) return;
  float* x = x0 + (int64_t)i * D0;
  x[0] = 1.f; x[1] = sa; x[2] = ss; x[3] = sq;
  const int comp = dpn > 1 ? free_map[i] % dpn : -1;
  x[4] = comp == 0; x[5] = comp == 1; x[6] = comp == 2;
  x[7] = deg / 40.f;
}

// A^ at the factor pattern entries (0 where A has no entry): LF_LPR lanes per
// row, one pattern entry per lane, a binary search in the row.
__global__ void lf_pattern_values(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                  const float* __restrict__ ahat, const int* __restrict__ lrp,
                                  const int* __restrict__ lci, float* __restrict__ al) {
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int i = (int)(tid / LF_LPR), l = (int)(tid % LF_LPR);
  if (i >= n) return;
  const int r0 = rp[i], r1 = rp[i + 1];
  for (int t = lrp[i] + l; t < lrp[i + 1]; t += LF_LPR) {
    const int j = lci[t];
    int lo = r0, hi = r1;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (ci[mid] < j) lo = mid + 1;
      else hi = mid;
    }
    al[t] = (lo < r1 && ci[lo] == j) ? ahat[lo] : 0.f;
  }
}

// ---- network forward ----------------------------------------------------------------

// Ya = |A^_off| X, Yb = A^_off X (rows of width DIN): DIN / 4 lanes per row,
// each accumulating four channels over the row in order (one 16-byte load of
// X per entry and lane).
template <int DIN>
__global__ void lf_agg(int n, const int* __restrict__ rp, const int* __restrict__ ci, const float* __restrict__ ahat,
                       const float* __restrict__ X, float* __restrict__ Ya, float* __restrict__ Yb) {
  constexpr int LPR = DIN / 4;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int i = (int)(tid / LPR), c4 = (int)(tid % LPR);
  if (i >= n) return;
  float4 a = make_float4(0.f, 0.f, 0.f, 0.f), b = a;
  for (int k = rp[i]; k < rp[i + 1]; ++k) {
    const int j = ci[k];
    if (j == i) continue;
    const float w = ahat[k], aw = fabsf(w);
    const float4 v = __ldg(reinterpret_cast<const float4*>(X + (int64_t)j * DIN) + c4);
    a.x += aw * v.x; a.y += aw * v.y; a.z += aw * v.z; a.w += aw * v.w;
    b.x += w * v.x; b.y += w * v.y; b.z += w * v.z; b.w += w * v.w;
  }
  reinterpret_cast<float4*>(Ya + (int64_t)i * DIN)[c4] = a;
  reinterpret_cast<float4*>(Yb + (int64_t)i * DIN)[c4] = b;
}

// H = tanh(Ws X + Wa Ya + Wb Yb + b)
template <int DIN>
__global__ void lf_layer(int n, const float* __restrict__ prm, int ows, int owa, int owb, int ob,
                         const float* __restrict__ X, const float* __restrict__ Ya, const float* __restrict__ Yb,
                         float* __restrict__ Hout) {
  __shared__ float w[3 * H * DIN + H];
  for (int t = threadIdx.x; t < H * DIN; t += blockDim.x) {
    w[t] = prm[ows + t];
    w[H * DIN + t] = prm[owa + t];
    w[2 * H * DIN + t] = prm[owb + t];
  }
  for (int t = threadIdx.x; t < H; t += blockDim.x) w[3 * H * DIN + t] = prm[ob + t];
  __syncthreads();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float x[DIN], ya[DIN], yb[DIN];
#pragma unroll
  for (int c = 0; c < DIN; ++c) {
    x[c] = X[(int64_t)i * DIN + c];
    ya[c] = Ya[(int64_t)i * DIN + c];
    yb[c] = Yb[(int64_t)i * DIN + c];
  }
#pragma unroll
  for (int o = 0; o < H; ++o) {
    float s = w[3 * H * DIN + o];
#pragma unroll
    for (int c = 0; c < DIN; ++c)
      s += w[o * DIN + c] * x[c] + w[H * DIN + o * DIN + c] * ya[c] + w[2 * H * DIN + o * DIN + c] * yb[c];
    Hout[(int64_t)i * H + o] = tanhf(s);
  }
}

// P = U h, Q = V h
__global__ void lf_head_nodes(int n, const float* __restrict__ prm, Off o, const float* __restrict__ Hh,
                              float* __restrict__ P, float* __restrict__ Q) {
  __shared__ float U[H * H], V[H * H];
  for (int t = threadIdx.x; t < H * H; t += blockDim.x) { U[t] = prm[o.U + t]; V[t] = prm[o.V + t]; }
  __syncthreads();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float h[H];
#pragma unroll
  for (int c = 0; c < H; ++c) h[c] = Hh[(int64_t)i * H + c];
#pragma unroll
  for (int a = 0; a < H; ++a) {
    float p = 0.f, qq = 0.f;
#pragma unroll
    for (int c = 0; c < H; ++c) { p += U[a * H + c] * h[c]; qq += V[a * H + c] * h[c]; }
    P[(int64_t)i * H + a] = p;
    Q[(int64_t)i * H + a] = qq;
  }
}

// L^_ij for every pattern entry: four lanes per row, each evaluating four
// channels of z_ij; the four partial sums are added across the lanes.
__global__ void lf_head_edges(int n, const float* __restrict__ prm, Off o, const int* __restrict__ lrp,
                              const int* __restrict__ lci, const float* __restrict__ al, const float* __restrict__ P,
                              const float* __restrict__ Q, float* __restrict__ lhat) {
  constexpr int LPR = H / 4;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int i = (int)(tid / LPR), c4 = (int)(tid % LPR);
  if (i >= n) return;  // whole sub-warps leave together
  float ue[4], ce[4], we[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) { ue[u] = prm[o.ue + 4 * c4 + u]; ce[u] = prm[o.ce + 4 * c4 + u]; we[u] = prm[o.we + 4 * c4 + u]; }
  const float w0 = prm[o.w0];
  const float4 p = reinterpret_cast<const float4*>(P + (int64_t)i * H)[c4];
  const unsigned m = subwarp_mask(LPR);
  for (int t = lrp[i]; t < lrp[i + 1]; ++t) {
    const int j = lci[t];
    const float a = al[t];
    const float4 q = __ldg(reinterpret_cast<const float4*>(Q + (int64_t)j * H) + c4);
    float v = we[0] * tanhf(p.x + q.x + ue[0] * a + ce[0]);
    v += we[1] * tanhf(p.y + q.y + ue[1] * a + ce[1]);
    v += we[2] * tanhf(p.z + q.z + ue[2] * a + ce[2]);
    v += we[3] * tanhf(p.w + q.w + ue[3] * a + ce[3]);
    for (int q2 = LPR / 2; q2 > 0; q2 >>= 1) v += __shfl_xor_sync(m, v, q2, LPR);
    if (c4 == 0) lhat[t] = w0 * a + v;
  }
}

// Kaporin terms, per row i with pattern P = (lower pattern of i, i) (ascending,
// i last) and g = (L^_i,P, 1):  w = A^[P,P] g,  q_i = g . w  (FP64 accumulation),
// sig_i = q_i^-1/2,  d loss / d L^_ij = 2 w_j / (n q_i),  loss += log q_i.
// One warp per row: lanes take pattern entries a and a + 32 and merge row
// P[a] of A^ with the pattern.  Rows longer than LF_MAXM set bit 0 of *flag,
// a non-positive q sets bit 1.
__global__ void __launch_bounds__(LF_THREADS) lf_kaporin_warp(int n, const int* __restrict__ rp,
                                                              const int* __restrict__ ci,
                                                              const float* __restrict__ ahat,
                                                              const int* __restrict__ lrp,
                                                              const int* __restrict__ lci,
                                                              const float* __restrict__ lhat,
                                                              float* __restrict__ sig, float* __restrict__ dlhat,
                                                              double* __restrict__ loss, int* __restrict__ flag) {
  constexpr int WPB = LF_THREADS / 32;
  __shared__ int Ps[WPB][LF_MAXM];
  __shared__ double gs[WPB][LF_MAXM];
  __shared__ double lsum[WPB];
  const int lane = threadIdx.x & 31, wb = threadIdx.x >> 5;
  const int i = blockIdx.x * WPB + wb;
  double lq = 0.0;
  if (i < n) {
    const int l0 = lrp[i], m = lrp[i + 1] - l0 + 1;
    if (m > LF_MAXM) {
      if (lane == 0) { atomicOr(flag, 1); sig[i] = 1.f; }
    } else {
      for (int a = lane; a < m - 1; a += 32) { Ps[wb][a] = lci[l0 + a]; gs[wb][a] = lhat[l0 + a]; }
      if (lane == 0) { Ps[wb][m - 1] = i; gs[wb][m - 1] = 1.0; }
      __syncwarp();
      double w[2] = {0.0, 0.0}, qp = 0.0;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int a = lane + 32 * h;
        if (a >= m) continue;
        const int r = Ps[wb][a];
        int k = rp[r], b = 0;
        const int ke = rp[r + 1];
        double sacc = 0.0;
        while (k < ke && b < m) {  // merge of two ascending lists
          const int c = ci[k], pb = Ps[wb][b];
          if (c == pb) { sacc += (double)ahat[k] * gs[wb][b]; ++k; ++b; }
          else if (c < pb) ++k;
          else ++b;
        }
        w[h] = sacc;
        qp += gs[wb][a] * sacc;
      }
      for (int o = 16; o > 0; o >>= 1) qp += __shfl_xor_sync(0xffffffffu, qp, o);
      if (!(qp > 0.0)) {
        if (lane == 0) { atomicOr(flag, 2); sig[i] = 1.f; }
      } else {
        if (lane == 0) { lq = log(qp); sig[i] = (float)(1.0 / sqrt(qp)); }
        if (dlhat) {
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int a = lane + 32 * h;
            if (a < m - 1) dlhat[l0 + a] = (float)(2.0 * w[h] / ((double)n * qp));
          }
        }
      }
    }
  }
  if (!loss) return;
  if (lane == 0) lsum[wb] = lq;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q2 = 0; q2 < WPB; ++q2) t += lsum[q2];
    atomicAdd(loss, t);
  }
}

// ---- node-block Kaporin terms --------------------------------------------------------
//
// When every free node has all its dofs free, row (g, a) of the factor has the
// pattern (all dofs of g's lower neighbour nodes, ascending; then (g, b) for
// b < a) and the rows of node g share their neighbour nodes H = (lower
// neighbours of g, g).  With g_a = (L^_(g,a), 1 at (g,a), 0 after it) on the
// dofs of H, w_a = A^[H,H] g_a and q_(g,a) = g_a . w_a; A^[H,H] is read as
// dpn x dpn blocks, so one block serves dpn^2 scalar terms of all dpn rows.

// Blocks of A^ on the node-group adjacency (zeroed beforehand): LF_LPR lanes
// per scalar row g*dpn + a stride over its entries; each entry's block is found
// by a binary search in g's neighbour groups (the list holds every group the
// node's rows reach).
__global__ void lf_blocks(int n, int dpn, const int* __restrict__ rp, const int* __restrict__ ci,
                          const float* __restrict__ ahat, const int* __restrict__ gptr, const int* __restrict__ glist,
                          float* __restrict__ ablk) {
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int row = (int)(tid / LF_LPR), l = (int)(tid % LF_LPR);
  if (row >= n) return;
  const int g = row / dpn, a = row % dpn, d2 = dpn * dpn;
  const int t0 = gptr[g], t1 = gptr[g + 1];
  for (int k = rp[row] + l; k < rp[row + 1]; k += LF_LPR) {
    const int c = ci[k], J = c / dpn, b = c % dpn;
    int lo = t0, hi = t1;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (glist[mid] < J) lo = mid + 1;
      else hi = mid;
    }
    if (lo < t1) ablk[(int64_t)lo * d2 + a * dpn + b] = ahat[k];
  }
}

// Every factor row's columns are the dofs of its node's lower neighbour groups
// (as the node-block operator lists them), then its own lower dofs.
__global__ void lf_check_blocks(int ngroups, int dpn, const int* __restrict__ lrp, const int* __restrict__ lci,
                                const int* __restrict__ gptr, const int* __restrict__ glist,
                                const int* __restrict__ nlow, int* __restrict__ flag) {
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (int64_t)ngroups * dpn) return;
  const int g = (int)(tid / dpn), a = (int)(tid % dpn);
  const int r0 = lrp[g * dpn + a], nl = nlow[g];
  if (lrp[g * dpn + a + 1] - r0 != dpn * nl + a) { atomicOr(flag, 1); return; }
  for (int p = 0; p < nl; ++p)
    for (int b = 0; b < dpn; ++b)
      if (lci[r0 + dpn * p + b] != glist[gptr[g] + p] * dpn + b) atomicOr(flag, 1);
  for (int b = 0; b < a; ++b)
    if (lci[r0 + dpn * nl + b] != g * dpn + b) atomicOr(flag, 1);
}

constexpr int KN_LANES = 8;  // lanes per node group (a structured tet mesh has 7 lower neighbours per node)

// Kaporin terms of node group g's dpn rows (see above); KN_LANES lanes per
// group, lane p owns pattern node H[p] (and H[p + KN_LANES], ...), merges that
// node's neighbour list with H and accumulates w for all dpn rows.  Same
// outputs and flags as lf_kaporin_warp.
template <int D>
__global__ void __launch_bounds__(LF_THREADS) lf_kaporin_nb(int ngroups, const int* __restrict__ gptr,
                                                            const int* __restrict__ glist,
                                                            const float* __restrict__ ablk,
                                                            const int* __restrict__ lrp, const int* __restrict__ nlow,
                                                            const float* __restrict__ lhat, float* __restrict__ sig,
                                                            float* __restrict__ dlhat, double* __restrict__ loss,
                                                            int* __restrict__ flag, int n) {
  constexpr int MAXH = LF_MAXM / D;  // the scalar kernel's row bound, in nodes
  constexpr int PASS = (MAXH + KN_LANES - 1) / KN_LANES;
  constexpr int NPB = LF_THREADS / KN_LANES;
  __shared__ int Hs[NPB][MAXH];
  __shared__ float gv[NPB][D][MAXH][D];
  __shared__ double lsum[LF_THREADS / 32];
  const int slot = threadIdx.x / KN_LANES, l = threadIdx.x % KN_LANES;
  const int g = blockIdx.x * NPB + slot;
  const unsigned mask = subwarp_mask(KN_LANES);
  double lq = 0.0;
  if (g < ngroups) {  // uniform over the sub-warp
    const int nl = nlow[g], nh = nl + 1;
    if (D * nh > LF_MAXM) {  // the longest of the group's rows has D * nl + D entries
      if (l < D) { atomicOr(flag, 1); sig[g * D + l] = 1.f; }
    } else {
      const int gp = gptr[g];
      for (int p = l; p < nh; p += KN_LANES) Hs[slot][p] = p < nl ? glist[gp + p] : g;
      for (int e = l; e < D * nh * D; e += KN_LANES) {
        const int a = e / (nh * D), p = (e / D) % nh, b = e % D;
        const int r0 = lrp[g * D + a];
        float v;
        if (p < nl) v = lhat[r0 + D * p + b];
        else v = b < a ? lhat[r0 + D * nl + b] : (b == a ? 1.f : 0.f);
        gv[slot][a][p][b] = v;
      }
      __syncwarp(mask);
      double w[PASS][D][D];
      double qp[D];
#pragma unroll
      for (int a = 0; a < D; ++a) qp[a] = 0.0;
#pragma unroll
      for (int ps = 0; ps < PASS; ++ps) {
#pragma unroll
        for (int a = 0; a < D; ++a)
#pragma unroll
          for (int b = 0; b < D; ++b) w[ps][a][b] = 0.0;
        const int p = l + ps * KN_LANES;
        if (p < nh) {
          const int h = Hs[slot][p];
          int q = 0;
          for (int t = gptr[h]; t < gptr[h + 1] && q < nh; ++t) {
            const int k = glist[t];
            while (q < nh && Hs[slot][q] < k) ++q;
            if (q < nh && Hs[slot][q] == k) {
              float bb[D * D];
#pragma unroll
              for (int u = 0; u < D * D; ++u) bb[u] = ablk[(int64_t)t * D * D + u];
#pragma unroll
              for (int a = 0; a < D; ++a)
#pragma unroll
                for (int b = 0; b < D; ++b) {
                  double acc = 0.0;
#pragma unroll
                  for (int c = 0; c < D; ++c) acc += (double)bb[b * D + c] * (double)gv[slot][a][q][c];
                  w[ps][a][b] += acc;
                }
              ++q;
            }
          }
#pragma unroll
          for (int a = 0; a < D; ++a)
#pragma unroll
            for (int b = 0; b < D; ++b) qp[a] += (double)gv[slot][a][p][b] * w[ps][a][b];
        }
      }
#pragma unroll
      for (int a = 0; a < D; ++a)
        for (int o = KN_LANES / 2; o > 0; o >>= 1) qp[a] += __shfl_xor_sync(mask, qp[a], o, KN_LANES);
#pragma unroll
      for (int a = 0; a < D; ++a) {
        const int row = g * D + a;
        if (!(qp[a] > 0.0)) {
          if (l == 0) { atomicOr(flag, 2); sig[row] = 1.f; }
          continue;
        }
        if (l == 0) { lq += log(qp[a]); sig[row] = (float)(1.0 / sqrt(qp[a])); }
        if (!dlhat) continue;
        const int r0 = lrp[row];
#pragma unroll
        for (int ps = 0; ps < PASS; ++ps) {
          const int p = l + ps * KN_LANES;
          if (p > nl) continue;
#pragma unroll
          for (int b = 0; b < D; ++b)
            if (p < nl || b < a) dlhat[r0 + D * p + b] = (float)(2.0 * w[ps][a][b] / ((double)n * qp[a]));
        }
      }
    }
  }
  if (!loss) return;
  for (int o = 16; o > 0; o >>= 1) lq += __shfl_xor_sync(0xffffffffu, lq, o);
  if ((threadIdx.x & 31) == 0) lsum[threadIdx.x >> 5] = lq;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q2 = 0; q2 < LF_THREADS / 32; ++q2) t += lsum[q2];
    atomicAdd(loss, t);
  }
}

// ---- backward -------------------------------------------------------------------------

// Block-reduce NV floats per thread, then one atomicAdd per value and block.
template <int NV>
__device__ __forceinline__ void block_atomic(float (&v)[NV], float* out) {
  __shared__ float sh[LF_THREADS / 32][NV];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < NV; ++c) {
    float x = v[c];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sh[wid][c] = x;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    float s = 0.f;
    for (int w = 0; w < LF_THREADS / 32; ++w) s += sh[w][threadIdx.x];
    atomicAdd(out + threadIdx.x, s);
  }
}

// Edge head backward: gradients of we, w0, ue, ce; dP (per row) and dQ (atomics).
__global__ void lf_head_edges_bwd(int n, const float* __restrict__ prm, Off o, float* __restrict__ grad,
                                  const int* __restrict__ lrp, const int* __restrict__ lci,
                                  const float* __restrict__ al, const float* __restrict__ P,
                                  const float* __restrict__ Q, const float* __restrict__ dlhat,
                                  float* __restrict__ dP, float* __restrict__ dQ) {
  __shared__ float ue[H], ce[H], we[H];
  for (int t = threadIdx.x; t < H; t += blockDim.x) { ue[t] = prm[o.ue + t]; ce[t] = prm[o.ce + t]; we[t] = prm[o.we + t]; }
  __syncthreads();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  float gwe[H], gue[H], gce[H], gw0[1] = {0.f};
#pragma unroll
  for (int c = 0; c < H; ++c) gwe[c] = gue[c] = gce[c] = 0.f;
  if (i < n) {
    float p[H], dp[H];
#pragma unroll
    for (int c = 0; c < H; ++c) { p[c] = P[(int64_t)i * H + c]; dp[c] = 0.f; }
    for (int t = lrp[i]; t < lrp[i + 1]; ++t) {
      const int j = lci[t];
      const float a = al[t], dl = dlhat[t];
      gw0[0] += dl * a;
#pragma unroll
      for (int c = 0; c < H; ++c) {
        const float z = tanhf(p[c] + Q[(int64_t)j * H + c] + ue[c] * a + ce[c]);
        gwe[c] += dl * z;
        const float da = dl * we[c] * (1.f - z * z);
        gue[c] += da * a;
        gce[c] += da;
        dp[c] += da;
        atomicAdd(dQ + (int64_t)j * H + c, da);
      }
    }
#pragma unroll
    for (int c = 0; c < H; ++c) dP[(int64_t)i * H + c] = dp[c];
  }
  block_atomic<H>(gwe, grad + o.we);
  __syncthreads();
  block_atomic<H>(gue, grad + o.ue);
  __syncthreads();
  block_atomic<H>(gce, grad + o.ce);
  __syncthreads();
  block_atomic<1>(gw0, grad + o.w0);
}

// out[a][b] += sum_i A_i[a] * B_i[b] (A rows of width DA, B rows of width DB); one
// thread per (a, b), rows in tiles of 32 through shared memory.
template <int DA, int DB>
__global__ void lf_outer(int n, const float* __restrict__ A, const float* __restrict__ B, float* __restrict__ out) {
  __shared__ float ta[32][DA], tb[32][DB];
  const int a = threadIdx.x / DB, b = threadIdx.x % DB;
  float s = 0.f;
  for (int base = blockIdx.x * 32; base < n; base += gridDim.x * 32) {
    for (int t = threadIdx.x; t < 32 * DA; t += blockDim.x) {
      const int r = base + t / DA;
      ta[t / DA][t % DA] = r < n ? A[(int64_t)r * DA + t % DA] : 0.f;
    }
    for (int t = threadIdx.x; t < 32 * DB; t += blockDim.x) {
      const int r = base + t / DB;
      tb[t / DB][t % DB] = r < n ? B[(int64_t)r * DB + t % DB] : 0.f;
    }
    __syncthreads();
    if (threadIdx.x < DA * DB)
      for (int r = 0; r < 32; ++r) s += ta[r][a] * tb[r][b];
    __syncthreads();
  }
  if (threadIdx.x < DA * DB) atomicAdd(out + a * DB + b, s);
}

// sum over rows of A (width D) into out[D]
template <int D>
__global__ void lf_colsum(int n, const float* __restrict__ A, float* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  float v[D];
#pragma unroll
  for (int c = 0; c < D; ++c) v[c] = i < n ? A[(int64_t)i * D + c] : 0.f;
  block_atomic<D>(v, out);
}

// Node head backward: dH = U^T dP + V^T dQ  (weight gradients via lf_outer)
__global__ void lf_head_nodes_bwd(int n, const float* __restrict__ prm, Off o, const float* __restrict__ dP,
                                  const float* __restrict__ dQ, float* __restrict__ dH) {
  __shared__ float U[H * H], V[H * H];
  for (int t = threadIdx.x; t < H * H; t += blockDim.x) { U[t] = prm[o.U + t]; V[t] = prm[o.V + t]; }
  __syncthreads();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float dp[H], dq[H];
#pragma unroll
  for (int c = 0; c < H; ++c) { dp[c] = dP[(int64_t)i * H + c]; dq[c] = dQ[(int64_t)i * H + c]; }
#pragma unroll
  for (int c = 0; c < H; ++c) {
    float s = 0.f;
#pragma unroll
    for (int a = 0; a < H; ++a) s += U[a * H + c] * dp[a] + V[a * H + c] * dq[a];
    dH[(int64_t)i * H + c] = s;
  }
}

// Layer backward, per row: dpre = dH (1 - H^2); S = Ws^T dpre; Ta = Wa^T dpre; Tb = Wb^T dpre.
template <int DIN>
__global__ void lf_layer_bwd(int n, const float* __restrict__ prm, int ows, int owa, int owb,
                             const float* __restrict__ Hout, const float* __restrict__ dH, float* __restrict__ dpre,
                             float* __restrict__ S, float* __restrict__ Ta, float* __restrict__ Tb) {
  __shared__ float w[3 * H * DIN];
  for (int t = threadIdx.x; t < H * DIN; t += blockDim.x) {
    w[t] = prm[ows + t];
    w[H * DIN + t] = prm[owa + t];
    w[2 * H * DIN + t] = prm[owb + t];
  }
  __syncthreads();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float d[H];
#pragma unroll
  for (int o = 0; o < H; ++o) {
    const float h = Hout[(int64_t)i * H + o];
    d[o] = dH[(int64_t)i * H + o] * (1.f - h * h);
    dpre[(int64_t)i * H + o] = d[o];
  }
#pragma unroll
  for (int c = 0; c < DIN; ++c) {
    float s = 0.f, a = 0.f, b = 0.f;
#pragma unroll
    for (int o = 0; o < H; ++o) {
      s += w[o * DIN + c] * d[o];
      a += w[H * DIN + o * DIN + c] * d[o];
      b += w[2 * H * DIN + o * DIN + c] * d[o];
    }
    S[(int64_t)i * DIN + c] = s;
    Ta[(int64_t)i * DIN + c] = a;
    Tb[(int64_t)i * DIN + c] = b;
  }
}

// dX = S + |A^_off| Ta + A^_off Tb
template <int DIN>
__global__ void lf_agg_bwd(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                           const float* __restrict__ ahat, const float* __restrict__ S, const float* __restrict__ Ta,
                           const float* __restrict__ Tb, float* __restrict__ dX) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s[DIN];
#pragma unroll
  for (int c = 0; c < DIN; ++c) s[c] = S[(int64_t)i * DIN + c];
  for (int k = rp[i]; k < rp[i + 1]; ++k) {
    const int j = ci[k];
    if (j == i) continue;
    const float w = ahat[k], aw = fabsf(w);
#pragma unroll
    for (int c = 0; c < DIN; ++c) s[c] += aw * Ta[(int64_t)j * DIN + c] + w * Tb[(int64_t)j * DIN + c];
  }
#pragma unroll
  for (int c = 0; c < DIN; ++c) dX[(int64_t)i * DIN + c] = s[c];
}

__global__ void lf_adam(int np, float* __restrict__ prm, const float* __restrict__ g, float* __restrict__ m1,
                        float* __restrict__ m2, float lr, float b1, float b2, float eps, float c1, float c2,
                        float clip) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  float gi = fminf(fmaxf(g[i], -clip), clip);
  m1[i] = b1 * m1[i] + (1.f - b1) * gi;
  m2[i] = b2 * m2[i] + (1.f - b2) * gi * gi;
  prm[i] -= lr * (m1[i] / c1) / (sqrtf(m2[i] / c2) + eps);
}

// FP64 factor of A from the network output: sigma^2 = sig^2 / d_i, L_ij = L^_ij sqrt(d_i / d_j).
__global__ void lf_to_factor(int n, const int* __restrict__ lrp, const int* __restrict__ lci,
                             const float* __restrict__ lhat, const float* __restrict__ sig,
                             const double* __restrict__ dis, double* __restrict__ sig2, double* __restrict__ lva) {
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int i = (int)(tid / LF_LPR), l = (int)(tid % LF_LPR);
  if (i >= n) return;
  const double di = dis[i];
  if (l == 0) {
    const double s = sig[i];
    sig2[i] = s * s * di * di;
  }
  for (int t = lrp[i] + l; t < lrp[i + 1]; t += LF_LPR) lva[t] = (double)lhat[t] * dis[lci[t]] / di;
}

int blocks(int64_t n) { return (int)((n + LF_THREADS - 1) / LF_THREADS); }

}  // namespace

int lf_param_count() { return offsets().total; }

void lf_init_params(uint64_t seed, float* h) {
  Off o = offsets();
  uint64_t st = seed * 0x9E3779B97F4A7C15ull + 12345;
  auto rnd = [&]() {  // splitmix64 -> uniform(-1, 1)
    st += 0x9E3779B97F4A7C15ull;
    uint64_t z = st;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (float)((double)(z >> 11) / 9007199254740992.0 * 2.0 - 1.0);
  };
  for (int i = 0; i < o.total; ++i) h[i] = 0.f;
  for (int l = 0; l < LF_LAYERS; ++l) {
    const float sc = 1.f / std::sqrt((float)(3 * o.din[l]));
    for (int t = 0; t < H * o.din[l]; ++t) {
      h[o.ws[l] + t] = sc * rnd();
      h[o.wa[l] + t] = sc * rnd();
      h[o.wb[l] + t] = sc * rnd();
    }
  }
  const float sh = 1.f / std::sqrt((float)H);
  for (int t = 0; t < H * H; ++t) { h[o.U + t] = sh * rnd(); h[o.V + t] = sh * rnd(); }
  for (int t = 0; t < H; ++t) { h[o.ue + t] = sh * rnd(); h[o.ce + t] = 0.1f * rnd(); }
  h[o.w0] = -1.f;  // we = 0: the first-order factor I - tril(A^)
}

void LfGraph::prepare(SystemData& S, const FsaiFactor& F) {
  cudaStream_t s = S.ctx->stream;
  n = (int)S.n_free;
  nnz = S.nnz;
  nnzl = F.nnz;
  ahat.alloc(std::max<int64_t>(nnz, 1), s);
  dis.alloc(n, s);
  x0.alloc((int64_t)n * D0, s);
  al.alloc(std::max<int64_t>(nnzl, 1), s);
  for (int l = 0; l < LF_LAYERS; ++l) {
    const int din = l == 0 ? D0 : H;
    ya[l].alloc((int64_t)n * din, s);
    yb[l].alloc((int64_t)n * din, s);
    h[l].alloc((int64_t)n * H, s);
  }
  P.alloc((int64_t)n * H, s);
  Q.alloc((int64_t)n * H, s);
  sig.alloc(n, s);
  lhat.alloc(std::max<int64_t>(nnzl, 1), s);
  flag.alloc(1, s);
  lf_prep<<<blocks(n), LF_THREADS, 0, s>>>(n, S.row_ptr.p, S.col.p, S.val.p, dis.p);
  TPT_CHECK_LAUNCH();
  lf_prep2<<<blocks((int64_t)n * LF_LPR), LF_THREADS, 0, s>>>(n, S.dpn, S.row_ptr.p, S.col.p, S.val.p, S.free_map.p, dis.p, ahat.p,
                                            x0.p);
  TPT_CHECK_LAUNCH();
  lf_pattern_values<<<blocks((int64_t)n * LF_LPR), LF_THREADS, 0, s>>>(n, S.row_ptr.p, S.col.p, ahat.p, F.rp.p, F.ci.p, al.p);
  TPT_CHECK_LAUNCH();
  if (nb_checked < 0) {  // once per system: does the factor pattern have the node-block shape?
    nb_checked = 0;
    if (S.dpn <= 3 && nb_build_operator(S) && S.nb.dpn == S.dpn) {
      const NbSell& N = S.nb;
      flag.zero();
      lf_check_blocks<<<blocks((int64_t)N.ngroups * N.dpn), LF_THREADS, 0, s>>>(N.ngroups, N.dpn, F.rp.p, F.ci.p,
                                                                             N.gptr.p, N.glist.p, N.nlow.p, flag.p);
      TPT_CHECK_LAUNCH();
      int f = 0;
      TPT_CUDA(cudaMemcpyAsync(&f, flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
      TPT_CUDA(cudaStreamSynchronize(s));
      nb_checked = f == 0 ? 1 : 0;
    }
  }
  nb = nb_checked == 1;
  if (nb) {
    const NbSell& N = S.nb;
    ablk.alloc(N.glist.n * N.dpn * N.dpn, s);
    ablk.zero();
    lf_blocks<<<blocks((int64_t)n * LF_LPR), LF_THREADS, 0, s>>>(n, N.dpn, S.row_ptr.p, S.col.p, ahat.p, N.gptr.p,
                                                                  N.glist.p, ablk.p);
    TPT_CHECK_LAUNCH();
  }
  ready = true;
}

namespace {

// Network forward to L^ and, through the Kaporin kernel, sig (and, when dlhat
// is given, the loss gradient with respect to L^; the loss sum goes to *loss).
void forward_impl(const SystemData& S, const FsaiFactor& F, LfGraph& G, const float* prm, float* dlhat,
                  double* loss) {
  cudaStream_t s = S.ctx->stream;
  const Off o = offsets();
  const int n = G.n;
  const float* in = G.x0.p;
  for (int l = 0; l < LF_LAYERS; ++l) {
    if (l == 0) {
      lf_agg<D0><<<blocks((int64_t)n * (D0 / 4)), LF_THREADS, 0, s>>>(n, S.row_ptr.p, S.col.p, G.ahat.p, in, G.ya[l].p, G.yb[l].p);
      TPT_CHECK_LAUNCH();
      lf_layer<D0><<<blocks(n), LF_THREADS, 0, s>>>(n, prm, o.ws[l], o.wa[l], o.wb[l], o.b[l], in, G.ya[l].p,
                                                    G.yb[l].p, G.h[l].p);
    } else {
      lf_agg<H><<<blocks((int64_t)n * (H / 4)), LF_THREADS, 0, s>>>(n, S.row_ptr.p, S.col.p, G.ahat.p, in, G.ya[l].p, G.yb[l].p);
      TPT_CHECK_LAUNCH();
      lf_layer<H><<<blocks(n), LF_THREADS, 0, s>>>(n, prm, o.ws[l], o.wa[l], o.wb[l], o.b[l], in, G.ya[l].p,
                                                   G.yb[l].p, G.h[l].p);
    }
    TPT_CHECK_LAUNCH();
    in = G.h[l].p;
  }
  lf_head_nodes<<<blocks(n), LF_THREADS, 0, s>>>(n, prm, o, in, G.P.p, G.Q.p);
  TPT_CHECK_LAUNCH();
  lf_head_edges<<<blocks((int64_t)n * (H / 4)), LF_THREADS, 0, s>>>(n, prm, o, F.rp.p, F.ci.p, G.al.p, G.P.p, G.Q.p, G.lhat.p);
  TPT_CHECK_LAUNCH();
  G.flag.zero();
  if (G.nb) {
    const NbSell& N = S.nb;
    const int nb_blocks = ceil_div(N.ngroups, LF_THREADS / KN_LANES);
#define TPT_LF_KN(D)                                                                                      \
  lf_kaporin_nb<D><<<nb_blocks, LF_THREADS, 0, s>>>(N.ngroups, N.gptr.p, N.glist.p, G.ablk.p, F.rp.p, N.nlow.p, \
                                                    G.lhat.p, G.sig.p, dlhat, loss, G.flag.p, n);
    if (N.dpn == 3) { TPT_LF_KN(3) }
    else if (N.dpn == 2) { TPT_LF_KN(2) }
    else { TPT_LF_KN(1) }
#undef TPT_LF_KN
  } else {
    lf_kaporin_warp<<<ceil_div(n, LF_THREADS / 32), LF_THREADS, 0, s>>>(n, S.row_ptr.p, S.col.p, G.ahat.p, F.rp.p,
                                                                        F.ci.p, G.lhat.p, G.sig.p, dlhat, loss,
                                                                        G.flag.p);
  }
  TPT_CHECK_LAUNCH();
}

}  // namespace

bool lf_forward(const SystemData& S, const FsaiFactor& F, LfGraph& G, const float* prm) {
  forward_impl(S, F, G, prm, nullptr, nullptr);
  int f = 0;
  TPT_CUDA(cudaMemcpyAsync(&f, G.flag.p, sizeof(int), cudaMemcpyDeviceToHost, S.ctx->stream));
  TPT_CUDA(cudaStreamSynchronize(S.ctx->stream));
  return f == 0;
}

double lf_loss_grad(const SystemData& S, const FsaiFactor& F, LfGraph& G, const float* prm, float* grad) {
  cudaStream_t s = S.ctx->stream;
  const Off o = offsets();
  const int n = G.n;
  DevBuf<double> loss;
  loss.alloc(1, s);
  loss.zero();
  DevBuf<float> dl;
  if (grad) dl.alloc(std::max<int64_t>(G.nnzl, 1), s);
  forward_impl(S, F, G, prm, grad ? dl.p : nullptr, loss.p);
  if (grad) {
    DevBuf<float> dP, dQ, dH, dpre, Sx, Ta, Tb, dX;
    dP.alloc((int64_t)n * H, s);
    dQ.alloc((int64_t)n * H, s);
    dQ.zero();
    dH.alloc((int64_t)n * H, s);
    dpre.alloc((int64_t)n * H, s);
    Sx.alloc((int64_t)n * H, s);
    Ta.alloc((int64_t)n * H, s);
    Tb.alloc((int64_t)n * H, s);
    dX.alloc((int64_t)n * H, s);
    lf_head_edges_bwd<<<blocks(n), LF_THREADS, 0, s>>>(n, prm, o, grad, F.rp.p, F.ci.p, G.al.p, G.P.p, G.Q.p, dl.p,
                                                       dP.p, dQ.p);
    TPT_CHECK_LAUNCH();
    const float* hl = G.h[LF_LAYERS - 1].p;
    const int og = std::min(1024, std::max(1, n / 32));
    lf_outer<H, H><<<og, 256, 0, s>>>(n, dP.p, hl, grad + o.U);
    TPT_CHECK_LAUNCH();
    lf_outer<H, H><<<og, 256, 0, s>>>(n, dQ.p, hl, grad + o.V);
    TPT_CHECK_LAUNCH();
    lf_head_nodes_bwd<<<blocks(n), LF_THREADS, 0, s>>>(n, prm, o, dP.p, dQ.p, dH.p);
    TPT_CHECK_LAUNCH();
    for (int l = LF_LAYERS - 1; l >= 0; --l) {
      const float* xin = l == 0 ? G.x0.p : G.h[l - 1].p;
      if (l == 0) {
        lf_layer_bwd<D0><<<blocks(n), LF_THREADS, 0, s>>>(n, prm, o.ws[l], o.wa[l], o.wb[l], G.h[l].p, dH.p, dpre.p,
                                                         Sx.p, Ta.p, Tb.p);
        TPT_CHECK_LAUNCH();
        lf_outer<H, D0><<<og, 256, 0, s>>>(n, dpre.p, xin, grad + o.ws[l]);
        lf_outer<H, D0><<<og, 256, 0, s>>>(n, dpre.p, G.ya[l].p, grad + o.wa[l]);
        lf_outer<H, D0><<<og, 256, 0, s>>>(n, dpre.p, G.yb[l].p, grad + o.wb[l]);
      } else {
        lf_layer_bwd<H><<<blocks(n), LF_THREADS, 0, s>>>(n, prm, o.ws[l], o.wa[l], o.wb[l], G.h[l].p, dH.p, dpre.p,
                                                        Sx.p, Ta.p, Tb.p);
        TPT_CHECK_LAUNCH();
        lf_outer<H, H><<<og, 256, 0, s>>>(n, dpre.p, xin, grad + o.ws[l]);
        lf_outer<H, H><<<og, 256, 0, s>>>(n, dpre.p, G.ya[l].p, grad + o.wa[l]);
        lf_outer<H, H><<<og, 256, 0, s>>>(n, dpre.p, G.yb[l].p, grad + o.wb[l]);
        TPT_CHECK_LAUNCH();
        lf_agg_bwd<H><<<blocks(n), LF_THREADS, 0, s>>>(n, S.row_ptr.p, S.col.p, G.ahat.p, Sx.p, Ta.p, Tb.p, dX.p);
        TPT_CHECK_LAUNCH();
        TPT_CUDA(cudaMemcpyAsync(dH.p, dX.p, (size_t)n * H * sizeof(float), cudaMemcpyDeviceToDevice, s));
      }
      TPT_CHECK_LAUNCH();
      lf_colsum<H><<<blocks(n), LF_THREADS, 0, s>>>(n, dpre.p, grad + o.b[l]);
      TPT_CHECK_LAUNCH();
    }
  }
  double h = 0.0;
  int f = 0;
  TPT_CUDA(cudaMemcpyAsync(&h, loss.p, sizeof(double), cudaMemcpyDeviceToHost, s));
  TPT_CUDA(cudaMemcpyAsync(&f, G.flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  TPT_CUDA(cudaStreamSynchronize(s));
  TPT_REQUIRE(f == 0, TPTFEM_ERR_NUMERIC,
              (f & 1) ? "learned FSAI: a factor pattern row exceeds the supported length"
                      : "learned FSAI: q_i <= 0 (the matrix is not positive definite in FP32)");
  return h / (double)n;
}

void lf_adam_step(cudaStream_t s, int np, float* prm, const float* grad, float* m1, float* m2, int step, float lr,
                  float clip) {
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, (float)step), c2 = 1.f - std::pow(b2, (float)step);
  lf_adam<<<blocks(np), LF_THREADS, 0, s>>>(np, prm, grad, m1, m2, lr, b1, b2, 1e-8f, c1, c2, clip);
  TPT_CHECK_LAUNCH();
}

void lf_factor_fp64(const SystemData& S, const FsaiFactor& F, const LfGraph& G, double* sig2, double* lva) {
  lf_to_factor<<<blocks((int64_t)G.n * LF_LPR), LF_THREADS, 0, S.ctx->stream>>>(G.n, F.rp.p, F.ci.p, G.lhat.p, G.sig.p, G.dis.p, sig2,
                                                              lva);
  TPT_CHECK_LAUNCH();
}

}  // namespace tptfem
