// coarse.cu -- aggregation coarse space with rigid-body modes for the
// two-level (additive) preconditioner  M^-1 = G^T G + P A_c^-1 P^T.
//
// The slow modes left by a sparse approximate inverse on an elongated,
// heterogeneous elastic body are smooth, near-rigid motions of large pieces
// of it.  Free mesh nodes are binned by coordinates into boxes (aggregates);
// on each aggregate the rigid-body modes (translations, and rotations about
// its centroid) span the coarse space, orthonormalised per aggregate (modes
// that an aggregate cannot carry, e.g. rotations of a single node, are
// dropped).  A_c = P^T A P is formed with one multi-vector operator product
// per colour (all modes at once): aggregates are coloured by bin coordinates
// mod 3, so an aggregate has at most one neighbour of each colour and
// P^T A (P E_colour) yields whole coarse columns without mixing.  A_c is
// factorised and inverted once per set-up, off the iteration path (cuSOLVER
// dpotrf, cuBLAS dtrsm and dsyrk), and kept as an explicit FP32 inverse, so each iteration adds one restriction, one coarse mat-vec
// and a prolongation that is fused into the FSAI transpose kernel.
// Requires the node-block layout (full node groups) and the mesh geometry.
#include <cub/device/device_radix_sort.cuh>
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <numeric>

#include "modes.cuh"
#include "objects.hpp"

namespace tptfem {

namespace {

constexpr int CS_THREADS = 256;
constexpr int CS_MAX_COARSE = 8192;

__device__ __forceinline__ int colour_of(const int* b) { return (b[0] % 3) + 3 * (b[1] % 3) + 9 * (b[2] % 3); }

// V[(g dpn + a) nm + m] = (P e_{c, m})_{g,a} for every mode m at once
// (colour < 0: every colour, i.e. P itself).
template <int DPN>
__global__ void cs_fill_modes(int ngroups, const int* __restrict__ agg, const int* __restrict__ abin,
                              const float* __restrict__ y, const double* __restrict__ T, int colour,
                              double* __restrict__ V) {
  constexpr int NM = rigid_modes(DPN);
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngroups) return;
  const int I = agg[g];
  double* out = V + (int64_t)g * DPN * NM;
  if (colour >= 0 && colour_of(abin + 3 * I) != colour) {
#pragma unroll
    for (int q = 0; q < DPN * NM; ++q) out[q] = 0.0;
    return;
  }
  double R[DPN][NM];
  mode_rows<DPN>(y + 3 * (int64_t)g, R);
  const double* t = T + (int64_t)I * NM * NM;
#pragma unroll
  for (int a = 0; a < DPN; ++a)
#pragma unroll
    for (int m = 0; m < NM; ++m) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < NM; ++k) s += R[a][k] * t[k * NM + m];
      out[a * NM + m] = s;
    }
}

// Raw moments of every column m of W (interleaved) over one segment:
// smom[(seg nm + m) nm + k] = sum over its groups of (R_g^T W_g[:, m])_k;
// groups without a neighbour of the colour are skipped.  W holds the groups
// from g0 on (0: all of them).
template <int DPN>
__global__ void __launch_bounds__(CS_THREADS) cs_moments_modes(const int* __restrict__ sbeg,
                                                               const int* __restrict__ send,
                                                               const int* __restrict__ alist,
                                                               const float* __restrict__ y,
                                                               const double* __restrict__ W,
                                                               double* __restrict__ smom,
                                                               const unsigned* __restrict__ gmask, int colour,
                                                               int g0) {
  constexpr int NM = rigid_modes(DPN);
  __shared__ double sh[CS_THREADS / 32][NM * NM];
  const int seg = blockIdx.x;
  double s[NM * NM];
#pragma unroll
  for (int q = 0; q < NM * NM; ++q) s[q] = 0.0;
  for (int t = sbeg[seg] + threadIdx.x; t < send[seg]; t += CS_THREADS) {
    const int g = alist[t];
    if (!((gmask[g] >> colour) & 1u)) continue;  // W_g is zero (and not written) for this colour
    double R[DPN][NM];
    mode_rows<DPN>(y + 3 * (int64_t)g, R);
    const double* wg = W + (int64_t)(g - g0) * DPN * NM;
#pragma unroll
    for (int a = 0; a < DPN; ++a)
#pragma unroll
      for (int m = 0; m < NM; ++m) {
        const double wa = wg[a * NM + m];
#pragma unroll
        for (int k = 0; k < NM; ++k) s[m * NM + k] += R[a][k] * wa;
      }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NM * NM; ++q) {
    double x = s[q];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sh[wid][q] = x;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < NM * NM; q += CS_THREADS) {
    double x = 0.0;
    for (int w = 0; w < CS_THREADS / 32; ++w) x += sh[w][q];
    smom[(int64_t)seg * NM * NM + q] = x;
  }
}

// Raw mode moments of one segment of an aggregate's group list:
// smom[seg][k] = sum over its groups of (R_g^T w_g)_k, block-reduced in a
// fixed order (w holds the groups from g0 on).
template <int DPN>
__global__ void __launch_bounds__(CS_THREADS) cs_moments(const int* __restrict__ sbeg, const int* __restrict__ send,
                                                         const int* __restrict__ alist, const float* __restrict__ y,
                                                         const double* __restrict__ w, double* __restrict__ smom,
                                                         int g0, const int* __restrict__ done = nullptr) {
  if (done && *done) return;  // the PCG iteration this belongs to was not needed
  constexpr int NM = rigid_modes(DPN);
  __shared__ double sh[CS_THREADS / 32][NM];
  const int seg = blockIdx.x;
  double s[NM];
#pragma unroll
  for (int k = 0; k < NM; ++k) s[k] = 0.0;
  for (int t = sbeg[seg] + threadIdx.x; t < send[seg]; t += CS_THREADS) {
    const int g = alist[t];
    double R[DPN][NM];
    mode_rows<DPN>(y + 3 * (int64_t)g, R);
#pragma unroll
    for (int a = 0; a < DPN; ++a) {
      const double wa = w[(int64_t)(g - g0) * DPN + a];
#pragma unroll
      for (int k = 0; k < NM; ++k) s[k] += R[a][k] * wa;
    }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NM; ++k) {
    double x = s[k];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sh[wid][k] = x;
  }
  __syncthreads();
  if (threadIdx.x < NM) {
    double x = 0.0;
    for (int q = 0; q < CS_THREADS / 32; ++q) x += sh[q][threadIdx.x];
    smom[(int64_t)seg * NM + threadIdx.x] = x;
  }
}

// Orthonormal-mode moments of aggregate I: T_I^T (sum of its segments' raw moments).
__device__ __forceinline__ double agg_moment(int I, int mp, int nm, const int* __restrict__ aseg,
                                             const double* __restrict__ smom, const double* __restrict__ T) {
  const double* t = T + (int64_t)I * nm * nm;
  double x = 0.0;
  for (int k = 0; k < nm; ++k) {
    double sk = 0.0;
    for (int q = aseg[I]; q < aseg[I + 1]; ++q) sk += smom[(int64_t)q * nm + k];
    x += t[k * nm + mp] * sk;
  }
  return x;
}

// yc = P^T r from the segment moments.
__global__ void cs_yc(int na, int nm, const int* __restrict__ aseg, const double* __restrict__ smom,
                      const double* __restrict__ T, double* __restrict__ yc, const int* __restrict__ done = nullptr) {
  if (done && *done) return;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < na * nm) yc[j] = agg_moment(j / nm, j % nm, nm, aseg, smom, T);
}

// uc = A_c^-1 yc: one warp per row, FP32 matrix (row stride ld, a multiple of
// 4, zero-padded), FP64 accumulation.  Each lane reads two adjacent matrix
// entries and the matching two coarse-vector entries (16 contiguous bytes per
// lane, so the shared-memory reads are conflict-free); eight loads per lane are
// kept in flight.
__global__ void __launch_bounds__(CS_THREADS) cs_gemv(int nc, int ld, const double* __restrict__ yc,
                                                      const float* __restrict__ Ainv, double* __restrict__ uc,
                                                      const int* __restrict__ done = nullptr) {
  if (done && *done) return;
  extern __shared__ double ys[];
  for (int j = threadIdx.x; j < ld; j += blockDim.x) ys[j] = j < nc ? yc[j] : 0.0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int row = blockIdx.x * (CS_THREADS / 32) + (threadIdx.x >> 5);
  if (row >= nc) return;
  const float2* a = reinterpret_cast<const float2*>(Ainv + (int64_t)row * ld);
  const double2* y2 = reinterpret_cast<const double2*>(ys);
  const int n2 = ld >> 1;
  double s = 0.0;
#pragma unroll 8
  for (int j = lane; j < n2; j += 32) {
    const float2 v = a[j];
    const double2 w = y2[j];
    s += (double)v.x * w.x;
    s += (double)v.y * w.y;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) uc[row] = s;
}

// cm = T uc per aggregate (raw-mode coefficients of P uc).
__global__ void cs_raw(int na, int nm, const double* __restrict__ T, const double* __restrict__ uc,
                       double* __restrict__ cm, const int* __restrict__ done = nullptr) {
  if (done && *done) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= na * nm) return;
  const int I = t / nm, k = t % nm;
  const double* tI = T + (int64_t)I * nm * nm + k * nm;
  double x = 0.0;
  for (int m = 0; m < nm; ++m) x += tI[m] * uc[(int64_t)I * nm + m];
  cm[t] = x;
}

// gid[g] = g and the group count of every aggregate (input of the group-list sort).
__global__ void cs_iota_count(int ngroups, const int* __restrict__ agg, int* __restrict__ gid, int* __restrict__ cnt) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngroups) return;
  gid[g] = g;
  atomicAdd(&cnt[agg[g]], 1);
}

__global__ void cs_group_colour(int ngroups, const int* __restrict__ agg, const int* __restrict__ abin,
                                unsigned char* __restrict__ gcol) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < ngroups) gcol[g] = (unsigned char)colour_of(abin + 3 * agg[g]);
}

// Per group, the colours among its neighbour groups (itself included); per
// chunk of 32 groups, their union.
__global__ void cs_colour_masks(int ngroups, const int* __restrict__ gptr, const int* __restrict__ glist,
                                const unsigned char* __restrict__ gcol, unsigned* __restrict__ gmask,
                                unsigned* __restrict__ cmask) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngroups) return;
  unsigned m = 0;
  for (int t = gptr[g]; t < gptr[g + 1]; ++t) m |= 1u << gcol[glist[t]];
  gmask[g] = m;
  atomicOr(cmask + (g >> 5), m);
}

// Column blocks (J, m) of A_c, one thread per (I, m, mp): J is I's unique
// neighbour (itself included) of the colour; the moments of W = A P E_colour
// give entry (I mp, J m).
__global__ void cs_columns_par(int na, int nm, const int* __restrict__ abin, const int* __restrict__ bin2agg, int bx,
                               int by, int bz, const int* __restrict__ aseg, const double* __restrict__ smom,
                               const double* __restrict__ T, int colour, double* __restrict__ Ac, int nc) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= na * nm * nm) return;
  const int I = t / (nm * nm), m = (t / nm) % nm, mp = t % nm;
  const int nbin[3] = {bx, by, bz};
  int jb[3];
  for (int d = 0; d < 3; ++d) {
    const int want = (colour / (d == 0 ? 1 : (d == 1 ? 3 : 9))) % 3;
    const int b = abin[3 * I + d];
    jb[d] = -1;
    for (int o = -1; o <= 1; ++o) {
      const int c = b + o;
      if (c >= 0 && c < nbin[d] && c % 3 == want) jb[d] = c;
    }
    if (jb[d] < 0) return;
  }
  const int J = bin2agg[((int64_t)jb[2] * by + jb[1]) * bx + jb[0]];
  if (J < 0) return;
  const double* tI = T + (int64_t)I * nm * nm;
  double x = 0.0;
  for (int k = 0; k < nm; ++k) {
    double sk = 0.0;
    for (int q = aseg[I]; q < aseg[I + 1]; ++q) sk += smom[((int64_t)q * nm + m) * nm + k];
    x += tI[k * nm + mp] * sk;
  }
  Ac[((int64_t)I * nm + mp) * nc + (int64_t)J * nm + m] = x;
}

// Rows/columns of dropped modes are zero: put 1 on their diagonal.
__global__ void cs_fix_diag(int nc, double* __restrict__ Ac) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nc && Ac[(int64_t)i * nc + i] == 0.0) Ac[(int64_t)i * nc + i] = 1.0;
}

// The n x n identity (column-major = row-major).
__global__ void cs_identity(int nc, double* __restrict__ out) {
  int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= (int64_t)nc * nc) return;
  out[id] = (id / nc == id % nc) ? 1.0 : 0.0;
}

// The inverse is left in one triangle (column-major lower = row-major
// upper of the stored array): mirror it and convert to FP32.
// Rows of out have stride ld >= nc; the padding columns are zero.
__global__ void cs_symmetrize(int nc, int ld, const double* __restrict__ A, float* __restrict__ out) {
  int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= (int64_t)nc * ld) return;
  const int i = (int)(id / ld), j = (int)(id % ld);
  if (j >= nc) { out[id] = 0.0f; return; }
  // column-major lower triangle: element (r, c) with r >= c at A[c * nc + r]
  const int r = i > j ? i : j, c = i > j ? j : i;
  out[id] = (float)A[(int64_t)c * nc + r];
}

// Every operator block (g, h) must join aggregates at most one bin apart.
__global__ void cs_check_adjacency(int ngroups, const int* __restrict__ gptr, const int* __restrict__ glist,
                                   const int* __restrict__ gbin, int* __restrict__ flag) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngroups) return;
  for (int t = gptr[g]; t < gptr[g + 1]; ++t) {
    const int h = glist[t];
    for (int d = 0; d < 3; ++d)
      if (abs(gbin[3 * g + d] - gbin[3 * h + d]) > 1) atomicOr(flag, 1);
  }
}

// ---- geometry of the coarse space (device) ----------------------------------------

// Node position of every group (its first dof's node), zero-padded to 3-D.
__global__ void cs_positions(int ngroups, int dpn, int cdim, const int* __restrict__ free_map,
                             const double* __restrict__ coords, double* __restrict__ pos) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngroups) return;
  const int node = free_map[(int64_t)g * dpn] / dpn;
  for (int d = 0; d < 3; ++d) pos[(int64_t)g * 3 + d] = d < cdim ? coords[(int64_t)node * cdim + d] : 0.0;
}

// Per-block min (part[6b..6b+2]) and max (part[6b+3..]) of the positions.
__global__ void __launch_bounds__(CS_THREADS) cs_bbox(int ngroups, const double* __restrict__ pos,
                                                      double* __restrict__ part) {
  __shared__ double sh[CS_THREADS][6];
  double v[6] = {1e300, 1e300, 1e300, -1e300, -1e300, -1e300};
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ngroups; g += gridDim.x * blockDim.x)
    for (int d = 0; d < 3; ++d) {
      const double x = pos[(int64_t)g * 3 + d];
      v[d] = fmin(v[d], x);
      v[3 + d] = fmax(v[3 + d], x);
    }
  for (int q = 0; q < 6; ++q) sh[threadIdx.x][q] = v[q];
  __syncthreads();
  for (int st = CS_THREADS / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int q = 0; q < 6; ++q)
        sh[threadIdx.x][q] = q < 3 ? fmin(sh[threadIdx.x][q], sh[threadIdx.x + st][q])
                                   : fmax(sh[threadIdx.x][q], sh[threadIdx.x + st][q]);
    __syncthreads();
  }
  if (threadIdx.x < 6) part[(int64_t)blockIdx.x * 6 + threadIdx.x] = sh[0][threadIdx.x];
}

// Bin of every group: k_d = min(bins_d - 1, floor((x_d - lo_d) / L_d * bins_d)).
__global__ void cs_bin(int ngroups, const double* __restrict__ pos, double lx, double ly, double lz, double Lx,
                       double Ly, double Lz, int bx, int by, int bz, int* __restrict__ gbin, int* __restrict__ binid,
                       int* __restrict__ used) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngroups) return;
  const double lo[3] = {lx, ly, lz}, L[3] = {Lx, Ly, Lz};
  const int nb[3] = {bx, by, bz};
  int64_t b = 0;
  for (int d = 2; d >= 0; --d) {
    int k = 0;
    if (L[d] > 0) k = min(nb[d] - 1, (int)floor((pos[(int64_t)g * 3 + d] - lo[d]) / L[d] * nb[d]));
    k = max(k, 0);
    gbin[(int64_t)g * 3 + d] = k;
    b = b * nb[d] + k;
  }
  binid[g] = (int)b;
  used[b] = 1;
}

__global__ void cs_mark_empty(int64_t nbins, const int* __restrict__ used, int* __restrict__ bin2agg) {
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nbins && !used[b]) bin2agg[b] = -1;
}

__global__ void cs_group_agg(int ngroups, const int* __restrict__ binid, const int* __restrict__ bin2agg,
                             int* __restrict__ agg) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < ngroups) agg[g] = bin2agg[binid[g]];
}

// Per aggregate (one block): centroid (stats[0..2]) and inertia about it
// (stats[3..11], sum |y|^2 I - y y^T), in a fixed summation order; bin of
// its first group.
__global__ void __launch_bounds__(CS_THREADS) cs_aggregate_stats(const int* __restrict__ aptr,
                                                                 const int* __restrict__ alist,
                                                                 const double* __restrict__ pos,
                                                                 const int* __restrict__ gbin,
                                                                 double* __restrict__ stats, int* __restrict__ abin) {
  __shared__ double sh[CS_THREADS][9];
  __shared__ double cen[3];
  const int A = blockIdx.x, b0 = aptr[A], b1 = aptr[A + 1];
  double v[9];
  for (int q = 0; q < 3; ++q) v[q] = 0.0;
  for (int t = b0 + threadIdx.x; t < b1; t += CS_THREADS)
    for (int d = 0; d < 3; ++d) v[d] += pos[(int64_t)alist[t] * 3 + d];
  for (int q = 0; q < 3; ++q) sh[threadIdx.x][q] = v[q];
  __syncthreads();
  for (int st = CS_THREADS / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int q = 0; q < 3; ++q) sh[threadIdx.x][q] += sh[threadIdx.x + st][q];
    __syncthreads();
  }
  if (threadIdx.x < 3) cen[threadIdx.x] = sh[0][threadIdx.x] / (double)(b1 - b0);
  __syncthreads();
  for (int q = 0; q < 9; ++q) v[q] = 0.0;
  for (int t = b0 + threadIdx.x; t < b1; t += CS_THREADS) {
    double y[3];
    for (int d = 0; d < 3; ++d) y[d] = pos[(int64_t)alist[t] * 3 + d] - cen[d];
    const double y2 = y[0] * y[0] + y[1] * y[1] + y[2] * y[2];
    for (int a = 0; a < 3; ++a)
      for (int c = 0; c < 3; ++c) v[a * 3 + c] += (a == c ? y2 : 0.0) - y[a] * y[c];
  }
  __syncthreads();
  for (int q = 0; q < 9; ++q) sh[threadIdx.x][q] = v[q];
  __syncthreads();
  for (int st = CS_THREADS / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int q = 0; q < 9; ++q) sh[threadIdx.x][q] += sh[threadIdx.x + st][q];
    __syncthreads();
  }
  if (threadIdx.x < 3) stats[(int64_t)A * 12 + threadIdx.x] = cen[threadIdx.x];
  if (threadIdx.x < 9) stats[(int64_t)A * 12 + 3 + threadIdx.x] = sh[0][threadIdx.x];
  if (threadIdx.x < 3) abin[A * 3 + threadIdx.x] = gbin[(int64_t)alist[b0] * 3 + threadIdx.x];
}

// y_g = position minus its aggregate's centroid (FP32).
__global__ void cs_relative(int ngroups, const int* __restrict__ agg, const double* __restrict__ pos,
                            const double* __restrict__ stats, float* __restrict__ y) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngroups) return;
  const int A = agg[g];
  for (int d = 0; d < 3; ++d)
    y[(int64_t)g * 3 + d] = (float)(pos[(int64_t)g * 3 + d] - stats[(int64_t)A * 12 + d]);
}

// Eigen-decomposition of a symmetric 3x3 matrix by cyclic Jacobi rotations
// (host, once per aggregate): A = V diag(w) V^T, V column-major in v[3][3].
void sym_eig3(double a[3][3], double w[3], double v[3][3]) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) v[i][j] = i == j;
  for (int sweep = 0; sweep < 50; ++sweep) {
    const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
    const double tr = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
    if (off <= 1e-30 * (tr + 1e-300)) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        if (a[p][q] == 0.0) continue;
        const double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < 3; ++k) {  // A <- A J
          const double akp = a[k][p], akq = a[k][q];
          a[k][p] = c * akp - s * akq;
          a[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 3; ++k) {  // A <- J^T A
          const double apk = a[p][k], aqk = a[q][k];
          a[p][k] = c * apk - s * aqk;
          a[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 3; ++k) {
          const double vkp = v[k][p], vkq = v[k][q];
          v[k][p] = c * vkp - s * vkq;
          v[k][q] = s * vkp + c * vkq;
        }
      }
  }
  for (int i = 0; i < 3; ++i) w[i] = a[i][i];
}

// One rank's rows of W = A (P E_colour) for every mode at once (a partitioned
// system: local CSR rows, gcol mapping local columns to global reduced
// indices): W[i nm + m] = sum over row i of a_ij P[j, m], the columns j of
// aggregates of the colour only.  One thread per row, entries in row order.
template <int DPN>
__global__ void cs_local_apply(int64_t nloc, const int* __restrict__ rp, const int* __restrict__ ci,
                               const double* __restrict__ va, const int* __restrict__ gcol,
                               const double* __restrict__ Pfull, const unsigned char* __restrict__ gcolour,
                               int colour, double* __restrict__ W) {
  constexpr int NM = rigid_modes(DPN);
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nloc) return;
  double s[NM];
#pragma unroll
  for (int m = 0; m < NM; ++m) s[m] = 0.0;
  for (int k = rp[i]; k < rp[i + 1]; ++k) {
    const int j = gcol[ci[k]];
    if (gcolour[j / DPN] != colour) continue;
    const double a = va[k];
    const double* pj = Pfull + (int64_t)j * NM;
#pragma unroll
    for (int m = 0; m < NM; ++m) s[m] += a * pj[m];
  }
#pragma unroll
  for (int m = 0; m < NM; ++m) W[i * NM + m] = s[m];
}

int blocks_for(int64_t n) { return (int)((n + CS_THREADS - 1) / CS_THREADS); }

}  // namespace

bool coarse_build(SystemData& S, int target) {
  CoarseSpace& C = S.coarse;
  if (C.state && C.target == target) return C.state == 1;
  C.state = 2;
  C.target = target;
  C.ready = false;
  ++C.generation;
  if (!S.mesh || S.nb.state != 1 || S.dpn < 1 || S.dpn > 3) return false;
  cudaStream_t s = S.ctx->stream;
  const MeshData& M = *S.mesh;
  const int dpn = S.dpn, ng = S.nb.ngroups, nm = rigid_modes(dpn), cdim = M.cdim;
  PhaseTimer tall(s, "coarse geometry");
  // node position of every group and the bounding box (device)
  DevBuf<double> pos, part;
  pos.alloc((size_t)ng * 3, s);
  const int pb = std::min(1024, blocks_for(ng));
  part.alloc((size_t)pb * 6, s);
  cs_positions<<<blocks_for(ng), CS_THREADS, 0, s>>>(ng, dpn, cdim, S.free_map.p, M.coords.p, pos.p);
  TPT_CHECK_LAUNCH();
  cs_bbox<<<pb, CS_THREADS, 0, s>>>(ng, pos.p, part.p);
  TPT_CHECK_LAUNCH();
  std::vector<double> hp((size_t)pb * 6);
  part.download(hp.data(), hp.size());
  TPT_CUDA(cudaStreamSynchronize(s));
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int q = 0; q < pb; ++q)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], hp[(size_t)q * 6 + d]);
      hi[d] = std::max(hi[d], hp[(size_t)q * 6 + 3 + d]);
    }
  double L[3], vol = 1.0;
  int nact = 0;
  for (int d = 0; d < 3; ++d) {
    L[d] = d < cdim ? hi[d] - lo[d] : 0.0;
    if (L[d] > 0) { vol *= L[d]; ++nact; }
  }
  if (nact == 0 || target < 1) return false;
  double H = std::pow(vol / (double)target, 1.0 / nact);
  // bins (device), non-empty bins -> aggregates, adjacency check; coarsen until valid
  DevBuf<int> gbin, binid, used, flag;
  gbin.alloc((size_t)ng * 3, s);
  binid.alloc(ng, s);
  flag.alloc(1, s);
  int na = 0;
  bool ok = false;
  for (int attempt = 0; attempt < 12 && !ok; ++attempt, H *= 1.25) {
    for (int d = 0; d < 3; ++d) C.bins[d] = L[d] > 0 ? std::max(1, (int)std::floor(L[d] / H)) : 1;
    const int64_t nbins = (int64_t)C.bins[0] * C.bins[1] * C.bins[2];
    if (nbins > (1 << 24)) continue;
    used.alloc(nbins + 1, s);
    used.zero();
    cs_bin<<<blocks_for(ng), CS_THREADS, 0, s>>>(ng, pos.p, lo[0], lo[1], lo[2], L[0], L[1], L[2], C.bins[0],
                                                   C.bins[1], C.bins[2], gbin.p, binid.p, used.p);
    TPT_CHECK_LAUNCH();
    C.bin2agg.alloc(nbins + 1, s);
    na = (int)exclusive_scan_i32(used.p, C.bin2agg.p, nbins, s);  // rank of each non-empty bin
    if ((int64_t)na * nm > CS_MAX_COARSE) continue;
    flag.zero();
    cs_check_adjacency<<<blocks_for(ng), CS_THREADS, 0, s>>>(ng, S.nb.gptr.p, S.nb.glist.p, gbin.p, flag.p);
    TPT_CHECK_LAUNCH();
    int f = 0;
    flag.download(&f, 1);
    TPT_CUDA(cudaStreamSynchronize(s));
    ok = f == 0;
    if (ok) {  // empty bins -> -1
      cs_mark_empty<<<blocks_for(nbins), CS_THREADS, 0, s>>>(nbins, used.p, C.bin2agg.p);
      TPT_CHECK_LAUNCH();
    }
  }
  if (!ok) return false;
  // aggregate of every group; the groups of each aggregate in ascending order
  // by a stable radix sort of (aggregate, group) on the device, and the
  // aggregates' offsets from their counts
  C.agg.alloc(ng, s);
  cs_group_agg<<<blocks_for(ng), CS_THREADS, 0, s>>>(ng, binid.p, C.bin2agg.p, C.agg.p);
  TPT_CHECK_LAUNCH();
  std::vector<int> aptr(na + 1, 0);
  C.alist.alloc(ng, s);
  {
    DevBuf<int> gid, skey, acnt;
    gid.alloc(ng, s);
    skey.alloc(ng, s);
    acnt.alloc(na + 1, s);
    acnt.zero();
    cs_iota_count<<<blocks_for(ng), CS_THREADS, 0, s>>>(ng, C.agg.p, gid.p, acnt.p);
    TPT_CHECK_LAUNCH();
    int bits = 1;
    while ((1 << bits) < na) ++bits;
    size_t tmp_bytes = 0;
    TPT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, C.agg.p, skey.p, gid.p, C.alist.p, ng, 0, bits, s));
    DevBuf<unsigned char> tmp;
    tmp.alloc(std::max<size_t>(tmp_bytes, 1), s);
    TPT_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, C.agg.p, skey.p, gid.p, C.alist.p, ng, 0, bits, s));
    std::vector<int> cnt(na);
    acnt.download(cnt.data(), na);
    TPT_CUDA(cudaStreamSynchronize(s));
    for (int i = 0; i < na; ++i) aptr[i + 1] = aptr[i] + cnt[i];
  }
  constexpr int CS_SEG = 1024;  // segments of at most CS_SEG groups (restriction work items)
  std::vector<int> sb, se, aseg(na + 1, 0);
  for (int i = 0; i < na; ++i) {
    for (int t = aptr[i]; t < aptr[i + 1]; t += CS_SEG) {
      sb.push_back(t);
      se.push_back(std::min(aptr[i + 1], t + CS_SEG));
    }
    aseg[i + 1] = (int)sb.size();
  }
  C.na = na;
  C.nm = nm;
  C.nc = na * nm;
  C.nseg = (int)sb.size();
  C.aptr.alloc(na + 1, s); C.aptr.upload(aptr.data(), na + 1);
  C.sbeg.alloc(C.nseg, s); C.sbeg.upload(sb.data(), C.nseg);
  C.send.alloc(C.nseg, s); C.send.upload(se.data(), C.nseg);
  C.aseg.alloc(na + 1, s); C.aseg.upload(aseg.data(), na + 1);
  C.smom.alloc((size_t)C.nseg * nm, s);
  // centroids, relative positions, inertia (device); mode transforms (host, per aggregate)
  DevBuf<double> stats;
  stats.alloc((size_t)na * 12, s);
  C.abin.alloc((size_t)na * 3, s);
  cs_aggregate_stats<<<na, CS_THREADS, 0, s>>>(C.aptr.p, C.alist.p, pos.p, gbin.p, stats.p, C.abin.p);
  TPT_CHECK_LAUNCH();
  C.y.alloc((size_t)ng * 3, s);
  cs_relative<<<blocks_for(ng), CS_THREADS, 0, s>>>(ng, C.agg.p, pos.p, stats.p, C.y.p);
  TPT_CHECK_LAUNCH();
  std::vector<double> st((size_t)na * 12);
  stats.download(st.data(), st.size());
  TPT_CUDA(cudaStreamSynchronize(s));
  std::vector<double> T((size_t)na * nm * nm, 0.0);
  for (int i = 0; i < na; ++i) {
    double* t = T.data() + (size_t)i * nm * nm;
    const double cnt = aptr[i + 1] - aptr[i];
    const double* in = st.data() + (size_t)i * 12 + 3;  // inertia, row-major 3 x 3
    for (int k = 0; k < dpn; ++k) t[k * nm + k] = 1.0 / std::sqrt(cnt);
    if (dpn == 2) {
      const double iz = in[8];  // sum of |y|^2 in the plane
      if (iz > 1e-12 * cnt * H * H) t[2 * nm + 2] = 1.0 / std::sqrt(iz);
    } else if (dpn == 3) {
      double a[3][3], w[3], v[3][3];
      for (int p2 = 0; p2 < 3; ++p2)
        for (int q = 0; q < 3; ++q) a[p2][q] = in[p2 * 3 + q];
      sym_eig3(a, w, v);
      const double wmax = std::max(w[0], std::max(w[1], w[2]));
      for (int q = 0; q < 3; ++q) {
        if (!(w[q] > 1e-9 * wmax) || !(wmax > 1e-12 * cnt * H * H)) continue;
        const double sc = 1.0 / std::sqrt(w[q]);
        for (int p2 = 0; p2 < 3; ++p2) t[(3 + p2) * nm + 3 + q] = v[p2][q] * sc;
      }
    }
  }
  C.T.alloc(T.size(), s); C.T.upload(T.data(), T.size());
  TPT_CUDA(cudaFuncSetAttribute(cs_gemv, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(CS_MAX_COARSE * sizeof(double))));
  C.Ac.alloc((size_t)C.nc * C.nc, s);
  C.info.alloc(1, s);  // on the context's stream, which outlives the engines' second streams
  C.ld = (C.nc + 3) & ~3;
  C.Ainv.alloc((size_t)C.nc * C.ld, s);
  C.yc.alloc(C.nc, s);
  C.uc.alloc(C.nc, s);
  C.cm.alloc(C.nc, s);
  C.Pfull.alloc((size_t)S.n_free * nm, s);
  C.gcolour.alloc(ng, s);
  cs_group_colour<<<blocks_for(ng), CS_THREADS, 0, s>>>(ng, C.agg.p, C.abin.p, C.gcolour.p);
  TPT_CHECK_LAUNCH();
  C.gmask.alloc(ng, s);
  C.cmask.alloc(S.nb.nchunks, s);
  C.cmask.zero();
  cs_colour_masks<<<blocks_for(ng), CS_THREADS, 0, s>>>(ng, S.nb.gptr.p, S.nb.glist.p, C.gcolour.p, C.gmask.p,
                                                         C.cmask.p);
  TPT_CHECK_LAUNCH();
#define TPT_CS_P(D)                                                                                       \
  cs_fill_modes<D><<<blocks_for(ng), CS_THREADS, 0, s>>>(ng, C.agg.p, C.abin.p, C.y.p, C.T.p, -1, C.Pfull.p); \
  TPT_CHECK_LAUNCH();
  if (dpn == 3) { TPT_CS_P(3) }
  else if (dpn == 2) { TPT_CS_P(2) }
  else { TPT_CS_P(1) }
#undef TPT_CS_P
  TPT_CUDA(cudaStreamSynchronize(s));  // host vectors above are released on return
  C.state = 1;
  return true;
}

bool coarse_assemble(SystemData& S) {
  if (!coarse_assemble_async(S, S.ctx->stream)) return false;
  return coarse_finish(S, S.ctx->stream);
}

bool coarse_finish(SystemData& S, cudaStream_t s) {
  CoarseSpace& C = S.coarse;
  int hinfo = 0;
  TPT_CUDA(cudaMemcpyAsync(&hinfo, C.info.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  TPT_CUDA(cudaStreamSynchronize(s));
  C.ready = hinfo == 0;  // otherwise the coarse matrix was not positive definite in FP64
  return C.ready;
}

bool coarse_assemble_async(SystemData& S, cudaStream_t s) {
  CoarseSpace& C = S.coarse;
  C.ready = false;
  if (C.state != 1) return false;
  const int dpn = S.dpn, nc = C.nc;
  TPT_CUDA(cudaMemsetAsync(C.Ac.p, 0, (size_t)nc * nc * sizeof(double), s));
  DevBuf<double> w, mom;
  w.alloc(S.n_free * C.nm, s);
  mom.alloc((size_t)C.nseg * C.nm * C.nm, s);
  const int ncx = std::min(3, C.bins[0]), ncy = std::min(3, C.bins[1]), ncz = std::min(3, C.bins[2]);
  for (int cz = 0; cz < ncz; ++cz)
    for (int cy = 0; cy < ncy; ++cy)
      for (int cx = 0; cx < ncx; ++cx) {
        const int colour = cx + 3 * cy + 9 * cz;
        nb_operator_apply_modes(S, C.Pfull.p, w.p, C.gcolour.p, colour, C.cmask.p, s);
#define TPT_CS_COL(D)                                                                                             \
  cs_moments_modes<D><<<C.nseg, CS_THREADS, 0, s>>>(C.sbeg.p, C.send.p, C.alist.p, C.y.p, w.p, mom.p, C.gmask.p,   \
                                                    colour, 0);                                                   \
  TPT_CHECK_LAUNCH();
        if (dpn == 3) { TPT_CS_COL(3) }
        else if (dpn == 2) { TPT_CS_COL(2) }
        else { TPT_CS_COL(1) }
#undef TPT_CS_COL
        cs_columns_par<<<blocks_for((int64_t)C.na * C.nm * C.nm), CS_THREADS, 0, s>>>(
            C.na, C.nm, C.abin.p, C.bin2agg.p, C.bins[0], C.bins[1], C.bins[2], C.aseg.p, mom.p, C.T.p, colour,
            C.Ac.p, nc);
        TPT_CHECK_LAUNCH();
      }
  coarse_factor_async(S.ctx, s, nc, C.ld, C.Ac.p, C.Ainv.p, C.info.p);
  return true;
}

bool coarse_factor(tptfem_context* ctx, int nc, int ld, double* Ac, float* Ainv) {
  cudaStream_t s = ctx->stream;
  DevBuf<int> info;
  info.alloc(1, s);
  coarse_factor_async(ctx, s, nc, ld, Ac, Ainv, info.p);
  int hinfo = 0;
  info.download(&hinfo, 1);
  TPT_CUDA(cudaStreamSynchronize(s));
  return hinfo == 0;  // otherwise not positive definite in FP64
}

void coarse_factor_async(tptfem_context* ctx, cudaStream_t s, int nc, int ld, double* Ac, float* Ainv, int* d_info) {
  cs_fix_diag<<<blocks_for(nc), CS_THREADS, 0, s>>>(nc, Ac);
  TPT_CHECK_LAUNCH();
  // Cholesky and inverse (symmetric: row-major storage = column-major storage)
  cusolverDnHandle_t h = (cusolverDnHandle_t)ctx->cusolver;
  if (!h) {
    TPT_REQUIRE(cusolverDnCreate(&h) == CUSOLVER_STATUS_SUCCESS, TPTFEM_ERR_DEVICE, "cusolverDnCreate failed");
    ctx->cusolver = h;
  }
  TPT_REQUIRE(cusolverDnSetStream(h, s) == CUSOLVER_STATUS_SUCCESS, TPTFEM_ERR_DEVICE, "cusolverDnSetStream failed");
  int lw1 = 0;
  TPT_REQUIRE(cusolverDnDpotrf_bufferSize(h, CUBLAS_FILL_MODE_LOWER, nc, Ac, nc, &lw1) == CUSOLVER_STATUS_SUCCESS,
              TPTFEM_ERR_DEVICE, "dpotrf_bufferSize failed");
  DevBuf<double> work;
  work.alloc(std::max(1, lw1), s);
  TPT_REQUIRE(cusolverDnDpotrf(h, CUBLAS_FILL_MODE_LOWER, nc, Ac, nc, work.p, lw1, d_info) ==
                  CUSOLVER_STATUS_SUCCESS, TPTFEM_ERR_DEVICE, "dpotrf failed");
  // (a failed Cholesky, d_info != 0, is left for the caller to read: the steps
  // below then produce values that are never used)
  // A_c^-1 = L^-T L^-1: L^-1 from one triangular solve with the identity
  // (lower triangular, zeros above), then one syrk into the lower triangle of
  // Ac -- large library calls instead of potri's many small ones
  DevBuf<double> linv;
  linv.alloc((size_t)nc * nc, s);
  cs_identity<<<blocks_for((int64_t)nc * nc), CS_THREADS, 0, s>>>(nc, linv.p);
  TPT_CHECK_LAUNCH();
  cublasHandle_t hb = (cublasHandle_t)ctx->cublas;
  if (!hb) {
    TPT_REQUIRE(cublasCreate(&hb) == CUBLAS_STATUS_SUCCESS, TPTFEM_ERR_DEVICE, "cublasCreate failed");
    ctx->cublas = hb;
  }
  TPT_REQUIRE(cublasSetStream(hb, s) == CUBLAS_STATUS_SUCCESS, TPTFEM_ERR_DEVICE, "cublasSetStream failed");
  const double one = 1.0, zero = 0.0;
  TPT_REQUIRE(cublasDtrsm(hb, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, nc, nc,
                          &one, Ac, nc, linv.p, nc) == CUBLAS_STATUS_SUCCESS,
              TPTFEM_ERR_DEVICE, "dtrsm failed");
  TPT_REQUIRE(cublasDsyrk(hb, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, nc, nc, &one, linv.p, nc, &zero, Ac, nc) ==
                  CUBLAS_STATUS_SUCCESS, TPTFEM_ERR_DEVICE, "dsyrk failed");
  cs_symmetrize<<<blocks_for((int64_t)nc * ld), CS_THREADS, 0, s>>>(nc, ld, Ac, Ainv);
  TPT_CHECK_LAUNCH();
}

void coarse_restrict_solve(const SystemData& S, const double* r, cudaStream_t s, const int* done) {
  const CoarseSpace& C = S.coarse;
#define TPT_CS_R(D)                                                                                           \
  cs_moments<D><<<C.nseg, CS_THREADS, 0, s>>>(C.sbeg.p, C.send.p, C.alist.p, C.y.p, r, C.smom.p, 0, done); \
  TPT_CHECK_LAUNCH();
  if (S.dpn == 3) { TPT_CS_R(3) }
  else if (S.dpn == 2) { TPT_CS_R(2) }
  else { TPT_CS_R(1) }
#undef TPT_CS_R
  cs_yc<<<blocks_for(C.nc), CS_THREADS, 0, s>>>(C.na, C.nm, C.aseg.p, C.smom.p, C.T.p, C.yc.p, done);
  TPT_CHECK_LAUNCH();
  cs_gemv<<<(C.nc + CS_THREADS / 32 - 1) / (CS_THREADS / 32), CS_THREADS, (size_t)C.ld * sizeof(double), s>>>(
      C.nc, C.ld, C.yc.p, C.Ainv.p, C.uc.p, done);
  TPT_CHECK_LAUNCH();
  cs_raw<<<blocks_for(C.nc), CS_THREADS, 0, s>>>(C.na, C.nm, C.T.p, C.uc.p, C.cm.p, done);
  TPT_CHECK_LAUNCH();
}

void coarse_download(const SystemData& S, int* na, int* nm, double* Ainv_out) {
  const CoarseSpace& C = S.coarse;
  if (na) *na = C.na;
  if (nm) *nm = C.nm;
  if (Ainv_out && C.ready) {  // the FP32 inverse of A_c, widened
    std::vector<float> f((size_t)C.nc * C.ld);
    C.Ainv.download(f.data(), f.size());
    TPT_CUDA(cudaStreamSynchronize(S.ctx->stream));
    for (int i = 0; i < C.nc; ++i)
      for (int j = 0; j < C.nc; ++j) Ainv_out[(size_t)i * C.nc + j] = f[(size_t)i * C.ld + j];
  }
}

int coarse_default_aggregates(const SystemData& S) {
  // about one aggregate per 2000 node groups for vector problems (6 or 3
  // rigid modes each) and per 700 for scalar ones (one constant mode each),
  // between 8 and 3000
  const int per = S.dpn == 1 ? 700 : 2000;
  return std::max(8, std::min(3000, S.nb.ngroups / per));
}

// ---- the coarse space of a row-partitioned system (dist.cu) -----------------------
// Every rank holds the whole system's aggregates and P (coarse_build); these
// work on its own groups only, so that the ranks' partial A_c and P^T r add
// up, over the ranks, to the whole system's.

void coarse_local_build(const SystemData& S, int64_t g0, int64_t g1, CoarseLocal& L) {
  const CoarseSpace& C = S.coarse;
  cudaStream_t s = S.ctx->stream;
  L.g0 = g0;
  L.g1 = g1;
  const int64_t ngl = g1 - g0;
  std::vector<int> agg(std::max<int64_t>(ngl, 1));
  if (ngl) {
    TPT_CUDA(cudaMemcpyAsync(agg.data(), C.agg.p + g0, ngl * sizeof(int), cudaMemcpyDeviceToHost, s));
    TPT_CUDA(cudaStreamSynchronize(s));
  }
  // the local groups of each aggregate, ascending (counting sort by aggregate)
  std::vector<int> cnt(C.na + 1, 0), list(std::max<int64_t>(ngl, 1));
  for (int64_t g = 0; g < ngl; ++g) cnt[agg[g] + 1]++;
  for (int i = 0; i < C.na; ++i) cnt[i + 1] += cnt[i];
  std::vector<int> pos(cnt.begin(), cnt.end() - 1);
  for (int64_t g = 0; g < ngl; ++g) list[pos[agg[g]]++] = (int)(g0 + g);
  constexpr int CS_SEG = 1024;
  std::vector<int> sb, se, aseg(C.na + 1, 0);
  for (int i = 0; i < C.na; ++i) {
    for (int t = cnt[i]; t < cnt[i + 1]; t += CS_SEG) {
      sb.push_back(t);
      se.push_back(std::min(cnt[i + 1], t + CS_SEG));
    }
    aseg[i + 1] = (int)sb.size();
  }
  L.nseg = (int)sb.size();
  L.alist.alloc(list.size(), s);
  L.alist.upload(list.data(), list.size());
  L.sbeg.alloc(std::max(L.nseg, 1), s);
  L.sbeg.upload(sb.data(), L.nseg);
  L.send.alloc(std::max(L.nseg, 1), s);
  L.send.upload(se.data(), L.nseg);
  L.aseg.alloc(C.na + 1, s);
  L.aseg.upload(aseg.data(), C.na + 1);
  L.smom.alloc((size_t)std::max(L.nseg, 1) * C.nm, s);
  TPT_CUDA(cudaStreamSynchronize(s));  // the host vectors are released on return
}

void coarse_local_matrix(const SystemData& S, const CoarseLocal& L, int64_t nloc, const int* rp, const int* ci,
                         const double* va, const int* gcol, double* Acp) {
  const CoarseSpace& C = S.coarse;
  cudaStream_t s = S.ctx->stream;
  const int dpn = S.dpn, nc = C.nc;
  TPT_CUDA(cudaMemsetAsync(Acp, 0, (size_t)nc * nc * sizeof(double), s));
  if (!nloc || !L.nseg) return;
  DevBuf<double> w, mom;
  w.alloc(nloc * C.nm, s);
  mom.alloc((size_t)L.nseg * C.nm * C.nm, s);
  const int ncx = std::min(3, C.bins[0]), ncy = std::min(3, C.bins[1]), ncz = std::min(3, C.bins[2]);
  for (int cz = 0; cz < ncz; ++cz)
    for (int cy = 0; cy < ncy; ++cy)
      for (int cx = 0; cx < ncx; ++cx) {
        const int colour = cx + 3 * cy + 9 * cz;
#define TPT_CS_LOC(D)                                                                                            \
  cs_local_apply<D><<<blocks_for(nloc), CS_THREADS, 0, s>>>(nloc, rp, ci, va, gcol, C.Pfull.p, C.gcolour.p, colour, \
                                                            w.p);                                                  \
  TPT_CHECK_LAUNCH();                                                                                              \
  cs_moments_modes<D><<<L.nseg, CS_THREADS, 0, s>>>(L.sbeg.p, L.send.p, L.alist.p, C.y.p, w.p, mom.p, C.gmask.p,   \
                                                    colour, (int)L.g0);                                            \
  TPT_CHECK_LAUNCH();
        if (dpn == 3) { TPT_CS_LOC(3) }
        else if (dpn == 2) { TPT_CS_LOC(2) }
        else { TPT_CS_LOC(1) }
#undef TPT_CS_LOC
        cs_columns_par<<<blocks_for((int64_t)C.na * C.nm * C.nm), CS_THREADS, 0, s>>>(
            C.na, C.nm, C.abin.p, C.bin2agg.p, C.bins[0], C.bins[1], C.bins[2], L.aseg.p, mom.p, C.T.p, colour, Acp,
            nc);
        TPT_CHECK_LAUNCH();
      }
}

void coarse_local_restrict(const SystemData& S, CoarseLocal& L, const double* r_loc, double* yc, cudaStream_t s) {
  const CoarseSpace& C = S.coarse;
  if (L.nseg) {
#define TPT_CS_LR(D)                                                                                              \
  cs_moments<D><<<L.nseg, CS_THREADS, 0, s>>>(L.sbeg.p, L.send.p, L.alist.p, C.y.p, r_loc, L.smom.p, (int)L.g0); \
  TPT_CHECK_LAUNCH();
    if (S.dpn == 3) { TPT_CS_LR(3) }
    else if (S.dpn == 2) { TPT_CS_LR(2) }
    else { TPT_CS_LR(1) }
#undef TPT_CS_LR
  }
  cs_yc<<<blocks_for(C.nc), CS_THREADS, 0, s>>>(C.na, C.nm, L.aseg.p, L.smom.p, C.T.p, yc);
  TPT_CHECK_LAUNCH();
}

void coarse_local_solve(const SystemData& S, int ld, const float* Ainv, const double* yc, double* uc, double* cm,
                        cudaStream_t s) {
  const CoarseSpace& C = S.coarse;
  cs_gemv<<<(C.nc + CS_THREADS / 32 - 1) / (CS_THREADS / 32), CS_THREADS, (size_t)ld * sizeof(double), s>>>(
      C.nc, ld, yc, Ainv, uc);
  TPT_CHECK_LAUNCH();
  cs_raw<<<blocks_for(C.nc), CS_THREADS, 0, s>>>(C.na, C.nm, C.T.p, uc, cm);
  TPT_CHECK_LAUNCH();
}

}  // namespace tptfem
