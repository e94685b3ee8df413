// topopt.cu -- batched 2-D SIMP topology optimisation (minimum compliance).
//
// Restates crates/tpt-fem-topopt/src/lib.rs (topopt_simp, topopt:342-385) for
// many independent instances at once.  One CTA owns one instance; each
// optimality-criteria iteration is two launches over all instances:
//   E_e = emin + rho_e^p (e0 - emin)                     (assemble, topopt:220-238)
//   K(E) u = f with Dirichlet dofs (the reference uses a dense LU):
//     topo_direct factors K_FF as a band (banded Cholesky, products on the FP64
//     tensor cores) and refines the solution to the residual tolerance; for
//     grids too wide for its band, or a breakdown, topo_iteration runs PCG in
//     FP64 on the matrix-free Q1 operator from the unit element matrix
//     (element_stiffness_unit, topopt:166-217), warm-started from the previous
//     displacement, preconditioned by Jacobi plus an aggregation coarse space of
//     plane rigid modes (M^-1 = D^-1 + P A_c^-1 P^T, A_c assembled and inverted
//     inside the instance's CTA every OC iteration)
//   c = f . u                                             (topopt:360,368)
//   dc_e = -p rho^(p-1) (e0 - emin) u_e^T K0 u_e           (topopt:371-375)
//   sensitivity filter (topopt:259-279) or the density filter of the 88-line
//     SIMP code, then the OC bisection (oc_update, topopt:284-331), all in
//     topo_iteration
// The launches of all iterations are captured in one CUDA graph.  Instances
// never wait on each other (no inter-CTA synchronisation); blocks are issued
// largest instance first.  The block size (threads per instance) is chosen by
// timing the first iteration with each candidate (the autotuner below) and
// cached in the context per batch shape.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <numeric>

#include "common.cuh"
#include "objects.hpp"

namespace tptfem {
namespace {

constexpr double RHO_MIN = 1e-3, RHO_MAX = 1.0, OC_DAMP = 0.5;  // topopt:54-62

constexpr int TP_MAXC = 384;  // coarse unknowns per instance (3 modes x 128 aggregates)

struct TopoInst {
  int nelx, nely, nx, ny, ne, ndof;
  int max_iter, density_filter, has_lift;
  int ag, nax, nay, nc;  // coarse space: aggregates of ag x ag nodes, nax x nay of them, 3 modes each
  // direct solve: banded Cholesky in the band ordering (node index i * ny + j when
  // yfast, else j * nx + i; dof 2 * node + component), half-bandwidth bw, npad
  // unknowns (ndof rounded up to the panel width; the extra ones are identity rows)
  int direct, bw, yfast, npad;
  int64_t eoff, doff, hoff, coff, toff, loff, yoff;
  double h, e0, penal, vol_frac, radius, move, emin;
  double ke0[64];  // element stiffness for E = 1, row-major 8 x 8
};

struct TopoArgs {
  const TopoInst* inst;
  const int* order;  // block -> instance, largest first
  int iter;
  int max_pcg;
  double tol;
  // element arrays (offset eoff)
  double *x, *phys, *E, *raw, *sens, *xnew;
  // dof arrays (offset doff)
  const double *f, *ulift, *ufix;
  const uint8_t* fixed;
  double *u, *r, *p, *q, *dinv, *b;
  double* Ac;        // coarse matrix, inverted in place (offset coff, nc x nc)
  double* Tm;        // per aggregate: 3 x 3 mode transform (offset toff)
  int coarse;        // 1: two-level preconditioner, 0: Jacobi only
  double* hist;      // compliance history (offset hoff)
  int* last_iters;   // per instance: PCG iterations of the latest solve
  long long* total_iters;
  int* flags;        // per instance: bit 0 PCG not converged, bit 1 breakdown
  // direct solves
  const int* dorder;       // block -> instance for the direct kernel, largest first
  double* L;               // band factors (offset loff, npad x (bw + 1), column k holds L(k + d, k))
  double* yb;              // band-ordered right-hand side / solution (offset yoff, npad)
  int* direct_ok;          // per instance: 1 when this iteration's direct solve succeeded
  long long* refine;       // per instance: iterative-refinement steps taken
};

// Block-wide sums (deterministic for a fixed block size).
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double s = threadIdx.x < NT / 32 ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) sh[64] = s;
  }
  __syncthreads();
  return sh[64];
}

template <int NT>
__device__ __forceinline__ void block_sum2(double& a, double& b, double* sh) {
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) { sh[threadIdx.x >> 5] = a; sh[32 + (threadIdx.x >> 5)] = b; }
  __syncthreads();
  if (threadIdx.x < 32) {
    double s = threadIdx.x < NT / 32 ? sh[threadIdx.x] : 0.0;
    double t = threadIdx.x < NT / 32 ? sh[32 + threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      s += __shfl_xor_sync(0xffffffffu, s, o);
      t += __shfl_xor_sync(0xffffffffu, t, o);
    }
    if (threadIdx.x == 0) { sh[64] = s; sh[65] = t; }
  }
  __syncthreads();
  a = sh[64];
  b = sh[65];
}

// local index of node (i, j) in the element whose origin is (i + di, j + dj),
// di, dj in {-1, 0}; element node order 00, 10, 11, 01 (Quad4, topopt:99-109)
__device__ __forceinline__ int local_node(int di, int dj) {
  const int ox = -di, oy = -dj;
  return oy == 0 ? ox : (ox == 1 ? 2 : 3);
}

// y = K(E) v on the grid's rows; rows of fixed dofs are set to 0 when `mask`.
// Node (i, j) gathers its <= 4 incident elements (origins (i-1..i, j-1..j)),
// each from its own 8 dof values (L1-resident), which keeps few values live.
// Returns this thread's part of v.y.
template <int NT>
__device__ double apply_k(const TopoInst& I, const double* __restrict__ E, const double* __restrict__ v,
                          double* __restrict__ y, const uint8_t* __restrict__ fixed, bool mask,
                          const double* __restrict__ ke) {
  const int nx = I.nx, nelx = I.nelx, nely = I.nely, nn = nx * I.ny;
  double dot = 0.0;
  for (int n = threadIdx.x; n < nn; n += NT) {
    const int i = n % nx, j = n / nx;
    double y0 = 0.0, y1 = 0.0;
#pragma unroll 1
    for (int q = 0; q < 4; ++q) {
      const int di = (q & 1) ? 0 : -1, dj = (q & 2) ? 0 : -1;
      const int ei = i + di, ej = j + dj;
      if (ei < 0 || ei >= nelx || ej < 0 || ej >= nely) continue;
      const int n0 = ej * nx + ei;
      const int ln = local_node(di, dj);
      const double* k0 = ke + (2 * ln) * 8;
      const double* k1 = k0 + 8;
      const int nd[4] = {n0, n0 + 1, n0 + nx + 1, n0 + nx};
      double s0 = 0.0, s1 = 0.0;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const double2 vv = __ldg(reinterpret_cast<const double2*>(v) + nd[k]);
        s0 += k0[2 * k] * vv.x + k0[2 * k + 1] * vv.y;
        s1 += k1[2 * k] * vv.x + k1[2 * k + 1] * vv.y;
      }
      const double Ee = __ldg(E + ej * nelx + ei);
      y0 += Ee * s0;
      y1 += Ee * s1;
    }
    if (mask) {
      if (fixed[2 * n]) y0 = 0.0;
      if (fixed[2 * n + 1]) y1 = 0.0;
    }
    reinterpret_cast<double2*>(y)[n] = make_double2(y0, y1);
    const double2 vn = reinterpret_cast<const double2*>(v)[n];
    dot += vn.x * y0 + vn.y * y1;
  }
  return dot;
}

// Filter weights w = R - d for d <= R (sensitivity filter, topopt:259-279) or
// w = max(0, R - d) (density filter) between element centres d apart.  The
// window spans W elements either side; windows up to TP_WMAX use a table of
// the weights by offset, filled once per instance (negative: outside the
// sensitivity filter's disc), so the sums need no square roots.
constexpr int TP_WMAX = 8;
constexpr int TP_WTAB = (2 * TP_WMAX + 1) * (2 * TP_WMAX + 1);

template <bool SENS>
__device__ __forceinline__ int filter_halfwidth(const TopoInst& I) {
  return SENS ? (int)floor(I.radius / I.h) + 1 : (int)ceil(I.radius / I.h);
}

template <bool SENS>
__device__ __forceinline__ double filter_weight(const TopoInst& I, double dx, double dy) {
  const double d2 = dx * dx + dy * dy, R = I.radius;
  if (SENS) return d2 <= R * R ? R - sqrt(d2) : -1.0;
  return fmax(0.0, R - sqrt(d2));
}

template <bool SENS, int NT>
__device__ void filter_table(const TopoInst& I, double* wt) {
  const int W = filter_halfwidth<SENS>(I), n = 2 * W + 1;
  if (W > TP_WMAX) return;
  for (int q = threadIdx.x; q < n * n; q += NT) {
    const int oy = q / n - W, ox = q % n - W;
    wt[q] = filter_weight<SENS>(I, ox * I.h, oy * I.h);
  }
}

// Sum over the filter window of element e of w * term, term = val[f] (1 when
// val is null), divided by div[f] when div is given; den = sum of w.
template <bool SENS>
__device__ __forceinline__ void filter_window(const TopoInst& I, int e, const double* __restrict__ val,
                                              const double* __restrict__ div, const double* __restrict__ wt,
                                              double& num, double& den) {
  const int ei = e % I.nelx, ej = e / I.nelx;
  const double h = I.h;
  const int w = filter_halfwidth<SENS>(I), n = 2 * w + 1;
  const bool tab = w <= TP_WMAX;
  const double cx = ((double)ei + 0.5) * h, cy = ((double)ej + 0.5) * h;
  num = 0.0;
  den = 0.0;
  for (int fj = max(0, ej - w); fj <= min(I.nely - 1, ej + w); ++fj)
    for (int fi = max(0, ei - w); fi <= min(I.nelx - 1, ei + w); ++fi) {
      const double wgt = tab ? wt[(fj - ej + w) * n + (fi - ei + w)]
                             : filter_weight<SENS>(I, cx - ((double)fi + 0.5) * h, cy - ((double)fj + 0.5) * h);
      if (SENS && wgt < 0.0) continue;
      const int f = fj * I.nelx + fi;
      double term = val ? val[f] : 1.0;
      if (div) term /= div[f];
      num += wgt * term;
      den += wgt;
    }
}

__device__ __forceinline__ double oc_candidate(double rho, double b, double lambda, double move) {
  const double ratio = b > 0.0 ? pow(b / lambda, OC_DAMP) : 0.0;
  const double c = rho * ratio;
  const double lo = fmax(rho - move, RHO_MIN), hi = fmin(rho + move, RHO_MAX);
  return fmin(fmax(c, lo), hi);
}

// ---- per-instance aggregation coarse space ----------------------------------------
// Aggregates are boxes of ag x ag nodes (the last row/column of boxes takes the
// remainder); each carries the three rigid modes of plane elasticity about the
// centre of its node box -- x, y translation and rotation (-y, x) --
// orthonormalised over its free dofs (modes it cannot carry are dropped).
// Colour of an aggregate = (ax mod 3, ay mod 3): an aggregate has at most one
// neighbour of each colour, so A_c = P^T K P comes column block by column block
// from 9 x 3 operator products.

struct AggBox {
  int i0, i1, j0, j1;
};

__device__ __forceinline__ AggBox agg_box(const TopoInst& I, int A) {
  const int ax = A % I.nax, ay = A / I.nax;
  AggBox b;
  b.i0 = ax * I.ag;
  b.i1 = ax == I.nax - 1 ? I.nx - 1 : b.i0 + I.ag - 1;
  b.j0 = ay * I.ag;
  b.j1 = ay == I.nay - 1 ? I.ny - 1 : b.j0 + I.ag - 1;
  return b;
}

__device__ __forceinline__ int agg_of(const TopoInst& I, int i, int j) {
  return min(i / I.ag, I.nax - 1) + I.nax * min(j / I.ag, I.nay - 1);
}

// raw modes of node (i, j) of box b: R[a][k], a = dof component, k = mode
__device__ __forceinline__ void modes2(const TopoInst& I, const AggBox& b, int i, int j, double (&R)[2][3]) {
  const double x = (i - 0.5 * (b.i0 + b.i1)) * I.h, y = (j - 0.5 * (b.j0 + b.j1)) * I.h;
  R[0][0] = 1.0; R[0][1] = 0.0; R[0][2] = -y;
  R[1][0] = 0.0; R[1][1] = 1.0; R[1][2] = x;
}

// Orthonormal mode transform of every aggregate (warp per aggregate): Gram
// matrix over free dofs G = L L^T (modes with no remaining weight dropped),
// T = L^-T.
template <int NT>
__device__ void coarse_transforms(const TopoInst& I, const uint8_t* __restrict__ fixed, double* __restrict__ Tm) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int na = I.nax * I.nay;
  for (int A = warp; A < na; A += NT / 32) {
    const AggBox b = agg_box(I, A);
    const int w = b.i1 - b.i0 + 1, cnt = w * (b.j1 - b.j0 + 1);
    double g[6] = {0, 0, 0, 0, 0, 0};  // 00 01 02 11 12 22
    for (int t = lane; t < cnt; t += 32) {
      const int i = b.i0 + t % w, j = b.j0 + t / w, n = j * I.nx + i;
      double R[2][3];
      modes2(I, b, i, j, R);
      for (int c = 0; c < 2; ++c) {
        if (fixed[2 * n + c]) continue;
        g[0] += R[c][0] * R[c][0]; g[1] += R[c][0] * R[c][1]; g[2] += R[c][0] * R[c][2];
        g[3] += R[c][1] * R[c][1]; g[4] += R[c][1] * R[c][2]; g[5] += R[c][2] * R[c][2];
      }
    }
    for (int q = 0; q < 6; ++q)
      for (int o = 16; o > 0; o >>= 1) g[q] += __shfl_xor_sync(0xffffffffu, g[q], o);
    if (lane == 0) {
      const double G[3][3] = {{g[0], g[1], g[2]}, {g[1], g[3], g[4]}, {g[2], g[4], g[5]}};
      const double tr = g[0] + g[3] + g[5];
      double L[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      bool keep[3];
      for (int k = 0; k < 3; ++k) {
        double sk = G[k][k];
        for (int q = 0; q < k; ++q) sk -= L[k][q] * L[k][q];
        keep[k] = sk > 1e-10 * tr && tr > 0.0;
        if (!keep[k]) continue;
        L[k][k] = sqrt(sk);
        for (int i2 = k + 1; i2 < 3; ++i2) {
          double v = G[i2][k];
          for (int q = 0; q < k; ++q) v -= L[i2][q] * L[k][q];
          L[i2][k] = v / L[k][k];
        }
      }
      double* T = Tm + (int64_t)A * 9;
      for (int m = 0; m < 3; ++m) {  // column m of L^-1, then T[k][m] = Linv[m][k]
        double xv[3];
        for (int i2 = 0; i2 < 3; ++i2) {
          if (!keep[i2]) { xv[i2] = 0.0; continue; }
          double v = (i2 == m) ? 1.0 : 0.0;
          for (int q = 0; q < i2; ++q) v -= L[i2][q] * xv[q];
          xv[i2] = v / L[i2][i2];
        }
        for (int k = 0; k < 3; ++k) T[m * 3 + k] = keep[m] ? xv[k] : 0.0;  // T^T stored: row m = mode m
      }
    }
  }
}

// s[k] = sum over aggregate A's nodes of R^T w (raw modes), warp-reduced (all lanes get it).
__device__ __forceinline__ void agg_moments(const TopoInst& I, int A, const double* __restrict__ w, double (&s)[3]) {
  const int lane = threadIdx.x & 31;
  const AggBox b = agg_box(I, A);
  const int wd = b.i1 - b.i0 + 1, cnt = wd * (b.j1 - b.j0 + 1);
  s[0] = s[1] = s[2] = 0.0;
  for (int t = lane; t < cnt; t += 32) {
    const int i = b.i0 + t % wd, j = b.j0 + t / wd, n = j * I.nx + i;
    double R[2][3];
    modes2(I, b, i, j, R);
    const double2 wn = reinterpret_cast<const double2*>(w)[n];
    for (int k = 0; k < 3; ++k) s[k] += R[0][k] * wn.x + R[1][k] * wn.y;
  }
  for (int k = 0; k < 3; ++k)
    for (int o = 16; o > 0; o >>= 1) s[k] += __shfl_xor_sync(0xffffffffu, s[k], o);
}

// A_c = P^T K_FF P, then its inverse in place (Gauss-Jordan; A_c is SPD).
template <int NT>
__device__ void coarse_assemble_invert(const TopoInst& I, const double* __restrict__ E,
                                       const uint8_t* __restrict__ fixed, const double* __restrict__ ke,
                                       const double* __restrict__ Tm, double* __restrict__ v, double* __restrict__ y,
                                       double* __restrict__ Ac, double* __restrict__ fcol) {
  const int nc = I.nc, na = I.nax * I.nay, nn = I.nx * I.ny;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int t = threadIdx.x; t < nc * nc; t += NT) Ac[t] = 0.0;
  for (int cy = 0; cy < min(3, I.nay); ++cy)
    for (int cx = 0; cx < min(3, I.nax); ++cx)
      for (int m = 0; m < 3; ++m) {
        __syncthreads();
        for (int n = threadIdx.x; n < nn; n += NT) {  // v = P e_(colour, m), zero on fixed dofs
          const int i = n % I.nx, j = n / I.nx, A = agg_of(I, i, j);
          double v0 = 0.0, v1 = 0.0;
          if ((A % I.nax) % 3 == cx && (A / I.nax) % 3 == cy) {
            double R[2][3];
            modes2(I, agg_box(I, A), i, j, R);
            const double* T = Tm + (int64_t)A * 9 + m * 3;
            v0 = fixed[2 * n] ? 0.0 : R[0][0] * T[0] + R[0][1] * T[1] + R[0][2] * T[2];
            v1 = fixed[2 * n + 1] ? 0.0 : R[1][0] * T[0] + R[1][1] * T[1] + R[1][2] * T[2];
          }
          reinterpret_cast<double2*>(v)[n] = make_double2(v0, v1);
        }
        __syncthreads();
        apply_k<NT>(I, E, v, y, fixed, true, ke);
        __syncthreads();
        for (int A = warp; A < na; A += NT / 32) {
          const int ax = A % I.nax, ay = A / I.nax;
          int jx = -1, jy = -1;
          for (int o = -1; o <= 1; ++o) {
            if (ax + o >= 0 && ax + o < I.nax && (ax + o) % 3 == cx) jx = ax + o;
            if (ay + o >= 0 && ay + o < I.nay && (ay + o) % 3 == cy) jy = ay + o;
          }
          if (jx < 0 || jy < 0) continue;
          const int J = jy * I.nax + jx;
          double sk[3];
          agg_moments(I, A, y, sk);
          if (lane < 3) {
            const double* T = Tm + (int64_t)A * 9 + lane * 3;  // mode `lane` of A
            Ac[(int64_t)(A * 3 + lane) * nc + J * 3 + m] = T[0] * sk[0] + T[1] * sk[1] + T[2] * sk[2];
          }
        }
      }
  __syncthreads();
  for (int i = threadIdx.x; i < nc; i += NT)
    if (Ac[(int64_t)i * nc + i] == 0.0) Ac[(int64_t)i * nc + i] = 1.0;  // dropped modes
  for (int k = 0; k < nc; ++k) {  // in-place Gauss-Jordan inversion
    __syncthreads();
    for (int i = threadIdx.x; i < nc; i += NT) fcol[i] = Ac[(int64_t)i * nc + k];
    __syncthreads();
    const double piv = fcol[k];
    for (int j = threadIdx.x; j < nc; j += NT)
      Ac[(int64_t)k * nc + j] = (j == k ? 1.0 : Ac[(int64_t)k * nc + j]) / piv;
    __syncthreads();
    for (int t = threadIdx.x; t < nc * nc; t += NT) {
      const int i = t / nc, j = t % nc;
      if (i == k) continue;
      const double akj = Ac[(int64_t)k * nc + j];
      Ac[t] = (j == k ? 0.0 : Ac[t]) - fcol[i] * akj;
    }
  }
  __syncthreads();
}

// uc = A_c^-1 P^T r and c_A = T_A uc_A (raw-mode coefficients per aggregate) into cm.
template <int NT>
__device__ void coarse_solve(const TopoInst& I, const double* __restrict__ Tm, const double* __restrict__ Ainv,
                             const double* __restrict__ r, double* __restrict__ yc, double* __restrict__ uc,
                             double* __restrict__ cm) {
  const int nc = I.nc, na = I.nax * I.nay;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  for (int A = warp; A < na; A += NT / 32) {
    double sk[3];
    agg_moments(I, A, r, sk);
    if (lane < 3) {
      const double* T = Tm + (int64_t)A * 9 + lane * 3;
      yc[A * 3 + lane] = T[0] * sk[0] + T[1] * sk[1] + T[2] * sk[2];
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nc; i += NT) {
    const double* row = Ainv + (int64_t)i * nc;
    double sum = 0.0;
    for (int j = 0; j < nc; ++j) sum += row[j] * yc[j];
    uc[i] = sum;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < na * 3; t += NT) {  // raw-mode coefficients: sum_m T[m][k] uc[m]
    const int A = t / 3, k = t % 3;
    const double* T = Tm + (int64_t)A * 9;
    cm[t] = T[0 * 3 + k] * uc[A * 3 + 0] + T[1 * 3 + k] * uc[A * 3 + 1] + T[2 * 3 + k] * uc[A * 3 + 2];
  }
  __syncthreads();
}

// z = D^-1 r + P uc (cm holds the raw-mode coefficients); returns this thread's part of r.z
template <int NT>
__device__ double two_level_z(const TopoInst& I, const double* __restrict__ r, const double* __restrict__ dinv,
                              const double* __restrict__ cm, double* __restrict__ z) {
  double rz = 0.0;
  for (int n = threadIdx.x; n < I.nx * I.ny; n += NT) {
    const int i = n % I.nx, j = n / I.nx, A = agg_of(I, i, j);
    double R[2][3];
    modes2(I, agg_box(I, A), i, j, R);
    const double2 rn = reinterpret_cast<const double2*>(r)[n];
    const double2 dn = reinterpret_cast<const double2*>(dinv)[n];
    const double c0 = cm[A * 3], c1 = cm[A * 3 + 1], c2 = cm[A * 3 + 2];
    // fixed dofs: dinv = 0 and r = 0, and P is zero there (v is masked)
    const double z0 = dn.x * rn.x + (dn.x != 0.0 ? R[0][0] * c0 + R[0][1] * c1 + R[0][2] * c2 : 0.0);
    const double z1 = dn.y * rn.y + (dn.y != 0.0 ? R[1][0] * c0 + R[1][1] * c1 + R[1][2] * c2 : 0.0);
    reinterpret_cast<double2*>(z)[n] = make_double2(z0, z1);
    rz += rn.x * z0 + rn.y * z1;
  }
  return rz;
}

// ---- per-instance direct solve: banded Cholesky ------------------------------------
// K_FF (fixed dofs replaced by identity rows and columns) is banded in the node
// ordering that runs along the shorter grid direction: node (i, j) couples with
// (i +- 1, j +- 1), so |row - col| <= bw = 2 min(nx, ny) + 3.  The factor L is
// computed panel by panel (TD_NB columns) in one CTA, with the right-hand side
// carried along as one extra row below the panel's R = bw + TD_NB rows, so that
// the forward substitution comes out of the same elimination:
//   1. A's entries of the panel's columns (rows >= the column, at most bw
//      below) from the element moduli and the unit element matrix, one thread
//      per (column, neighbour node); the right-hand-side row holds b;
//   2. S = L(panel rows, earlier columns) L(panel columns, earlier columns)^T
//      over the bw earlier columns (the right-hand-side row uses y of those
//      columns), staged from the band storage in chunks of TD_JC columns that
//      are prefetched into registers one chunk ahead; each thread accumulates
//      a 4 x 4 tile of the panel in registers;
//   3. P = A - S is eliminated in registers four columns at a time: the thread
//      holding the 4 x 4 diagonal block factors it, the other threads of that
//      column group eliminate their rows with it, then every later column is
//      updated (two barriers per group);
//   4. the columns are scaled by the pivots' inverse square roots into the band
//      storage, and the right-hand-side row gives y of the panel's unknowns.
// The backward substitution reads the stored panels in reverse.  The residual
// of the result is checked on the matrix-free operator and, if needed,
// corrected by iterative refinement with the stored factor.
constexpr int TD_NT = 512;     // threads of the direct kernel
constexpr int TD_NB = 32;      // panel width
constexpr int TD_JC = 16;      // earlier columns staged per chunk
constexpr int TD_MAXBW = 221;  // largest half-bandwidth: the panel's rows + the right-hand-side row in 4 x 4 tiles
constexpr int TD_RSMAX = 256;  //   (at most TD_RSMAX / 4 row tiles x TD_NB / 4 column tiles = TD_NT threads)
constexpr int TD_NSTAGE = 4;   // chunk buffers: TD_NSTAGE - 1 chunks in flight
constexpr int TD_REFINE = 4;   // iterative-refinement steps at most
static_assert((TD_RSMAX / 4) * (TD_NB / 4) <= TD_NT, "panel tiles must fit the block");
static_assert(TD_NT == 16 * TD_NB, "backward dot products use 16 lanes per panel column");

// rows stored per panel: R = bw + TD_NB matrix rows, the right-hand-side row R, padding to 4
__host__ __device__ inline int td_rs(int bw) { return (bw + TD_NB + 1 + 7) & ~7; }
// column-group buffers: row r at (r / 4) * 6 + r % 4 (two padding doubles per
// four rows), so the 4-row tiles of consecutive threads fall in distinct banks
__host__ __device__ inline int td_cs(int rs) { return rs / 4 * 6; }
__host__ __device__ inline int64_t td_smem_doubles(int bw) {
  const int rs = td_rs(bw);
  return (int64_t)TD_NB * rs + (int64_t)TD_NSTAGE * TD_JC * rs + 8LL * td_cs(rs);
}
static_assert(((TD_MAXBW + TD_NB + 1 + 7) & ~7) <= TD_RSMAX, "TD_MAXBW must fit TD_RSMAX");
constexpr int TD_MAXT = (TD_RSMAX / 8) * (TD_NB / 8) / (TD_NT / 32);  // 8 x 8 product tiles per warp
static_assert((TD_NT / 32) % (TD_NB / 8) == 0, "a warp's product tiles share one column block");
static_assert(TD_JC == TD_NT / 32, "one staged column per warp and chunk");

// 8-byte asynchronous copy global -> shared (zero-filled when !valid), and its
// group commit / wait (cp.async, PTX ISA).
__device__ __forceinline__ void td_cp8(double* sdst, const double* gsrc, bool valid) {
  const unsigned saddr = static_cast<unsigned>(__cvta_generic_to_shared(sdst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(saddr), "l"(gsrc), "r"(valid ? 8 : 0)
               : "memory");
}
__device__ __forceinline__ void td_cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void td_cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// D = A B + D on one 8 x 8 x 4 FP64 tensor-core tile (mma.sync m8n8k4, PTX ISA
// fragment layout: lane l holds A(l / 4, l % 4), B(l % 4, l / 4) and
// D(l / 4, 2 (l % 4) + {0, 1})).
__device__ __forceinline__ void td_mma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// 1 / x by Newton-Raphson from a single-precision seed (two steps: the seed's
// 2^-23 relative error squares to below double rounding); x = pivots, which
// lie well inside the single-precision range (else the plain division).
__device__ __forceinline__ double td_rcp(double x) {
  const double ax = fabs(x);
  if (!(ax > 1e-30 && ax < 1e30)) return 1.0 / x;
  double r = (double)__frcp_rn((float)x);
  r = r * (2.0 - x * r);
  return r * (2.0 - x * r);
}

__device__ __forceinline__ int band_index(const TopoInst& I, int i, int j, int comp) {
  return 2 * (I.yfast ? i * I.ny + j : j * I.nx + i) + comp;
}

// original dof (2 (j nx + i) + comp) of band unknown k < ndof
__device__ __forceinline__ int band_to_dof(const TopoInst& I, int k) {
  const int m = k >> 1, comp = k & 1;
  const int i = I.yfast ? m / I.ny : m % I.nx;
  const int j = I.yfast ? m % I.ny : m / I.nx;
  return 2 * (j * I.nx + i) + comp;
}

__device__ __forceinline__ int dof_to_band(const TopoInst& I, int d) {
  const int n = d >> 1;
  return band_index(I, n % I.nx, n / I.nx, d & 1);
}

// Entries A(row, k) of band column k for the rows of node (i + di, j + dj),
// both components, rows >= k, into col[row - K]: the sum over the elements
// that hold both nodes.  Identity for fixed dofs and padding unknowns k >= ndof
// (written by the node's own entry, di = dj = 0).  The moduli and fixed flags
// are all loaded before any is used (one round of memory latency).
__device__ void band_column_entries(const TopoInst& I, const double* __restrict__ E,
                                    const uint8_t* __restrict__ fixed, const double* __restrict__ ke, int k, int K,
                                    int di, int dj, double* __restrict__ col) {
  const bool self = di == 0 && dj == 0;
  const int kk = min(k, I.ndof - 1);
  const int m = kk >> 1, comp = kk & 1;
  const int i = I.yfast ? m / I.ny : m % I.nx;
  const int j = I.yfast ? m % I.ny : m / I.nx;
  const int i2 = i + di, j2 = j + dj;
  const bool node2 = i2 >= 0 && i2 < I.nx && j2 >= 0 && j2 < I.ny;
  const int n2 = node2 ? j2 * I.nx + i2 : j * I.nx + i;
  // the (up to) four elements around node (i, j): origins (i - 1 + a, j - 1 + b)
  double Ee[4];
  bool inE[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int ei = i - 1 + (q & 1), ej = j - 1 + (q >> 1);
    inE[q] = ei >= 0 && ei < I.nelx && ej >= 0 && ej < I.nely;
    Ee[q] = inE[q] ? E[ej * I.nelx + ei] : 0.0;
  }
  const bool fcol = fixed[2 * (j * I.nx + i) + comp];
  const bool f2[2] = {fixed[2 * n2] != 0, fixed[2 * n2 + 1] != 0};
  if (k >= I.ndof || fcol) {
    if (self) col[k - K] = 1.0;
    return;
  }
  if (!node2) return;
#pragma unroll
  for (int c2 = 0; c2 < 2; ++c2) {
    const int row = band_index(I, i2, j2, c2);
    if (row < k || f2[c2]) continue;
    double v = 0.0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int ei = i - 1 + (q & 1), ej = j - 1 + (q >> 1);
      // element (ei, ej) holds node (i2, j2) too
      if (!inE[q] || i2 < ei || i2 > ei + 1 || j2 < ej || j2 > ej + 1) continue;
      const int lc = 2 * local_node(ei - i, ej - j) + comp;
      const int lr = 2 * local_node(ei - i2, ej - j2) + c2;
      v += Ee[q] * ke[lr * 8 + lc];
    }
    col[row - K] = v;
  }
}

// Panel K of L from the band storage into Pa (column-major, rows r = 0..R-1 of
// the window starting at K; zero outside the band).
template <int NT>
__device__ void band_load_panel(int K, int bw, int RS, const double* Lb, double* Pa) {
  const int R = bw + TD_NB, ld = bw + 1;
  for (int q = threadIdx.x; q < TD_NB * RS; q += NT) {
    const int c = q / RS, r = q - c * RS;
    Pa[q] = (r >= c && r - c <= bw && r < R) ? Lb[(int64_t)(K + c) * ld + (r - c)] : 0.0;
  }
}

// Forward substitution for panel K (L in Pa): y[K..K+NB) from the diagonal
// block, then y[K+NB .. K+R) -= L(below) y[K..K+NB).
template <int NT>
__device__ void band_forward_panel(int K, int np, int bw, int RS, const double* Pa, double* yb, double* ysm) {
  const int t = threadIdx.x, R = bw + TD_NB;
  if (t < 32) {
    double v = yb[K + t];
    const double dl = 1.0 / Pa[t * RS + t];
    double y = 0.0;
    for (int c = 0; c < TD_NB; ++c) {
      const double yc = __shfl_sync(0xffffffffu, v, c) * __shfl_sync(0xffffffffu, dl, c);
      if (t == c) y = yc;
      if (t > c) v -= Pa[c * RS + t] * yc;
    }
    yb[K + t] = y;
    ysm[t] = y;
  }
  __syncthreads();
  for (int r = TD_NB + t; r < R && K + r < np; r += NT) {
    double s = 0.0;
#pragma unroll 8
    for (int c = 0; c < TD_NB; ++c) s += Pa[c * RS + r] * ysm[c];
    yb[K + r] -= s;
  }
  __syncthreads();
}

// Backward substitution x = L^-T y over all panels, in place in yb.  The
// panels stream from the band storage through three shared-memory buffers
// (sm, sm + TD_NB RS, sm + 2 TD_NB RS) by cp.async, two panels ahead.
template <int NT>
__device__ void band_backward(int np, int bw, int RS, const double* Lb, double* yb, double* sm, double* tsm) {
  const int t = threadIdx.x, R = bw + TD_NB, ld = bw + 1, nl = TD_NB * RS;
  const int wc0 = t / RS, wr0 = t - wc0 * RS, wdc = NT / RS, wdr = NT - wdc * RS;
  const int npan = np / TD_NB;
  // panel p (from the last) into buffer p % 3: value w = c * RS + r holds L(K + r, K + c)
  auto issue = [&](int pp) {
    if (pp < npan) {
      const int K = np - TD_NB * (pp + 1);
      double* B = sm + (pp % 3) * nl;
      int c = wc0, r = wr0;
      for (int w = t; w < nl; w += NT) {
        const bool in = r >= c && r - c <= bw && r < R;
        td_cp8(B + w, in ? Lb + (int64_t)(K + c) * ld + (r - c) : Lb, in);
        c += wdc;
        r += wdr;
        if (r >= RS) { r -= RS; ++c; }
      }
    }
    td_cp_commit();
  };
  issue(0);
  issue(1);
  for (int pp = 0; pp < npan; ++pp) {
    td_cp_wait<1>();
    __syncthreads();  // panel pp has landed everywhere; buffer (pp + 2) % 3 is free
    issue(pp + 2);
    const int K = np - TD_NB * (pp + 1);
    const double* Pa = sm + (pp % 3) * nl;
    {
      const int c = t >> 4, s = t & 15;
      double sum = 0.0;
      for (int r = TD_NB + s; r < R && K + r < np; r += 16) sum += Pa[c * RS + r] * yb[K + r];
      for (int o = 8; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
      if (s == 0) tsm[c] = yb[K + c] - sum;
    }
    __syncthreads();
    if (t < 32) {
      double v = tsm[t];
      const double dl = 1.0 / Pa[t * RS + t];
      double x = 0.0;
      for (int c = TD_NB - 1; c >= 0; --c) {
        const double xc = __shfl_sync(0xffffffffu, v, c) * __shfl_sync(0xffffffffu, dl, c);
        if (t == c) x = xc;
        if (t < c) v -= Pa[t * RS + c] * xc;  // L(K + c, K + t)
      }
      yb[K + t] = x;
    }
  }
  td_cp_wait<0>();
  __syncthreads();
}

// Factor K_FF = L L^T into Lb and solve L y = yb in place.  False on a
// non-positive pivot.
template <int NT>
__device__ bool band_factor_forward(const TopoInst& I, const double* __restrict__ E, const uint8_t* __restrict__ fixed,
                                    const double* __restrict__ ke, double* Lb, double* yb, double* sm, double* piv,
                                    int* bad) {
  const int bw = I.bw, ld = bw + 1, np = I.npad;
  const int R = bw + TD_NB, RS = td_rs(bw);  // row R: right-hand side
  double* Pa = sm;                    // TD_NB x RS, column-major: A of the panel
  double* Wc = sm + TD_NB * RS;       // TD_NSTAGE x TD_JC x RS: staged earlier columns
  const int CS = td_cs(RS);
  double* cg = Wc + TD_NSTAGE * TD_JC * RS;  // 4 x CS: the eliminated column group (padded rows)
  double* cgs = cg + 4 * CS;                 // 4 x CS: the same, divided by the pivots
  __shared__ double dfac[16], dinv[4];
  const int t = threadIdx.x;
  // elimination tiles, column-tile major: the threads of a warp share their
  // column tile (one code path per warp in each elimination phase)
  const int nrt = RS / 4;
  const bool act = t < nrt * (TD_NB / 4);
  const int tc = t / nrt, tr = t - tc * nrt;
  const int r0 = 4 * tr, c0 = 4 * tc;
  const int nw = TD_JC * RS;  // staged values per chunk
  const int lane = t & 31, warp = t >> 5;
  const int rlast = RS - 8;   // first row of the last row block (holds row R)
  // Pa is zero at the start of every panel: zeroed here, and each panel's
  // write-out zeroes the entries it copies (the others are written as zero)
  for (int q = t; q < TD_NB * RS; q += NT) Pa[q] = 0.0;
  __syncthreads();
  for (int K = 0; K < np; K += TD_NB) {
    // S over chunk ch of the earlier columns: staged value w = j * RS + r holds
    // L(K + r, jlo + ch * TD_JC + j), row R holds y of that column
    const int jlo = max(0, K - bw), nch = (K - jlo + TD_JC - 1) / TD_JC;
    // chunk ch: warp w stages column gj = jlo + ch TD_JC + w, its lanes the rows
    // (L(K + r, gj) sits at Lb[gj ld + K - gj + r] while r <= rmax = bw - K + gj).
    // The products read a column's rows only up to rmax + 10 (the row blocks a
    // 4-column step needs) and the last row block (right-hand side, row R), so
    // only rows < rmax + 17 and that block are staged (zero beyond the band);
    // columns past the panel start (gj >= K) are staged as zeros throughout.
#define TD_ISSUE(ch)                                                                    \
  {                                                                                     \
    if ((ch) < nch) {                                                                   \
      const int gj = jlo + (ch) * TD_JC + warp;                                         \
      double* Wj = Wc + ((ch) % TD_NSTAGE) * nw + warp * RS;                            \
      const bool live = gj < K;                                                         \
      const double* col = Lb + (int64_t)gj * ld + (K - gj);                             \
      const int rmax = live ? bw - (K - gj) : -1;                                       \
      const int rz = live ? min(rmax + 17, rlast) : rlast;                              \
      for (int r = lane; r < rz; r += 32) td_cp8(Wj + r, r <= rmax ? col + r : Lb, r <= rmax); \
      if (lane < 8) td_cp8(Wj + rlast + lane, live && rlast + lane == R ? yb + gj : Lb,  \
                           live && rlast + lane == R);                                  \
    }                                                                                   \
    td_cp_commit();                                                                     \
  }
    // S on the tensor cores: warp w owns the 8 x 8 tiles i = 0, 1, .. of row block
    // rb0 + 4 i (rb0 = w / 4) and column block cb = w % 4, two accumulators per
    // lane and tile
    const int cb = warp & 3, rb0 = warp >> 2;
    const int nmine = (RS / 8 - rb0 + 3) >> 2;                           // this warp's tiles
    const int irhs = ((rlast / 8 - rb0) & 3) == 0 ? (rlast / 8 - rb0) >> 2 : -1;  // its right-hand-side tile
    double s0[TD_MAXT], s1[TD_MAXT];
#pragma unroll
    for (int i = 0; i < TD_MAXT; ++i) s0[i] = s1[i] = 0.0;
#pragma unroll
    for (int ch = 0; ch < TD_NSTAGE - 1; ++ch) TD_ISSUE(ch);  // in flight during the assembly
    if (t < TD_NB * 9) {
      const int c = t / 9, nb = t - 9 * c;
      band_column_entries(I, E, fixed, ke, K + c, K, nb % 3 - 1, nb / 3 - 1, Pa + c * RS);
      if (nb == 4) Pa[c * RS + R] = yb[K + c];
    }
    for (int ch = 0; ch < nch; ++ch) {
      td_cp_wait<TD_NSTAGE - 2>();  // chunk ch has landed (this thread's copies)
      __syncthreads();               // ... everyone's; chunk ch - 1's buffer is free
      TD_ISSUE(ch + TD_NSTAGE - 1);
      const int j0 = jlo + ch * TD_JC;
      const double* Wl = Wc + (ch % TD_NSTAGE) * nw + (lane & 3) * RS + (lane >> 2);
      double bf[TD_JC / 4];
#pragma unroll
      for (int ks = 0; ks < TD_JC / 4; ++ks) bf[ks] = Wl[ks * 4 * RS + cb * 8];
      // row block rb is zero in columns below K + 8 rb - bw (band): tile i needs the
      // 4-column steps ks >= kmin0 + 8 i (all of them for the right-hand-side tile)
      const int kmin0 = (K + 8 * rb0 - bw - j0) >> 2;  // ceil((K + 8 rb0 - bw - j0 - 3) / 4)
#pragma unroll
      for (int i = 0; i < TD_MAXT; ++i) {
        if (i >= nmine) break;
        const int km = i == irhs ? 0 : kmin0 + 8 * i;
        if (km > TD_JC / 4 - 1) continue;
        const double* Wi = Wl + (rb0 + 4 * i) * 8;
#pragma unroll
        for (int ks = 0; ks < TD_JC / 4; ++ks)
          if (ks >= km) td_mma(s0[i], s1[i], Wi[ks * 4 * RS], bf[ks]);
      }
    }
    td_cp_wait<0>();
    __syncthreads();  // also publishes the assembly when there are no chunks
#undef TD_ISSUE
    // P = A - S in Pa, then into the 4 x 4 register tiles of the elimination
#pragma unroll
    for (int i = 0; i < TD_MAXT; ++i) {
      if (i < nmine) {
        const int r = (rb0 + 4 * i) * 8 + (lane >> 2), c = cb * 8 + 2 * (lane & 3);
        Pa[c * RS + r] -= s0[i];
        Pa[(c + 1) * RS + r] -= s1[i];
      }
    }
    __syncthreads();
    double p[4][4];
#pragma unroll
    for (int b2 = 0; b2 < 4; ++b2) {
      double2 v01 = make_double2(0.0, 0.0), v23 = v01;
      if (act) {
        v01 = *reinterpret_cast<const double2*>(Pa + (c0 + b2) * RS + r0);
        v23 = *reinterpret_cast<const double2*>(Pa + (c0 + b2) * RS + r0 + 2);
      }
      p[0][b2] = v01.x; p[1][b2] = v01.y; p[2][b2] = v23.x; p[3][b2] = v23.y;
    }
    // elimination, column group g = columns 4g .. 4g + 3
    for (int g = 0; g < TD_NB / 4; ++g) {
      if (act && tr == g && tc == g) {  // the diagonal block
        bool okp = true;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const double pv = p[k][k];
          okp = okp && pv > 0.0 && isfinite(pv);
          const double iv = td_rcp(pv);
          dinv[k] = iv;
          piv[4 * g + k] = pv;
#pragma unroll
          for (int c2 = k + 1; c2 < 4; ++c2) {
            const double f = p[c2][k] * iv;
#pragma unroll
            for (int r2 = c2; r2 < 4; ++r2) p[r2][c2] -= p[r2][k] * f;
          }
        }
        if (!okp) *bad = 1;
#pragma unroll
        for (int a2 = 0; a2 < 4; ++a2)
#pragma unroll
          for (int b2 = 0; b2 < 4; ++b2) dfac[a2 * 4 + b2] = p[a2][b2];
      }
      __syncthreads();
      if (act && tc == g) {  // the column group's other rows, then publish the group
        if (tr != g) {
#pragma unroll
          for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int c2 = k + 1; c2 < 4; ++c2) {
              const double f = dfac[c2 * 4 + k] * dinv[k];
#pragma unroll
              for (int a2 = 0; a2 < 4; ++a2) p[a2][c2] -= p[a2][k] * f;
            }
        }
        const int o6 = 6 * tr;  // padded position of row r0
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const double ivk = dinv[k];
          *reinterpret_cast<double2*>(cg + k * CS + o6) = make_double2(p[0][k], p[1][k]);
          *reinterpret_cast<double2*>(cg + k * CS + o6 + 2) = make_double2(p[2][k], p[3][k]);
          *reinterpret_cast<double2*>(cgs + k * CS + o6) = make_double2(p[0][k] * ivk, p[1][k] * ivk);
          *reinterpret_cast<double2*>(cgs + k * CS + o6 + 2) = make_double2(p[2][k] * ivk, p[3][k] * ivk);
        }
      }
      __syncthreads();
      if (act && tc > g) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const double2 l01 = *reinterpret_cast<const double2*>(cg + k * CS + 6 * tr);
          const double2 l23 = *reinterpret_cast<const double2*>(cg + k * CS + 6 * tr + 2);
          const double2 f01 = *reinterpret_cast<const double2*>(cgs + k * CS + 6 * tc);
          const double2 f23 = *reinterpret_cast<const double2*>(cgs + k * CS + 6 * tc + 2);
          const double l[4] = {l01.x, l01.y, l23.x, l23.y}, f[4] = {f01.x, f01.y, f23.x, f23.y};
#pragma unroll
          for (int a2 = 0; a2 < 4; ++a2)
#pragma unroll
            for (int b2 = 0; b2 < 4; ++b2) p[a2][b2] -= l[a2] * f[b2];
        }
      }
    }
    __syncthreads();
    if (*bad) return false;
    // L = P diag(pivots)^-1/2 into Pa (zero outside the band), y of the panel's unknowns
    if (act) {  // rows past R stay zero; row R's entry is rewritten by the next assembly
#pragma unroll
      for (int b2 = 0; b2 < 4; ++b2) {
        const int c = c0 + b2;
        const double sc = rsqrt(piv[c]);
        double v[4];
#pragma unroll
        for (int a2 = 0; a2 < 4; ++a2) {
          const int r = r0 + a2;
          v[a2] = r >= c && r - c <= bw && r < R ? p[a2][b2] * sc : 0.0;
          if (r == R) yb[K + c] = p[a2][b2] * sc;
        }
        *reinterpret_cast<double2*>(Pa + c * RS + r0) = make_double2(v[0], v[1]);
        *reinterpret_cast<double2*>(Pa + c * RS + r0 + 2) = make_double2(v[2], v[3]);
      }
    }
    __syncthreads();
    for (int c = warp; c < TD_NB; c += NT / 32)  // coalesced copy to the band storage
      for (int d = lane; d <= bw; d += 32) {
        Lb[(int64_t)(K + c) * ld + d] = Pa[c * RS + c + d];
        Pa[c * RS + c + d] = 0.0;
      }
    __syncthreads();
  }
  return true;
}

// One displacement solve per instance and OC iteration by the banded Cholesky
// factor (instances marked direct; the others and failed ones are solved by
// PCG in topo_iteration).  Writes u (original dof order) and b; moduli as in
// topo_iteration.
template <int NT>
__global__ void __launch_bounds__(NT, 1) topo_direct(TopoArgs a) {
  extern __shared__ __align__(16) double dsm[];
  __shared__ double ke[64];
  __shared__ double red[72];
  __shared__ double piv[TD_NB], ysm[TD_NB], tsm[TD_NB];
  __shared__ int bad;
  __shared__ TopoInst I;
  const int idx = a.dorder[blockIdx.x];
  if (threadIdx.x == 0) {
    I = a.inst[idx];
    bad = 0;
  }
  __syncthreads();
  if (a.iter >= max(I.max_iter, 1)) return;
  for (int t = threadIdx.x; t < 64; t += NT) ke[t] = I.ke0[t];
  const int ne = I.ne, nd = I.ndof, np = I.npad;
  const double* phys = a.phys + I.eoff;
  double* E = a.E + I.eoff;
  const double* f = a.f + I.doff;
  const uint8_t* fixed = a.fixed + I.doff;
  double* u = a.u + I.doff;
  double* r = a.r + I.doff;
  double* q = a.q + I.doff;
  double* b = a.b + I.doff;
  double* Lb = a.L + I.loff;
  double* yb = a.yb + I.yoff;
  if (a.iter == 0 && threadIdx.x == 0) {
    a.total_iters[idx] = 0;
    a.flags[idx] = 0;
    a.refine[idx] = 0;
  }
  const double emin = I.emin, de = I.e0 - I.emin;
  for (int e = threadIdx.x; e < ne; e += NT) E[e] = emin + pow(a.iter == 0 ? I.vol_frac : phys[e], I.penal) * de;
  __syncthreads();
  if (I.has_lift) {
    apply_k<NT>(I, E, a.ulift + I.doff, q, fixed, false, ke);
    __syncthreads();
    for (int d = threadIdx.x; d < nd; d += NT) b[d] = fixed[d] ? 0.0 : f[d] - q[d];
  } else {
    for (int d = threadIdx.x; d < nd; d += NT) b[d] = fixed[d] ? 0.0 : f[d];
  }
  __syncthreads();
  for (int k = threadIdx.x; k < np; k += NT) yb[k] = k < nd ? b[band_to_dof(I, k)] : 0.0;
  __syncthreads();
  const int RS = td_rs(I.bw);
  bool ok = band_factor_forward<NT>(I, E, fixed, ke, Lb, yb, dsm, piv, &bad);
  int steps = 0;
  if (ok) {
    band_backward<NT>(np, I.bw, RS, Lb, yb, dsm, tsm);
    for (int d = threadIdx.x; d < nd; d += NT) u[d] = fixed[d] ? 0.0 : yb[dof_to_band(I, d)];
    const double stop = a.tol * a.tol;
    for (;;) {
      __syncthreads();
      apply_k<NT>(I, E, u, q, fixed, true, ke);
      __syncthreads();
      double rr = 0.0, bb = 0.0;
      for (int d = threadIdx.x; d < nd; d += NT) {
        const double rd = fixed[d] ? 0.0 : b[d] - q[d];
        r[d] = rd;
        rr += rd * rd;
        bb += b[d] * b[d];
      }
      block_sum2<NT>(rr, bb, red);
      if (rr <= stop * bb) break;
      if (steps == TD_REFINE) { ok = false; break; }
      ++steps;
      for (int k = threadIdx.x; k < np; k += NT) yb[k] = k < nd ? r[band_to_dof(I, k)] : 0.0;
      __syncthreads();
      for (int K = 0; K < np; K += TD_NB) {
        band_load_panel<NT>(K, I.bw, RS, Lb, dsm);
        __syncthreads();
        band_forward_panel<NT>(K, np, I.bw, RS, dsm, yb, ysm);
      }
      band_backward<NT>(np, I.bw, RS, Lb, yb, dsm, tsm);
      for (int d = threadIdx.x; d < nd; d += NT)
        if (!fixed[d]) u[d] += yb[dof_to_band(I, d)];
    }
  }
  if (threadIdx.x == 0) {
    a.direct_ok[idx] = ok ? 1 : 0;
    a.refine[idx] += steps;
  }
}

template <int NT>
__global__ void __launch_bounds__(NT, 1) topo_iteration(TopoArgs a) {
  __shared__ double ke[64];
  __shared__ double red[72];
  __shared__ TopoInst I;
  const int idx = a.order[blockIdx.x];
  if (threadIdx.x == 0) I = a.inst[idx];
  __syncthreads();
  if (a.iter >= max(I.max_iter, 1)) return;
  for (int t = threadIdx.x; t < 64; t += NT) ke[t] = I.ke0[t];
  const int ne = I.ne, nd = I.ndof;
  double* x = a.x + I.eoff;
  double* phys = a.phys + I.eoff;
  double* E = a.E + I.eoff;
  double* raw = a.raw + I.eoff;
  double* sens = a.sens + I.eoff;
  double* xnew = a.xnew + I.eoff;
  const double* f = a.f + I.doff;
  const double* ufix = a.ufix + I.doff;
  const uint8_t* fixed = a.fixed + I.doff;
  double* u = a.u + I.doff;
  double* r = a.r + I.doff;
  double* p = a.p + I.doff;
  double* q = a.q + I.doff;
  double* dinv = a.dinv + I.doff;
  double* b = a.b + I.doff;
  const double emin = I.emin, de = I.e0 - I.emin;
  // solved by topo_direct in this iteration (u and b are set)
  const bool solved = I.direct && a.direct_ok[idx];

  if (a.iter == 0) {  // uniform start (topopt:353), zero initial guess
    for (int e = threadIdx.x; e < ne; e += NT) { x[e] = I.vol_frac; phys[e] = I.vol_frac; }
    if (!solved) {
      for (int d = threadIdx.x; d < nd; d += NT) u[d] = 0.0;
      if (threadIdx.x == 0 && !I.direct) { a.total_iters[idx] = 0; a.flags[idx] = 0; }
    }
  }
  __syncthreads();
  // moduli (assemble, topopt:224)
  for (int e = threadIdx.x; e < ne; e += NT) E[e] = emin + pow(phys[e], I.penal) * de;
  __syncthreads();
  if (!solved) {
    // Jacobi diagonal of K_FF
    for (int n = threadIdx.x; n < I.nx * I.ny; n += NT) {
      const int i = n % I.nx, j = n / I.nx;
      double d0 = 0.0, d1 = 0.0;
      for (int dj = -1; dj <= 0; ++dj)
        for (int di = -1; di <= 0; ++di) {
          const int ei = i + di, ej = j + dj;
          if (ei < 0 || ei >= I.nelx || ej < 0 || ej >= I.nely) continue;
          const int ln = local_node(di, dj);
          const double Ee = E[ej * I.nelx + ei];
          d0 += Ee * ke[(2 * ln) * 8 + 2 * ln];
          d1 += Ee * ke[(2 * ln + 1) * 8 + 2 * ln + 1];
        }
      dinv[2 * n] = fixed[2 * n] ? 0.0 : 1.0 / d0;
      dinv[2 * n + 1] = fixed[2 * n + 1] ? 0.0 : 1.0 / d1;
    }
    // right-hand side: b = f_F - K_FD u_D (reduce_system lifting, first bcs value)
    if (I.has_lift) {
      apply_k<NT>(I, E, a.ulift + I.doff, q, fixed, false, ke);
      __syncthreads();
      for (int d = threadIdx.x; d < nd; d += NT) b[d] = fixed[d] ? 0.0 : f[d] - q[d];
    } else {
      for (int d = threadIdx.x; d < nd; d += NT) b[d] = fixed[d] ? 0.0 : f[d];
    }
    __syncthreads();
    // two-level preconditioner (per-instance coarse space): transforms once, A_c^-1 per OC iteration
    __shared__ double yc[TP_MAXC], uc[TP_MAXC], cm[TP_MAXC];
    const bool two = a.coarse && I.nc > 0;
    double* Ac = a.Ac + I.coff;
    double* Tm = a.Tm + I.toff;
    if (two) {
      if (a.iter == 0) coarse_transforms<NT>(I, fixed, Tm);
      __syncthreads();
      coarse_assemble_invert<NT>(I, E, fixed, ke, Tm, p, q, Ac, yc);
    }
    // r = b - K x0 (warm start), z = M r, p = z
    apply_k<NT>(I, E, u, q, fixed, true, ke);
    __syncthreads();
    double rz = 0.0, rr = 0.0, bb = 0.0;
    for (int d = threadIdx.x; d < nd; d += NT) {
      const double rd = b[d] - q[d];
      r[d] = rd;
      rr += rd * rd;
      bb += b[d] * b[d];
      if (!two) {
        const double z = dinv[d] * rd;
        p[d] = z;
        rz += rd * z;
      }
    }
    if (two) {
      coarse_solve<NT>(I, Tm, Ac, r, yc, uc, cm);
      rz = two_level_z<NT>(I, r, dinv, cm, p);
    }
    block_sum2<NT>(rz, rr, red);
    bb = block_sum<NT>(bb, red);
    const double stop = a.tol * a.tol * bb;
    int it = 0;
    bool conv = rr <= stop;
    while (!conv && it < a.max_pcg) {
      double pq = apply_k<NT>(I, E, p, q, fixed, true, ke);
      pq = block_sum<NT>(pq, red);
      if (!(pq > 0.0)) {
        if (threadIdx.x == 0) atomicOr(a.flags + idx, 2);
        break;
      }
      const double alpha = rz / pq;
      double rzn = 0.0, rrn = 0.0;
      for (int d = threadIdx.x; d < nd; d += NT) {
        u[d] += alpha * p[d];
        const double rd = r[d] - alpha * q[d];
        r[d] = rd;
        if (!two) rzn += rd * dinv[d] * rd;
        rrn += rd * rd;
      }
      block_sum2<NT>(rzn, rrn, red);
      ++it;
      conv = rrn <= stop;
      if (conv) break;
      if (two) {  // z = D^-1 r + P A_c^-1 P^T r into q
        coarse_solve<NT>(I, Tm, Ac, r, yc, uc, cm);
        rzn = two_level_z<NT>(I, r, dinv, cm, q);
        rzn = block_sum<NT>(rzn, red);
        const double beta = rzn / rz;
        rz = rzn;
        for (int d = threadIdx.x; d < nd; d += NT) p[d] = q[d] + beta * p[d];
      } else {
        const double beta = rzn / rz;
        rz = rzn;
        for (int d = threadIdx.x; d < nd; d += NT) p[d] = dinv[d] * r[d] + beta * p[d];
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      a.last_iters[idx] = it;
      a.total_iters[idx] += it;
      if (!conv) atomicOr(a.flags + idx, 1);
    }
  }  // !solved
  // compliance c = f . u, u with the fixed dofs' (last) values (topopt:360,368)
  double c = 0.0;
  for (int d = threadIdx.x; d < nd; d += NT) c += f[d] * (fixed[d] ? ufix[d] : u[d]);
  c = block_sum<NT>(c, red);
  if (threadIdx.x == 0) {
    if (a.iter == 0) a.hist[I.hoff] = c;
    if (I.max_iter > 0) a.hist[I.hoff + a.iter + 1] = c;
  }
  if (I.max_iter == 0) return;  // the initial solve only (topopt:356-360)
  __shared__ double wtab[TP_WTAB];
  if (I.density_filter) filter_table<false, NT>(I, wtab);
  else filter_table<true, NT>(I, wtab);
  __syncthreads();
  // raw sensitivity (topopt:371-375), element_quad_form (topopt:241-254)
  for (int e = threadIdx.x; e < ne; e += NT) {
    const int ei = e % I.nelx, ej = e / I.nelx;
    const int n0 = ej * I.nx + ei;
    const int nodes[4] = {n0, n0 + 1, n0 + I.nx + 1, n0 + I.nx};
    double ue[8];
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int c2 = 0; c2 < 2; ++c2) {
        const int d = 2 * nodes[k] + c2;
        ue[2 * k + c2] = fixed[d] ? ufix[d] : u[d];
      }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) s += ue[i] * ke[i * 8 + j] * ue[j];
    raw[e] = -I.penal * pow(phys[e], I.penal - 1.0) * de * s;
  }
  __syncthreads();
  if (!I.density_filter) {
    // filter_sensitivity (topopt:259-279), then oc_update (topopt:284-331)
    for (int e = threadIdx.x; e < ne; e += NT) {
      double num, den;
      filter_window<true>(I, e, raw, nullptr, wtab, num, den);
      sens[e] = den > 0.0 ? num / den : raw[e];
    }
    __syncthreads();
    const double target = I.vol_frac * (double)ne;
    double lo = 1e-9, hi = 1e9, lambda = 1.0;
    for (int k = 0; k < 60; ++k) {
      lambda = 0.5 * (lo + hi);
      double s = 0.0;
      for (int e = threadIdx.x; e < ne; e += NT) s += oc_candidate(x[e], -sens[e], lambda, I.move);
      s = block_sum<NT>(s, red);
      if (s > target) lo = lambda; else hi = lambda;
    }
    for (int e = threadIdx.x; e < ne; e += NT) {
      const double v = oc_candidate(x[e], -sens[e], lambda, I.move);
      x[e] = v;
      phys[e] = v;
    }
  } else {
    // density filter (88-line code): dc = H (dc / Hs), dv = H (1 / Hs); OC on
    // the design with the volume of the filtered (physical) densities.
    // E (free until the next launch) holds Hs, sens = dc, raw = dv.
    for (int e = threadIdx.x; e < ne; e += NT) {
      double num, den;
      filter_window<false>(I, e, nullptr, nullptr, wtab, num, den);
      E[e] = den;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < ne; e += NT) {
      double num, den;
      filter_window<false>(I, e, raw, E, wtab, num, den);
      sens[e] = num;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < ne; e += NT) {
      double num, den;
      filter_window<false>(I, e, nullptr, E, wtab, num, den);
      raw[e] = num;
    }
    __syncthreads();
    const double target = I.vol_frac * (double)ne;
    double l1 = 0.0, l2 = 1e9;
    for (int guard = 0; guard < 200 && (l2 - l1) / (l1 + l2) > 1e-3; ++guard) {
      const double lmid = 0.5 * (l2 + l1);
      for (int e = threadIdx.x; e < ne; e += NT) {
        const double oc = x[e] * sqrt(fmax(0.0, -sens[e] / raw[e] / lmid));
        xnew[e] = fmax(0.0, fmax(x[e] - I.move, fmin(1.0, fmin(x[e] + I.move, oc))));
      }
      __syncthreads();
      double s = 0.0;
      for (int e = threadIdx.x; e < ne; e += NT) {
        double num, den;
        filter_window<false>(I, e, xnew, nullptr, wtab, num, den);
        const double v = num / E[e];
        phys[e] = v;
        s += v;
      }
      s = block_sum<NT>(s, red);
      if (s > target) l1 = lmid; else l2 = lmid;
    }
    for (int e = threadIdx.x; e < ne; e += NT) x[e] = xnew[e];
  }
}

void launch_nt(int nt, int nblocks, const TopoArgs& a, cudaStream_t s) {
  switch (nt) {
    case 256: topo_iteration<256><<<nblocks, 256, 0, s>>>(a); break;
    case 512: topo_iteration<512><<<nblocks, 512, 0, s>>>(a); break;
    default: topo_iteration<1024><<<nblocks, 1024, 0, s>>>(a); break;
  }
  TPT_CHECK_LAUNCH();
}

// element_stiffness_unit (topopt:166-217) in the reference's operation order
// (host code, compiled without floating-point contraction).
void element_stiffness_unit(double nu, double h, double* ke) {
  const double c = 1.0 / (1.0 - nu * nu);
  const double d[3][3] = {{c, c * nu, 0.0}, {c * nu, c, 0.0}, {0.0, 0.0, c * (1.0 - nu) / 2.0}};
  const double gp[2] = {-1.0 / std::sqrt(3.0), 1.0 / std::sqrt(3.0)}, gw[2] = {1.0, 1.0};  // gauss_legendre(2)
  const double jdet = h * h / 4.0, scale = 2.0 / h;
  const double s4[4] = {-1.0, 1.0, 1.0, -1.0}, t4[4] = {-1.0, -1.0, 1.0, 1.0};  // Quad4 corners
  for (int t = 0; t < 64; ++t) ke[t] = 0.0;
  for (int qa = 0; qa < 2; ++qa)
    for (int qb = 0; qb < 2; ++qb) {
      const double xi = gp[qa], eta = gp[qb], w = gw[qa] * gw[qb];
      double bm[3][8] = {{0}};
      for (int n = 0; n < 4; ++n) {  // Quad4::grad (element:141-153), scaled to x, y
        const double gx = 0.25 * s4[n] * (1.0 + t4[n] * eta), gy = 0.25 * (1.0 + s4[n] * xi) * t4[n];
        const double nx_ = scale * gx, ny_ = scale * gy;
        bm[0][2 * n] = nx_;
        bm[1][2 * n + 1] = ny_;
        bm[2][2 * n] = ny_;
        bm[2][2 * n + 1] = nx_;
      }
      double db[3][8];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 8; ++j) {
          double s = 0.0;
          for (int k = 0; k < 3; ++k) s += d[i][k] * bm[k][j];
          db[i][j] = s;
        }
      for (int i = 0; i < 8; ++i)
        for (int j = 0; j < 8; ++j) {
          double s = 0.0;
          for (int k = 0; k < 3; ++k) s += bm[k][i] * db[k][j];
          ke[i * 8 + j] += w * jdet * s;
        }
    }
}

}  // namespace

void topopt_element_stiffness(double nu, double h, double* ke) { element_stiffness_unit(nu, h, ke); }

// Host driver: validate, pack, tune, capture, run.
void topopt_batch(tptfem_context* ctx, const tptfem_topopt_instance* in, int n, const tptfem_topopt_opts* opts,
                  double* compliance, double* densities, tptfem_topopt_stats* stats) {
  cudaStream_t s = ctx->stream;
  TPT_REQUIRE(n >= 1 && in && compliance && densities, TPTFEM_ERR_INVALID_ARG, "topopt: no instances or outputs");
  const double tol = opts && opts->rel_tol > 0 ? opts->rel_tol : 1e-10;
  const int max_pcg = opts && opts->max_pcg_iter > 0 ? opts->max_pcg_iter : 50000;
  std::vector<TopoInst> inst(n);
  int64_t eoff = 0, doff = 0, hoff = 0, coff = 0, toff = 0;
  const bool two_level = !(opts && opts->plain_jacobi);
  const bool allow_direct = !(opts && opts->pcg_only);
  size_t free_b = 0, total_b = 0;
  TPT_CUDA(cudaMemGetInfo(&free_b, &total_b));
  const int64_t band_budget = (int64_t)(free_b / 2 / sizeof(double));  // factor storage, in doubles
  int64_t loff = 0, yoff = 0;
  int launches = 0;
  for (int k = 0; k < n; ++k) {
    const tptfem_topopt_instance& P = in[k];
    TPT_REQUIRE(P.nelx >= 1 && P.nely >= 1 && (int64_t)(P.nelx + 1) * (P.nely + 1) * 2 < (1LL << 30),
                TPTFEM_ERR_INVALID_ARG, "topopt: grid size out of range");
    TPT_REQUIRE(P.max_iter >= 0 && P.max_iter <= 100000, TPTFEM_ERR_INVALID_ARG, "topopt: max_iter out of range");
    TPT_REQUIRE(P.h > 0 && P.e0 > 0 && P.nu > -1 && P.nu < 0.5 && P.vol_frac > 0 && P.vol_frac <= 1 &&
                    P.penal >= 1 && P.filter_radius > 0 && P.move_limit > 0 && P.emin >= 0 && P.emin < P.e0,
                TPTFEM_ERR_INVALID_ARG, "topopt: parameter out of range");
    TopoInst& I = inst[k];
    std::memset(&I, 0, sizeof(I));
    I.nelx = P.nelx; I.nely = P.nely; I.nx = P.nelx + 1; I.ny = P.nely + 1;
    I.ne = P.nelx * P.nely; I.ndof = 2 * I.nx * I.ny;
    I.max_iter = P.max_iter; I.density_filter = P.density_filter != 0;
    I.eoff = eoff; I.doff = doff; I.hoff = hoff;
    I.h = P.h; I.e0 = P.e0; I.penal = P.penal; I.vol_frac = P.vol_frac; I.radius = P.filter_radius;
    I.move = P.move_limit; I.emin = P.emin;
    element_stiffness_unit(P.nu, P.h, I.ke0);
    // direct solve when the band fits the kernel's panel and the factor fits the memory budget
    I.yfast = I.ny <= I.nx;
    I.bw = 2 * std::min(I.nx, I.ny) + 3;
    I.npad = (I.ndof + TD_NB - 1) / TD_NB * TD_NB;
    const int64_t lsize = (int64_t)I.npad * (I.bw + 1);
    I.direct = allow_direct && I.bw <= TD_MAXBW && loff + lsize <= band_budget;
    I.loff = loff;
    I.yoff = yoff;
    if (I.direct) {
      loff += lsize;
      yoff += I.npad;
    }
    // coarse space: about 48 aggregates of ag x ag nodes (at least 4 x 4)
    I.ag = std::max(4, (int)std::ceil(std::sqrt((double)I.nx * I.ny / 48.0)));
    I.nax = std::max(1, I.nx / I.ag);
    I.nay = std::max(1, I.ny / I.ag);
    while (3 * I.nax * I.nay > TP_MAXC) {
      ++I.ag;
      I.nax = std::max(1, I.nx / I.ag);
      I.nay = std::max(1, I.ny / I.ag);
    }
    I.nc = two_level && !I.direct ? 3 * I.nax * I.nay : 0;
    I.coff = coff;
    I.toff = toff;
    coff += (int64_t)I.nc * I.nc;
    toff += (int64_t)I.nax * I.nay * 9;
    eoff += I.ne;
    doff += I.ndof;
    hoff += P.max_iter + 1;
    launches = std::max(launches, std::max(P.max_iter, 1));  // max_iter 0 still solves once
  }
  // loads and Dirichlet data (first bcs value lifts, last overwrites: assembly:525,555-557)
  std::vector<double> f(doff, 0.0), ulift(doff, 0.0), ufix(doff, 0.0);
  std::vector<uint8_t> fixed(doff, 0);
  for (int k = 0; k < n; ++k) {
    const tptfem_topopt_instance& P = in[k];
    TopoInst& I = inst[k];
    double* fk = f.data() + I.doff;
    if (P.f) {
      for (int d = 0; d < I.ndof; ++d) {
        TPT_REQUIRE(std::isfinite(P.f[d]), TPTFEM_ERR_INVALID_ARG, "topopt: non-finite load");
        fk[d] = P.f[d];
      }
    } else {
      TPT_REQUIRE(P.load_dof >= 0 && P.load_dof < I.ndof && std::isfinite(P.load_value), TPTFEM_ERR_INVALID_ARG,
                  "topopt: point load out of range");
      fk[P.load_dof] = P.load_value;
    }
    uint8_t* fx = fixed.data() + I.doff;
    std::vector<uint8_t> seen(I.ndof, 0);
    if (P.bc_dof) {
      TPT_REQUIRE(P.nbc >= 0, TPTFEM_ERR_INVALID_ARG, "topopt: negative Dirichlet count");
      for (int64_t t = 0; t < P.nbc; ++t) {
        const int64_t d = P.bc_dof[t];
        TPT_REQUIRE(d >= 0 && d < I.ndof, TPTFEM_ERR_INVALID_ARG, "topopt: Dirichlet dof out of range");
        const double v = P.bc_val ? P.bc_val[t] : 0.0;
        TPT_REQUIRE(std::isfinite(v), TPTFEM_ERR_INVALID_ARG, "topopt: non-finite Dirichlet value");
        if (!seen[d]) { ulift[I.doff + d] = v; seen[d] = 1; }
        ufix[I.doff + d] = v;
        fx[d] = 1;
      }
    } else {  // cantilever_load (topopt:398-415): the whole left edge
      for (int j = 0; j < I.ny; ++j) { fx[2 * j * I.nx] = 1; fx[2 * j * I.nx + 1] = 1; }
    }
    for (int d = 0; d < I.ndof; ++d) if (ulift[I.doff + d] != 0.0) I.has_lift = 1;
  }
  // largest instances first (an instance solved directly costs topo_iteration its filter and OC work only)
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  auto weight = [&](int k) {
    return (int64_t)inst[k].ndof * std::max(inst[k].max_iter, 1) * (inst[k].direct ? 1 : 64);
  };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return weight(a) > weight(b); });
  // the direct kernel's blocks: largest band work (npad bw^2) first
  std::vector<int> dorder;
  int64_t td_smem = 0;
  for (int k = 0; k < n; ++k)
    if (inst[k].direct) {
      dorder.push_back(k);
      td_smem = std::max(td_smem, td_smem_doubles(inst[k].bw) * (int64_t)sizeof(double));
    }
  std::stable_sort(dorder.begin(), dorder.end(), [&](int a, int b) {
    return (int64_t)inst[a].npad * inst[a].bw * inst[a].bw > (int64_t)inst[b].npad * inst[b].bw * inst[b].bw;
  });
  const int ndirect = (int)dorder.size();
  if (ndirect)
    TPT_CUDA(cudaFuncSetAttribute(topo_direct<TD_NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)td_smem));

  DevBuf<TopoInst> d_inst;
  DevBuf<int> d_order, d_last, d_flags, d_dorder, d_ok;
  DevBuf<long long> d_total, d_refine;
  DevBuf<double> dL, dyb;
  DevBuf<double> ex, ephys, eE, eraw, esens, exnew, df, dlift, dfix, du, dr, dp, dq, ddinv, db, dhist, dAc, dTm;
  DevBuf<uint8_t> dfixed;
  d_inst.alloc(n, s); d_order.alloc(n, s); d_last.alloc(n, s); d_flags.alloc(n, s); d_total.alloc(n, s);
  d_ok.alloc(n, s); d_refine.alloc(n, s); d_dorder.alloc(std::max(ndirect, 1), s);
  dL.alloc(std::max<int64_t>(loff, 1), s);
  dyb.alloc(std::max<int64_t>(yoff, 1), s);
  for (auto* v : {&ex, &ephys, &eE, &eraw, &esens, &exnew}) v->alloc(std::max<int64_t>(eoff, 1), s);
  for (auto* v : {&df, &dlift, &dfix, &du, &dr, &dp, &dq, &ddinv, &db}) v->alloc(std::max<int64_t>(doff, 1), s);
  dfixed.alloc(std::max<int64_t>(doff, 1), s);
  dhist.alloc(std::max<int64_t>(hoff, 1), s);
  dAc.alloc(std::max<int64_t>(coff, 1), s);
  dTm.alloc(std::max<int64_t>(toff, 1), s);
  d_inst.upload(inst.data(), n);
  d_order.upload(order.data(), n);
  df.upload(f.data(), doff);
  dlift.upload(ulift.data(), doff);
  dfix.upload(ufix.data(), doff);
  dfixed.upload(fixed.data(), doff);
  if (ndirect) d_dorder.upload(dorder.data(), ndirect);
  d_last.zero(); d_flags.zero(); d_total.zero(); dhist.zero(); d_ok.zero(); d_refine.zero();

  TopoArgs a{};
  a.inst = d_inst.p; a.order = d_order.p; a.iter = 0; a.max_pcg = max_pcg; a.tol = tol;
  a.x = ex.p; a.phys = ephys.p; a.E = eE.p; a.raw = eraw.p; a.sens = esens.p; a.xnew = exnew.p;
  a.f = df.p; a.ulift = dlift.p; a.ufix = dfix.p; a.fixed = dfixed.p;
  a.u = du.p; a.r = dr.p; a.p = dp.p; a.q = dq.p; a.dinv = ddinv.p; a.b = db.p;
  a.hist = dhist.p; a.last_iters = d_last.p; a.total_iters = d_total.p; a.flags = d_flags.p;
  a.Ac = dAc.p; a.Tm = dTm.p; a.coarse = two_level ? 1 : 0;
  a.dorder = d_dorder.p; a.L = dL.p; a.yb = dyb.p; a.direct_ok = d_ok.p; a.refine = d_refine.p;
  auto launch_direct = [&]() {
    if (!ndirect) return;
    topo_direct<TD_NT><<<ndirect, TD_NT, td_smem, s>>>(a);
    TPT_CHECK_LAUNCH();
  };

  cudaEvent_t ev0 = ctx->ev[0], ev1 = ctx->ev[1], ev2 = ctx->ev[2];
  float tune_ms = 0.f;
  // autotuner: threads per instance, chosen by timing the first iteration
  int nt = opts && (opts->block_threads == 256 || opts->block_threads == 512 || opts->block_threads == 1024)
               ? opts->block_threads : 0;
  uint64_t sig = 1469598103934665603ull;
  for (int k = 0; k < n; ++k)
    for (uint64_t v : {(uint64_t)inst[k].nelx, (uint64_t)inst[k].nely, (uint64_t)inst[k].density_filter,
                       (uint64_t)inst[k].nc, (uint64_t)inst[k].direct})
      sig = (sig ^ v) * 1099511628211ull;
  if (!nt) {
    auto it = ctx->topo_tuned.find(sig);
    if (it != ctx->topo_tuned.end()) nt = it->second;
  }
  if (!nt) {
    float best = 1e30f;
    TPT_CUDA(cudaEventRecord(ev0, s));
    a.iter = 0;
    launch_direct();  // the candidates time the remaining work of iteration 0
    for (int cand : {256, 512, 1024}) {
      float ms = 0.f;
      TPT_CUDA(cudaEventRecord(ev1, s));
      a.iter = 0;
      launch_nt(cand, n, a, s);
      TPT_CUDA(cudaEventRecord(ev2, s));
      TPT_CUDA(cudaEventSynchronize(ev2));
      TPT_CUDA(cudaEventElapsedTime(&ms, ev1, ev2));
      if (ms < best) { best = ms; nt = cand; }
    }
    TPT_CUDA(cudaEventRecord(ev1, s));
    TPT_CUDA(cudaEventSynchronize(ev1));
    TPT_CUDA(cudaEventElapsedTime(&tune_ms, ev0, ev1));
    ctx->topo_tuned[sig] = nt;
  }
  // all iterations as one graph (iteration 0 re-initialises the state)
  float run_ms = 0.f;
  const bool graph = !opts || opts->use_graph;
  cudaGraphExec_t exec = nullptr;
  if (graph) {
    cudaGraph_t g = nullptr;
    TPT_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < launches; ++k) {
      a.iter = k;
      launch_direct();
      switch (nt) {
        case 256: topo_iteration<256><<<n, 256, 0, s>>>(a); break;
        case 512: topo_iteration<512><<<n, 512, 0, s>>>(a); break;
        default: topo_iteration<1024><<<n, 1024, 0, s>>>(a); break;
      }
    }
    cudaError_t ce = cudaStreamEndCapture(s, &g);
    TPT_CUDA(ce);
    ce = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    TPT_CUDA(ce);
  }
  TPT_CUDA(cudaEventRecord(ev0, s));
  if (graph) {
    TPT_CUDA(cudaGraphLaunch(exec, s));
  } else {
    for (int k = 0; k < launches; ++k) {
      a.iter = k;
      launch_direct();
      launch_nt(nt, n, a, s);
    }
  }
  TPT_CUDA(cudaEventRecord(ev1, s));
  const cudaError_t se = cudaEventSynchronize(ev1);
  if (exec) cudaGraphExecDestroy(exec);
  TPT_CUDA(se);
  TPT_CUDA(cudaGetLastError());
  TPT_CUDA(cudaEventElapsedTime(&run_ms, ev0, ev1));
  // results: reference-mode instances report the design, density-filter ones
  // the physical (filtered) densities
  std::vector<double> hist(std::max<int64_t>(hoff, 1)), xs(std::max<int64_t>(eoff, 1)), ps(std::max<int64_t>(eoff, 1));
  std::vector<long long> total(n), refine(n);
  std::vector<int> flags(n);
  d_refine.download(refine.data(), n);
  dhist.download(hist.data(), hoff);
  ex.download(xs.data(), eoff);
  ephys.download(ps.data(), eoff);
  d_total.download(total.data(), n);
  d_flags.download(flags.data(), n);
  TPT_CUDA(cudaStreamSynchronize(s));
  std::copy(hist.begin(), hist.begin() + hoff, compliance);
  for (const TopoInst& I : inst) {
    const std::vector<double>& src = I.density_filter ? ps : xs;
    std::copy(src.begin() + I.eoff, src.begin() + I.eoff + I.ne, densities + I.eoff);
  }
  long long tot = 0, ref = 0;
  int bad = 0;
  for (int k = 0; k < n; ++k) { tot += total[k]; ref += refine[k]; bad += flags[k] != 0; }
  if (stats) {
    stats->total_ms = run_ms;
    stats->tune_ms = tune_ms;
    stats->pcg_iterations = tot;
    stats->block_threads = nt;
    stats->not_converged = bad;
    stats->refinement_steps = ref;
    stats->direct_instances = ndirect;
  }
  TPT_REQUIRE(bad == 0, TPTFEM_ERR_NOT_CONVERGED, "topopt: a displacement solve did not converge");
}

}  // namespace tptfem
