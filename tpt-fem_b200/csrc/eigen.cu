// eigen.cu -- Lanczos and power iteration on a device CSR matrix.
//
// Restates lanczos_eigs (crates/tpt-fem-eigen/src/lib.rs:134-262) and
// power_iteration (lib.rs:62-88) with the matrix-vector products on the GPU:
//   * Lanczos from v0 = e_0 with full re-orthogonalisation; the reference
//     does one modified Gram-Schmidt pass over v_0..v_j, here classical
//     Gram-Schmidt runs twice (two passes of V^T w and w -= V p), which is as
//     stable and reads the basis with two coalesced sweeps instead of j+1;
//   * alpha_j = (A v_j) . v_j before the re-orthogonalisation, beta_j = |w|,
//     stop at beta < 1e-12 or after lanczos_dim vectors, as the reference;
//   * the tridiagonal T is diagonalised on the host by the reference's cyclic
//     Jacobi method (lib.rs:166-214), Ritz vectors V q_i normalised on the GPU.
// The basis lives in HBM as lanczos_dim columns of n doubles.  Dot products
// are reduced per block and the block partials summed on the host in a fixed
// order, so results are reproducible.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "objects.hpp"

namespace tptfem {

namespace {

constexpr int EG_THREADS = 256;
constexpr int EG_MAXK = 64;  // basis columns per re-orthogonalisation tile

int eg_blocks(int64_t n) { return std::max(1, std::min(sm_count() * 4, ceil_div(n, EG_THREADS))); }

// partial[b * nk + k] = sum over this block's rows of V[:, k0 + k] . w
__global__ void __launch_bounds__(EG_THREADS) eg_project(int64_t n, int nk, const double* __restrict__ V, int64_t ld,
                                                         const double* __restrict__ w, double* __restrict__ partial) {
  __shared__ double sh[EG_THREADS / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int k = 0; k < nk; ++k) {
    const double* v = V + (int64_t)k * ld;
    double s = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * EG_THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * EG_THREADS)
      s += v[i] * w[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) sh[wid] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int q = 0; q < EG_THREADS / 32; ++q) t += sh[q];
      partial[(int64_t)blockIdx.x * nk + k] = t;
    }
    __syncthreads();
  }
}

// w -= V[:, 0..nk) c   (c in shared memory)
__global__ void eg_subtract(int64_t n, int nk, const double* __restrict__ V, int64_t ld, const double* __restrict__ c,
                            double* __restrict__ w) {
  __shared__ double cs[EG_MAXK];
  for (int k = threadIdx.x; k < nk; k += blockDim.x) cs[k] = c[k];
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double s = w[i];
    for (int k = 0; k < nk; ++k) s -= cs[k] * V[(int64_t)k * ld + i];
    w[i] = s;
  }
}

// y = V[:, 0..nk) c   (Ritz vector assembly)
__global__ void eg_combine(int64_t n, int nk, const double* __restrict__ V, int64_t ld, const double* __restrict__ c,
                           double* __restrict__ y) {
  __shared__ double cs[EG_MAXK];
  for (int k = threadIdx.x; k < nk; k += blockDim.x) cs[k] = c[k];
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double s = y[i];
    for (int k = 0; k < nk; ++k) s += cs[k] * V[(int64_t)k * ld + i];
    y[i] = s;
  }
}

__global__ void eg_scale(int64_t n, const double* __restrict__ x, double a, double* __restrict__ y) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = x[i] * a;
}

__global__ void eg_start_ramp(int64_t n, double* __restrict__ x) {  // x_i = i + 1
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = (double)(i + 1);
}

struct Eg {
  tptfem_context* ctx;
  const MatrixData& M;
  int64_t n;
  int blocks;
  DevBuf<double> part, coef;
  std::vector<double> hpart;
  Eg(tptfem_context* c, const MatrixData& m) : ctx(c), M(m), n(m.nrows), blocks(eg_blocks(m.nrows)) {
    part.alloc((size_t)blocks * EG_MAXK, c->stream);
    coef.alloc(EG_MAXK, c->stream);
    hpart.resize((size_t)blocks * EG_MAXK);
  }
  void matvec(const double* x, double* y) {
    csr_matvec_f64(ctx, n, M.row_ptr.p, M.col.p, M.val.p, x, y);
  }
  // out[k] = V[:, k0 + k] . w for k < nk (nk <= EG_MAXK), block partials summed in order
  void project(const double* V, int64_t ld, int nk, const double* w, double* out) {
    eg_project<<<blocks, EG_THREADS, 0, ctx->stream>>>(n, nk, V, ld, w, part.p);
    TPT_CHECK_LAUNCH();
    TPT_CUDA(cudaMemcpyAsync(hpart.data(), part.p, (size_t)blocks * nk * sizeof(double), cudaMemcpyDeviceToHost,
                             ctx->stream));
    TPT_CUDA(cudaStreamSynchronize(ctx->stream));
    for (int k = 0; k < nk; ++k) {
      double s = 0.0;
      for (int b = 0; b < blocks; ++b) s += hpart[(size_t)b * nk + k];
      out[k] = s;
    }
  }
  double dot(const double* a, const double* b) {
    double r;
    project(a, n, 1, b, &r);
    return r;
  }
  // w -= V[:, 0..k) p  or  y += V[:, 0..k) p, in tiles of EG_MAXK columns
  void apply(const double* V, int64_t ld, int k, const double* p, double* w, bool subtract) {
    for (int k0 = 0; k0 < k; k0 += EG_MAXK) {
      const int nk = std::min(EG_MAXK, k - k0);
      TPT_CUDA(cudaMemcpyAsync(coef.p, p + k0, nk * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
      if (subtract) eg_subtract<<<blocks, EG_THREADS, 0, ctx->stream>>>(n, nk, V + k0 * ld, ld, coef.p, w);
      else eg_combine<<<blocks, EG_THREADS, 0, ctx->stream>>>(n, nk, V + k0 * ld, ld, coef.p, w);
      TPT_CHECK_LAUNCH();
    }
    TPT_CUDA(cudaStreamSynchronize(ctx->stream));  // p is host memory the copies read
  }
  void scale(const double* x, double a, double* y) {
    eg_scale<<<blocks, EG_THREADS, 0, ctx->stream>>>(n, x, a, y);
    TPT_CHECK_LAUNCH();
  }
};

// Cyclic Jacobi eigen-decomposition of a dense symmetric matrix
// (crates/tpt-fem-eigen/src/lib.rs:166-214, same sweep order and threshold);
// eigenvectors as columns of v.
void jacobi_sym(std::vector<std::vector<double>>& a, int max_sweeps, std::vector<double>& eig,
                std::vector<std::vector<double>>& v) {
  const size_t n = a.size();
  v.assign(n, std::vector<double>(n, 0.0));
  for (size_t i = 0; i < n; ++i) v[i][i] = 1.0;
  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    bool changed = false;
    for (size_t p = 0; p < n; ++p)
      for (size_t q = p + 1; q < n; ++q) {
        if (!(std::fabs(a[p][q]) > 1e-12)) continue;
        changed = true;
        const double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
        const double t = theta >= 0.0 ? 1.0 / (theta + std::sqrt(1.0 + theta * theta))
                                      : 1.0 / (theta - std::sqrt(1.0 + theta * theta));
        const double c = 1.0 / std::sqrt(1.0 + t * t), s = t * c;
        for (size_t i = 0; i < n; ++i) {
          const double aip = a[i][p], aiq = a[i][q];
          a[i][p] = c * aip - s * aiq;
          a[i][q] = s * aip + c * aiq;
        }
        for (size_t i = 0; i < n; ++i) {
          const double api = a[p][i], aqi = a[q][i];
          a[p][i] = c * api - s * aqi;
          a[q][i] = s * api + c * aqi;
        }
        for (size_t i = 0; i < n; ++i) {
          const double vip = v[i][p], viq = v[i][q];
          v[i][p] = c * vip - s * viq;
          v[i][q] = s * vip + c * viq;
        }
      }
    if (!changed) break;
  }
  eig.resize(n);
  for (size_t i = 0; i < n; ++i) eig[i] = a[i][i];
}

}  // namespace

int lanczos_eigs(tptfem_context* ctx, const MatrixData& M, int num, int largest, int dim, double* values,
                 double* vectors) {
  const int64_t n = M.nrows;
  TPT_REQUIRE(n > 0 && M.ref_ncols <= n, TPTFEM_ERR_INVALID_ARG, "Lanczos needs a square matrix");
  TPT_REQUIRE(dim >= 1 && num >= 0, TPTFEM_ERR_INVALID_ARG, "lanczos_dim must be >= 1 and num >= 0");
  dim = (int)std::min<int64_t>(dim, n);
  cudaStream_t s = ctx->stream;
  Eg E(ctx, M);
  DevBuf<double> V, w;
  V.alloc((size_t)n * dim, s);
  w.alloc(n, s);
  TPT_CUDA(cudaMemsetAsync(V.p, 0, (size_t)n * sizeof(double), s));
  const double one = 1.0;
  TPT_CUDA(cudaMemcpyAsync(V.p, &one, sizeof(double), cudaMemcpyHostToDevice, s));  // v0 = e_0
  std::vector<double> alpha, beta, p(dim);
  int m = 0;
  for (int j = 0; j < dim; ++j) {
    const double* vj = V.p + (int64_t)j * n;
    E.matvec(vj, w.p);
    alpha.push_back(E.dot(w.p, vj));
    m = j + 1;
    for (int pass = 0; pass < 2; ++pass) {  // full re-orthogonalisation against v_0..v_j
      for (int k0 = 0; k0 <= j; k0 += EG_MAXK) E.project(V.p + (int64_t)k0 * n, n, std::min(EG_MAXK, j + 1 - k0),
                                                         w.p, p.data() + k0);
      E.apply(V.p, n, j + 1, p.data(), w.p, true);
    }
    if (j + 1 == dim) break;
    const double b = std::sqrt(E.dot(w.p, w.p));
    if (b < 1e-12) break;
    beta.push_back(b);
    E.scale(w.p, 1.0 / b, V.p + (int64_t)(j + 1) * n);
  }
  std::vector<std::vector<double>> T(m, std::vector<double>(m, 0.0)), Q;
  for (int i = 0; i < m; ++i) T[i][i] = alpha[i];
  for (int i = 0; i + 1 < m; ++i) T[i][i + 1] = T[i + 1][i] = beta[i];
  std::vector<double> eig;
  jacobi_sym(T, 200, eig, Q);
  std::vector<int> idx(m);
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return eig[a] < eig[b]; });
  const int take = std::min(num, m);
  std::vector<int> order(take);
  for (int t = 0; t < take; ++t) order[t] = largest ? idx[m - 1 - t] : idx[t];
  std::vector<double> q(m);
  for (int t = 0; t < take; ++t) {
    const int i = order[t];
    values[t] = eig[i];
    if (!vectors) continue;
    for (int r = 0; r < m; ++r) q[r] = Q[r][i];
    TPT_CUDA(cudaMemsetAsync(w.p, 0, (size_t)n * sizeof(double), s));
    E.apply(V.p, n, m, q.data(), w.p, false);
    const double nv = std::sqrt(E.dot(w.p, w.p));
    E.scale(w.p, 1.0 / nv, w.p);
    TPT_CUDA(cudaMemcpyAsync(vectors + (size_t)t * n, w.p, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  TPT_CUDA(cudaStreamSynchronize(s));
  return take;
}

int power_iteration(tptfem_context* ctx, const MatrixData& M, int max_iter, double tol, double* lambda, double* x_out) {
  const int64_t n = M.nrows;
  TPT_REQUIRE(n > 0 && M.ref_ncols <= n, TPTFEM_ERR_INVALID_ARG, "power iteration needs a square matrix");
  cudaStream_t s = ctx->stream;
  Eg E(ctx, M);
  DevBuf<double> x, y;
  x.alloc(n, s);
  y.alloc(n, s);
  eg_start_ramp<<<E.blocks, EG_THREADS, 0, s>>>(n, x.p);
  TPT_CHECK_LAUNCH();
  E.scale(x.p, 1.0 / std::sqrt(E.dot(x.p, x.p)), x.p);
  double lam = 0.0;
  int it = 0;
  for (; it < max_iter; ++it) {
    E.matvec(x.p, y.p);
    E.scale(y.p, 1.0 / std::sqrt(E.dot(y.p, y.p)), x.p);
    E.matvec(x.p, y.p);
    const double nw = E.dot(x.p, y.p) / E.dot(x.p, x.p);  // rayleigh (lib.rs:38-40)
    if (std::fabs(nw - lam) < tol * std::max(std::fabs(nw), 1.0)) {
      lam = nw;
      ++it;
      break;
    }
    lam = nw;
  }
  *lambda = lam;
  if (x_out) x.download(x_out, n);
  TPT_CUDA(cudaStreamSynchronize(s));
  return it;
}

}  // namespace tptfem
