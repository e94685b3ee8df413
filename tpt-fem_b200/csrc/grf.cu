// grf.cu -- seeded Gaussian random field by random Fourier features, the
// input generator of the heterogeneous-Poisson configuration:
//
//   g(x) = scale * sum_m cos(w_m . x + phi_m),   scale = sqrt(2 / M),
//
// evaluated for many points.  The frequencies w (3 x M, row-major) and phases
// phi come from the caller (a seeded host RNG), so a field is defined by its
// seed alone; the sum runs over m in ascending order with the dot product
// formed as ((x w0 + y w1) + z w2) + phi without contraction, so every GPU
// running this library produces the same bits for the same inputs.
#include <algorithm>

#include "objects.hpp"

namespace tptfem {
namespace {

constexpr int GRF_THREADS = 256;
constexpr int64_t GRF_CHUNK = 1 << 22;  // points per device pass (96 MB of coordinates)

__global__ void __launch_bounds__(GRF_THREADS) grf_kernel(int64_t n, int M, const double* __restrict__ pts,
                                                          const double* __restrict__ wphi, double scale,
                                                          double* __restrict__ out) {
  extern __shared__ double sh[];  // w0[M], w1[M], w2[M], phi[M]
  for (int i = threadIdx.x; i < 4 * M; i += blockDim.x) sh[i] = wphi[i];
  __syncthreads();
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    const double x = pts[3 * p], y = pts[3 * p + 1], z = pts[3 * p + 2];
    double acc = 0.0;
    for (int m = 0; m < M; ++m) {
      const double a = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, sh[m]), __dmul_rn(y, sh[M + m])),
                                           __dmul_rn(z, sh[2 * M + m])),
                                 sh[3 * M + m]);
      acc = __dadd_rn(acc, cos(a));
    }
    out[p] = __dmul_rn(acc, scale);
  }
}

}  // namespace

void grf_eval(tptfem_context* ctx, const double* h_points, int64_t n, const double* h_w, const double* h_phi, int M,
              double scale, double* h_out) {
  TPT_REQUIRE(M >= 1 && M <= GRF_MAX_FEATURES, TPTFEM_ERR_INVALID_ARG, "feature count must be in 1..2048");
  cudaStream_t s = ctx->stream;
  std::vector<double> wphi(4 * (size_t)M);
  std::copy(h_w, h_w + 3 * (size_t)M, wphi.begin());
  std::copy(h_phi, h_phi + M, wphi.begin() + 3 * (size_t)M);
  DevBuf<double> d_wphi, d_pts, d_out;
  d_wphi.alloc(wphi.size(), s);
  d_wphi.upload(wphi.data(), wphi.size());
  const int64_t chunk = std::min<int64_t>(n, GRF_CHUNK);
  d_pts.alloc(3 * chunk, s);
  d_out.alloc(chunk, s);
  const size_t shmem = 4 * (size_t)M * sizeof(double);
  TPT_CUDA(cudaFuncSetAttribute(grf_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem));
  for (int64_t p0 = 0; p0 < n; p0 += chunk) {
    const int64_t len = std::min(chunk, n - p0);
    host_to_device(ctx, d_pts.p, h_points + 3 * p0, 3 * len * sizeof(double));
    const int grid = (int)std::min<int64_t>(ceil_div(len, GRF_THREADS), (int64_t)sm_count() * 8);
    grf_kernel<<<grid, GRF_THREADS, shmem, s>>>(len, M, d_pts.p, d_wphi.p, scale, d_out.p);
    TPT_CHECK_LAUNCH();
    device_to_host(ctx, h_out + p0, d_out.p, len * sizeof(double));
  }
  TPT_CUDA(cudaStreamSynchronize(s));
}

}  // namespace tptfem
