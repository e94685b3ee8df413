// noalloc.cu -- relative residual ||b - A x||_2 / ||b||_2 of a device-resident
// CSR system without allocating any device memory.
//
// Some callers cannot let a library allocate: applications that reserve all of
// the GPU's memory up front under a fixed budget (an allocation could fail or
// evict their own buffers), or that run this check inside a tight time-step or
// optimisation loop where cudaMalloc/cudaFree would add a device-wide
// synchronisation to every call.  For them this entry point takes every input
// and output from the caller and keeps its only scratch -- the per-block
// partial sums, the last-block ticket, the two totals and an error flag -- in
// the file-scope array below.
//
// The array is a fixed NOALLOC_SLOTS doubles (16,448 bytes), resident on every
// GPU that loads the library until the process exits.  All calls share it: it
// keeps the previous call's contents, so each call clears the ticket and flag
// it needs at zero before launching, and calls whose kernels overlap on the
// GPU (different streams, or several host threads) race on it and must be
// serialised by the caller.  The array's device address is looked up once per
// device and cached; a call that fails with a device error drops the cached
// address (and SM count), so the next call looks them up again -- after a
// cudaDeviceReset, for instance.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <mutex>

#include "objects.hpp"

namespace tptfem {
namespace {

constexpr int SPMV_THREADS = 256;

// Error-free transformations (Knuth TwoSum; TwoProduct through FMA).
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  const double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}
__device__ __forceinline__ void two_prod(double a, double b, double& p, double& e) {
  p = a * b;
  e = __fma_rn(a, b, -p);
}

// Fixed-order block sum of two doubles (result in thread 0).
__device__ __forceinline__ void block_sum2(double (&v)[2]) {
  __shared__ double sh[2][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_down_sync(0xffffffffu, v[i], o);
  __syncthreads();
  if (lane == 0) { sh[0][wid] = v[0]; sh[1][wid] = v[1]; }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      double t = lane < nw ? sh[i][lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
      v[i] = t;
    }
  }
}

// Per-block partials in `partials`, then a fixed-order sum by the last block to
// arrive (atomic ticket).  True in thread 0 of the last block, totals in v.
__device__ __forceinline__ bool grid_sum2(double (&v)[2], double* partials, unsigned* ticket) {
  block_sum2(v);
  __shared__ bool last;
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = v[0];
    partials[gridDim.x + blockIdx.x] = v[1];
    __threadfence();
    last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double acc[2] = {0.0, 0.0};
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
    acc[0] += __ldcg(partials + b);
    acc[1] += __ldcg(partials + gridDim.x + b);
  }
  block_sum2(acc);
  if (threadIdx.x == 0) {
    v[0] = acc[0];
    v[1] = acc[1];
    *ticket = 0;
  }
  return threadIdx.x == 0;
}

constexpr int NOALLOC_MAX_BLOCKS = 1024;                  // grid limit of the residual kernel
constexpr int NOALLOC_PARTIALS = 2 * NOALLOC_MAX_BLOCKS;  // two sums per block
constexpr int NOALLOC_OUT = NOALLOC_PARTIALS;             // ||r||^2, ||b||^2
constexpr int NOALLOC_TICKET = NOALLOC_PARTIALS + 2;      // unsigned in a double slot
constexpr int NOALLOC_FLAG = NOALLOC_PARTIALS + 3;        // unsigned in a double slot
constexpr int NOALLOC_SLOTS = NOALLOC_PARTIALS + 8;

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_SLOTS];

constexpr unsigned FLAG_COLUMN = 1u;  // a column index outside [0, n)
constexpr unsigned FLAG_ROW = 2u;     // a row range outside [0, nnz] or reversed

constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};
int g_noalloc_sms[NOALLOC_MAX_DEVICES] = {};

// Residual row sums as in residual_f64 (compensated), without storing r.  A
// row whose range [rp[row], rp[row+1]) is reversed or leaves [0, nnz), and a
// column index outside [0, n), are flagged and skipped, so malformed arrays
// never send a load outside the nnz entries the caller declared.
template <int LANES>
__global__ void __launch_bounds__(SPMV_THREADS) residual_norms_noalloc(int n, int nnz, const int* __restrict__ rp,
                                                                       const int* __restrict__ ci,
                                                                       const double* __restrict__ va,
                                                                       const double* __restrict__ x,
                                                                       const double* __restrict__ b,
                                                                       double* scratch) {
  constexpr int RPW = 32 / LANES;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int sub = (threadIdx.x & 31) / LANES;
  const int lane = threadIdx.x & (LANES - 1);
  unsigned* ticket = reinterpret_cast<unsigned*>(scratch + NOALLOC_TICKET);
  unsigned* flag = reinterpret_cast<unsigned*>(scratch + NOALLOC_FLAG);
  double d[2] = {0.0, 0.0};
  for (int base = warp * RPW; base < n; base += nwarps * RPW) {
    const int row = base + sub;
    const bool valid = row < n;
    double hi = 0.0, lo = 0.0;
    if (valid) {
      int kb = rp[row], ke = rp[row + 1];
      if (kb < 0 || ke > nnz || kb > ke) {
        if (lane == 0) atomicOr(flag, FLAG_ROW);
        kb = ke = 0;
      }
      for (int k = kb + lane; k < ke; k += LANES) {
        const int c = ci[k];
        if (c < 0 || c >= n) { atomicOr(flag, FLAG_COLUMN); continue; }
        double p, pe, s, se;
        two_prod(va[k], x[c], p, pe);
        two_sum(hi, p, s, se);
        hi = s;
        lo += pe + se;
      }
    }
#pragma unroll
    for (int o = LANES / 2; o > 0; o >>= 1) {
      const double oh = __shfl_down_sync(0xffffffffu, hi, o, LANES);
      const double ol = __shfl_down_sync(0xffffffffu, lo, o, LANES);
      double s, se;
      two_sum(hi, oh, s, se);
      hi = s;
      lo += ol + se;
    }
    if (valid && lane == 0) {
      double r1, e1;
      two_sum(b[row], -hi, r1, e1);
      const double ri = r1 + (e1 - lo);
      d[0] += ri * ri;
      d[1] += b[row] * b[row];
    }
  }
  if (grid_sum2(d, scratch, ticket)) {
    scratch[NOALLOC_OUT] = d[0];
    scratch[NOALLOC_OUT + 1] = d[1];
  }
}

void put_err(char* buf, size_t len, const char* msg) {
  if (!buf || !len) return;
  size_t m = std::strlen(msg);
  if (m >= len) m = len - 1;
  std::memcpy(buf, msg, m);
  buf[m] = 0;
}

}  // namespace
}  // namespace tptfem

using namespace tptfem;

extern "C" tptfem_status tptfem_rel_residual_noalloc(int device, void* stream, int64_t n, const int32_t* row_ptrs,
                                                     const int32_t* col_ind, const double* values, const double* x,
                                                     const double* b, double* rel_residual, char* err,
                                                     size_t err_len) {
  put_err(err, err_len, "");
  if (!row_ptrs || !col_ind || !values || !x || !b || !rel_residual) {
    put_err(err, err_len, "a pointer argument is NULL");
    return TPTFEM_ERR_INVALID_ARG;
  }
  if (n < 1 || n > INT_MAX - 1) {
    put_err(err, err_len, "n must be in 1..2147483646 (int32 rows and columns)");
    return TPTFEM_ERR_INVALID_ARG;
  }
  if (device < 0 || device >= NOALLOC_MAX_DEVICES) {
    put_err(err, err_len, "device index out of range");
    return TPTFEM_ERR_INVALID_ARG;
  }
  int prev = 0;
  if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess) {
    put_err(err, err_len, "cannot make the requested device current");
    return TPTFEM_ERR_DEVICE;
  }
  tptfem_status rc = TPTFEM_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  do {
    double* scratch = nullptr;
    int sms = 0;
    {
      // once per device, with that device current: the host-side symbol is only
      // a stand-in, the kernel needs the device address of the array
      std::lock_guard<std::mutex> lock(g_noalloc_mu);
      if (!g_noalloc_ptr[device]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
          put_err(err, err_len, "cudaGetSymbolAddress failed for the scratch array");
          rc = TPTFEM_ERR_DEVICE;
          break;
        }
        int count = 0;
        if (cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || count < 1) {
          put_err(err, err_len, "cannot read the device's multiprocessor count");
          rc = TPTFEM_ERR_DEVICE;
          break;
        }
        g_noalloc_ptr[device] = static_cast<double*>(p);
        g_noalloc_sms[device] = count;
      }
      scratch = g_noalloc_ptr[device];
      sms = g_noalloc_sms[device];
    }
    int nnz = 0;
    if (cudaMemcpyAsync(&nnz, row_ptrs + n, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      put_err(err, err_len, "reading row_ptrs[n] failed");
      rc = TPTFEM_ERR_DEVICE;
      break;
    }
    if (nnz < 0) {
      put_err(err, err_len, "row_ptrs[n] (the number of stored entries) is negative");
      rc = TPTFEM_ERR_INVALID_ARG;
      break;
    }
    const double avg = (double)nnz / (double)n;
    const int lanes = avg <= 3 ? 2 : avg <= 12 ? 4 : avg <= 40 ? 8 : avg <= 96 ? 16 : 32;
    int grid = (int)std::min<int64_t>((n * lanes + SPMV_THREADS - 1) / SPMV_THREADS, NOALLOC_MAX_BLOCKS);
    grid = std::max(1, std::min(grid, sms * 8));
    // the ticket and the flag must start at zero; partials are overwritten
    if (cudaMemsetAsync(scratch + NOALLOC_TICKET, 0, 2 * sizeof(double), s) != cudaSuccess) {
      put_err(err, err_len, "clearing the scratch array failed");
      rc = TPTFEM_ERR_DEVICE;
      break;
    }
    const int nn = (int)n;
    switch (lanes) {
      case 2: residual_norms_noalloc<2><<<grid, SPMV_THREADS, 0, s>>>(nn, nnz, row_ptrs, col_ind, values, x, b, scratch); break;
      case 4: residual_norms_noalloc<4><<<grid, SPMV_THREADS, 0, s>>>(nn, nnz, row_ptrs, col_ind, values, x, b, scratch); break;
      case 8: residual_norms_noalloc<8><<<grid, SPMV_THREADS, 0, s>>>(nn, nnz, row_ptrs, col_ind, values, x, b, scratch); break;
      case 16: residual_norms_noalloc<16><<<grid, SPMV_THREADS, 0, s>>>(nn, nnz, row_ptrs, col_ind, values, x, b, scratch); break;
      default: residual_norms_noalloc<32><<<grid, SPMV_THREADS, 0, s>>>(nn, nnz, row_ptrs, col_ind, values, x, b, scratch); break;
    }
    double out[4] = {0.0, 0.0, 0.0, 0.0};
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(out, scratch + NOALLOC_OUT, 4 * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      put_err(err, err_len, "residual kernel failed");
      rc = TPTFEM_ERR_DEVICE;
      break;
    }
    unsigned bad = 0;
    std::memcpy(&bad, &out[3], sizeof(unsigned));
    if (bad & FLAG_ROW) {
      put_err(err, err_len, "row_ptrs is not non-decreasing within [0, row_ptrs[n]]");
      rc = TPTFEM_ERR_INVALID_ARG;
      break;
    }
    if (bad) {
      put_err(err, err_len, "a column index is outside [0, n)");
      rc = TPTFEM_ERR_INVALID_ARG;
      break;
    }
    const double r2 = out[0], b2 = out[1];
    *rel_residual = b2 > 0.0 ? std::sqrt(r2) / std::sqrt(b2) : std::sqrt(r2);
  } while (false);
  if (rc == TPTFEM_ERR_DEVICE) {
    // the cached address may be stale (e.g. after a device reset): look it up again next time
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    g_noalloc_ptr[device] = nullptr;
    g_noalloc_sms[device] = 0;
  }
  cudaSetDevice(prev);
  return rc;
}
