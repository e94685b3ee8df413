// common.cuh -- internal plumbing shared by the tptfem CUDA sources.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>
#include <vector>

#include "../../include/tptfem.h"

namespace tptfem {

// A status + message carried from the failing call up to the C ABI.
struct Error {
  tptfem_status status;
  std::string msg;
};

#define TPT_CUDA(call)                                                                       \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      throw ::tptfem::Error{TPTFEM_ERR_DEVICE, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
  } while (0)

#define TPT_CHECK_LAUNCH() TPT_CUDA(cudaGetLastError())

#define TPT_REQUIRE(cond, status, msg)                  \
  do {                                                  \
    if (!(cond)) throw ::tptfem::Error{(status), (msg)}; \
  } while (0)

// Stream-ordered device buffer (cudaMallocAsync on the owning stream).
template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t s = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n), s(o.s) { o.p = nullptr; o.n = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) { release(); p = o.p; n = o.n; s = o.s; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DevBuf() { release(); }
  void alloc(size_t count, cudaStream_t stream) {
    release();
    s = stream;
    n = count;
    if (count) {
      cudaError_t e = cudaMallocAsync((void**)&p, count * sizeof(T), stream);
      if (e != cudaSuccess) {
        p = nullptr; n = 0;
        throw Error{TPTFEM_ERR_OUT_OF_MEMORY, std::string("device allocation failed: ") + cudaGetErrorString(e)};
      }
    }
  }
  void release() {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    n = 0;
  }
  void zero() {
    if (n) TPT_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
  }
  void upload(const T* h, size_t count) {
    if (count) TPT_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void download(T* h, size_t count) const {
    if (count) TPT_CUDA(cudaMemcpyAsync(h, p, count * sizeof(T), cudaMemcpyDeviceToHost, s));
  }
};

inline int ceil_div(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

// Error-free transformations (Knuth TwoSum; TwoProduct through FMA), for the
// compensated FP64 residuals of the solvers.
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  const double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}
__device__ __forceinline__ void two_prod(double a, double b, double& p, double& e) {
  p = a * b;
  e = __fma_rn(a, b, -p);
}

// Number of SMs of the current device (cached per process; all B200s have 148).
int sm_count();

// Exclusive scan of n int32 counts into out (n+1 entries, out[n] = total).
// Returns the total; throws CREATION when it exceeds INT32_MAX.
int64_t exclusive_scan_i32(const int* in, int* out, int64_t n, cudaStream_t s);

}  // namespace tptfem
