// staging.cu -- host <-> device transfers of large user arrays.
//
// The C ABI takes ordinary (pageable) host arrays.  Large ones are copied by
// several host threads into the context's pinned staging buffer (kept between
// calls, grown on demand) and moved by one DMA, instead of the driver's
// single-threaded pageable path; connectivity is narrowed to int32 and
// coefficients are checked on the way.  Small arrays go directly.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "objects.hpp"

namespace tptfem {

namespace {

constexpr size_t STAGE_MIN_BYTES = 1u << 20;  // below this the direct copy is as fast

// f(begin, end) on contiguous ranges of [0, n), one host thread per range.
template <typename Fn>
void parallel_ranges(size_t n, Fn f) {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t nt = std::min<size_t>(std::min(16u, hw), std::max<size_t>(1, n / (1u << 16)));
  if (nt <= 1) {
    f(size_t(0), n);
    return;
  }
  std::vector<std::thread> th;
  th.reserve(nt);
  for (size_t t = 0; t < nt; ++t) th.emplace_back(f, n * t / nt, n * (t + 1) / nt);
  for (auto& x : th) x.join();
}

void* stage(tptfem_context* ctx, size_t bytes) {
  if (ctx->h_stage_bytes < bytes) {
    if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
    ctx->h_stage = nullptr;
    ctx->h_stage_bytes = 0;
    TPT_CUDA(cudaHostAlloc(&ctx->h_stage, bytes, cudaHostAllocDefault));
    ctx->h_stage_bytes = bytes;
  }
  return ctx->h_stage;
}

void dma_in(tptfem_context* ctx, void* dst, const void* pinned, size_t bytes) {
  TPT_CUDA(cudaMemcpyAsync(dst, pinned, bytes, cudaMemcpyHostToDevice, ctx->stream));
  TPT_CUDA(cudaStreamSynchronize(ctx->stream));  // the staging buffer is reused by the next call
}

}  // namespace

void host_to_device(tptfem_context* ctx, void* dst, const void* src, size_t bytes) {
  if (!bytes) return;
  if (bytes < STAGE_MIN_BYTES) {
    TPT_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
    return;
  }
  char* p = static_cast<char*>(stage(ctx, bytes));
  const char* s = static_cast<const char*>(src);
  parallel_ranges(bytes, [&](size_t b, size_t e) { std::memcpy(p + b, s + b, e - b); });
  dma_in(ctx, dst, p, bytes);
}

void device_to_host(tptfem_context* ctx, void* dst, const void* src, size_t bytes) {
  if (!bytes) return;
  if (bytes < STAGE_MIN_BYTES) {
    TPT_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    TPT_CUDA(cudaStreamSynchronize(ctx->stream));
    return;
  }
  char* p = static_cast<char*>(stage(ctx, bytes));
  TPT_CUDA(cudaMemcpyAsync(p, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  TPT_CUDA(cudaStreamSynchronize(ctx->stream));
  char* d = static_cast<char*>(dst);
  parallel_ranges(bytes, [&](size_t b, size_t e) { std::memcpy(d + b, p + b, e - b); });
}

bool host_to_device_ids(tptfem_context* ctx, int* dst, const int64_t* src, size_t count, int64_t limit) {
  if (!count) return true;
  int* p = static_cast<int*>(stage(ctx, count * sizeof(int)));
  std::atomic<bool> ok(true);
  parallel_ranges(count, [&](size_t b, size_t e) {
    bool good = true;
    for (size_t i = b; i < e; ++i) {
      const int64_t v = src[i];
      good &= v >= 0 && v < limit;
      p[i] = (int)v;
    }
    if (!good) ok = false;
  });
  if (!ok) return false;
  dma_in(ctx, dst, p, count * sizeof(int));
  return true;
}

bool host_to_device_finite(tptfem_context* ctx, double* dst, const double* src, size_t count) {
  if (!count) return true;
  double* p = static_cast<double*>(stage(ctx, count * sizeof(double)));
  std::atomic<bool> ok(true);
  parallel_ranges(count, [&](size_t b, size_t e) {
    bool good = true;
    for (size_t i = b; i < e; ++i) {
      good &= std::isfinite(src[i]);
      p[i] = src[i];
    }
    if (!good) ok = false;
  });
  if (!ok) return false;
  dma_in(ctx, dst, p, count * sizeof(double));
  return true;
}

}  // namespace tptfem
