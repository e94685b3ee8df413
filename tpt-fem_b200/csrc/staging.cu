// staging.cu -- host <-> device transfers of large user arrays.
//
// The C ABI takes ordinary (pageable) host arrays.  Large ones are copied by
// several host threads into the context's pinned staging buffer (kept between
// calls, grown on demand) in chunks, each moved by its own DMA as soon as it is
// filled (downloads the same way in reverse), instead of the driver's
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
constexpr size_t STAGE_CHUNK = 8u << 20;      // pipelined transfers move chunks of this size

unsigned stage_threads(size_t bytes) {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  return (unsigned)std::max<size_t>(1, std::min<size_t>(std::min(16u, hw), bytes / (1u << 18)));
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

// Host -> device through the pinned buffer, pipelined: n staged elements of
// `elem` bytes in chunks; host thread t fills its slice of every chunk in turn
// (fill(i0, i1) writes staged elements [i0, i1) and returns false if the
// input there is invalid), and this thread issues each chunk's DMA as soon as
// every slice of it is in, so the copies overlap the host work on the next
// chunks.  Returns false if any fill did.
template <typename Fill>
bool staged_in(tptfem_context* ctx, void* dst, size_t n, size_t elem, Fill fill) {
  const size_t bytes = n * elem;
  char* p = static_cast<char*>(stage(ctx, bytes));
  const size_t cel = std::max<size_t>(1, STAGE_CHUNK / elem), nchunk = (n + cel - 1) / cel;
  const unsigned nt = stage_threads(bytes);
  std::vector<std::atomic<unsigned>> done(nchunk);
  for (auto& d : done) d.store(0);
  std::atomic<bool> ok(true);
  auto work = [&](unsigned t) {
    for (size_t c = 0; c < nchunk; ++c) {
      const size_t c0 = c * cel, c1 = std::min(n, c0 + cel), len = c1 - c0;
      const size_t b = c0 + len * t / nt, e = c0 + len * (t + 1) / nt;
      if (b < e && !fill(b, e)) ok = false;
      done[c].fetch_add(1, std::memory_order_release);
    }
  };
  std::vector<std::thread> th;
  for (unsigned t = 1; t < nt; ++t) th.emplace_back(work, t);
  // this thread fills slice 0 of each chunk, then issues the chunk once all
  // slices are in (a copy error is raised only after the workers have finished)
  cudaError_t err = cudaSuccess;
  for (size_t c = 0; c < nchunk; ++c) {
    const size_t c0 = c * cel, c1 = std::min(n, c0 + cel), len = c1 - c0;
    const size_t e = c0 + len / nt;
    if (c0 < e && !fill(c0, e)) ok = false;
    done[c].fetch_add(1, std::memory_order_release);
    while (done[c].load(std::memory_order_acquire) < nt) std::this_thread::yield();
    if (err == cudaSuccess)
      err = cudaMemcpyAsync(static_cast<char*>(dst) + c0 * elem, p + c0 * elem, len * elem, cudaMemcpyHostToDevice,
                            ctx->stream);
  }
  for (auto& x : th) x.join();
  TPT_CUDA(err);
  TPT_CUDA(cudaStreamSynchronize(ctx->stream));  // the staging buffer is reused by the next call
  return ok;
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
  staged_in(ctx, dst, bytes, 1, [&](size_t b, size_t e) {
    std::memcpy(p + b, s + b, e - b);
    return true;
  });
}

// Device -> host through the pinned buffer, pipelined: chunk c's DMA is
// followed by an event; host thread t copies its slice of each chunk out once
// that chunk's event has completed, while the next chunks are still moving.
void device_to_host(tptfem_context* ctx, void* dst, const void* src, size_t bytes) {
  if (!bytes) return;
  if (bytes < STAGE_MIN_BYTES) {
    TPT_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    TPT_CUDA(cudaStreamSynchronize(ctx->stream));
    return;
  }
  char* p = static_cast<char*>(stage(ctx, bytes));
  const size_t nchunk = (bytes + STAGE_CHUNK - 1) / STAGE_CHUNK;
  std::vector<cudaEvent_t> ev(nchunk, nullptr);
  for (size_t c = 0; c < nchunk; ++c) {
    TPT_CUDA(cudaEventCreateWithFlags(&ev[c], cudaEventDisableTiming));
    const size_t c0 = c * STAGE_CHUNK, len = std::min(bytes, c0 + STAGE_CHUNK) - c0;
    TPT_CUDA(cudaMemcpyAsync(p + c0, static_cast<const char*>(src) + c0, len, cudaMemcpyDeviceToHost, ctx->stream));
    TPT_CUDA(cudaEventRecord(ev[c], ctx->stream));
  }
  const unsigned nt = stage_threads(bytes);
  char* d = static_cast<char*>(dst);
  std::atomic<int> err(0);
  auto work = [&](unsigned t) {
    for (size_t c = 0; c < nchunk; ++c) {
      if (cudaEventSynchronize(ev[c]) != cudaSuccess) { err = 1; return; }
      const size_t c0 = c * STAGE_CHUNK, len = std::min(bytes, c0 + STAGE_CHUNK) - c0;
      const size_t b = c0 + len * t / nt, e = c0 + len * (t + 1) / nt;
      std::memcpy(d + b, p + b, e - b);
    }
  };
  std::vector<std::thread> th;
  for (unsigned t = 1; t < nt; ++t) th.emplace_back(work, t);
  work(0);
  for (auto& x : th) x.join();
  for (auto e : ev) cudaEventDestroy(e);
  TPT_REQUIRE(!err, TPTFEM_ERR_DEVICE, "device-to-host copy failed");
}

bool host_to_device_ids(tptfem_context* ctx, int* dst, const int64_t* src, size_t count, int64_t limit) {
  if (!count) return true;
  int* p = static_cast<int*>(stage(ctx, count * sizeof(int)));
  return staged_in(ctx, dst, count, sizeof(int), [&](size_t b, size_t e) {
    bool good = true;
    for (size_t i = b; i < e; ++i) {
      const int64_t v = src[i];
      good &= v >= 0 && v < limit;
      p[i] = (int)v;
    }
    return good;
  });
}

bool host_to_device_finite(tptfem_context* ctx, double* dst, const double* src, size_t count) {
  if (!count) return true;
  double* p = static_cast<double*>(stage(ctx, count * sizeof(double)));
  return staged_in(ctx, dst, count, sizeof(double), [&](size_t b, size_t e) {
    bool good = true;
    for (size_t i = b; i < e; ++i) {
      good &= std::isfinite(src[i]);
      p[i] = src[i];
    }
    return good;
  });
}

}  // namespace tptfem
