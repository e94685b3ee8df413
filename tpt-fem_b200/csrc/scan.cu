// scan.cu -- exclusive prefix sum of int32 counts (row/segment pointers).
//
// Three passes over tiles of 2048 items: tile sums, one-block scan of the
// tile sums (int64, so an overflow of int32 is detected, not wrapped), and a
// rescan of every tile with its offset.
#include "common.cuh"

namespace tptfem {

namespace {
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ long long block_exclusive_scan(long long v, long long* total) {
  __shared__ long long warp_tot[SCAN_THREADS / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  long long x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[wid] = x;
  __syncthreads();
  if (wid == 0) {
    long long t = lane < SCAN_THREADS / 32 ? warp_tot[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      long long y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    if (lane < SCAN_THREADS / 32) warp_tot[lane] = t;
  }
  __syncthreads();
  long long base = wid ? warp_tot[wid - 1] : 0;
  if (total) *total = warp_tot[SCAN_THREADS / 32 - 1];
  long long r = base + x - v;
  __syncthreads();
  return r;
}

__global__ void tile_sums(const int* __restrict__ in, long long* __restrict__ sums, int64_t n) {
  int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
  long long s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    int64_t i = base + (int64_t)k * SCAN_THREADS + threadIdx.x;
    if (i < n) s += in[i];
  }
  long long tot;
  block_exclusive_scan(s, &tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void scan_sums(long long* __restrict__ sums, int64_t nb, long long* __restrict__ total) {
  long long carry = 0;
  for (int64_t c = 0; c < nb; c += SCAN_THREADS) {
    int64_t i = c + threadIdx.x;
    long long v = i < nb ? sums[i] : 0;
    long long tot;
    long long ex = block_exclusive_scan(v, &tot);
    if (i < nb) sums[i] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void tile_scan(const int* __restrict__ in, int* __restrict__ out, const long long* __restrict__ offs,
                          int64_t n) {
  int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
  int v[SCAN_ITEMS];
  long long s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    int64_t i = base + k;
    v[k] = i < n ? in[i] : 0;
    s += v[k];
  }
  long long run = offs[blockIdx.x] + block_exclusive_scan(s, nullptr);
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    int64_t i = base + k;
    if (i < n) out[i] = (int)run;
    run += v[k];
  }
}

__global__ void write_total(int* out, int64_t n, const long long* total) {
  long long t = *total;
  out[n] = t > 0x7fffffffLL ? -1 : (int)t;
}
}  // namespace

int64_t exclusive_scan_i32(const int* in, int* out, int64_t n, cudaStream_t s) {
  int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
  DevBuf<long long> sums;
  sums.alloc(nb + 1, s);
  if (nb > 0) {
    tile_sums<<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, sums.p, n);
    TPT_CHECK_LAUNCH();
    scan_sums<<<1, SCAN_THREADS, 0, s>>>(sums.p, nb, sums.p + nb);
    TPT_CHECK_LAUNCH();
  } else {
    TPT_CUDA(cudaMemsetAsync(sums.p, 0, sizeof(long long), s));
  }
  long long total = 0;
  TPT_CUDA(cudaMemcpyAsync(&total, sums.p + nb, sizeof(long long), cudaMemcpyDeviceToHost, s));
  TPT_CUDA(cudaStreamSynchronize(s));
  TPT_REQUIRE(total <= 0x7fffffffLL, TPTFEM_ERR_CREATION,
              "prefix sum exceeds the int32 index range of the device format");
  if (nb > 0) {
    tile_scan<<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, out, sums.p, n);
    TPT_CHECK_LAUNCH();
  }
  write_total<<<1, 1, 0, s>>>(out, n, sums.p + nb);
  TPT_CHECK_LAUNCH();
  return total;
}

int sm_count() {
  static int cached = 0;
  if (!cached) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&cached, cudaDevAttrMultiProcessorCount, dev);
    if (cached <= 0) cached = 148;
  }
  return cached;
}

}  // namespace tptfem
