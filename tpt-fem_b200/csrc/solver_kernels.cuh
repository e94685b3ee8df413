// solver_kernels.cuh -- device kernels of the PCG engine (solver.cu) and the
// FSAI preconditioner apply.  Included by solver.cu only.
#pragma once
#include <cuda_fp16.h>

#include <cmath>

#include "common.cuh"

namespace tptfem {

constexpr int VEC_THREADS = 256;
constexpr int SPMV_THREADS = 256;

enum { PC_JACOBI = 0, PC_FSAI = 1 };

struct PcgState {
  double rz[2];   // r.z by iteration parity
  double rz_old;  // rz used by the last alpha (for beta after a reliable update)
  double pq;
  double rr;      // recursive ||r||^2
  double upd2;    // request a reliable update when rr <= upd2
  int done;       // 0 running, 2 breakdown, 3 iteration cap, 4 update requested
  int iters;
  int max_iters;
  int pad;
  unsigned ticket[8];
};

// Preconditioner handed to the engine: Jacobi (dinv) or a factorised sparse
// approximate inverse M^-1 = G^T G with G = diag(sigma) (I + L), L strictly
// lower triangular: sigma^2 in FP32 and L in FP16 (CSR) with an explicit
// transpose (CSR), so both halves of the apply are row gathers.
template <typename T>
struct Precond {
  int kind = PC_JACOBI;
  const T* dinv = nullptr;
  int n = 0;
  int lanes = 4, grid = 1;
  const float* sigma2 = nullptr;
  const int* g_rp = nullptr;
  const int* g_ci = nullptr;
  const __half* g_va = nullptr;
  const int* gt_rp = nullptr;
  const int* gt_ci = nullptr;
  const __half* gt_va = nullptr;
};

// ---- deterministic reductions -------------------------------------------------------

template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV]) {
  __shared__ double sh[NV][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_down_sync(0xffffffffu, v[i], o);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int i = 0; i < NV; ++i) sh[i][wid] = v[i];
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      double t = lane < nw ? sh[i][lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
      v[i] = t;
    }
  }
}

// Per-block partials, then a fixed-order sum by the last block to arrive.
// Returns true in thread 0 of the last block, with the totals in v.
template <int NV>
__device__ __forceinline__ bool grid_sum(double (&v)[NV], double* partials, unsigned* ticket) {
  block_sum<NV>(v);
  __shared__ bool last;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) partials[i * gridDim.x + blockIdx.x] = v[i];
    __threadfence();
    unsigned t = atomicAdd(ticket, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double acc[NV];
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    acc[i] = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) acc[i] += __ldcg(partials + i * gridDim.x + b);
  }
  block_sum<NV>(acc);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) v[i] = acc[i];
    *ticket = 0;
  }
  return threadIdx.x == 0;
}

// ---- SpMV ------------------------------------------------------------------------

template <typename TA, typename TV>
__device__ __forceinline__ TA to_acc(TV v) {
  return (TA)v;
}
template <>
__device__ __forceinline__ double to_acc<double, __half>(__half v) {
  return (double)__half2float(v);
}
template <>
__device__ __forceinline__ float to_acc<float, __half>(__half v) {
  return __half2float(v);
}

// Row sum with LANES threads per row; every lane of a warp runs the same number
// of trips, so the segment shuffles are always converged.
template <typename TV, typename TX, typename TA, int LANES>
__device__ __forceinline__ TA row_dot(const int* __restrict__ rp, const int* __restrict__ ci,
                                      const TV* __restrict__ va, const TX* __restrict__ x, int row, bool valid) {
  TA s = TA(0);
  if (valid) {
    const int b = rp[row], e = rp[row + 1];
    for (int k = b + (threadIdx.x & (LANES - 1)); k < e; k += LANES) s += to_acc<TA>(va[k]) * (TA)__ldg(x + ci[k]);
  }
#pragma unroll
  for (int o = LANES / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, LANES);
  return s;
}

// y = A x (accumulated in TY); DOT: also pq = x.y into st->pq (breakdown if <= 0).
template <typename TV, typename TX, typename TY, int LANES, bool DOT>
__global__ void __launch_bounds__(SPMV_THREADS) spmv_kernel(int n, const int* __restrict__ rp,
                                                            const int* __restrict__ ci, const TV* __restrict__ va,
                                                            const TX* __restrict__ x, TY* __restrict__ y,
                                                            PcgState* st, double* partials, bool skip_done) {
  if (skip_done && st->done) return;
  constexpr int RPW = 32 / LANES;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int sub = (threadIdx.x & 31) / LANES;
  const bool head = (threadIdx.x & (LANES - 1)) == 0;
  double d[1] = {0.0};
  for (int base = warp * RPW; base < n; base += nwarps * RPW) {
    const int row = base + sub;
    const bool valid = row < n;
    TY s = row_dot<TV, TX, TY, LANES>(rp, ci, va, x, row, valid);
    if (valid && head) {
      y[row] = s;
      if (DOT) d[0] += (double)x[row] * (double)s;
    }
  }
  if (DOT) {
    if (grid_sum<1>(d, partials, &st->ticket[0])) {
      st->pq = d[0];
      if (!(d[0] > 0.0)) st->done = 2;  // p.Ap <= 0 or NaN
    }
  }
}

// FSAI first half: t = sigma^2 * (r + L r).  Skipped once done.
template <typename T, int LANES>
__global__ void __launch_bounds__(SPMV_THREADS) fsai_lower(int n, const int* __restrict__ rp,
                                                           const int* __restrict__ ci, const __half* __restrict__ va,
                                                           const float* __restrict__ sigma2,
                                                           const T* __restrict__ r, T* __restrict__ t,
                                                           const PcgState* st) {
  if (st->done) return;
  constexpr int RPW = 32 / LANES;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int sub = (threadIdx.x & 31) / LANES;
  const bool head = (threadIdx.x & (LANES - 1)) == 0;
  for (int base = warp * RPW; base < n; base += nwarps * RPW) {
    const int row = base + sub;
    const bool valid = row < n;
    T s = row_dot<__half, T, T, LANES>(rp, ci, va, r, row, valid);
    if (valid && head) t[row] = (T)sigma2[row] * (r[row] + s);
  }
}

// FSAI second half: z = t + L^T t and rz = r.z into st->rz[par ^ 1].
template <typename T, int LANES>
__global__ void __launch_bounds__(SPMV_THREADS) fsai_upper_rz(int n, const int* __restrict__ rp,
                                                              const int* __restrict__ ci,
                                                              const __half* __restrict__ va,
                                                              const T* __restrict__ t, const T* __restrict__ r,
                                                              T* __restrict__ z, PcgState* st, double* partials,
                                                              int par) {
  if (st->done) return;
  constexpr int RPW = 32 / LANES;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int sub = (threadIdx.x & 31) / LANES;
  const bool head = (threadIdx.x & (LANES - 1)) == 0;
  double d[1] = {0.0};
  for (int base = warp * RPW; base < n; base += nwarps * RPW) {
    const int row = base + sub;
    const bool valid = row < n;
    T s = row_dot<__half, T, T, LANES>(rp, ci, va, t, row, valid);
    if (valid && head) {
      const T zi = t[row] + s;
      z[row] = zi;
      d[0] += (double)r[row] * (double)zi;
    }
  }
  if (grid_sum<1>(d, partials, &st->ticket[3])) {
    st->rz[par ^ 1] = d[0];
    if (!(d[0] > 0.0)) st->done = 2;  // preconditioner not SPD
  }
}

// ---- PCG vector kernels ------------------------------------------------------------

template <typename T>
struct Pair;
template <>
struct Pair<double> { using type = double2; };
template <>
struct Pair<float> { using type = float2; };

// K2: alpha = rz/pq; xl += alpha p; r -= alpha q; rr (and, Jacobi, rz' = r.D^-1 r).
// Two elements per thread and step (8- or 16-byte loads; vectors are whole
// stream-ordered allocations, so 16-byte aligned).
template <typename T, bool JACOBI>
__global__ void __launch_bounds__(VEC_THREADS) pcg_update(int n, int par, T* __restrict__ xl, T* __restrict__ r,
                                                          const T* __restrict__ p, const T* __restrict__ q,
                                                          const T* __restrict__ dinv, PcgState* st,
                                                          double* partials) {
  if (st->done) return;
  using V = typename Pair<T>::type;
  const double rz = st->rz[par];
  const T a = (T)(rz / st->pq);
  double v[2] = {0.0, 0.0};
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  for (int i = tid; i < (n >> 1); i += stride) {
    V xv = reinterpret_cast<V*>(xl)[i], rv = reinterpret_cast<V*>(r)[i];
    const V pv = reinterpret_cast<const V*>(p)[i], qv = reinterpret_cast<const V*>(q)[i];
    xv.x += a * pv.x;
    xv.y += a * pv.y;
    rv.x = rv.x - a * qv.x;
    rv.y = rv.y - a * qv.y;
    reinterpret_cast<V*>(xl)[i] = xv;
    reinterpret_cast<V*>(r)[i] = rv;
    if (JACOBI) {
      const V dv = reinterpret_cast<const V*>(dinv)[i];
      v[0] += (double)rv.x * (double)(dv.x * rv.x) + (double)rv.y * (double)(dv.y * rv.y);
    }
    v[1] += (double)rv.x * (double)rv.x + (double)rv.y * (double)rv.y;
  }
  if ((n & 1) && tid == 0) {
    const int i = n - 1;
    xl[i] += a * p[i];
    const T ri = r[i] - a * q[i];
    r[i] = ri;
    if (JACOBI) v[0] += (double)ri * (double)(dinv[i] * ri);
    v[1] += (double)ri * (double)ri;
  }
  if (grid_sum<2>(v, partials, &st->ticket[1])) {
    if (JACOBI) st->rz[par ^ 1] = v[0];
    st->rz_old = rz;
    st->rr = v[1];
    st->iters += 1;
    if (!(v[1] == v[1]) || !(v[0] == v[0])) st->done = 2;
    else if (v[1] <= st->upd2) st->done = 4;
    else if (st->iters >= st->max_iters) st->done = 3;
  }
}

// K3: p = z + beta p, z = D^-1 r (Jacobi) or the FSAI output.
template <typename T, bool JACOBI>
__global__ void __launch_bounds__(VEC_THREADS) pcg_direction(int n, int par, const T* __restrict__ r,
                                                             T* __restrict__ p, const T* __restrict__ dinv,
                                                             const T* __restrict__ z, const PcgState* st) {
  if (st->done) return;
  using V = typename Pair<T>::type;
  const T beta = (T)(st->rz[par ^ 1] / st->rz[par]);
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  for (int i = tid; i < (n >> 1); i += stride) {
    V pv = reinterpret_cast<V*>(p)[i], zv;
    if (JACOBI) {
      const V dv = reinterpret_cast<const V*>(dinv)[i], rv = reinterpret_cast<const V*>(r)[i];
      zv.x = dv.x * rv.x;
      zv.y = dv.y * rv.y;
    } else {
      zv = reinterpret_cast<const V*>(z)[i];
    }
    pv.x = zv.x + beta * pv.x;
    pv.y = zv.y + beta * pv.y;
    reinterpret_cast<V*>(p)[i] = pv;
  }
  if ((n & 1) && tid == 0) p[n - 1] = (JACOBI ? dinv[n - 1] * r[n - 1] : z[n - 1]) + beta * p[n - 1];
}

__global__ void init_state(PcgState* st, int max_iters) {
  st->rz[0] = st->rz[1] = 0.0;
  st->rz_old = INFINITY;
  st->pq = 0.0;
  st->rr = 0.0;
  st->upd2 = 0.0;
  st->done = 0;
  st->iters = 0;
  st->max_iters = max_iters;
}

// Reliable update, part 1: r = (T) r_hi, xl = 0, rr (and Jacobi rz -> rz[0]); done = 0.
template <typename T>
__global__ void __launch_bounds__(VEC_THREADS) reset_residual(int n, const double* __restrict__ r_hi,
                                                              T* __restrict__ r, T* __restrict__ xl,
                                                              const T* __restrict__ dinv, PcgState* st,
                                                              double* partials, double upd2) {
  double v[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    T ri = (T)r_hi[i];
    r[i] = ri;
    xl[i] = T(0);
    if (dinv) v[0] += (double)ri * (double)(dinv[i] * ri);
    v[1] += (double)ri * (double)ri;
  }
  if (grid_sum<2>(v, partials, &st->ticket[2])) {
    if (dinv) st->rz[0] = v[0];
    st->rr = v[1];
    st->upd2 = upd2;
    st->done = 0;
  }
}

// Reliable update, part 2: p = z + (rz[0] / rz_old) p (beta = 0 on the first call).
template <typename T>
__global__ void __launch_bounds__(VEC_THREADS) reset_direction(int n, const T* __restrict__ r, T* __restrict__ p,
                                                               const T* __restrict__ dinv, const T* __restrict__ z,
                                                               const PcgState* st) {
  const T beta = (T)(st->rz[0] / st->rz_old);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = (dinv ? dinv[i] * r[i] : z[i]) + beta * p[i];
}

template <typename T>
__global__ void accumulate(int n, const T* __restrict__ xl, double* __restrict__ x) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] += (double)xl[i];
}

// dinv = 1 / diag(A); flags rows whose diagonal is missing or not positive.
template <typename T>
__global__ void jacobi_diag(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                            const double* __restrict__ va, T* __restrict__ dinv, int* flag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double d = 0.0;
  for (int k = rp[i]; k < rp[i + 1]; ++k)
    if (ci[k] == i) d = va[k];
  if (!(d > 0.0)) atomicOr(flag, 1);
  dinv[i] = (T)(1.0 / d);
}

// FP64 true residual r = b - A x, computed with compensated (double-double)
// accumulation so r is the residual of the FP64 vector x rounded once, not a
// sum whose cancellation noise (eps * || |A||x| ||) can exceed the target;
// and ||r||^2 into *out2 via the ticket.
template <int LANES>
__global__ void __launch_bounds__(SPMV_THREADS) residual_f64(int n, const int* __restrict__ rp,
                                                             const int* __restrict__ ci,
                                                             const double* __restrict__ va,
                                                             const double* __restrict__ x,
                                                             const double* __restrict__ b, double* __restrict__ r,
                                                             double* out2, unsigned* ticket, double* partials) {
  constexpr int RPW = 32 / LANES;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int sub = (threadIdx.x & 31) / LANES;
  const int lane = threadIdx.x & (LANES - 1);
  double d[1] = {0.0};
  for (int base = warp * RPW; base < n; base += nwarps * RPW) {
    const int row = base + sub;
    const bool valid = row < n;
    double hi = 0.0, lo = 0.0;
    if (valid) {
      const int kb = rp[row], ke = rp[row + 1];
      for (int k = kb + lane; k < ke; k += LANES) {
        double p, pe, s, se;
        two_prod(va[k], __ldg(x + ci[k]), p, pe);
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
      r[row] = ri;
      d[0] += ri * ri;
    }
  }
  if (grid_sum<1>(d, partials, ticket)) *out2 = d[0];
}

__global__ void to_f32(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}

__global__ void sumsq_kernel(int n, const double* __restrict__ b, double* out, unsigned* ticket, double* partials) {
  double v[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[0] += b[i] * b[i];
  if (grid_sum<1>(v, partials, ticket)) *out = v[0];
}

// z = G^T G r with rz = r.z into st->rz[par ^ 1].  Skipped once done.
template <typename T>
void fsai_apply(const Precond<T>& pc, int n, const T* r, T* t, T* z, PcgState* st, double* partials, int par,
                cudaStream_t s) {
#define TPT_FSAI_CASE(L)                                                                                       \
  case L:                                                                                                      \
    fsai_lower<T, L><<<pc.grid, SPMV_THREADS, 0, s>>>(n, pc.g_rp, pc.g_ci, pc.g_va, pc.sigma2, r, t, st);      \
    TPT_CHECK_LAUNCH();                                                                                        \
    fsai_upper_rz<T, L><<<pc.grid, SPMV_THREADS, 0, s>>>(n, pc.gt_rp, pc.gt_ci, pc.gt_va, t, r, z, st,         \
                                                         partials, par);                                       \
    TPT_CHECK_LAUNCH();                                                                                        \
    break;
  switch (pc.lanes) {
    TPT_FSAI_CASE(2)
    TPT_FSAI_CASE(4)
    TPT_FSAI_CASE(8)
    default: TPT_FSAI_CASE(16)
  }
#undef TPT_FSAI_CASE
}

}  // namespace tptfem
