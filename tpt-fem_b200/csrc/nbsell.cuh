// nbsell.cuh -- NB-SELL apply kernels (see nbsell.cu for the layout).
// One warp per chunk of 32 node groups, one thread per group; each thread
// accumulates its DPN rows in registers.  Included by solver.cu.
#pragma once
#include <cuda_fp16.h>

#include "modes.cuh"
#include "solver_kernels.cuh"

namespace tptfem {

// y = K x (FP64 blocks); DOT: pq = x.y into st->pq (breakdown if <= 0).
template <int DPN, bool DOT>
__global__ void __launch_bounds__(SPMV_THREADS) nb_spmv(int ngroups, const int* __restrict__ cptr,
                                                        const int* __restrict__ bcol,
                                                        const double* __restrict__ bval,
                                                        const double* __restrict__ x, double* __restrict__ y,
                                                        PcgState* st, double* partials, bool skip_done) {
  if (skip_done && st->done) return;
  constexpr int D2 = DPN * DPN;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const int nchunks = (ngroups + 31) >> 5;
  double d[1] = {0.0};
  for (int c = warp; c < nchunks; c += nw) {
    const int g = c * 32 + lane;
    if (g < ngroups) {
      double acc[DPN];
#pragma unroll
      for (int a = 0; a < DPN; ++a) acc[a] = 0.0;
      const int s1 = cptr[c + 1];
      for (int s = cptr[c]; s < s1; ++s) {
        const int J = bcol[(int64_t)s * 32 + lane];
        double xj[DPN];
#pragma unroll
        for (int b = 0; b < DPN; ++b) xj[b] = __ldg(x + (int64_t)J * DPN + b);
        const double* v = bval + (int64_t)s * D2 * 32 + lane;
#pragma unroll
        for (int a = 0; a < DPN; ++a)
#pragma unroll
          for (int b = 0; b < DPN; ++b) acc[a] += v[(a * DPN + b) * 32] * xj[b];
      }
#pragma unroll
      for (int a = 0; a < DPN; ++a) {
        y[(int64_t)g * DPN + a] = acc[a];
        if (DOT) d[0] += x[(int64_t)g * DPN + a] * acc[a];
      }
    }
  }
  if (DOT) {
    if (grid_sum<1>(d, partials, &st->ticket[0])) {
      st->pq = d[0];
      if (!(d[0] > 0.0)) st->done = 2;
    }
  }
}

// y = K x from the symmetric half storage (nb_build_sym): diagonal block,
// strictly-lower blocks, and the transposes of the lower blocks of the upper
// neighbours, read where their rows store them.  Step k handles lower slot k
// and upper slot nu-1-k (upper columns descending): block (J, g) is then read
// by row g in the same step in which row J reads it as its own lower block
// (J's lower list is ascending), so the two reads of a block by concurrently
// running warps are close in time and the second one is an L2 hit.
// K is symmetric up to FP64 rounding of the element matrices; this operator
// uses its lower half for both halves.
// At most 40 registers (6 resident blocks per SM): the kernel is latency-bound,
// more warps in flight beat more registers per warp (0.222 -> 0.189 ms at 4.2M dofs).
template <int DPN, bool DOT>
__global__ void __launch_bounds__(SPMV_THREADS, 6) nb_spmv_sym(int ngroups, const int* __restrict__ lcptr,
                                                            const int* __restrict__ lcol,
                                                            const double* __restrict__ lval,
                                                            const double* __restrict__ dval,
                                                            const int* __restrict__ ucptr,
                                                            const int* __restrict__ ucol,
                                                            const int* __restrict__ ubase,
                                                            const double* __restrict__ x, double* __restrict__ y,
                                                            PcgState* st, double* partials, bool skip_done) {
  if (skip_done && st->done) return;
  constexpr int D2 = DPN * DPN;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const int nchunks = (ngroups + 31) >> 5;
  double d[1] = {0.0};
  for (int c = warp; c < nchunks; c += nw) {
    const int g = c * 32 + lane;
    if (g < ngroups) {
      double xg[DPN], acc[DPN];
#pragma unroll
      for (int b = 0; b < DPN; ++b) xg[b] = x[(int64_t)g * DPN + b];
#pragma unroll
      for (int a = 0; a < DPN; ++a) {
        double s = 0.0;
#pragma unroll
        for (int b = 0; b < DPN; ++b) s += dval[((int64_t)c * D2 + a * DPN + b) * 32 + lane] * xg[b];
        acc[a] = s;
      }
      // lower slot k and upper slot (nu - 1 - k) in the same step
      const int l0 = lcptr[c], nl = lcptr[c + 1] - l0;
      const int u0 = ucptr[c], nu = ucptr[c + 1] - u0;
      const int steps = nl > nu ? nl : nu;
      for (int k = 0; k < steps; ++k) {
        if (k < nu) {
          const int64_t idx = (int64_t)(u0 + nu - 1 - k) * 32 + lane;
          const int base = ubase[idx];
          if (base >= 0) {
            const int J = ucol[idx];
            double xj[DPN];
#pragma unroll
            for (int b = 0; b < DPN; ++b) xj[b] = __ldg(x + (int64_t)J * DPN + b);
            const double* v = lval + base;
#pragma unroll
            for (int a = 0; a < DPN; ++a)
#pragma unroll
              for (int b = 0; b < DPN; ++b) acc[a] += __ldg(v + (b * DPN + a) * 32) * xj[b];
          }
        }
        if (k < nl) {
          const int64_t s = l0 + k;
          const int J = lcol[s * 32 + lane];
          double xj[DPN];
#pragma unroll
          for (int b = 0; b < DPN; ++b) xj[b] = __ldg(x + (int64_t)J * DPN + b);
          const double* v = lval + s * D2 * 32 + lane;
#pragma unroll
          for (int a = 0; a < DPN; ++a)
#pragma unroll
            for (int b = 0; b < DPN; ++b) acc[a] += v[(a * DPN + b) * 32] * xj[b];
        }
      }
#pragma unroll
      for (int a = 0; a < DPN; ++a) {
        y[(int64_t)g * DPN + a] = acc[a];
        if (DOT) d[0] += xg[a] * acc[a];
      }
    }
  }
  if (DOT) {
    if (grid_sum<1>(d, partials, &st->ticket[0])) {
      st->pq = d[0];
      if (!(d[0] > 0.0)) st->done = 2;
    }
  }
}

// Y = K X for NV interleaved vectors (X[(row) * NV + v]) from the symmetric
// half storage: each block is read once for all vectors.  Used to form
// coarse-space products P^T A P (set-up only, not on the iteration path):
// with gcol set, the rows of groups whose colour differs from `colour` count
// as zero, so X can hold P for every colour at once; such blocks are not read.
// With cmask set, chunks whose bit `colour` is clear (no group in them has a
// neighbour of that colour) are skipped and their rows of Y left unwritten.
template <int DPN, int NV>
__global__ void __launch_bounds__(SPMV_THREADS) nb_spmv_sym_multi(int ngroups, const int* __restrict__ lcptr,
                                                                  const int* __restrict__ lcol,
                                                                  const double* __restrict__ lval,
                                                                  const double* __restrict__ dval,
                                                                  const int* __restrict__ ucptr,
                                                                  const int* __restrict__ ucol,
                                                                  const int* __restrict__ ubase,
                                                                  const double* __restrict__ X,
                                                                  double* __restrict__ Y,
                                                                  const unsigned char* __restrict__ gcol,
                                                                  int colour,
                                                                  const unsigned* __restrict__ cmask) {
  constexpr int D2 = DPN * DPN;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const int nchunks = (ngroups + 31) >> 5;
  for (int c = warp; c < nchunks; c += nw) {
    if (cmask && !((cmask[c] >> colour) & 1u)) continue;  // uniform over the warp
    const int g = c * 32 + lane;
    if (g >= ngroups) continue;
    double acc[DPN][NV];
#pragma unroll
    for (int a = 0; a < DPN; ++a)
#pragma unroll
      for (int v = 0; v < NV; ++v) acc[a][v] = 0.0;
    auto wanted = [&](int J) { return !gcol || __ldg(gcol + J) == colour; };
    auto add = [&](const double (&blk)[D2], int J, bool transposed) {
#pragma unroll
      for (int b = 0; b < DPN; ++b)
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const double xv = __ldg(X + ((int64_t)J * DPN + b) * NV + v);
#pragma unroll
          for (int a = 0; a < DPN; ++a) acc[a][v] += (transposed ? blk[b * DPN + a] : blk[a * DPN + b]) * xv;
        }
    };
    if (wanted(g)) {
      double blk[D2];
#pragma unroll
      for (int q = 0; q < D2; ++q) blk[q] = dval[((int64_t)c * D2 + q) * 32 + lane];
      add(blk, g, false);
    }
    for (int s = lcptr[c]; s < lcptr[c + 1]; ++s) {
      const int J = lcol[(int64_t)s * 32 + lane];
      if (!wanted(J)) continue;
      double blk[D2];
#pragma unroll
      for (int q = 0; q < D2; ++q) blk[q] = lval[((int64_t)s * D2 + q) * 32 + lane];
      add(blk, J, false);
    }
    for (int s = ucptr[c]; s < ucptr[c + 1]; ++s) {
      const int64_t idx = (int64_t)s * 32 + lane;
      const int base = ubase[idx];
      if (base < 0) continue;
      const int J = ucol[idx];
      if (!wanted(J)) continue;
      double blk[D2];
#pragma unroll
      for (int q = 0; q < D2; ++q) blk[q] = __ldg(lval + base + q * 32);
      add(blk, J, true);
    }
#pragma unroll
    for (int a = 0; a < DPN; ++a)
#pragma unroll
      for (int v = 0; v < NV; ++v) Y[((int64_t)g * DPN + a) * NV + v] = acc[a][v];
  }
}

// One FP16 block of a factor slot: 8 values in a 16-byte word (row-major
// entries 0..7) plus the 9th entry (3x3) in a separate 2-byte array, so a lane
// issues two loads per block.  For DPN = 2 the word holds all 4 entries; for
// DPN = 1 the single value is stored in the 2-byte array only.
template <int DPN>
__device__ __forceinline__ void load_half_block(const uint4* __restrict__ pack, const __half* __restrict__ tail,
                                                int64_t idx, float (&v)[DPN * DPN]) {
  if constexpr (DPN == 1) {  // one value: it lives in the 2-byte array alone
    v[0] = __half2float(__ldg(tail + idx));
  } else {
    const uint4 w = __ldg(pack + idx);
    const __half2* h = reinterpret_cast<const __half2*>(&w);
    float f[8];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float2 p = __half22float2(h[i]);
      f[2 * i] = p.x;
      f[2 * i + 1] = p.y;
    }
#pragma unroll
    for (int q = 0; q < DPN * DPN && q < 8; ++q) v[q] = f[q];
    if constexpr (DPN * DPN == 9) v[8] = __half2float(tail[idx]);
  }
}

// t = sigma^2 * (r + L r), L in packed FP16 blocks.  Skipped once done.
template <int DPN>
__global__ void __launch_bounds__(SPMV_THREADS) nb_fsai_lower(int ngroups, const int* __restrict__ cptr,
                                                              const int* __restrict__ bcol,
                                                              const uint4* __restrict__ pack,
                                                              const __half* __restrict__ tail,
                                                              const __half* __restrict__ dval,
                                                              const float* __restrict__ sigma2,
                                                              const double* __restrict__ r, double* __restrict__ t,
                                                              const PcgState* st) {
  if (st->done) return;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const int nchunks = (ngroups + 31) >> 5;
  for (int c = warp; c < nchunks; c += nw) {
    const int g = c * 32 + lane;
    if (g >= ngroups) continue;
    double own[DPN], acc[DPN];
#pragma unroll
    for (int a = 0; a < DPN; ++a) acc[a] = own[a] = r[(int64_t)g * DPN + a];
    int q = 0;
#pragma unroll
    for (int a = 1; a < DPN; ++a)
#pragma unroll
      for (int b = 0; b < a; ++b, ++q)
        acc[a] += (double)__half2float(dval[((int64_t)c * 3 + q) * 32 + lane]) * own[b];
    const int s1 = cptr[c + 1];
#pragma unroll 2
    for (int s = cptr[c]; s < s1; ++s) {
      const int64_t idx = (int64_t)s * 32 + lane;
      const int J = bcol[idx];
      double xj[DPN];
#pragma unroll
      for (int b = 0; b < DPN; ++b) xj[b] = __ldg(r + (int64_t)J * DPN + b);
      float v[DPN * DPN];
      load_half_block<DPN>(pack, tail, idx, v);
#pragma unroll
      for (int a = 0; a < DPN; ++a)
#pragma unroll
        for (int b = 0; b < DPN; ++b) acc[a] += (double)v[a * DPN + b] * xj[b];
    }
#pragma unroll
    for (int a = 0; a < DPN; ++a) t[(int64_t)g * DPN + a] = (double)sigma2[(int64_t)g * DPN + a] * acc[a];
  }
}

// z = t + L^T t (transposed packed FP16 blocks) [+ P uc, the coarse
// correction, when cs.agg is set] and rz = r.z into st->rz[par ^ 1].
template <int DPN>
__global__ void __launch_bounds__(SPMV_THREADS) nb_fsai_upper_rz(int ngroups, const int* __restrict__ cptr,
                                                                 const int* __restrict__ bcol,
                                                                 const uint4* __restrict__ pack,
                                                                 const __half* __restrict__ tail,
                                                                 const __half* __restrict__ dval,
                                                                 const double* __restrict__ t,
                                                                 const double* __restrict__ r,
                                                                 double* __restrict__ z, PcgState* st,
                                                                 double* partials, int par, CoarseArgs cs) {
  if (st->done) return;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const int nchunks = (ngroups + 31) >> 5;
  double d[1] = {0.0};
  for (int c = warp; c < nchunks; c += nw) {
    const int g = c * 32 + lane;
    if (g >= ngroups) continue;
    double own[DPN], acc[DPN];
#pragma unroll
    for (int a = 0; a < DPN; ++a) acc[a] = own[a] = t[(int64_t)g * DPN + a];
    int q = 0;
#pragma unroll
    for (int a = 1; a < DPN; ++a)
#pragma unroll
      for (int b = 0; b < a; ++b, ++q)
        acc[b] += (double)__half2float(dval[((int64_t)c * 3 + q) * 32 + lane]) * own[a];
    const int s1 = cptr[c + 1];
#pragma unroll 2
    for (int s = cptr[c]; s < s1; ++s) {
      const int64_t idx = (int64_t)s * 32 + lane;
      const int J = bcol[idx];
      double xj[DPN];
#pragma unroll
      for (int b = 0; b < DPN; ++b) xj[b] = __ldg(t + (int64_t)J * DPN + b);
      float v[DPN * DPN];
      load_half_block<DPN>(pack, tail, idx, v);
#pragma unroll
      for (int a = 0; a < DPN; ++a)
#pragma unroll
        for (int b = 0; b < DPN; ++b) acc[a] += (double)v[a * DPN + b] * xj[b];
    }
    if (cs.agg) {  // z_g += R_g cm_I, cm_I = T_I uc_I
      constexpr int NM = rigid_modes(DPN);
      const double* cI = cs.cm + (int64_t)cs.agg[g] * NM;
      double cm[NM];
#pragma unroll
      for (int k = 0; k < NM; ++k) cm[k] = __ldg(cI + k);
      double R[DPN][NM];
      mode_rows<DPN>(cs.y + 3 * (int64_t)g, R);
#pragma unroll
      for (int a = 0; a < DPN; ++a)
#pragma unroll
        for (int k = 0; k < NM; ++k) acc[a] += R[a][k] * cm[k];
    }
#pragma unroll
    for (int a = 0; a < DPN; ++a) {
      z[(int64_t)g * DPN + a] = acc[a];
      d[0] += r[(int64_t)g * DPN + a] * acc[a];
    }
  }
  if (grid_sum<1>(d, partials, &st->ticket[3])) {
    st->rz[par ^ 1] = d[0];
    if (!(d[0] > 0.0)) st->done = 2;
  }
}

}  // namespace tptfem
