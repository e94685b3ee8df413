// modes.cuh -- rigid-body modes of a mesh node for the aggregation coarse
// space (coarse.cu) and its prolongation (fused into nbsell.cuh's FSAI kernel).
#pragma once

namespace tptfem {

// Modes per node group: DPN 3: 3 translations + 3 rotations; DPN 2: 2 + 1; DPN 1: 1.
__host__ __device__ constexpr int rigid_modes(int dpn) { return dpn == 1 ? 1 : (dpn == 2 ? 3 : 6); }

// R[a][k]: component a of raw mode k at position y (relative to the
// aggregate's centroid).  DPN 3: translations x, y, z, then rotations e_k x y;
// DPN 2: x, y, rotation about z; DPN 1: the constant.
template <int DPN>
__device__ __forceinline__ void mode_rows(const float* __restrict__ y3, double (&R)[DPN][rigid_modes(DPN)]) {
  if constexpr (DPN == 1) {
    R[0][0] = 1.0;
  } else if constexpr (DPN == 2) {
    const double y0 = y3[0], y1 = y3[1];
    R[0][0] = 1.0; R[0][1] = 0.0; R[0][2] = -y1;
    R[1][0] = 0.0; R[1][1] = 1.0; R[1][2] = y0;
  } else {
    const double y0 = y3[0], y1 = y3[1], y2 = y3[2];
    R[0][0] = 1.0; R[0][1] = 0.0; R[0][2] = 0.0; R[0][3] = 0.0; R[0][4] = y2;  R[0][5] = -y1;
    R[1][0] = 0.0; R[1][1] = 1.0; R[1][2] = 0.0; R[1][3] = -y2; R[1][4] = 0.0; R[1][5] = y0;
    R[2][0] = 0.0; R[2][1] = 0.0; R[2][2] = 1.0; R[2][3] = y1;  R[2][4] = -y0; R[2][5] = 0.0;
  }
}

// Coarse prolongation arguments for the FSAI transpose kernel (null: off).
struct CoarseArgs {
  const int* agg = nullptr;    // per group: aggregate
  const float* y = nullptr;    // per group: relative position (3 floats)
  const double* cm = nullptr;  // per aggregate: raw-mode coefficients T uc (nm values)
};

}  // namespace tptfem
