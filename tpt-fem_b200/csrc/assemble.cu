// assemble.cu -- element stiffness/load kernels and the element->CSR scatter.
//
// Design: "row gather".  One thread owns one global row (node n, component a)
// and walks the elements incident to n in ascending element id.  For each it
// recomputes the element geometry and the element-matrix ROW belonging to
// (n, a), and adds every entry into a dense per-row accumulator over n's
// neighbour columns (shared memory).  Because one thread adds the
// contributions of an entry in element order starting from +0.0, the result
// is bit-identical to Coo::to_csr's sequential duplicate sum
// (crates/tpt-fem-sparse/src/lib.rs:144-163), with no atomics and no COO
// triplet array in HBM.  A slot enters the pattern iff at least one element
// contributed a value != 0.0, which is the reference's zero-skip
// (crates/tpt-fem-assembly/src/lib.rs:469-472).
//
// The element formulas reproduce the reference's FP64 operation order
// exactly; this file is compiled with -fmad=false so no multiply-add is
// contracted.  Products with a structural zero of B or D are omitted: they
// add a signed zero to a sum, which never changes a stored value.
//
// Reference functions restated here (crates/...):
//   tpt-fem-element/src/lib.rs     624-740  Map, mat_det, mat_inv, physical_grad
//   tpt-fem-thermal/src/lib.rs     132-196  poisson_element_matrix / source_vector
//   tpt-fem-elasticity/src/lib.rs  197-348  constitutive, b_matrix, element matrix, body vector
//   tpt-fem-assembly/src/lib.rs    394-420, 601-667  surface, apply_neumann_order
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "objects.hpp"

namespace tptfem {

namespace {

// ---- quadrature tables (host-computed with the reference's expressions) ----
struct QuadTab {
  int nq;
  double w[25];
  double ns[25][4];     // shape values per point and node
  double lg[25][4][2];  // Quad4 reference gradients per point and node
};
__constant__ QuadTab c_cell;

struct FaceTab {
  int nq;
  double w[4];
  double ns[4][3];
};
__constant__ FaceTab c_face;

// gauss_legendre (crates/tpt-fem-quadrature/src/lib.rs:118-162)
bool gauss_legendre(int order, double* p, double* w) {
  switch (order) {
    case 1: p[0] = 0.0; w[0] = 2.0; return true;
    case 2: p[0] = -1.0 / std::sqrt(3.0); p[1] = 1.0 / std::sqrt(3.0); w[0] = w[1] = 1.0; return true;
    case 3:
      p[0] = 0.0; p[1] = -std::sqrt(3.0 / 5.0); p[2] = std::sqrt(3.0 / 5.0);
      w[0] = 8.0 / 9.0; w[1] = 5.0 / 9.0; w[2] = 5.0 / 9.0;
      return true;
    case 4: {
      const double pp[4] = {-0.3399810435848563, 0.3399810435848563, -0.8611363115940526, 0.8611363115940526};
      const double ww[4] = {0.6521451548625461, 0.6521451548625461, 0.3478548451374539, 0.3478548451374539};
      for (int i = 0; i < 4; ++i) { p[i] = pp[i]; w[i] = ww[i]; }
      return true;
    }
    case 5: {
      const double pp[5] = {0.0, -0.5384693101056831, 0.5384693101056831, -0.9061798459386640, 0.9061798459386640};
      const double ww[5] = {0.5688888888888889, 0.4786286704993665, 0.4786286704993665, 0.2369268850561891,
                            0.2369268850561891};
      for (int i = 0; i < 5; ++i) { p[i] = pp[i]; w[i] = ww[i]; }
      return true;
    }
    default: return false;
  }
}

// cell_quad (crates/tpt-fem-thermal/src/lib.rs:29-92) for Tet4 / Tri3 / Quad4, plus
// the shape values and reference gradients at each point.
QuadTab make_cell_tab(int cell, int order) {
  QuadTab t{};
  if (cell == TPTFEM_CELL_TET4) {  // tetrahedron(Degree2), quadrature:282-289; order ignored
    const double a = 0.5854101966249685, b = 0.1381966011250105;
    const double pts[4][3] = {{a, b, b}, {b, a, b}, {b, b, a}, {b, b, b}};
    t.nq = 4;
    for (int q = 0; q < 4; ++q) {
      t.w[q] = 1.0 / 24.0;
      double x = pts[q][0], y = pts[q][1], z = pts[q][2];
      t.ns[q][0] = 1.0 - x - y - z;
      t.ns[q][1] = x; t.ns[q][2] = y; t.ns[q][3] = z;
    }
    return t;
  }
  if (cell == TPTFEM_CELL_TRI3) {  // triangle(Degree2), quadrature:223-234; order ignored
    const double pts[3][2] = {{2.0 / 3.0, 1.0 / 6.0}, {1.0 / 6.0, 2.0 / 3.0}, {1.0 / 6.0, 1.0 / 6.0}};
    t.nq = 3;
    for (int q = 0; q < 3; ++q) {
      t.w[q] = 1.0 / 6.0;
      double x = pts[q][0], y = pts[q][1];
      t.ns[q][0] = 1.0 - x - y;  // Tri3 shape (element:106-120)
      t.ns[q][1] = x; t.ns[q][2] = y;
    }
    return t;
  }
  double p[5], w[5];
  TPT_REQUIRE(gauss_legendre(order, p, w), TPTFEM_ERR_INVALID_ARG, "quad_order must be in 1..=5");
  const double s[4] = {-1.0, 1.0, 1.0, -1.0}, tt[4] = {-1.0, -1.0, 1.0, 1.0};
  int q = 0;
  for (int ia = 0; ia < order; ++ia)
    for (int ib = 0; ib < order; ++ib, ++q) {  // tensor_square: outer a, inner b (quadrature:180-191)
      double x = p[ia], y = p[ib];
      t.w[q] = w[ia] * w[ib];
      for (int i = 0; i < 4; ++i) {  // Quad4 shape/grad (element:135-153)
        t.ns[q][i] = 0.25 * (1.0 + s[i] * x) * (1.0 + tt[i] * y);
        t.lg[q][i][0] = 0.25 * s[i] * (1.0 + tt[i] * y);
        t.lg[q][i][1] = 0.25 * (1.0 + s[i] * x) * tt[i];
      }
    }
  t.nq = q;
  return t;
}

// face_quad (crates/tpt-fem-assembly/src/lib.rs:336-358) at FACE_QUAD_ORDER = 2.
FaceTab make_face_tab(int cell) {
  FaceTab f{};
  if (cell == TPTFEM_CELL_TET4) {  // triangle(Degree2) on Tri3 faces
    const double pts[3][2] = {{2.0 / 3.0, 1.0 / 6.0}, {1.0 / 6.0, 2.0 / 3.0}, {1.0 / 6.0, 1.0 / 6.0}};
    f.nq = 3;
    for (int q = 0; q < 3; ++q) {
      f.w[q] = 1.0 / 6.0;
      double x = pts[q][0], y = pts[q][1];
      f.ns[q][0] = 1.0 - x - y; f.ns[q][1] = x; f.ns[q][2] = y;
    }
  } else {  // gauss_legendre(2) on Line2 edges
    double p[2], w[2];
    gauss_legendre(2, p, w);
    f.nq = 2;
    for (int q = 0; q < 2; ++q) {
      f.w[q] = w[q];
      f.ns[q][0] = (1.0 - p[q]) / 2.0;
      f.ns[q][1] = (1.0 + p[q]) / 2.0;
    }
  }
  return f;
}

// ---- element geometry ---------------------------------------------------------

// Tet4: J[p][r] = X[r+1][p] - X[0][p] (what Map::from_nodes_and_grad's running
// sum gives for the constant Tet4 gradients), det/inverse by cofactors in the
// order of element:624-680, physical gradients as physical_grad's running sum.
struct TetGeom {
  double g[4][3];
  double adet;
};

__device__ __forceinline__ bool tet_geom(const double (&X)[4][3], TetGeom& G) {
  double m[9];
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int r = 0; r < 3; ++r) m[p * 3 + r] = X[r + 1][p] - X[0][p];
  double c0 = m[4] * m[8] - m[5] * m[7];
  double c1 = m[3] * m[8] - m[5] * m[6];
  double c2 = m[3] * m[7] - m[4] * m[6];
  double det = m[0] * c0 - m[1] * c1 + m[2] * c2;
  double inv = 1.0 / det;
  double iv[9];
  iv[0] = c0 * inv;
  iv[1] = (m[2] * m[7] - m[1] * m[8]) * inv;
  iv[2] = (m[1] * m[5] - m[2] * m[4]) * inv;
  iv[3] = (m[5] * m[6] - m[3] * m[8]) * inv;
  iv[4] = (m[0] * m[8] - m[2] * m[6]) * inv;
  iv[5] = (m[2] * m[3] - m[0] * m[5]) * inv;
  iv[6] = c2 * inv;
  iv[7] = (m[1] * m[6] - m[0] * m[7]) * inv;
  iv[8] = (m[0] * m[4] - m[1] * m[3]) * inv;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    G.g[0][i] = (-iv[i] - iv[3 + i]) - iv[6 + i];
    G.g[1][i] = iv[i];
    G.g[2][i] = iv[3 + i];
    G.g[3][i] = iv[6 + i];
  }
  G.adet = fabs(det);
  return isfinite(inv) && isfinite(det);
}

// Tri3: J[p][r] = X[r+1][p] - X[0][p] (the running sum of Map::from_nodes_and_grad
// for the constant Tri3 gradients), det and inverse by the 2 x 2 cofactors of
// element:624-680, physical gradients as physical_grad's running sum.
struct TriGeom {
  double g[3][2];
  double adet;
};

__device__ __forceinline__ bool tri_geom(const double (&X)[4][2], TriGeom& G) {
  double m[4];
#pragma unroll
  for (int p = 0; p < 2; ++p)
#pragma unroll
    for (int r = 0; r < 2; ++r) m[p * 2 + r] = X[r + 1][p] - X[0][p];
  double det = m[0] * m[3] - m[1] * m[2];
  double inv = 1.0 / det;
  double iv[4] = {m[3] * inv, -m[1] * inv, -m[2] * inv, m[0] * inv};
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    G.g[0][i] = -iv[i] - iv[2 + i];
    G.g[1][i] = iv[i];
    G.g[2][i] = iv[2 + i];
  }
  G.adet = fabs(det);
  return isfinite(inv) && isfinite(det);
}

// Quad4 at one quadrature point: J by the running sum over the 4 nodes.
struct QuadGeom {
  double g[4][2];
  double adet;
};

__device__ __forceinline__ bool quad_geom(const double (&X)[4][2], int q, QuadGeom& G) {
  double m[4];
#pragma unroll
  for (int p = 0; p < 2; ++p)
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      double s = X[0][p] * c_cell.lg[q][0][r];
      s = s + X[1][p] * c_cell.lg[q][1][r];
      s = s + X[2][p] * c_cell.lg[q][2][r];
      s = s + X[3][p] * c_cell.lg[q][3][r];
      m[p * 2 + r] = s;
    }
  double det = m[0] * m[3] - m[1] * m[2];
  double inv = 1.0 / det;
  double iv[4] = {m[3] * inv, -m[1] * inv, -m[2] * inv, m[0] * inv};
#pragma unroll
  for (int n = 0; n < 4; ++n)
#pragma unroll
    for (int i = 0; i < 2; ++i) G.g[n][i] = c_cell.lg[q][n][0] * iv[i] + c_cell.lg[q][n][1] * iv[2 + i];
  G.adet = fabs(det);
  return isfinite(inv) && isfinite(det);
}

// ---- element rows -------------------------------------------------------------

// Isotropic constitutive constants (elasticity:197-233) for one element.
struct Dmat {
  double d00, d01, dsh;  // diagonal normal, off-diagonal normal, shear
};

__device__ __forceinline__ Dmat make_d(int model, double e, double nu) {
  Dmat D;
  if (model == TPTFEM_MODEL_CONTINUUM_3D) {
    double c = e / ((1.0 + nu) * (1.0 - 2.0 * nu));
    D.d00 = (1.0 - nu) * c;
    D.d01 = c * nu;
    D.dsh = (1.0 - 2.0 * nu) / 2.0 * c;
  } else if (model == TPTFEM_MODEL_PLANE_STRESS) {
    double c = e / (1.0 - nu * nu);
    D.d00 = c;
    D.d01 = c * nu;
    D.dsh = c * (1.0 - nu) / 2.0;
  } else {  // plane strain
    double c = e / ((1.0 + nu) * (1.0 - 2.0 * nu));
    D.d00 = c * (1.0 - nu);
    D.d01 = c * nu;
    D.dsh = c * (1.0 - 2.0 * nu) / 2.0;
  }
  return D;
}

// sum_{s,t} (B_l[s][a] * D[s][t]) * B_j[t][b] over the structurally non-zero
// terms, in the reference's s-major, t-minor order (elasticity:292-306).
__device__ __forceinline__ double bdb3(const double* gl, const double* gj, int a, int b, const Dmat& D) {
  const double m = D.d00, cn = D.d01, d = D.dsh;
  switch (a * 3 + b) {
    case 0: return ((gl[0] * m) * gj[0] + (gl[1] * d) * gj[1]) + (gl[2] * d) * gj[2];
    case 1: return (gl[0] * cn) * gj[1] + (gl[1] * d) * gj[0];
    case 2: return (gl[0] * cn) * gj[2] + (gl[2] * d) * gj[0];
    case 3: return (gl[1] * cn) * gj[0] + (gl[0] * d) * gj[1];
    case 4: return ((gl[1] * m) * gj[1] + (gl[0] * d) * gj[0]) + (gl[2] * d) * gj[2];
    case 5: return (gl[1] * cn) * gj[2] + (gl[2] * d) * gj[1];
    case 6: return (gl[2] * cn) * gj[0] + (gl[0] * d) * gj[2];
    case 7: return (gl[2] * cn) * gj[1] + (gl[1] * d) * gj[2];
    default: return ((gl[2] * m) * gj[2] + (gl[1] * d) * gj[1]) + (gl[0] * d) * gj[0];
  }
}

__device__ __forceinline__ double bdb2(const double* gl, const double* gj, int a, int b, const Dmat& D) {
  switch (a * 2 + b) {
    case 0: return (gl[0] * D.d00) * gj[0] + (gl[1] * D.dsh) * gj[1];
    case 1: return (gl[0] * D.d01) * gj[1] + (gl[1] * D.dsh) * gj[0];
    case 2: return (gl[1] * D.d01) * gj[0] + (gl[0] * D.dsh) * gj[1];
    default: return (gl[1] * D.d00) * gj[1] + (gl[0] * D.dsh) * gj[0];
  }
}

struct ElemIn {
  const double* coords;
  int cdim;
  const int* conn;
  const double* coef;
  int per_elem;
  int model;
  double nu;
};

// SD: spatial dimension; NV: nodes per element (arrays below hold 4 slots,
// a Tri3 element uses the first 3).
template <int CELL>
struct CellTraits;
template <>
struct CellTraits<TPTFEM_CELL_TET4> {
  static constexpr int SD = 3, NV = 4;
};
template <>
struct CellTraits<TPTFEM_CELL_QUAD4> {
  static constexpr int SD = 2, NV = 4;
};
template <>
struct CellTraits<TPTFEM_CELL_TRI3> {
  static constexpr int SD = 2, NV = 3;
};

template <int CELL>
__device__ __forceinline__ void load_elem(const ElemIn& in, int e, double (&X)[4][CellTraits<CELL>::SD],
                                          int (&nodes)[4]) {
  constexpr int NV = CellTraits<CELL>::NV;
  if constexpr (NV == 4) {
    int4 c = reinterpret_cast<const int4*>(in.conn)[e];
    nodes[0] = c.x; nodes[1] = c.y; nodes[2] = c.z; nodes[3] = c.w;
  } else {
#pragma unroll
    for (int j = 0; j < NV; ++j) nodes[j] = __ldg(in.conn + (int64_t)e * NV + j);
#pragma unroll
    for (int j = NV; j < 4; ++j) nodes[j] = nodes[0];
  }
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int p = 0; p < CellTraits<CELL>::SD; ++p) X[j][p] = __ldg(in.coords + (int64_t)nodes[j] * in.cdim + p);
}

// ---- boundary faces -------------------------------------------------------------

template <int CELL>
struct FaceTraits;
template <>
struct FaceTraits<TPTFEM_CELL_TET4> {
  static constexpr int NF = 4, FN = 3;
  __device__ static int node(int f, int q) {
    const int t[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
    return t[f][q];
  }
};
template <>
struct FaceTraits<TPTFEM_CELL_QUAD4> {
  static constexpr int NF = 4, FN = 2;
  __device__ static int node(int f, int q) {
    const int t[4][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}};
    return t[f][q];
  }
};
template <>
struct FaceTraits<TPTFEM_CELL_TRI3> {
  static constexpr int NF = 3, FN = 2;
  __device__ static int node(int f, int q) {
    const int t[3][2] = {{1, 2}, {2, 0}, {0, 1}};
    return t[f][q];
  }
};

// Measure and outward unit normal of face fl of an element, as
// apply_neumann_order / apply_robin_order compute them (assembly:394-420,
// 617-653): tangents from the face's reference gradients, the normal turned
// to point from the element centroid to the face centroid.
template <int CELL, int SD>
__device__ __forceinline__ void face_geometry(const double (&X)[4][SD], const int (&fl)[3], double& measure,
                                              double (&nrm)[SD]) {
  constexpr int FN = FaceTraits<CELL>::FN, NV = CellTraits<CELL>::NV;
  if constexpr (CELL == TPTFEM_CELL_TET4) {
    double t0[3], t1[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      t0[d] = X[fl[1]][d] - X[fl[0]][d];
      t1[d] = X[fl[2]][d] - X[fl[0]][d];
    }
    double c[3] = {t0[1] * t1[2] - t0[2] * t1[1], t0[2] * t1[0] - t0[0] * t1[2], t0[0] * t1[1] - t0[1] * t1[0]};
    measure = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    for (int d = 0; d < 3; ++d) nrm[d] = c[d] / measure;
  } else {
    double t[2];
#pragma unroll
    for (int d = 0; d < 2; ++d) t[d] = -0.5 * X[fl[0]][d] + 0.5 * X[fl[1]][d];
    measure = sqrt(t[0] * t[0] + t[1] * t[1]);
    double n0 = -t[1], n1 = t[0];
    double ln = sqrt(n0 * n0 + n1 * n1);
    nrm[0] = n0 / ln;
    nrm[1] = n1 / ln;
  }
  double ec[SD], fc[SD];
#pragma unroll
  for (int d = 0; d < SD; ++d) {
    double s = 0.0;
    for (int j = 0; j < NV; ++j) s = s + X[j][d];
    ec[d] = s / (double)NV;
    double f = 0.0;
    for (int q = 0; q < FN; ++q) f = f + X[fl[q]][d];
    fc[d] = f / (double)FN;
  }
  double dd = nrm[0] * (fc[0] - ec[0]);
  for (int d = 1; d < SD; ++d) dd = dd + nrm[d] * (fc[d] - ec[d]);
  if (dd < 0.0)
    for (int d = 0; d < SD; ++d) nrm[d] = -nrm[d];
}

// Row (l, a) of the element matrix: out[j*DPN + b] for the element's 4 nodes.
// PHYS 0: poisson_element_matrix with conductivity k; PHYS 1: elasticity.
template <int CELL, int PHYS, int DPN>
__device__ __forceinline__ bool element_row(const double (&X)[4][CellTraits<CELL>::SD], double coef, int model,
                                            double nu, int l, int a, double (&out)[4 * DPN]) {
  bool ok = true;
  if constexpr (CELL == TPTFEM_CELL_TET4) {
    TetGeom G;
    ok = tet_geom(X, G);
    const double w = c_cell.w[0];
    if constexpr (PHYS == 0) {
      const double wk = w * coef;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        double dot = G.g[l][0] * G.g[j][0] + G.g[l][1] * G.g[j][1] + G.g[l][2] * G.g[j][2];
        double t = wk * dot * G.adet;
        double v = t + t;  // four identical quadrature points, summed in order
        v = v + t;
        out[j] = v + t;
      }
    } else {
      Dmat D = make_d(model, coef, nu);
      const double wd = w * G.adet;
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          double t = wd * bdb3(G.g[l], G.g[j], a, b, D);
          double v = t + t;
          v = v + t;
          out[j * 3 + b] = v + t;
        }
    }
  } else if constexpr (CELL == TPTFEM_CELL_TRI3) {  // constant Jacobian, three equal-weight points
    TriGeom G;
    ok = tri_geom(X, G);
    const double w = c_cell.w[0];
    if constexpr (PHYS == 0) {
      const double wk = w * coef;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        double dot = G.g[l][0] * G.g[j][0] + G.g[l][1] * G.g[j][1];
        double t = wk * dot * G.adet;
        double v = t + t;  // three identical quadrature points, summed in order
        out[j] = v + t;
      }
    } else {
      Dmat D = make_d(model, coef, nu);
      const double wd = w * G.adet;
#pragma unroll
      for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
          double t = wd * bdb2(G.g[l], G.g[j], a, b, D);
          double v = t + t;
          out[j * 2 + b] = v + t;
        }
    }
  } else {  // Quad4: the Jacobian varies per point
#pragma unroll
    for (int i = 0; i < 4 * DPN; ++i) out[i] = 0.0;
    Dmat D;
    if constexpr (PHYS == 1) D = make_d(model, coef, nu);
    const int nq = c_cell.nq;
    for (int q = 0; q < nq; ++q) {
      QuadGeom G;
      ok &= quad_geom(X, q, G);
      const double w = c_cell.w[q];
      if constexpr (PHYS == 0) {
        const double wk = w * coef;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          double dot = G.g[l][0] * G.g[j][0] + G.g[l][1] * G.g[j][1];
          out[j] = out[j] + wk * dot * G.adet;
        }
      } else {
        const double wd = w * G.adet;
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
          for (int b = 0; b < 2; ++b) out[j * 2 + b] = out[j * 2 + b] + wd * bdb2(G.g[l], G.g[j], a, b, D);
      }
    }
  }
  return ok;
}

// COUNT: non-zeros per row; FILL: columns and values at row_ptr; NUMERIC: values
// into an existing pattern (checked); PADDED: columns and values of row r at
// r * maxc in a scratch array plus the count, compacted afterwards (one pass of
// element work instead of COUNT + FILL).
enum { MODE_COUNT = 0, MODE_FILL = 1, MODE_NUMERIC = 2, MODE_PADDED = 3 };

struct RowArgs {
  ElemIn in;
  const int* ne_ptr;
  const int* ne;
  const uchar4* slot;
  const int* nb_ptr;
  const int* nb;
  int64_t nrows;
  int* row_cnt;        // COUNT
  const int* row_ptr;  // FILL / NUMERIC
  int* col;            // FILL writes, NUMERIC checks
  double* val;
  int* flag;           // bit 0: bad element geometry, bit 1: pattern changed
  int maxc;            // accumulator slots per thread (max neighbours * DPN)
  // apply_robin term (robin != 0): h on the boundary faces selected by
  // (raxis, rsign), every boundary face when raxis < 0
  const unsigned char* bface;
  int robin, raxis;
  double rsign, rh;
  // per-point Robin coefficient (rpts != nullptr), indexed like TractionArgs::g
  const double* rpts;
  const int* face_off;
};

// One thread per global row.  Shared memory holds the row's dense accumulator
// (double) and non-zero flags (byte), slot-major so a warp touches consecutive
// words.
template <int CELL, int PHYS, int DPN, int MODE>
__global__ void __launch_bounds__(128) assemble_rows(RowArgs A) {
  extern __shared__ double sh[];
  const int T = blockDim.x;
  const int tid = threadIdx.x;
  const int64_t r = (int64_t)blockIdx.x * T + tid;
  if (r >= A.nrows) return;
  const int n = (int)(r / DPN), a = (int)(r % DPN);
  const int nb0 = A.nb_ptr[n];
  const int ncand = (A.nb_ptr[n + 1] - nb0) * DPN;
  double* acc = sh;
  unsigned char* nzf = reinterpret_cast<unsigned char*>(sh + (size_t)A.maxc * T);
  for (int s = 0; s < ncand; ++s) {
    acc[s * T + tid] = 0.0;
    nzf[s * T + tid] = 0;
  }
  bool ok = true;
  const int k1 = A.ne_ptr[n + 1];
  for (int k = A.ne_ptr[n]; k < k1; ++k) {
    const int pe = A.ne[k];
    const int e = pe >> 2, l = pe & 3;
    const uchar4 sl = A.slot[k];
    double X[4][CellTraits<CELL>::SD];
    int nodes[4];
    load_elem<CELL>(A.in, e, X, nodes);
    const double coef = A.in.coef[A.in.per_elem ? e : 0];
    double out[4 * DPN];
    ok &= element_row<CELL, PHYS, DPN>(X, coef, A.in.model, A.in.nu, l, a, out);
    const int sj[4] = {sl.x, sl.y, sl.z, sl.w};
#pragma unroll
    for (int j = 0; j < CellTraits<CELL>::NV; ++j)
#pragma unroll
      for (int b = 0; b < DPN; ++b) {
        const int s = (sj[j] * DPN + b) * T + tid;
        const double v = out[j * DPN + b];
        acc[s] = acc[s] + v;
        nzf[s] |= (unsigned char)(v != 0.0);
      }
  }
  if (A.robin) {
    // apply_robin_order (assembly:684-753): after every element contribution,
    // h N_k N_l w |face| for each selected boundary face holding this node, in
    // (element, face, quadrature point) order; every pair gets an entry.
    constexpr int SD = CellTraits<CELL>::SD, FN = FaceTraits<CELL>::FN, NF = FaceTraits<CELL>::NF;
    for (int k = A.ne_ptr[n]; k < k1; ++k) {
      const int pe = A.ne[k];
      const int e = pe >> 2, l = pe & 3;
      const unsigned bm = A.bface[e];
      if (!bm) continue;
      double X[4][SD];
      int nodes[4];
      load_elem<CELL>(A.in, e, X, nodes);
      const uchar4 sl = A.slot[k];
      const int sj[4] = {sl.x, sl.y, sl.z, sl.w};
      for (int fi = 0; fi < NF; ++fi) {
        if (!(bm & (1u << fi))) continue;
        int fl[3];
        int kpos = -1;
        for (int q = 0; q < FN; ++q) {
          fl[q] = FaceTraits<CELL>::node(fi, q);
          if (fl[q] == l) kpos = q;
        }
        if (kpos < 0) continue;
        double measure, nrm[SD];
        face_geometry<CELL, SD>(X, fl, measure, nrm);
        const double hsel = (A.raxis < 0 || nrm[A.raxis] * A.rsign > 0.5) ? A.rh : 0.0;
        const int64_t fp = A.rpts ? (int64_t)(A.face_off[e] + __popc(bm & ((1u << fi) - 1u))) * c_face.nq : 0;
        for (int q = 0; q < c_face.nq; ++q) {
          const double h = A.rpts ? A.rpts[fp + q] : hsel;
          const double wmh = c_face.w[q] * measure * h * c_face.ns[q][kpos];
          for (int lf = 0; lf < FN; ++lf) {
            const int s = (sj[fl[lf]] * DPN + a) * T + tid;
            acc[s] = acc[s] + wmh * c_face.ns[q][lf];
            nzf[s] = 1;
          }
        }
      }
    }
  }
  if (!ok) atomicOr(A.flag, 1);
  if (MODE == MODE_COUNT) {
    int c = 0;
    for (int s = 0; s < ncand; ++s) c += nzf[s * T + tid];
    A.row_cnt[r] = c;
  } else if (MODE == MODE_PADDED) {
    int c = 0;
    int* pc = A.col + r * A.maxc;
    double* pv = A.val + r * A.maxc;
    for (int s = 0; s < ncand; ++s) {
      if (!nzf[s * T + tid]) continue;
      pc[c] = A.nb[nb0 + s / DPN] * DPN + s % DPN;
      pv[c] = acc[s * T + tid];
      ++c;
    }
    A.row_cnt[r] = c;
  } else {
    int o = A.row_ptr[r];
    const int end = A.row_ptr[r + 1];
    bool same = true;
    for (int s = 0; s < ncand; ++s) {
      if (!nzf[s * T + tid]) continue;
      const int cidx = A.nb[nb0 + s / DPN] * DPN + s % DPN;
      if (MODE == MODE_FILL) {
        A.col[o] = cidx;
        A.val[o] = acc[s * T + tid];
      } else {
        if (o >= end || A.col[o] != cidx) { same = false; break; }
        A.val[o] = acc[s * T + tid];
      }
      ++o;
    }
    if (MODE == MODE_NUMERIC && (!same || o != end)) atomicOr(A.flag, 2);
  }
}

// Tet4 rows, one warp per node: the node's rows (n, 0..DPN-1) against its
// neighbour slots, lane k owning slot k (at most 32 neighbours) and holding
// the DPN x DPN accumulators of that column block in registers.  First each
// lane takes one incident element and computes the node's element-row blocks
// against the element's four nodes (shared memory, with each block's slot);
// then the lanes walk the elements in ascending id and the lane owning a
// block's slot adds it, so every entry is summed in element order from +0.0
// as in assemble_rows (and in Coo::to_csr's duplicate sum).  Same modes and
// outputs as assemble_rows.
constexpr int AN_WARPS = 4;     // warps per block
constexpr int AN_MAXDEG = 32;   // incident elements per node handled here (one per lane)

template <int PHYS, int DPN>
__global__ void __launch_bounds__(32 * AN_WARPS) assemble_nodes_tet(RowArgs A, int64_t n_nodes, int mode) {
  constexpr int D2 = DPN * DPN;
  __shared__ double blk[AN_WARPS][AN_MAXDEG][4][D2];
  __shared__ uchar4 bslot[AN_WARPS][AN_MAXDEG];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t n = (int64_t)blockIdx.x * AN_WARPS + w;
  if (n >= n_nodes) return;  // whole warps leave together
  const int k0 = A.ne_ptr[n], deg = A.ne_ptr[n + 1] - k0;
  bool ok = true;
  if (lane < deg) {
    const int pe = A.ne[k0 + lane];
    const int e = pe >> 2, l = pe & 3;
    double X[4][3];
    int nodes[4];
    load_elem<TPTFEM_CELL_TET4>(A.in, e, X, nodes);
    TetGeom G;
    ok = tet_geom(X, G);
    const double coef = A.in.coef[A.in.per_elem ? e : 0];
    const double w0 = c_cell.w[0];
    if constexpr (PHYS == 0) {
      const double wk = w0 * coef;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        double dot = G.g[l][0] * G.g[j][0] + G.g[l][1] * G.g[j][1] + G.g[l][2] * G.g[j][2];
        double t = wk * dot * G.adet;
        double v = t + t;  // four identical quadrature points, summed in order
        v = v + t;
        blk[w][lane][j][0] = v + t;
      }
    } else {
      const Dmat D = make_d(A.in.model, coef, A.in.nu);
      const double wd = w0 * G.adet;
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int a = 0; a < DPN; ++a)
#pragma unroll
          for (int b = 0; b < DPN; ++b) {
            double t = wd * bdb3(G.g[l], G.g[j], a, b, D);
            double v = t + t;
            v = v + t;
            blk[w][lane][j][a * DPN + b] = v + t;
          }
    }
    bslot[w][lane] = A.slot[k0 + lane];
  }
  __syncwarp();
  double acc[D2];
  unsigned nz = 0;  // bit a * DPN + b
#pragma unroll
  for (int q = 0; q < D2; ++q) acc[q] = 0.0;
  for (int i = 0; i < deg; ++i) {
    const uchar4 sl = bslot[w][i];
    const int j = sl.x == lane ? 0 : (sl.y == lane ? 1 : (sl.z == lane ? 2 : (sl.w == lane ? 3 : -1)));
    if (j < 0) continue;
#pragma unroll
    for (int q = 0; q < D2; ++q) {
      const double v = blk[w][i][j][q];
      acc[q] = acc[q] + v;
      nz |= (unsigned)(v != 0.0) << q;
    }
  }
  if (__any_sync(0xffffffffu, !ok) && lane == 0) atomicOr(A.flag, 1);
  const int nb0 = A.nb_ptr[n], nnb = A.nb_ptr[n + 1] - nb0;
  const bool mine = lane < nnb;
  const int col0 = mine ? A.nb[nb0 + lane] * DPN : 0;
#pragma unroll
  for (int a = 0; a < DPN; ++a) {
    const int64_t r = n * DPN + a;
    const unsigned rowbits = mine ? (nz >> (a * DPN)) & ((1u << DPN) - 1u) : 0u;
    const int cnt = __popc(rowbits);
    int pre = cnt;  // inclusive scan over lanes = slots in column order
    for (int o2 = 1; o2 < 32; o2 <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, pre, o2);
      if (lane >= o2) pre += t;
    }
    const int total = __shfl_sync(0xffffffffu, pre, 31);
    int off = pre - cnt;
    if (mode == MODE_COUNT || mode == MODE_PADDED) {
      if (lane == 0) A.row_cnt[r] = total;
      if (mode == MODE_COUNT) continue;
    }
    int base = 0, end = 0;
    if (mode != MODE_PADDED) {
      base = A.row_ptr[r];
      end = A.row_ptr[r + 1];
      if (mode == MODE_NUMERIC && lane == 0 && end - base != total) atomicOr(A.flag, 2);
    }
    int* cdst = mode == MODE_PADDED ? A.col + r * A.maxc : A.col + base;
    double* vdst = mode == MODE_PADDED ? A.val + r * A.maxc : A.val + base;
#pragma unroll
    for (int b = 0; b < DPN; ++b) {
      if (!((rowbits >> b) & 1u)) continue;
      const int cidx = col0 + b;
      if (mode == MODE_NUMERIC) {
        if (base + off >= end || cdst[off] != cidx) atomicOr(A.flag, 2);
        else vdst[off] = acc[a * DPN + b];
      } else {
        cdst[off] = cidx;
        vdst[off] = acc[a * DPN + b];
      }
      ++off;
    }
  }
}

// ---- Tet4 rows through ordered chains ---------------------------------------------
// assemble_nodes_tet adds each incidence's blocks into the node's slots in a
// loop over all incidences in which only the few lanes owning the element's
// slots work, with an FP64 compare per value for the pattern; its issue slots,
// not HBM, are the limit.  tet_node_rows keeps one warp per node but sums
// every slot over a precomputed chain -- the incidences whose element holds
// that slot's node, in ascending element id -- so each addition is done by
// the lane that needs it, and the node's own slot (whose chain has every
// incident element) is spread over one lane per entry.  A one-element
// "record" (gradients, w|det|, constitutive constants) is formed per
// incidence; the value stores stream past L2 (st.global.cs).  Forming the
// records once per element in a separate pass and reading them back from an
// L2-resident ring was measured slower (6.2 against 3.3 ms at 280x70x70)
// than forming them per incidence, and was not kept.
//
// Record (16 doubles): g[4][3], the element's physical gradients, then
//   elasticity: w |det|, D00, D01, Dshear;  Poisson: w k, |det|, 0, 0.
// Per entry the four identical quadrature points add t = (w|det|) s four
// times from 0.0: 0 + t = t and t + t = 2t are exact, so the sum is
// fl(fl(3t) + t), the same bits in two operations instead of four.
constexpr int TR_DOUBLES = 16;  // doubles per element record
constexpr int TN_WARPS = 2;     // warps (nodes) per block of tet_node_rows
constexpr int TN_MAXDEG = 32;   // incident elements per node handled by one warp (at most)
// Resident blocks per SM the register budget of tet_node_rows is cut for:
// 16 (64 registers) by default; TPTFEM_TET_MINB=8 gives the compiler 80.
int tet_minb() {
  static int v = -1;
  if (v < 0) {
    const char* e = std::getenv("TPTFEM_TET_MINB");
    v = (e && std::atoi(e) == 8) ? 8 : 16;
  }
  return v;
}

// Element e's record (geometry and constitutive constants); false for a
// degenerate element.
template <int PHYS>
__device__ __forceinline__ bool tet_record(const ElemIn& in, int64_t e, double (&r)[TR_DOUBLES]) {
  double X[4][3];
  int nodes[4];
  load_elem<TPTFEM_CELL_TET4>(in, (int)e, X, nodes);
  TetGeom G;
  const bool ok = tet_geom(X, G);
  const double coef = in.coef[in.per_elem ? e : 0];
  const double w0 = c_cell.w[0];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k) r[i * 3 + k] = G.g[i][k];
  if constexpr (PHYS == 1) {
    const Dmat D = make_d(in.model, coef, in.nu);
    r[12] = w0 * G.adet;
    r[13] = D.d00;
    r[14] = D.d01;
    r[15] = D.dsh;
  } else {
    r[12] = w0 * coef;
    r[13] = G.adet;
    r[14] = r[15] = 0.0;
  }
  return ok;
}

// Chains (once per mesh): node n's entries in neighbour slot s are summed over
// the incidences whose element holds slot s's node, in ascending element id;
// give every (incidence k, element node j) a position in its slot's chain:
// chains are stored one after another in slot order, coff[nb_ptr[n] + s] is
// where slot s's chain starts (the last ends at 4 * deg), and cpos[k] holds
// the positions of incidence k's four blocks.  One warp per node; one ballot
// per slot gives the incidences of that slot in ascending order.
__global__ void tet_chains(int64_t n_nodes, const int* __restrict__ ne_ptr, const uchar4* __restrict__ slot,
                           const int* __restrict__ nb_ptr, uchar4* __restrict__ cpos,
                           unsigned char* __restrict__ coff) {
  const int lane = threadIdx.x & 31;
  const int64_t n = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (n >= n_nodes) return;
  const int k0 = ne_ptr[n], deg = ne_ptr[n + 1] - k0;
  const int nb0 = nb_ptr[n], nnb = nb_ptr[n + 1] - nb0;
  const uchar4 sl = lane < deg ? slot[k0 + lane] : make_uchar4(255, 255, 255, 255);
  unsigned mymask = 0;
  for (int t = 0; t < nnb; ++t) {
    const unsigned m = __ballot_sync(0xffffffffu, sl.x == t || sl.y == t || sl.z == t || sl.w == t);
    if (lane == t) mymask = m;
  }
  const int len = __popc(mymask);
  int pre = len;
  for (int o2 = 1; o2 < 32; o2 <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, pre, o2);
    if (lane >= o2) pre += t;
  }
  if (lane < nnb) coff[nb0 + lane] = (unsigned char)(pre - len);
  const int sj[4] = {sl.x, sl.y, sl.z, sl.w};
  const unsigned below = (1u << lane) - 1u;
  int pos[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int s = sj[j] & 31;
    pos[j] = __shfl_sync(0xffffffffu, pre - len, s) + __popc(__shfl_sync(0xffffffffu, mymask, s) & below);
  }
  if (lane < deg) cpos[k0 + lane] = make_uchar4(pos[0], pos[1], pos[2], pos[3]);
}

// One warp per node of [n0, n1).
//  1. Lane k takes incidence k (element e_k, the node's local index l_k), reads
//     e_k's record and forms the node's blocks against the element's four
//     nodes (9 entries each for elasticity), writing block j at its chain
//     position cpos[k].j with the mask of its non-zero entries.
//  2. Each slot's chain is summed entry by entry from +0.0 in chain order --
//     ascending element id, Coo::to_csr's sequential duplicate sum
//     (crates/tpt-fem-sparse/src/lib.rs:144-163) -- with the masks ORed: lane s
//     for the other slots, D2 lanes (one entry each) for the node's own slot,
//     whose chain holds every incident element.
//  3. Lane s writes slot s's entries to the node's rows (one scan gives the
//     positions in all DPN rows).
//   COUNT / FILL / PADDED: as assemble_nodes_tet; the masks are stored per
//     neighbour entry (nzm[nb_ptr[n] + s]).
//   NUMERIC: the masks must equal the stored ones (else flag bit 2: the
//     pattern changed); values go to the positions the pattern gives them,
//     without reading the column indices back.
template <int PHYS, int DPN, int MAXDEG, int MINB>
__global__ void __launch_bounds__(32 * TN_WARPS, MINB) tet_node_rows(RowArgs A, int64_t n0, int64_t n1,
                                                                     const uchar4* __restrict__ cpos,
                                                                     const unsigned char* __restrict__ coff,
                                                                     unsigned short* __restrict__ nzm, int mode) {
  constexpr int D2 = DPN * DPN;
  constexpr int CS = DPN == 1 ? 1 : 10;  // chain entry stride in doubles (16-byte rows for DPN 3)
  __shared__ __align__(16) double chain[TN_WARPS][4 * MAXDEG][CS];
  __shared__ unsigned short cnz[TN_WARPS][4 * MAXDEG];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t n = n0 + (int64_t)blockIdx.x * TN_WARPS + w;
  if (n >= n1) return;  // whole warps leave together
  const int k0 = A.ne_ptr[n], deg = A.ne_ptr[n + 1] - k0;
  const int nb0 = A.nb_ptr[n], nnb = A.nb_ptr[n + 1] - nb0;
  // slot data first, so its loads overlap the block work
  const bool mine = lane < nnb;
  int col = 0, c0 = 0, c1 = 0;
  if (mine) {
    col = A.nb[nb0 + lane];
    c0 = coff[nb0 + lane];
    c1 = lane + 1 < nnb ? coff[nb0 + lane + 1] : 4 * deg;
  }
  // 1. blocks into their chains
  if (lane < deg) {
    const int pe = A.ne[k0 + lane];
    const uchar4 cp = cpos[k0 + lane];
    double r[TR_DOUBLES];
    if (!tet_record<PHYS>(A.in, pe >> 2, r)) atomicOr(A.flag, 1);
    const int l = pe & 3;
    double gl[3];  // the node's own gradient row, selected without a dynamic register index
#pragma unroll
    for (int c = 0; c < 3; ++c) gl[c] = l == 0 ? r[c] : (l == 1 ? r[3 + c] : (l == 2 ? r[6 + c] : r[9 + c]));
    const int pj[4] = {cp.x, cp.y, cp.z, cp.w};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const double* gj = r + 3 * j;
      double v[D2];
      if constexpr (PHYS == 0) {
        const double dot = gl[0] * gj[0] + gl[1] * gj[1] + gl[2] * gj[2];
        const double t = r[12] * dot * r[13];
        v[0] = 3.0 * t + t;
      } else {
        const double wd = r[12], m = r[13], cn = r[14], d = r[15];
        const double pm0 = gl[0] * m, pm1 = gl[1] * m, pm2 = gl[2] * m;
        const double pc0 = gl[0] * cn, pc1 = gl[1] * cn, pc2 = gl[2] * cn;
        const double pd0 = gl[0] * d, pd1 = gl[1] * d, pd2 = gl[2] * d;
        // bdb3's sums, term for term
        const double sm[9] = {(pm0 * gj[0] + pd1 * gj[1]) + pd2 * gj[2], pc0 * gj[1] + pd1 * gj[0],
                              pc0 * gj[2] + pd2 * gj[0],                  pc1 * gj[0] + pd0 * gj[1],
                              (pm1 * gj[1] + pd0 * gj[0]) + pd2 * gj[2], pc1 * gj[2] + pd2 * gj[1],
                              pc2 * gj[0] + pd0 * gj[2],                  pc2 * gj[1] + pd1 * gj[2],
                              (pm2 * gj[2] + pd1 * gj[1]) + pd0 * gj[0]};
#pragma unroll
        for (int q = 0; q < 9; ++q) {
          const double t = wd * sm[q];
          v[q] = 3.0 * t + t;
        }
      }
      unsigned msk = 0;
#pragma unroll
      for (int q = 0; q < D2; ++q) msk |= (unsigned)(v[q] != 0.0) << q;
      double* dst = chain[w][pj[j]];
      if constexpr (DPN == 1) {
        dst[0] = v[0];
      } else {
#pragma unroll
        for (int q = 0; q < 4; ++q) reinterpret_cast<double2*>(dst)[q] = make_double2(v[2 * q], v[2 * q + 1]);
        dst[8] = v[8];
      }
      cnz[w][pj[j]] = (unsigned short)msk;
    }
  }
  __syncwarp();
  // 2. ordered chain sums, in two loops so that neither runs the other's body:
  //  a. lane s (a slot other than the node's own) sums its chain, all D2
  //     entries per element (its chain is short: the elements sharing an edge);
  //  b. the node's own slot, whose chain holds every incident element: lane q
  //     (< D2) sums entry q, and the sums move to the slot's lane.
  const unsigned selfm = __ballot_sync(0xffffffffu, mine && col == (int)n);
  const int self = selfm ? __ffs(selfm) - 1 : -1;
  double acc[D2];
#pragma unroll
  for (int q = 0; q < D2; ++q) acc[q] = 0.0;
  unsigned nzb = 0;
  {
    const bool own = mine && lane != self;
    const int e1 = own ? c1 : 0;
    for (int c = own ? c0 : 0; c < e1; ++c) {
      const double* e = chain[w][c];
      if constexpr (DPN == 1) {
        acc[0] = acc[0] + e[0];
      } else {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const double2 v = reinterpret_cast<const double2*>(e)[q];
          acc[2 * q] = acc[2 * q] + v.x;
          acc[2 * q + 1] = acc[2 * q + 1] + v.y;
        }
        acc[8] = acc[8] + e[8];
      }
      nzb |= cnz[w][c];
    }
  }
  if (self >= 0) {
    const int sc0 = __shfl_sync(0xffffffffu, c0, self), sc1 = __shfl_sync(0xffffffffu, c1, self);
    double sv = 0.0;
    unsigned snz = 0;
    if (lane < D2) {  // loads run ahead of the dependent additions, four at a time
      int c = sc0;
      for (; c + 4 <= sc1; c += 4) {
        const double v0 = chain[w][c][lane], v1 = chain[w][c + 1][lane], v2 = chain[w][c + 2][lane],
                     v3 = chain[w][c + 3][lane];
        snz |= cnz[w][c] | cnz[w][c + 1] | cnz[w][c + 2] | cnz[w][c + 3];
        sv = sv + v0;
        sv = sv + v1;
        sv = sv + v2;
        sv = sv + v3;
      }
      for (; c < sc1; ++c) {
        sv = sv + chain[w][c][lane];
        snz |= cnz[w][c];
      }
    }
#pragma unroll
    for (int q = 0; q < D2; ++q) {
      const double t = __shfl_sync(0xffffffffu, sv, q);
      if (lane == self) acc[q] = t;
    }
    const unsigned tn = __shfl_sync(0xffffffffu, snz, 0);
    if (lane == self) nzb = tn;
  }
  // 3. rows
  const unsigned nz = mine ? nzb : 0u;
  if (mine) {
    if (mode == MODE_NUMERIC) {
      if (nzm[nb0 + lane] != (unsigned short)nz) atomicOr(A.flag, 2);
    } else {
      nzm[nb0 + lane] = (unsigned short)nz;
    }
  }
  // the DPN rows' counts packed in one word (8 bits each; a row has at most
  // 3 * 32 entries), so one scan over the lanes gives every row's positions
  unsigned packed = 0;
#pragma unroll
  for (int a = 0; a < DPN; ++a) packed |= (unsigned)__popc((nz >> (a * DPN)) & ((1u << DPN) - 1u)) << (8 * a);
  unsigned pr = packed;
  for (int o2 = 1; o2 < 32; o2 <<= 1) {
    const unsigned t = __shfl_up_sync(0xffffffffu, pr, o2);
    if (lane >= o2) pr += t;
  }
  const unsigned totals = __shfl_sync(0xffffffffu, pr, 31);
  const int col0 = col * DPN;
#pragma unroll
  for (int a = 0; a < DPN; ++a) {
    const int64_t r = n * DPN + a;
    const unsigned rowbits = (nz >> (a * DPN)) & ((1u << DPN) - 1u);
    const int total = (totals >> (8 * a)) & 255u;
    int off = (int)((pr >> (8 * a)) & 255u) - __popc(rowbits);
    if (mode == MODE_COUNT || mode == MODE_PADDED) {
      if (lane == 0) A.row_cnt[r] = total;
      if (mode == MODE_COUNT) continue;
    }
    int base = 0, rlen = A.maxc;
    if (mode != MODE_PADDED) {
      base = A.row_ptr[r];
      rlen = A.row_ptr[r + 1] - base;
      if (mode == MODE_NUMERIC && lane == 0 && rlen != total) atomicOr(A.flag, 2);
    }
    int* cdst = mode == MODE_PADDED ? A.col + r * A.maxc : A.col + base;
    double* vdst = mode == MODE_PADDED ? A.val + r * A.maxc : A.val + base;
#pragma unroll
    for (int b = 0; b < DPN; ++b) {
      if (!((rowbits >> b) & 1u)) continue;
      if (off < rlen) {  // a changed pattern (flagged) may not fit the row
        if (mode != MODE_NUMERIC) cdst[off] = col0 + b;
        __stcs(vdst + off, acc[a * DPN + b]);
      }
      ++off;
    }
  }
}

// ---- loads ----------------------------------------------------------------------

struct LoadArgs {
  ElemIn in;
  const int* ne_ptr;
  const int* ne;
  int64_t n_nodes;
  double b[3];  // source value (Poisson) or body force (elasticity)
  // per-quadrature-point values instead of b (nullptr: constant b): KIND 0 one
  // source value per (element, point), KIND 1 DPN body-force components
  const double* pv;
  double* rhs;
  int* flag;
};

// rhs[n*DPN + a] = sum over incident elements (ascending id) of the element
// load entry, like the reference's `rhs[node] += f[i]` loops.
// KIND 0: poisson_source_vector (thermal:163-196); KIND 1: elasticity_body_vector (elasticity:312-348).
template <int CELL, int KIND, int DPN>
__global__ void load_rows(LoadArgs A) {
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= A.n_nodes) return;
  double acc[DPN];
#pragma unroll
  for (int a = 0; a < DPN; ++a) acc[a] = 0.0;
  bool ok = true;
  for (int k = A.ne_ptr[n]; k < A.ne_ptr[n + 1]; ++k) {
    const int e = A.ne[k] >> 2, l = A.ne[k] & 3;
    double X[4][CellTraits<CELL>::SD];
    int nodes[4];
    load_elem<CELL>(A.in, e, X, nodes);
    double f[DPN];
#pragma unroll
    for (int a = 0; a < DPN; ++a) f[a] = 0.0;
    const int nq = c_cell.nq;
    // the source value or body force at point q: the constant, or the caller's
    // value at that point
    auto bval = [&](int q, int a) { return A.pv ? A.pv[((int64_t)e * nq + q) * DPN + a] : A.b[a]; };
    if constexpr (CELL == TPTFEM_CELL_TET4) {
      TetGeom G;
      ok &= tet_geom(X, G);
      for (int q = 0; q < nq; ++q) {
        const double w = c_cell.w[q], N = c_cell.ns[q][l];
        if (KIND == 0) f[0] = f[0] + w * bval(q, 0) * N * G.adet;
        else
#pragma unroll
          for (int a = 0; a < DPN; ++a) f[a] = f[a] + w * N * bval(q, a) * G.adet;
      }
    } else if constexpr (CELL == TPTFEM_CELL_TRI3) {
      TriGeom G;
      ok &= tri_geom(X, G);
      for (int q = 0; q < nq; ++q) {
        const double w = c_cell.w[q], N = c_cell.ns[q][l];
        if (KIND == 0) f[0] = f[0] + w * bval(q, 0) * N * G.adet;
        else
#pragma unroll
          for (int a = 0; a < DPN; ++a) f[a] = f[a] + w * N * bval(q, a) * G.adet;
      }
    } else {
      for (int q = 0; q < nq; ++q) {
        QuadGeom G;
        ok &= quad_geom(X, q, G);
        const double w = c_cell.w[q], N = c_cell.ns[q][l];
        if (KIND == 0) f[0] = f[0] + w * bval(q, 0) * N * G.adet;
        else
#pragma unroll
          for (int a = 0; a < DPN; ++a) f[a] = f[a] + w * N * bval(q, a) * G.adet;
      }
    }
#pragma unroll
    for (int a = 0; a < DPN; ++a) acc[a] = acc[a] + f[a];
  }
  if (!ok) atomicOr(A.flag, 1);
#pragma unroll
  for (int a = 0; a < DPN; ++a) A.rhs[n * DPN + a] = acc[a];
}

struct TractionArgs {
  ElemIn in;
  const int* ne_ptr;
  const int* ne;
  const unsigned char* bface;
  int64_t n_nodes;
  int dpn, axis;
  double sign;
  double t[3];
  // general flux (g != nullptr): g at every boundary-face quadrature point,
  // indexed (face_off[e] + rank of the face among e's boundary faces) * nqf + q,
  // added to the components in comp_mask
  const double* g;
  const int* face_off;
  unsigned comp_mask;
  double* rhs;
};

// apply_neumann_order (assembly:601-667) with the face-selector flux, one
// thread per node visiting its boundary faces in (element, face) order.
template <int CELL>
__global__ void traction_rows(TractionArgs A) {
  constexpr int SD = CellTraits<CELL>::SD;
  constexpr int FN = FaceTraits<CELL>::FN, NF = FaceTraits<CELL>::NF;
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= A.n_nodes) return;
  double acc[3];
  for (int c = 0; c < A.dpn; ++c) acc[c] = A.rhs[n * A.dpn + c];
  for (int k = A.ne_ptr[n]; k < A.ne_ptr[n + 1]; ++k) {
    const int e = A.ne[k] >> 2, l = A.ne[k] & 3;
    const unsigned bm = A.bface[e];
    if (!bm) continue;
    double X[4][SD];
    int nodes[4];
    load_elem<CELL>(A.in, e, X, nodes);
    for (int fi = 0; fi < NF; ++fi) {
      if (!(bm & (1u << fi))) continue;
      int fl[3];
      int kpos = -1;
      for (int q = 0; q < FN; ++q) {
        fl[q] = FaceTraits<CELL>::node(fi, q);
        if (fl[q] == l) kpos = q;
      }
      if (kpos < 0) continue;
      double measure, nrm[SD];
      face_geometry<CELL, SD>(X, fl, measure, nrm);
      if (A.g) {
        const int64_t fp = (int64_t)(A.face_off[e] + __popc(bm & ((1u << fi) - 1u))) * c_face.nq;
        for (int q = 0; q < c_face.nq; ++q) {
          const double wm = c_face.w[q] * measure, N = c_face.ns[q][kpos], g = A.g[fp + q];
          for (int c = 0; c < A.dpn; ++c)
            if (A.comp_mask & (1u << c)) acc[c] = acc[c] + wm * g * N;
        }
        continue;
      }
      const bool sel = nrm[A.axis] * A.sign > 0.5;
      for (int q = 0; q < c_face.nq; ++q) {
        const double wm = c_face.w[q] * measure, N = c_face.ns[q][kpos];
        for (int c = 0; c < A.dpn; ++c) {
          const double g = sel ? A.t[c] : 0.0;
          acc[c] = acc[c] + wm * g * N;
        }
      }
    }
  }
  for (int c = 0; c < A.dpn; ++c) A.rhs[n * A.dpn + c] = acc[c];
}

// ---- quadrature points for caller-evaluated sources and fluxes ---------------

// Physical quadrature points of every element, x_q[d] = sum_k N_k(xi_q) X_k[d]
// summed over k from 0.0 for each of the cdim stored coordinates, as
// poisson_source_vector / elasticity_body_vector form the point they hand to
// the source closure (thermal:163-196, elasticity:312-348).  Output
// ((e * nq) + q) * cdim + d.
template <int CELL>
__global__ void quad_points(ElemIn in, int64_t n_elems, double* __restrict__ out) {
  constexpr int NV = CellTraits<CELL>::NV;
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_elems) return;
  int nodes[4];
  for (int j = 0; j < NV; ++j) nodes[j] = in.conn[e * NV + j];
  const int nq = c_cell.nq;
  for (int q = 0; q < nq; ++q)
    for (int d = 0; d < in.cdim; ++d) {
      double x = 0.0;
      for (int k = 0; k < NV; ++k) x = x + c_cell.ns[q][k] * in.coords[(int64_t)nodes[k] * in.cdim + d];
      out[(e * nq + q) * in.cdim + d] = x;
    }
}

__global__ void face_counts(int64_t n_elems, const unsigned char* __restrict__ bface, int* __restrict__ cnt) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n_elems) cnt[e] = __popc((unsigned)bface[e]);
}

// Boundary-face quadrature points and outward unit normals in (element, face,
// point) order -- the order boundary_faces lists the faces in
// (assembly:563-583) -- with x_q summed over the face's nodes as
// apply_neumann_order / apply_robin_order do (assembly:601-667, 684-753).
template <int CELL>
__global__ void face_points(ElemIn in, int64_t n_elems, const unsigned char* __restrict__ bface,
                            const int* __restrict__ face_off, double* __restrict__ xo, double* __restrict__ no) {
  constexpr int SD = CellTraits<CELL>::SD, FN = FaceTraits<CELL>::FN, NF = FaceTraits<CELL>::NF;
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_elems) return;
  const unsigned bm = bface[e];
  if (!bm) return;
  double X[4][SD];
  int nodes[4];
  load_elem<CELL>(in, (int)e, X, nodes);
  int rank = 0;
  for (int fi = 0; fi < NF; ++fi) {
    if (!(bm & (1u << fi))) continue;
    int fl[3];
    for (int q = 0; q < FN; ++q) fl[q] = FaceTraits<CELL>::node(fi, q);
    double measure, nrm[SD];
    face_geometry<CELL, SD>(X, fl, measure, nrm);
    const int64_t fp = (int64_t)(face_off[e] + rank) * c_face.nq;
    for (int q = 0; q < c_face.nq; ++q) {
      for (int d = 0; d < SD; ++d) {
        double x = 0.0;
        for (int k = 0; k < FN; ++k) x = x + c_face.ns[q][k] * X[fl[k]][d];
        xo[(fp + q) * SD + d] = x;
        no[(fp + q) * SD + d] = nrm[d];
      }
    }
    ++rank;
  }
}

ElemIn elem_in(const MeshData& m, const double* coef, int per_elem, int model, double nu) {
  ElemIn in;
  in.coords = m.coords.p;
  in.cdim = m.cdim;
  in.conn = m.conn.p;
  in.coef = coef;
  in.per_elem = per_elem;
  in.model = model;
  in.nu = nu;
  return in;
}

void set_cell_tab(const MeshData& m, int quad_order, cudaStream_t s) {
  QuadTab t = make_cell_tab(m.cell, quad_order);
  TPT_CUDA(cudaMemcpyToSymbolAsync(c_cell, &t, sizeof(t), 0, cudaMemcpyHostToDevice, s));
}

// Boundary faces and the face quadrature (FACE_QUAD_ORDER 2) for a Robin term.
void set_robin_faces(MeshData& m, int axis, cudaStream_t s) {
  const int sd = m.cell == TPTFEM_CELL_TET4 ? 3 : 2;
  TPT_REQUIRE(axis < sd, TPTFEM_ERR_INVALID_ARG, "robin axis out of range for the mesh dimension");
  mesh_build_boundary_faces(m);
  mesh_build_face_offsets(m);
  FaceTab f = make_face_tab(m.cell);
  TPT_CUDA(cudaMemcpyToSymbolAsync(c_face, &f, sizeof(f), 0, cudaMemcpyHostToDevice, s));
}

int read_flag(tptfem_context* ctx) {
  TPT_CUDA(cudaMemcpyAsync(ctx->h_pinned, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  TPT_CUDA(cudaStreamSynchronize(ctx->stream));
  return ctx->h_pinned[0];
}

void tet_build_chains(MeshData& m) {
  if (m.tchains) return;
  cudaStream_t s = m.ctx->stream;
  m.cpos.alloc(std::max<size_t>(m.ne.n, 1), s);
  m.coff.alloc(std::max<size_t>(m.nb.n, 1), s);
  tet_chains<<<ceil_div(m.n_nodes * 32, 256), 256, 0, s>>>(m.n_nodes, m.ne_ptr.p, m.slot.p, m.nb_ptr.p, m.cpos.p,
                                                          m.coff.p);
  TPT_CHECK_LAUNCH();
  m.tchains = true;
}

template <int PHYS, int DPN>
void launch_tet_chains(MatrixData& M, int mode, const RowArgs& A, cudaStream_t s) {
  MeshData& m = *M.mesh;
  tet_build_chains(m);
  if (M.nzmask.n != m.nb.n) M.nzmask.alloc(m.nb.n, s);
  const int grid = ceil_div(m.n_nodes, TN_WARPS);
  // fewer incidences per node, less shared memory per warp, more warps per SM
  const bool d24 = m.max_deg <= 24, b16 = tet_minb() == 16;
  auto go = [&](auto kern) {
    kern<<<grid, 32 * TN_WARPS, 0, s>>>(A, 0, m.n_nodes, m.cpos.p, m.coff.p, M.nzmask.p, mode);
  };
  if (d24 && b16) go(tet_node_rows<PHYS, DPN, 24, 16>);
  else if (d24) go(tet_node_rows<PHYS, DPN, 24, 8>);
  else if (b16) go(tet_node_rows<PHYS, DPN, 32, 16>);
  else go(tet_node_rows<PHYS, DPN, 32, 8>);
  TPT_CHECK_LAUNCH();
}

// TPTFEM_TET_ASM=warp selects assemble_nodes_tet instead of tet_node_rows
// (for A/B timing; both give the same bits).
bool tet_warp_kernel() {
  static int v = -1;
  if (v < 0) {
    const char* e = std::getenv("TPTFEM_TET_ASM");
    v = (e && std::strcmp(e, "warp") == 0) ? 1 : 0;
  }
  return v == 1;
}

template <int PHYS, int DPN>
void launch_nodes_tet(int mode, const RowArgs& A, int64_t n_nodes, cudaStream_t s) {
  assemble_nodes_tet<PHYS, DPN><<<ceil_div(n_nodes, AN_WARPS), 32 * AN_WARPS, 0, s>>>(A, n_nodes, mode);
  TPT_CHECK_LAUNCH();
}

template <int CELL, int PHYS, int DPN>
void launch_rows(int mode, const RowArgs& A, cudaStream_t s) {
  // Threads per block: the dense accumulator (9 bytes per slot and thread)
  // must fit in shared memory.
  int threads = 128;
  while (threads > 32 && (size_t)threads * A.maxc * 9 > 200 * 1024) threads -= 32;
  size_t smem = (size_t)threads * A.maxc * 9;
  TPT_REQUIRE(smem <= 227 * 1024, TPTFEM_ERR_CREATION, "node valence too high for the device assembly path");
  auto run = [&](auto kern) {
    TPT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<ceil_div(A.nrows, threads), threads, smem, s>>>(A);
    TPT_CHECK_LAUNCH();
  };
  if (mode == MODE_COUNT) run(assemble_rows<CELL, PHYS, DPN, MODE_COUNT>);
  else if (mode == MODE_FILL) run(assemble_rows<CELL, PHYS, DPN, MODE_FILL>);
  else if (mode == MODE_PADDED) run(assemble_rows<CELL, PHYS, DPN, MODE_PADDED>);
  else run(assemble_rows<CELL, PHYS, DPN, MODE_NUMERIC>);
}

void dispatch_rows(MatrixData& M, int mode, const RowArgs& A, cudaStream_t s) {
  const int cell = M.mesh->cell;
  const MeshData& m = *M.mesh;
  if (cell == TPTFEM_CELL_TET4 && !A.robin && m.max_nb <= 32 && m.max_deg <= TN_MAXDEG && !tet_warp_kernel()) {
    // a warp per node: at most 32 neighbour slots and incident elements
    if (M.physics == 0) launch_tet_chains<0, 1>(M, mode, A, s);
    else launch_tet_chains<1, 3>(M, mode, A, s);
  } else if (cell == TPTFEM_CELL_TET4 && !A.robin && m.max_nb <= 32 && m.max_deg <= AN_MAXDEG) {
    if (M.physics == 0) launch_nodes_tet<0, 1>(mode, A, m.n_nodes, s);
    else launch_nodes_tet<1, 3>(mode, A, m.n_nodes, s);
  } else if (cell == TPTFEM_CELL_TET4) {
    if (M.physics == 0) launch_rows<TPTFEM_CELL_TET4, 0, 1>(mode, A, s);
    else launch_rows<TPTFEM_CELL_TET4, 1, 3>(mode, A, s);
  } else if (cell == TPTFEM_CELL_TRI3) {
    if (M.physics == 0) launch_rows<TPTFEM_CELL_TRI3, 0, 1>(mode, A, s);
    else launch_rows<TPTFEM_CELL_TRI3, 1, 2>(mode, A, s);
  } else {
    if (M.physics == 0) launch_rows<TPTFEM_CELL_QUAD4, 0, 1>(mode, A, s);
    else launch_rows<TPTFEM_CELL_QUAD4, 1, 2>(mode, A, s);
  }
}

RowArgs row_args(MatrixData& M) {
  MeshData& m = *M.mesh;
  RowArgs A;
  A.in = elem_in(m, M.coef.p, M.per_element, M.model, M.nu);
  A.ne_ptr = m.ne_ptr.p;
  A.ne = m.ne.p;
  A.slot = m.slot.p;
  A.nb_ptr = m.nb_ptr.p;
  A.nb = m.nb.p;
  A.nrows = M.nrows;
  A.row_cnt = nullptr;
  A.row_ptr = M.row_ptr.p;
  A.col = M.col.p;
  A.val = M.val.p;
  A.flag = M.ctx->d_flag;
  A.maxc = m.max_nb * M.dpn;
  A.bface = M.robin ? m.bface.p : nullptr;
  A.robin = M.robin;
  A.raxis = M.robin_axis;
  A.rsign = M.robin_sign;
  A.rh = M.robin_h;
  A.rpts = (M.robin && M.robin_pts.n) ? M.robin_pts.p : nullptr;
  A.face_off = A.rpts ? m.face_off.p : nullptr;
  return A;
}

// Largest row/column index with an entry, plus one (what Coo::to_csr reports
// as nrows / ncols, crates/tpt-fem-sparse/src/lib.rs:124-139).
__global__ void ref_dims(const int* __restrict__ rp, const int* __restrict__ col, int64_t nrows, int* out) {
  int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrows) return;
  int b = rp[r], e = rp[r + 1];
  if (e > b) {
    atomicMax(out, (int)r);
    atomicMax(out + 1, col[e - 1]);
  }
}

// Padded rows -> CSR: one warp per row, lanes over its entries.
__global__ void compact_rows(int64_t nrows, int maxc, const int* __restrict__ pcol, const double* __restrict__ pval,
                             const int* __restrict__ row_ptr, int* __restrict__ col, double* __restrict__ val) {
  const int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= nrows) return;
  const int o = row_ptr[r], c = row_ptr[r + 1] - o;
  for (int i = lane; i < c; i += 32) {
    col[o + i] = pcol[r * maxc + i];
    val[o + i] = pval[r * maxc + i];
  }
}

// Scratch budget of the one-pass (padded) assembly; larger meshes count first.
constexpr int64_t PADDED_ASSEMBLY_BYTES = 12LL << 30;

}  // namespace

void assemble_matrix(MatrixData& M) {
  MeshData& m = *M.mesh;
  tptfem_context* ctx = M.ctx;
  cudaStream_t s = ctx->stream;
  TPT_REQUIRE(m.cell == TPTFEM_CELL_TET4 || m.cell == TPTFEM_CELL_QUAD4 || m.cell == TPTFEM_CELL_TRI3,
              TPTFEM_ERR_INVALID_ARG, "device assembly supports Tet4, Quad4 and Tri3 meshes");
  if (M.physics == 1) {
    bool okm = (m.cell == TPTFEM_CELL_TET4 && M.model == TPTFEM_MODEL_CONTINUUM_3D) ||
               ((m.cell == TPTFEM_CELL_QUAD4 || m.cell == TPTFEM_CELL_TRI3) &&
                (M.model == TPTFEM_MODEL_PLANE_STRESS || M.model == TPTFEM_MODEL_PLANE_STRAIN));
    TPT_REQUIRE(okm, TPTFEM_ERR_MODEL_DIM_MISMATCH,
                "elasticity model/dimension mismatch: model is incompatible with the mesh's spatial dimension");
  }
  M.dpn = M.physics == 0 ? 1 : (m.cell == TPTFEM_CELL_TET4 ? 3 : 2);
  mesh_build_adjacency(m);
  set_cell_tab(m, M.quad_order, s);
  if (M.robin) set_robin_faces(m, M.robin_axis, s);
  M.nrows = m.n_nodes * M.dpn;
  TPT_REQUIRE(M.nrows < (1LL << 31), TPTFEM_ERR_CREATION, "row count exceeds the int32 device index range");
  DevBuf<int> cnt;
  cnt.alloc(M.nrows + 1, s);
  TPT_CUDA(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), s));
  RowArgs A = row_args(M);
  A.row_cnt = cnt.p;
  const int64_t padded = M.nrows * (int64_t)A.maxc;
  if (padded * 12 <= PADDED_ASSEMBLY_BYTES) {  // one element pass into padded rows, then compaction
    DevBuf<int> pcol;
    DevBuf<double> pval;
    pcol.alloc(std::max<int64_t>(padded, 1), s);
    pval.alloc(std::max<int64_t>(padded, 1), s);
    A.col = pcol.p;
    A.val = pval.p;
    dispatch_rows(M, MODE_PADDED, A, s);
    TPT_REQUIRE((read_flag(ctx) & 1) == 0, TPTFEM_ERR_NUMERIC,
                "degenerate element: zero or non-finite Jacobian determinant");
    M.row_ptr.alloc(M.nrows + 1, s);
    M.nnz = exclusive_scan_i32(cnt.p, M.row_ptr.p, M.nrows, s);
    M.col.alloc(M.nnz, s);
    M.val.alloc(M.nnz, s);
    compact_rows<<<ceil_div(M.nrows * 32, 256), 256, 0, s>>>(M.nrows, A.maxc, pcol.p, pval.p, M.row_ptr.p, M.col.p,
                                                             M.val.p);
    TPT_CHECK_LAUNCH();
  } else {
    dispatch_rows(M, MODE_COUNT, A, s);
    TPT_REQUIRE((read_flag(ctx) & 1) == 0, TPTFEM_ERR_NUMERIC,
                "degenerate element: zero or non-finite Jacobian determinant");
    M.row_ptr.alloc(M.nrows + 1, s);
    M.nnz = exclusive_scan_i32(cnt.p, M.row_ptr.p, M.nrows, s);
    M.col.alloc(M.nnz, s);
    M.val.alloc(M.nnz, s);
    A = row_args(M);
    dispatch_rows(M, MODE_FILL, A, s);
  }
  DevBuf<int> dims;
  dims.alloc(2, s);
  TPT_CUDA(cudaMemsetAsync(dims.p, 0, 2 * sizeof(int), s));
  ref_dims<<<ceil_div(M.nrows, 256), 256, 0, s>>>(M.row_ptr.p, M.col.p, M.nrows, dims.p);
  TPT_CHECK_LAUNCH();
  int hd[2];
  TPT_CUDA(cudaMemcpyAsync(hd, dims.p, sizeof(hd), cudaMemcpyDeviceToHost, s));
  TPT_CUDA(cudaStreamSynchronize(s));
  M.ref_nrows = (int64_t)hd[0] + 1;
  M.ref_ncols = (int64_t)hd[1] + 1;
}

bool reassemble_values(MatrixData& M) {
  tptfem_context* ctx = M.ctx;
  cudaStream_t s = ctx->stream;
  set_cell_tab(*M.mesh, M.quad_order, s);
  if (M.robin) set_robin_faces(*M.mesh, M.robin_axis, s);
  TPT_CUDA(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), s));
  RowArgs A = row_args(M);
  dispatch_rows(M, MODE_NUMERIC, A, s);
  int f = read_flag(ctx);
  TPT_REQUIRE((f & 1) == 0, TPTFEM_ERR_NUMERIC, "degenerate element: zero or non-finite Jacobian determinant");
  return (f & 2) == 0;
}

double profile_numeric_assembly(MatrixData& M, int reps) {
  tptfem_context* ctx = M.ctx;
  cudaStream_t s = ctx->stream;
  set_cell_tab(*M.mesh, M.quad_order, s);
  if (M.robin) set_robin_faces(*M.mesh, M.robin_axis, s);
  TPT_CUDA(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), s));
  RowArgs A = row_args(M);
  dispatch_rows(M, MODE_NUMERIC, A, s);  // warm-up (module load, caches)
  TPT_CUDA(cudaEventRecord(ctx->ev[0], s));
  for (int r = 0; r < reps; ++r) dispatch_rows(M, MODE_NUMERIC, A, s);
  TPT_CUDA(cudaEventRecord(ctx->ev[1], s));
  TPT_CUDA(cudaEventSynchronize(ctx->ev[1]));
  float ms = 0.f;
  TPT_CUDA(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
  const int f = read_flag(ctx);
  TPT_REQUIRE(f == 0, TPTFEM_ERR_NUMERIC, "profiled re-assembly: degenerate element or changed pattern");
  return (double)ms / std::max(reps, 1);
}

void load_poisson_source(MeshData& m, double src, int quad_order, double* d_rhs, const double* d_pts) {
  tptfem_context* ctx = m.ctx;
  cudaStream_t s = ctx->stream;
  mesh_build_adjacency(m);
  set_cell_tab(m, quad_order, s);
  TPT_CUDA(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), s));
  LoadArgs A;
  A.in = elem_in(m, nullptr, 0, 0, 0.0);
  A.ne_ptr = m.ne_ptr.p;
  A.ne = m.ne.p;
  A.n_nodes = m.n_nodes;
  A.b[0] = src; A.b[1] = A.b[2] = 0.0;
  A.pv = d_pts;
  A.rhs = d_rhs;
  A.flag = ctx->d_flag;
  if (m.cell == TPTFEM_CELL_TET4) load_rows<TPTFEM_CELL_TET4, 0, 1><<<ceil_div(m.n_nodes, 128), 128, 0, s>>>(A);
  else if (m.cell == TPTFEM_CELL_TRI3) load_rows<TPTFEM_CELL_TRI3, 0, 1><<<ceil_div(m.n_nodes, 128), 128, 0, s>>>(A);
  else load_rows<TPTFEM_CELL_QUAD4, 0, 1><<<ceil_div(m.n_nodes, 128), 128, 0, s>>>(A);
  TPT_CHECK_LAUNCH();
  TPT_REQUIRE((read_flag(ctx) & 1) == 0, TPTFEM_ERR_NUMERIC, "degenerate element in load integration");
}

void load_body(MeshData& m, const double* body, int quad_order, double* d_rhs, const double* d_pts) {
  tptfem_context* ctx = m.ctx;
  cudaStream_t s = ctx->stream;
  mesh_build_adjacency(m);
  set_cell_tab(m, quad_order, s);
  TPT_CUDA(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), s));
  LoadArgs A;
  A.in = elem_in(m, nullptr, 0, 0, 0.0);
  A.ne_ptr = m.ne_ptr.p;
  A.ne = m.ne.p;
  A.n_nodes = m.n_nodes;
  A.b[0] = A.b[1] = A.b[2] = 0.0;
  if (body) { A.b[0] = body[0]; A.b[1] = body[1]; A.b[2] = m.cell == TPTFEM_CELL_TET4 ? body[2] : 0.0; }
  A.pv = d_pts;
  A.rhs = d_rhs;
  A.flag = ctx->d_flag;
  if (m.cell == TPTFEM_CELL_TET4) load_rows<TPTFEM_CELL_TET4, 1, 3><<<ceil_div(m.n_nodes, 128), 128, 0, s>>>(A);
  else if (m.cell == TPTFEM_CELL_TRI3) load_rows<TPTFEM_CELL_TRI3, 1, 2><<<ceil_div(m.n_nodes, 128), 128, 0, s>>>(A);
  else load_rows<TPTFEM_CELL_QUAD4, 1, 2><<<ceil_div(m.n_nodes, 128), 128, 0, s>>>(A);
  TPT_CHECK_LAUNCH();
  TPT_REQUIRE((read_flag(ctx) & 1) == 0, TPTFEM_ERR_NUMERIC, "degenerate element in load integration");
}

void apply_traction(MeshData& m, int dpn, int axis, double sign, const double* t, double* d_rhs) {
  cudaStream_t s = m.ctx->stream;
  const int sd = m.cell == TPTFEM_CELL_TET4 ? 3 : 2;
  TPT_REQUIRE(dpn >= 1 && dpn <= 3, TPTFEM_ERR_INVALID_ARG, "dofs_per_node must be 1..3");
  TPT_REQUIRE(axis >= 0 && axis < sd, TPTFEM_ERR_INVALID_ARG, "axis out of range for the mesh dimension");
  mesh_build_boundary_faces(m);
  FaceTab f = make_face_tab(m.cell);
  TPT_CUDA(cudaMemcpyToSymbolAsync(c_face, &f, sizeof(f), 0, cudaMemcpyHostToDevice, s));
  TractionArgs A;
  A.in = elem_in(m, nullptr, 0, 0, 0.0);
  A.ne_ptr = m.ne_ptr.p;
  A.ne = m.ne.p;
  A.bface = m.bface.p;
  A.n_nodes = m.n_nodes;
  A.dpn = dpn;
  A.axis = axis;
  A.sign = sign;
  for (int c = 0; c < 3; ++c) A.t[c] = c < dpn ? t[c] : 0.0;
  A.g = nullptr;
  A.face_off = nullptr;
  A.comp_mask = 0u;
  A.rhs = d_rhs;
  if (m.cell == TPTFEM_CELL_TET4) traction_rows<TPTFEM_CELL_TET4><<<ceil_div(m.n_nodes, 128), 128, 0, s>>>(A);
  else if (m.cell == TPTFEM_CELL_TRI3) traction_rows<TPTFEM_CELL_TRI3><<<ceil_div(m.n_nodes, 128), 128, 0, s>>>(A);
  else traction_rows<TPTFEM_CELL_QUAD4><<<ceil_div(m.n_nodes, 128), 128, 0, s>>>(A);
  TPT_CHECK_LAUNCH();
}

int cell_point_count(int cell, int quad_order) { return make_cell_tab(cell, quad_order).nq; }

int face_point_count(int cell) { return make_face_tab(cell).nq; }

void mesh_quad_points(MeshData& m, int quad_order, double* d_out) {
  cudaStream_t s = m.ctx->stream;
  set_cell_tab(m, quad_order, s);
  const ElemIn in = elem_in(m, nullptr, 0, 0, 0.0);
  const int grid = ceil_div(m.n_elems, 128);
  if (m.cell == TPTFEM_CELL_TET4) quad_points<TPTFEM_CELL_TET4><<<grid, 128, 0, s>>>(in, m.n_elems, d_out);
  else if (m.cell == TPTFEM_CELL_TRI3) quad_points<TPTFEM_CELL_TRI3><<<grid, 128, 0, s>>>(in, m.n_elems, d_out);
  else quad_points<TPTFEM_CELL_QUAD4><<<grid, 128, 0, s>>>(in, m.n_elems, d_out);
  TPT_CHECK_LAUNCH();
}

void mesh_build_face_offsets(MeshData& m) {
  if (m.foffs) return;
  mesh_build_boundary_faces(m);
  cudaStream_t s = m.ctx->stream;
  DevBuf<int> cnt;
  cnt.alloc(m.n_elems, s);
  face_counts<<<ceil_div(m.n_elems, 128), 128, 0, s>>>(m.n_elems, m.bface.p, cnt.p);
  TPT_CHECK_LAUNCH();
  m.face_off.alloc(m.n_elems + 1, s);
  m.n_bfaces = exclusive_scan_i32(cnt.p, m.face_off.p, m.n_elems, s);
  m.foffs = true;
}

void mesh_face_points(MeshData& m, double* d_x, double* d_n) {
  mesh_build_face_offsets(m);
  cudaStream_t s = m.ctx->stream;
  FaceTab f = make_face_tab(m.cell);
  TPT_CUDA(cudaMemcpyToSymbolAsync(c_face, &f, sizeof(f), 0, cudaMemcpyHostToDevice, s));
  const ElemIn in = elem_in(m, nullptr, 0, 0, 0.0);
  const int grid = ceil_div(m.n_elems, 128);
  if (m.cell == TPTFEM_CELL_TET4)
    face_points<TPTFEM_CELL_TET4><<<grid, 128, 0, s>>>(in, m.n_elems, m.bface.p, m.face_off.p, d_x, d_n);
  else if (m.cell == TPTFEM_CELL_TRI3)
    face_points<TPTFEM_CELL_TRI3><<<grid, 128, 0, s>>>(in, m.n_elems, m.bface.p, m.face_off.p, d_x, d_n);
  else
    face_points<TPTFEM_CELL_QUAD4><<<grid, 128, 0, s>>>(in, m.n_elems, m.bface.p, m.face_off.p, d_x, d_n);
  TPT_CHECK_LAUNCH();
}

void apply_neumann_points(MeshData& m, int dpn, const double* d_g, unsigned comp_mask, double* d_rhs) {
  cudaStream_t s = m.ctx->stream;
  TPT_REQUIRE(dpn >= 1 && dpn <= 3, TPTFEM_ERR_INVALID_ARG, "dofs_per_node must be 1..3");
  mesh_build_face_offsets(m);
  FaceTab f = make_face_tab(m.cell);
  TPT_CUDA(cudaMemcpyToSymbolAsync(c_face, &f, sizeof(f), 0, cudaMemcpyHostToDevice, s));
  TractionArgs A;
  A.in = elem_in(m, nullptr, 0, 0, 0.0);
  A.ne_ptr = m.ne_ptr.p;
  A.ne = m.ne.p;
  A.bface = m.bface.p;
  A.n_nodes = m.n_nodes;
  A.dpn = dpn;
  A.axis = 0;
  A.sign = 1.0;
  A.t[0] = A.t[1] = A.t[2] = 0.0;
  A.g = d_g;
  A.face_off = m.face_off.p;
  A.comp_mask = comp_mask;
  A.rhs = d_rhs;
  if (m.cell == TPTFEM_CELL_TET4) traction_rows<TPTFEM_CELL_TET4><<<ceil_div(m.n_nodes, 128), 128, 0, s>>>(A);
  else if (m.cell == TPTFEM_CELL_TRI3) traction_rows<TPTFEM_CELL_TRI3><<<ceil_div(m.n_nodes, 128), 128, 0, s>>>(A);
  else traction_rows<TPTFEM_CELL_QUAD4><<<ceil_div(m.n_nodes, 128), 128, 0, s>>>(A);
  TPT_CHECK_LAUNCH();
}

}  // namespace tptfem
