// oracle.cpp -- CPU restatement of tpt-fem's assembly -> CSR -> solve path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: it restates, in
// plain C++ and in the reference's own floating-point operation order, the
// Rust functions that the CUDA library replaces.  Only tests/, the smoke test
// and bench.py's CPU-baseline leg load it; the product path never does.
//
// Build flags matter: -O2 -ffp-contract=off -fno-fast-math (no FMA
// contraction, no reassociation), so every a*b+c rounds twice exactly as the
// reference's Rust code does.
//
// Reference files followed (paths relative to the tpt-fem project root):
//   crates/tpt-fem-mesh-gen/src/lib.rs      61-67 (orient3), 422-495 (box_mesh)
//   crates/tpt-fem-quadrature/src/lib.rs    118-162, 180-191, 223-234, 279-289
//   crates/tpt-fem-element/src/lib.rs       86-180 (shape/grad), 624-740 (Map)
//   crates/tpt-fem-thermal/src/lib.rs       29-92, 132-240
//   crates/tpt-fem-elasticity/src/lib.rs    117-183, 197-381
//   crates/tpt-fem-assembly/src/lib.rs      27-96, 336-667
//   crates/tpt-fem-sparse/src/lib.rs        114-278
//
// The reference's dense LU lives in the un-vendored crate
// tpt-math-linalg-dense 0.1.0 (called at crates/tpt-fem-sparse/src/lib.rs:268-274);
// a textbook partial-pivot LU stands in for it here.  Below the 1e-9..1e-10
// tolerances of the reference's own solve tests that LU is parity-unpinned.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

using std::vector;
typedef int64_t i64;

namespace {

enum Cell { LINE = 1, TRI = 2, QUAD = 3, TET = 4 };

struct OMesh {
  int cell = TET;
  int cdim = 3;  // number of coordinates stored per node
  vector<vector<double>> nodes;
  vector<vector<i64>> elems;
};

// Rust's `Iterator::sum` for f64 starts from -0.0 (std, since 1.82).
double rsum_dot(const vector<double>& a, const vector<double>& b) {
  double s = -0.0;
  size_t n = std::min(a.size(), b.size());
  for (size_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

int ref_dim(int cell) {
  switch (cell) {
    case LINE: return 1;
    case TRI: return 2;
    case QUAD: return 2;
    default: return 3;
  }
}

// ---- quadrature: crates/tpt-fem-quadrature/src/lib.rs ---------------------

// gauss_legendre (lib.rs:118-162)
void gauss_legendre(int order, vector<double>& p, vector<double>& w) {
  switch (order) {
    case 1: p = {0.0}; w = {2.0}; break;
    case 2: p = {-1.0 / std::sqrt(3.0), 1.0 / std::sqrt(3.0)}; w = {1.0, 1.0}; break;
    case 3:
      p = {0.0, -std::sqrt(3.0 / 5.0), std::sqrt(3.0 / 5.0)};
      w = {8.0 / 9.0, 5.0 / 9.0, 5.0 / 9.0};
      break;
    case 4:
      p = {-0.3399810435848563, 0.3399810435848563, -0.8611363115940526, 0.8611363115940526};
      w = {0.6521451548625461, 0.6521451548625461, 0.3478548451374539, 0.3478548451374539};
      break;
    case 5:
      p = {0.0, -0.5384693101056831, 0.5384693101056831, -0.9061798459386640, 0.9061798459386640};
      w = {0.5688888888888889, 0.4786286704993665, 0.4786286704993665, 0.2369268850561891,
           0.2369268850561891};
      break;
    default: p.clear(); w.clear();  // the reference panics here
  }
}

// cell_quad (thermal/src/lib.rs:29-92, identical in elasticity:117-183);
// tensor_square (quadrature:180-191): outer loop a, inner loop b.
bool cell_quad(int cell, int order, vector<vector<double>>& pts, vector<double>& wts) {
  pts.clear(); wts.clear();
  if (cell == LINE) {
    vector<double> p, w; gauss_legendre(order, p, w);
    if (p.empty()) return false;
    for (size_t i = 0; i < p.size(); ++i) { pts.push_back({p[i]}); wts.push_back(w[i]); }
  } else if (cell == TRI) {  // triangle(Degree2), quadrature:223-234
    pts = {{2.0 / 3.0, 1.0 / 6.0}, {1.0 / 6.0, 2.0 / 3.0}, {1.0 / 6.0, 1.0 / 6.0}};
    wts = {1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0};
  } else if (cell == QUAD) {
    vector<double> p, w; gauss_legendre(order, p, w);
    if (p.empty()) return false;
    for (size_t a = 0; a < p.size(); ++a)
      for (size_t b = 0; b < p.size(); ++b) { pts.push_back({p[a], p[b]}); wts.push_back(w[a] * w[b]); }
  } else if (cell == TET) {  // tetrahedron(Degree2), quadrature:282-289; ignores `order`
    const double a = 0.5854101966249685, b = 0.1381966011250105;
    pts = {{a, b, b}, {b, a, b}, {b, b, a}, {b, b, b}};
    wts = {1.0 / 24.0, 1.0 / 24.0, 1.0 / 24.0, 1.0 / 24.0};
  } else {
    return false;
  }
  return true;
}

// ---- reference elements: crates/tpt-fem-element/src/lib.rs ----------------

vector<vector<double>> ref_nodes(int cell) {
  switch (cell) {
    case LINE: return {{-1.0}, {1.0}};
    case TRI: return {{0.0, 0.0}, {1.0, 0.0}, {0.0, 1.0}};
    case QUAD: return {{-1.0, -1.0}, {1.0, -1.0}, {1.0, 1.0}, {-1.0, 1.0}};
    default: return {{0.0, 0.0, 0.0}, {1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
  }
}

vector<double> ref_shape(int cell, const vector<double>& xi) {
  switch (cell) {
    case LINE: { double x = xi[0]; return {(1.0 - x) / 2.0, (1.0 + x) / 2.0}; }
    case TRI: { double x = xi[0], y = xi[1]; return {1.0 - x - y, x, y}; }
    case QUAD: {  // element:135-140
      double x = xi[0], y = xi[1];
      const double s[4] = {-1.0, 1.0, 1.0, -1.0}, t[4] = {-1.0, -1.0, 1.0, 1.0};
      vector<double> r(4);
      for (int i = 0; i < 4; ++i) r[i] = 0.25 * (1.0 + s[i] * x) * (1.0 + t[i] * y);
      return r;
    }
    default: { double x = xi[0], y = xi[1], z = xi[2]; return {1.0 - x - y - z, x, y, z}; }
  }
}

vector<vector<double>> ref_grad(int cell, const vector<double>& xi) {
  switch (cell) {
    case LINE: return {{-0.5}, {0.5}};
    case TRI: return {{-1.0, -1.0}, {1.0, 0.0}, {0.0, 1.0}};
    case QUAD: {  // element:141-153
      double x = xi[0], y = xi[1];
      const double s[4] = {-1.0, 1.0, 1.0, -1.0}, t[4] = {-1.0, -1.0, 1.0, 1.0};
      vector<vector<double>> g(4, vector<double>(2));
      for (int i = 0; i < 4; ++i) {
        g[i][0] = 0.25 * s[i] * (1.0 + t[i] * y);
        g[i][1] = 0.25 * (1.0 + s[i] * x) * t[i];
      }
      return g;
    }
    default: return {{-1.0, -1.0, -1.0}, {1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
  }
}

// mat_det / mat_inv (element:624-680), cofactor formulas in source order.
double mat_det(int n, const vector<double>& m) {
  if (n == 1) return m[0];
  if (n == 2) return m[0] * m[3] - m[1] * m[2];
  return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
         m[2] * (m[3] * m[7] - m[4] * m[6]);
}

vector<double> mat_inv(int n, const vector<double>& m) {
  if (n == 1) return {1.0 / m[0]};
  if (n == 2) {
    double det = m[0] * m[3] - m[1] * m[2];
    double inv = 1.0 / det;
    return {m[3] * inv, -m[1] * inv, -m[2] * inv, m[0] * inv};
  }
  double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
               m[2] * (m[3] * m[7] - m[4] * m[6]);
  double inv = 1.0 / det;
  return {(m[4] * m[8] - m[5] * m[7]) * inv, (m[2] * m[7] - m[1] * m[8]) * inv,
          (m[1] * m[5] - m[2] * m[4]) * inv, (m[5] * m[6] - m[3] * m[8]) * inv,
          (m[0] * m[8] - m[2] * m[6]) * inv, (m[2] * m[3] - m[0] * m[5]) * inv,
          (m[3] * m[7] - m[4] * m[6]) * inv, (m[1] * m[6] - m[0] * m[7]) * inv,
          (m[0] * m[4] - m[1] * m[3]) * inv};
}

struct Map {
  int dim;
  vector<double> jac, inv;
  double det;  // signed, as element:716 stores it; callers take fabs
};

// Map::from_nodes_and_grad (element:702-724): J[p][r] += X_n[p]*dN_n/dxi_r, node by node.
Map map_from(const vector<vector<double>>& phys, const vector<vector<double>>& lg) {
  Map mp;
  int n = (int)lg[0].size();
  mp.dim = n;
  mp.jac.assign(n * n, 0.0);
  for (size_t k = 0; k < phys.size() && k < lg.size(); ++k)
    for (int p = 0; p < n; ++p)
      for (int r = 0; r < n; ++r) mp.jac[p * n + r] += phys[k][p] * lg[k][r];
  mp.det = mat_det(n, mp.jac);
  mp.inv = mat_inv(n, mp.jac);
  return mp;
}

// Map::physical_grad (element:729-740)
vector<double> physical_grad(const Map& mp, const vector<double>& local) {
  int n = mp.dim;
  vector<double> out(n, 0.0);
  for (int i = 0; i < n; ++i) {
    double s = 0.0;
    for (int r = 0; r < n; ++r) s += local[r] * mp.inv[r * n + i];
    out[i] = s;
  }
  return out;
}

vector<vector<double>> elem_phys(const OMesh& m, i64 eid) {
  vector<vector<double>> phys;
  for (i64 nd : m.elems[eid]) phys.push_back(m.nodes[nd]);
  return phys;
}

// ---- thermal: crates/tpt-fem-thermal/src/lib.rs -----------------------------

// poisson_element_matrix (thermal:132-160)
bool poisson_element_matrix(const OMesh& m, i64 eid, double cond, int qo, vector<vector<double>>& k) {
  auto phys = elem_phys(m, eid);
  vector<vector<double>> qp; vector<double> qw;
  if (!cell_quad(m.cell, qo, qp, qw)) return false;
  size_t n = phys.size();
  k.assign(n, vector<double>(n, 0.0));
  for (size_t q = 0; q < qp.size(); ++q) {
    double w = qw[q];
    auto local = ref_grad(m.cell, qp[q]);
    Map mp = map_from(phys, local);
    double det = std::fabs(mp.det);
    vector<vector<double>> g;
    for (auto& l : local) g.push_back(physical_grad(mp, l));
    for (size_t i = 0; i < n; ++i)
      for (size_t j = 0; j < n; ++j) k[i][j] += w * cond * rsum_dot(g[i], g[j]) * det;
  }
  return true;
}

// poisson_source_vector (thermal:163-196) with a source given as a callback
// of the physical quadrature point (or a constant when cb == nullptr).
typedef double (*source_cb)(const double* x, int dim, void* ud);
bool poisson_source_vector(const OMesh& m, i64 eid, double s_const, source_cb cb, void* ud, int qo,
                           vector<double>& f) {
  auto phys = elem_phys(m, eid);
  vector<vector<double>> qp; vector<double> qw;
  if (!cell_quad(m.cell, qo, qp, qw)) return false;
  size_t n = phys.size();
  f.assign(n, 0.0);
  for (size_t q = 0; q < qp.size(); ++q) {
    double w = qw[q];
    auto ns = ref_shape(m.cell, qp[q]);
    auto local = ref_grad(m.cell, qp[q]);
    Map mp = map_from(phys, local);
    double det = std::fabs(mp.det);
    vector<double> x(phys[0].size(), 0.0);
    for (size_t k = 0; k < n; ++k)
      for (size_t d = 0; d < x.size(); ++d) x[d] += ns[k] * phys[k][d];
    double s = cb ? cb(x.data(), (int)x.size(), ud) : s_const;
    for (size_t i = 0; i < n; ++i) f[i] += w * s * ns[i] * det;
  }
  return true;
}

// ---- elasticity: crates/tpt-fem-elasticity/src/lib.rs -----------------------

enum Model { BAR = 0, PLANE_STRESS = 1, PLANE_STRAIN = 2, CONTINUUM3D = 3 };

// constitutive (elasticity:197-238)
bool constitutive(int model, double e, double nu, int dim, vector<vector<double>>& d) {
  if (model == BAR && dim == 1) { d = {{e}}; return true; }
  if (model == PLANE_STRESS && dim == 2) {
    double c = e / (1.0 - nu * nu);
    d = {{c, c * nu, 0.0}, {c * nu, c, 0.0}, {0.0, 0.0, c * (1.0 - nu) / 2.0}};
    return true;
  }
  if (model == PLANE_STRAIN && dim == 2) {
    double c = e / ((1.0 + nu) * (1.0 - 2.0 * nu));
    d = {{c * (1.0 - nu), c * nu, 0.0}, {c * nu, c * (1.0 - nu), 0.0}, {0.0, 0.0, c * (1.0 - 2.0 * nu) / 2.0}};
    return true;
  }
  if (model == CONTINUUM3D && dim == 3) {
    double c = e / ((1.0 + nu) * (1.0 - 2.0 * nu));
    double mm = (1.0 - nu) * c;
    double dd = (1.0 - 2.0 * nu) / 2.0 * c;
    d = {{mm, c * nu, c * nu, 0.0, 0.0, 0.0}, {c * nu, mm, c * nu, 0.0, 0.0, 0.0},
         {c * nu, c * nu, mm, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, dd, 0.0, 0.0},
         {0.0, 0.0, 0.0, 0.0, dd, 0.0},       {0.0, 0.0, 0.0, 0.0, 0.0, dd}};
    return true;
  }
  return false;  // ElasticityError::ModelDimMismatch
}

// b_matrix (elasticity:242-258): Voigt xx,yy,zz,xy,yz,zx with engineering shear.
vector<vector<double>> b_matrix(const vector<double>& g, int dim) {
  if (dim == 1) return {{g[0]}};
  if (dim == 2) return {{g[0], 0.0}, {0.0, g[1]}, {g[1], g[0]}};
  return {{g[0], 0.0, 0.0}, {0.0, g[1], 0.0}, {0.0, 0.0, g[2]},
          {g[1], g[0], 0.0}, {0.0, g[2], g[1]}, {g[2], 0.0, g[0]}};
}

int strain_dim(int dim) { return dim == 1 ? 1 : (dim == 2 ? 3 : 6); }

// elasticity_element_matrix (elasticity:262-309)
bool elasticity_element_matrix(const OMesh& m, i64 eid, int model, double young, double nu, int qo,
                               vector<vector<double>>& k) {
  auto phys = elem_phys(m, eid);
  int dim = ref_dim(m.cell);
  size_t n = phys.size();
  int nstr = strain_dim(dim);
  vector<vector<double>> d;
  if (!constitutive(model, young, nu, dim, d)) return false;
  vector<vector<double>> qp; vector<double> qw;
  if (!cell_quad(m.cell, qo, qp, qw)) return false;
  k.assign(n * dim, vector<double>(n * dim, 0.0));
  for (size_t q = 0; q < qp.size(); ++q) {
    double w = qw[q];
    auto local = ref_grad(m.cell, qp[q]);
    Map mp = map_from(phys, local);
    double det = std::fabs(mp.det);
    vector<vector<vector<double>>> b;
    for (size_t i = 0; i < n; ++i) b.push_back(b_matrix(physical_grad(mp, local[i]), dim));
    for (size_t i = 0; i < n; ++i)
      for (size_t j = 0; j < n; ++j)
        for (int a = 0; a < dim; ++a)
          for (int bb = 0; bb < dim; ++bb) {
            double s = 0.0;
            for (int s_ = 0; s_ < nstr; ++s_)
              for (int t = 0; t < nstr; ++t) s += b[i][s_][a] * d[s_][t] * b[j][t][bb];
            k[i * dim + a][j * dim + bb] += w * det * s;
          }
  }
  return true;
}

// elasticity_body_vector (elasticity:312-348) with the body force given as a
// callback of the physical quadrature point (or a constant when cb == nullptr).
typedef void (*body_cb)(const double* x, int dim, double* out, void* ud);
bool elasticity_body_vector(const OMesh& m, i64 eid, const double* body, body_cb cb, void* ud, int qo,
                            vector<double>& f) {
  auto phys = elem_phys(m, eid);
  int dim = ref_dim(m.cell);
  size_t n = phys.size();
  vector<vector<double>> qp; vector<double> qw;
  if (!cell_quad(m.cell, qo, qp, qw)) return false;
  f.assign(n * dim, 0.0);
  for (size_t q = 0; q < qp.size(); ++q) {
    double w = qw[q];
    auto ns = ref_shape(m.cell, qp[q]);
    auto local = ref_grad(m.cell, qp[q]);
    Map mp = map_from(phys, local);
    double det = std::fabs(mp.det);
    vector<double> x(phys[0].size(), 0.0), bq(3, 0.0);
    const double* b = body;
    if (cb) {
      for (size_t k = 0; k < n; ++k)
        for (size_t d = 0; d < x.size(); ++d) x[d] += ns[k] * phys[k][d];
      cb(x.data(), (int)x.size(), bq.data(), ud);
      b = bq.data();
    }
    for (size_t i = 0; i < n; ++i)
      for (int a = 0; a < dim; ++a) f[i * dim + a] += w * ns[i] * b[a] * det;
  }
  return true;
}

// ---- sparse: crates/tpt-fem-sparse/src/lib.rs --------------------------------

struct Coo {
  vector<i64> rows, cols;
  vector<double> vals;
  void push(i64 r, i64 c, double v) { rows.push_back(r); cols.push_back(c); vals.push_back(v); }
};

struct Csr {
  i64 nrows = 0, ncols = 0;
  vector<i64> row_ptrs, col_ind;
  vector<double> values;
};

// Coo::to_csr (sparse:122-175): stable sort by (row, col), then sequential
// left-to-right summation of duplicates in push order.
Csr to_csr(const Coo& c) {
  Csr out;
  size_t n = c.rows.size();
  i64 mr = 0, mc = 0;
  for (size_t i = 0; i < n; ++i) { mr = std::max(mr, c.rows[i]); mc = std::max(mc, c.cols[i]); }
  out.nrows = n ? mr + 1 : 1;  // max over rows chained with 0, plus 1
  out.ncols = n ? mc + 1 : 1;
  vector<i64> perm(n);
  std::iota(perm.begin(), perm.end(), 0);
  std::stable_sort(perm.begin(), perm.end(), [&](i64 a, i64 b) {
    if (c.rows[a] != c.rows[b]) return c.rows[a] < c.rows[b];
    return c.cols[a] < c.cols[b];
  });
  out.row_ptrs.assign(out.nrows + 1, 0);
  size_t k = 0;
  while (k < n) {
    i64 r = c.rows[perm[k]], cc = c.cols[perm[k]];
    double sum = c.vals[perm[k]];
    size_t kk = k + 1;
    while (kk < n && c.rows[perm[kk]] == r && c.cols[perm[kk]] == cc) { sum += c.vals[perm[kk]]; ++kk; }
    out.col_ind.push_back(cc);
    out.values.push_back(sum);
    out.row_ptrs[r + 1] += 1;
    k = kk;
  }
  for (i64 r = 0; r < out.nrows; ++r) out.row_ptrs[r + 1] += out.row_ptrs[r];
  return out;
}

// Csr::matvec (sparse:195-205)
vector<double> matvec(const Csr& a, const double* x, i64 xlen) {
  vector<double> y(std::max(a.nrows, xlen), 0.0);
  for (i64 r = 0; r < a.nrows; ++r) {
    double s = 0.0;
    for (i64 c = a.row_ptrs[r]; c < a.row_ptrs[r + 1]; ++c) s += a.values[c] * x[a.col_ind[c]];
    y[r] = s;
  }
  return y;
}

// Stand-in for tpt_math_linalg_dense::DMatrix::solve: partial-pivot LU on a
// column-major dense matrix (the fill of sparse:262-268).
bool dense_lu_solve(i64 n, vector<double>& a, vector<double>& b, std::string& err) {
  vector<i64> piv(n);
  for (i64 k = 0; k < n; ++k) {
    i64 p = k;
    double best = std::fabs(a[k + k * n]);
    for (i64 i = k + 1; i < n; ++i) {
      double v = std::fabs(a[i + k * n]);
      if (v > best) { best = v; p = i; }
    }
    if (!(best > 0.0)) { err = "matrix is singular"; return false; }
    piv[k] = p;
    if (p != k) {
      for (i64 j = 0; j < n; ++j) std::swap(a[k + j * n], a[p + j * n]);
      std::swap(b[k], b[p]);
    }
    double akk = a[k + k * n];
    for (i64 i = k + 1; i < n; ++i) a[i + k * n] /= akk;
    for (i64 j = k + 1; j < n; ++j) {
      double akj = a[k + j * n];
      if (akj == 0.0) continue;
      for (i64 i = k + 1; i < n; ++i) a[i + j * n] -= a[i + k * n] * akj;
    }
  }
  for (i64 i = 0; i < n; ++i) {  // forward substitution, unit lower
    double s = b[i];
    for (i64 j = 0; j < i; ++j) s -= a[i + j * n] * b[j];
    b[i] = s;
  }
  for (i64 i = n - 1; i >= 0; --i) {  // back substitution
    double s = b[i];
    for (i64 j = i + 1; j < n; ++j) s -= a[i + j * n] * b[j];
    b[i] = s / a[i + i * n];
  }
  return true;
}

// solve / solve_multi (sparse:225-278): second to_csr, dense fill, LU.
bool solve(const Coo& coo, const vector<double>& rhs, vector<double>& x, std::string& err) {
  Csr csr = to_csr(coo);
  i64 n = csr.nrows;
  if (csr.ncols != n) { err = "solve requires a square matrix"; return false; }
  if ((i64)rhs.size() != n) { err = "rhs length does not match matrix dimension"; return false; }
  if (n > 20000) { err = "dense LU oracle limited to n <= 20000"; return false; }
  vector<double> data((size_t)n * n, 0.0);
  for (i64 r = 0; r < n; ++r)
    for (i64 idx = csr.row_ptrs[r]; idx < csr.row_ptrs[r + 1]; ++idx)
      data[r + csr.col_ind[idx] * n] += csr.values[idx];
  x = rhs;
  return dense_lu_solve(n, data, x, err);
}

struct Reduced {
  Coo kred;
  vector<double> fred;
  vector<i64> free;
};

// reduce_system (assembly:504-535): lifting uses the FIRST bcs entry for a dof.
Reduced reduce_system(const Coo& coo, const vector<double>& rhs, const vector<std::pair<i64, double>>& bcs) {
  i64 n = (i64)rhs.size();
  Csr csr = to_csr(coo);
  std::unordered_set<i64> fixed;
  for (auto& b : bcs) fixed.insert(b.first);
  Reduced red;
  for (i64 i = 0; i < n; ++i) if (!fixed.count(i)) red.free.push_back(i);
  std::unordered_map<i64, i64> free_idx;
  for (size_t k = 0; k < red.free.size(); ++k) free_idx[red.free[k]] = (i64)k;
  red.fred.assign(red.free.size(), 0.0);
  for (i64 fdof : red.free) {
    double r = rhs[fdof];
    if (fdof < csr.nrows) {
      for (i64 c = csr.row_ptrs[fdof]; c < csr.row_ptrs[fdof + 1]; ++c) {
        i64 col = csr.col_ind[c];
        double v = csr.values[c];
        if (fixed.count(col)) {
          double val = 0.0;
          for (auto& b : bcs) if (b.first == col) { val = b.second; break; }
          r -= v * val;
        } else {
          red.kred.push(free_idx[fdof], free_idx[col], v);
        }
      }
    }
    red.fred[free_idx[fdof]] = r;
  }
  return red;
}

// solve_with_dirichlet (assembly:543-559): fixed dofs get the LAST bcs value.
bool solve_with_dirichlet(const Coo& coo, const vector<double>& rhs, const vector<std::pair<i64, double>>& bcs,
                          vector<double>& u, std::string& err) {
  Reduced red = reduce_system(coo, rhs, bcs);
  vector<double> x;
  if (!solve(red.kred, red.fred, x, err)) return false;
  u.assign(rhs.size(), 0.0);
  for (size_t i = 0; i < red.free.size(); ++i) u[red.free[i]] = x[i];
  for (auto& b : bcs) u[b.first] = b.second;
  return true;
}

// ---- assembly: crates/tpt-fem-assembly/src/lib.rs ----------------------------

// assemble / try_assemble (assembly:428-480): zero-skip, element then i then j order.
void scatter_element(Coo& coo, const vector<i64>& en, int dpn, const vector<vector<double>>& k) {
  size_t nd = k.size();
  for (size_t i = 0; i < nd; ++i)
    for (size_t j = 0; j < nd; ++j) {
      double kij = k[i][j];
      if (kij == 0.0) continue;
      i64 gi = en[i / dpn] * dpn + (i64)(i % dpn);
      i64 gj = en[j / dpn] * dpn + (i64)(j % dpn);
      coo.push(gi, gj, kij);
    }
}

struct FaceDef { vector<int> nodes; int face; };

// Face tables (assembly:38-96).
vector<FaceDef> faces_of(int cell) {
  switch (cell) {
    case LINE: return {{{0}, LINE}, {{1}, LINE}};
    case TRI: return {{{1, 2}, LINE}, {{2, 0}, LINE}, {{0, 1}, LINE}};
    case QUAD: return {{{0, 1}, LINE}, {{1, 2}, LINE}, {{2, 3}, LINE}, {{3, 0}, LINE}};
    default: return {{{1, 2, 3}, TRI}, {{0, 2, 3}, TRI}, {{0, 1, 3}, TRI}, {{0, 1, 2}, TRI}};
  }
}

// boundary_faces (assembly:563-583): faces whose sorted node key occurs once.
vector<std::pair<i64, int>> boundary_faces(const OMesh& m) {
  // Counting the sorted node keys by sorting them (rather than the reference's
  // HashMap) gives the same set; the output keeps element-then-face order.
  auto faces = faces_of(m.cell);
  const size_t nf = faces.size(), ne = m.elems.size();
  struct Key { std::array<i64, 4> k; i64 idx; };
  vector<Key> keys(ne * nf);
  for (size_t e = 0; e < ne; ++e)
    for (size_t fi = 0; fi < nf; ++fi) {
      Key& kk = keys[e * nf + fi];
      kk.k.fill(-1);
      size_t q = 0;
      for (int i : faces[fi].nodes) kk.k[q++] = m.elems[e][i];
      std::sort(kk.k.begin(), kk.k.begin() + q);
      kk.idx = (i64)(e * nf + fi);
    }
  std::sort(keys.begin(), keys.end(), [](const Key& a, const Key& b) { return a.k < b.k; });
  vector<char> once(ne * nf, 0);
  for (size_t a = 0; a < keys.size();) {
    size_t b = a + 1;
    while (b < keys.size() && keys[b].k == keys[a].k) ++b;
    if (b - a == 1) once[keys[a].idx] = 1;
    a = b;
  }
  vector<std::pair<i64, int>> out;
  for (size_t e = 0; e < ne; ++e)
    for (size_t fi = 0; fi < nf; ++fi)
      if (once[e * nf + fi]) out.push_back({(i64)e, (int)fi});
  return out;
}

vector<double> mean_of(const vector<vector<double>>& pts) {
  vector<double> m(pts[0].size(), 0.0);
  for (auto& p : pts) for (size_t d = 0; d < p.size(); ++d) m[d] += p[d];
  for (auto& v : m) v /= (double)pts.size();
  return m;
}

double norm_of(const vector<double>& a) { return std::sqrt(rsum_dot(a, a)); }

// surface (assembly:394-420)
void surface(const vector<vector<double>>& tangents, int dim, double& measure, vector<double>& n) {
  if (tangents.size() == 1) {
    auto& t = tangents[0];
    measure = norm_of(t);
    n.assign(dim, 0.0);
    n[0] = -t[1];
    n[1] = t[0];
    double ln = norm_of(n);
    for (auto& v : n) v /= ln;
  } else {
    auto& a = tangents[0]; auto& b = tangents[1];
    vector<double> c = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
    measure = norm_of(c);
    n = c;
    double ln = norm_of(n);
    for (auto& v : n) v /= ln;
  }
}

typedef double (*flux_cb)(const double* x, const double* nrm, int dim, void* ud);

// apply_neumann_order (assembly:601-667). `comp_mask` (bit c set = keep
// component c) lets a caller turn the reference's scalar-tiled flux into a
// vector traction, exactly as a caller of the reference would by discarding
// the unwanted components afterwards.
void apply_neumann(const OMesh& m, int dpn, flux_cb cb, void* ud, double* rhs, int order, unsigned comp_mask) {
  auto faces = faces_of(m.cell);
  for (auto& bf : boundary_faces(m)) {
    i64 eid = bf.first;
    const FaceDef& f = faces[bf.second];
    auto phys = elem_phys(m, eid);
    vector<vector<double>> qp; vector<double> qw;
    cell_quad(f.face, order, qp, qw);
    int dim = (int)phys[0].size();
    auto ec = mean_of(phys);
    vector<vector<double>> fc;
    for (int i : f.nodes) fc.push_back(phys[i]);
    auto fcen = mean_of(fc);
    for (size_t q = 0; q < qp.size(); ++q) {
      double w = qw[q];
      auto ns = ref_shape(f.face, qp[q]);
      auto ng = ref_grad(f.face, qp[q]);
      vector<double> xp(dim, 0.0);
      for (size_t k = 0; k < f.nodes.size(); ++k)
        for (int d = 0; d < dim; ++d) xp[d] += ns[k] * phys[f.nodes[k]][d];
      size_t fd = ng[0].size();
      vector<vector<double>> tangents(fd, vector<double>(dim, 0.0));
      for (size_t mm = 0; mm < fd; ++mm)
        for (size_t k = 0; k < f.nodes.size(); ++k)
          for (int d = 0; d < dim; ++d) tangents[mm][d] += ng[k][mm] * phys[f.nodes[k]][d];
      double measure; vector<double> normal;
      surface(tangents, dim, measure, normal);
      vector<double> dir(dim);
      for (int d = 0; d < dim; ++d) dir[d] = fcen[d] - ec[d];
      if (rsum_dot(normal, dir) < 0.0) for (auto& v : normal) v = -v;
      double g = cb(xp.data(), normal.data(), dim, ud);
      for (size_t k = 0; k < f.nodes.size(); ++k) {
        i64 base = m.elems[eid][f.nodes[k]] * dpn;
        for (int c = 0; c < dpn; ++c)
          if (comp_mask & (1u << c)) rhs[base + c] += w * measure * g * ns[k];
      }
    }
  }
}

// apply_robin_order (assembly:684-753): for every boundary face and face
// quadrature point, h(x, n) N_k N_l is pushed onto `coo` for each pair (k, l)
// of the face's nodes and each component, after whatever `coo` already holds
// (solve_poisson calls it after `assemble`, thermal:235-237).  No zero-skip.
void apply_robin(const OMesh& m, int dpn, flux_cb cb, void* ud, Coo& coo, int order) {
  auto faces = faces_of(m.cell);
  for (auto& bf : boundary_faces(m)) {
    i64 eid = bf.first;
    const FaceDef& f = faces[bf.second];
    auto phys = elem_phys(m, eid);
    vector<vector<double>> qp; vector<double> qw;
    cell_quad(f.face, order, qp, qw);
    int dim = (int)phys[0].size();
    auto ec = mean_of(phys);
    vector<vector<double>> fc;
    for (int i : f.nodes) fc.push_back(phys[i]);
    auto fcen = mean_of(fc);
    for (size_t q = 0; q < qp.size(); ++q) {
      double w = qw[q];
      auto ns = ref_shape(f.face, qp[q]);
      auto ng = ref_grad(f.face, qp[q]);
      vector<double> xp(dim, 0.0);
      for (size_t k = 0; k < f.nodes.size(); ++k)
        for (int d = 0; d < dim; ++d) xp[d] += ns[k] * phys[f.nodes[k]][d];
      size_t fd = ng[0].size();
      vector<vector<double>> tangents(fd, vector<double>(dim, 0.0));
      for (size_t mm = 0; mm < fd; ++mm)
        for (size_t k = 0; k < f.nodes.size(); ++k)
          for (int d = 0; d < dim; ++d) tangents[mm][d] += ng[k][mm] * phys[f.nodes[k]][d];
      double measure; vector<double> normal;
      surface(tangents, dim, measure, normal);
      vector<double> dir(dim);
      for (int d = 0; d < dim; ++d) dir[d] = fcen[d] - ec[d];
      if (rsum_dot(normal, dir) < 0.0) for (auto& v : normal) v = -v;
      double h = cb(xp.data(), normal.data(), dim, ud);
      for (size_t k = 0; k < f.nodes.size(); ++k)
        for (size_t l = 0; l < f.nodes.size(); ++l) {
          i64 bi = m.elems[eid][f.nodes[k]] * dpn, bj = m.elems[eid][f.nodes[l]] * dpn;
          for (int c = 0; c < dpn; ++c) coo.push(bi + c, bj + c, w * measure * h * ns[k] * ns[l]);
        }
    }
  }
}

// Built-in flux: value `val` where the outward normal's `axis` component
// times `sign` exceeds 0.5, zero elsewhere (a traction on one box face).
struct FaceSel { int axis; double sign; double val; };
double facesel_flux(const double*, const double* n, int, void* ud) {
  FaceSel* s = (FaceSel*)ud;
  if (s->axis < 0) return s->val;  // every boundary face
  return (n[s->axis] * s->sign > 0.5) ? s->val : 0.0;
}

// ---- mesh generation: crates/tpt-fem-mesh-gen/src/lib.rs --------------------

double orient3(const double* a, const double* b, const double* c, const double* d) {
  double ab[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  double ac[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
  double ad[3] = {d[0] - a[0], d[1] - a[1], d[2] - a[2]};
  return ab[0] * (ac[1] * ad[2] - ac[2] * ad[1]) - ab[1] * (ac[0] * ad[2] - ac[2] * ad[0]) +
         ab[2] * (ac[0] * ad[1] - ac[1] * ad[0]);
}

}  // namespace

// =============================================================================
// extern "C" surface used by tests/ (ctypes).  Handles are opaque pointers.
// =============================================================================
extern "C" {

struct OrcMesh { OMesh m; };
struct OrcCoo { Coo c; };
struct OrcCsr { Csr c; };
struct OrcReduced { Reduced r; };

static thread_local std::string g_err;
const char* orc_last_error() { return g_err.c_str(); }

// box_mesh (mesh-gen:422-495).  coords: N x 3, conn: E x 4.
void orc_box_mesh_sizes(const i64 n[3], i64* n_nodes, i64* n_elems) {
  *n_nodes = (n[0] + 1) * (n[1] + 1) * (n[2] + 1);
  *n_elems = 6 * n[0] * n[1] * n[2];
}

void orc_box_mesh(const double mn[3], const double mx[3], const i64 n[3], double* coords, i64* conn) {
  i64 nx = n[0], ny = n[1], nz = n[2];
  auto id = [&](i64 i, i64 j, i64 k) { return (i * (ny + 1) + j) * (nz + 1) + k; };
  for (i64 i = 0; i <= nx; ++i)
    for (i64 j = 0; j <= ny; ++j)
      for (i64 k = 0; k <= nz; ++k) {
        double t = nx > 0 ? (double)i / (double)nx : 0.0;
        double u = ny > 0 ? (double)j / (double)ny : 0.0;
        double w = nz > 0 ? (double)k / (double)nz : 0.0;
        double* c = coords + 3 * id(i, j, k);
        c[0] = mn[0] + t * (mx[0] - mn[0]);
        c[1] = mn[1] + u * (mx[1] - mn[1]);
        c[2] = mn[2] + w * (mx[2] - mn[2]);
      }
  // The orientation test evaluates the corners of the first brick (the
  // reference's `corner` closure shadows the loop indices), so it is the
  // same for every brick.
  auto corner = [&](i64 i, i64 j, i64 k, double* o) {
    double t = nx > 0 ? (double)i / (double)nx : 0.0;
    double u = ny > 0 ? (double)j / (double)ny : 0.0;
    double w = nz > 0 ? (double)k / (double)nz : 0.0;
    o[0] = mn[0] + t * (mx[0] - mn[0]);
    o[1] = mn[1] + u * (mx[1] - mn[1]);
    o[2] = mn[2] + w * (mx[2] - mn[2]);
  };
  static const int cof[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  static const int tets[6][4] = {{0, 1, 2, 6}, {0, 2, 3, 6}, {0, 3, 7, 6},
                                 {0, 7, 4, 6}, {0, 4, 5, 6}, {0, 5, 1, 6}};
  double co[8][3];
  for (int c = 0; c < 8; ++c) corner(cof[c][0], cof[c][1], cof[c][2], co[c]);
  bool swap[6];
  for (int t = 0; t < 6; ++t)
    swap[t] = orient3(co[tets[t][0]], co[tets[t][1]], co[tets[t][2]], co[tets[t][3]]) < 0.0;
  i64 e = 0;
  for (i64 i = 0; i < nx; ++i)
    for (i64 j = 0; j < ny; ++j)
      for (i64 k = 0; k < nz; ++k) {
        i64 idc[8];
        for (int c = 0; c < 8; ++c) idc[c] = id(i + cof[c][0], j + cof[c][1], k + cof[c][2]);
        for (int t = 0; t < 6; ++t) {
          i64 tv[4] = {idc[tets[t][0]], idc[tets[t][1]], idc[tets[t][2]], idc[tets[t][3]]};
          if (swap[t]) std::swap(tv[1], tv[2]);
          for (int q = 0; q < 4; ++q) conn[4 * e + q] = tv[q];
          ++e;
        }
      }
}

OrcMesh* orc_mesh_new(int cell, int cdim, const double* coords, i64 n_nodes, const i64* conn, i64 n_elems, int npe) {
  OrcMesh* h = new OrcMesh;
  h->m.cell = cell;
  h->m.cdim = cdim;
  h->m.nodes.resize(n_nodes);
  for (i64 i = 0; i < n_nodes; ++i) h->m.nodes[i].assign(coords + cdim * i, coords + cdim * (i + 1));
  h->m.elems.resize(n_elems);
  for (i64 e = 0; e < n_elems; ++e) h->m.elems[e].assign(conn + npe * e, conn + npe * (e + 1));
  return h;
}
void orc_mesh_free(OrcMesh* h) { delete h; }

// Single-element kernels (the closures handed to `assemble`).
int orc_poisson_element_matrix(OrcMesh* h, i64 eid, double k, int qo, double* out) {
  vector<vector<double>> ke;
  if (!poisson_element_matrix(h->m, eid, k, qo, ke)) return 1;
  size_t n = ke.size();
  for (size_t i = 0; i < n; ++i) for (size_t j = 0; j < n; ++j) out[i * n + j] = ke[i][j];
  return 0;
}
int orc_elasticity_element_matrix(OrcMesh* h, i64 eid, int model, double E, double nu, int qo, double* out) {
  vector<vector<double>> ke;
  if (!elasticity_element_matrix(h->m, eid, model, E, nu, qo, ke)) return 1;
  size_t n = ke.size();
  for (size_t i = 0; i < n; ++i) for (size_t j = 0; j < n; ++j) out[i * n + j] = ke[i][j];
  return 0;
}

// assemble(mesh, 1, |e| poisson_element_matrix(mesh, e, k[e], qo)).
// `k` holds one value per element, or one value if k_per_elem == 0.
OrcCoo* orc_assemble_poisson(OrcMesh* h, const double* k, int k_per_elem, int qo) {
  OrcCoo* c = new OrcCoo;
  vector<vector<double>> ke;
  for (size_t e = 0; e < h->m.elems.size(); ++e) {
    if (!poisson_element_matrix(h->m, (i64)e, k[k_per_elem ? e : 0], qo, ke)) { delete c; g_err = "bad quadrature order"; return nullptr; }
    scatter_element(c->c, h->m.elems[e], 1, ke);
  }
  return c;
}

// try_assemble(mesh, dim, |e| elasticity_element_matrix(mesh, e, model, E[e], nu, qo)).
OrcCoo* orc_assemble_elasticity(OrcMesh* h, int model, const double* E, int e_per_elem, double nu, int qo) {
  OrcCoo* c = new OrcCoo;
  int dim = ref_dim(h->m.cell);
  vector<vector<double>> ke;
  for (size_t e = 0; e < h->m.elems.size(); ++e) {
    if (!elasticity_element_matrix(h->m, (i64)e, model, E[e_per_elem ? e : 0], nu, qo, ke)) {
      delete c; g_err = "elasticity model/dimension mismatch"; return nullptr;
    }
    scatter_element(c->c, h->m.elems[e], dim, ke);
  }
  return c;
}

// assemble(mesh, dpn, closure) with the closure's matrices given explicitly
// (n_elems blocks of nd x nd, nd = nodes_per_elem * dpn).
OrcCoo* orc_assemble_given(OrcMesh* h, int dpn, const double* mats) {
  OrcCoo* c = new OrcCoo;
  size_t npe = h->m.elems.empty() ? 0 : h->m.elems[0].size();
  size_t nd = npe * dpn;
  vector<vector<double>> ke(nd, vector<double>(nd));
  for (size_t e = 0; e < h->m.elems.size(); ++e) {
    for (size_t i = 0; i < nd; ++i) for (size_t j = 0; j < nd; ++j) ke[i][j] = mats[e * nd * nd + i * nd + j];
    scatter_element(c->c, h->m.elems[e], dpn, ke);
  }
  return c;
}

// Selected rows of Coo::to_csr(assemble(...)) (sparse:122-175 over
// assembly:428-480) for meshes too large to hold the whole COO.  The triplets
// that global row r receives are the zero-skipped entries of local row r of
// each element containing r's node, pushed in element id order and, within an
// element, in local column order (scatter_element above).  The stable sort by
// (row, col) keeps that push order among equal columns, so sorting one row's
// triplets stably by column and summing equal columns left to right gives
// exactly that row of the CSR.  kind 0: poisson_element_matrix (coef = k);
// kind 1: elasticity_element_matrix (coef = E, with model and nu).  coef holds
// one value per element, or one value if coef_per_elem == 0.  Rows are
// independent, so they are computed in parallel.
struct OrcRows { vector<i64> ptr, cols; vector<double> vals; };

OrcRows* orc_csr_rows(OrcMesh* h, int kind, int model, const double* coef, int coef_per_elem, double nu, int qo,
                      const i64* rows, i64 nrows) {
  const OMesh& m = h->m;
  const int dpn = kind == 0 ? 1 : ref_dim(m.cell);
  const i64 nn = (i64)m.nodes.size();
  vector<char> need(nn, 0);
  for (i64 k = 0; k < nrows; ++k) {
    if (rows[k] < 0 || rows[k] / dpn >= nn) { g_err = "row outside the mesh"; return nullptr; }
    need[rows[k] / dpn] = 1;
  }
  vector<vector<i64>> inc(nn);
  for (size_t e = 0; e < m.elems.size(); ++e)
    for (i64 nd : m.elems[e]) if (need[nd]) inc[nd].push_back((i64)e);
  vector<vector<std::pair<i64, double>>> out(nrows);
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(| : bad)
  for (i64 k = 0; k < nrows; ++k) {
    const i64 node = rows[k] / dpn, comp = rows[k] % dpn;
    vector<std::pair<i64, double>> t;
    vector<vector<double>> ke;
    for (i64 e : inc[node]) {
      const double c = coef[coef_per_elem ? e : 0];
      const bool ok = kind == 0 ? poisson_element_matrix(m, e, c, qo, ke)
                                : elasticity_element_matrix(m, e, model, c, nu, qo, ke);
      if (!ok) { bad = 1; break; }
      const vector<i64>& en = m.elems[e];
      for (size_t a = 0; a < en.size(); ++a) {
        if (en[a] != node) continue;
        const size_t i = a * dpn + (size_t)comp;
        for (size_t j = 0; j < ke[i].size(); ++j) {
          const double kij = ke[i][j];
          if (kij == 0.0) continue;
          t.push_back({en[j / dpn] * dpn + (i64)(j % dpn), kij});
        }
      }
    }
    std::stable_sort(t.begin(), t.end(), [](const std::pair<i64, double>& x, const std::pair<i64, double>& y) {
      return x.first < y.first;
    });
    for (size_t q = 0; q < t.size();) {
      double sum = t[q].second;
      size_t qq = q + 1;
      while (qq < t.size() && t[qq].first == t[q].first) sum += t[qq++].second;
      out[k].push_back({t[q].first, sum});
      q = qq;
    }
  }
  if (bad) { g_err = "element matrix failed (quadrature order or model)"; return nullptr; }
  OrcRows* r = new OrcRows;
  r->ptr.assign(nrows + 1, 0);
  for (i64 k = 0; k < nrows; ++k) {
    r->ptr[k + 1] = r->ptr[k] + (i64)out[k].size();
    for (auto& p : out[k]) { r->cols.push_back(p.first); r->vals.push_back(p.second); }
  }
  return r;
}
i64 orc_rows_nnz(OrcRows* r) { return (i64)r->cols.size(); }
void orc_rows_copy(OrcRows* r, i64* ptr, i64* cols, double* vals) {
  std::memcpy(ptr, r->ptr.data(), r->ptr.size() * sizeof(i64));
  if (!r->cols.empty()) {
    std::memcpy(cols, r->cols.data(), r->cols.size() * sizeof(i64));
    std::memcpy(vals, r->vals.data(), r->vals.size() * sizeof(double));
  }
}
void orc_rows_free(OrcRows* r) { delete r; }

// Selected nodes of the Poisson load loop of solve_poisson (thermal:224-230):
// rhs[node] receives f_e[i] of every element containing it, in element id
// order, starting from 0.0 -- the same additions the whole loop makes on that
// entry.  Source constant s.
int orc_load_poisson_rows(OrcMesh* h, double s, int qo, const i64* nodes, i64 n, double* out) {
  const OMesh& m = h->m;
  const i64 nn = (i64)m.nodes.size();
  vector<i64> slot(nn, -1);
  for (i64 k = 0; k < n; ++k) {
    if (nodes[k] < 0 || nodes[k] >= nn) { g_err = "node outside the mesh"; return 1; }
    slot[nodes[k]] = k;
  }
  vector<double> acc(n, 0.0), f;
  for (size_t e = 0; e < m.elems.size(); ++e) {
    bool hit = false;
    for (i64 nd : m.elems[e]) hit |= slot[nd] >= 0;
    if (!hit) continue;
    if (!poisson_source_vector(m, (i64)e, s, nullptr, nullptr, qo, f)) { g_err = "bad quadrature order"; return 1; }
    for (size_t i = 0; i < m.elems[e].size(); ++i)
      if (slot[m.elems[e][i]] >= 0) acc[slot[m.elems[e][i]]] += f[i];
  }
  for (i64 k = 0; k < n; ++k) out[k] = acc[slot[nodes[k]]];
  return 0;
}

OrcCoo* orc_coo_new() { return new OrcCoo; }
void orc_coo_push(OrcCoo* c, i64 r, i64 col, double v) { c->c.push(r, col, v); }
i64 orc_coo_len(OrcCoo* c) { return (i64)c->c.rows.size(); }
void orc_coo_copy(OrcCoo* c, i64* rows, i64* cols, double* vals) {
  size_t n = c->c.rows.size();
  if (n == 0) return;
  std::memcpy(rows, c->c.rows.data(), n * sizeof(i64));
  std::memcpy(cols, c->c.cols.data(), n * sizeof(i64));
  std::memcpy(vals, c->c.vals.data(), n * sizeof(double));
}
void orc_coo_free(OrcCoo* c) { delete c; }

OrcCsr* orc_to_csr(OrcCoo* c) { OrcCsr* o = new OrcCsr; o->c = to_csr(c->c); return o; }
void orc_csr_dims(OrcCsr* a, i64* nrows, i64* ncols, i64* nnz) {
  *nrows = a->c.nrows; *ncols = a->c.ncols; *nnz = (i64)a->c.values.size();
}
void orc_csr_copy(OrcCsr* a, i64* row_ptrs, i64* col_ind, double* values) {
  std::memcpy(row_ptrs, a->c.row_ptrs.data(), (a->c.nrows + 1) * sizeof(i64));
  size_t nnz = a->c.values.size();
  if (nnz) {
    std::memcpy(col_ind, a->c.col_ind.data(), nnz * sizeof(i64));
    std::memcpy(values, a->c.values.data(), nnz * sizeof(double));
  }
}
OrcCsr* orc_csr_from_arrays(i64 nrows, i64 ncols, const i64* row_ptrs, const i64* col_ind, const double* values) {
  OrcCsr* o = new OrcCsr;
  o->c.nrows = nrows; o->c.ncols = ncols;
  o->c.row_ptrs.assign(row_ptrs, row_ptrs + nrows + 1);
  i64 nnz = row_ptrs[nrows];
  o->c.col_ind.assign(col_ind, col_ind + nnz);
  o->c.values.assign(values, values + nnz);
  return o;
}
void orc_csr_free(OrcCsr* a) { delete a; }

// Csr::matvec; y must hold max(nrows, xlen) entries.
void orc_csr_matvec(OrcCsr* a, const double* x, i64 xlen, double* y) {
  auto v = matvec(a->c, x, xlen);
  std::memcpy(y, v.data(), v.size() * sizeof(double));
}

// Poisson load loop of solve_poisson (thermal:224-230).
int orc_load_poisson_source(OrcMesh* h, double s, int qo, double* rhs) {
  vector<double> f;
  for (size_t e = 0; e < h->m.elems.size(); ++e) {
    if (!poisson_source_vector(h->m, (i64)e, s, nullptr, nullptr, qo, f)) return 1;
    for (size_t i = 0; i < h->m.elems[e].size(); ++i) rhs[h->m.elems[e][i]] += f[i];
  }
  return 0;
}
int orc_load_poisson_source_cb(OrcMesh* h, source_cb cb, void* ud, int qo, double* rhs) {
  vector<double> f;
  for (size_t e = 0; e < h->m.elems.size(); ++e) {
    if (!poisson_source_vector(h->m, (i64)e, 0.0, cb, ud, qo, f)) return 1;
    for (size_t i = 0; i < h->m.elems[e].size(); ++i) rhs[h->m.elems[e][i]] += f[i];
  }
  return 0;
}

// Body-force load loop of solve_elasticity (elasticity:371-379).
int orc_load_body(OrcMesh* h, const double* body, int qo, double* rhs) {
  int dim = ref_dim(h->m.cell);
  vector<double> f;
  for (size_t e = 0; e < h->m.elems.size(); ++e) {
    if (!elasticity_body_vector(h->m, (i64)e, body, nullptr, nullptr, qo, f)) return 1;
    for (size_t i = 0; i < h->m.elems[e].size(); ++i)
      for (int a = 0; a < dim; ++a) rhs[h->m.elems[e][i] * dim + a] += f[i * dim + a];
  }
  return 0;
}

// The same with a body-force callback of the quadrature point.
int orc_load_body_cb(OrcMesh* h, body_cb cb, void* ud, int qo, double* rhs) {
  int dim = ref_dim(h->m.cell);
  vector<double> f;
  for (size_t e = 0; e < h->m.elems.size(); ++e) {
    if (!elasticity_body_vector(h->m, (i64)e, nullptr, cb, ud, qo, f)) return 1;
    for (size_t i = 0; i < h->m.elems[e].size(); ++i)
      for (int a = 0; a < dim; ++a) rhs[h->m.elems[e][i] * dim + a] += f[i * dim + a];
  }
  return 0;
}

// apply_neumann_order with a caller flux callback.
void orc_apply_neumann_cb(OrcMesh* h, int dpn, flux_cb cb, void* ud, int order, unsigned comp_mask, double* rhs) {
  apply_neumann(h->m, dpn, cb, ud, rhs, order, comp_mask);
}
// apply_neumann_order with the built-in face-selector flux (traction t on the
// faces whose outward normal satisfies sign*n[axis] > 0.5), applied to the
// components in comp_mask.
void orc_apply_traction(OrcMesh* h, int dpn, int axis, double sign, double val, unsigned comp_mask, double* rhs) {
  FaceSel s{axis, sign, val};
  apply_neumann(h->m, dpn, facesel_flux, &s, rhs, 2, comp_mask);
}
// apply_robin_order with the built-in face selector (axis < 0: every boundary face).
void orc_apply_robin(OrcCoo* c, OrcMesh* h, int dpn, int axis, double sign, double val) {
  FaceSel s{axis, sign, val};
  apply_robin(h->m, dpn, facesel_flux, &s, c->c, 2);
}
void orc_apply_robin_cb(OrcCoo* c, OrcMesh* h, int dpn, flux_cb cb, void* ud, int order) {
  apply_robin(h->m, dpn, cb, ud, c->c, order);
}
i64 orc_boundary_face_count(OrcMesh* h) { return (i64)boundary_faces(h->m).size(); }

OrcReduced* orc_reduce_system(OrcCoo* c, const double* rhs, i64 n, const i64* bc_dof, const double* bc_val, i64 nbc) {
  vector<std::pair<i64, double>> bcs;
  for (i64 i = 0; i < nbc; ++i) bcs.push_back({bc_dof[i], bc_val[i]});
  OrcReduced* r = new OrcReduced;
  r->r = reduce_system(c->c, vector<double>(rhs, rhs + n), bcs);
  return r;
}
i64 orc_reduced_nfree(OrcReduced* r) { return (i64)r->r.free.size(); }
OrcCoo* orc_reduced_kred(OrcReduced* r) { OrcCoo* c = new OrcCoo; c->c = r->r.kred; return c; }
void orc_reduced_copy(OrcReduced* r, double* fred, i64* free) {
  size_t n = r->r.free.size();
  if (!n) return;
  std::memcpy(fred, r->r.fred.data(), n * sizeof(double));
  std::memcpy(free, r->r.free.data(), n * sizeof(i64));
}
void orc_reduced_free(OrcReduced* r) { delete r; }

int orc_solve(OrcCoo* c, const double* rhs, i64 n, double* x) {
  vector<double> xs;
  if (!solve(c->c, vector<double>(rhs, rhs + n), xs, g_err)) return 1;
  std::memcpy(x, xs.data(), xs.size() * sizeof(double));
  return 0;
}

int orc_solve_with_dirichlet(OrcCoo* c, const double* rhs, i64 n, const i64* bc_dof, const double* bc_val, i64 nbc,
                             double* u) {
  vector<std::pair<i64, double>> bcs;
  for (i64 i = 0; i < nbc; ++i) bcs.push_back({bc_dof[i], bc_val[i]});
  vector<double> us;
  if (!solve_with_dirichlet(c->c, vector<double>(rhs, rhs + n), bcs, us, g_err)) return 1;
  std::memcpy(u, us.data(), us.size() * sizeof(double));
  return 0;
}

// ---- CPU Jacobi-PCG ------------------------------------------------------------
// NOT reference code: the reference has no iterative solver.  This is the CPU
// restatement of the plain method the GPU library runs, FP64 Jacobi-PCG, used
// as the oracle for large systems and as the timed CPU baseline.  Like the GPU
// solver it stops on the TRUE relative residual ||b - A x||_2 / ||b||_2 <= tol:
// the recursion runs until its updated residual meets tol, then the true
// residual is computed, and if that still exceeds tol the recursion restarts
// from it (at most 8 restarts).  `nthreads` <= 0 uses every OpenMP thread.
// Returns the total iterations, negated when max_it was reached first;
// *relres gets the true final relative residual.
}  // extern "C"
template <typename I>
i64 pcg_jacobi(i64 n, const I* rp, const I* ci, const double* va, const double* b, double* x, double tol, i64 max_it,
               int nthreads, double* relres) {
#ifdef _OPENMP
  // every call sets its own team size, so a one-thread call leaves no residue
  omp_set_num_threads(nthreads > 0 ? nthreads : omp_get_num_procs());
#endif
  vector<double> r(n), z(n), p(n), q(n), dinv(n);
  double bb = 0.0;
#pragma omp parallel for reduction(+ : bb) schedule(static)
  for (i64 i = 0; i < n; ++i) {
    double d = 0.0;
    for (i64 k = rp[i]; k < rp[i + 1]; ++k) if ((i64)ci[k] == i) d += va[k];
    dinv[i] = 1.0 / d;
    x[i] = 0.0;
    r[i] = b[i];
    bb += b[i] * b[i];
  }
  const double bnorm = std::sqrt(bb);
  if (bnorm == 0.0) { if (relres) *relres = 0.0; return 0; }
  i64 it = 0;
  double res = bb;
  for (int restart = 0;; ++restart) {
    double rz = 0.0, rr = 0.0;
#pragma omp parallel for reduction(+ : rz, rr) schedule(static)
    for (i64 i = 0; i < n; ++i) {
      z[i] = dinv[i] * r[i];
      p[i] = z[i];
      rz += r[i] * z[i];
      rr += r[i] * r[i];
    }
    while (std::sqrt(rr) > tol * bnorm && it < max_it) {
      double pq = 0.0;
#pragma omp parallel for reduction(+ : pq) schedule(static)
      for (i64 i = 0; i < n; ++i) {
        double s = 0.0;
        for (i64 k = rp[i]; k < rp[i + 1]; ++k) s += va[k] * p[ci[k]];
        q[i] = s;
        pq += p[i] * s;
      }
      const double alpha = rz / pq;
      double rz_new = 0.0, rr_new = 0.0;
#pragma omp parallel for reduction(+ : rz_new, rr_new) schedule(static)
      for (i64 i = 0; i < n; ++i) {
        x[i] += alpha * p[i];
        r[i] -= alpha * q[i];
        z[i] = dinv[i] * r[i];
        rz_new += r[i] * z[i];
        rr_new += r[i] * r[i];
      }
      const double beta = rz_new / rz;
      rz = rz_new;
      rr = rr_new;
#pragma omp parallel for schedule(static)
      for (i64 i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
      ++it;
    }
    res = 0.0;
#pragma omp parallel for reduction(+ : res) schedule(static)
    for (i64 i = 0; i < n; ++i) {
      double s = 0.0;
      for (i64 k = rp[i]; k < rp[i + 1]; ++k) s += va[k] * x[ci[k]];
      r[i] = b[i] - s;
      res += r[i] * r[i];
    }
    if (std::sqrt(res) <= tol * bnorm || it >= max_it || restart >= 8) break;
  }
  if (relres) *relres = std::sqrt(res) / bnorm;
  return std::sqrt(res) > tol * bnorm ? -it : it;
}
extern "C" {

i64 orc_pcg_jacobi(i64 n, const i64* rp, const i64* ci, const double* va, const double* b, double* x, double tol,
                   i64 max_it, int nthreads, double* relres) {
  return pcg_jacobi<i64>(n, rp, ci, va, b, x, tol, max_it, nthreads, relres);
}
// The same with int32 row pointers and columns (12 bytes per stored entry
// instead of 16: the form a tuned CPU solver would use).
i64 orc_pcg_jacobi_i32(i64 n, const int32_t* rp, const int32_t* ci, const double* va, const double* b, double* x,
                       double tol, i64 max_it, int nthreads, double* relres) {
  return pcg_jacobi<int32_t>(n, rp, ci, va, b, x, tol, max_it, nthreads, relres);
}

// Map::from_nodes_and_grad at reference point xi (element:702-724).
void orc_map(int cell, const double* X, int npe, int cdim, const double* xi, double* jac, double* det, double* inv) {
  vector<vector<double>> phys(npe);
  for (int k = 0; k < npe; ++k) phys[k].assign(X + k * cdim, X + (k + 1) * cdim);
  int rd = ref_dim(cell);
  Map mp = map_from(phys, ref_grad(cell, vector<double>(xi, xi + rd)));
  for (int i = 0; i < rd * rd; ++i) { jac[i] = mp.jac[i]; inv[i] = mp.inv[i]; }
  *det = mp.det;
}

// cell_quad points/weights (thermal:29-92); returns the point count.
int orc_cell_quad(int cell, int order, double* pts, double* w) {
  vector<vector<double>> p; vector<double> ww;
  if (!cell_quad(cell, order, p, ww)) return 0;
  int rd = ref_dim(cell);
  for (size_t q = 0; q < p.size(); ++q) {
    for (int d = 0; d < rd; ++d) pts[q * rd + d] = p[q][d];
    w[q] = ww[q];
  }
  return (int)p.size();
}

// ---- classic FSAI ----------------------------------------------------------------
// NOT reference code (the reference has no iterative solver): CPU restatement
// of Kolotilina-Yeremin FSAI on the lower-triangular pattern, the checker for
// the device factor.  Row i: P = { j <= i in row i }, solve A[P,P] y = e_last
// by dense Cholesky, G[i,P] = y / sqrt(y_last).  Returns nullptr when a
// principal block is not positive definite.
// lrp/lci: the strictly-lower pattern of each row (nullptr: tril(A) minus the
// diagonal).  Output: CSR of G itself (pattern + diagonal, values y/sqrt(y_i)).
OrcCsr* orc_fsai(i64 n, const i64* rp, const i64* ci, const double* va, const i64* lrp, const i64* lci) {
  OrcCsr* o = new OrcCsr;
  o->c.nrows = n; o->c.ncols = n;
  o->c.row_ptrs.assign(n + 1, 0);
  auto lookup = [&](i64 r, i64 c) {
    const i64* b = ci + rp[r];
    const i64* e = ci + rp[r + 1];
    const i64* it = std::lower_bound(b, e, c);
    return (it != e && *it == c) ? va[rp[r] + (it - b)] : 0.0;
  };
  for (i64 i = 0; i < n; ++i) {
    vector<i64> P;
    if (lrp) {
      for (i64 k = lrp[i]; k < lrp[i + 1]; ++k) P.push_back(lci[k]);
    } else {
      for (i64 k = rp[i]; k < rp[i + 1]; ++k) if (ci[k] < i) P.push_back(ci[k]);
    }
    P.push_back(i);
    size_t m = P.size();
    vector<double> L(m * m, 0.0);
    for (size_t a = 0; a < m; ++a)
      for (size_t b = 0; b <= a; ++b) L[a * m + b] = lookup(P[a], P[b]);
    for (size_t a = 0; a < m; ++a)
      for (size_t b = 0; b <= a; ++b) {
        double s = L[a * m + b];
        for (size_t t = 0; t < b; ++t) s -= L[a * m + t] * L[b * m + t];
        if (a == b) {
          if (!(s > 0.0)) { delete o; g_err = "FSAI block not positive definite"; return nullptr; }
          L[a * m + a] = std::sqrt(s);
        } else {
          L[a * m + b] = s / L[b * m + b];
        }
      }
    vector<double> y(m, 0.0);
    y[m - 1] = 1.0 / L[(m - 1) * m + (m - 1)];
    for (i64 a = (i64)m - 1; a >= 0; --a) {
      double s = y[a];
      for (size_t t = a + 1; t < m; ++t) s -= L[t * m + a] * y[t];
      y[a] = s / L[a * m + a];
    }
    double sc = 1.0 / std::sqrt(y[m - 1]);
    for (size_t a = 0; a < m; ++a) { o->c.col_ind.push_back(P[a]); o->c.values.push_back(y[a] * sc); }
    o->c.row_ptrs[i + 1] = (i64)o->c.col_ind.size();
  }
  return o;
}

int orc_max_threads() {
#ifdef _OPENMP
  return omp_get_num_procs();
#else
  return 1;
#endif
}

}  // extern "C"

// ---- topology optimisation: crates/tpt-fem-topopt/src/lib.rs -----------------
//
// Restatement of topopt_simp (topopt:342-385) and its helpers, plus a second
// mode with the density filter and the OC loop of the published 88-line SIMP
// code (Andreassen, Clausen, Schevenels, Lazarov, Sigmund, Struct. Multidisc.
// Optim. 43 (2011) 1-16), which the reference does not have.  The solve is
// either the reference's own path (solve_with_dirichlet: reduce, CSR, dense LU)
// or a banded Cholesky of the same reduced matrix in y-fastest node order
// (for grids where an n^2 dense matrix is out of reach).
namespace {

const double TOPO_RHO_MIN = 1e-3, TOPO_RHO_MAX = 1.0, TOPO_OC_DAMP = 0.5;  // topopt:54-62

// element_stiffness_unit (topopt:166-217), E = 1, 2x2 Gauss, square of side h.
vector<double> topo_ke0(double nu, double h) {
  const double c = 1.0 / (1.0 - nu * nu);
  const double d[3][3] = {{c, c * nu, 0.0}, {c * nu, c, 0.0}, {0.0, 0.0, c * (1.0 - nu) / 2.0}};
  vector<double> p, w;
  gauss_legendre(2, p, w);
  const double jdet = h * h / 4.0;
  const double scale = 2.0 / h;
  vector<double> ke(64, 0.0);
  for (size_t a = 0; a < p.size(); ++a)
    for (size_t b = 0; b < p.size(); ++b) {
      vector<double> xi = {p[a], p[b]};
      const double wt = w[a] * w[b];
      vector<vector<double>> dn = ref_grad(QUAD, xi);
      double bm[3][8] = {{0}};
      for (int n = 0; n < 4; ++n) {
        const double nx_ = scale * dn[n][0], ny_ = scale * dn[n][1];
        bm[0][2 * n] = nx_;
        bm[1][2 * n + 1] = ny_;
        bm[2][2 * n] = ny_;
        bm[2][2 * n + 1] = nx_;
      }
      double db[3][8];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 8; ++j) {
          double s = 0.0;
          for (int k = 0; k < 3; ++k) s += d[i][k] * bm[k][j];
          db[i][j] = s;
        }
      for (int i = 0; i < 8; ++i)
        for (int j = 0; j < 8; ++j) {
          double s = 0.0;
          for (int k = 0; k < 3; ++k) s += bm[k][i] * db[k][j];
          ke[i * 8 + j] += wt * jdet * s;
        }
    }
  return ke;
}

struct TopoGrid {  // Grid::new(nelx + 1, nely + 1, h) (topopt:89-116)
  i64 nx, ny, nelx, nely;
  double h;
  i64 n_elem() const { return nelx * nely; }
  void nodes(i64 e, i64 out[4]) const {
    const i64 ei = e % nelx, ej = e / nelx;
    out[0] = ej * nx + ei;
    out[1] = ej * nx + ei + 1;
    out[2] = (ej + 1) * nx + ei + 1;
    out[3] = (ej + 1) * nx + ei;
  }
  void center(i64 e, double c[2]) const {
    c[0] = ((double)(e % nelx) + 0.5) * h;
    c[1] = ((double)(e / nelx) + 0.5) * h;
  }
};

// assemble (topopt:220-238): all 64 entries, E(rho) = emin + rho^p (e0 - emin).
Coo topo_assemble(const TopoGrid& g, const vector<double>& rho, const vector<double>& ke0, double e0, double penal,
                  double emin) {
  Coo coo;
  for (i64 e = 0; e < g.n_elem(); ++e) {
    const double er = emin + std::pow(rho[e], penal) * (e0 - emin);
    i64 nd[4];
    g.nodes(e, nd);
    i64 gd[8];
    for (int k = 0; k < 4; ++k) { gd[2 * k] = 2 * nd[k]; gd[2 * k + 1] = 2 * nd[k] + 1; }
    for (int i = 0; i < 8; ++i)
      for (int j = 0; j < 8; ++j) coo.push(gd[i], gd[j], er * ke0[i * 8 + j]);
  }
  return coo;
}

// element_quad_form (topopt:241-254)
double topo_quad_form(const vector<double>& ke0, const vector<double>& u, const i64 nd[4]) {
  double ue[8];
  for (int k = 0; k < 4; ++k) { ue[2 * k] = u[2 * nd[k]]; ue[2 * k + 1] = u[2 * nd[k] + 1]; }
  double s = 0.0;
  for (int i = 0; i < 8; ++i)
    for (int j = 0; j < 8; ++j) s += ue[i] * ke0[i * 8 + j] * ue[j];
  return s;
}

// filter_sensitivity (topopt:259-279).  The reference loops over every element
// f; only f with d^2 <= R^2 contribute, so the loop here visits the window of
// element rows/columns within R (+1) in the same ascending f order.
vector<double> topo_filter_sensitivity(const TopoGrid& g, const vector<double>& raw, double radius) {
  const double r2 = radius * radius;
  const i64 w = (i64)std::floor(radius / g.h) + 1;
  vector<double> out(raw.size(), 0.0);
  for (i64 e = 0; e < g.n_elem(); ++e) {
    double ce[2];
    g.center(e, ce);
    const i64 ei = e % g.nelx, ej = e / g.nelx;
    double num = 0.0, den = 0.0;
    for (i64 fj = std::max<i64>(0, ej - w); fj <= std::min(g.nely - 1, ej + w); ++fj)
      for (i64 fi = std::max<i64>(0, ei - w); fi <= std::min(g.nelx - 1, ei + w); ++fi) {
        const i64 f = fj * g.nelx + fi;
        double cf[2];
        g.center(f, cf);
        const double dx = ce[0] - cf[0], dy = ce[1] - cf[1];
        const double d2 = dx * dx + dy * dy;
        if (d2 <= r2) {
          const double wt = radius - std::sqrt(d2);
          num += wt * raw[f];
          den += wt;
        }
      }
    out[e] = den > 0.0 ? num / den : raw[e];
  }
  return out;
}

// oc_update (topopt:284-331): 60 bisection steps on [1e-9, 1e9].
vector<double> topo_oc_update(const vector<double>& rho, const vector<double>& sens, double vol_frac,
                              double move_limit) {
  const size_t n = rho.size();
  const double target = vol_frac * (double)n;
  vector<double> b(n);
  for (size_t e = 0; e < n; ++e) b[e] = -sens[e];
  auto cand = [&](size_t e, double lambda) {
    const double ratio = b[e] > 0.0 ? std::pow(b[e] / lambda, TOPO_OC_DAMP) : 0.0;
    const double c = rho[e] * ratio;
    const double lo = std::max(rho[e] - move_limit, TOPO_RHO_MIN), hi = std::min(rho[e] + move_limit, TOPO_RHO_MAX);
    return std::min(std::max(c, lo), hi);  // f64::clamp(lo, hi), lo <= hi here
  };
  double lo = 1e-9, hi = 1e9, lambda = 1.0;
  for (int it = 0; it < 60; ++it) {
    lambda = 0.5 * (lo + hi);
    double sum = 0.0;
    for (size_t e = 0; e < n; ++e) sum += cand(e, lambda);
    if (sum > target) lo = lambda; else hi = lambda;
  }
  vector<double> out(n);
  for (size_t e = 0; e < n; ++e) out[e] = cand(e, lambda);
  return out;
}

// Density filter of the 88-line code: y = H x / Hs, H_ef = max(0, rmin - d_ef).
void topo_density_filter(const TopoGrid& g, double rmin, const vector<double>& x, vector<double>& y,
                         const vector<double>* scale_in = nullptr) {
  const i64 w = (i64)std::ceil(rmin / g.h);
  y.assign(x.size(), 0.0);
  for (i64 e = 0; e < g.n_elem(); ++e) {
    const i64 ei = e % g.nelx, ej = e / g.nelx;
    double ce[2];
    g.center(e, ce);
    double num = 0.0, den = 0.0;
    for (i64 fj = std::max<i64>(0, ej - w); fj <= std::min(g.nely - 1, ej + w); ++fj)
      for (i64 fi = std::max<i64>(0, ei - w); fi <= std::min(g.nelx - 1, ei + w); ++fi) {
        const i64 f = fj * g.nelx + fi;
        double cf[2];
        g.center(f, cf);
        const double dx = ce[0] - cf[0], dy = ce[1] - cf[1];
        const double wt = std::max(0.0, rmin - std::sqrt(dx * dx + dy * dy));
        num += wt * (scale_in ? x[f] / (*scale_in)[f] : x[f]);
        den += wt;
      }
    y[e] = scale_in ? num : num / den;
  }
}

vector<double> topo_filter_weight_sums(const TopoGrid& g, double rmin) {
  vector<double> ones(g.n_elem(), 1.0), hs;
  const i64 w = (i64)std::ceil(rmin / g.h);
  hs.assign(g.n_elem(), 0.0);
  for (i64 e = 0; e < g.n_elem(); ++e) {
    const i64 ei = e % g.nelx, ej = e / g.nelx;
    double ce[2];
    g.center(e, ce);
    double den = 0.0;
    for (i64 fj = std::max<i64>(0, ej - w); fj <= std::min(g.nely - 1, ej + w); ++fj)
      for (i64 fi = std::max<i64>(0, ei - w); fi <= std::min(g.nelx - 1, ei + w); ++fi) {
        double cf[2];
        g.center(fj * g.nelx + fi, cf);
        const double dx = ce[0] - cf[0], dy = ce[1] - cf[1];
        den += std::max(0.0, rmin - std::sqrt(dx * dx + dy * dy));
      }
    hs[e] = den;
  }
  return hs;
}

// Reduced solve by banded Cholesky: free dofs renumbered y-fastest
// (node (i, j) -> i * ny + j), band stored row-wise as A[r][r - c], c <= r.
bool topo_banded_solve(const TopoGrid& g, const Coo& coo, const vector<double>& f,
                       const vector<std::pair<i64, double>>& bcs, vector<double>& u, std::string& err) {
  Reduced red = reduce_system(coo, f, bcs);
  Csr k = to_csr(red.kred);
  const i64 n = (i64)red.free.size();
  vector<i64> newid(n), order(n);
  for (i64 r = 0; r < n; ++r) {
    const i64 dof = red.free[r], node = dof / 2;
    order[r] = ((node % g.nx) * g.ny + node / g.nx) * 2 + dof % 2;
  }
  vector<i64> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  std::sort(idx.begin(), idx.end(), [&](i64 a, i64 b) { return order[a] < order[b]; });
  for (i64 p = 0; p < n; ++p) newid[idx[p]] = p;
  i64 bw = 0;
  for (i64 r = 0; r < k.nrows; ++r)
    for (i64 t = k.row_ptrs[r]; t < k.row_ptrs[r + 1]; ++t) bw = std::max<i64>(bw, std::llabs(newid[r] - newid[k.col_ind[t]]));
  const i64 W = bw + 1;
  vector<double> B((size_t)n * W, 0.0);
  for (i64 r = 0; r < k.nrows; ++r)
    for (i64 t = k.row_ptrs[r]; t < k.row_ptrs[r + 1]; ++t) {
      const i64 a = newid[r], c = newid[k.col_ind[t]];
      if (c <= a) B[a * W + (a - c)] = k.values[t];
    }
  for (i64 j = 0; j < n; ++j) {  // L L^T, column j
    double s = B[j * W];
    for (i64 t = std::max<i64>(0, j - bw); t < j; ++t) s -= B[j * W + (j - t)] * B[j * W + (j - t)];
    if (!(s > 0.0)) { err = "topopt banded Cholesky: matrix not positive definite"; return false; }
    const double ljj = std::sqrt(s);
    B[j * W] = ljj;
    for (i64 i = j + 1; i <= std::min(n - 1, j + bw); ++i) {
      double v = B[i * W + (i - j)];
      for (i64 t = std::max<i64>(0, i - bw); t < j; ++t) v -= B[i * W + (i - t)] * B[j * W + (j - t)];
      B[i * W + (i - j)] = v / ljj;
    }
  }
  vector<double> y(n);
  for (i64 r = 0; r < n; ++r) y[newid[r]] = red.fred[r];
  for (i64 i = 0; i < n; ++i) {
    double s = y[i];
    for (i64 t = std::max<i64>(0, i - bw); t < i; ++t) s -= B[i * W + (i - t)] * y[t];
    y[i] = s / B[i * W];
  }
  for (i64 i = n - 1; i >= 0; --i) {
    double s = y[i];
    for (i64 t = i + 1; t <= std::min(n - 1, i + bw); ++t) s -= B[t * W + (t - i)] * y[t];
    y[i] = s / B[i * W];
  }
  u.assign(f.size(), 0.0);
  for (i64 r = 0; r < n; ++r) u[red.free[r]] = y[newid[r]];
  for (auto& b : bcs) u[b.first] = b.second;
  return true;
}

struct TopoArgs {
  i64 nelx, nely;
  double h, e0, nu, vol_frac, penal, radius, move_limit, emin;
  i64 max_iter;
  int density_filter, banded;
};

// topopt_simp (topopt:342-385); with density_filter the 88-line code's filter,
// sensitivity chain rule and OC loop on physical densities.
bool topo_run(const TopoArgs& a, const vector<double>& f, const vector<std::pair<i64, double>>& bcs,
              vector<double>& compliance, vector<double>& rho_out, std::string& err) {
  TopoGrid g{a.nelx + 1, a.nely + 1, a.nelx, a.nely, a.h};
  const i64 ne = g.n_elem();
  const vector<double> ke0 = topo_ke0(a.nu, a.h);
  vector<double> x(ne, a.vol_frac), phys = x, u;
  auto fe = [&](const vector<double>& rho) {
    Coo coo = topo_assemble(g, rho, ke0, a.e0, a.penal, a.emin);
    return a.banded ? topo_banded_solve(g, coo, f, bcs, u, err) : solve_with_dirichlet(coo, f, bcs, u, err);
  };
  auto dot = [&]() {
    double s = -0.0;
    for (size_t i = 0; i < f.size(); ++i) s += f[i] * u[i];
    return s;
  };
  compliance.clear();
  if (!fe(phys)) return false;
  compliance.push_back(dot());
  vector<double> hs = a.density_filter ? topo_filter_weight_sums(g, a.radius) : vector<double>();
  for (i64 it = 0; it < a.max_iter; ++it) {
    if (!fe(phys)) return false;
    compliance.push_back(dot());
    vector<double> raw(ne);
    for (i64 e = 0; e < ne; ++e) {
      i64 nd[4];
      g.nodes(e, nd);
      const double q = topo_quad_form(ke0, u, nd);
      raw[e] = -a.penal * std::pow(phys[e], a.penal - 1.0) * (a.e0 - a.emin) * q;
    }
    if (!a.density_filter) {
      x = topo_oc_update(x, topo_filter_sensitivity(g, raw, a.radius), a.vol_frac, a.move_limit);
      phys = x;
    } else {
      vector<double> dc, dv, ones(ne, 1.0);
      topo_density_filter(g, a.radius, raw, dc, &hs);
      topo_density_filter(g, a.radius, ones, dv, &hs);
      double l1 = 0.0, l2 = 1e9;
      vector<double> xn(ne);
      const double target = a.vol_frac * (double)ne;
      while ((l2 - l1) / (l1 + l2) > 1e-3) {
        const double lmid = 0.5 * (l2 + l1);
        for (i64 e = 0; e < ne; ++e) {
          const double oc = x[e] * std::sqrt(-dc[e] / dv[e] / lmid);
          xn[e] = std::max(0.0, std::max(x[e] - a.move_limit, std::min(1.0, std::min(x[e] + a.move_limit, oc))));
        }
        topo_density_filter(g, a.radius, xn, phys);
        double s = 0.0;
        for (i64 e = 0; e < ne; ++e) s += phys[e];
        if (s > target) l1 = lmid; else l2 = lmid;
      }
      x = xn;
    }
  }
  rho_out = a.density_filter ? phys : x;
  return true;
}

}  // namespace

extern "C" {

void orc_topopt_ke0(double nu, double h, double* out) {
  vector<double> k = topo_ke0(nu, h);
  std::copy(k.begin(), k.end(), out);
}

void orc_topopt_filter_sensitivity(i64 nelx, i64 nely, double h, const double* raw, double radius, double* out) {
  TopoGrid g{nelx + 1, nely + 1, nelx, nely, h};
  vector<double> r(raw, raw + nelx * nely);
  vector<double> o = topo_filter_sensitivity(g, r, radius);
  std::copy(o.begin(), o.end(), out);
}

void orc_topopt_oc_update(i64 n, const double* rho, const double* sens, double vol_frac, double move_limit,
                          double* out) {
  vector<double> o = topo_oc_update(vector<double>(rho, rho + n), vector<double>(sens, sens + n), vol_frac, move_limit);
  std::copy(o.begin(), o.end(), out);
}

// Runs one instance; compliance_out holds max_iter + 1 values, rho_out nelx * nely.
int orc_topopt(i64 nelx, i64 nely, double h, double e0, double nu, double vol_frac, double penal, double radius,
               double move_limit, double emin, i64 max_iter, int density_filter, int banded, const double* f,
               const i64* bc_dof, const double* bc_val, i64 nbc, double* compliance_out, double* rho_out) {
  TopoArgs a{nelx, nely, h, e0, nu, vol_frac, penal, radius, move_limit, emin, max_iter, density_filter, banded};
  vector<double> fv(f, f + 2 * (nelx + 1) * (nely + 1));
  vector<std::pair<i64, double>> bcs;
  for (i64 i = 0; i < nbc; ++i) bcs.push_back({bc_dof[i], bc_val[i]});
  vector<double> c, r;
  if (!topo_run(a, fv, bcs, c, r, g_err)) return 1;
  std::copy(c.begin(), c.end(), compliance_out);
  std::copy(r.begin(), r.end(), rho_out);
  return 0;
}

}  // extern "C"
