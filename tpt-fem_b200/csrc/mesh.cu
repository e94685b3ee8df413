// mesh.cu -- device box mesher and the node->element adjacency every
// assembly kernel walks.
//
// The adjacency is the backbone of the deterministic "row gather" design: a
// row's owner thread visits the elements incident to its node in ascending
// element id, which is exactly the order in which Coo::to_csr sums duplicate
// triplets (crates/tpt-fem-sparse/src/lib.rs:144-163) and in which the
// reference's load loops add into rhs (crates/tpt-fem-thermal/src/lib.rs:224-230).
// Compiled with -fmad=false: coordinates follow box_mesh's rounding exactly.
#include <cmath>

#include "objects.hpp"

namespace tptfem {

namespace {

// box_mesh node coordinates (crates/tpt-fem-mesh-gen/src/lib.rs:427-439):
// node (i,j,k) -> id (i*(ny+1)+j)*(nz+1)+k, x = min + (i/nx)*(max-min).
__global__ void box_nodes(double* __restrict__ xyz, int nx, int ny, int nz, double mn0, double mn1, double mn2,
                          double ex0, double ex1, double ex2) {
  int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t nn = (int64_t)(nx + 1) * (ny + 1) * (nz + 1);
  if (id >= nn) return;
  int k = (int)(id % (nz + 1));
  int64_t r = id / (nz + 1);
  int j = (int)(r % (ny + 1));
  int i = (int)(r / (ny + 1));
  double t = nx > 0 ? (double)i / (double)nx : 0.0;
  double u = ny > 0 ? (double)j / (double)ny : 0.0;
  double w = nz > 0 ? (double)k / (double)nz : 0.0;
  xyz[3 * id + 0] = mn0 + t * ex0;
  xyz[3 * id + 1] = mn1 + u * ex1;
  xyz[3 * id + 2] = mn2 + w * ex2;
}

// Six tets per brick sharing the 0-6 diagonal (mesh-gen:459-490); `swap` bit t
// set when orient3 of tet t is negative.
__global__ void box_tets(int* __restrict__ conn, int nx, int ny, int nz, unsigned swap) {
  int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t nb = (int64_t)nx * ny * nz;
  if (b >= nb) return;
  int k = (int)(b % nz);
  int64_t r = b / nz;
  int j = (int)(r % ny);
  int i = (int)(r / ny);
  auto id = [&](int di, int dj, int dk) { return ((i + di) * (ny + 1) + (j + dj)) * (nz + 1) + (k + dk); };
  int c[8] = {id(0, 0, 0), id(1, 0, 0), id(1, 1, 0), id(0, 1, 0), id(0, 0, 1), id(1, 0, 1), id(1, 1, 1), id(0, 1, 1)};
  const int tets[6][4] = {{0, 1, 2, 6}, {0, 2, 3, 6}, {0, 3, 7, 6}, {0, 7, 4, 6}, {0, 4, 5, 6}, {0, 5, 1, 6}};
#pragma unroll
  for (int t = 0; t < 6; ++t) {
    int v0 = c[tets[t][0]], v1 = c[tets[t][1]], v2 = c[tets[t][2]], v3 = c[tets[t][3]];
    if (swap & (1u << t)) { int tmp = v1; v1 = v2; v2 = tmp; }
    int4 q = make_int4(v0, v1, v2, v3);
    reinterpret_cast<int4*>(conn)[6 * b + t] = q;
  }
}

__global__ void count_incidence(const int* __restrict__ conn, int64_t n_ent, int* __restrict__ cnt) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_ent) atomicAdd(&cnt[conn[i]], 1);
}

__global__ void fill_incidence(const int* __restrict__ conn, int64_t n_ent, int npe, const int* __restrict__ ptr,
                               int* __restrict__ cursor, int* __restrict__ ne) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_ent) return;
  int node = conn[i];
  int e = (int)(i / npe), l = (int)(i % npe);
  int pos = ptr[node] + atomicAdd(&cursor[node], 1);
  ne[pos] = (e << 2) | l;
}

// Sort each node's incidence segment by element id (insertion sort: segments
// hold a few dozen entries) and record the largest degree.
__global__ void sort_incidence(const int* __restrict__ ptr, int* __restrict__ ne, int64_t n_nodes,
                               int* __restrict__ max_deg) {
  int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= n_nodes) return;
  int b = ptr[n], e = ptr[n + 1];
  for (int i = b + 1; i < e; ++i) {
    int v = ne[i];
    int j = i - 1;
    while (j >= b && ne[j] > v) { ne[j + 1] = ne[j]; --j; }
    ne[j + 1] = v;
  }
  atomicMax(max_deg, e - b);
}

constexpr int MAX_NB = 255;  // neighbour positions are stored as uint8

// Sorted unique neighbour nodes of node n (itself included).  COUNT pass
// writes the count; FILL pass writes the list.  Sets *err when a node has
// more than MAX_NB neighbours.
template <bool FILL>
__global__ void neighbours(const int* __restrict__ conn, int npe, const int* __restrict__ ne_ptr,
                           const int* __restrict__ ne, int64_t n_nodes, int* __restrict__ cnt,
                           const int* __restrict__ nb_ptr, int* __restrict__ nb, int* __restrict__ err,
                           int* __restrict__ max_nb) {
  int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= n_nodes) return;
  int list[MAX_NB + 1];
  int len = 0;
  bool overflow = false;
  for (int k = ne_ptr[n]; k < ne_ptr[n + 1] && !overflow; ++k) {
    int e = ne[k] >> 2;
    for (int j = 0; j < npe; ++j) {
      int v = conn[(int64_t)e * npe + j];
      int lo = 0, hi = len;
      while (lo < hi) { int mid = (lo + hi) >> 1; if (list[mid] < v) lo = mid + 1; else hi = mid; }
      if (lo < len && list[lo] == v) continue;
      if (len == MAX_NB) { overflow = true; break; }
      for (int t = len; t > lo; --t) list[t] = list[t - 1];
      list[lo] = v;
      ++len;
    }
  }
  if (overflow) { atomicExch(err, 1); return; }
  if (!FILL) {
    cnt[n] = len;
    atomicMax(max_nb, len);
  } else {
    int o = nb_ptr[n];
    for (int t = 0; t < len; ++t) nb[o + t] = list[t];
  }
}

// For incidence entry k (node n, element e): position of each element node in
// n's neighbour list.
__global__ void incidence_slots(const int* __restrict__ conn, int npe, const int* __restrict__ ne_ptr,
                                const int* __restrict__ ne, int64_t n_nodes, const int* __restrict__ nb_ptr,
                                const int* __restrict__ nb, uchar4* __restrict__ slot) {
  int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= n_nodes) return;
  int b = nb_ptr[n], len = nb_ptr[n + 1] - b;
  for (int k = ne_ptr[n]; k < ne_ptr[n + 1]; ++k) {
    int e = ne[k] >> 2;
    unsigned char s[4] = {0, 0, 0, 0};
    for (int j = 0; j < npe; ++j) {
      int v = conn[(int64_t)e * npe + j];
      int lo = 0, hi = len;
      while (lo < hi) { int mid = (lo + hi) >> 1; if (nb[b + mid] < v) lo = mid + 1; else hi = mid; }
      s[j] = (unsigned char)lo;
    }
    slot[k] = make_uchar4(s[0], s[1], s[2], s[3]);
  }
}

// Boundary faces (crates/tpt-fem-assembly/src/lib.rs:563-583): a face is on the
// boundary iff no other element holds all of its nodes.  Face tables follow
// TRI_FACES / QUAD_FACES / TET_FACES (assembly:46-96).
__global__ void boundary_face_mask(const int* __restrict__ conn, int cell, int npe, const int* __restrict__ ne_ptr,
                                   const int* __restrict__ ne, int64_t n_elems, unsigned char* __restrict__ mask) {
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_elems) return;
  if (cell == TPTFEM_CELL_TET4) {
    // Faces 1..3 (opposite vertices 1..3) contain vertex 0: one scan of vertex
    // 0's incident elements serves all three; face 0 = (1, 2, 3) scans vertex
    // 1's.  A face is interior iff another element holds its three vertices.
    const int4 me = reinterpret_cast<const int4*>(conn)[e];
    auto holds = [](const int4& c, int v) { return c.x == v || c.y == v || c.z == v || c.w == v; };
    bool sh1 = false, sh2 = false, sh3 = false, sh0 = false;
    for (int k = ne_ptr[me.x]; k < ne_ptr[me.x + 1]; ++k) {
      const int o = ne[k] >> 2;
      if (o == (int)e) continue;
      const int4 c = reinterpret_cast<const int4*>(conn)[o];
      const bool h1 = holds(c, me.y), h2 = holds(c, me.z), h3 = holds(c, me.w);
      sh1 |= h2 && h3;
      sh2 |= h1 && h3;
      sh3 |= h1 && h2;
    }
    for (int k = ne_ptr[me.y]; k < ne_ptr[me.y + 1] && !sh0; ++k) {
      const int o = ne[k] >> 2;
      if (o == (int)e) continue;
      const int4 c = reinterpret_cast<const int4*>(conn)[o];
      sh0 = holds(c, me.z) && holds(c, me.w);
    }
    mask[e] = (unsigned char)((sh0 ? 0 : 1) | (sh1 ? 0 : 2) | (sh2 ? 0 : 4) | (sh3 ? 0 : 8));
    return;
  }
  const int tet_f[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
  const int quad_f[4][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}};
  const int tri_f[3][2] = {{1, 2}, {2, 0}, {0, 1}};
  const int nf = cell == TPTFEM_CELL_TRI3 ? 3 : 4, fn = (cell == TPTFEM_CELL_TET4) ? 3 : 2;
  unsigned char m = 0;
  for (int f = 0; f < nf; ++f) {
    int v[3];
    for (int q = 0; q < fn; ++q)
      v[q] = conn[e * npe + (cell == TPTFEM_CELL_TET4 ? tet_f[f][q]
                                                       : (cell == TPTFEM_CELL_TRI3 ? tri_f[f][q] : quad_f[f][q]))];
    bool shared = false;
    for (int k = ne_ptr[v[0]]; k < ne_ptr[v[0] + 1] && !shared; ++k) {
      int o = ne[k] >> 2;
      if (o == (int)e) continue;
      int hit = 1;
      for (int q = 1; q < fn; ++q) {
        bool found = false;
        for (int j = 0; j < npe; ++j) found |= (conn[(int64_t)o * npe + j] == v[q]);
        hit &= found;
      }
      shared = hit;
    }
    if (!shared) m |= (unsigned char)(1u << f);
  }
  mask[e] = m;
}

double orient3(const double* a, const double* b, const double* c, const double* d) {
  double ab[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  double ac[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
  double ad[3] = {d[0] - a[0], d[1] - a[1], d[2] - a[2]};
  return ab[0] * (ac[1] * ad[2] - ac[2] * ad[1]) - ab[1] * (ac[0] * ad[2] - ac[2] * ad[0]) +
         ab[2] * (ac[0] * ad[1] - ac[1] * ad[0]);
}

}  // namespace

void mesh_box(MeshData& m, const double mn[3], const double mx[3], const int64_t n[3]) {
  cudaStream_t s = m.ctx->stream;
  int64_t nx = n[0], ny = n[1], nz = n[2];
  TPT_REQUIRE(nx >= 1 && ny >= 1 && nz >= 1, TPTFEM_ERR_INVALID_ARG, "box_mesh needs at least one cell per axis");
  int64_t nn = (nx + 1) * (ny + 1) * (nz + 1);
  int64_t ne = 6 * nx * ny * nz;
  TPT_REQUIRE(nn < (1LL << 31) && ne < (1LL << 29), TPTFEM_ERR_INVALID_ARG, "box_mesh too large for int32 ids");
  m.cell = TPTFEM_CELL_TET4;
  m.cdim = 3;
  m.npe = 4;
  m.n_nodes = nn;
  m.n_elems = ne;
  m.coords.alloc(nn * 3, s);
  m.conn.alloc(ne * 4, s);
  double ex[3] = {mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2]};
  box_nodes<<<ceil_div(nn, 256), 256, 0, s>>>(m.coords.p, (int)nx, (int)ny, (int)nz, mn[0], mn[1], mn[2], ex[0],
                                               ex[1], ex[2]);
  TPT_CHECK_LAUNCH();
  // Orientation of the six tets, evaluated on the first brick's corners as the
  // reference's `corner` closure does (mesh-gen:441-450, 476-479).
  const int cof[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  const int tets[6][4] = {{0, 1, 2, 6}, {0, 2, 3, 6}, {0, 3, 7, 6}, {0, 7, 4, 6}, {0, 4, 5, 6}, {0, 5, 1, 6}};
  double co[8][3];
  for (int c = 0; c < 8; ++c) {
    double t = (double)cof[c][0] / (double)nx, u = (double)cof[c][1] / (double)ny, w = (double)cof[c][2] / (double)nz;
    co[c][0] = mn[0] + t * (mx[0] - mn[0]);
    co[c][1] = mn[1] + u * (mx[1] - mn[1]);
    co[c][2] = mn[2] + w * (mx[2] - mn[2]);
  }
  unsigned swap = 0;
  for (int t = 0; t < 6; ++t)
    if (orient3(co[tets[t][0]], co[tets[t][1]], co[tets[t][2]], co[tets[t][3]]) < 0.0) swap |= 1u << t;
  int64_t nb = nx * ny * nz;
  box_tets<<<ceil_div(nb, 256), 256, 0, s>>>(m.conn.p, (int)nx, (int)ny, (int)nz, swap);
  TPT_CHECK_LAUNCH();
}

void mesh_build_adjacency(MeshData& m) {
  if (m.adj) return;
  cudaStream_t s = m.ctx->stream;
  int64_t nn = m.n_nodes, n_ent = m.n_elems * m.npe;
  DevBuf<int> cnt;
  cnt.alloc(nn + 1, s);
  cnt.zero();
  count_incidence<<<ceil_div(n_ent, 256), 256, 0, s>>>(m.conn.p, n_ent, cnt.p);
  TPT_CHECK_LAUNCH();
  m.ne_ptr.alloc(nn + 1, s);
  exclusive_scan_i32(cnt.p, m.ne_ptr.p, nn, s);
  m.ne.alloc(n_ent, s);
  cnt.zero();
  fill_incidence<<<ceil_div(n_ent, 256), 256, 0, s>>>(m.conn.p, n_ent, m.npe, m.ne_ptr.p, cnt.p, m.ne.p);
  TPT_CHECK_LAUNCH();
  DevBuf<int> scratch;
  scratch.alloc(4, s);
  scratch.zero();
  int* d_maxdeg = scratch.p;
  int* d_err = scratch.p + 1;
  int* d_maxnb = scratch.p + 2;
  sort_incidence<<<ceil_div(nn, 128), 128, 0, s>>>(m.ne_ptr.p, m.ne.p, nn, d_maxdeg);
  TPT_CHECK_LAUNCH();
  neighbours<false><<<ceil_div(nn, 128), 128, 0, s>>>(m.conn.p, m.npe, m.ne_ptr.p, m.ne.p, nn, cnt.p, nullptr,
                                                         nullptr, d_err, d_maxnb);
  TPT_CHECK_LAUNCH();
  int h[4];
  TPT_CUDA(cudaMemcpyAsync(h, scratch.p, 4 * sizeof(int), cudaMemcpyDeviceToHost, s));
  TPT_CUDA(cudaStreamSynchronize(s));
  TPT_REQUIRE(h[1] == 0, TPTFEM_ERR_CREATION, "a node has more than 255 neighbours (valence limit of the device path)");
  m.max_deg = h[0];
  m.max_nb = h[2];
  m.nb_ptr.alloc(nn + 1, s);
  int64_t tot = exclusive_scan_i32(cnt.p, m.nb_ptr.p, nn, s);
  m.nb.alloc(tot, s);
  neighbours<true><<<ceil_div(nn, 128), 128, 0, s>>>(m.conn.p, m.npe, m.ne_ptr.p, m.ne.p, nn, nullptr, m.nb_ptr.p,
                                                        m.nb.p, d_err, d_maxnb);
  TPT_CHECK_LAUNCH();
  m.slot.alloc(n_ent, s);
  incidence_slots<<<ceil_div(nn, 128), 128, 0, s>>>(m.conn.p, m.npe, m.ne_ptr.p, m.ne.p, nn, m.nb_ptr.p, m.nb.p,
                                                     m.slot.p);
  TPT_CHECK_LAUNCH();
  m.adj = true;
}

void mesh_build_boundary_faces(MeshData& m) {
  if (m.bfaces) return;
  mesh_build_adjacency(m);
  cudaStream_t s = m.ctx->stream;
  m.bface.alloc(m.n_elems, s);
  boundary_face_mask<<<ceil_div(m.n_elems, 128), 128, 0, s>>>(m.conn.p, m.cell, m.npe, m.ne_ptr.p, m.ne.p,
                                                              m.n_elems, m.bface.p);
  TPT_CHECK_LAUNCH();
  m.bfaces = true;
}

}  // namespace tptfem
