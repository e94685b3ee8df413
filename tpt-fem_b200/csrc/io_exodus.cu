// io_exodus.cu -- Exodus II export of device-resident meshes.
//
// Restates write_exodus / mesh_to_exodus_bytes (crates/tpt-fem-io-exodus/src/
// lib.rs:384-563) and its NetCDF-3 classic (CDF-1) encoder (lib.rs:84-192):
// the same dimensions, variables, order, big-endian encodings and 4-byte
// padding, so that the files are interchangeable.  A device mesh has one
// cell type, hence one element block.  Coordinates are stored as NC_FLOAT
// (single precision), as the reference stores them.
#include <cstring>
#include <string>
#include <vector>

#include "objects.hpp"

namespace tptfem {

namespace {

constexpr uint32_t NC_DIMENSION = 10, NC_VARIABLE = 11, NC_FLOAT = 5, NC_INT = 4, NC_CHAR = 2;
constexpr uint32_t LEN_NAME = 33;

struct NcDim {
  std::string name;
  uint32_t size;
};

struct NcVar {
  std::string name;
  uint32_t dtype;
  std::vector<uint32_t> dims;
  std::string data;  // big-endian payload
};

void be32(std::string& o, uint32_t v) {
  const char b[4] = {(char)(v >> 24), (char)(v >> 16), (char)(v >> 8), (char)v};
  o.append(b, 4);
}

void pad4(std::string& o) {
  while (o.size() % 4) o.push_back('\0');
}

void name(std::string& o, const std::string& n) {
  o.push_back((char)(unsigned char)std::min<size_t>(n.size(), 255));
  o += n;
  pad4(o);
}

uint32_t vsize(const std::vector<NcDim>& dims, const NcVar& v) {
  uint64_t s = v.dtype == NC_CHAR ? 1 : 4;
  for (uint32_t d : v.dims) s *= dims[d].size;
  TPT_REQUIRE(s <= 0xffffffffull, TPTFEM_ERR_INVALID_ARG, "Exodus variable too large for a CDF-1 file");
  return (uint32_t)s;
}

std::string header(const std::vector<NcDim>& dims, const std::vector<NcVar>& vars,
                   const std::vector<uint32_t>& begins) {
  std::string h("CDF\x01", 4);
  be32(h, 0);  // numrecs
  be32(h, NC_DIMENSION);
  be32(h, (uint32_t)dims.size());
  for (const auto& d : dims) {
    name(h, d.name);
    be32(h, d.size);
  }
  be32(h, NC_VARIABLE);
  be32(h, (uint32_t)vars.size());
  for (size_t i = 0; i < vars.size(); ++i) {
    const NcVar& v = vars[i];
    name(h, v.name);
    be32(h, (uint32_t)v.dims.size());
    for (uint32_t d : v.dims) be32(h, d);
    be32(h, 0);  // attributes
    be32(h, v.dtype);
    be32(h, vsize(dims, v));
    be32(h, begins[i]);
  }
  be32(h, 0);  // NC_END
  return h;
}

std::string floats(const std::vector<double>& v) {
  std::string o;
  o.reserve(v.size() * 4);
  for (double x : v) {
    const float f = (float)x;
    uint32_t u;
    std::memcpy(&u, &f, 4);
    be32(o, u);
  }
  return o;
}

std::string ints(const std::vector<int64_t>& v) {
  std::string o;
  o.reserve(v.size() * 4);
  for (int64_t x : v) be32(o, (uint32_t)x);
  return o;
}

const char* exodus_cell_name(int cell) {
  switch (cell) {
    case TPTFEM_CELL_TRI3: return "TRI3";
    case TPTFEM_CELL_QUAD4: return "QUAD4";
    default: return "TET4";
  }
}

}  // namespace

std::string exodus_bytes(const MeshData& m) {
  cudaStream_t s = m.ctx->stream;
  std::vector<double> xyz((size_t)m.n_nodes * m.cdim);
  std::vector<int> conn((size_t)m.n_elems * m.npe);
  m.coords.download(xyz.data(), xyz.size());
  m.conn.download(conn.data(), conn.size());
  TPT_CUDA(cudaStreamSynchronize(s));
  const uint32_t nn = (uint32_t)m.n_nodes, ne = (uint32_t)m.n_elems;
  std::vector<NcDim> dims = {{"num_nodes", nn}, {"num_elem", ne}, {"num_elem_blk", 1}, {"num_node_sets", 0},
                             {"num_side_sets", 0}, {"len_name", LEN_NAME}, {"four", 4}, {"time_step", 1},
                             {"num_dim", 3}, {"eb0_n", ne}, {"eb0_np", (uint32_t)m.npe}};
  std::vector<NcVar> vars;
  vars.push_back({"time_whole", NC_FLOAT, {7}, floats({0.0})});
  std::vector<double> c3((size_t)m.n_nodes * 3);
  for (int64_t i = 0; i < m.n_nodes; ++i)
    for (int d = 0; d < 3; ++d) c3[(size_t)i * 3 + d] = d < m.cdim ? xyz[(size_t)i * m.cdim + d] : 0.0;
  vars.push_back({"coords", NC_FLOAT, {0, 8}, floats(c3)});
  vars.push_back({"elem_blk_id", NC_INT, {2}, ints({1})});
  vars.push_back({"eb_status", NC_INT, {2}, ints({1})});
  vars.push_back({"eb_prop1", NC_INT, {2}, ints({1})});
  std::string nm(exodus_cell_name(m.cell));
  nm.resize(LEN_NAME, '\0');
  vars.push_back({"eb_names", NC_CHAR, {5, 2}, nm});
  std::vector<int64_t> c1(conn.begin(), conn.end());
  for (auto& v : c1) v += 1;  // Exodus node ids are 1-based
  vars.push_back({"connect1", NC_INT, {9, 10}, ints(c1)});
  std::vector<int64_t> emap(ne), nmap(nn);
  for (uint32_t i = 0; i < ne; ++i) emap[i] = i + 1;
  for (uint32_t i = 0; i < nn; ++i) nmap[i] = i + 1;
  vars.push_back({"elem_num_map", NC_INT, {1}, ints(emap)});
  vars.push_back({"node_num_map", NC_INT, {0}, ints(nmap)});
  // begins: header length (with placeholder begins), then each payload padded to 4
  std::vector<uint32_t> begins(vars.size(), 0);
  uint64_t cursor = (header(dims, vars, begins).size() + 3) & ~uint64_t(3);
  for (size_t i = 0; i < vars.size(); ++i) {
    begins[i] = (uint32_t)cursor;
    cursor = (cursor + vsize(dims, vars[i]) + 3) & ~uint64_t(3);
  }
  TPT_REQUIRE(cursor <= 0xffffffffull, TPTFEM_ERR_INVALID_ARG, "mesh too large for a CDF-1 Exodus file");
  std::string out = header(dims, vars, begins);
  pad4(out);
  for (const auto& v : vars) {
    out += v.data;
    pad4(out);
  }
  return out;
}

}  // namespace tptfem
