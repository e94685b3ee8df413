// io_vtk.cu -- legacy VTK export of device-resident meshes and per-node fields.
//
// Restates write_vtk / write_vtk_with_data (crates/tpt-fem-io-vtk/src/lib.rs:
// 117-196).  The reference builds a vtkio model (mesh_to_vtk) and lets the
// third-party crate `vtkio` (not vendored) serialise it.  This file writes the
// same bytes directly; the layout below is the one the reference's own output
// files show (mesh_gen_box_structured.vtk, thermal_solve.vtk,
// elasticity_frame.vtk):
//   "# vtk DataFile Version 4.1\n" title "\n" "BINARY\n" "\n"
//   "DATASET UNSTRUCTURED_GRID\n" "POINTS <n> double\n" <3n big-endian f64> "\n"
//   "\nCELLS <m> <m + sum of node counts>\n" <big-endian i32: count, ids...> "\n"
//   "\nCELL_TYPES <m>\n" <m big-endian i32> "\n"
//   "\nPOINT_DATA <n>\n"
//   per field: "\nSCALARS <name> double 1\nLOOKUP_TABLE default\n" <n big-endian f64> "\n"
//   "\nCELL_DATA <m>\n" "\n"
// Points are padded to three coordinates with 0.0 (mesh_to_vtk:125-131).
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "objects.hpp"

namespace tptfem {

namespace {

void put_be64(std::string& out, double v) {
  uint64_t u;
  std::memcpy(&u, &v, 8);
  char b[8];
  for (int i = 0; i < 8; ++i) b[i] = (char)((u >> (56 - 8 * i)) & 0xff);
  out.append(b, 8);
}

void put_be32(std::string& out, uint32_t u) {
  char b[4];
  for (int i = 0; i < 4; ++i) b[i] = (char)((u >> (24 - 8 * i)) & 0xff);
  out.append(b, 4);
}

// VTK cell type numbers of the linear cells (vtk_cell_type, io-vtk:102-115).
uint32_t vtk_cell(int cell) {
  switch (cell) {
    case TPTFEM_CELL_TRI3: return 5;   // VTK_TRIANGLE
    case TPTFEM_CELL_QUAD4: return 9;  // VTK_QUAD
    default: return 10;                // VTK_TETRA
  }
}

}  // namespace

std::string vtk_legacy_binary(const MeshData& m, const std::string& title, const std::vector<std::string>& names,
                              const std::vector<const double*>& values) {
  cudaStream_t s = m.ctx->stream;
  std::vector<double> xyz((size_t)m.n_nodes * m.cdim);
  std::vector<int> conn((size_t)m.n_elems * m.npe);
  m.coords.download(xyz.data(), xyz.size());
  m.conn.download(conn.data(), conn.size());
  TPT_CUDA(cudaStreamSynchronize(s));
  for (const auto& nm : names)
    TPT_REQUIRE(!nm.empty() && nm.find_first_of(" \t\n") == std::string::npos, TPTFEM_ERR_INVALID_ARG,
                "field names must be non-empty and free of white space");
  TPT_REQUIRE(title.find('\n') == std::string::npos, TPTFEM_ERR_INVALID_ARG, "the title must be one line");
  std::string out;
  out.reserve((size_t)m.n_nodes * (24 + 8 * values.size()) + (size_t)m.n_elems * 4 * (m.npe + 2) + 512);
  out += "# vtk DataFile Version 4.1\n";
  out += title + "\n";
  out += "BINARY\n\nDATASET UNSTRUCTURED_GRID\n";
  out += "POINTS " + std::to_string(m.n_nodes) + " double\n";
  for (int64_t i = 0; i < m.n_nodes; ++i)
    for (int d = 0; d < 3; ++d) put_be64(out, d < m.cdim ? xyz[(size_t)i * m.cdim + d] : 0.0);
  out += "\n";
  out += "\nCELLS " + std::to_string(m.n_elems) + " " + std::to_string(m.n_elems * (m.npe + 1)) + "\n";
  for (int64_t e = 0; e < m.n_elems; ++e) {
    put_be32(out, (uint32_t)m.npe);
    for (int j = 0; j < m.npe; ++j) put_be32(out, (uint32_t)conn[(size_t)e * m.npe + j]);
  }
  out += "\n";
  out += "\nCELL_TYPES " + std::to_string(m.n_elems) + "\n";
  const uint32_t ct = vtk_cell(m.cell);
  for (int64_t e = 0; e < m.n_elems; ++e) put_be32(out, ct);
  out += "\n";
  out += "\nPOINT_DATA " + std::to_string(m.n_nodes) + "\n";
  for (size_t f = 0; f < names.size(); ++f) {
    out += "\nSCALARS " + names[f] + " double 1\nLOOKUP_TABLE default\n";
    for (int64_t i = 0; i < m.n_nodes; ++i) put_be64(out, values[f][i]);
    out += "\n";
  }
  out += "\nCELL_DATA " + std::to_string(m.n_elems) + "\n";
  out += "\n";
  return out;
}

void write_file(const char* path, const std::string& bytes) {
  std::ofstream f(path, std::ios::binary | std::ios::trunc);
  TPT_REQUIRE(f.good(), TPTFEM_ERR_INVALID_ARG, std::string("cannot open ") + path + " for writing");
  f.write(bytes.data(), (std::streamsize)bytes.size());
  f.close();
  TPT_REQUIRE(f.good(), TPTFEM_ERR_INVALID_ARG, std::string("writing ") + path + " failed");
}

}  // namespace tptfem
