// gmsh v4.1 ASCII mesh reader (src/mesh/mod_gmsh_reader.f90:gmsh_read and its section readers):
// nodes, first-order volume elements (second-order tets and hexes by their corner nodes) and the
// surface elements of 2-D physical groups, as the raw arrays dpm_create takes.  Mesh ingestion is
// host work (a text file); the geometry, face matching and operators are built on the device.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace dpm {

struct GmshMesh {
  std::vector<double> xyz;           // [n_nodes][3], nodes in file order
  std::vector<int> cell_type;        // ElemType of each volume element, file order
  std::vector<int64_t> cell_off;     // [n_cells+1]
  std::vector<int> cell_nodes;       // 0-based node indices, gmsh local ordering
  std::vector<int64_t> bface_off;    // [n_bfaces+1]
  std::vector<int> bface_nodes;
  std::vector<int> bface_patch;      // 0-based patch index
  std::vector<std::string> patch_names;
};

// Returns 0, or -1 when the file cannot be opened, -2 when it is malformed or holds what the
// reference refuses (binary files, element types other than points, lines, triangles, quads,
// tets, hexes, prisms, pyramids, 10-node tets and 20-node hexes; a surface element outside every
// 2-D physical group); *err says which.
int read_gmsh(const std::string& path, GmshMesh& g, std::string* err);

// Writes g as a gmsh v4.1 ASCII file: one volume entity, one surface entity per patch, one 2-D
// physical group per patch (tags 1..n in patch order) and one 3-D group "fluid".
int write_gmsh(const std::string& path, const GmshMesh& g, std::string* err);

}  // namespace dpm
