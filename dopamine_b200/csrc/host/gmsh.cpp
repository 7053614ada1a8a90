// gmsh v4.1 ASCII reader and writer; see gmsh.hpp.  The reader follows the reference's section
// readers line for line (src/mesh/mod_gmsh_reader.f90:45-236, 618-734, 987-1014): every list-
// directed read there consumes one line, so this parser is line-based too.
#include "gmsh.hpp"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string_view>

#include "../../../include/dopamine_b200.h"
#include "mesh.hpp"

namespace dpm {
namespace {

// gmsh element codes (mod_gmsh_reader.f90:14-23)
constexpr int G_LINE2 = 1, G_TRI3 = 2, G_QUAD4 = 3, G_TET4 = 4, G_HEX8 = 5, G_PRISM6 = 6, G_PYR5 = 7, G_TET10 = 11,
              G_HEX20 = 17, G_POINT = 15;

int nodes_per_element(int t) {  // gmsh_nodes_per_element
  switch (t) {
    case G_LINE2: return 2;
    case G_TRI3: return 3;
    case G_QUAD4: return 4;
    case G_TET4: return 4;
    case G_HEX8: return 8;
    case G_PRISM6: return 6;
    case G_PYR5: return 5;
    case G_TET10: return 10;
    case G_HEX20: return 20;
    case G_POINT: return 1;
  }
  return -1;
}
// volume element -> (cell type, corner nodes used)
bool volume_type(int t, int& type, int& corners) {
  switch (t) {
    case G_TET4: case G_TET10: type = EL_TET4; corners = 4; return true;
    case G_HEX8: case G_HEX20: type = EL_HEX8; corners = 8; return true;
    case G_PRISM6: type = EL_PRISM6; corners = 6; return true;
    case G_PYR5: type = EL_PYR5; corners = 5; return true;
  }
  return false;
}
bool boundary_type(int t) { return t == G_TRI3 || t == G_QUAD4; }

struct Lines {
  const char* p;
  const char* end;
  bool next(std::string_view& out) {
    if (p >= end) return false;
    const char* s = p;
    while (p < end && *p != '\n') ++p;
    const char* e = p;
    if (p < end) ++p;
    if (e > s && e[-1] == '\r') --e;
    out = std::string_view(s, (size_t)(e - s));
    return true;
  }
};

void split(std::string_view line, std::vector<std::string_view>& tok) {
  tok.clear();
  size_t i = 0, n = line.size();
  while (i < n) {
    while (i < n && (line[i] == ' ' || line[i] == '\t')) ++i;
    if (i >= n) break;
    size_t s = i;
    while (i < n && line[i] != ' ' && line[i] != '\t') ++i;
    tok.push_back(line.substr(s, i - s));
  }
}

bool to_ll(std::string_view t, long long& v) {
  char buf[64];
  if (t.empty() || t.size() >= sizeof(buf)) return false;
  std::memcpy(buf, t.data(), t.size());
  buf[t.size()] = 0;
  char* e = nullptr;
  v = std::strtoll(buf, &e, 10);
  return e && *e == 0;
}
bool to_d(std::string_view t, double& v) {
  char buf[64];
  if (t.empty() || t.size() >= sizeof(buf)) return false;
  std::memcpy(buf, t.data(), t.size());
  buf[t.size()] = 0;
  char* e = nullptr;
  v = std::strtod(buf, &e);
  return e && *e == 0;
}

std::string_view trim(std::string_view s) {
  size_t a = 0, b = s.size();
  while (a < b && (s[a] == ' ' || s[a] == '\t')) ++a;
  while (b > a && (s[b - 1] == ' ' || s[b - 1] == '\t')) --b;
  return s.substr(a, b - a);
}

struct Elem {
  int etype, phys;
  int64_t first;  // into the node-tag pool
  int nn;
};

}  // namespace

int read_gmsh(const std::string& path, GmshMesh& g, std::string* err) {
  auto fail = [&](int code, const std::string& msg) {
    if (err) *err = msg;
    return code;
  };
  std::ifstream in(path, std::ios::binary);
  if (!in) return fail(-1, "cannot open file: " + path);
  std::string text((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
  Lines L{text.data(), text.data() + text.size()};
  std::string_view line;
  std::vector<std::string_view> tok;
  struct Group { int dim, tag; std::string name; };
  std::vector<Group> groups;
  struct EntPhys { int dim, tag, phys; };
  std::vector<EntPhys> ent;
  std::vector<long long> node_tags;
  std::vector<double> coords;
  std::vector<Elem> elems;
  std::vector<long long> pool;
  bool got_nodes = false, got_elements = false;
  auto need = [&](size_t n, const char* what) -> bool {
    if (!L.next(line)) return false;
    split(line, tok);
    (void)what;
    return tok.size() >= n;
  };
  auto lookup = [&](int dim, int tag) {  // lookup_entity_phys_tag: first match, else -1
    for (const auto& e : ent)
      if (e.dim == dim && e.tag == tag) return e.phys;
    return -1;
  };
  while (L.next(line)) {
    std::string_view t = trim(line);
    if (t == "$MeshFormat") {
      double ver;
      long long ft;
      if (!need(2, "format") || !to_d(tok[0], ver) || !to_ll(tok[1], ft)) return fail(-2, "malformed $MeshFormat");
      if (ver < 4.0) return fail(-2, "only gmsh format 4 files are read (found an older format)");
      if (ft != 0) return fail(-2, "only ASCII gmsh files are read (found a binary file)");
    } else if (t == "$PhysicalNames") {  // read_physical_names
      long long n;
      if (!need(1, "count") || !to_ll(tok[0], n) || n < 0) return fail(-2, "malformed $PhysicalNames");
      groups.clear();
      for (long long i = 0; i < n; ++i) {
        long long d, tg;
        if (!need(3, "group") || !to_ll(tok[0], d) || !to_ll(tok[1], tg)) return fail(-2, "malformed physical name");
        // the name: the rest of the line after the two integers, quotes stripped
        const size_t pos = (size_t)(tok[1].data() - line.data());
        std::string_view rest = trim(line.substr(pos + tok[1].size()));
        std::string name(rest);
        if (name.size() >= 2 && name.front() == '"') name = name.substr(1, name.size() - 2);
        groups.push_back({(int)d, (int)tg, name});
      }
    } else if (t == "$Entities") {  // read_entities_v4, parse_entity_line_for_phys
      long long cnt[4];
      if (!need(4, "counts")) return fail(-2, "malformed $Entities");
      for (int k = 0; k < 4; ++k)
        if (!to_ll(tok[k], cnt[k])) return fail(-2, "malformed $Entities");
      ent.clear();
      for (int dim = 0; dim < 4; ++dim)
        for (long long i = 0; i < cnt[dim]; ++i) {
          if (!L.next(line)) return fail(-2, "truncated $Entities");
          split(line, tok);
          long long etag, nphys, phys;
          if (tok.size() < 8 || !to_ll(tok[0], etag) || !to_ll(tok[7], nphys)) continue;
          if (nphys <= 0 || (long long)tok.size() < 8 + nphys || !to_ll(tok[8], phys)) continue;
          ent.push_back({dim, (int)etag, (int)phys});
        }
    } else if (t == "$Nodes") {  // read_nodes_v4
      long long nb, nn, mn, mx;
      if (!need(4, "header") || !to_ll(tok[0], nb) || !to_ll(tok[1], nn) || !to_ll(tok[2], mn) || !to_ll(tok[3], mx) ||
          nn < 0 || nb < 0)
        return fail(-2, "malformed $Nodes header");
      node_tags.assign(nn, 0);
      coords.assign(3 * nn, 0.0);
      long long off = 0;
      for (long long b = 0; b < nb; ++b) {
        long long edim, etag, par, n;
        if (!need(4, "block") || !to_ll(tok[0], edim) || !to_ll(tok[1], etag) || !to_ll(tok[2], par) ||
            !to_ll(tok[3], n) || n < 0 || off + n > nn)
          return fail(-2, "malformed $Nodes block");
        for (long long i = 0; i < n; ++i)
          if (!need(1, "tag") || !to_ll(tok[0], node_tags[off + i])) return fail(-2, "malformed node tag");
        for (long long i = 0; i < n; ++i)
          if (!need(3, "xyz") || !to_d(tok[0], coords[3 * (off + i)]) || !to_d(tok[1], coords[3 * (off + i) + 1]) ||
              !to_d(tok[2], coords[3 * (off + i) + 2]))
            return fail(-2, "malformed node coordinates");
        off += n;
      }
      if (off != nn) return fail(-2, "$Nodes blocks do not add up to the node count");
      got_nodes = true;
    } else if (t == "$Elements") {  // read_elements_v4
      long long nb, ne, mn, mx;
      if (!need(4, "header") || !to_ll(tok[0], nb) || !to_ll(tok[1], ne) || !to_ll(tok[2], mn) || !to_ll(tok[3], mx) ||
          ne < 0 || nb < 0)
        return fail(-2, "malformed $Elements header");
      elems.clear();
      elems.reserve(ne);
      pool.clear();
      for (long long b = 0; b < nb; ++b) {
        long long edim, etag, et, n;
        if (!need(4, "block") || !to_ll(tok[0], edim) || !to_ll(tok[1], etag) || !to_ll(tok[2], et) ||
            !to_ll(tok[3], n) || n < 0)
          return fail(-2, "malformed $Elements block");
        int nn = nodes_per_element((int)et);
        if (nn < 1)
          return fail(-2, "unsupported gmsh element type " + std::to_string(et) +
                              " (supported: first-order line, tri, quad, tet, hex, prism, pyramid, point)");
        int phys = lookup((int)edim, (int)etag);
        for (long long i = 0; i < n; ++i) {
          if (!need((size_t)nn + 1, "element")) return fail(-2, "malformed element line");
          Elem e{(int)et, phys, (int64_t)pool.size(), nn};
          for (int k = 0; k < nn; ++k) {
            long long v;
            if (!to_ll(tok[1 + k], v)) return fail(-2, "malformed element node");
            pool.push_back(v);
          }
          elems.push_back(e);
        }
      }
      if ((long long)elems.size() != ne) return fail(-2, "$Elements blocks do not add up to the element count");
      got_elements = true;
    }
  }
  if (!got_nodes) return fail(-2, "missing $Nodes section");
  if (!got_elements) return fail(-2, "missing $Elements section");

  // build_mesh_from_gmsh: node tags -> local indices, volume and boundary elements in file order
  long long max_tag = 0;
  for (long long t : node_tags) max_tag = std::max(max_tag, t);
  if (max_tag > 4000000000LL) return fail(-2, "node tags beyond the supported range");
  std::vector<int> t2l((size_t)max_tag + 1, -1);
  for (size_t i = 0; i < node_tags.size(); ++i) {
    if (node_tags[i] < 1) return fail(-2, "node tag below 1");
    t2l[(size_t)node_tags[i]] = (int)i;
  }
  auto local = [&](long long tag, int& out) {
    if (tag < 1 || tag > max_tag || t2l[(size_t)tag] < 0) return false;
    out = t2l[(size_t)tag];
    return true;
  };
  g = GmshMesh();
  g.xyz = coords;
  g.cell_off.push_back(0);
  g.bface_off.push_back(0);
  const int n_phys = (int)groups.size();
  std::vector<int> face_group;  // group index (0-based) per boundary element
  for (const Elem& e : elems) {
    int type, corners;
    if (volume_type(e.etype, type, corners)) {
      for (int k = 0; k < corners; ++k) {
        int v;
        if (!local(pool[e.first + k], v)) return fail(-2, "element references an unknown node");
        g.cell_nodes.push_back(v);
      }
      g.cell_type.push_back(type);
      g.cell_off.push_back((int64_t)g.cell_nodes.size());
    } else if (boundary_type(e.etype)) {
      for (int k = 0; k < e.nn; ++k) {
        int v;
        if (!local(pool[e.first + k], v)) return fail(-2, "element references an unknown node");
        g.bface_nodes.push_back(v);
      }
      g.bface_off.push_back((int64_t)g.bface_nodes.size());
      int grp = -1;
      for (int j = 0; j < n_phys; ++j)
        if (groups[j].dim == 2 && groups[j].tag == e.phys) { grp = j; break; }
      if (n_phys > 0 && grp < 0)
        return fail(-2, "boundary element with physical tag " + std::to_string(e.phys) +
                            " belongs to no 2-D physical group");
      face_group.push_back(grp);
    }
  }
  // build_patches: the 2-D groups that hold faces, in group order
  if (n_phys == 0) {
    if (!face_group.empty()) g.patch_names.push_back("boundary");
    g.bface_patch.assign(face_group.size(), 0);
  } else {
    std::vector<int64_t> count(n_phys, 0);
    for (int j : face_group) count[j]++;
    std::vector<int> compact(n_phys, -1);
    for (int j = 0; j < n_phys; ++j)
      if (count[j] > 0) {
        compact[j] = (int)g.patch_names.size();
        g.patch_names.push_back(groups[j].name);
      }
    g.bface_patch.resize(face_group.size());
    for (size_t i = 0; i < face_group.size(); ++i) g.bface_patch[i] = compact[face_group[i]];
  }
  return 0;
}

int write_gmsh(const std::string& path, const GmshMesh& g, std::string* err) {
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) {
    if (err) *err = "cannot create file: " + path;
    return -1;
  }
  const int np = (int)g.patch_names.size();
  const int64_t nn = (int64_t)g.xyz.size() / 3, nc = (int64_t)g.cell_type.size(), nb = (int64_t)g.bface_patch.size();
  std::fprintf(f, "$MeshFormat\n4.1 0 8\n$EndMeshFormat\n$PhysicalNames\n%d\n", np + 1);
  for (int p = 0; p < np; ++p) std::fprintf(f, "2 %d \"%s\"\n", p + 1, g.patch_names[p].c_str());
  std::fprintf(f, "3 %d \"fluid\"\n$EndPhysicalNames\n$Entities\n0 0 %d 1\n", np + 1, np);
  for (int p = 0; p < np; ++p) std::fprintf(f, "%d 0 0 0 0 0 0 1 %d 0\n", p + 1, p + 1);
  std::fprintf(f, "1 0 0 0 0 0 0 1 %d 0\n$EndEntities\n", np + 1);
  std::fprintf(f, "$Nodes\n1 %lld 1 %lld\n3 1 0 %lld\n", (long long)nn, (long long)nn, (long long)nn);
  for (int64_t i = 0; i < nn; ++i) std::fprintf(f, "%lld\n", (long long)(i + 1));
  for (int64_t i = 0; i < nn; ++i)
    std::fprintf(f, "%.17g %.17g %.17g\n", g.xyz[3 * i], g.xyz[3 * i + 1], g.xyz[3 * i + 2]);
  std::fprintf(f, "$EndNodes\n");
  // element blocks: runs of one type; boundary faces patch by patch in their order, then cells
  struct Block { int dim, tag, type; std::vector<int64_t> items; };
  std::vector<Block> blocks;
  for (int p = 0; p < np; ++p)
    for (int64_t b = 0; b < nb; ++b) {
      if (g.bface_patch[b] != p) continue;
      int t = (g.bface_off[b + 1] - g.bface_off[b]) == 3 ? G_TRI3 : G_QUAD4;
      if (blocks.empty() || blocks.back().dim != 2 || blocks.back().tag != p + 1 || blocks.back().type != t)
        blocks.push_back({2, p + 1, t, {}});
      blocks.back().items.push_back(b);
    }
  for (int64_t c = 0; c < nc; ++c) {
    int t = g.cell_type[c];  // ElemType codes are the gmsh first-order codes
    if (blocks.empty() || blocks.back().dim != 3 || blocks.back().type != t) blocks.push_back({3, 1, t, {}});
    blocks.back().items.push_back(c);
  }
  std::fprintf(f, "$Elements\n%zu %lld 1 %lld\n", blocks.size(), (long long)(nb + nc), (long long)(nb + nc));
  long long tag = 1;
  for (const Block& bl : blocks) {
    std::fprintf(f, "%d %d %d %zu\n", bl.dim, bl.tag, bl.type, bl.items.size());
    for (int64_t i : bl.items) {
      std::fprintf(f, "%lld", tag++);
      if (bl.dim == 2)
        for (int64_t k = g.bface_off[i]; k < g.bface_off[i + 1]; ++k) std::fprintf(f, " %d", g.bface_nodes[k] + 1);
      else
        for (int64_t k = g.cell_off[i]; k < g.cell_off[i + 1]; ++k) std::fprintf(f, " %d", g.cell_nodes[k] + 1);
      std::fprintf(f, "\n");
    }
  }
  std::fprintf(f, "$EndElements\n");
  bool ok = std::fclose(f) == 0;
  if (!ok && err) *err = "write failed: " + path;
  return ok ? 0 : -1;
}

}  // namespace dpm

// ---- C-ABI ------------------------------------------------------------------------------------

struct dpm_gmsh {
  dpm::GmshMesh g;
};

extern "C" int dpm_gmsh_read(const char* path, dpm_gmsh_t** out, char* errbuf, int errlen) {
  if (!path || !out) return DPM_ERR_ARG;
  *out = nullptr;
  auto* h = new dpm_gmsh();
  std::string err;
  int rc = dpm::read_gmsh(path, h->g, &err);
  if (rc) {
    delete h;
    if (errbuf && errlen > 0) std::snprintf(errbuf, (size_t)errlen, "%s", err.c_str());
    return rc == -1 ? DPM_ERR_ARG : DPM_ERR_MESH;
  }
  *out = h;
  return DPM_OK;
}

extern "C" int dpm_gmsh_sizes(const dpm_gmsh_t* h, int64_t* n_nodes, int64_t* n_cells, int64_t* n_cell_nodes,
                              int64_t* n_bfaces, int64_t* n_bface_nodes, int* n_patches) {
  if (!h) return DPM_ERR_ARG;
  const auto& g = h->g;
  if (n_nodes) *n_nodes = (int64_t)g.xyz.size() / 3;
  if (n_cells) *n_cells = (int64_t)g.cell_type.size();
  if (n_cell_nodes) *n_cell_nodes = (int64_t)g.cell_nodes.size();
  if (n_bfaces) *n_bfaces = (int64_t)g.bface_patch.size();
  if (n_bface_nodes) *n_bface_nodes = (int64_t)g.bface_nodes.size();
  if (n_patches) *n_patches = (int)g.patch_names.size();
  return DPM_OK;
}

extern "C" int dpm_gmsh_fill(const dpm_gmsh_t* h, double* xyz, int* cell_type, int64_t* cell_off, int* cell_nodes,
                             int64_t* bface_off, int* bface_nodes, int* bface_patch) {
  if (!h) return DPM_ERR_ARG;
  const auto& g = h->g;
  auto cp = [](auto* dst, const auto& v) {
    if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
  };
  cp(xyz, g.xyz); cp(cell_type, g.cell_type); cp(cell_off, g.cell_off); cp(cell_nodes, g.cell_nodes);
  cp(bface_off, g.bface_off); cp(bface_nodes, g.bface_nodes); cp(bface_patch, g.bface_patch);
  return DPM_OK;
}

extern "C" const char* dpm_gmsh_patch_name(const dpm_gmsh_t* h, int k) {
  if (!h || k < 0 || k >= (int)h->g.patch_names.size()) return nullptr;
  return h->g.patch_names[k].c_str();
}

extern "C" int dpm_gmsh_free(dpm_gmsh_t* h) {
  if (!h) return DPM_ERR_ARG;
  delete h;
  return DPM_OK;
}

extern "C" int dpm_gmsh_write(const char* path, const dpm_raw_mesh_t* m, const char* const* patch_names) {
  if (!path || !m || (m->n_patches > 0 && !patch_names)) return DPM_ERR_ARG;
  dpm::GmshMesh g;
  g.xyz.assign(m->xyz, m->xyz + 3 * m->n_nodes);
  g.cell_type.assign(m->cell_type, m->cell_type + m->n_cells);
  g.cell_off.assign(m->cell_off, m->cell_off + m->n_cells + 1);
  g.cell_nodes.assign(m->cell_nodes, m->cell_nodes + m->cell_off[m->n_cells]);
  g.bface_off.assign(m->bface_off, m->bface_off + m->n_bfaces + 1);
  g.bface_nodes.assign(m->bface_nodes, m->bface_nodes + m->bface_off[m->n_bfaces]);
  g.bface_patch.assign(m->bface_patch, m->bface_patch + m->n_bfaces);
  for (int p = 0; p < m->n_patches; ++p) g.patch_names.push_back(patch_names[p] ? patch_names[p] : "");
  std::string err;
  return dpm::write_gmsh(path, g, &err) ? DPM_ERR_ARG : DPM_OK;
}
