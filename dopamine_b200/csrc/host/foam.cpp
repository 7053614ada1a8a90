// OpenFOAM polyMesh reader, src/mesh/mod_foam_reader.f90:foam_read and its file readers: points,
// faces, owner, neighbour and boundary of a polyMesh directory, ASCII or binary (byte order and
// label / scalar sizes from the header's arch entry; faces as a faceList or a faceCompactList),
// as the face-based arrays of dpm_create_poly.  Mesh ingestion is host work; the set-up of the
// mesh itself is on the device (setup_gpu.cu) or in build_mesh_poly (mesh.cpp).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <string_view>
#include <vector>

#include "../../../include/dopamine_b200.h"
#include "mesh.hpp"

namespace dpm {

struct FoamMesh {
  std::vector<double> xyz;
  std::vector<int64_t> face_off{0};
  std::vector<int> face_nodes, owner, neighbour;
  std::vector<std::string> patch_name, patch_type;
  std::vector<int64_t> patch_start, patch_nfaces;
};

namespace {

// Tokens of an OpenFOAM dictionary file: words and numbers, and ( ) { } ; as single tokens;
// // and /* */ comments skipped.
struct Toks {
  std::string text;
  size_t p = 0;
  bool read(const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    if (!in) return false;
    text.assign((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    return true;
  }
  void skip() {
    for (;;) {
      while (p < text.size() && (text[p] == ' ' || text[p] == '\t' || text[p] == '\n' || text[p] == '\r')) ++p;
      if (p + 1 < text.size() && text[p] == '/' && text[p + 1] == '/') {
        while (p < text.size() && text[p] != '\n') ++p;
        continue;
      }
      if (p + 1 < text.size() && text[p] == '/' && text[p + 1] == '*') {
        size_t e = text.find("*/", p + 2);
        p = e == std::string::npos ? text.size() : e + 2;
        continue;
      }
      break;
    }
  }
  bool next(std::string_view& t) {
    skip();
    if (p >= text.size()) return false;
    const char ch = text[p];
    if (ch == '(' || ch == ')' || ch == '{' || ch == '}' || ch == ';') {
      t = std::string_view(&text[p], 1);
      ++p;
      return true;
    }
    size_t s = p;
    if (ch == '"') {  // quoted word
      ++p;
      while (p < text.size() && text[p] != '"') ++p;
      if (p < text.size()) ++p;
    } else {
      while (p < text.size() && !std::strchr(" \t\r\n(){};", text[p])) ++p;
    }
    t = std::string_view(&text[s], p - s);
    return true;
  }
};

bool to_ll(std::string_view t, long long& v) {
  if (t.empty() || t.size() > 30) return false;
  char buf[32];
  std::memcpy(buf, t.data(), t.size());
  buf[t.size()] = 0;
  char* e = nullptr;
  v = std::strtoll(buf, &e, 10);
  return *e == 0;
}
bool to_d(std::string_view t, double& v) {
  if (t.empty() || t.size() > 60) return false;
  char buf[64];
  std::memcpy(buf, t.data(), t.size());
  buf[t.size()] = 0;
  char* e = nullptr;
  v = std::strtod(buf, &e);
  return *e == 0;
}

// Header facts of a polyMesh file (foam_probe_file): format, byte order and label / scalar
// sizes of binary data, class.
struct Arch {
  bool binary = false, little = true;
  int label = 4, scalar = 8;
  std::string cls;
};

// Opens a polyMesh file and moves past its FoamFile header (foam_skip_header), reading the format,
// arch and class entries.
int open_list(Toks& T, const std::string& path, std::string* err, Arch& A) {
  if (!T.read(path)) {
    if (err) *err = "cannot open " + path;
    return -1;
  }
  std::string_view t;
  size_t save = T.p;
  if (T.next(t) && t == "FoamFile") {
    if (!T.next(t) || t != "{") {
      if (err) *err = "malformed FoamFile header in " + path;
      return -2;
    }
    std::string key;
    int depth = 1;
    while (depth > 0 && T.next(t)) {
      if (t == "{") ++depth;
      else if (t == "}") --depth;
      else if (t == ";") key.clear();
      else if (key.empty()) key = std::string(t);
      else if (key == "format") A.binary = t == "binary";
      else if (key == "class") A.cls = std::string(t);
      else if (key == "arch") {
        const std::string a(t);
        if (a.find("MSB") != std::string::npos) A.little = false;
        if (a.find("label=64") != std::string::npos) A.label = 8;
        if (a.find("scalar=32") != std::string::npos) A.scalar = 4;
      }
    }
  } else {
    T.p = save;
  }
  return 0;
}

// "N (" of a list; N >= 0.  In a binary file the data starts right after '(' (no whitespace is
// skipped there: a value's first byte may look like whitespace).
bool list_head(Toks& T, long long& n) {
  std::string_view t;
  if (!T.next(t) || !to_ll(t, n) || n < 0) return false;
  return T.next(t) && t == "(";
}

// Raw binary label / scalar at the cursor, in the file's byte order.
bool raw_bytes(Toks& T, const Arch& A, int size, unsigned char* out) {
  if (T.p + size > T.text.size()) return false;
  for (int i = 0; i < size; ++i) out[i] = (unsigned char)T.text[T.p + (A.little ? i : size - 1 - i)];
  T.p += size;
  return true;
}
bool raw_label(Toks& T, const Arch& A, long long& v) {
  unsigned char b[8];
  if (!raw_bytes(T, A, A.label, b)) return false;
  if (A.label == 8) {
    int64_t x;
    std::memcpy(&x, b, 8);
    v = x;
  } else {
    int32_t x;
    std::memcpy(&x, b, 4);
    v = x;
  }
  return true;
}
bool raw_scalar(Toks& T, const Arch& A, double& v) {
  unsigned char b[8];
  if (!raw_bytes(T, A, A.scalar, b)) return false;
  if (A.scalar == 8) {
    std::memcpy(&v, b, 8);
  } else {
    float x;
    std::memcpy(&x, b, 4);
    v = x;
  }
  return true;
}
bool label_at(Toks& T, const Arch& A, long long& v) {
  if (A.binary) return raw_label(T, A, v);
  std::string_view t;
  return T.next(t) && to_ll(t, v);
}

int read_labels(const std::string& path, std::vector<int>& out, std::string* err) {
  Toks T;
  Arch A;
  int rc = open_list(T, path, err, A);
  if (rc) return rc;
  long long n;
  std::string_view t;
  if (!list_head(T, n)) {
    if (err) *err = "malformed label list in " + path;
    return -2;
  }
  out.resize(n);
  for (long long i = 0; i < n; ++i) {
    long long v;
    if (!label_at(T, A, v)) {
      if (err) *err = "malformed label in " + path;
      return -2;
    }
    out[i] = (int)v;
  }
  if (!T.next(t) || t != ")") {
    if (err) *err = "label list of " + path + " does not end after its count";
    return -2;
  }
  return 0;
}

}  // namespace

int read_foam(const std::string& dir, FoamMesh& M, std::string* err) {
  M = FoamMesh();
  std::string_view t;
  auto fail = [&](const std::string& msg) {
    if (err) *err = msg;
    return -2;
  };
  {  // points: N ( (x y z) ... ), or N raw scalar triples in a binary file
    Toks T;
    Arch A;
    int rc = open_list(T, dir + "/points", err, A);
    if (rc) return rc;
    long long n;
    if (!list_head(T, n)) return fail("malformed point list in " + dir + "/points");
    M.xyz.resize(3 * n);
    for (long long i = 0; i < n; ++i) {
      if (A.binary) {
        for (int k = 0; k < 3; ++k)
          if (!raw_scalar(T, A, M.xyz[3 * i + k])) return fail("truncated binary points in " + dir + "/points");
        continue;
      }
      if (!T.next(t) || t != "(") return fail("malformed point in " + dir + "/points");
      for (int k = 0; k < 3; ++k)
        if (!T.next(t) || !to_d(t, M.xyz[3 * i + k])) return fail("malformed coordinate in " + dir + "/points");
      if (!T.next(t) || t != ")") return fail("malformed point in " + dir + "/points");
    }
    if (A.binary && (!T.next(t) || t != ")")) return fail("binary point list of " + dir + "/points does not end");
  }
  {  // faces: a faceList N ( k(a b ...) ... ), or a faceCompactList (offsets N+1, then the
     // concatenated node labels); in binary files the compact form is recognised by its leading
     // 0 label as well (foam_read_faces_binary)
    Toks T;
    Arch A;
    int rc = open_list(T, dir + "/faces", err, A);
    if (rc) return rc;
    long long n;
    if (!list_head(T, n)) return fail("malformed face list in " + dir + "/faces");
    bool compact = A.cls == "faceCompactList";
    if (A.binary && !compact && n >= 2) {
      const size_t save = T.p;
      long long first;
      if (!raw_label(T, A, first)) return fail("truncated binary faces in " + dir + "/faces");
      T.p = save;
      compact = first == 0;
    }
    if (compact) {
      if (n < 1) return fail("compact-face offset table too small in " + dir + "/faces");
      M.face_off.resize(n);
      for (long long i = 0; i < n; ++i) {
        long long v;
        if (!label_at(T, A, v)) return fail("malformed compact-face offset in " + dir + "/faces");
        M.face_off[i] = v;
        if ((i == 0 && v != 0) || (i > 0 && v < M.face_off[i - 1]))
          return fail("compact-face offsets must start at 0 and not decrease in " + dir + "/faces");
      }
      long long m2;
      if (!T.next(t) || t != ")" || !list_head(T, m2)) return fail("malformed compact-face lists in " + dir + "/faces");
      if (m2 != M.face_off[n - 1]) return fail("compact offsets mismatch in " + dir + "/faces");
      M.face_nodes.resize(m2);
      for (long long j = 0; j < m2; ++j) {
        long long v;
        if (!label_at(T, A, v)) return fail("malformed compact-face node in " + dir + "/faces");
        M.face_nodes[j] = (int)v;
      }
    } else {
      M.face_off.reserve(n + 1);
      for (long long i = 0; i < n; ++i) {
        long long k;
        if (A.binary) {
          if (!raw_label(T, A, k) || k < 0) return fail("malformed binary face in " + dir + "/faces");
          for (long long j = 0; j < k; ++j) {
            long long v;
            if (!raw_label(T, A, v)) return fail("truncated binary faces in " + dir + "/faces");
            M.face_nodes.push_back((int)v);
          }
        } else {
          if (!T.next(t) || !to_ll(t, k) || k < 0) return fail("malformed face size in " + dir + "/faces");
          if (!T.next(t) || t != "(") return fail("malformed face in " + dir + "/faces");
          for (long long j = 0; j < k; ++j) {
            long long v;
            if (!T.next(t) || !to_ll(t, v)) return fail("malformed face node in " + dir + "/faces");
            M.face_nodes.push_back((int)v);
          }
          if (!T.next(t) || t != ")") return fail("malformed face in " + dir + "/faces");
        }
        M.face_off.push_back((int64_t)M.face_nodes.size());
      }
    }
  }
  int rc = read_labels(dir + "/owner", M.owner, err);
  if (rc) return rc;
  rc = read_labels(dir + "/neighbour", M.neighbour, err);
  if (rc) return rc;
  if (M.owner.size() != M.face_off.size() - 1) return fail("owner and faces lists differ in length");
  if (M.neighbour.size() > M.owner.size()) return fail("more neighbours than faces");
  {  // boundary: N ( name { type t; nFaces n; startFace s; ... } ... )
    Toks T;
    Arch A;
    rc = open_list(T, dir + "/boundary", err, A);
    if (rc) return rc;
    long long n;
    if (!list_head(T, n)) return fail("malformed patch list in " + dir + "/boundary");
    for (long long i = 0; i < n; ++i) {
      if (!T.next(t)) return fail("truncated patch list in " + dir + "/boundary");
      std::string name(t);
      if (!T.next(t) || t != "{") return fail("malformed patch entry in " + dir + "/boundary");
      std::string type = "patch";
      long long nfc = 0, start = 0;
      std::string key;
      std::vector<std::string> vals;
      int depth = 1;
      while (depth > 0) {
        if (!T.next(t)) return fail("truncated patch entry in " + dir + "/boundary");
        if (t == "{" || t == "(") { ++depth; continue; }
        if (t == "}" || t == ")") { --depth; continue; }
        if (depth > 1) continue;  // nested lists and dictionaries (inGroups, ...) are skipped
        if (t == ";") {
          if (!vals.empty()) {
            if (key == "type") type = vals[0];
            else if (key == "nFaces" && !to_ll(vals[0], nfc)) return fail("malformed nFaces in " + dir + "/boundary");
            else if (key == "startFace" && !to_ll(vals[0], start)) return fail("malformed startFace in " + dir + "/boundary");
          }
          key.clear();
          vals.clear();
        } else if (key.empty()) {
          key = std::string(t);
        } else {
          vals.emplace_back(t);
        }
      }
      M.patch_name.push_back(name);
      M.patch_type.push_back(type);
      M.patch_start.push_back(start);
      M.patch_nfaces.push_back(nfc);
    }
  }
  return 0;
}

}  // namespace dpm

// ---- C-ABI ------------------------------------------------------------------------------------

struct dpm_foam {
  dpm::FoamMesh m;
};

extern "C" int dpm_foam_read(const char* polymesh_dir, dpm_foam_t** out, char* errbuf, int errlen) {
  if (!polymesh_dir || !out) return DPM_ERR_ARG;
  *out = nullptr;
  auto* h = new dpm_foam();
  std::string err;
  int rc = dpm::read_foam(polymesh_dir, h->m, &err);
  if (rc) {
    delete h;
    if (errbuf && errlen > 0) std::snprintf(errbuf, (size_t)errlen, "%s", err.c_str());
    return rc == -1 ? DPM_ERR_ARG : DPM_ERR_MESH;
  }
  *out = h;
  return DPM_OK;
}

extern "C" int dpm_foam_sizes(const dpm_foam_t* h, int64_t* n_points, int64_t* n_faces, int64_t* n_face_nodes,
                              int64_t* n_int_faces, int* n_patches) {
  if (!h) return DPM_ERR_ARG;
  const auto& m = h->m;
  if (n_points) *n_points = (int64_t)m.xyz.size() / 3;
  if (n_faces) *n_faces = (int64_t)m.owner.size();
  if (n_face_nodes) *n_face_nodes = (int64_t)m.face_nodes.size();
  if (n_int_faces) *n_int_faces = (int64_t)m.neighbour.size();
  if (n_patches) *n_patches = (int)m.patch_name.size();
  return DPM_OK;
}

extern "C" int dpm_foam_fill(const dpm_foam_t* h, double* xyz, int64_t* face_off, int* face_nodes, int* owner,
                             int* neighbour, int64_t* patch_start, int64_t* patch_nfaces) {
  if (!h) return DPM_ERR_ARG;
  const auto& m = h->m;
  auto cp = [](auto* dst, const auto& v) {
    if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
  };
  cp(xyz, m.xyz); cp(face_off, m.face_off); cp(face_nodes, m.face_nodes); cp(owner, m.owner);
  cp(neighbour, m.neighbour); cp(patch_start, m.patch_start); cp(patch_nfaces, m.patch_nfaces);
  return DPM_OK;
}

extern "C" const char* dpm_foam_patch_name(const dpm_foam_t* h, int k) {
  if (!h || k < 0 || k >= (int)h->m.patch_name.size()) return nullptr;
  return h->m.patch_name[k].c_str();
}

extern "C" const char* dpm_foam_patch_type(const dpm_foam_t* h, int k) {
  if (!h || k < 0 || k >= (int)h->m.patch_type.size()) return nullptr;
  return h->m.patch_type[k].c_str();
}

extern "C" int dpm_foam_free(dpm_foam_t* h) {
  if (!h) return DPM_ERR_ARG;
  delete h;
  return DPM_OK;
}

extern "C" int dpm_poly_cell_geometry(const dpm_poly_mesh_t* pm, const int* patch_bc, double* centroid, double* volume,
                                      char* errbuf, int errlen) {
  if (!pm || (pm->n_patches > 0 && !patch_bc)) return DPM_ERR_ARG;
  dpm::PolyMesh p;
  p.n_points = pm->n_points; p.xyz = pm->xyz; p.n_faces = pm->n_faces; p.face_off = pm->face_off;
  p.face_nodes = pm->face_nodes; p.owner = pm->owner; p.n_int_faces = pm->n_int_faces; p.neighbour = pm->neighbour;
  p.n_patches = pm->n_patches; p.patch_start = pm->patch_start; p.patch_nfaces = pm->patch_nfaces;
  dpm::Mesh m;
  std::string err;
  if (dpm::build_mesh_poly(p, patch_bc, m, &err)) {
    if (errbuf && errlen > 0) std::snprintf(errbuf, (size_t)errlen, "%s", err.c_str());
    return DPM_ERR_MESH;
  }
  if (centroid) std::memcpy(centroid, m.centroid.data(), m.centroid.size() * sizeof(double));
  if (volume) std::memcpy(volume, m.volume.data(), m.volume.size() * sizeof(double));
  return DPM_OK;
}
