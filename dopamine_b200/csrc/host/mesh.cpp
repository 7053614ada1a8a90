// Host mesh set-up; see mesh.hpp.  Every routine names the reference routine it restates.
#include "mesh.hpp"

#include <algorithm>
#include <parallel/algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <numeric>

namespace dpm {
namespace {

inline void cross3(const double a[3], const double b[3], double c[3]) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
inline double dot3(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// Local faces of each element type (src/mesh/mod_gmsh_reader.f90:get_element_faces, 0-based).
int element_faces(int type, const int* n, int fn[6][4], int nn[6]) {
  auto set = [&](int k, std::initializer_list<int> l) {
    int i = 0;
    for (int v : l) fn[k][i++] = n[v];
    nn[k] = i;
  };
  switch (type) {
    case EL_TET4:
      set(0, {0, 1, 2}); set(1, {0, 1, 3}); set(2, {1, 2, 3}); set(3, {0, 2, 3});
      return 4;
    case EL_HEX8:
      set(0, {0, 1, 2, 3}); set(1, {4, 5, 6, 7}); set(2, {0, 1, 5, 4});
      set(3, {2, 3, 7, 6}); set(4, {0, 3, 7, 4}); set(5, {1, 2, 6, 5});
      return 6;
    case EL_PRISM6:
      set(0, {0, 1, 2}); set(1, {3, 4, 5}); set(2, {0, 1, 4, 3}); set(3, {1, 2, 5, 4}); set(4, {0, 2, 5, 3});
      return 5;
    case EL_PYR5:
      set(0, {0, 1, 2, 3}); set(1, {0, 1, 4}); set(2, {1, 2, 4}); set(3, {2, 3, 4}); set(4, {0, 3, 4});
      return 5;
  }
  return 0;
}

// Exact tet centroid and volume (mod_gmsh_reader.f90:tet_geometry).
void tet_geometry(const double* p1, const double* p2, const double* p3, const double* p4, double c[3], double& v) {
  double a[3], b[3], d[3];
  for (int k = 0; k < 3; ++k) { a[k] = p2[k] - p1[k]; b[k] = p3[k] - p1[k]; d[k] = p4[k] - p1[k]; }
  v = std::fabs(a[0] * (b[1] * d[2] - b[2] * d[1]) - a[1] * (b[0] * d[2] - b[2] * d[0]) +
                a[2] * (b[0] * d[1] - b[1] * d[0])) / 6.0;
  for (int k = 0; k < 3; ++k) c[k] = (((p1[k] + p2[k]) + p3[k]) + p4[k]) / 4.0;
}

// Hex / prism / pyramid geometry by tet decomposition (mod_gmsh_reader.f90:hex_geometry etc).
void cell_geometry(int type, const int* n, const double* xyz, double c[3], double& vol) {
  static const int hex_t[5][4] = {{0, 1, 3, 4}, {1, 2, 3, 6}, {3, 4, 6, 7}, {1, 4, 5, 6}, {1, 3, 4, 6}};
  static const int pri_t[3][4] = {{0, 1, 2, 3}, {1, 3, 4, 2}, {2, 3, 4, 5}};
  static const int pyr_t[2][4] = {{0, 1, 3, 4}, {1, 2, 3, 4}};
  auto P = [&](int i) { return xyz + 3 * (int64_t)n[i]; };
  if (type == EL_TET4) {
    tet_geometry(P(0), P(1), P(2), P(3), c, vol);
    return;
  }
  const int(*t)[4] = nullptr;
  int nt = 0;
  if (type == EL_HEX8) { t = hex_t; nt = 5; }
  else if (type == EL_PRISM6) { t = pri_t; nt = 3; }
  else if (type == EL_PYR5) { t = pyr_t; nt = 2; }
  vol = 0.0;
  c[0] = c[1] = c[2] = 0.0;
  for (int i = 0; i < nt; ++i) {
    double tc[3], tv;
    tet_geometry(P(t[i][0]), P(t[i][1]), P(t[i][2]), P(t[i][3]), tc, tv);
    vol += tv;
    for (int k = 0; k < 3; ++k) c[k] += tv * tc[k];
  }
  if (vol > SMALL)
    for (int k = 0; k < 3; ++k) c[k] /= vol;
}

// Face centre (vertex mean) and area vector by a fan from the centre
// (mod_gmsh_reader.f90:compute_face_geometry).
void face_geometry(const int* fn, int nf, const double* xyz, double centre[3], double normal[3], double& area) {
  centre[0] = centre[1] = centre[2] = 0.0;
  for (int i = 0; i < nf; ++i)
    for (int k = 0; k < 3; ++k) centre[k] += xyz[3 * (int64_t)fn[i] + k];
  for (int k = 0; k < 3; ++k) centre[k] /= (double)nf;
  double acc[3] = {0, 0, 0};
  for (int i = 0; i < nf; ++i) {
    const double* pi = xyz + 3 * (int64_t)fn[i];
    const double* pj = xyz + 3 * (int64_t)fn[(i + 1) % nf];
    double a[3], b[3], cr[3];
    for (int k = 0; k < 3; ++k) { a[k] = pi[k] - centre[k]; b[k] = pj[k] - centre[k]; }
    cross3(a, b, cr);
    for (int k = 0; k < 3; ++k) acc[k] += 0.5 * cr[k];
  }
  area = std::sqrt(acc[0] * acc[0] + acc[1] * acc[1] + acc[2] * acc[2]);
  for (int k = 0; k < 3; ++k) normal[k] = acc[k] / (area + SMALL);
}

struct FaceKey {
  std::array<int, 4> k;
  bool operator<(const FaceKey& o) const { return k < o.k; }
  bool operator==(const FaceKey& o) const { return k == o.k; }
};

FaceKey canonical(const int* fn, int nf) {
  FaceKey key;
  key.k = {-1, -1, -1, -1};
  for (int i = 0; i < nf; ++i) key.k[i] = fn[i];
  for (int i = 1; i < nf; ++i) {  // insertion sort, as canonical_face_nodes
    int t = key.k[i], j = i - 1;
    while (j >= 0 && key.k[j] > t) { key.k[j + 1] = key.k[j]; --j; }
    key.k[j + 1] = t;
  }
  return key;
}

void invert3x3(const double A[3][3], double Ainv[3][3], double& det) {
  double c11 = A[1][1] * A[2][2] - A[1][2] * A[2][1];
  double c12 = -(A[1][0] * A[2][2] - A[1][2] * A[2][0]);
  double c13 = A[1][0] * A[2][1] - A[1][1] * A[2][0];
  double c21 = -(A[0][1] * A[2][2] - A[0][2] * A[2][1]);
  double c22 = A[0][0] * A[2][2] - A[0][2] * A[2][0];
  double c23 = -(A[0][0] * A[2][1] - A[0][1] * A[2][0]);
  double c31 = A[0][1] * A[1][2] - A[0][2] * A[1][1];
  double c32 = -(A[0][0] * A[1][2] - A[0][2] * A[1][0]);
  double c33 = A[0][0] * A[1][1] - A[0][1] * A[1][0];
  det = A[0][0] * c11 + A[0][1] * c12 + A[0][2] * c13;
  double m = std::max(std::fabs(det), SMALL);
  double idet = 1.0 / (det < 0 ? -m : m);
  Ainv[0][0] = c11 * idet; Ainv[0][1] = c21 * idet; Ainv[0][2] = c31 * idet;
  Ainv[1][0] = c12 * idet; Ainv[1][1] = c22 * idet; Ainv[1][2] = c32 * idet;
  Ainv[2][0] = c13 * idet; Ainv[2][1] = c23 * idet; Ainv[2][2] = c33 * idet;
}

// Periodic patch matching (src/bc/mod_bc_setup.f90:try_pair_patches).
bool try_pair(const Mesh& m, int p, int q, double& max_err, std::vector<int>& map) {
  int64_t n = m.patch_nfaces[p];
  if (n == 0 || n != m.patch_nfaces[q]) return false;
  std::vector<double> cp(3 * n), cq(3 * n);
  double sp[3] = {0, 0, 0}, sq[3] = {0, 0, 0}, np_[3] = {0, 0, 0}, nq[3] = {0, 0, 0};
  for (int64_t i = 0; i < n; ++i) {
    int64_t fp = m.n_int_faces + m.patch_start[p] + i, fq = m.n_int_faces + m.patch_start[q] + i;
    for (int k = 0; k < 3; ++k) {
      cp[3 * i + k] = m.centre[3 * fp + k];
      cq[3 * i + k] = m.centre[3 * fq + k];
    }
  }
  for (int64_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) {
      sp[k] += cp[3 * i + k];
      sq[k] += cq[3 * i + k];
      np_[k] += m.normal[3 * (m.n_int_faces + m.patch_start[p] + i) + k];
      nq[k] += m.normal[3 * (m.n_int_faces + m.patch_start[q] + i) + k];
    }
  double shift[3];
  for (int k = 0; k < 3; ++k) shift[k] = sq[k] / (double)n - sp[k] / (double)n;
  double avg_dot = dot3(np_, nq);
  double scale = 1.0;
  for (int64_t i = 0; i < 3 * n; ++i) scale = std::max(scale, std::max(std::fabs(cp[i]), std::fabs(cq[i])));
  double tol = 1.0e-5 * scale;
  const double KC1 = 3.14159265358979, KC2 = 2.71828182845904, KC3 = 1.41421356237310;
  std::vector<double> kp(n), kq(n);
  std::vector<int> op(n), oq(n);
  for (int64_t i = 0; i < n; ++i) {
    kp[i] = KC1 * (cp[3 * i] + shift[0]) + KC2 * (cp[3 * i + 1] + shift[1]) + KC3 * (cp[3 * i + 2] + shift[2]);
    kq[i] = KC1 * cq[3 * i] + KC2 * cq[3 * i + 1] + KC3 * cq[3 * i + 2];
    op[i] = oq[i] = (int)i;
  }
  std::sort(op.begin(), op.end(), [&](int a, int b) { return kp[a] < kp[b] || (kp[a] == kp[b] && a < b); });
  std::sort(oq.begin(), oq.end(), [&](int a, int b) { return kq[a] < kq[b] || (kq[a] == kq[b] && a < b); });
  map.assign(n, -1);
  max_err = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    map[op[i]] = oq[i];
    double d2 = 0;
    for (int k = 0; k < 3; ++k) {
      double d = cq[3 * oq[i] + k] - (cp[3 * op[i] + k] + shift[k]);
      d2 += d * d;
    }
    max_err = std::max(max_err, std::sqrt(d2));
  }
  return max_err <= tol && avg_dot < 0.0;
}

}  // namespace

void build_cell_faces(Mesh& m) {
  const int64_t nc = m.n_cells, nf = m.n_faces;
  // Cell -> face CSR (mod_mesh.f90:mesh_build_connectivity).
  m.cell_face_off.assign(nc + 1, 0);
  for (int64_t f = 0; f < nf; ++f) {
    m.cell_face_off[m.owner[f] + 1]++;
    if (m.neighbour[f] >= 0) m.cell_face_off[m.neighbour[f] + 1]++;
  }
  for (int64_t c = 0; c < nc; ++c) m.cell_face_off[c + 1] += m.cell_face_off[c];
  m.cell_faces.assign(m.cell_face_off[nc], -1);
  {
    std::vector<int64_t> cur(m.cell_face_off.begin(), m.cell_face_off.end() - 1);
    for (int64_t f = 0; f < nf; ++f) {
      m.cell_faces[cur[m.owner[f]]++] = (int)f;
      if (m.neighbour[f] >= 0) m.cell_faces[cur[m.neighbour[f]]++] = (int)f;
    }
  }
}

int build_periodic(Mesh& m, std::string* err) {
  const int64_t nfi = m.n_int_faces, nfb = m.n_bnd_faces;
  // Periodic pairing (src/bc/mod_bc_setup.f90:build_periodic_pairs).
  m.periodic_pair.assign(nfb, -1);
  m.periodic_pair_dcf.assign(nfb, 0.0);
  std::vector<int> per;
  for (int p = 0; p < m.n_patches; ++p)
    if (m.patch_bc[p] == BC_PERIODIC) per.push_back(p);
  if (!per.empty()) {
    std::vector<uint8_t> used(m.n_patches, 0);
    for (size_t i = 0; i < per.size(); ++i) {
      int p = per[i];
      if (used[p]) continue;
      int best_q = -1;
      double best_err = 1e300;
      std::vector<int> best_map, map;
      for (size_t j = i + 1; j < per.size(); ++j) {
        int q = per[j];
        if (used[q]) continue;
        double e;
        if (try_pair(m, p, q, e, map) && e < best_err) {
          best_err = e;
          best_q = q;
          best_map = map;
        }
      }
      if (best_q < 0) {
        if (err) *err = "no periodic partner for a periodic patch";
        return -4;
      }
      for (int64_t k = 0; k < (int64_t)best_map.size(); ++k) {
        int64_t fbp = m.patch_start[p] + k, fbq = m.patch_start[best_q] + best_map[k];
        m.periodic_pair[fbp] = (int)fbq;
        m.periodic_pair[fbq] = (int)fbp;
        m.periodic_pair_dcf[fbp] = m.d_cf[nfi + fbq];
        m.periodic_pair_dcf[fbq] = m.d_cf[nfi + fbp];
      }
      used[p] = used[best_q] = 1;
    }
    // finalize_periodic_partner_metrics
    for (int64_t b = 0; b < nfb; ++b) {
      if (m.periodic_pair_dcf[b] > 0.0) continue;
      if (m.periodic_pair[b] >= 0) m.periodic_pair_dcf[b] = m.d_cf[nfi + m.periodic_pair[b]];
      if (m.periodic_pair_dcf[b] <= 0.0) m.periodic_pair_dcf[b] = m.d_cf[nfi + b];
    }
  }
  // Periodic interpolation weight (mod_mesh.f90:mesh_build_soa_mirror).
  m.periodic_gc.assign(nfb, 0.5);
  for (int64_t b = 0; b < nfb; ++b)
    if (m.periodic_pair_dcf[b] > 0.0)
      m.periodic_gc[b] = m.periodic_pair_dcf[b] / (m.d_cf[nfi + b] + m.periodic_pair_dcf[b] + SMALL);

  return 0;
}

// The part of the set-up that both the element path (build_mesh) and the polyhedral path
// (build_mesh_poly) share, once faces (owner, neighbour, patch, area, centre, normal), cells
// (centroid, volume, vertex lists) and patches are in m: cell -> face lists, face metrics,
// periodic pairing, LS stencil.
int finish_mesh(Mesh& m, std::string* err) {
  const int64_t nc = m.n_cells, nf = m.n_faces, nfi = m.n_int_faces, nfb = m.n_bnd_faces;
  build_cell_faces(m);

  // Face geometry (mod_mesh.f90:mesh_compute_geometry, mesh_tag_refinement_faces).
  m.sf.assign(3 * nf, 0.0);
  m.d_cf.assign(nf, 0.0);
  m.gc.assign(nf, 0.0);
  m.eps.assign(3 * nf, 0.0);
  m.skew.assign(nf, 0.0);
  m.is_refine.assign(nf, 0);
#pragma omp parallel for schedule(static)
  for (int64_t f = 0; f < nf; ++f) {
    for (int k = 0; k < 3; ++k) m.sf[3 * f + k] = m.area[f] * m.normal[3 * f + k];
    const double* co = &m.centroid[3 * (int64_t)m.owner[f]];
    const double* ce = &m.centre[3 * f];
    if (m.neighbour[f] >= 0) {
      const double* cn = &m.centroid[3 * (int64_t)m.neighbour[f]];
      double d_on[3], d_oc[3];
      for (int k = 0; k < 3; ++k) { d_on[k] = cn[k] - co[k]; d_oc[k] = ce[k] - co[k]; }
      double d_on2 = d_on[0] * d_on[0] + d_on[1] * d_on[1] + d_on[2] * d_on[2];
      m.d_cf[f] = std::max(std::sqrt(d_on2), 1.0e-30);
      double w = dot3(d_oc, d_on) / (d_on2 + SMALL);
      m.gc[f] = std::max(0.0, std::min(1.0, 1.0 - w));
      double em[3], s2 = 0.0;
      for (int k = 0; k < 3; ++k) {
        m.eps[3 * f + k] = ce[k] - (co[k] + (1.0 - m.gc[f]) * (cn[k] - co[k]));
        em[k] = ce[k] - 0.5 * (co[k] + cn[k]);
        s2 += em[k] * em[k];
      }
      m.skew[f] = std::sqrt(s2) / std::max(m.d_cf[f], 1.0e-30);
      m.is_refine[f] = m.skew[f] > REFINE_SKEW_TOL;
    } else {
      double d[3];
      for (int k = 0; k < 3; ++k) d[k] = ce[k] - co[k];
      m.d_cf[f] = std::max(std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]), 1.0e-30);
      m.gc[f] = 1.0;
    }
  }

  {
    int rc = build_periodic(m, err);
    if (rc) return rc;
  }
  // Least-squares stencil: face neighbours (periodic partners across seams), then
  // vertex-sharing cells, inverse-distance weights (mod_mesh.f90:mesh_build_ls_stencil).
  int max_faces = 1;
  for (int64_t c = 0; c < nc; ++c) max_faces = std::max<int>(max_faces, (int)(m.cell_face_off[c + 1] - m.cell_face_off[c]));
  const int max_stencil = std::max(32, 4 * max_faces);
  std::vector<int> cnt(nc, 0), tnb((size_t)nc * max_stencil, -1), tface((size_t)nc * max_stencil, -1);
  std::vector<uint8_t> tper((size_t)nc * max_stencil, 0);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < nc; ++i) {
    for (int64_t idx = m.cell_face_off[i]; idx < m.cell_face_off[i + 1]; ++idx) {
      int f = m.cell_faces[idx];
      int nb = m.owner[f];
      if (nb == i) nb = m.neighbour[f];
      bool is_per = false;
      if (nb < 0) {
        int64_t fb = f - nfi;
        int p = m.patch[f];
        if (p >= 0 && m.patch_bc[p] == BC_PERIODIC) {
          int pb = m.periodic_pair[fb];
          if (pb >= 0) nb = m.owner[nfi + pb];
          if (nb >= 0) is_per = true;
        }
        if (nb < 0) nb = -1;
      }
      size_t s = (size_t)i * max_stencil + cnt[i]++;
      tnb[s] = nb;
      tper[s] = is_per;
      if (nb == -1) tface[s] = f;
    }
  }
  {
    const int64_t nv = m.n_vertices;
    const int64_t* coff = m.cell_vert_off.data();
    const int* cnodes = m.cell_vertices.data();
    std::vector<int64_t> voff(nv + 1, 0);
    for (int64_t c = 0; c < nc; ++c)
      for (int64_t k = coff[c]; k < coff[c + 1]; ++k) voff[cnodes[k] + 1]++;
    for (int64_t v = 0; v < nv; ++v) voff[v + 1] += voff[v];
    std::vector<int> vcell(voff[nv]);
    std::vector<int64_t> vp(voff.begin(), voff.end() - 1);
    for (int64_t c = 0; c < nc; ++c)
      for (int64_t k = coff[c]; k < coff[c + 1]; ++k) vcell[vp[cnodes[k]]++] = (int)c;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nc; ++i) {
      int* nbs = &tnb[(size_t)i * max_stencil];
      for (int64_t k = coff[i]; k < coff[i + 1]; ++k) {
        int v = cnodes[k];
        for (int64_t kk = voff[v]; kk < voff[v + 1]; ++kk) {
          int cnb = vcell[kk];
          if (cnb == i) continue;
          bool found = false;
          for (int j = 0; j < cnt[i]; ++j)
            if (nbs[j] == cnb) { found = true; break; }
          if (found) continue;
          if (cnt[i] < max_stencil) {
            size_t s = (size_t)i * max_stencil + cnt[i]++;
            tnb[s] = cnb;
            tper[s] = 0;
            tface[s] = -1;
          }
        }
      }
    }
  }
  m.ls_off.assign(nc + 1, 0);
  for (int64_t i = 0; i < nc; ++i) m.ls_off[i + 1] = m.ls_off[i] + cnt[i];
  const int64_t ns = m.ls_off[nc];
  m.ls_cell.assign(ns, -1);
  m.ls_face.assign(ns, -1);
  m.ls_w.assign(3 * ns, 0.0);
  int64_t n_deg = 0;
#pragma omp parallel for schedule(static) reduction(+ : n_deg)
  for (int64_t i = 0; i < nc; ++i) {
    const int64_t off = m.ls_off[i];
    auto offset_of = [&](int idx, double d[3]) {
      size_t s = (size_t)i * max_stencil + idx;
      int nb = tnb[s];
      const double* ci = &m.centroid[3 * i];
      if (nb >= 0 && tper[s]) {
        int f = m.cell_faces[m.cell_face_off[i] + idx];
        double dpo = m.d_cf[f], dpn = dpo;
        int64_t fb = f - nfi;
        if (fb >= 0 && fb < nfb && m.periodic_pair_dcf[fb] > 0.0) dpn = m.periodic_pair_dcf[fb];
        for (int k = 0; k < 3; ++k) d[k] = (dpo + dpn) * m.normal[3 * (int64_t)f + k];
      } else if (nb >= 0) {
        for (int k = 0; k < 3; ++k) d[k] = m.centroid[3 * (int64_t)nb + k] - ci[k];
      } else {
        int f = m.cell_faces[m.cell_face_off[i] + idx];
        for (int k = 0; k < 3; ++k) d[k] = m.centre[3 * (int64_t)f + k] - ci[k];
      }
    };
    double A[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int idx = 0; idx < cnt[i]; ++idx) {
      size_t s = (size_t)i * max_stencil + idx;
      m.ls_cell[off + idx] = tnb[s];
      m.ls_face[off + idx] = tface[s];
      double d[3];
      offset_of(idx, d);
      double w = 1.0 / (std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) + SMALL);
      double ww = w * w;
      A[0][0] += ww * d[0] * d[0]; A[0][1] += ww * d[0] * d[1];
      A[0][2] += ww * d[0] * d[2]; A[1][1] += ww * d[1] * d[1];
      A[1][2] += ww * d[1] * d[2]; A[2][2] += ww * d[2] * d[2];
    }
    A[1][0] = A[0][1]; A[2][0] = A[0][2]; A[2][1] = A[1][2];
    double scale = (A[0][0] + A[1][1] + A[2][2]) / 3.0;
    double Ai[3][3], det;
    invert3x3(A, Ai, det);
    if (scale <= 0.0 || std::fabs(det) < LS_DET_TOL * (scale * scale * scale)) {
      for (int k = 0; k < 3; ++k) A[k][k] += LS_REG_FRAC * std::max(scale, SMALL);
      invert3x3(A, Ai, det);
      n_deg++;
    }
    for (int idx = 0; idx < cnt[i]; ++idx) {
      double d[3];
      offset_of(idx, d);
      double w = 1.0 / (std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) + SMALL);
      double r[3] = {w * w * d[0], w * w * d[1], w * w * d[2]};
      for (int k = 0; k < 3; ++k) m.ls_w[3 * (off + idx) + k] = Ai[k][0] * r[0] + Ai[k][1] * r[1] + Ai[k][2] * r[2];
    }
  }
  m.ls_degenerate = n_deg;
  return 0;
}

int build_mesh(const RawMesh& raw, const int* patch_bc, Mesh& m, std::string* err) {
  auto fail = [&](int code, const char* msg) {
    if (err) *err = msg;
    return code;
  };
  const int64_t nc = raw.n_cells;
  m = Mesh();
  m.n_cells = nc;
  m.n_patches = raw.n_patches;
  m.n_vertices = raw.n_nodes;
  m.vertices.assign(raw.xyz, raw.xyz + 3 * raw.n_nodes);
  m.cell_vert_off.assign(raw.cell_off, raw.cell_off + nc + 1);
  m.cell_vertices.assign(raw.cell_nodes, raw.cell_nodes + raw.cell_off[nc]);

  // Cell centroids and volumes (mod_gmsh_reader.f90:build_mesh_from_gmsh).
  m.centroid.assign(3 * nc, 0.0);
  m.volume.assign(nc, 0.0);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < nc; ++c)
    cell_geometry(raw.cell_type[c], raw.cell_nodes + raw.cell_off[c], raw.xyz, &m.centroid[3 * c], m.volume[c]);

  // Face matching.  The reference walks cells in order with a hash table; an interior face is
  // created when its second cell reaches it, so ordering (second cell, local face) reproduces
  // its face numbering (mod_gmsh_reader.f90:build_faces_from_cells).
  struct Rec { FaceKey key; int cell; int fi; };
  // (key, cell, local face) is a strict total order over distinct records, so any sort gives the
  // same sequence; the parallel one is used.
  std::vector<int64_t> roff(nc + 1, 0);
  int bad_type = 0;
#pragma omp parallel for schedule(static) reduction(| : bad_type)
  for (int64_t c = 0; c < nc; ++c) {
    int fn[6][4], nn[6];
    int nfc = element_faces(raw.cell_type[c], raw.cell_nodes + raw.cell_off[c], fn, nn);
    if (nfc == 0) bad_type = 1;
    roff[c + 1] = nfc;
  }
  if (bad_type) return fail(-1, "unsupported element type");
  for (int64_t c = 0; c < nc; ++c) roff[c + 1] += roff[c];
  std::vector<Rec> recs(roff[nc]);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < nc; ++c) {
    int fn[6][4], nn[6];
    int nfc = element_faces(raw.cell_type[c], raw.cell_nodes + raw.cell_off[c], fn, nn);
    for (int i = 0; i < nfc; ++i) recs[roff[c] + i] = {canonical(fn[i], nn[i]), (int)c, i};
  }
  __gnu_parallel::sort(recs.begin(), recs.end(), [](const Rec& a, const Rec& b) {
    if (a.key < b.key) return true;
    if (b.key < a.key) return false;
    return a.cell < b.cell || (a.cell == b.cell && a.fi < b.fi);
  });
  struct IntFace { int second_cell, second_fi, owner; };
  std::vector<IntFace> ifaces;
  std::vector<uint8_t> matched(recs.size(), 0);  // 1: part of an interior pair or a boundary face
  for (size_t i = 0; i < recs.size();) {
    size_t j = i + 1;
    while (j < recs.size() && recs[j].key == recs[i].key) ++j;
    if (j - i >= 2) {
      ifaces.push_back({recs[i + 1].cell, recs[i + 1].fi, recs[i].cell});
      for (size_t k = i; k < j; ++k) matched[k] = 1;
    }
    i = j;
  }
  __gnu_parallel::sort(ifaces.begin(), ifaces.end(), [](const IntFace& a, const IntFace& b) {
    return a.second_cell < b.second_cell || (a.second_cell == b.second_cell && a.second_fi < b.second_fi);
  });
  const int64_t nfi = (int64_t)ifaces.size();
  const int64_t nfb = raw.n_bfaces;
  const int64_t nf = nfi + nfb;
  m.n_int_faces = nfi;
  m.n_bnd_faces = nfb;
  m.n_faces = nf;
  m.owner.assign(nf, -1);
  m.neighbour.assign(nf, -1);
  m.patch.assign(nf, -1);
  m.area.assign(nf, 0.0);
  m.centre.assign(3 * nf, 0.0);
  m.normal.assign(3 * nf, 0.0);
#pragma omp parallel for schedule(static)
  for (int64_t f = 0; f < nfi; ++f) {
    const IntFace& F = ifaces[f];
    int fn[6][4], nn[6];
    element_faces(raw.cell_type[F.second_cell], raw.cell_nodes + raw.cell_off[F.second_cell], fn, nn);
    m.owner[f] = F.owner;
    m.neighbour[f] = F.second_cell;
    face_geometry(fn[F.second_fi], nn[F.second_fi], raw.xyz, &m.centre[3 * f], &m.normal[3 * f], m.area[f]);
    double d[3];
    for (int k = 0; k < 3; ++k) d[k] = m.centroid[3 * F.second_cell + k] - m.centroid[3 * F.owner + k];
    if (dot3(&m.normal[3 * f], d) < 0.0)
      for (int k = 0; k < 3; ++k) m.normal[3 * f + k] = -m.normal[3 * f + k];
  }
  // Boundary faces in element order, then regrouped by patch.
  std::vector<int> b_owner(nfb), b_patch(nfb);
  std::vector<int64_t> b_rec(nfb, -1);
  std::vector<double> b_centre(3 * nfb), b_normal(3 * nfb), b_area(nfb);
  // The first failing boundary face decides the message, as in a sequential walk.
  int64_t first_bad = nfb;
#pragma omp parallel for schedule(static) reduction(min : first_bad)
  for (int64_t b = 0; b < nfb; ++b) {
    const int* fn = raw.bface_nodes + raw.bface_off[b];
    int nn = (int)(raw.bface_off[b + 1] - raw.bface_off[b]);
    if (nn < 3 || nn > 4) { first_bad = std::min(first_bad, b); continue; }
    FaceKey key = canonical(fn, nn);
    Rec probe{key, -1, -1};
    auto it = std::lower_bound(recs.begin(), recs.end(), probe, [](const Rec& a, const Rec& p) { return a.key < p.key; });
    if (it == recs.end() || !(it->key == key)) { first_bad = std::min(first_bad, b); continue; }
    b_rec[b] = it - recs.begin();
    b_owner[b] = it->cell;
    b_patch[b] = raw.bface_patch[b];
    face_geometry(fn, nn, raw.xyz, &b_centre[3 * b], &b_normal[3 * b], b_area[b]);
    double d[3];
    for (int k = 0; k < 3; ++k) d[k] = b_centre[3 * b + k] - m.centroid[3 * it->cell + k];
    if (dot3(&b_normal[3 * b], d) < 0.0)
      for (int k = 0; k < 3; ++k) b_normal[3 * b + k] = -b_normal[3 * b + k];
  }
  if (first_bad < nfb) {
    int nn = (int)(raw.bface_off[first_bad + 1] - raw.bface_off[first_bad]);
    return fail(-2, (nn < 3 || nn > 4) ? "boundary face with other than 3 or 4 nodes" : "boundary face has no owner cell");
  }
  for (int64_t b = 0; b < nfb; ++b) matched[b_rec[b]] = 1;
  for (size_t i = 0; i < recs.size(); ++i)
    if (!matched[i]) return fail(-3, "unlabelled boundary faces (open cells)");
  m.patch_start.assign(m.n_patches, 0);
  m.patch_nfaces.assign(m.n_patches, 0);
  for (int64_t b = 0; b < nfb; ++b) m.patch_nfaces[b_patch[b]]++;
  for (int p = 1; p < m.n_patches; ++p) m.patch_start[p] = m.patch_start[p - 1] + m.patch_nfaces[p - 1];
  {
    std::vector<int64_t> cursor(m.patch_start);
    for (int64_t b = 0; b < nfb; ++b) {
      int64_t i = cursor[b_patch[b]]++;
      int64_t f = nfi + i;
      m.owner[f] = b_owner[b];
      m.patch[f] = b_patch[b];
      m.area[f] = b_area[b];
      for (int k = 0; k < 3; ++k) {
        m.centre[3 * f + k] = b_centre[3 * b + k];
        m.normal[3 * f + k] = b_normal[3 * b + k];
      }
    }
  }
  m.patch_bc.assign(patch_bc, patch_bc + m.n_patches);
  return finish_mesh(m, err);
}

// Polygon face geometry (src/mesh/mod_mesh.f90:compute_polygon_face_geometry): area vector by a
// fan from the first node, centre weighted by the fan triangles' signed areas.
static void polygon_geometry(const int* fn, int nn, const double* xyz, double centre[3], double normal[3],
                             double& area) {
  centre[0] = centre[1] = centre[2] = 0.0;
  if (nn < 3) {
    area = SMALL;
    normal[0] = normal[1] = normal[2] = 0.0;
    return;
  }
  const double* pref = xyz + 3 * (int64_t)fn[0];
  double nacc[3] = {0.0, 0.0, 0.0};
  for (int i = 1; i < nn - 1; ++i) {
    const double* pi = xyz + 3 * (int64_t)fn[i];
    const double* pj = xyz + 3 * (int64_t)fn[i + 1];
    double a[3], b[3], c[3];
    for (int k = 0; k < 3; ++k) { a[k] = pi[k] - pref[k]; b[k] = pj[k] - pref[k]; }
    cross3(a, b, c);
    for (int k = 0; k < 3; ++k) nacc[k] = nacc[k] + 0.5 * c[k];
  }
  area = std::sqrt(nacc[0] * nacc[0] + nacc[1] * nacc[1] + nacc[2] * nacc[2]) + SMALL;
  for (int k = 0; k < 3; ++k) normal[k] = nacc[k] / area;
  double asum = 0.0;
  for (int i = 1; i < nn - 1; ++i) {
    const double* pi = xyz + 3 * (int64_t)fn[i];
    const double* pj = xyz + 3 * (int64_t)fn[i + 1];
    double a[3], b[3], c[3];
    for (int k = 0; k < 3; ++k) { a[k] = pi[k] - pref[k]; b[k] = pj[k] - pref[k]; }
    cross3(a, b, c);
    double tv[3];
    for (int k = 0; k < 3; ++k) tv[k] = 0.5 * c[k];
    const double ta = dot3(tv, normal);
    for (int k = 0; k < 3; ++k) centre[k] = centre[k] + ta * ((pref[k] + pi[k]) + pj[k]) / 3.0;
    asum = asum + ta;
  }
  if (std::fabs(asum) > SMALL)
    for (int k = 0; k < 3; ++k) centre[k] = centre[k] / asum;
  else
    for (int k = 0; k < 3; ++k) centre[k] = pref[k];
}

int build_mesh_poly(const PolyMesh& pm, const int* patch_bc, Mesh& m, std::string* err) {
  auto fail = [&](int code, const char* msg) {
    if (err) *err = msg;
    return code;
  };
  const int64_t nf = pm.n_faces, nfi = pm.n_int_faces, nfb = nf - nfi, nv = pm.n_points;
  if (nf < 1 || nfi < 0 || nfi > nf) return fail(-5, "face counts out of range");
  // foam_read: cell count from owner and neighbour, upper-triangular internal faces
  int64_t mx = -1;
  for (int64_t f = 0; f < nf; ++f) {
    if (pm.owner[f] < 0) return fail(-5, "negative cell index in owner/neighbour (corrupt polyMesh files)");
    mx = std::max<int64_t>(mx, pm.owner[f]);
  }
  for (int64_t f = 0; f < nfi; ++f) {
    if (pm.neighbour[f] < 0) return fail(-5, "negative cell index in owner/neighbour (corrupt polyMesh files)");
    mx = std::max<int64_t>(mx, pm.neighbour[f]);
  }
  for (int64_t f = 0; f < nfi; ++f)
    if (pm.owner[f] >= pm.neighbour[f]) return fail(-6, "OpenFOAM upper-triangular convention violated");
  for (int64_t k = 0; k < pm.face_off[nf]; ++k)
    if (pm.face_nodes[k] < 0 || pm.face_nodes[k] >= nv) return fail(-5, "face node index out of range");
  const int64_t nc = mx + 1;
  m = Mesh();
  m.n_cells = nc;
  m.n_faces = nf;
  m.n_int_faces = nfi;
  m.n_bnd_faces = nfb;
  m.n_patches = pm.n_patches;
  m.n_vertices = nv;
  m.vertices.assign(pm.xyz, pm.xyz + 3 * nv);
  // patches (foam_read_boundary, validate_foam_boundary_connectivity)
  m.patch.assign(nf, -1);
  m.patch_start.assign(m.n_patches, 0);
  m.patch_nfaces.assign(m.n_patches, 0);
  int n_periodic = 0;
  for (int p = 0; p < m.n_patches; ++p) {
    const int64_t s0 = pm.patch_start[p] - nfi, n = pm.patch_nfaces[p];
    if (s0 < 0 || n < 0) return fail(-7, "boundary connectivity invalid (patch has invalid start_face/n_faces)");
    if (s0 + n > nfb) return fail(-7, "patch face range exceeds boundary faces");
    m.patch_start[p] = s0;
    m.patch_nfaces[p] = n;
    for (int64_t f = nfi + s0; f < nfi + s0 + n; ++f) m.patch[f] = p;
    if (patch_bc[p] == BC_PERIODIC) n_periodic++;
  }
  for (int64_t f = nfi; f < nf; ++f)
    if (m.patch[f] < 0) return fail(-7, "boundary faces not mapped to a patch");
  if (n_periodic % 2) return fail(-8, "odd number of periodic patches");
  m.patch_bc.assign(patch_bc, patch_bc + m.n_patches);
  // faces
  m.owner.assign(pm.owner, pm.owner + nf);
  m.neighbour.assign(nf, -1);
  for (int64_t f = 0; f < nfi; ++f) m.neighbour[f] = pm.neighbour[f];
  m.area.assign(nf, 0.0);
  m.centre.assign(3 * nf, 0.0);
  m.normal.assign(3 * nf, 0.0);
#pragma omp parallel for schedule(static)
  for (int64_t f = 0; f < nf; ++f)
    polygon_geometry(pm.face_nodes + pm.face_off[f], (int)(pm.face_off[f + 1] - pm.face_off[f]), pm.xyz,
                     &m.centre[3 * f], &m.normal[3 * f], m.area[f]);
  // cell moments (mod_mesh.f90:compute_polyhedron_cell_moments), about the first vertex of the
  // first face (in face order) that touches the cell
  std::vector<double> ref(3 * nc, 0.0), mom(3 * nc, 0.0);
  std::vector<uint8_t> ref_set(nc, 0);
  m.volume.assign(nc, 0.0);
  m.centroid.assign(3 * nc, 0.0);
  for (int64_t f = 0; f < nf; ++f) {
    if (pm.face_off[f + 1] - pm.face_off[f] < 3) continue;
    for (int side = 0; side < 2; ++side) {
      const int64_t c = side == 0 ? m.owner[f] : m.neighbour[f];
      if (c < 0 || ref_set[c]) continue;
      for (int k = 0; k < 3; ++k) ref[3 * c + k] = pm.xyz[3 * (int64_t)pm.face_nodes[pm.face_off[f]] + k];
      ref_set[c] = 1;
    }
  }
  for (int64_t f = 0; f < nf; ++f) {
    const int64_t s0 = pm.face_off[f], s1 = pm.face_off[f + 1];
    if (s1 - s0 < 3) continue;
    for (int side = 0; side < 2; ++side) {
      const int64_t c = side == 0 ? m.owner[f] : m.neighbour[f];
      if (c < 0) break;
      const double* r = &ref[3 * c];
      double v0[3];
      for (int k = 0; k < 3; ++k) v0[k] = pm.xyz[3 * (int64_t)pm.face_nodes[s0] + k] - r[k];
      for (int64_t i = s0 + 1; i < s1 - 1; ++i) {
        double v1[3], v2[3], cr[3];
        for (int k = 0; k < 3; ++k) {
          v1[k] = pm.xyz[3 * (int64_t)pm.face_nodes[i] + k] - r[k];
          v2[k] = pm.xyz[3 * (int64_t)pm.face_nodes[i + 1] + k] - r[k];
        }
        cross3(v1, v2, cr);
        const double sv = dot3(v0, cr) / 6.0;
        double sm[3];
        for (int k = 0; k < 3; ++k) sm[k] = sv * ((v0[k] + v1[k]) + v2[k]) / 4.0;
        if (side == 0) {
          m.volume[c] = m.volume[c] + sv;
          for (int k = 0; k < 3; ++k) mom[3 * c + k] = mom[3 * c + k] + sm[k];
        } else {
          m.volume[c] = m.volume[c] - sv;
          for (int k = 0; k < 3; ++k) mom[3 * c + k] = mom[3 * c + k] - sm[k];
        }
      }
    }
  }
  for (int64_t c = 0; c < nc; ++c) {
    if (std::fabs(m.volume[c]) > SMALL)
      for (int k = 0; k < 3; ++k) m.centroid[3 * c + k] = ref[3 * c + k] + mom[3 * c + k] / m.volume[c];
    m.volume[c] = std::fabs(m.volume[c]);
  }
  // cell vertex lists (mod_foam_reader.f90:build_cell_topology_metadata): the cell's owner faces
  // in face order, then its neighbour faces, each vertex at its first appearance
  {
    std::vector<int64_t> cnt(nc + 1, 0);
    for (int64_t f = 0; f < nf; ++f) cnt[m.owner[f] + 1]++;
    for (int64_t f = 0; f < nfi; ++f) cnt[m.neighbour[f] + 1]++;
    for (int64_t c = 0; c < nc; ++c) cnt[c + 1] += cnt[c];
    std::vector<int> cfaces(cnt[nc]);
    std::vector<int64_t> pos(cnt.begin(), cnt.end() - 1);
    for (int64_t f = 0; f < nf; ++f) cfaces[pos[m.owner[f]]++] = (int)f;
    for (int64_t f = 0; f < nfi; ++f) cfaces[pos[m.neighbour[f]]++] = (int)f;
    std::vector<int64_t> mark(nv, -1);
    m.cell_vert_off.assign(nc + 1, 0);
    m.cell_vertices.clear();
    for (int64_t c = 0; c < nc; ++c) {
      for (int64_t q = cnt[c]; q < cnt[c + 1]; ++q) {
        const int f = cfaces[q];
        for (int64_t k = pm.face_off[f]; k < pm.face_off[f + 1]; ++k) {
          const int v = pm.face_nodes[k];
          if (mark[v] == c) continue;
          mark[v] = c;
          m.cell_vertices.push_back(v);
        }
      }
      m.cell_vert_off[c + 1] = (int64_t)m.cell_vertices.size();
    }
  }
  return finish_mesh(m, err);
}

}  // namespace dpm
