// Static operators; see ops.hpp.
#include "ops.hpp"

#include <algorithm>
#include <cmath>

namespace dpm {
namespace {

constexpr double NONORTHO_SIN2_TOL = 1.0e-10;  // src/numerics/mod_nonortho.f90:7

inline double dot(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// Over-relaxed Jasak k-vector, k = S - |S|^2/(S.d) d (src/numerics/mod_nonortho.f90:65-99).
void jasak_k(const double* sf, const double* d, double min_cos, double* k) {
  double len = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  if (len < 1.0e-30) { k[0] = k[1] = k[2] = 0.0; return; }
  double inv = 1.0 / len, sdd = dot(sf, d) * inv, dl = sdd * len, s2 = dot(sf, sf);
  if (min_cos > 0.0) dl = std::max(dl, min_cos * std::sqrt(s2) * len);
  if (dl > 1.0e-30)
    for (int i = 0; i < 3; ++i) k[i] = sf[i] - (s2 / dl) * d[i];
  else
    for (int i = 0; i < 3; ++i) k[i] = sf[i] - (sdd * inv) * d[i];
}

double det3(const double* A) {
  return A[0] * (A[4] * A[8] - A[7] * A[5]) - A[3] * (A[1] * A[8] - A[7] * A[2]) + A[6] * (A[1] * A[5] - A[4] * A[2]);
}

template <class T>
void ell_from_lists(const std::vector<std::vector<T>>& lists, int64_t nc, int& width, std::vector<T>& out, T pad) {
  width = 0;
  for (auto& l : lists) width = std::max<int>(width, (int)l.size());
  out.assign((size_t)std::max(width, 1) * nc, pad);
  for (int64_t c = 0; c < nc; ++c)
    for (size_t s = 0; s < lists[c].size(); ++s) out[s * nc + c] = lists[c][s];
}

}  // namespace

int build_static_ops(const Mesh& m, const dpm_patch_cfg_t* pc, const dpm_params_t& P, StaticOps& S) {
  // Every per-cell sum is a gather over the cell's sorted lists, in the order the reference's
  // global face loops add the terms, so the cells can be built in parallel.
  const int64_t nc = m.n_cells, nf = m.n_faces, nfi = m.n_int_faces, nb = m.n_bnd_faces;
  S = StaticOps();
  S.nc = nc; S.nf = nf; S.nfi = nfi; S.nb = nb;
  S.bnd_bc.assign(nb, BC_ZEROGRADIENT);
  S.bnd_pnb.assign(nb, -1);
  for (int64_t b = 0; b < nb; ++b) {
    int p = m.patch[nfi + b];
    if (p >= 0) S.bnd_bc[b] = pc[p].bc_id;
    if (S.bnd_bc[b] == BC_PERIODIC) {
      int n = m.periodic_partner_cell(b);
      S.bnd_pnb[b] = (n == m.owner[nfi + b]) ? -1 : n;
    }
  }
  // Pressure-solver face list and coefficients (mod_pressure_solver.f90:pressure_solver_init):
  // periodic pairs contribute to the diagonal first, interior faces next, outlet rows last.
  std::vector<int64_t> per_canon;  // boundary index of the canonical face of each periodic pair
  for (int q = 0; q < m.n_patches; ++q) {
    if (pc[q].bc_id != BC_PERIODIC) continue;
    for (int64_t k = 0; k < m.patch_nfaces[q]; ++k) {
      int64_t b = m.patch_start[q] + k;
      int o = m.owner[nfi + b], n = m.periodic_partner_cell(b);
      if (n < 0 || n <= o) continue;  // canonical side: owner has the smaller cell id
      per_canon.push_back(b);
    }
  }
  S.nfp = nfi + (int64_t)per_canon.size();
  const int64_t nfp = S.nfp;
  S.ps_o.resize(nfp); S.ps_n.resize(nfp); S.ps_f.resize(nfp);
  S.ps_coeff.assign(nfp, 0.0); S.ps_gcf.assign(nfp, 0.0); S.ps_gcw.assign(nfp, 0.0);
  S.ps_k.assign(3 * nfp, 0.0); S.ps_krc.assign(3 * nfp, 0.0);
  S.diag.assign(nc, 0.0);
  std::vector<int> bps(nb, -1);            // pressure-solver index of a periodic boundary face
  std::vector<uint8_t> bcanon(nb, 0);      // its canonical side
  for (size_t k = 0; k < per_canon.size(); ++k) {
    int64_t b = per_canon[k], f = nfi + b, i = nfi + (int64_t)k;
    int o = m.owner[f], n = m.periodic_partner_cell(b);
    int pb = m.periodic_pair[b];
    int64_t pf = pb >= 0 ? nfi + pb : -1;
    double pdcf = m.periodic_pair_dcf[b];
    if (pdcf <= SMALL && pf >= 0) pdcf = m.d_cf[pf];
    if (pdcf <= SMALL) pdcf = m.d_cf[f];
    double area = m.area[f];
    if (pf >= 0) area = 0.5 * (area + m.area[pf]);
    double coeff = area / (m.d_cf[f] + pdcf + SMALL);
    S.ps_o[i] = o; S.ps_n[i] = n; S.ps_f[i] = (int)f;
    S.ps_coeff[i] = coeff;
    // face-velocity weight from the two owner-to-face distances (mod_fv_solver.f90:2541-2560)
    double d_o = m.d_cf[f], d_n = d_o;
    if (m.periodic_pair_dcf[b] > SMALL) d_n = m.periodic_pair_dcf[b];
    if (d_n <= SMALL && pf >= 0) d_n = m.d_cf[pf];
    double dt_ = d_o + d_n;
    S.ps_gcf[i] = dt_ > SMALL ? d_n / dt_ : 0.5;
    S.ps_gcw[i] = m.periodic_gc[b];
    bps[b] = (int)i;
    bcanon[b] = 1;
    if (pb >= 0) bps[pb] = (int)i;
  }
  const double cfl = P.pressure_min_cos_theta;
  int bad_coeff = 0;
#pragma omp parallel for schedule(static) reduction(| : bad_coeff)
  for (int64_t f = 0; f < nfi; ++f) {
    int o = m.owner[f], n = m.neighbour[f];
    S.ps_o[f] = o; S.ps_n[f] = n; S.ps_f[f] = (int)f;
    S.ps_gcf[f] = m.gc[f]; S.ps_gcw[f] = m.gc[f];
    double d[3];
    for (int k = 0; k < 3; ++k) d[k] = m.centroid[3 * n + k] - m.centroid[3 * o + k];
    double dor = dot(d, &m.normal[3 * f]);
    if (cfl > 0.0 && dor < cfl * m.d_cf[f]) dor = cfl * m.d_cf[f];
    double coeff = dor > SMALL ? m.area[f] / dor : m.area[f] / (m.d_cf[f] + SMALL);
    if (!(std::fabs(coeff) <= 1.7976931348623157e308) || coeff <= SMALL) bad_coeff = 1;
    S.ps_coeff[f] = coeff;
  }
  if (bad_coeff) return DPM_ERR_MESH;
  S.bnd_cb.assign(nb, 0.0);
  S.bnd_kout.assign(3 * nb, 0.0);
  S.n_outlet = 0;
  std::vector<double> bdiag(nb, 0.0);      // outlet row's diagonal term of a boundary face
  std::vector<uint8_t> bdiag_on(nb, 0);
  for (int q = 0; q < m.n_patches; ++q) {
    if (pc[q].bc_id != BC_OUTLET) continue;
    for (int64_t k = 0; k < m.patch_nfaces[q]; ++k) {
      int64_t b = m.patch_start[q] + k, f = nfi + b;
      int o = m.owner[f];
      double d[3];
      for (int j = 0; j < 3; ++j) d[j] = m.centre[3 * f + j] - m.centroid[3 * o + j];
      double dpb = std::fabs(dot(d, &m.normal[3 * f]));
      S.n_outlet++;
      // coefficient of the flux/velocity corrections (mod_fv_solver.f90:2860-2866)
      S.bnd_cb[b] = m.area[f] / std::max(dpb, SMALL);
      if (dpb <= SMALL) dpb = m.d_cf[f];
      if (cfl > 0.0) dpb = std::max(dpb, cfl * m.d_cf[f]);
      if (dpb <= SMALL) continue;
      double cb = m.area[f] / dpb;
      bdiag[b] = cb;
      bdiag_on[b] = 1;
      S.dir_rows.push_back(o);
      S.dir_vals.push_back(cb * pc[q].p_val);
    }
  }
  // Per-cell lists (ELL [slot][nc], PAD): faces ascending, boundary faces ascending, and the
  // pressure-solver entries idx (owner side) / ~idx (neighbour side) ascending in idx.
  {
    int w_f = 0, w_b = 0, w_p = 0;
#pragma omp parallel for schedule(static) reduction(max : w_f, w_b, w_p)
    for (int64_t c = 0; c < nc; ++c) {
      int nbd = 0, np = 0;
      for (int64_t k = m.cell_face_off[c]; k < m.cell_face_off[c + 1]; ++k) {
        const int f = m.cell_faces[k];
        if (f >= nfi) {
          ++nbd;
          if (bps[f - nfi] >= 0) ++np;
        } else {
          ++np;
        }
      }
      w_f = std::max(w_f, (int)(m.cell_face_off[c + 1] - m.cell_face_off[c]));
      w_b = std::max(w_b, nbd);
      w_p = std::max(w_p, np);
    }
    S.S = w_f; S.SB = w_b; S.SP = w_p;
    S.cell_face.assign((size_t)std::max(w_f, 1) * nc, PAD);
    S.cell_bnd.assign((size_t)std::max(w_b, 1) * nc, PAD);
    S.cell_ps.assign((size_t)std::max(w_p, 1) * nc, PAD);
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nc; ++c) {
      int s = 0, nbd = 0, np = 0;
      std::vector<int> e;
      e.reserve(8);
      for (int64_t k = m.cell_face_off[c]; k < m.cell_face_off[c + 1]; ++k, ++s) {
        const int f = m.cell_faces[k];
        S.cell_face[(size_t)s * nc + c] = f;
        if (f < nfi) {
          e.push_back(m.owner[f] == c ? f : ~f);
        } else {
          const int64_t b = f - nfi;
          S.cell_bnd[(size_t)nbd++ * nc + c] = (int)b;
          if (bps[b] >= 0) e.push_back(bcanon[b] ? bps[b] : ~bps[b]);
        }
      }
      std::sort(e.begin(), e.end(), [](int a, int b) { return (a >= 0 ? a : ~a) < (b >= 0 ? b : ~b); });
      for (int v : e) S.cell_ps[(size_t)np++ * nc + c] = v;
    }
  }
  // Diagonal: periodic pairs, then interior faces, then outlet rows, each in list order.
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < nc; ++c) {
    double dg = 0.0;
    for (int pass = 0; pass < 2; ++pass)
      for (int q = 0; q < S.SP; ++q) {
        const int e = S.cell_ps[(size_t)q * nc + c];
        if (e == PAD) break;
        const int i = e >= 0 ? e : ~e;
        if ((pass == 0) == (i >= nfi)) dg += S.ps_coeff[i];
      }
    for (int q = 0; q < S.SB; ++q) {
      const int b = S.cell_bnd[(size_t)q * nc + c];
      if (b == PAD) break;
      if (bdiag_on[b]) dg += bdiag[b];
    }
    if (!(dg > SMALL) || !(dg <= 1.7976931348623157e308)) dg = 1.0;
    S.diag[c] = dg;
  }

  // Non-orthogonal correction (mod_fv_solver.f90:detect_nonortho_skip, build_nonortho_cache).
  int64_t n_active = 0;
  std::vector<double> kk(3 * nfp, 0.0), kb(3 * nb, 0.0);
#pragma omp parallel for schedule(static) reduction(+ : n_active)
  for (int64_t i = 0; i < nfp; ++i) {
    int o = S.ps_o[i], n = S.ps_n[i];
    const double* sf = &m.sf[3 * (int64_t)S.ps_f[i]];
    double d[3], k[3];
    for (int j = 0; j < 3; ++j) d[j] = m.centroid[3 * n + j] - m.centroid[3 * o + j];
    jasak_k(sf, d, cfl, k);
    if (dot(k, k) >= NONORTHO_SIN2_TOL * dot(sf, sf)) {
      n_active++;
      for (int j = 0; j < 3; ++j) kk[3 * i + j] = k[j];
    }
  }
  for (int64_t b = 0; b < nb; ++b) {
    if (S.bnd_bc[b] != BC_OUTLET) continue;
    int64_t f = nfi + b;
    int o = m.owner[f];
    double d[3], k[3];
    for (int j = 0; j < 3; ++j) d[j] = m.centre[3 * f + j] - m.centroid[3 * o + j];
    jasak_k(&m.sf[3 * f], d, cfl, k);
    if (dot(k, k) >= NONORTHO_SIN2_TOL * dot(&m.sf[3 * f], &m.sf[3 * f])) {
      n_active++;
      for (int j = 0; j < 3; ++j) kb[3 * b + j] = k[j];
    }
  }
  int n_gradbc = 0;
  for (int q = 0; q < m.n_patches; ++q) {
    int b = pc[q].bc_id;
    if (!(b == BC_OUTLET || b == BC_PERIODIC || b == BC_WALL_NOSLIP || b == BC_WALL_VELOCITY ||
          b == BC_WALL_MODEL || b == BC_SLIP || b == BC_SYMMETRY))
      n_gradbc++;
  }
  S.skip_nonortho = (n_active == 0);
  S.skip_grad_p = S.skip_nonortho && n_gradbc == 0;
  S.n_nonortho_corr = P.n_nonortho_corr > 0 ? P.n_nonortho_corr : (S.skip_nonortho ? 1 : 2);
  if (!S.skip_nonortho) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nfp; ++i)
      for (int j = 0; j < 3; ++j) S.ps_k[j * nfp + i] = kk[3 * i + j];
    for (int64_t b = 0; b < nb; ++b)
      for (int j = 0; j < 3; ++j) S.bnd_kout[j * nb + b] = kb[3 * b + j];
    if (!P.rhie_chow_dual) S.ps_krc = S.ps_k;  // Rhie-Chow k: same vector, same activity test
  }
  S.diag_interface = false;
  for (int64_t f = 0; f < nfi; ++f)
    if (m.is_refine[f]) { S.diag_interface = true; break; }
  S.V_min = 1e300; S.V_total = 0.0;
  for (int64_t c = 0; c < nc; ++c) { S.V_min = std::min(S.V_min, m.volume[c]); S.V_total += m.volume[c]; }

  // Assembled matrix, row-sorted (pressure_backend_petsc.c:330-360 stores AIJ rows sorted): the
  // row's (self, diag) then one entry per pressure-solver face in idx order, stable-sorted by
  // column, equal columns summed in that order; ELL [WA][nc], padded with (self, 0).
  {
    auto row = [&](int64_t c, std::vector<std::pair<int, double>>& r) {
      r.clear();
      r.push_back({(int)c, S.diag[c]});
      for (int q = 0; q < S.SP; ++q) {
        const int e = S.cell_ps[(size_t)q * nc + c];
        if (e == PAD) break;
        const int i = e >= 0 ? e : ~e;
        if (S.ps_coeff[i] == 0.0) continue;
        r.push_back({e >= 0 ? S.ps_n[i] : S.ps_o[i], -S.ps_coeff[i]});
      }
      std::stable_sort(r.begin(), r.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
      size_t u = 0;
      for (size_t k = 0; k < r.size(); ++k) {
        if (u > 0 && r[u - 1].first == r[k].first) r[u - 1].second += r[k].second;
        else r[u++] = r[k];
      }
      r.resize(u);
    };
    int wa = 0;
#pragma omp parallel reduction(max : wa)
    {
      std::vector<std::pair<int, double>> r;
#pragma omp for schedule(static)
      for (int64_t c = 0; c < nc; ++c) {
        row(c, r);
        wa = std::max(wa, (int)r.size());
      }
    }
    S.WA = wa;
    if (S.WA > 16) return DPM_ERR_UNSUPPORTED;
    S.A_col.assign((size_t)std::max(wa, 1) * nc, 0);
    S.A_val.assign((size_t)std::max(wa, 1) * nc, 0.0);
#pragma omp parallel
    {
      std::vector<std::pair<int, double>> r;
#pragma omp for schedule(static)
      for (int64_t c = 0; c < nc; ++c) {
        row(c, r);
        // pad every row to the full width with (self, 0): fixed-length rows, no early exit on the GPU
        for (int w = 0; w < wa; ++w) {
          S.A_col[(size_t)w * nc + c] = w < (int)r.size() ? r[w].first : (int)c;
          S.A_val[(size_t)w * nc + c] = w < (int)r.size() ? r[w].second : 0.0;
        }
      }
    }
  }
  // LS stencil as ELL.
  {
    int W = 0;
    for (int64_t c = 0; c < nc; ++c) W = std::max<int>(W, (int)(m.ls_off[c + 1] - m.ls_off[c]));
    S.W = W;
    S.ls_idx.assign((size_t)std::max(W, 1) * nc, PAD);
    S.ls_w.assign((size_t)3 * std::max(W, 1) * nc, 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nc; ++c)
      for (int64_t k = m.ls_off[c]; k < m.ls_off[c + 1]; ++k) {
        int s = (int)(k - m.ls_off[c]);
        int n = m.ls_cell[k];
        int v;
        if (n >= 0) v = n;
        else {
          int f = m.ls_face[k];
          int64_t b = f >= 0 ? f - nfi : -1;
          v = (b >= 0 && b < nb) ? -(int)(b + 1) : -(int)(nb + 1);  // -(nb+1): use the cell value
        }
        S.ls_idx[(size_t)s * nc + c] = v;
        for (int j = 0; j < 3; ++j) S.ls_w[((size_t)j * W + s) * nc + c] = m.ls_w[3 * k + j];
      }
  }
  // Reconstruction operator T^-1 (mod_fv_solver.f90:build_reconstruct_operator, invert_sym3):
  // the cell's pressure-solver faces in idx order, then its non-periodic boundary faces.
  S.Tinv.assign(9 * nc, 0.0);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < nc; ++c) {
    double A[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    auto add = [&](int64_t f) {
      const double* n = &m.normal[3 * f];
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) A[i + 3 * j] += m.area[f] * n[i] * n[j];
    };
    for (int q = 0; q < S.SP; ++q) {
      const int e = S.cell_ps[(size_t)q * nc + c];
      if (e == PAD) break;
      add(S.ps_f[e >= 0 ? e : ~e]);
    }
    for (int q = 0; q < S.SB; ++q) {
      const int b = S.cell_bnd[(size_t)q * nc + c];
      if (b == PAD) break;
      if (S.bnd_bc[b] != BC_PERIODIC) add(nfi + b);
    }
    // A(i,j) = A[(i-1) + 3(j-1)]
    double a11 = A[0], a21 = A[1], a31 = A[2], a12 = A[3], a22 = A[4], a32 = A[5], a13 = A[6], a23 = A[7], a33 = A[8];
    double c11 = a22 * a33 - a23 * a32, c12 = a13 * a32 - a12 * a33, c13 = a12 * a23 - a13 * a22;
    double c22 = a11 * a33 - a13 * a31, c23 = a13 * a21 - a11 * a23, c33 = a11 * a22 - a12 * a21;
    double det = a11 * c11 + a12 * (a23 * a31 - a21 * a33) + a13 * (a21 * a32 - a22 * a31);
    double tr = a11 + a22 + a33, mt = std::max(tr, SMALL);
    double* Ti = &S.Tinv[9 * c];
    if (std::fabs(det) <= 1.0e-12 * mt * mt * mt) {
      Ti[0] = Ti[4] = Ti[8] = 3.0 / mt;
      continue;
    }
    Ti[0] = c11 / det; Ti[3] = c12 / det; Ti[6] = c13 / det;
    Ti[1] = c12 / det; Ti[4] = c22 / det; Ti[7] = c23 / det;
    Ti[2] = c13 / det; Ti[5] = c23 / det; Ti[8] = c33 / det;
  }
  // SGS filter tensor with det G = V^2 and two face-area smoothing passes
  // (src/sgs/mod_vreman.f90:build_filter_tensor, smooth_filter_tensor): a cell's interior faces
  // in face order.
  {
    S.G.assign(9 * nc, 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nc; ++c) {
      double g[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int64_t k = m.cell_face_off[c]; k < m.cell_face_off[c + 1]; ++k) {
        int64_t f = m.cell_faces[k];
        double dx[3];
        for (int j = 0; j < 3; ++j) dx[j] = m.centre[3 * f + j] - m.centroid[3 * c + j];
        for (int n = 0; n < 3; ++n)
          for (int i = 0; i < 3; ++i) g[i + 3 * n] += m.area[f] * dx[i] * dx[n];
      }
      double dt = det3(g), t = (g[0] + g[4] + g[8]) / 3.0, t3 = t * t * t;
      if (t3 > 0.0 && dt > 1.0e-12 * t3) {
        double s = std::pow(m.volume[c] * m.volume[c] / dt, 1.0 / 3.0);
        for (int j = 0; j < 9; ++j) S.G[9 * c + j] = s * g[j];
      } else {
        double d2 = std::pow(m.volume[c], 2.0 / 3.0);
        S.G[9 * c] = S.G[9 * c + 4] = S.G[9 * c + 8] = d2;
      }
    }
    std::vector<double> Gn(9 * nc);
    for (int pass = 0; pass < 2; ++pass) {
#pragma omp parallel for schedule(static)
      for (int64_t c = 0; c < nc; ++c) {
        double gn[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, ws = 0.0;
        for (int64_t k = m.cell_face_off[c]; k < m.cell_face_off[c + 1]; ++k) {
          const int f = m.cell_faces[k];
          if (f >= nfi) continue;
          const int other = m.owner[f] == c ? m.neighbour[f] : m.owner[f];
          const double a = m.area[f];
          for (int j = 0; j < 9; ++j) gn[j] += a * S.G[9 * (int64_t)other + j];
          ws += a;
        }
        for (int j = 0; j < 9; ++j)
          Gn[9 * c + j] = ws > SMALL ? 0.5 * S.G[9 * c + j] + 0.5 * gn[j] / ws : S.G[9 * c + j];
      }
      S.G.swap(Gn);
    }
  }
  // Wall-model sampling distance (src/sgs/mod_wall_model.f90:find_sample_cell, h_wm <= 0).
  S.y_w.assign(nb, 0.0);
  for (int64_t b = 0; b < nb; ++b) {
    if (S.bnd_bc[b] != BC_WALL_MODEL) continue;
    int64_t f = nfi + b;
    int o = m.owner[f];
    double d[3], nin[3];
    for (int j = 0; j < 3; ++j) { d[j] = m.centroid[3 * o + j] - m.centre[3 * f + j]; nin[j] = -m.normal[3 * f + j]; }
    S.y_w[b] = std::fabs(dot(d, nin)) + SMALL;
  }
  S.wblend.assign(nf, 1.0);
#pragma omp parallel for schedule(static)
  for (int64_t f = 0; f < nfi; ++f) S.wblend[f] = refine_blend_weight(m.skew[f]);
  return 0;
}

}  // namespace dpm
