// ORACLE — test infrastructure only.  A CPU restatement of the reference's RK3W fractional-step
// time step (AkshayPatil1994/dopamine, Fortran) used as the parity checker for the sm_100a
// product path and as the timed CPU baseline.  Nothing in the product links, imports or
// executes this file.  Every routine cites the reference routine it follows; face loops run in
// the reference's face order and accumulate in the same sequence, and the Poisson solve follows
// PETSc's KSPCG (unpreconditioned residual norm, nonzero initial guess, constant null space,
// Jacobi preconditioner) as configured in src/solver/pressure_backend_petsc.c:381-463.
//
// Pinning: checked against the reference's regression CSVs (tests/regression/reference/*.csv)
// for the cases whose meshes can be regenerated without gmsh; see tests/test_oracle_golden.py.
//
// Mesh geometry, periodic pairing and LS stencils come from the shared host set-up
// (dopamine_b200/csrc/host/mesh.cpp), the restatement of src/mesh/mod_mesh.f90 set-up.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#include "../dopamine_b200/csrc/host/mesh.hpp"
#include "../include/dopamine_b200.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {
using namespace dpm;

constexpr double KAPPA = 0.41;                  // src/mod_parameters.f90:14
constexpr double BLOG = 5.2;                    // src/mod_parameters.f90:17
constexpr double C_VREMAN = 0.025;              // src/mod_parameters.f90:20
constexpr double NU_SGS_STAB_FRAC = 0.4;        // src/sgs/mod_vreman.f90:34
constexpr double NONORTHO_SIN2_TOL = 1.0e-10;   // src/numerics/mod_nonortho.f90:7
constexpr double NONORTHO_PHI_TOL = 1.0e-3;     // src/solver/mod_fv_solver.f90:116
constexpr double AMD_ALPHA_SQ_MIN = 1.0e-20;    // src/sgs/mod_amd.f90:18
constexpr double AMD_ROUNDOFF_FRAC = 1.0e-12;   // src/sgs/mod_amd.f90:22
const double RK3W_ALPHA[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};   // src/mod_parameters.f90:64
const double RK3W_BETA[3] = {0.0, -17.0 / 60.0, -5.0 / 12.0};
const double RK3W_GAMMA[3] = {8.0 / 15.0, 2.0 / 15.0, 1.0 / 3.0};
const double RK3W_C[3] = {0.0, 8.0 / 15.0, 2.0 / 3.0};

inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline bool finite(double x) { return std::fabs(x) <= 1.79769313486231570e308; }
inline bool is_wall(int bc) {
  return bc == BC_WALL_NOSLIP || bc == BC_WALL_MODEL || bc == BC_WALL_VELOCITY || bc == BC_SLIP || bc == BC_SYMMETRY;
}

// src/numerics/mod_nonortho.f90:65-99
void kfactor_limited(const double* sf, const double* d_on, double min_cos, double* k) {
  double len = std::sqrt(d_on[0] * d_on[0] + d_on[1] * d_on[1] + d_on[2] * d_on[2]);
  if (len < 1.0e-30) { k[0] = k[1] = k[2] = 0.0; return; }
  double inv = 1.0 / len;
  double sdd = dot3(sf, d_on) * inv;
  double d_len = sdd * len;
  double sf_sq = sf[0] * sf[0] + sf[1] * sf[1] + sf[2] * sf[2];
  if (min_cos > 0.0) d_len = std::max(d_len, min_cos * std::sqrt(sf_sq) * len);
  if (d_len > 1.0e-30) {
    for (int i = 0; i < 3; ++i) k[i] = sf[i] - (sf_sq / d_len) * d_on[i];
  } else {
    for (int i = 0; i < 3; ++i) k[i] = sf[i] - (sdd * inv) * d_on[i];
  }
}

// src/sgs/mod_wall_model.f90:50-64
void reichardt_uplus(double yp, double c_buf, double& up, double& dup) {
  const double A1 = 11.0, A2 = 0.33, A1I = 1.0 / A1;
  double e1 = std::exp(-yp * A1I), e2 = std::exp(-A2 * yp);
  up = std::log(1.0 + KAPPA * yp) / KAPPA + c_buf * (1.0 - e1 - yp * A1I * e2);
  dup = 1.0 / (1.0 + KAPPA * yp) + c_buf * (A1I * e1 - A1I * e2 + yp * A1I * A2 * e2);
}

// src/sgs/mod_wall_model.f90:67-114
void wall_stress_newton(double u_par, double y_w, double nu, double& u_tau, double& tau_mag, bool& capped) {
  const double C_BUF = BLOG - std::log(KAPPA) / KAPPA;
  capped = false;
  if (u_par <= SMALL || y_w <= SMALL) { u_tau = 0.0; tau_mag = 0.0; return; }
  u_tau = std::max(0.01 * u_par, std::sqrt(nu * u_par / (y_w + SMALL)));
  double inv_nu = 1.0 / (nu + SMALL), ywn = y_w * inv_nu;
  for (int it = 0; it < 50; ++it) {
    double yp = u_tau * ywn, up, dup;
    reichardt_uplus(yp, C_BUF, up, dup);
    double f = u_par / (u_tau + SMALL) - up;
    double df = -u_par / (u_tau * u_tau + SMALL) - dup * ywn;
    double s = df >= 0.0 ? SMALL : -SMALL;
    double un = u_tau - f / (df + s);
    un = std::min(std::max(un, 0.1 * u_tau), 10.0 * u_tau);
    if (std::fabs(un - u_tau) < 1.0e-8 * un) { u_tau = un; break; }
    u_tau = un;
  }
  capped = (u_tau * ywn < 1.0);
  tau_mag = u_tau * u_tau;
}

// src/sgs/mod_amd.f90:31-66
double amd_point(const double* a, const double* G, double c_amd) {
  // a, G column-major 3x3: a[i + 3j] = alpha(i+1, j+1)
  double asq = 0.0;
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) asq += a[i + 3 * j] * a[i + 3 * j];
  double num = 0.0;
  for (int n = 0; n < 3; ++n)
    for (int mm = 0; mm < 3; ++mm) {
      double beta = 0.0;
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) beta += G[i + 3 * j] * a[i + 3 * mm] * a[j + 3 * n];
      num -= beta * a[mm + 3 * n];
    }
  double trg = G[0] + G[4] + G[8];
  if (asq > AMD_ALPHA_SQ_MIN && num > AMD_ROUNDOFF_FRAC * trg * asq * std::sqrt(asq)) return c_amd * num / asq;
  return 0.0;
}

double det3(const double* A) {  // column-major
  auto a = [&](int i, int j) { return A[(i - 1) + 3 * (j - 1)]; };
  return a(1, 1) * (a(2, 2) * a(3, 3) - a(2, 3) * a(3, 2)) - a(1, 2) * (a(2, 1) * a(3, 3) - a(2, 3) * a(3, 1)) +
         a(1, 3) * (a(2, 1) * a(3, 2) - a(2, 2) * a(3, 1));
}

struct Solver {
  Mesh m;
  dpm_params_t P{};
  std::vector<dpm_patch_cfg_t> pc;
  int64_t nc = 0, nf = 0, nfi = 0, nb = 0;
  int nthreads = 1;

  // primary fields (AoS, Fortran layout)
  std::vector<double> U, p, p_old, T, nu_sgs, U_bnd, p_bnd, phi_prev, phi_prev_bnd, tau_w;
  // temperature and passive scalars (scalar-major [s][nc] / [s][nb] / [s][nc][3])
  std::vector<double> T_bnd, grad_T, H_T, H_T0, conv_T, visc_T;
  int ns = 0;
  std::vector<double> Cs, C_bnd, grad_C, H_C, H_C0, conv_C, visc_C;
  // MOST surface layer: per-face Obukhov length and kinematic heat flux, domain-mean L
  std::vector<double> L_bnd, q_w;
  double L_obukhov = 0.0;
  std::vector<double> grad_U, face_flux, U_face, inv_vol;
  std::vector<double> H_U, H_U0, rhs_p, conv_U, visc_U, gp, gp_rc, gp_cell, p_tot, p_tot_bnd, phi_it, Tinv;
  std::vector<uint8_t> built;
  bool u_face_ready = false;
  double time = 0.0;
  int64_t step = 0;

  // patch classification (mod_fv_solver.f90:build_patch_classification)
  std::vector<int64_t> per_bf, nper_bf;
  int64_t n_outlet = 0;
  double V_min = 0, V_total = 0, p_atol_factor = 1.0e-15;
  bool diag_interface = false;

  // pressure-solver face list (mod_pressure_solver.f90:pressure_solver_init)
  int64_t nfp = 0;
  std::vector<int> ps_owner, ps_nb, ps_mesh;
  std::vector<uint8_t> ps_skip;
  std::vector<double> ps_coeff, ps_diag;
  std::vector<int> dir_rows;
  std::vector<double> dir_vals;
  // CSR of the assembled matrix, columns sorted (as PETSc AIJ stores them)
  std::vector<int64_t> A_off;
  std::vector<int> A_col;
  std::vector<double> A_val;
  // optional record of the pressure systems solved (right-hand side, initial guess, atol), for
  // tests that study the solver on the systems the time step produces
  bool record = false;
  std::vector<std::vector<double>> rec_rhs, rec_x0;
  std::vector<double> rec_atol;

  // non-orthogonal caches (mod_fv_solver.f90:detect_nonortho_skip, build_nonortho_cache)
  bool skip_nonortho = false, skip_grad_p = false;
  std::vector<double> k_int, k_bnd;
  std::vector<uint8_t> act_int, act_bnd;

  // SGS filter tensor and wall-model sampling
  std::vector<double> Gf;
  std::vector<double> y_w;
  std::vector<int> sample_cell;
  std::vector<double> u_par_filt;
  bool filt_ready = false;

  // ABL inlet mean and temperature per boundary face, and the synthetic-eddy state
  // (src/abl/mod_abl_types.f90:SEMState, src/abl/mod_sem_inflow.f90)
  std::vector<double> abl_mean, abl_T, sem_fluc;
  struct Sem {
    bool initialized = false, dfsem = true, per1 = false, per2 = false;
    double n_in[3] = {0, 0, 0}, x_inlet[3] = {0, 0, 0}, t1[3] = {0, 0, 0}, t2[3] = {0, 0, 0};
    double t1_min = 0, t1_max = 0, t2_min = 0, t2_max = 0, period1 = 0, period2 = 0, per1_lo = 0, per2_lo = 0;
    double sigma = 0, rsup = 0, box_volume = 0, u_convect = 0, lam_ref = 0, sig_min = 0;
    int n = 0;
    std::vector<double> pos, amp, frame, sig, ampl;
    uint64_t rng = 88172645463325252ULL;
  } sem;

  // body forces (mod_fv_solver.f90:959-983, :1662-1699), nudging profiles
  // (src/abl/mod_abl_weather.f90:NudgingData) and passive-scalar sources (src/mod_scalar.f90)
  double mass_flux_force[3] = {0.0, 0.0, 0.0};
  int nd_nt = 0, nd_nz = 0;
  std::vector<double> nd_times, nd_z, nd_U, nd_T;  // U (3, nz, nt), T (nz, nt) Fortran order
  struct Src {
    dpm_scalar_source_t d;
    std::vector<double> tags;
  };
  std::vector<Src> srcs;

  // exact cell projection (src/numerics/mod_cell_projection.f90:cell_proj_t): pressure-face list
  // with interpolation weights, outlet faces, and the last step's iteration counts
  bool cp_on = false;
  std::vector<int> cp_own, cp_nbr, cp_bcell;
  std::vector<double> cp_sf, cp_gc, cp_bsf;
  int cp_iters = 0, cp_precond_iters = 0;

  // last-step diagnostics
  int last_solves = 0, last_iters = 0;
  double last_resid = 0.0, last_dt = 0.0;

  int bc_of_face(int64_t f) const { return m.patch[f] >= 0 ? pc[m.patch[f]].bc_id : BC_ZEROGRADIENT; }

  // ------------------------------------------------------------------------------------------
  int init(const dpm_raw_mesh_t* raw, const dpm_patch_cfg_t* patches, const dpm_params_t* prm, std::string* err) {
    RawMesh r;
    r.n_nodes = raw->n_nodes; r.xyz = raw->xyz; r.n_cells = raw->n_cells; r.cell_type = raw->cell_type;
    r.cell_off = raw->cell_off; r.cell_nodes = raw->cell_nodes; r.n_bfaces = raw->n_bfaces;
    r.bface_off = raw->bface_off; r.bface_nodes = raw->bface_nodes; r.bface_patch = raw->bface_patch;
    r.n_patches = raw->n_patches;
    std::vector<int> pbc(raw->n_patches);
    for (int i = 0; i < raw->n_patches; ++i) pbc[i] = patches[i].bc_id;
    int rc = build_mesh(r, pbc.data(), m, err);
    if (rc) return rc;
    P = *prm;
    if (P.cell_projection != DPM_CELL_PROJECTION_LS && P.cell_projection != DPM_CELL_PROJECTION_EXACT) {
      if (err) *err = "cell_projection must be LS or EXACT";
      return DPM_ERR_ARG;
    }
    pc.assign(patches, patches + raw->n_patches);
    nc = m.n_cells; nf = m.n_faces; nfi = m.n_int_faces; nb = m.n_bnd_faces;
    U.assign(3 * nc, 0.0); p.assign(nc, 0.0); p_old.assign(nc, 0.0); T.assign(nc, P.T_ref);
    nu_sgs.assign(nc, 0.0); U_bnd.assign(3 * nb, 0.0); p_bnd.assign(nb, 0.0);
    phi_prev.assign(nc, 0.0); phi_prev_bnd.assign(nb, 0.0); tau_w.assign(3 * nb, 0.0);
    grad_U.assign(9 * nc, 0.0); face_flux.assign(nf, 0.0); U_face.assign(nf, 0.0);
    T_bnd.assign(nb, P.T_ref); grad_T.assign(3 * nc, 0.0); H_T.assign(nc, 0.0); H_T0.assign(nc, 0.0);
    conv_T.assign(nc, 0.0); visc_T.assign(nc, 0.0);
    ns = std::max(0, std::min(P.n_scalars, 4));
    Cs.assign((size_t)ns * nc, 0.0); C_bnd.assign((size_t)ns * nb, 0.0); grad_C.assign((size_t)ns * 3 * nc, 0.0);
    H_C.assign((size_t)ns * nc, 0.0); H_C0.assign((size_t)ns * nc, 0.0); conv_C.assign(nc, 0.0); visc_C.assign(nc, 0.0);
    L_bnd.assign(nb, 0.0); q_w.assign(nb, 0.0); L_obukhov = P.abl_L_obukhov;
    auto scalar_ok = [](int sch) {
      return sch == DPM_SCHEME_CDS || sch == DPM_SCHEME_QUICK || sch == DPM_SCHEME_VANLEER_TVD || sch == DPM_SCHEME_KOREN_TVD;
    };
    if ((P.boussinesq && !scalar_ok(P.temperature_scheme)) || (ns > 0 && !scalar_ok(P.scalar_scheme))) {
      if (err) *err = "scalar advection scheme must be CDS, QUICK, VANLEER_TVD or KOREN_TVD";
      return DPM_ERR_UNSUPPORTED;
    }
    inv_vol.resize(nc);
    for (int64_t c = 0; c < nc; ++c) inv_vol[c] = 1.0 / std::max(m.volume[c], SMALL);
    H_U.assign(3 * nc, 0.0); H_U0.assign(3 * nc, 0.0); rhs_p.assign(nc, 0.0);
    conv_U.assign(3 * nc, 0.0); visc_U.assign(3 * nc, 0.0); gp.assign(3 * nc, 0.0); gp_rc.assign(3 * nc, 0.0);
    gp_cell.assign(3 * nc, 0.0); p_tot.assign(nc, 0.0); p_tot_bnd.assign(nb, 0.0); phi_it.assign(nc, 0.0);
    built.assign(nf, 0);
    Tinv.assign(9 * nc, 0.0);
    for (int64_t c = 0; c < nc; ++c) Tinv[9 * c] = Tinv[9 * c + 4] = Tinv[9 * c + 8] = 1.0;
    abl_inlet_profiles();
    // build_patch_classification
    for (int q = 0; q < m.n_patches; ++q)
      for (int64_t f = 0; f < m.patch_nfaces[q]; ++f)
        (pc[q].bc_id == BC_PERIODIC ? per_bf : nper_bf).push_back(m.patch_start[q] + f);
    n_outlet = 0;
    for (int q = 0; q < m.n_patches; ++q)
      if (pc[q].bc_id == BC_OUTLET) n_outlet += m.patch_nfaces[q];
    apply_velocity_bc(-1, false);
    apply_pressure_bc(p.data(), -1, false, false);
    apply_temperature_bc(-1);
    for (int sc = 0; sc < ns; ++sc) apply_scalar_bc(sc, -1);
    // initialize_velocity_from_bc
    double u0[3] = {0, 0, 0};
    for (int q = 0; q < m.n_patches; ++q)
      if (pc[q].bc_id == BC_INLET) { for (int k = 0; k < 3; ++k) u0[k] = pc[q].U_val[k]; break; }
    for (int64_t c = 0; c < nc; ++c)
      for (int k = 0; k < 3; ++k) U[3 * c + k] = u0[k];
    pressure_solver_init();
    V_min = 1e300; V_total = 0.0;
    for (int64_t c = 0; c < nc; ++c) { V_min = std::min(V_min, m.volume[c]); V_total += m.volume[c]; }
    p_atol_factor = 1.0e-15;
    detect_nonortho_skip();
    build_nonortho_cache();
    build_reconstruct_operator();
    diag_interface = false;
    for (int64_t f = 0; f < nfi; ++f)
      if (m.is_refine[f]) { diag_interface = true; break; }
    build_filter_tensor();
    build_cell_projection();
    if (P.use_sem && sem_init()) update_sem_inflow(time, false, 0.0);  // mod_fv_solver.f90:486-492
    return 0;
  }

  // ------------------------------------------------------------------ ABL inlet (mod_abl_profiles.f90)
  static double ustar_from_ref(double u_ref, double z_ref, double z0) {
    return (z_ref > z0 && z0 > SMALL && u_ref > SMALL) ? KAPPA * u_ref / std::log(z_ref / z0) : 0.05 * u_ref;
  }
  static double u_profile(double z, double u_star, double z0) {  // neutral (L = 0)
    if (z <= z0 || u_star <= SMALL || z0 <= SMALL) return 0.0;
    return (u_star / KAPPA) * std::log(z / z0);
  }
  double patch_z0m(int q) const { return pc[q].abl_z0_m > 0.0 ? pc[q].abl_z0_m : P.abl_z0_m; }
  double patch_z0h(int q) const { return pc[q].abl_z0_h > 0.0 ? pc[q].abl_z0_h : P.abl_z0_h; }
  // the log-law mean (mod_bc.f90:352-372) and temperature (:557-562, abl_T_profile) of each
  // ABL-inlet face; the synthetic fluctuation starts at zero
  void abl_inlet_profiles() {
    abl_mean.assign(3 * nb, 0.0);
    abl_T.assign(nb, P.T_ref);
    sem_fluc.assign(3 * nb, 0.0);
    const double wr = P.abl_wind_dir_deg * 3.14159265358979323846 / 180.0;
    for (int64_t fb = 0; fb < nb; ++fb) {
      int64_t fg = nfi + fb;
      if (bc_of_face(fg) != BC_ABL_INLET) continue;
      const int q = m.patch[fg];
      const double z = m.centre[3 * fg + 2];
      const double us = ustar_from_ref(P.abl_u_ref, P.abl_z_ref, patch_z0m(q));
      const double um = u_profile(z, us, patch_z0m(q));
      abl_mean[3 * fb] = -um * std::sin(wr);
      abl_mean[3 * fb + 1] = -um * std::cos(wr);
      const double z0h = patch_z0h(q);
      const double ts = (P.abl_z_ref > z0h && z0h > SMALL) ? KAPPA * (P.abl_T_ref - P.abl_T_surface) / std::log(P.abl_z_ref / z0h) : 0.0;
      double Tz = P.abl_T_surface;
      if (!(z <= z0h || std::fabs(ts) <= SMALL || z0h <= SMALL)) Tz = P.abl_T_surface + (ts / KAPPA) * std::log(z / z0h);
      abl_T[fb] = Tz;
    }
  }

  // ------------------------------------------------------------------ synthetic eddies (mod_sem_inflow.f90)
  static constexpr double SEM_SMALL = 1.0e-16, SEM_PI = 3.14159265358979323846;
  double sem_rand() {  // :50-55, xorshift64
    sem.rng ^= sem.rng << 13;
    sem.rng ^= sem.rng >> 7;
    sem.rng ^= sem.rng << 17;
    return (double)(sem.rng & 4503599627370495ULL) / 4503599627370496.0;
  }
  static void cross(const double* a, const double* b, double* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
  }
  // sem_inlet_frame + sem_detect_periodic (:59-165)
  bool sem_frame() {
    double ns[3] = {0, 0, 0}, xs[3] = {0, 0, 0}, asum = 0.0;
    for (int64_t fb = 0; fb < nb; ++fb) {
      int64_t fg = nfi + fb;
      if (bc_of_face(fg) != BC_ABL_INLET) continue;
      double a = m.area[fg];
      for (int k = 0; k < 3; ++k) { ns[k] = ns[k] + a * m.normal[3 * fg + k]; xs[k] = xs[k] + a * m.centre[3 * fg + k]; }
      asum = asum + a;
    }
    if (!(asum > SEM_SMALL)) return false;
    double nl = std::sqrt(ns[0] * ns[0] + ns[1] * ns[1] + ns[2] * ns[2]);
    if (nl <= SEM_SMALL) return false;
    for (int k = 0; k < 3; ++k) { sem.n_in[k] = -ns[k] / nl; sem.x_inlet[k] = xs[k] / asum; }
    const double ez[3] = {0, 0, 1}, ex[3] = {1, 0, 0};
    cross(std::fabs(sem.n_in[2]) < 0.9 ? ez : ex, sem.n_in, sem.t1);
    double tl = std::max(std::sqrt(sem.t1[0] * sem.t1[0] + sem.t1[1] * sem.t1[1] + sem.t1[2] * sem.t1[2]), SEM_SMALL);
    for (int k = 0; k < 3; ++k) sem.t1[k] = sem.t1[k] / tl;
    cross(sem.n_in, sem.t1, sem.t2);
    double lo[2] = {1.7976931348623157e308, 1.7976931348623157e308}, hi[2] = {-1.7976931348623157e308, -1.7976931348623157e308};
    for (int64_t fb = 0; fb < nb; ++fb) {
      int64_t fg = nfi + fb;
      if (bc_of_face(fg) != BC_ABL_INLET) continue;
      double d[3];
      for (int k = 0; k < 3; ++k) d[k] = m.centre[3 * fg + k] - sem.x_inlet[k];
      double s1 = dot3(d, sem.t1), s2 = dot3(d, sem.t2);
      lo[0] = std::min(lo[0], s1); hi[0] = std::max(hi[0], s1);
      lo[1] = std::min(lo[1], s2); hi[1] = std::max(hi[1], s2);
    }
    sem.t1_min = lo[0]; sem.t1_max = hi[0]; sem.t2_min = lo[1]; sem.t2_max = hi[1];
    double plo[2] = {1.7976931348623157e308, 1.7976931348623157e308}, phi2[2] = {-1.7976931348623157e308, -1.7976931348623157e308};
    for (int k = 0; k < 2; ++k) {
      const double* tk = k == 0 ? sem.t1 : sem.t2;
      for (int64_t fb = 0; fb < nb; ++fb) {
        int64_t fg = nfi + fb;
        if (bc_of_face(fg) != BC_PERIODIC) continue;
        if (std::fabs(dot3(&m.normal[3 * fg], tk)) < 0.99) continue;
        double d[3];
        for (int j = 0; j < 3; ++j) d[j] = m.centre[3 * fg + j] - sem.x_inlet[j];
        double sv = dot3(d, tk);
        plo[k] = std::min(plo[k], sv); phi2[k] = std::max(phi2[k], sv);
      }
    }
    sem.per1 = sem.per2 = false;
    sem.period1 = sem.period2 = 0.0;
    if (phi2[0] - plo[0] > SEM_SMALL && plo[0] <= sem.t1_min + SEM_SMALL && phi2[0] >= sem.t1_max - SEM_SMALL) {
      sem.per1 = true; sem.period1 = phi2[0] - plo[0]; sem.per1_lo = plo[0];
    }
    if (phi2[1] - plo[1] > SEM_SMALL && plo[1] <= sem.t2_min + SEM_SMALL && phi2[1] >= sem.t2_max - SEM_SMALL) {
      sem.per2 = true; sem.period2 = phi2[1] - plo[1]; sem.per2_lo = plo[1];
    }
    return true;
  }
  // sem_target_at (:663-711) without a profile table: mean (global axes) and R = [uu,vv,ww,uv,uw,vw]
  void sem_target(double z, double um[3], double R[6]) const {
    const double z0 = P.abl_z0_m, zf = std::max(z0, 1.0e-6), zz = std::max(z, zf);
    const double us = ustar_from_ref(P.abl_u_ref, P.abl_z_ref, z0);
    double umag = P.sem_mean_law == DPM_SEM_MEAN_POWER ? P.abl_u_ref * std::pow(zz / std::max(P.abl_z_ref, SEM_SMALL), P.sem_alpha)
                                                       : u_profile(z, us, z0);
    const double wr = P.abl_wind_dir_deg * SEM_PI / 180.0;
    um[0] = -umag * std::sin(wr); um[1] = -umag * std::cos(wr); um[2] = 0.0;
    for (int k = 0; k < 6; ++k) R[k] = 0.0;
    if (P.sem_Iu_ref > 0.0) {
      const double zi = std::max(z, 10.0 * z0);
      const double Iu = P.sem_Iu_ref * std::log(std::max(P.abl_z_ref, 1.0001 * z0) / z0) / std::log(zi / z0);
      umag = P.sem_mean_law == DPM_SEM_MEAN_POWER ? P.abl_u_ref * std::pow(std::max(zi, zf) / std::max(P.abl_z_ref, SEM_SMALL), P.sem_alpha)
                                                  : u_profile(zi, us, z0);
      const double su = Iu * umag, sv = P.sem_Iv_ratio * su, sw = P.sem_Iw_ratio * su;
      R[0] = su * su; R[1] = sv * sv; R[2] = sw * sw;
      R[4] = P.sem_rho_uw * su * sw;
    } else {
      R[0] = (2.4 * us) * (2.4 * us);
      R[1] = (1.9 * us) * (1.9 * us);
      R[2] = (1.25 * us) * (1.25 * us);
      R[4] = -(us * us);
    }
  }
  // sem_stress_at (:725-748): Rm (row-major 3x3) in the mean-wind frame and the frame axes Wr
  void sem_stress(double z, double Rm[9], double Wr[9]) const {
    double um[3], R[6];
    sem_target(z, um, R);
    Rm[0] = R[0]; Rm[4] = R[1]; Rm[8] = R[2];
    Rm[1] = R[3]; Rm[3] = R[3];
    Rm[2] = R[4]; Rm[6] = R[4];
    Rm[5] = R[5]; Rm[7] = R[5];
    const double wr = P.abl_wind_dir_deg * SEM_PI / 180.0;
    // columns e_s, e_n, e_z
    Wr[0] = -std::sin(wr); Wr[3] = -std::cos(wr); Wr[6] = 0.0;
    Wr[1] = std::cos(wr);  Wr[4] = -std::sin(wr); Wr[7] = 0.0;
    Wr[2] = 0.0;           Wr[5] = 0.0;           Wr[8] = 1.0;
  }
  // sem_eigen3 (:752-792): cyclic Jacobi, A = V diag(lam) V^T (row-major V, columns the vectors)
  static void eigen3(const double Ain[9], double lam[3], double V[9]) {
    double A[3][3], W[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) A[i][j] = Ain[3 * i + j];
    for (int sweep = 1; sweep <= 30; ++sweep) {
      double off = std::fabs(A[0][1]) + std::fabs(A[0][2]) + std::fabs(A[1][2]);
      if (off <= 1.0e-15 * (std::fabs(A[0][0]) + std::fabs(A[1][1]) + std::fabs(A[2][2]) + SEM_SMALL)) break;
      for (int p = 0; p < 2; ++p)
        for (int q = p + 1; q < 3; ++q) {
          double apq = A[p][q];
          if (std::fabs(apq) <= SEM_SMALL) continue;
          double th = (A[q][q] - A[p][p]) / (2.0 * apq);
          double t = std::copysign(1.0, th) / (std::fabs(th) + std::sqrt(th * th + 1.0));
          double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c, tau = sn / (1.0 + c);
          A[p][p] = A[p][p] - t * apq;
          A[q][q] = A[q][q] + t * apq;
          A[p][q] = 0.0; A[q][p] = 0.0;
          for (int k = 0; k < 3; ++k) {
            if (k != p && k != q) {
              double akp = A[k][p], akq = A[k][q];
              A[k][p] = akp - sn * (akq + tau * akp); A[p][k] = A[k][p];
              A[k][q] = akq + sn * (akp - tau * akq); A[q][k] = A[k][q];
            }
            double vkp = W[k][p], vkq = W[k][q];
            W[k][p] = vkp - sn * (vkq + tau * vkp);
            W[k][q] = vkq + sn * (vkp - tau * vkq);
          }
        }
    }
    lam[0] = A[0][0]; lam[1] = A[1][1]; lam[2] = A[2][2];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) V[3 * i + j] = W[i][j];
  }
  // sem_reference_scales (:795-841)
  void sem_scales() {
    const int nl = 65;
    std::vector<double> zl(nl);
    const double zlo = sem.x_inlet[2] + sem.t2_min, zhi = sem.x_inlet[2] + sem.t2_max;
    for (int k = 1; k <= nl - 1; ++k) zl[k - 1] = zlo + (zhi - zlo) * (double)(k - 1) / (double)(nl - 2);
    zl[nl - 1] = P.abl_z_ref;
    double lmax = SEM_SMALL;
    double Rm[9], Wr[9], lam[3], V[9];
    for (int k = 0; k < nl; ++k) {
      sem_stress(zl[k], Rm, Wr);
      eigen3(Rm, lam, V);
      lmax = std::max(lmax, std::max(lam[0], std::max(lam[1], lam[2])));
    }
    sem.lam_ref = lmax;
    sem.rsup = sem.sigma;
    double fmin = 1.0;
    for (int k = 0; k < nl; ++k) {
      sem_stress(zl[k], Rm, Wr);
      eigen3(Rm, lam, V);
      double mx = std::max(lam[0], std::max(lam[1], lam[2])), mn = std::min(lam[0], std::min(lam[1], lam[2]));
      if (mx >= 0.25 * lmax) fmin = std::min(fmin, std::max(0.2, std::sqrt(std::max(mn, 0.0) / lmax)));
    }
    sem.sig_min = sem.sigma * fmin;
  }
  // sem_place_eddy (:320-338)
  void sem_place(int i, double sv, bool new_amp) {
    double a = sem.t1_min + (sem.t1_max - sem.t1_min) * sem_rand();
    double b = sem.t2_min + (sem.t2_max - sem.t2_min) * sem_rand();
    for (int k = 0; k < 3; ++k) sem.pos[3 * i + k] = sem.x_inlet[k] + sv * sem.n_in[k] + a * sem.t1[k] + b * sem.t2[k];
    if (new_amp)
      for (int k = 0; k < 3; ++k) sem.amp[3 * i + k] = std::copysign(1.0, sem_rand() - 0.5);
  }
  // sem_init + sem_setup + sem_balance_amplitudes (:176-316); false without an ABL inlet
  bool sem_init() {
    sem = Sem();
    if (!sem_frame()) return false;
    const int ne = std::max(1, P.sem_n_eddies);
    sem.n = ne;
    sem.pos.assign(3 * ne, 0.0);
    sem.amp.assign(3 * ne, 0.0);
    const double span1 = sem.t1_max - sem.t1_min, span2 = sem.t2_max - sem.t2_min;
    sem.sigma = P.sem_sigma <= SEM_SMALL ? 0.1 * std::min(span1, span2) : P.sem_sigma;
    if (sem.sigma <= SEM_SMALL) sem.sigma = 0.1 * P.abl_z_ref;
    sem.dfsem = P.sem_type != DPM_SEM_JARRIN;
    sem.rsup = sem.sigma;
    if (sem.dfsem) {
      sem.frame.assign(9 * ne, 0.0);
      sem.sig.assign(3 * ne, 0.0);
      sem.ampl.assign(3 * ne, 0.0);
      sem_scales();
    }
    if (sem.per1) { sem.t1_min = sem.per1_lo; sem.t1_max = sem.per1_lo + sem.period1; }
    else { sem.t1_min = sem.t1_min - sem.rsup; sem.t1_max = sem.t1_max + sem.rsup; }
    if (sem.per2) { sem.t2_min = sem.per2_lo; sem.t2_max = sem.per2_lo + sem.period2; }
    else { sem.t2_min = sem.t2_min - sem.rsup; sem.t2_max = sem.t2_max + sem.rsup; }
    sem.box_volume = 2.0 * sem.rsup * (sem.t1_max - sem.t1_min) * (sem.t2_max - sem.t2_min);
    sem.u_convect = std::max(P.abl_u_ref, SEM_SMALL);
    sem.rng = 88172645463325252ULL;
    if (P.sem_seed != 0) {
      sem.rng = 88172645463325252ULL ^ ((uint64_t)(int64_t)P.sem_seed * 2654435761ULL);
      if (sem.rng == 0) sem.rng = 88172645463325252ULL;
      for (int i = 0; i < 8; ++i) sem_rand();
    }
    for (int i = 0; i < ne; ++i) sem_place(i, sem.rsup * (2.0 * sem_rand() - 1.0), true);
    for (int k = 0; k < 3; ++k) {  // sem_balance_amplitudes
      double ssum = 0.0;
      for (int i = 0; i < ne; ++i) ssum = ssum + sem.amp[3 * i + k];
      for (int i = 0; i < ne; ++i) {
        if (std::fabs(ssum) < 1.0) break;
        if (sem.amp[3 * i + k] * ssum > 0.0) {
          sem.amp[3 * i + k] = -sem.amp[3 * i + k];
          ssum = ssum + 2.0 * sem.amp[3 * i + k];
        }
      }
    }
    if (sem.dfsem) sem_prepare();
    sem.initialized = true;
    return true;
  }
  // sem_prepare (:867-892)
  void sem_prepare() {
    if (!sem.dfsem) return;
    const double DF_I = 32.0 * SEM_PI / 945.0;
    for (int i = 0; i < sem.n; ++i) {
      double Rm[9], Wr[9], lam[3], V[9];
      sem_stress(sem.pos[3 * i + 2], Rm, Wr);
      eigen3(Rm, lam, V);
      double s[3];
      for (int j = 0; j < 3; ++j) {
        for (int r = 0; r < 3; ++r) {  // Vg = Wr V, column j
          double acc = 0.0;
          for (int k = 0; k < 3; ++k) acc = acc + Wr[3 * r + k] * V[3 * k + j];
          sem.frame[9 * i + 3 * j + r] = acc;
        }
        s[j] = sem.sigma * std::max(0.2, std::sqrt(std::max(lam[j], 0.0) / sem.lam_ref));
      }
      for (int j = 0; j < 3; ++j) sem.sig[3 * i + j] = s[j];
      const double K = (double)sem.n * s[0] * s[1] * s[2] * DF_I / sem.box_volume;
      double b[3], A[3];
      for (int j = 0; j < 3; ++j) b[j] = std::max(lam[j], 0.0) / (K * (s[j] * s[j]));
      A[0] = 0.5 * (b[1] + b[2] - b[0]);
      A[1] = 0.5 * (b[0] + b[2] - b[1]);
      A[2] = 0.5 * (b[0] + b[1] - b[2]);
      for (int j = 0; j < 3; ++j) sem.ampl[3 * i + j] = std::sqrt(std::max(A[j], 0.0)) * sem.amp[3 * i + j];
    }
  }
  // the eddy offset wrapped across periodic inlet directions (add_eddy, :968-976 / :1024-1032)
  void sem_wrap(double d[3]) const {
    if (sem.per1) {
      double k = std::round(dot3(d, sem.t1) / sem.period1);
      for (int j = 0; j < 3; ++j) d[j] = d[j] - sem.period1 * k * sem.t1[j];
    }
    if (sem.per2) {
      double k = std::round(dot3(d, sem.t2) / sem.period2);
      for (int j = 0; j < 3; ++j) d[j] = d[j] - sem.period2 * k * sem.t2[j];
    }
  }
  // sem_velocity_at_face (:933-978) and sem_velocity_jarrin (:980-1039), every eddy in index order
  void sem_face(const double* centre, bool look_ahead, double tau, double uf[3]) const {
    double xs[3];
    for (int k = 0; k < 3; ++k) xs[k] = look_ahead ? centre[k] - sem.u_convect * tau * sem.n_in[k] : centre[k];
    uf[0] = uf[1] = uf[2] = 0.0;
    if (sem.dfsem) {
      const double rs2 = sem.rsup * sem.rsup;
      for (int e = 0; e < sem.n; ++e) {
        double d[3];
        for (int k = 0; k < 3; ++k) d[k] = xs[k] - sem.pos[3 * e + k];
        sem_wrap(d);
        if (d[0] * d[0] + d[1] * d[1] + d[2] * d[2] >= rs2) continue;
        const double* fr = &sem.frame[9 * e];
        const double* sg = &sem.sig[3 * e];
        const double* al = &sem.ampl[3 * e];
        double r[3], d2 = 0.0;
        for (int j = 0; j < 3; ++j) {
          r[j] = dot3(d, fr + 3 * j) / sg[j];
          d2 = d2 + r[j] * r[j];
        }
        if (d2 >= 1.0) continue;
        const double g = 1.0 - d2;
        const double up0 = sg[0] * g * (r[1] * al[2] - r[2] * al[1]);
        const double up1 = sg[1] * g * (r[2] * al[0] - r[0] * al[2]);
        const double up2 = sg[2] * g * (r[0] * al[1] - r[1] * al[0]);
        for (int k = 0; k < 3; ++k) uf[k] = uf[k] + (up0 * fr[k] + up1 * fr[3 + k] + up2 * fr[6 + k]);
      }
      return;
    }
    double um[3], R[6];
    sem_target(centre[2], um, R);
    const double wr = P.abl_wind_dir_deg * SEM_PI / 180.0;
    const double sg = std::max(sem.sigma, SEM_SMALL);
    const double norm = 1.5450968080927583 * std::sqrt(sem.box_volume / (sg * sg * sg)) / std::sqrt((double)sem.n);
    double iso[3] = {0, 0, 0};
    for (int e = 0; e < sem.n; ++e) {
      double d[3];
      for (int k = 0; k < 3; ++k) d[k] = xs[k] - sem.pos[3 * e + k];
      sem_wrap(d);
      if (std::fabs(d[0]) >= sg || std::fabs(d[1]) >= sg || std::fabs(d[2]) >= sg) continue;
      const double rr = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) / sg;
      const double tent = std::max(0.0, 1.0 - rr);
      if (tent <= 0.0) continue;
      for (int k = 0; k < 3; ++k) iso[k] = iso[k] + norm * tent * sem.amp[3 * e + k];
    }
    // sem_cholesky (:651-661)
    double L11 = std::sqrt(std::max(R[0], SEM_SMALL));
    double L21 = R[3] / L11, L31 = R[4] / L11;
    double L22 = std::sqrt(std::max(R[1] - L21 * L21, SEM_SMALL));
    double L32 = (R[5] - L31 * L21) / L22;
    double L33 = std::sqrt(std::max(R[2] - L31 * L31 - L32 * L32, SEM_SMALL));
    const double a0 = L11 * iso[0], a1 = L21 * iso[0] + L22 * iso[1], a2 = L31 * iso[0] + L32 * iso[1] + L33 * iso[2];
    uf[0] = -a0 * std::sin(wr) + a1 * std::cos(wr);
    uf[1] = -a0 * std::cos(wr) - a1 * std::sin(wr);
    uf[2] = a2;
  }
  // update_sem_inflow (mod_fv_solver.f90:2062-2119): the fluctuation of every ABL-inlet face, then
  // the mean inflow it adds removed along each face normal
  void update_sem_inflow(double /*t*/, bool look_ahead, double tau) {
    std::fill(sem_fluc.begin(), sem_fluc.end(), 0.0);
    if (!sem.initialized) return;
    sem_prepare();
    double b1 = 0.0, b2 = 0.0;
    for (int64_t fb = 0; fb < nb; ++fb) {
      int64_t fg = nfi + fb;
      if (bc_of_face(fg) != BC_ABL_INLET) continue;
      double uf[3];
      sem_face(&m.centre[3 * fg], look_ahead, tau, uf);
      for (int k = 0; k < 3; ++k) sem_fluc[3 * fb + k] = uf[k];
      b1 = b1 + dot3(uf, &m.sf[3 * fg]);
      b2 = b2 + m.area[fg];
    }
    if (b2 <= SMALL) return;
    const double delta = b1 / b2;
    for (int64_t fb = 0; fb < nb; ++fb) {
      int64_t fg = nfi + fb;
      if (bc_of_face(fg) != BC_ABL_INLET) continue;
      for (int k = 0; k < 3; ++k) sem_fluc[3 * fb + k] = sem_fluc[3 * fb + k] - delta * m.normal[3 * fg + k];
    }
  }
  // sem_advance (:341-358)
  void sem_advance(double dt) {
    if (!sem.initialized) return;
    const double disp = sem.u_convect * dt;
    for (int i = 0; i < sem.n; ++i) {
      double d[3];
      for (int k = 0; k < 3; ++k) sem.pos[3 * i + k] = sem.pos[3 * i + k] + disp * sem.n_in[k];
      for (int k = 0; k < 3; ++k) d[k] = sem.pos[3 * i + k] - sem.x_inlet[k];
      if (dot3(d, sem.n_in) > sem.rsup) sem_place(i, -sem.rsup, false);
    }
  }

  // src/solver/mod_pressure_solver.f90:100-452
  void pressure_solver_init() {
    int64_t n_per_edges = 0;
    auto per_nb = [&](int64_t f_bnd) -> int {
      int pb = m.periodic_pair[f_bnd];
      return pb >= 0 ? m.owner[nfi + pb] : -1;
    };
    for (int q = 0; q < m.n_patches; ++q) {
      if (pc[q].bc_id != BC_PERIODIC) continue;
      for (int64_t fl = 0; fl < m.patch_nfaces[q]; ++fl) {
        int64_t fb = m.patch_start[q] + fl;
        int nbc = per_nb(fb);
        int o = m.owner[nfi + fb];
        if (nbc < 0 || o == nbc || o >= nbc) continue;
        n_per_edges++;
      }
    }
    nfp = nfi + n_per_edges;
    ps_owner.assign(nfp, -1); ps_nb.assign(nfp, -1); ps_mesh.assign(nfp, -1);
    ps_skip.assign(nfp, 0); ps_coeff.assign(nfp, 0.0); ps_diag.assign(nc, 0.0);
    for (int64_t i = 0; i < nfi; ++i) { ps_owner[i] = m.owner[i]; ps_mesh[i] = (int)i; ps_nb[i] = m.neighbour[i]; }
    int64_t idx = nfi;
    for (int q = 0; q < m.n_patches; ++q) {
      if (pc[q].bc_id != BC_PERIODIC) continue;
      for (int64_t fl = 0; fl < m.patch_nfaces[q]; ++fl) {
        int64_t fb = m.patch_start[q] + fl, fg = nfi + fb;
        int nbc = per_nb(fb);
        int o = m.owner[fg];
        if (nbc < 0 || o == nbc || o >= nbc) continue;
        ps_owner[idx] = o; ps_mesh[idx] = (int)fg; ps_nb[idx] = nbc;
        int pbd = m.periodic_pair[fb];
        double pair_dcf = m.periodic_pair_dcf[fb];
        int64_t pf = pbd >= 0 ? nfi + pbd : -1;
        if (pair_dcf <= SMALL && pf >= 0) pair_dcf = m.d_cf[pf];
        if (pair_dcf <= SMALL) pair_dcf = m.d_cf[fg];
        double d_per = m.d_cf[fg] + pair_dcf;
        double area_f = m.area[fg];
        if (pf >= 0) area_f = 0.5 * (area_f + m.area[pf]);
        double coeff = area_f / (d_per + SMALL);
        ps_coeff[idx] = coeff;
        ps_diag[o] += coeff;
        ps_diag[nbc] += coeff;
        idx++;
      }
    }
    double cos_floor = P.pressure_min_cos_theta;
    for (int64_t i = 0; i < nfi; ++i) {
      int o = m.owner[i], n = m.neighbour[i];
      double d[3];
      for (int k = 0; k < 3; ++k) d[k] = m.centroid[3 * n + k] - m.centroid[3 * o + k];
      double d_ortho = dot3(d, &m.normal[3 * i]);
      if (cos_floor > 0.0 && d_ortho < cos_floor * m.d_cf[i]) d_ortho = cos_floor * m.d_cf[i];
      double coeff = d_ortho > SMALL ? m.area[i] / d_ortho : m.area[i] / (m.d_cf[i] + SMALL);
      if (!finite(coeff) || coeff <= SMALL) { ps_skip[i] = 1; continue; }
      ps_coeff[i] = coeff;
      ps_diag[o] += coeff;
      ps_diag[n] += coeff;
    }
    dir_rows.clear(); dir_vals.clear();
    for (int q = 0; q < m.n_patches; ++q) {
      if (pc[q].bc_id != BC_OUTLET) continue;
      for (int64_t fl = 0; fl < m.patch_nfaces[q]; ++fl) {
        int64_t fg = nfi + m.patch_start[q] + fl;
        int o = m.owner[fg];
        double d[3];
        for (int k = 0; k < 3; ++k) d[k] = m.centre[3 * fg + k] - m.centroid[3 * o + k];
        double dpb = std::fabs(dot3(d, &m.normal[3 * fg]));
        if (dpb <= SMALL) dpb = m.d_cf[fg];
        if (cos_floor > 0.0) dpb = std::max(dpb, cos_floor * m.d_cf[fg]);
        if (dpb <= SMALL) continue;
        double cb = m.area[fg] / dpb;
        if (!finite(cb) || cb <= SMALL) continue;
        ps_diag[o] += cb;
        dir_rows.push_back(o);
        dir_vals.push_back(cb * pc[q].p_val);
      }
    }
    for (int64_t c = 0; c < nc; ++c)
      if (!finite(ps_diag[c]) || ps_diag[c] <= SMALL) ps_diag[c] = 1.0;
    // Assemble the AIJ matrix (pressure_backend_petsc.c:330-360): diag, -coeff off-diagonals.
    std::vector<std::vector<std::pair<int, double>>> rows(nc);
    for (int64_t c = 0; c < nc; ++c) rows[c].push_back({(int)c, ps_diag[c]});
    for (int64_t i = 0; i < nfp; ++i) {
      if (ps_skip[i] || ps_coeff[i] == 0.0) continue;
      rows[ps_owner[i]].push_back({ps_nb[i], -ps_coeff[i]});
      rows[ps_nb[i]].push_back({ps_owner[i], -ps_coeff[i]});
    }
    A_off.assign(nc + 1, 0);
    A_col.clear(); A_val.clear();
    for (int64_t c = 0; c < nc; ++c) {
      auto& r = rows[c];
      std::stable_sort(r.begin(), r.end(), [](auto& a, auto& b) { return a.first < b.first; });
      for (size_t j = 0; j < r.size(); ++j) {
        if (!A_col.empty() && (int64_t)A_col.size() > A_off[c] && A_col.back() == r[j].first) {
          A_val.back() += r[j].second;  // ADD_VALUES on a repeated entry
        } else {
          A_col.push_back(r[j].first);
          A_val.push_back(r[j].second);
        }
      }
      A_off[c + 1] = (int64_t)A_col.size();
    }
  }

  // src/solver/mod_fv_solver.f90:1864-1941
  void detect_nonortho_skip() {
    int64_t n_active = 0, n_gradbc = 0;
    for (int64_t i = 0; i < nfp; ++i) {
      if (ps_skip[i]) continue;
      int o = ps_owner[i], n = ps_nb[i];
      int64_t fm = ps_mesh[i];
      double d[3], k[3];
      for (int j = 0; j < 3; ++j) d[j] = m.centroid[3 * n + j] - m.centroid[3 * o + j];
      kfactor_limited(&m.sf[3 * fm], d, P.pressure_min_cos_theta, k);
      if (dot3(k, k) >= NONORTHO_SIN2_TOL * dot3(&m.sf[3 * fm], &m.sf[3 * fm])) n_active++;
    }
    for (int64_t fb : nper_bf) {
      int64_t fg = nfi + fb;
      if (bc_of_face(fg) != BC_OUTLET) continue;
      int o = m.owner[fg];
      double d[3], k[3];
      for (int j = 0; j < 3; ++j) d[j] = m.centre[3 * fg + j] - m.centroid[3 * o + j];
      kfactor_limited(&m.sf[3 * fg], d, P.pressure_min_cos_theta, k);
      if (dot3(k, k) >= NONORTHO_SIN2_TOL * dot3(&m.sf[3 * fg], &m.sf[3 * fg])) n_active++;
    }
    for (int q = 0; q < m.n_patches; ++q) {
      int b = pc[q].bc_id;
      if (!(b == BC_OUTLET || b == BC_PERIODIC || b == BC_WALL_NOSLIP || b == BC_WALL_VELOCITY ||
            b == BC_WALL_MODEL || b == BC_SLIP || b == BC_SYMMETRY))
        n_gradbc++;
    }
    skip_nonortho = (n_active == 0);
    skip_grad_p = skip_nonortho && (n_gradbc == 0);
    if (P.n_nonortho_corr <= 0) P.n_nonortho_corr = skip_nonortho ? 1 : 2;
  }

  // src/solver/mod_fv_solver.f90:1943-1997
  void build_nonortho_cache() {
    k_int.assign(3 * nfp, 0.0); act_int.assign(nfp, 0);
    k_bnd.assign(3 * nper_bf.size(), 0.0); act_bnd.assign(nper_bf.size(), 0);
    if (skip_nonortho) return;
    for (int64_t i = 0; i < nfp; ++i) {
      if (ps_skip[i]) continue;
      int o = ps_owner[i], n = ps_nb[i];
      int64_t fm = ps_mesh[i];
      double d[3], k[3];
      for (int j = 0; j < 3; ++j) d[j] = m.centroid[3 * n + j] - m.centroid[3 * o + j];
      kfactor_limited(&m.sf[3 * fm], d, P.pressure_min_cos_theta, k);
      if (dot3(k, k) >= NONORTHO_SIN2_TOL * dot3(&m.sf[3 * fm], &m.sf[3 * fm])) {
        for (int j = 0; j < 3; ++j) k_int[3 * i + j] = k[j];
        act_int[i] = 1;
      }
    }
    for (size_t ib = 0; ib < nper_bf.size(); ++ib) {
      int64_t fg = nfi + nper_bf[ib];
      if (bc_of_face(fg) != BC_OUTLET) continue;
      int o = m.owner[fg];
      double d[3], k[3];
      for (int j = 0; j < 3; ++j) d[j] = m.centre[3 * fg + j] - m.centroid[3 * o + j];
      kfactor_limited(&m.sf[3 * fg], d, P.pressure_min_cos_theta, k);
      if (dot3(k, k) >= NONORTHO_SIN2_TOL * dot3(&m.sf[3 * fg], &m.sf[3 * fg])) {
        for (int j = 0; j < 3; ++j) k_bnd[3 * ib + j] = k[j];
        act_bnd[ib] = 1;
      }
    }
  }

  // src/solver/mod_fv_solver.f90:3410-3495 (T = sum |Sf| n n^T over closing faces, inverted)
  void build_reconstruct_operator() {
    std::vector<double> Tm(9 * nc, 0.0);
    auto add = [&](int c, int64_t f) {
      const double* n = &m.normal[3 * f];
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) Tm[9 * c + i + 3 * j] += m.area[f] * n[i] * n[j];
    };
    for (int64_t i = 0; i < nfp; ++i) {
      if (ps_skip[i]) continue;
      add(ps_owner[i], ps_mesh[i]);
      add(ps_nb[i], ps_mesh[i]);
    }
    for (int64_t fb : nper_bf) add(m.owner[nfi + fb], nfi + fb);
    for (int64_t c = 0; c < nc; ++c) {
      const double* A = &Tm[9 * c];
      auto a = [&](int i, int j) { return A[(i - 1) + 3 * (j - 1)]; };
      double c11 = a(2, 2) * a(3, 3) - a(2, 3) * a(3, 2);
      double c12 = a(1, 3) * a(3, 2) - a(1, 2) * a(3, 3);
      double c13 = a(1, 2) * a(2, 3) - a(1, 3) * a(2, 2);
      double c22 = a(1, 1) * a(3, 3) - a(1, 3) * a(3, 1);
      double c23 = a(1, 3) * a(2, 1) - a(1, 1) * a(2, 3);
      double c33 = a(1, 1) * a(2, 2) - a(1, 2) * a(2, 1);
      double det = a(1, 1) * c11 + a(1, 2) * (a(2, 3) * a(3, 1) - a(2, 1) * a(3, 3)) +
                   a(1, 3) * (a(2, 1) * a(3, 2) - a(2, 2) * a(3, 1));
      double tr = a(1, 1) + a(2, 2) + a(3, 3);
      double* Ti = &Tinv[9 * c];
      double mt = std::max(tr, SMALL);
      if (std::fabs(det) <= 1.0e-12 * mt * mt * mt) {
        for (int k = 0; k < 9; ++k) Ti[k] = 0.0;
        Ti[0] = Ti[4] = Ti[8] = 3.0 / mt;
        continue;
      }
      // Ti column-major: Ti[(i-1) + 3(j-1)] = Ainv(i,j)
      Ti[0] = c11 / det; Ti[3] = c12 / det; Ti[6] = c13 / det;
      Ti[1] = c12 / det; Ti[4] = c22 / det; Ti[7] = c23 / det;
      Ti[2] = c13 / det; Ti[5] = c23 / det; Ti[8] = c33 / det;
    }
  }

  // src/sgs/mod_vreman.f90:168-264 (build_filter_tensor + smooth_filter_tensor)
  void build_filter_tensor() {
    Gf.assign(9 * nc, 0.0);
    for (int64_t c = 0; c < nc; ++c) {
      double d2 = std::pow(m.volume[c], 2.0 / 3.0);
      double g[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int64_t k = m.cell_face_off[c]; k < m.cell_face_off[c + 1]; ++k) {
        int f = m.cell_faces[k];
        double dx[3];
        for (int j = 0; j < 3; ++j) dx[j] = m.centre[3 * (int64_t)f + j] - m.centroid[3 * c + j];
        for (int n = 0; n < 3; ++n)
          for (int mm = 0; mm < 3; ++mm) g[mm + 3 * n] += m.area[f] * dx[mm] * dx[n];
      }
      double det = det3(g);
      double t = (g[0] + g[4] + g[8]) / 3.0;
      double tr3 = t * t * t;
      if (tr3 > 0.0 && det > 1.0e-12 * tr3) {
        double s = std::pow(m.volume[c] * m.volume[c] / det, 1.0 / 3.0);
        for (int j = 0; j < 9; ++j) Gf[9 * c + j] = s * g[j];
      } else {
        Gf[9 * c] = Gf[9 * c + 4] = Gf[9 * c + 8] = d2;
      }
    }
    std::vector<double> gnb(9 * nc), ws(nc);
    for (int pass = 0; pass < 2; ++pass) {
      std::fill(gnb.begin(), gnb.end(), 0.0);
      std::fill(ws.begin(), ws.end(), 0.0);
      for (int64_t f = 0; f < nf; ++f) {
        int o = m.owner[f], n = m.neighbour[f];
        if (n < 0) continue;
        double a = m.area[f];
        for (int j = 0; j < 9; ++j) gnb[9 * o + j] += a * Gf[9 * n + j];
        ws[o] += a;
        for (int j = 0; j < 9; ++j) gnb[9 * n + j] += a * Gf[9 * o + j];
        ws[n] += a;
      }
      for (int64_t c = 0; c < nc; ++c)
        if (ws[c] > SMALL)
          for (int j = 0; j < 9; ++j) Gf[9 * c + j] = 0.5 * Gf[9 * c + j] + 0.5 * gnb[9 * c + j] / ws[c];
    }
  }

  // ---------------------------------------------------------------- boundary conditions
  // src/bc/mod_bc.f90:196-380.  filt: -1 all faces, 0 non-periodic only, 1 periodic only.
  void apply_velocity_bc(int filt, bool have_grad) {
    for (int64_t fb = 0; fb < nb; ++fb) {
      int64_t fg = nfi + fb;
      int bc = bc_of_face(fg);
      if (filt == 1 && bc != BC_PERIODIC) continue;
      if (filt == 0 && bc == BC_PERIODIC) continue;
      int o = m.owner[fg];
      const double* n = &m.normal[3 * fg];
      double u[3] = {U_bnd[3 * fb], U_bnd[3 * fb + 1], U_bnd[3 * fb + 2]};
      switch (bc) {
        case BC_INLET:
          for (int k = 0; k < 3; ++k) u[k] = pc[m.patch[fg]].U_val[k];
          break;
        case BC_ABL_INLET:  // mod_bc.f90:352-372: the log-law mean plus the synthetic fluctuation
          for (int k = 0; k < 3; ++k) u[k] = abl_mean[3 * fb + k] + sem_fluc[3 * fb + k];
          break;
        case BC_OUTLET:
        case BC_ZEROGRADIENT: {
          for (int k = 0; k < 3; ++k) u[k] = U[3 * o + k];
          if (have_grad) {
            double d[3];
            for (int k = 0; k < 3; ++k) d[k] = m.centre[3 * fg + k] - m.centroid[3 * o + k];
            for (int k = 0; k < 3; ++k)
              u[k] = u[k] + grad_U[9 * o + 3 * k] * d[0] + grad_U[9 * o + 3 * k + 1] * d[1] + grad_U[9 * o + 3 * k + 2] * d[2];
          }
          break;
        }
        case BC_WALL_NOSLIP:
        case BC_WALL_MODEL:
          u[0] = u[1] = u[2] = 0.0;
          break;
        case BC_WALL_VELOCITY: {
          for (int k = 0; k < 3; ++k) u[k] = pc[m.patch[fg]].U_val[k];
          double un = u[0] * n[0] + u[1] * n[1] + u[2] * n[2];
          for (int k = 0; k < 3; ++k) u[k] = u[k] - un * n[k];
          break;
        }
        case BC_PERIODIC: {
          for (int k = 0; k < 3; ++k) u[k] = U[3 * o + k];
          int pnb = m.periodic_partner_cell(fb);
          if (pnb >= 0 && pnb != o) {
            double w = m.periodic_gc[fb];
            for (int k = 0; k < 3; ++k) u[k] = w * u[k] + (1.0 - w) * U[3 * pnb + k];
          }
          break;
        }
        case BC_SLIP:
        case BC_SYMMETRY: {
          for (int k = 0; k < 3; ++k) u[k] = U[3 * o + k];
          double un = u[0] * n[0] + u[1] * n[1] + u[2] * n[2];
          for (int k = 0; k < 3; ++k) u[k] = u[k] - un * n[k];
          break;
        }
        default:
          break;
      }
      for (int k = 0; k < 3; ++k) U_bnd[3 * fb + k] = u[k];
    }
  }

  // src/bc/mod_bc.f90:383-486.  pf: cell pressure-like field; writes p_bnd.
  void apply_pressure_bc(const double* pf, int filt, bool have_grad, bool increment) {
    double oscale = increment ? 0.0 : 1.0;
    for (int64_t fb = 0; fb < nb; ++fb) {
      int64_t fg = nfi + fb;
      int bc = bc_of_face(fg);
      if (filt == 1 && bc != BC_PERIODIC) continue;
      if (filt == 0 && bc == BC_PERIODIC) continue;
      int o = m.owner[fg];
      switch (bc) {
        case BC_OUTLET:
          p_bnd[fb] = oscale * pc[m.patch[fg]].p_val;
          break;
        case BC_PERIODIC: {
          int pnb = m.periodic_partner_cell(fb);
          if (pnb >= 0 && pnb != o) p_bnd[fb] = m.periodic_gc[fb] * pf[o] + (1.0 - m.periodic_gc[fb]) * pf[pnb];
          else p_bnd[fb] = pf[o];
          break;
        }
        case BC_WALL_NOSLIP: case BC_WALL_VELOCITY: case BC_WALL_MODEL: case BC_SLIP: case BC_SYMMETRY:
          p_bnd[fb] = pf[o] - 0.0;  // a_wall = 0: p_bnd = p_o - (a_wall.n) d_ortho
          break;
        default:
          if (have_grad) {
            double d[3];
            for (int k = 0; k < 3; ++k) d[k] = m.centre[3 * fg + k] - m.centroid[3 * o + k];
            p_bnd[fb] = pf[o] + gp[3 * o] * d[0] + gp[3 * o + 1] * d[1] + gp[3 * o + 2] * d[2];
          } else {
            p_bnd[fb] = pf[o];
          }
      }
    }
  }

  void refresh_halos_and_bc() {  // src/solver/mod_fv_solver.f90:985-1001, 2024-2059
    apply_velocity_bc(0, true);
    apply_pressure_bc(p.data(), 0, !skip_grad_p, false);
    apply_temperature_bc(0);
    for (int sc = 0; sc < ns; ++sc) apply_scalar_bc(sc, 0);
    apply_velocity_bc(1, true);
    apply_pressure_bc(p.data(), 1, !skip_grad_p, false);
    apply_temperature_bc(1);
    for (int sc = 0; sc < ns; ++sc) apply_scalar_bc(sc, 1);
  }

  // src/bc/mod_bc.f90:489-588 (apply_temperature_bc; every caller passes grad_T, so the default
  // branch always extrapolates with it).
  void apply_temperature_bc(int filt) {
    for (int64_t fb = 0; fb < nb; ++fb) {
      int64_t fg = nfi + fb;
      int bc = bc_of_face(fg);
      if (filt == 1 && bc != BC_PERIODIC) continue;
      if (filt == 0 && bc == BC_PERIODIC) continue;
      int o = m.owner[fg];
      switch (bc) {
        case BC_INLET:
        case BC_FIXEDTEMP:
          T_bnd[fb] = pc[m.patch[fg]].T_val;
          break;
        case BC_ABL_INLET:  // mod_bc.f90:559-562
          T_bnd[fb] = abl_T[fb];
          break;
        case BC_PERIODIC: {
          int pnb = m.periodic_partner_cell(fb);
          if (pnb >= 0 && pnb != o) T_bnd[fb] = m.periodic_gc[fb] * T[o] + (1.0 - m.periodic_gc[fb]) * T[pnb];
          else T_bnd[fb] = T[o];
          break;
        }
        default: {
          double d[3];
          for (int k = 0; k < 3; ++k) d[k] = m.centre[3 * fg + k] - m.centroid[3 * o + k];
          T_bnd[fb] = T[o] + grad_T[3 * o] * d[0] + grad_T[3 * o + 1] * d[1] + grad_T[3 * o + 2] * d[2];
        }
      }
    }
  }

  // src/bc/mod_bc.f90:591-680 (apply_passive_scalar_bc; modes 0 zero gradient, 1 Dirichlet,
  // 2 Neumann with a constant flux per area; the face diffusivity uses the global Pr_t, as the
  // reference's callers pass it, mod_fv_solver.f90:2049-2056)
  void apply_scalar_bc(int sc, int filt) {
    const double* C = &Cs[(size_t)sc * nc];
    double* Cb = &C_bnd[(size_t)sc * nb];
    for (int64_t fb = 0; fb < nb; ++fb) {
      int64_t fg = nfi + fb;
      int bc = bc_of_face(fg);
      if (filt == 1 && bc != BC_PERIODIC) continue;
      if (filt == 0 && bc == BC_PERIODIC) continue;
      int o = m.owner[fg];
      if (bc == BC_PERIODIC) {
        int pnb = m.periodic_partner_cell(fb);
        if (pnb >= 0 && pnb != o) Cb[fb] = m.periodic_gc[fb] * C[o] + (1.0 - m.periodic_gc[fb]) * C[pnb];
        else Cb[fb] = C[o];
        continue;
      }
      const int q = m.patch[fg];
      const int mode = q >= 0 ? pc[q].scalar_mode[sc] : 0;
      if (mode == 1) {
        Cb[fb] = pc[q].scalar_value[sc];
      } else if (mode == 2) {
        double alpha = P.scalar_diffusivity[sc] + nu_sgs[o] / P.Pr_t;
        double d = std::max(m.d_cf[fg], SMALL);
        Cb[fb] = alpha > SMALL ? C[o] + pc[q].scalar_value[sc] * d / alpha : C[o];
      } else {
        Cb[fb] = C[o];
      }
    }
  }
  void apply_scalar_bcs_all() {  // apply_scalar_bc (mod_fv_solver.f90:2005-2022), after each step
    apply_temperature_bc(-1);
    for (int sc = 0; sc < ns; ++sc) apply_scalar_bc(sc, -1);
  }
  void velocity_bc_refresh() {  // the apply_velocity_bc pair after each U update
    apply_velocity_bc(0, true);
    apply_velocity_bc(1, true);
  }
  void apply_pressure_bc_o2(bool incr) {  // src/solver/mod_fv_solver.f90:2324-2338
    apply_pressure_bc(p.data(), 0, !skip_grad_p, incr);
  }

  // ---------------------------------------------------------------- gradients
  // src/numerics/mod_gradient.f90:425-613 (CPU path)
  void ls_gradient_vector(const double* Uc, const double* Ub, double* g) {
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t c = 0; c < nc; ++c) {
      double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int64_t k = m.ls_off[c]; k < m.ls_off[c + 1]; ++k) {
        int n = m.ls_cell[k];
        double un[3];
        if (n < 0) {
          int f = m.ls_face[k];
          int64_t bi = f >= 0 ? f - nfi : -1;
          if (bi >= 0 && bi < nb) for (int j = 0; j < 3; ++j) un[j] = Ub[3 * bi + j];
          else for (int j = 0; j < 3; ++j) un[j] = Uc[3 * c + j];
        } else {
          for (int j = 0; j < 3; ++j) un[j] = Uc[3 * (int64_t)n + j];
        }
        for (int j = 0; j < 3; ++j) {
          double du = un[j] - Uc[3 * c + j];
          for (int i = 0; i < 3; ++i) acc[i + 3 * j] += m.ls_w[3 * k + i] * du;
        }
      }
      for (int j = 0; j < 9; ++j) g[9 * c + j] = acc[j];
    }
  }
  // src/numerics/mod_gradient.f90:307-423 (CPU path)
  void ls_gradient_scalar(const double* phi, const double* pb, double* g) {
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t c = 0; c < nc; ++c) {
      double acc[3] = {0, 0, 0};
      for (int64_t k = m.ls_off[c]; k < m.ls_off[c + 1]; ++k) {
        int n = m.ls_cell[k];
        double v;
        if (n < 0) {
          int f = m.ls_face[k];
          int64_t bi = f >= 0 ? f - nfi : -1;
          v = (bi >= 0 && bi < nb) ? pb[bi] : phi[c];
        } else {
          v = phi[n];
        }
        double d = v - phi[c];
        for (int i = 0; i < 3; ++i) acc[i] += m.ls_w[3 * k + i] * d;
      }
      for (int i = 0; i < 3; ++i) g[3 * c + i] = acc[i];
    }
  }
  // src/numerics/mod_gradient.f90:38-168 (serial path): grad_c = (1/V_c) sum_f phi_f S_f, with
  // phi_f the gc-interpolated face value (+ mean previous gradient . eps when gprev is given,
  // faded by the refinement blend on interior faces) or the boundary value.  Each cell sums its
  // faces in face order, as the face loop of the reference adds them.
  void gg_gradient_scalar(const double* phi, const double* pb, double* g, const double* gprev) {
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t c = 0; c < nc; ++c) {
      double acc[3] = {0, 0, 0};
      for (int64_t k = m.cell_face_off[c]; k < m.cell_face_off[c + 1]; ++k) {
        const int f = m.cell_faces[k];
        const double* sf = &m.sf[3 * (size_t)f];
        if (f < nfi) {
          const int o = m.owner[f], n = m.neighbour[f];
          const double w = m.gc[f];
          double pf;
          if (gprev) {
            const double* e = &m.eps[3 * (size_t)f];
            double gm[3];
            for (int i = 0; i < 3; ++i) gm[i] = w * gprev[3 * (size_t)o + i] + (1.0 - w) * gprev[3 * (size_t)n + i];
            const double plain = w * phi[o] + (1.0 - w) * phi[n];
            pf = plain + (gm[0] * e[0] + gm[1] * e[1] + gm[2] * e[2]);
            const double wb = refine_blend_weight(m.skew[f]);
            if (wb < 1.0) pf = plain + wb * (pf - plain);
          } else {
            pf = w * phi[o] + (1.0 - w) * phi[n];
          }
          if (o == c) for (int i = 0; i < 3; ++i) acc[i] = acc[i] + pf * sf[i];
          else for (int i = 0; i < 3; ++i) acc[i] = acc[i] - pf * sf[i];
        } else {
          const double pf = pb[f - nfi];
          for (int i = 0; i < 3; ++i) acc[i] = acc[i] + pf * sf[i];
        }
      }
      const double v = m.volume[c];
      for (int i = 0; i < 3; ++i) g[3 * c + i] = v > SMALL ? acc[i] * (1.0 / v) : acc[i];
    }
  }
  // src/numerics/mod_gradient.f90:172-304: the same per component, grad_U(i, j) = dU_j/dx_i.
  void gg_gradient_vector(const double* Uc, const double* Ub, double* g, const double* gprev) {
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t c = 0; c < nc; ++c) {
      double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int64_t k = m.cell_face_off[c]; k < m.cell_face_off[c + 1]; ++k) {
        const int f = m.cell_faces[k];
        const double* sf = &m.sf[3 * (size_t)f];
        double uf[3];
        bool own = true;
        if (f < nfi) {
          const int o = m.owner[f], n = m.neighbour[f];
          own = o == c;
          const double w = m.gc[f];
          if (gprev) {
            const double* e = &m.eps[3 * (size_t)f];
            for (int j = 0; j < 3; ++j) {
              double gm[3];
              for (int i = 0; i < 3; ++i)
                gm[i] = w * gprev[9 * (size_t)o + i + 3 * j] + (1.0 - w) * gprev[9 * (size_t)n + i + 3 * j];
              uf[j] = w * Uc[3 * (size_t)o + j] + (1.0 - w) * Uc[3 * (size_t)n + j] + (gm[0] * e[0] + gm[1] * e[1] + gm[2] * e[2]);
            }
            const double wb = refine_blend_weight(m.skew[f]);
            if (wb < 1.0)
              for (int j = 0; j < 3; ++j) {
                const double plain = w * Uc[3 * (size_t)o + j] + (1.0 - w) * Uc[3 * (size_t)n + j];
                uf[j] = plain + wb * (uf[j] - plain);
              }
          } else {
            for (int j = 0; j < 3; ++j) uf[j] = w * Uc[3 * (size_t)o + j] + (1.0 - w) * Uc[3 * (size_t)n + j];
          }
        } else {
          for (int j = 0; j < 3; ++j) uf[j] = Ub[3 * (size_t)(f - nfi) + j];
        }
        for (int j = 0; j < 3; ++j)
          for (int i = 0; i < 3; ++i) {
            if (own) acc[i + 3 * j] = acc[i + 3 * j] + uf[j] * sf[i];
            else acc[i + 3 * j] = acc[i + 3 * j] - uf[j] * sf[i];
          }
      }
      const double v = m.volume[c];
      for (int j = 0; j < 9; ++j) g[9 * c + j] = v > SMALL ? acc[j] * (1.0 / v) : acc[j];
    }
  }
  bool green_gauss() const { return P.gradient_scheme == DPM_GRAD_GREEN_GAUSS; }
  int gg_sweeps() const { return P.gg_iterations > 0 ? P.gg_iterations : 2; }
  // src/solver/mod_fv_solver.f90:2341-2369 gradient_of_scalar
  void gradient_of_scalar(const double* phi, const double* pb, double* g) {
    if (!green_gauss()) {
      ls_gradient_scalar(phi, pb, g);
      return;
    }
    gg_gradient_scalar(phi, pb, g, nullptr);
    std::vector<double> prev;
    for (int it = 2; it <= gg_sweeps(); ++it) {
      prev.assign(g, g + 3 * nc);
      gg_gradient_scalar(phi, pb, g, prev.data());
    }
  }
  // src/solver/mod_fv_solver.f90:1003-1077
  void compute_all_gradients() {
    if (!green_gauss()) {
      ls_gradient_vector(U.data(), U_bnd.data(), grad_U.data());
      if (P.boussinesq) ls_gradient_scalar(T.data(), T_bnd.data(), grad_T.data());
      for (int sc = 0; sc < ns; ++sc)
        ls_gradient_scalar(&Cs[(size_t)sc * nc], &C_bnd[(size_t)sc * nb], &grad_C[(size_t)sc * 3 * nc]);
      return;
    }
    gg_gradient_vector(U.data(), U_bnd.data(), grad_U.data(), nullptr);
    if (P.boussinesq) gg_gradient_scalar(T.data(), T_bnd.data(), grad_T.data(), nullptr);
    for (int sc = 0; sc < ns; ++sc)
      gg_gradient_scalar(&Cs[(size_t)sc * nc], &C_bnd[(size_t)sc * nb], &grad_C[(size_t)sc * 3 * nc], nullptr);
    std::vector<double> prev;
    for (int it = 2; it <= gg_sweeps(); ++it) {
      prev = grad_U;
      gg_gradient_vector(U.data(), U_bnd.data(), grad_U.data(), prev.data());
      if (P.boussinesq) {
        prev = grad_T;
        gg_gradient_scalar(T.data(), T_bnd.data(), grad_T.data(), prev.data());
      }
      for (int sc = 0; sc < ns; ++sc) {
        double* gcs = &grad_C[(size_t)sc * 3 * nc];
        prev.assign(gcs, gcs + 3 * nc);
        gg_gradient_scalar(&Cs[(size_t)sc * nc], &C_bnd[(size_t)sc * nb], gcs, prev.data());
      }
    }
  }
  void compute_pressure_gradient() {
    if (skip_grad_p) return;
    gradient_of_scalar(p.data(), p_bnd.data(), gp.data());
  }

  // ---------------------------------------------------------------- SGS
  void sgs_viscosity(double dt_stab) {
    if (P.sgs_model == DPM_SGS_NONE) { std::fill(nu_sgs.begin(), nu_sgs.end(), 0.0); return; }
    if (P.sgs_model == DPM_SGS_VREMAN) {  // src/sgs/mod_vreman.f90:50-153
#pragma omp parallel for schedule(static) num_threads(nthreads)
      for (int64_t c = 0; c < nc; ++c) {
        const double* a = &grad_U[9 * c];  // a[m + 3i] = alpha(m,i)
        const double* G = &Gf[9 * c];
        double beta[9];
        for (int j = 0; j < 3; ++j)
          for (int i = 0; i <= j; ++i) {
            double s = 0.0;
            for (int n = 0; n < 3; ++n)
              for (int mm = 0; mm < 3; ++mm) s += G[mm + 3 * n] * a[mm + 3 * i] * a[n + 3 * j];
            beta[i + 3 * j] = s;
          }
        double asq = a[0] * a[0] + a[3] * a[3] + a[6] * a[6] + a[1] * a[1] + a[4] * a[4] + a[7] * a[7] +
                     a[2] * a[2] + a[5] * a[5] + a[8] * a[8];
        double b11 = beta[0], b22 = beta[4], b33 = beta[8], b12 = beta[3], b13 = beta[6], b23 = beta[7];
        double B = b11 * b22 - b12 * b12 + b11 * b33 - b13 * b13 + b22 * b33 - b23 * b23;
        double nu_c = (asq > SMALL && B > 0.0) ? C_VREMAN * std::sqrt(B / asq) : 0.0;
        double cap = NU_SGS_STAB_FRAC * std::pow(m.volume[c], 2.0 / 3.0) / std::max(dt_stab, SMALL);
        nu_sgs[c] = std::min(nu_c, cap);
      }
      return;
    }
    if (P.sgs_model == DPM_SGS_SMAGORINSKY) {  // src/sgs/mod_vreman.f90:295-364
#pragma omp parallel for schedule(static) num_threads(nthreads)
      for (int64_t c = 0; c < nc; ++c) {
        const double* g = &grad_U[9 * c];
        double SS = 0.0;
        for (int j = 0; j < 3; ++j)
          for (int i = 0; i < 3; ++i) {
            double s = 0.5 * (g[i + 3 * j] + g[j + 3 * i]);
            SS += s * s;
          }
        double Sn = std::sqrt(2.0 * SS);
        double delta = std::max(std::pow(std::max(det3(&Gf[9 * c]), 0.0), 1.0 / 6.0), SMALL);
        double nu_c = (0.1 * delta) * (0.1 * delta) * Sn;
        double cap = NU_SGS_STAB_FRAC * delta * delta / std::max(dt_stab, SMALL);
        nu_sgs[c] = std::min(nu_c, cap);
      }
      return;
    }
    if (P.sgs_model == DPM_SGS_AMD) {  // src/sgs/mod_amd.f90:69-207
      for (int64_t c = 0; c < nc; ++c) {
        double nu_c = amd_point(&grad_U[9 * c], &Gf[9 * c], P.c_amd);
        double cap = NU_SGS_STAB_FRAC * std::pow(m.volume[c], 2.0 / 3.0) / std::max(dt_stab, SMALL);
        nu_sgs[c] = std::min(nu_c, cap);
      }
      if (P.amd_wall_gradient && nb > 0) {
        for (int64_t fb = 0; fb < nb; ++fb) {
          int64_t fg = nfi + fb;
          if (bc_of_face(fg) != BC_WALL_MODEL) continue;
          int o = m.owner[fg];
          double nrm[3], d[3];
          for (int k = 0; k < 3; ++k) { nrm[k] = -m.normal[3 * fg + k]; d[k] = m.centre[3 * fg + k] - m.centroid[3 * o + k]; }
          double yw = std::fabs(dot3(d, nrm));
          double un = dot3(&U[3 * o], nrm);
          double ut[3];
          for (int k = 0; k < 3; ++k) ut[k] = U[3 * o + k] - un * nrm[k];
          double utm = std::sqrt(ut[0] * ut[0] + ut[1] * ut[1] + ut[2] * ut[2]);
          if (utm <= 1.0e-14 || yw <= SMALL) continue;
          double utau, taum;
          bool cap;
          wall_stress_newton(utm, yw, P.nu, utau, taum, cap);
          double gw = utau / (KAPPA * yw);
          double a[9];
          for (int k = 0; k < 9; ++k) a[k] = grad_U[9 * o + k];
          double dold[3], dt_[3];
          for (int j = 0; j < 3; ++j) dold[j] = nrm[0] * a[0 + 3 * j] + nrm[1] * a[1 + 3 * j] + nrm[2] * a[2 + 3 * j];
          double dn = dot3(dold, nrm);
          for (int j = 0; j < 3; ++j) dt_[j] = gw * ut[j] / utm - (dold[j] - dn * nrm[j]);
          for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) a[i + 3 * j] += nrm[i] * dt_[j];
          double nu_c = amd_point(a, &Gf[9 * o], P.c_amd);
          double cp = NU_SGS_STAB_FRAC * std::pow(m.volume[o], 2.0 / 3.0) / std::max(dt_stab, SMALL);
          nu_sgs[o] = std::min(nu_c, cp);
        }
      }
      return;
    }
  }

  // ---------------------------------------------------------------- wall model
  // src/sgs/mod_wall_model.f90:176-313
  void wall_model(double dt_filter) {
    if (y_w.empty()) {
      y_w.assign(nb, 0.0);
      sample_cell.assign(nb, -1);
      u_par_filt.assign(3 * nb, 0.0);
      for (int64_t fb = 0; fb < nb; ++fb) {
        int64_t fg = nfi + fb;
        if (bc_of_face(fg) != BC_WALL_MODEL) continue;
        int o = m.owner[fg];
        double d[3];
        for (int k = 0; k < 3; ++k) d[k] = m.centroid[3 * o + k] - m.centre[3 * fg + k];
        double nin[3] = {-m.normal[3 * fg], -m.normal[3 * fg + 1], -m.normal[3 * fg + 2]};
        sample_cell[fb] = o;
        y_w[fb] = std::fabs(dot3(d, nin)) + SMALL;
      }
    }
    double t_use = P.wall_model_filter_time, tf = P.wall_model_filter_tf_fac;
    bool adaptive = tf > SMALL;
    bool do_filter = (t_use > SMALL || adaptive);
    bool seed = !filt_ready;
    double w_filt = (do_filter && !adaptive) ? dt_filter / (t_use + dt_filter) : 0.0;
    for (int64_t fb = 0; fb < nb; ++fb) {
      int64_t fg = nfi + fb;
      if (bc_of_face(fg) != BC_WALL_MODEL) continue;
      const double* n = &m.normal[3 * fg];
      int cs = sample_cell[fb] >= 0 ? sample_cell[fb] : m.owner[fg];
      double yw = y_w[fb];
      double un = U[3 * cs] * n[0] + U[3 * cs + 1] * n[1] + U[3 * cs + 2] * n[2];
      double u[3];
      for (int k = 0; k < 3; ++k) u[k] = U[3 * cs + k] - un * n[k];
      if (do_filter) {
        double* uf = &u_par_filt[3 * fb];
        if (seed) {
          for (int k = 0; k < 3; ++k) uf[k] = u[k];
        } else {
          double e = w_filt;
          if (adaptive) {
            e = 0.0;
            if (dt_filter > 0.0) {
              double upm = std::sqrt(uf[0] * uf[0] + uf[1] * uf[1] + uf[2] * uf[2]), utp, tp;
              bool cp;
              wall_stress_newton(upm, yw, P.nu, utp, tp, cp);
              e = 1.0;
              if (utp > SMALL) e = std::min(1.0, dt_filter * KAPPA * utp / (tf * yw));
            }
          }
          for (int k = 0; k < 3; ++k) uf[k] = uf[k] + e * (u[k] - uf[k]);
        }
        for (int k = 0; k < 3; ++k) u[k] = uf[k];
      }
      double um = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
      double utau, tm;
      bool cp;
      wall_stress_newton(um, yw, P.nu, utau, tm, cp);
      double sc = -tm / (um + SMALL);
      for (int k = 0; k < 3; ++k) tau_w[3 * fb + k] = sc * u[k];
    }
    if (t_use > SMALL || adaptive) filt_ready = true;
  }

  // ---------------------------------------------------------------- MOST surface layer
  // src/abl/mod_abl_profiles.f90:51-86 (Businger-Dyer stable branch, Paulson unstable branch)
  static double most_psi_m(double z) {
    if (std::fabs(z) < 1.0e-6) return 0.0;
    if (z > 0.0) return -5.0 * z;
    double x = std::pow(1.0 - 16.0 * z, 0.25);
    return 2.0 * std::log((1.0 + x) / 2.0) + std::log((1.0 + x * x) / 2.0) - 2.0 * std::atan(x) + M_PI / 2.0;
  }
  static double most_psi_h(double z) {
    if (std::fabs(z) < 1.0e-6) return 0.0;
    if (z > 0.0) return -5.0 * z;
    double y = std::pow(1.0 - 16.0 * z, 0.5);
    return 2.0 * std::log((1.0 + y) / 2.0);
  }
  static constexpr double MOST_KAPPA = 0.41, MOST_G = 9.81, MOST_L_CLIP = 5000.0;  // mod_parameters, mod_abl_wall
  static double fsign(double a, double b) { return b >= 0.0 ? std::fabs(a) : -std::fabs(a); }
  // L = u*^2 T_ref / (kappa g T*), kept away from 0 and clipped (mod_abl_wall.f90:L_from)
  static double most_L_from(double us, double ts, double tref) {
    if (std::fabs(ts) > SMALL) {
      double L = us * us * tref / (MOST_KAPPA * MOST_G * ts);
      L = fsign(std::max(std::fabs(L), 0.001), L);
      if (std::fabs(L) > MOST_L_CLIP) L = fsign(MOST_L_CLIP, L);
      return L;
    }
    return MOST_L_CLIP;
  }
  static void most_residuals(double us, double ts, double L, double up, double To, double Ts, double yw, double z0m,
                             double z0h, double& Fu, double& FT) {
    double pmz = most_psi_m(yw / L), pmz0 = most_psi_m(z0m / L);
    double phz = most_psi_h(yw / L), phz0 = most_psi_h(z0h / L);
    double dm = std::log(yw / z0m) - pmz + pmz0;
    double dh = std::log(yw / z0h) - phz + phz0;
    if (std::fabs(dm) < SMALL) dm = fsign(SMALL, dm);
    if (std::fabs(dh) < SMALL) dh = fsign(SMALL, dh);
    Fu = us - MOST_KAPPA * up / dm;
    FT = ts - MOST_KAPPA * (To - Ts) / dh;
  }
  // src/abl/mod_abl_wall.f90:156-231 (most_iterate: relaxed Newton on (u*, T*) with a
  // finite-difference Jacobian, L re-derived after every update)
  static void most_iterate(double up, double To, double Ts, double yw, double z0m, double z0h, double L_init,
                           double& us_out, double& ts_out, double& L_out) {
    const double tref = To;
    double us = std::max(SMALL, MOST_KAPPA * up / std::max(SMALL, std::log(yw / z0m)));
    double ts = 0.1 * (To - Ts);
    double L = std::fabs(L_init) < SMALL ? MOST_L_CLIP : L_init;
    for (int it = 1; it <= 20; ++it) {
      L = fsign(std::max(std::fabs(L), 0.001), L);
      if (std::fabs(L) > MOST_L_CLIP) L = fsign(MOST_L_CLIP, L);
      double Fu, FT, Fu_p, FT_p;
      most_residuals(us, ts, L, up, To, Ts, yw, z0m, z0h, Fu, FT);
      if (std::fabs(Fu) < 1.0e-8 && std::fabs(FT) < 1.0e-8) break;
      double du_eps = std::max(1.0e-6, 1.0e-6 * std::fabs(us));
      double dT_eps = std::max(1.0e-6, 1.0e-6 * std::fabs(ts));
      most_residuals(us + du_eps, ts, most_L_from(us + du_eps, ts, tref), up, To, Ts, yw, z0m, z0h, Fu_p, FT_p);
      double dFu_du = (Fu_p - Fu) / du_eps, dFT_du = (FT_p - FT) / du_eps;
      most_residuals(us, ts + dT_eps, most_L_from(us, ts + dT_eps, tref), up, To, Ts, yw, z0m, z0h, Fu_p, FT_p);
      double dFu_dT = (Fu_p - Fu) / dT_eps, dFT_dT = (FT_p - FT) / dT_eps;
      double den = dFu_du * dFT_dT - dFu_dT * dFT_du;
      if (std::fabs(den) < SMALL) break;
      double dus = -(dFT_dT * Fu - dFu_dT * FT) / den;
      double dts = -(dFu_du * FT - dFT_du * Fu) / den;
      us = us + 0.5 * dus;
      ts = ts + 0.5 * dts;
      us = std::max(SMALL, std::min(us, 0.5 * up));
      L = most_L_from(us, ts, tref);
    }
    us_out = us; ts_out = ts; L_out = L;
  }
  // src/abl/mod_abl_wall.f90:62-153 (abl_wall_model; global roughness, owner-cell sampling at the
  // wall-normal distance of its centroid)
  void most_wall_model(bool update_L) {
    const double L_cfg = L_obukhov;
    double L_sum = 0.0;
    int64_t nwf = 0;
    for (int64_t fb = 0; fb < nb; ++fb) {
      int64_t fg = nfi + fb;
      if (bc_of_face(fg) != BC_WALL_MODEL) continue;
      int o = m.owner[fg];
      const double* n = &m.normal[3 * fg];
      double yw = std::fabs((m.centre[3 * fg] - m.centroid[3 * o]) * n[0] + (m.centre[3 * fg + 1] - m.centroid[3 * o + 1]) * n[1] +
                            (m.centre[3 * fg + 2] - m.centroid[3 * o + 2]) * n[2]) + SMALL;
      const double* u = &U[3 * o];
      double un = u[0] * n[0] + u[1] * n[1] + u[2] * n[2];
      double t0 = u[0] - un * n[0], t1 = u[1] - un * n[1], t2 = u[2] - un * n[2];
      double upm = std::sqrt(t0 * t0 + t1 * t1 + t2 * t2);
      if (upm > SMALL) { t0 /= upm; t1 /= upm; t2 /= upm; }
      else { t0 = t1 = t2 = 0.0; }
      double Lg = L_bnd[fb];
      if (std::fabs(Lg) < SMALL) Lg = L_cfg;
      double us, ts, Ln;
      // src/abl/mod_abl_wall.f90:45-50, :248-257: the patch's roughness when set, else the global
      const dpm_patch_cfg_t& q = pc[m.patch[fg]];
      const double z0m = std::max(q.abl_z0_m > 0.0 ? q.abl_z0_m : P.abl_z0_m, SMALL);
      const double z0h = std::max(q.abl_z0_h > 0.0 ? q.abl_z0_h : P.abl_z0_h, SMALL);
      most_iterate(upm, T[o], P.abl_T_surface, yw, z0m, z0h, Lg, us, ts, Ln);
      L_bnd[fb] = Ln;
      L_sum += Ln;
      nwf++;
      tau_w[3 * fb] = -us * us * t0;
      tau_w[3 * fb + 1] = -us * us * t1;
      tau_w[3 * fb + 2] = -us * us * t2;
      q_w[fb] = -us * ts;
    }
    if (P.abl_compute_L && update_L && nwf > 0) L_obukhov = L_sum / (double)nwf;
  }

  // ---------------------------------------------------------------- advection
  int periodic_nb(int64_t fb, int o) const {  // soa_resolve_periodic_nb_dev, single-rank
    int n = m.periodic_partner_cell(fb);
    if (n == o) n = -1;
    return n;
  }

  // src/numerics/mod_advection.f90:1013-1197
  void advection_kep(double* rhs) {
    std::vector<double> div(nc, 0.0);
    std::fill(rhs, rhs + 3 * nc, 0.0);
    for (int64_t f = 0; f < nf; ++f) {
      int o = m.owner[f], n = m.neighbour[f];
      const double* sf = &m.sf[3 * f];
      int64_t fb = 0;
      int bc = -1, npr = -1;
      double Uf[3], Fn;
      if (n >= 0) {
        for (int k = 0; k < 3; ++k) Uf[k] = m.gc[f] * U[3 * o + k] + (1.0 - m.gc[f]) * U[3 * n + k];
        Fn = U_face[f];
      } else {
        fb = f - nfi;
        bc = bc_of_face(f);
        if (bc == BC_PERIODIC) npr = periodic_nb(fb, o);
        if (bc == BC_PERIODIC && npr >= 0) {
          double w = m.periodic_gc[fb];
          for (int k = 0; k < 3; ++k) Uf[k] = w * U[3 * o + k] + (1.0 - w) * U[3 * npr + k];
        } else {
          for (int k = 0; k < 3; ++k) Uf[k] = U_bnd[3 * fb + k];
        }
        if (bc == BC_PERIODIC || bc == BC_OUTLET) Fn = U_face[f];
        else if (is_wall(bc)) Fn = 0.0;
        else Fn = dot3(Uf, sf);
      }
      div[o] += Fn;
      if (n >= 0) div[n] -= Fn;
      for (int k = 0; k < 3; ++k) {
        double phi;
        if (n >= 0) phi = 0.5 * (U[3 * o + k] + U[3 * n + k]);
        else if (npr >= 0) phi = 0.5 * (U[3 * o + k] + U[3 * npr + k]);
        else phi = Uf[k];
        rhs[3 * o + k] -= Fn * phi * inv_vol[o];
        if (n >= 0) rhs[3 * n + k] += Fn * phi * inv_vol[n];
      }
    }
    for (int64_t c = 0; c < nc; ++c)
      for (int k = 0; k < 3; ++k) rhs[3 * c + k] += 0.5 * U[3 * c + k] * div[c] * inv_vol[c];
  }

  // src/numerics/mod_advection.f90:1200-1392
  void advection_cds(double* rhs) {
    std::fill(rhs, rhs + 3 * nc, 0.0);
    for (int64_t f = 0; f < nf; ++f) {
      int o = m.owner[f], n = m.neighbour[f];
      int64_t fb = 0;
      int bc = -1, npr = -1;
      double Fn;
      if (n >= 0) {
        Fn = U_face[f];
      } else {
        fb = f - nfi;
        bc = bc_of_face(f);
        if (bc == BC_PERIODIC || bc == BC_OUTLET) Fn = U_face[f];
        else if (is_wall(bc)) Fn = 0.0;
        else Fn = dot3(&U_bnd[3 * fb], &m.sf[3 * f]);
      }
      bool has_rec = n >= 0;
      if (!has_rec && bc == BC_PERIODIC) {
        npr = periodic_nb(fb, o);
        has_rec = npr >= 0;
      }
      int ns = has_rec ? (n >= 0 ? n : npr) : -1;
      for (int k = 0; k < 3; ++k) {
        double phi;
        if (has_rec) {
          double gcv = f >= nfi ? m.periodic_gc[fb] : m.gc[f];
          double plain = gcv * U[3 * o + k] + (1.0 - gcv) * U[3 * ns + k];
          if (f < nfi) {
            double gm[3], ph;
            for (int i = 0; i < 3; ++i) gm[i] = gcv * grad_U[9 * o + 3 * k + i] + (1.0 - gcv) * grad_U[9 * (int64_t)ns + 3 * k + i];
            ph = plain + dot3(gm, &m.eps[3 * f]);
            double wb = refine_blend_weight(m.skew[f]);
            if (wb < 1.0) ph = plain + wb * (ph - plain);
            phi = ph;
          } else {
            phi = plain;
          }
        } else {
          phi = U_bnd[3 * fb + k];
        }
        if (!finite(phi)) phi = 0.0;
        rhs[3 * o + k] -= Fn * phi * inv_vol[o];
        if (n >= 0) rhs[3 * n + k] += Fn * phi * inv_vol[n];
      }
    }
  }

  // Reconstruction context of face f for flux Fn (mod_advection.f90:2386-2498).
  struct Ctx { int up, down; double x_up[3], x_down[3], x_face[3], up_shift[3], dir[3], s_face, s_down; };
  bool recon_context(int64_t f, double Fn, Ctx& c) const {
    c.up = c.down = -1;
    for (int k = 0; k < 3; ++k) { c.x_up[k] = c.x_down[k] = c.up_shift[k] = c.dir[k] = 0.0; c.x_face[k] = m.centre[3 * f + k]; }
    c.s_face = c.s_down = 0.0;
    int o = m.owner[f], n = m.neighbour[f];
    if (n >= 0) {
      if (Fn >= 0.0) { c.up = o; c.down = n; } else { c.up = n; c.down = o; }
      for (int k = 0; k < 3; ++k) { c.x_up[k] = m.centroid[3 * c.up + k]; c.x_down[k] = m.centroid[3 * c.down + k]; }
    } else {
      if (bc_of_face(f) != BC_PERIODIC) return false;
      int64_t fb = f - nfi;
      int pcell = periodic_nb(fb, o);
      int pb = m.periodic_pair[fb];
      int64_t pf = pb >= 0 ? nfi + pb : -1;
      if (pcell < 0 && pf >= 0) pcell = m.owner[pf];
      if (pcell < 0) return false;
      double d_per;
      if (pf >= 0) d_per = m.d_cf[f] + m.d_cf[pf];
      else if (m.periodic_pair_dcf[fb] > SMALL) d_per = m.d_cf[f] + m.periodic_pair_dcf[fb];
      else d_per = 2.0 * m.d_cf[f];
      double shift[3];
      for (int k = 0; k < 3; ++k) shift[k] = (m.centroid[3 * o + k] + d_per * m.normal[3 * f + k]) - m.centroid[3 * pcell + k];
      if (Fn >= 0.0) {
        c.up = o; c.down = pcell;
        for (int k = 0; k < 3; ++k) { c.x_up[k] = m.centroid[3 * o + k]; c.x_down[k] = m.centroid[3 * pcell + k] + shift[k]; }
      } else {
        c.up = pcell; c.down = o;
        for (int k = 0; k < 3; ++k) {
          c.up_shift[k] = shift[k];
          c.x_up[k] = m.centroid[3 * pcell + k] + c.up_shift[k];
          c.x_down[k] = m.centroid[3 * o + k];
        }
      }
    }
    double dv[3], dn;
    for (int k = 0; k < 3; ++k) dv[k] = c.x_face[k] - c.x_up[k];
    dn = std::sqrt(dot3(dv, dv));
    if (dn <= SMALL) {
      for (int k = 0; k < 3; ++k) dv[k] = c.x_down[k] - c.x_up[k];
      dn = std::sqrt(dot3(dv, dv));
    }
    if (dn <= SMALL) return false;
    for (int k = 0; k < 3; ++k) c.dir[k] = dv[k] / dn;
    double a[3], b[3];
    for (int k = 0; k < 3; ++k) { a[k] = c.x_face[k] - c.x_up[k]; b[k] = c.x_down[k] - c.x_up[k]; }
    c.s_face = dot3(a, c.dir);
    c.s_down = dot3(b, c.dir);
    if (c.s_face <= SMALL || c.s_down <= c.s_face) {
      for (int k = 0; k < 3; ++k) dv[k] = c.x_down[k] - c.x_up[k];
      dn = std::sqrt(dot3(dv, dv));
      if (dn <= SMALL) return false;
      for (int k = 0; k < 3; ++k) c.dir[k] = dv[k] / dn;
      c.s_face = dot3(a, c.dir);
      c.s_down = dot3(b, c.dir);
    }
    if (c.s_down <= SMALL) return false;
    c.s_face = std::min(std::max(c.s_face, 0.0), c.s_down);
    return true;
  }

  // mod_advection.f90:2501-2549
  int far_upwind(const Ctx& c) const {
    int far = -1;
    if (c.up < 0 || c.up >= nc || c.down >= nc) return far;
    double best_align = -1.0, best_perp2 = 1e308;
    for (int64_t fi = m.cell_face_off[c.up]; fi < m.cell_face_off[c.up + 1]; ++fi) {
      int fj = m.cell_faces[fi];
      int n = m.owner[fj];
      if (n == c.up) n = m.neighbour[fj];
      if (n < 0) {
        if (fj >= nfi && bc_of_face(fj) == BC_PERIODIC) n = periodic_nb(fj - nfi, c.up);
      }
      if (n == c.down || n < 0) continue;
      double d[3];
      for (int k = 0; k < 3; ++k) d[k] = m.centroid[3 * n + k] + c.up_shift[k] - c.x_up[k];
      double s = dot3(d, c.dir);
      if (s >= -1.0e-12) continue;
      double dist2 = std::max(dot3(d, d), SMALL);
      double align = -s / std::sqrt(dist2);
      double perp2 = std::max(0.0, dist2 - s * s);
      if (align > best_align + 1.0e-12 ||
          (std::fabs(align - best_align) <= 1.0e-12 && perp2 < best_perp2 - 1.0e-12) ||
          (std::fabs(align - best_align) <= 1.0e-12 && std::fabs(perp2 - best_perp2) <= 1.0e-12 && n < far)) {
        best_align = align; best_perp2 = perp2; far = n;
      }
    }
    return far;
  }

  static double clampv(double x, double lo, double hi) {
    double l = std::min(lo, hi), h = std::max(lo, hi);
    return std::min(std::max(x, l), h);
  }

  // mod_advection.f90:2632-2722: QUICK fit on the upwind cell's neighbours, K components at once
  // (phi_at(cell, k), grad_at(cell, k, i) give the field and its cell gradient).
  template <int K, class PhiAt, class GradAt>
  void quick_fit(const Ctx& c, PhiAt phi_at, GradAt grad_at, double* phi_f) const {
    bool have_grad = c.up < nc && c.down < nc;
    double phU[K], phD[K], gup[K][3];
    for (int k = 0; k < K; ++k) {
      phU[k] = phi_at(c.up, k);
      phD[k] = phi_at(c.down, k);
      for (int i = 0; i < 3; ++i) gup[k][i] = have_grad ? grad_at(c.up, k, i) : 0.0;
    }
    auto axial = [&](double far, double up, const double* g, const double* dv, double s) {
      double t[3];
      for (int i = 0; i < 3; ++i) t[i] = dv[i] - s * c.dir[i];
      return far - up - dot3(g, t);
    };
    double dv[3];
    for (int i = 0; i < 3; ++i) dv[i] = c.x_down[i] - c.x_up[i];
    double dist2 = std::max(dot3(dv, dv), SMALL);
    double w = 1.0 / dist2;
    double a11 = w * c.s_down * c.s_down, a12 = a11 * c.s_down, a22 = a12 * c.s_down, lin_den = a11;
    int nfit = 1;
    double b1[K], b2[K], ln[K];
    for (int k = 0; k < K; ++k) {
      double dp = axial(phD[k], phU[k], gup[k], dv, c.s_down);
      b1[k] = w * c.s_down * dp;
      b2[k] = w * c.s_down * c.s_down * dp;
      ln[k] = b1[k];
    }
    if (c.up < nc && c.down < nc) {
      for (int64_t fi = m.cell_face_off[c.up]; fi < m.cell_face_off[c.up + 1]; ++fi) {
        int fj = m.cell_faces[fi];
        int n = m.owner[fj];
        if (n == c.up) n = m.neighbour[fj];
        if (n < 0 || n == c.down) continue;
        double d[3];
        for (int i = 0; i < 3; ++i) d[i] = m.centroid[3 * n + i] + c.up_shift[i] - c.x_up[i];
        double s = dot3(d, c.dir);
        if (s >= -1.0e-12) continue;
        double d2 = std::max(dot3(d, d), SMALL);
        if (s * s < 0.25 * d2) continue;
        double al = std::min(1.0, -s / std::sqrt(d2));
        double wt = (0.25 + al * al) / d2;
        a11 += wt * s * s; a12 += wt * s * s * s; a22 += wt * s * s * s * s; lin_den += wt * s * s;
        for (int k = 0; k < K; ++k) {
          double dp = axial(phi_at(n, k), phU[k], gup[k], d, s);
          b1[k] += wt * s * dp; b2[k] += wt * s * s * dp; ln[k] += wt * s * dp;
        }
        nfit++;
      }
    }
    double det = a11 * a22 - a12 * a12;
    for (int k = 0; k < K; ++k) {
      double a1, a2;
      if (nfit >= 2 && std::fabs(det) > SMALL) {
        a1 = (b1[k] * a22 - b2[k] * a12) / det;
        a2 = (-b1[k] * a12 + b2[k] * a11) / det;
      } else if (lin_den > SMALL) {
        a1 = ln[k] / lin_den; a2 = 0.0;
      } else {
        a1 = (phD[k] - phU[k]) / std::max(c.s_down, SMALL); a2 = 0.0;
      }
      double v = phU[k] + a1 * c.s_face + a2 * c.s_face * c.s_face;
      phi_f[k] = clampv(v, std::min(phU[k], phD[k]), std::max(phU[k], phD[k]));
    }
  }
  void quick3(const Ctx& c, double* phi_f) const {
    quick_fit<3>(c, [&](int cell, int k) { return U[3 * (int64_t)cell + k]; },
                 [&](int cell, int k, int i) { return grad_U[9 * (int64_t)cell + 3 * k + i]; }, phi_f);
  }

  // mod_advection.f90:2725-2791
  double tvd(int scheme, const double* phi, int stride, const Ctx& c, int far) const {
    double pU = phi[stride * (int64_t)c.up], pD = phi[stride * (int64_t)c.down];
    double sdn = (pD - pU) / std::max(c.s_down, SMALL), psi = 0.0;
    if (far >= 0 && std::fabs(sdn) > SMALL) {
      double xf[3];
      for (int k = 0; k < 3; ++k) xf[k] = m.centroid[3 * far + k] + c.up_shift[k] - c.x_up[k];
      double s_up = -dot3(xf, c.dir);
      if (s_up <= SMALL) {
        psi = 0.0;
      } else {
        double pUU = phi[stride * (int64_t)far];
        double r = ((pU - pUU) / s_up) / sdn;
        if (scheme == DPM_SCHEME_VANLEER_TVD) {
          psi = (r + std::fabs(r)) / (1.0 + std::fabs(r));
          psi = std::max(0.0, std::min(psi, 2.0));
        } else {
          psi = std::max(0.0, std::min(std::min(2.0 * r, (1.0 + 2.0 * r) / 3.0), 2.0));
        }
      }
    }
    return clampv(pU + psi * sdn * c.s_face, std::min(pU, pD), std::max(pU, pD));
  }

  // src/numerics/mod_advection.f90:1396-1635
  void advection_recon(int scheme, double* rhs) {
    std::fill(rhs, rhs + 3 * nc, 0.0);
    for (int64_t f = 0; f < nf; ++f) {
      int o = m.owner[f], n = m.neighbour[f];
      int64_t fb = f >= nfi ? f - nfi : 0;
      double Fn;
      if (n >= 0) Fn = U_face[f];
      else {
        int bc = bc_of_face(f);
        Fn = is_wall(bc) ? 0.0 : U_face[f];
      }
      Ctx c;
      bool ok = recon_context(f, Fn, c);
      int far = -1;
      if (ok && scheme != DPM_SCHEME_QUICK) far = far_upwind(c);
      if (!finite(Fn)) Fn = 0.0;
      double pq[3] = {0, 0, 0};
      if (ok && scheme == DPM_SCHEME_QUICK) quick3(c, pq);
      for (int k = 0; k < 3; ++k) {
        double phi;
        if (ok) {
          if (scheme == DPM_SCHEME_QUICK) phi = pq[k];
          else phi = tvd(scheme, &U[k], 3, c, far);
          if (!finite(phi)) phi = (Fn >= 0.0 || n < 0) ? U[3 * o + k] : U[3 * n + k];
        } else {
          phi = U_bnd[3 * fb + k];
        }
        if (!finite(phi)) phi = 0.0;
        rhs[3 * o + k] -= Fn * phi * inv_vol[o];
        if (n >= 0) rhs[3 * n + k] += Fn * phi * inv_vol[n];
      }
    }
  }

  void advection(double* rhs) {
    if (P.scheme == DPM_SCHEME_KEP) advection_kep(rhs);
    else if (P.scheme == DPM_SCHEME_CDS) advection_cds(rhs);
    else advection_recon(P.scheme, rhs);
  }

  // ---------------------------------------------------------------- viscous
  // src/numerics/mod_viscous.f90:37-282
  static double ortho_weight(double sdd, double area) {
    return area * std::max(0.0, std::min(1.0, sdd / (area + SMALL)));
  }
  void viscous(double* rhs) {
    std::fill(rhs, rhs + 3 * nc, 0.0);
    for (int64_t f = 0; f < nf; ++f) {
      int o = m.owner[f], n = m.neighbour[f];
      const double* sf = &m.sf[3 * f];
      const double* nh = &m.normal[3 * f];
      double st[3] = {0, 0, 0};
      auto face_stress = [&](int nbc, double gcv, double nu_eff, const double* d_on, double dlen) {
        double sdd = dot3(sf, d_on) / dlen;
        double dperp[3];
        for (int k = 0; k < 3; ++k) dperp[k] = sf[k] - (sdd / dlen) * d_on[k];
        double wo = ortho_weight(sdd, m.area[f]);
        double gf[9];
        for (int j = 0; j < 9; ++j) gf[j] = gcv * grad_U[9 * o + j] + (1.0 - gcv) * grad_U[9 * (int64_t)nbc + j];
        for (int k = 0; k < 3; ++k) {
          // gf[i + 3k] = dU_k/dx_i ; gf(k,:) = dU_j/dx_k over j: gf[k + 3j]
          double t1 = (U[3 * (int64_t)nbc + k] - U[3 * o + k]) * wo / dlen;
          double t2 = gf[0 + 3 * k] * dperp[0] + gf[1 + 3 * k] * dperp[1] + gf[2 + 3 * k] * dperp[2];
          double t3 = gf[k + 0] * sf[0] + gf[k + 3] * sf[1] + gf[k + 6] * sf[2];
          st[k] = nu_eff * (t1 + t2 + t3);
        }
      };
      if (n >= 0) {
        double gcv = m.gc[f];
        double nu_eff = P.nu + gcv * nu_sgs[o] + (1.0 - gcv) * nu_sgs[n];
        double d[3];
        for (int k = 0; k < 3; ++k) d[k] = m.centroid[3 * n + k] - m.centroid[3 * o + k];
        double dl = std::sqrt(dot3(d, d)) + SMALL;
        face_stress(n, gcv, nu_eff, d, dl);
      } else {
        int64_t fb = f - nfi;
        int bc = bc_of_face(f);
        if (bc == BC_PERIODIC) {
          int npr = periodic_nb(fb, o);
          int pb = m.periodic_pair[fb];
          int64_t pf = pb >= 0 ? nfi + pb : -1;
          if (npr >= 0) {
            double dper, gcp;
            if (pf >= 0) { dper = m.d_cf[f] + m.d_cf[pf]; gcp = m.d_cf[pf] / (dper + SMALL); }
            else if (m.periodic_pair_dcf[fb] > SMALL) { dper = m.d_cf[f] + m.periodic_pair_dcf[fb]; gcp = m.periodic_pair_dcf[fb] / (dper + SMALL); }
            else { dper = 2.0 * m.d_cf[f]; gcp = 0.5; }
            double nu_eff = P.nu + gcp * nu_sgs[o] + (1.0 - gcp) * nu_sgs[npr];
            double d[3] = {dper * nh[0], dper * nh[1], dper * nh[2]};
            face_stress(npr, gcp, nu_eff, d, dper + SMALL);
          } else {
            double nu_eff = P.nu + nu_sgs[o];
            for (int k = 0; k < 3; ++k) st[k] = nu_eff * ((U_bnd[3 * fb + k] - U[3 * o + k]) / (m.d_cf[f] + SMALL)) * m.area[f];
          }
        } else if (bc == BC_WALL_MODEL) {
          // traction enters through add_wall_stress_to_rhs
        } else {
          double nu_eff = P.nu + nu_sgs[o];
          double d[3];
          for (int k = 0; k < 3; ++k) d[k] = m.centre[3 * f + k] - m.centroid[3 * o + k];
          double dl = std::sqrt(dot3(d, d)) + SMALL;
          double sdd = dot3(sf, d) / dl, dperp[3];
          for (int k = 0; k < 3; ++k) dperp[k] = sf[k] - (sdd / dl) * d[k];
          double wo = ortho_weight(sdd, m.area[f]);
          const double* g = &grad_U[9 * o];
          for (int k = 0; k < 3; ++k) {
            double t1 = (U_bnd[3 * fb + k] - U[3 * o + k]) * wo / dl;
            double t2 = g[0 + 3 * k] * dperp[0] + g[1 + 3 * k] * dperp[1] + g[2 + 3 * k] * dperp[2];
            double t3 = g[k] * sf[0] + g[k + 3] * sf[1] + g[k + 6] * sf[2];
            st[k] = nu_eff * (t1 + t2 + t3);
          }
        }
      }
      for (int k = 0; k < 3; ++k) rhs[3 * o + k] += st[k] * inv_vol[o];
      if (n >= 0)
        for (int k = 0; k < 3; ++k) rhs[3 * n + k] -= st[k] * inv_vol[n];
    }
  }

  // advection_rhs_scalar_cds_soa / _recon_soa (src/numerics/mod_advection.f90:267-675): face flux
  // is the projected U_face on every non-wall face, zero on walls.
  void advection_scalar(int scheme, const double* phi, const double* phib, const double* gphi, double* rhs) {
    std::fill(rhs, rhs + nc, 0.0);
    for (int64_t f = 0; f < nf; ++f) {
      int o = m.owner[f], n = m.neighbour[f];
      int64_t fb = f >= nfi ? f - nfi : 0;
      int bc = n >= 0 ? -1 : bc_of_face(f);
      double Fn = (n < 0 && is_wall(bc)) ? 0.0 : U_face[f];
      double phf;
      if (scheme == DPM_SCHEME_CDS) {
        int npr = -1;
        bool has_rec = n >= 0;
        if (!has_rec && bc == BC_PERIODIC) {
          npr = periodic_nb(fb, o);
          has_rec = npr >= 0;
        }
        if (has_rec) {
          int ns_ = n >= 0 ? n : npr;
          double gcv = f >= nfi ? m.periodic_gc[fb] : m.gc[f];
          double plain = gcv * phi[o] + (1.0 - gcv) * phi[ns_];
          if (f < nfi) {
            double gm[3];
            for (int i = 0; i < 3; ++i) gm[i] = gcv * gphi[3 * o + i] + (1.0 - gcv) * gphi[3 * (int64_t)ns_ + i];
            double ph = plain + dot3(gm, &m.eps[3 * f]);
            double wb = refine_blend_weight(m.skew[f]);
            if (wb < 1.0) ph = plain + wb * (ph - plain);
            phf = ph;
          } else {
            phf = plain;
          }
          if (!finite(phf)) phf = (Fn >= 0.0 || n < 0) ? phi[o] : phi[n];
        } else {
          phf = phib[fb];
        }
      } else {
        Ctx c;
        bool ok = recon_context(f, Fn, c);
        if (ok) {
          if (scheme == DPM_SCHEME_QUICK) {
            quick_fit<1>(c, [&](int cell, int) { return phi[cell]; },
                         [&](int cell, int, int i) { return gphi[3 * (int64_t)cell + i]; }, &phf);
          } else {
            phf = tvd(scheme, phi, 1, c, far_upwind(c));
          }
          if (!finite(phf)) phf = (Fn >= 0.0 || n < 0) ? phi[o] : phi[n];
        } else {
          phf = phib[fb];
        }
      }
      if (!finite(Fn)) Fn = 0.0;
      if (!finite(phf)) phf = 0.0;
      rhs[o] -= Fn * phf * inv_vol[o];
      if (n >= 0) rhs[n] += Fn * phf * inv_vol[n];
    }
  }

  // src/numerics/mod_viscous.f90:286-507 (viscous_rhs_scalar): alpha_eff = alpha + nu_t / Pr_t,
  // over-relaxed normal part with the clamped orthogonality weight, gc-mean gradient on the
  // transverse part; every non-periodic boundary face by the Jasak split against phi_bnd.
  void viscous_scalar(const double* phi, double alpha, double prt, const double* gphi, const double* phib,
                      double* rhs) {
    std::fill(rhs, rhs + nc, 0.0);
    for (int64_t f = 0; f < nf; ++f) {
      int o = m.owner[f], n = m.neighbour[f];
      const double* sf = &m.sf[3 * f];
      double flux = 0.0;
      auto pair_flux = [&](int nbc, double gcv, double aeff, const double* d_on, double dlen) {
        double sdd = dot3(sf, d_on) / dlen;
        double dperp[3], gf[3];
        for (int k = 0; k < 3; ++k) {
          dperp[k] = sf[k] - (sdd / dlen) * d_on[k];
          gf[k] = gcv * gphi[3 * o + k] + (1.0 - gcv) * gphi[3 * (int64_t)nbc + k];
        }
        double dphi = (phi[nbc] - phi[o]) * ortho_weight(sdd, m.area[f]) / dlen + dot3(gf, dperp);
        return aeff * dphi;
      };
      auto bnd_flux = [&](int64_t fb) {
        double aeff = alpha + nu_sgs[o] / prt;
        double d[3];
        for (int k = 0; k < 3; ++k) d[k] = m.centre[3 * f + k] - m.centroid[3 * o + k];
        double dl = std::sqrt(dot3(d, d)) + SMALL;
        double sdd = dot3(sf, d) / dl, dperp[3];
        for (int k = 0; k < 3; ++k) dperp[k] = sf[k] - (sdd / dl) * d[k];
        double dphi = (phib[fb] - phi[o]) * ortho_weight(sdd, m.area[f]) / dl + dot3(&gphi[3 * o], dperp);
        return aeff * dphi;
      };
      if (n >= 0) {
        double gcv = m.gc[f];
        double aeff = alpha + (gcv * nu_sgs[o] + (1.0 - gcv) * nu_sgs[n]) / prt;
        double d[3];
        for (int k = 0; k < 3; ++k) d[k] = m.centroid[3 * n + k] - m.centroid[3 * o + k];
        flux = pair_flux(n, gcv, aeff, d, std::sqrt(dot3(d, d)) + SMALL);
      } else {
        int64_t fb = f - nfi;
        if (bc_of_face(f) == BC_PERIODIC) {
          int npr = periodic_nb(fb, o);
          int pb = m.periodic_pair[fb];
          int64_t pf = pb >= 0 ? nfi + pb : -1;
          if (npr >= 0) {
            double dper, gcp;
            if (pf >= 0) { dper = m.d_cf[f] + m.d_cf[pf]; gcp = m.d_cf[pf] / (dper + SMALL); }
            else if (m.periodic_pair_dcf[fb] > SMALL) { dper = m.d_cf[f] + m.periodic_pair_dcf[fb]; gcp = m.periodic_pair_dcf[fb] / (dper + SMALL); }
            else { dper = 2.0 * m.d_cf[f]; gcp = 0.5; }
            double aeff = alpha + (gcp * nu_sgs[o] + (1.0 - gcp) * nu_sgs[npr]) / prt;
            const double* nh = &m.normal[3 * f];
            double d[3] = {dper * nh[0], dper * nh[1], dper * nh[2]};
            flux = pair_flux(npr, gcp, aeff, d, dper + SMALL);
          } else {
            flux = bnd_flux(fb);
          }
        } else {
          flux = bnd_flux(fb);
        }
      }
      rhs[o] += flux * inv_vol[o];
      if (n >= 0) rhs[n] -= flux * inv_vol[n];
    }
  }

  // src/solver/mod_fv_solver.f90:1617-1762 (momentum part)
  void explicit_rhs() {
    advection(conv_U.data());
    viscous(visc_U.data());
    double fbg[3];
    body_force(time, fbg);
    const double* om = P.omega_rot;
    for (int64_t c = 0; c < nc; ++c) {
      for (int k = 0; k < 3; ++k) H_U[3 * c + k] = conv_U[3 * c + k] + visc_U[3 * c + k] + fbg[k];
      if (P.use_rotation) {
        const double* u = &U[3 * c];
        H_U[3 * c] = H_U[3 * c] - 2.0 * (om[1] * u[2] - om[2] * u[1]);
        H_U[3 * c + 1] = H_U[3 * c + 1] - 2.0 * (om[2] * u[0] - om[0] * u[2]);
        H_U[3 * c + 2] = H_U[3 * c + 2] - 2.0 * (om[0] * u[1] - om[1] * u[0]);
      }
      if (P.boussinesq)
        for (int k = 0; k < 3; ++k) H_U[3 * c + k] = H_U[3 * c + k] - P.beta * (T[c] - P.T_ref) * P.g[k];
    }
    // add_wall_stress_to_rhs (mod_fv_solver.f90:2238-2276)
    for (int64_t fb = 0; fb < nb; ++fb) {
      int64_t fg = nfi + fb;
      if (bc_of_face(fg) != BC_WALL_MODEL) continue;
      int o = m.owner[fg];
      double w = m.area[fg] / m.volume[o];
      for (int k = 0; k < 3; ++k) H_U[3 * o + k] = H_U[3 * o + k] + tau_w[3 * fb + k] * w;
    }
    // temperature (solved when Boussinesq is on) and passive scalars
    if (P.boussinesq) {
      advection_scalar(P.temperature_scheme, T.data(), T_bnd.data(), grad_T.data(), conv_T.data());
      viscous_scalar(T.data(), P.alpha_T, P.Pr_t, grad_T.data(), T_bnd.data(), visc_T.data());
      for (int64_t c = 0; c < nc; ++c) H_T[c] = conv_T[c] + visc_T[c];
      if (P.wall_model == DPM_WM_MOST)  // add_wall_heat_flux_to_rhs (mod_fv_solver.f90:2279-2313)
        for (int64_t fb = 0; fb < nb; ++fb) {
          int64_t fg = nfi + fb;
          if (bc_of_face(fg) != BC_WALL_MODEL) continue;
          int o = m.owner[fg];
          H_T[o] = H_T[o] + q_w[fb] * m.area[fg] / m.volume[o];
        }
    } else {
      std::fill(H_T.begin(), H_T.end(), 0.0);
    }
    for (int sc = 0; sc < ns; ++sc) {
      const double* C = &Cs[(size_t)sc * nc];
      const double* Cb = &C_bnd[(size_t)sc * nb];
      const double* gC = &grad_C[(size_t)sc * 3 * nc];
      advection_scalar(P.scalar_scheme, C, Cb, gC, conv_C.data());
      viscous_scalar(C, P.scalar_diffusivity[sc], P.scalar_pr_t[sc], gC, Cb, visc_C.data());
      for (int64_t c = 0; c < nc; ++c) H_C[(size_t)sc * nc + c] = conv_C[c] + visc_C[c];
    }
    add_scalar_sources(time);
    if (P.use_nudging) nudging_apply(time);
  }

  // body_force_now (mod_fv_solver.f90:2903-2922), as compute_explicit_rhs assembles it (:1662-1675)
  void body_force(double t, double f[3]) const {
    for (int k = 0; k < 3; ++k) f[k] = P.constant_mass_flux_forcing ? mass_flux_force[k] : P.f_const[k];
    if (P.use_harmonic_forcing) {
      const double* fd = P.forcing_dir;
      double dn = std::sqrt(fd[0] * fd[0] + fd[1] * fd[1] + fd[2] * fd[2]);
      double hd[3] = {1.0, 0.0, 0.0};
      if (dn > SMALL)
        for (int k = 0; k < 3; ++k) hd[k] = fd[k] / dn;
      double hs = P.forcing_amp * std::cos(P.forcing_omega * t + P.forcing_phase);
      for (int k = 0; k < 3; ++k) f[k] = f[k] + hs * hd[k];
    }
  }
  // update_mass_flux_forcing (:959-983)
  void update_mass_flux_forcing(double dt) {
    double m1 = 0.0, m2 = 0.0, m3 = 0.0;
    for (int64_t c = 0; c < nc; ++c) {
      m1 = m1 + U[3 * c] * m.volume[c];
      m2 = m2 + U[3 * c + 1] * m.volume[c];
      m3 = m3 + U[3 * c + 2] * m.volume[c];
    }
    const double mom[3] = {m1, m2, m3};
    for (int k = 0; k < 3; ++k) mass_flux_force[k] = (P.U_bulk_target[k] - mom[k] / std::max(V_total, SMALL)) / dt;
  }
  // interp_find_indices (src/abl/mod_abl_weather.f90:335-366), 0-based
  static void interp_find(const std::vector<double>& a, double v, int& i1, int& i2, double& w) {
    const int n = (int)a.size();
    i1 = 0;
    i2 = n - 1;
    for (int i = 0; i < n - 1; ++i)
      if (v >= a[i] && v <= a[i + 1]) { i1 = i; i2 = i + 1; break; }
    const double den = a[i2] - a[i1];
    if (std::fabs(den) < 1.0e-16) w = 0.0;
    else w = std::max(0.0, std::min(1.0, (v - a[i1]) / den));
  }
  // nudging_apply_rhs + nudging_interpolate (:233-333), dt the handle's P.dt as the caller passes it
  void nudging_apply(double t) {
    if (nd_nt < 1) return;
    const double zs = P.nudging_z_start, zt = P.nudging_z_full;
    double coeff = 1.0 / std::max(P.nudging_tau, 1.0e-16);
    if (P.dt > 1.0e-16) coeff = std::min(coeff, 0.5 / P.dt);
    int it1, it2;
    double wt;
    interp_find(nd_times, t, it1, it2, wt);
    for (int64_t c = 0; c < nc; ++c) {
      const double z = m.centroid[3 * c + 2];
      if (z < zs) continue;
      const double ramp = zt > zs ? std::min(1.0, (z - zs) / (zt - zs)) : 1.0;
      int iz1, iz2;
      double wz;
      interp_find(nd_z, z, iz1, iz2, wz);
      auto Up = [&](int j, int iz, int it) { return nd_U[3 * ((size_t)iz + (size_t)nd_nz * it) + j]; };
      auto Tp = [&](int iz, int it) { return nd_T[(size_t)iz + (size_t)nd_nz * it]; };
      double ur[3];
      for (int j = 0; j < 3; ++j)
        ur[j] = (1.0 - wt) * (1.0 - wz) * Up(j, iz1, it1) + wt * (1.0 - wz) * Up(j, iz1, it2) +
                (1.0 - wt) * wz * Up(j, iz2, it1) + wt * wz * Up(j, iz2, it2);
      const double tr = (1.0 - wt) * (1.0 - wz) * Tp(iz1, it1) + wt * (1.0 - wz) * Tp(iz1, it2) +
                        (1.0 - wt) * wz * Tp(iz2, it1) + wt * wz * Tp(iz2, it2);
      H_U[3 * c] = H_U[3 * c] - ramp * coeff * (U[3 * c] - ur[0]);
      H_U[3 * c + 1] = H_U[3 * c + 1] - ramp * coeff * (U[3 * c + 1] - ur[1]);
      if (!P.nudging_horizontal_only) H_U[3 * c + 2] = H_U[3 * c + 2] - ramp * coeff * (U[3 * c + 2] - ur[2]);
      H_T[c] = H_T[c] - ramp * coeff * (T[c] - tr);
    }
  }
  // scalar_source_value_at (src/mod_scalar.f90:133-229)
  static double source_value(const Src& s, const double* x, double t) {
    const dpm_scalar_source_t& d = s.d;
    if (!d.enabled) return 0.0;
    auto dist2 = [](const double* a, const double* b) {
      double r = 0.0;
      for (int k = 0; k < 3; ++k) r = r + (a[k] - b[k]) * (a[k] - b[k]);
      return r;
    };
    auto unit = [](const double* v, double* u) {
      double n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
      if (n <= SMALL) { u[0] = 0.0; u[1] = 0.0; u[2] = 1.0; }
      else for (int k = 0; k < 3; ++k) u[k] = v[k] / n;
    };
    auto slab = [&](double half) {
      double u[3], r[3];
      unit(d.normal, u);
      for (int k = 0; k < 3; ++k) r[k] = x[k] - d.center[k];
      return std::fabs(r[0] * u[0] + r[1] * u[1] + r[2] * u[2]) <= std::max(half, SMALL);
    };
    double w = 0.0;
    switch (d.src_kind) {
      case DPM_SCALAR_SRC_POINT:
        if (dist2(x, d.center) <= std::max(d.radius, SMALL) * std::max(d.radius, SMALL)) w = 1.0;
        break;
      case DPM_SCALAR_SRC_LINE: {
        double ab[3], den = 0.0, tt = 0.0, pr[3];
        for (int k = 0; k < 3; ++k) { ab[k] = d.p1[k] - d.p0[k]; den = den + ab[k] * ab[k]; }
        double dd;
        if (den <= SMALL) {
          dd = std::sqrt(dist2(x, d.p0));
        } else {
          for (int k = 0; k < 3; ++k) tt = tt + (x[k] - d.p0[k]) * ab[k];
          tt = std::max(0.0, std::min(1.0, tt / den));
          for (int k = 0; k < 3; ++k) pr[k] = d.p0[k] + tt * ab[k];
          dd = std::sqrt(dist2(x, pr));
        }
        if (dd <= std::max(d.radius, SMALL)) w = 1.0;
        break;
      }
      case DPM_SCALAR_SRC_SURFACE:
        if (slab(d.half_thickness)) {
          if (d.radius > 0.0) { if (dist2(x, d.center) <= d.radius * d.radius) w = 1.0; }
          else w = 1.0;
        }
        break;
      case DPM_SCALAR_SRC_OBJ:
        if (!s.tags.empty()) {
          double dm = 1.7976931348623157e308;
          for (size_t i = 0; i + 2 < s.tags.size(); i += 3) {
            double di = std::sqrt(dist2(x, &s.tags[i]));
            if (di < dm) dm = di;
          }
          if (dm <= std::max(d.tag_radius, SMALL)) w = 1.0;
        }
        break;
      default:
        if (d.shape == DPM_SCALAR_SHAPE_BOX) {
          if (x[0] >= d.box_min[0] && x[1] >= d.box_min[1] && x[2] >= d.box_min[2] && x[0] <= d.box_max[0] &&
              x[1] <= d.box_max[1] && x[2] <= d.box_max[2])
            w = 1.0;
        } else if (d.shape == DPM_SCALAR_SHAPE_PLANE) {
          if (slab(d.half_thickness)) w = 1.0;
        } else {
          if (dist2(x, d.center) <= std::max(d.radius, SMALL) * std::max(d.radius, SMALL)) w = 1.0;
        }
    }
    const double ts = d.time_mode == DPM_SCALAR_TIME_HARMONIC ? std::cos(d.omega * t + d.phase) : 1.0;
    return d.magnitude * ts * w;
  }
  // add_scalar_source_terms (mod_fv_solver.f90:1764-1784)
  void add_scalar_sources(double t) {
    if (ns <= 0) return;
    for (const Src& s : srcs) {
      if (!s.d.enabled) continue;
      const int sid = s.d.scalar_id;
      if (sid < 1 || sid > ns) continue;
      for (int64_t c = 0; c < nc; ++c) {
        const double v = source_value(s, &m.centroid[3 * c], t);
        if (std::fabs(v) > SMALL) H_C[(size_t)(sid - 1) * nc + c] = H_C[(size_t)(sid - 1) * nc + c] + v;
      }
    }
  }

  // ---------------------------------------------------------------- projection
  // src/solver/mod_fv_solver.f90:2389-2752
  void face_fluxes_and_rhs(double dt, bool incr) {
    if (!skip_grad_p) {
      if (incr) {
        for (int64_t c = 0; c < nc; ++c) p_tot[c] = phi_prev[c] + p[c];
        for (int64_t b = 0; b < nb; ++b) p_tot_bnd[b] = phi_prev_bnd[b] + p_bnd[b];
        gradient_of_scalar(p_tot.data(), p_tot_bnd.data(), gp.data());
      } else {
        gradient_of_scalar(p.data(), p_bnd.data(), gp.data());
      }
    }
    std::fill(rhs_p.begin(), rhs_p.end(), 0.0);
    std::fill(face_flux.begin(), face_flux.end(), 0.0);
    std::fill(built.begin(), built.end(), 0);
    for (int64_t i = 0; i < nfp; ++i) {
      if (ps_skip[i]) continue;
      int o = ps_owner[i], n = ps_nb[i];
      int64_t fm = ps_mesh[i];
      double gcf;
      if (fm < nfi) {
        gcf = m.gc[fm];
      } else {
        int64_t fb = fm - nfi;
        double d_o = m.d_cf[fm], d_n = d_o;
        if (m.periodic_pair_dcf[fb] > SMALL) d_n = m.periodic_pair_dcf[fb];
        if (d_n <= SMALL && m.periodic_pair[fb] >= 0) d_n = m.d_cf[nfi + m.periodic_pair[fb]];
        double d_t = d_o + d_n;
        gcf = d_t > SMALL ? d_n / d_t : 0.5;
      }
      double d_on[3];
      for (int k = 0; k < 3; ++k) d_on[k] = m.centroid[3 * n + k] - m.centroid[3 * o + k];
      const double* sf = &m.sf[3 * fm];
      double Uf[3], plain[3];
      for (int k = 0; k < 3; ++k) plain[k] = gcf * U[3 * o + k] + (1.0 - gcf) * U[3 * n + k];
      if (fm < nfi) {
        double wb = refine_blend_weight(m.skew[fm]);
        const double g = m.gc[fm];
        for (int j = 0; j < 3; ++j) {
          double ue = g * U[3 * o + j] + (1.0 - g) * U[3 * n + j];
          double gm[3];
          for (int i = 0; i < 3; ++i) gm[i] = g * grad_U[9 * o + 3 * j + i] + (1.0 - g) * grad_U[9 * (int64_t)n + 3 * j + i];
          ue = ue + gm[0] * m.eps[3 * fm] + gm[1] * m.eps[3 * fm + 1] + gm[2] * m.eps[3 * fm + 2];
          Uf[j] = plain[j] + wb * (ue - plain[j]);
        }
      } else {
        for (int k = 0; k < 3; ++k) Uf[k] = plain[k];
      }
      double flux = Uf[0] * sf[0] + Uf[1] * sf[1] + Uf[2] * sf[2];
      double krc[3] = {0, 0, 0};
      if (!skip_nonortho && !P.rhie_chow_dual) {
        double k[3];
        kfactor_limited(sf, d_on, P.pressure_min_cos_theta, k);
        if (dot3(k, k) >= NONORTHO_SIN2_TOL * dot3(sf, sf)) for (int j = 0; j < 3; ++j) krc[j] = k[j];
      }
      double gm[3], smk[3];
      for (int j = 0; j < 3; ++j) { gm[j] = gcf * gp_rc[3 * o + j] + (1.0 - gcf) * gp_rc[3 * n + j]; smk[j] = sf[j] - krc[j]; }
      double rc = dot3(gm, smk) - ps_coeff[i] * (phi_prev[n] - phi_prev[o]);
      flux = flux + dt * rc;
      face_flux[fm] = flux;
      built[fm] = 1;
      rhs_p[o] -= flux;
      rhs_p[n] += flux;
    }
    for (int64_t fb : nper_bf) {
      int64_t fg = nfi + fb;
      int o = m.owner[fg];
      int bc = bc_of_face(fg);
      double flux = is_wall(bc) ? 0.0 : dot3(&U_bnd[3 * fb], &m.sf[3 * fg]);
      if (cp_on && bc == BC_OUTLET) {  // compact old-pressure term, so that p_new = p_b there (:2625-2633)
        double d[3];
        for (int k = 0; k < 3; ++k) d[k] = m.centre[3 * fg + k] - m.centroid[3 * o + k];
        double c_b = m.area[fg] / std::max(std::fabs(dot3(d, &m.normal[3 * fg])), SMALL);
        flux = flux - dt * c_b * (pc[m.patch[fg]].p_val - phi_prev[o]);
      }
      face_flux[fg] = flux;
      built[fg] = 1;
      rhs_p[o] -= flux;
    }
    for (int64_t fb : per_bf) {
      int64_t fg = nfi + fb;
      if (built[fg]) continue;
      int o = m.owner[fg];
      int pb = m.periodic_pair[fb];
      if (pb >= 0 && built[nfi + pb]) {
        face_flux[fg] = -face_flux[nfi + pb];
        built[fg] = 1;
        continue;
      }
      int npr = pb >= 0 ? m.owner[nfi + pb] : -1;
      if (npr >= 0) {
        double s = 0;
        for (int k = 0; k < 3; ++k) s += (U[3 * o + k] + U[3 * npr + k]) * m.sf[3 * fg + k];
        face_flux[fg] = 0.5 * s;
      } else {
        face_flux[fg] = dot3(&U[3 * o], &m.sf[3 * fg]);
      }
      built[fg] = 1;
    }
    double rdt = 1.0 / std::max(dt, SMALL);
    for (int64_t c = 0; c < nc; ++c) rhs_p[c] *= rdt;
    if (!skip_nonortho) {
      for (int64_t i = 0; i < nfp; ++i) {
        if (ps_skip[i] || !act_int[i]) continue;
        int o = ps_owner[i], n = ps_nb[i];
        int64_t fm = ps_mesh[i];
        double gw = fm >= nfi ? m.periodic_gc[fm - nfi] : m.gc[fm];
        double cross = 0;
        for (int j = 0; j < 3; ++j) cross += (gw * gp[3 * o + j] + (1.0 - gw) * gp[3 * n + j]) * k_int[3 * i + j];
        rhs_p[o] += cross;
        rhs_p[n] -= cross;
      }
      for (size_t ib = 0; ib < nper_bf.size(); ++ib) {
        int64_t fg = nfi + nper_bf[ib];
        if (bc_of_face(fg) != BC_OUTLET || !act_bnd[ib]) continue;
        int o = m.owner[fg];
        rhs_p[o] += dot3(&gp[3 * o], &k_bnd[3 * ib]);
      }
    }
  }

  // src/solver/mod_fv_solver.f90:2756-2902
  void correct_face_fluxes(double dt, bool ptot) {
    for (int64_t i = 0; i < nfp; ++i) {
      if (ps_skip[i]) continue;
      int o = ps_owner[i], n = ps_nb[i];
      int64_t fm = ps_mesh[i];
      face_flux[fm] = face_flux[fm] - dt * ps_coeff[i] * (p[n] - p[o]);
      if (act_int[i]) {
        double g = fm >= nfi ? m.periodic_gc[fm - nfi] : m.gc[fm];
        double cross = 0;
        for (int j = 0; j < 3; ++j) cross += (g * gp[3 * o + j] + (1.0 - g) * gp[3 * n + j]) * k_int[3 * i + j];
        face_flux[fm] = face_flux[fm] - dt * cross;
      }
    }
    for (size_t ib = 0; ib < nper_bf.size(); ++ib) {
      int64_t fb = nper_bf[ib], fg = nfi + fb;
      if (bc_of_face(fg) != BC_OUTLET) continue;
      int o = m.owner[fg];
      double d[3];
      for (int k = 0; k < 3; ++k) d[k] = m.centre[3 * fg + k] - m.centroid[3 * o + k];
      double dor = std::max(std::fabs(dot3(d, &m.normal[3 * fg])), SMALL);
      double coeff = m.area[fg] / dor;
      double pv = ptot ? pc[m.patch[fg]].p_val : 0.0;
      face_flux[fg] = face_flux[fg] - dt * coeff * (pv - p[o]);
      if (act_bnd[ib]) face_flux[fg] = face_flux[fg] - dt * dot3(&gp[3 * o], &k_bnd[3 * ib]);
    }
    for (int64_t fb : per_bf) {
      int pb = m.periodic_pair[fb];
      if (pb < 0) continue;
      int os = m.owner[nfi + fb], op = m.owner[nfi + pb];
      if (os == op) continue;
      if (os > op) face_flux[nfi + fb] = -face_flux[nfi + pb];
    }
  }

  // src/solver/mod_fv_solver.f90:2927-3151
  void correct_velocity(double dt, bool with_cross, bool ptot) {
    bool do_cross = with_cross && !skip_nonortho;
    std::fill(gp_cell.begin(), gp_cell.end(), 0.0);
    for (int64_t i = 0; i < nfp; ++i) {
      if (ps_skip[i]) continue;
      int o = ps_owner[i], n = ps_nb[i];
      int64_t fm = ps_mesh[i];
      double g = ps_coeff[i] * (p[n] - p[o]);
      if (do_cross && act_int[i]) {
        double gw = fm >= nfi ? m.periodic_gc[fm - nfi] : m.gc[fm];
        double cross = 0;
        for (int j = 0; j < 3; ++j) cross += (gw * gp[3 * o + j] + (1.0 - gw) * gp[3 * n + j]) * k_int[3 * i + j];
        g = g + cross;
      }
      const double* nh = &m.normal[3 * fm];
      for (int k = 0; k < 3; ++k) gp_cell[3 * o + k] = gp_cell[3 * o + k] + g * nh[k];
      for (int k = 0; k < 3; ++k) gp_cell[3 * n + k] = gp_cell[3 * n + k] + g * nh[k];
    }
    for (size_t ib = 0; ib < nper_bf.size(); ++ib) {
      int64_t fg = nfi + nper_bf[ib];
      if (bc_of_face(fg) != BC_OUTLET) continue;
      int o = m.owner[fg];
      double d[3];
      for (int k = 0; k < 3; ++k) d[k] = m.centre[3 * fg + k] - m.centroid[3 * o + k];
      double dor = std::max(std::fabs(dot3(d, &m.normal[3 * fg])), SMALL);
      double coeff = m.area[fg] / dor;
      double g = coeff * ((ptot ? pc[m.patch[fg]].p_val : 0.0) - p[o]);
      if (do_cross && act_bnd[ib]) g = g + dot3(&gp[3 * o], &k_bnd[3 * ib]);
      for (int k = 0; k < 3; ++k) gp_cell[3 * o + k] = gp_cell[3 * o + k] + g * m.normal[3 * fg + k];
    }
    if (!do_cross) {
      double bb = P.boussinesq ? P.beta : 0.0;
      double fb_now[3];
      body_force(time, fb_now);
      for (int64_t fb : nper_bf) {
        int64_t fg = nfi + fb;
        if (bc_of_face(fg) == BC_OUTLET) continue;
        int o = m.owner[fg];
        double d[3];
        for (int k = 0; k < 3; ++k) d[k] = fb_now[k] - bb * (T[o] - P.T_ref) * P.g[k];
        const double* nh = &m.normal[3 * fg];
        double fn = (d[0] * nh[0] + d[1] * nh[1] + d[2] * nh[2]) * m.area[fg];
        for (int k = 0; k < 3; ++k) gp_cell[3 * o + k] = gp_cell[3 * o + k] + fn * nh[k];
      }
    }
    for (int64_t c = 0; c < nc; ++c) {
      const double* Ti = &Tinv[9 * c];
      double* g = &gp_cell[3 * c];
      double g1 = Ti[0] * g[0] + Ti[3] * g[1] + Ti[6] * g[2];
      double g2 = Ti[1] * g[0] + Ti[4] * g[1] + Ti[7] * g[2];
      double g3 = Ti[2] * g[0] + Ti[5] * g[1] + Ti[8] * g[2];
      g[0] = g1; g[1] = g2; g[2] = g3;
      U[3 * c] = U[3 * c] - dt * g1;
      U[3 * c + 1] = U[3 * c + 1] - dt * g2;
      U[3 * c + 2] = U[3 * c + 2] - dt * g3;
    }
  }

  // src/solver/mod_fv_solver.f90:3610-3641
  void anchor_pressure() {
    if (n_outlet > 0) return;
    double s = 0.0;
    for (int64_t c = 0; c < nc; ++c) s += p[c] * m.volume[c];
    double shift = V_total > 0.0 ? s / V_total : 0.0;
    for (int64_t c = 0; c < nc; ++c) p[c] = p[c] - shift;
  }

  // ---------------------------------------------------------------- Poisson solve
  void matvec(const double* x, double* y) const {
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int64_t r = 0; r < nc; ++r) {
      double s = 0.0;
      for (int64_t k = A_off[r]; k < A_off[r + 1]; ++k) s += A_val[k] * x[A_col[k]];
      y[r] = s;
    }
  }
  double vdot(const double* a, const double* b) const {
    double s = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : s) num_threads(nthreads)
    for (int64_t i = 0; i < nc; ++i) s += a[i] * b[i];
    return s;
  }
  void remove_mean(double* v) const {  // MatNullSpaceRemove with the constant vector
    double s = 0.0;
    for (int64_t i = 0; i < nc; ++i) s += v[i];
    double mn = s / (double)nc;
    for (int64_t i = 0; i < nc; ++i) v[i] -= mn;
  }

  // PETSc KSPSolve_CG with KSP_NORM_UNPRECONDITIONED and a Jacobi PC (x: guess in, solution
  // out).  Returns the KSPConvergedReason; *its and *rnorm as KSPGetIterationNumber / true residual.
  int cg(const double* b_in, double* x, double rtol, double atol, int maxit, bool guess_zero, int* its, double* resid) {
    const bool nullsp = dir_rows.empty();
    std::vector<double> b(b_in, b_in + nc), r(nc), z(nc), pv(nc), w(nc);
    if (nullsp) remove_mean(b.data());
    if (guess_zero) std::fill(x, x + nc, 0.0);
    matvec(x, r.data());
    for (int64_t i = 0; i < nc; ++i) r[i] = b[i] - r[i];
    double dp = std::sqrt(vdot(r.data(), r.data()));
    double rnorm0;
    if (!guess_zero) {
      double sn = std::sqrt(vdot(b.data(), b.data()));
      rnorm0 = sn == 0.0 ? dp : sn;
    } else {
      rnorm0 = dp;
    }
    double ttol = std::max(rtol * rnorm0, atol);
    const double divtol = 1.0e5;
    int reason = 0;
    *its = 0;
    auto converged = [&](double rn) {
      if (!finite(rn)) return -9;
      if (rn <= ttol) return rn < atol ? 3 : 2;
      if (rn >= divtol * rnorm0) return -4;
      return 0;
    };
    reason = converged(dp);
    if (!reason) {
      auto pcapply = [&]() {
        for (int64_t i = 0; i < nc; ++i) z[i] = r[i] / A_val_diag(i);
        if (nullsp) remove_mean(z.data());
      };
      pcapply();
      double beta = vdot(z.data(), r.data()), betaold = 0.0, dpi = 0.0, dpiold;
      int i = 0;
      do {
        *its = i + 1;
        if (beta == 0.0) { reason = 3; break; }
        if (i > 0 && beta * betaold < 0.0) { reason = -8; break; }
        if (i == 0) {
          pv = z;
        } else {
          double bb = beta / betaold;
          for (int64_t k = 0; k < nc; ++k) pv[k] = z[k] + bb * pv[k];
        }
        dpiold = dpi;
        matvec(pv.data(), w.data());
        dpi = vdot(pv.data(), w.data());
        betaold = beta;
        if (dpi == 0.0 || (i > 0 && ((dpi > 0) - (dpi < 0)) * ((dpiold > 0) - (dpiold < 0)) < 0)) {
          reason = dpi == 0.0 ? 3 : -10;
          break;
        }
        double a = beta / dpi;
        for (int64_t k = 0; k < nc; ++k) { x[k] += a * pv[k]; r[k] -= a * w[k]; }
        dp = std::sqrt(vdot(r.data(), r.data()));
        reason = converged(dp);
        if (reason) break;
        pcapply();
        beta = vdot(z.data(), r.data());
        i++;
      } while (i < maxit);
      if (!reason && i >= maxit) reason = -3;
    }
    // true residual with the caller's right-hand side (KSPBuildResidual)
    matvec(x, w.data());
    double s = 0.0;
    for (int64_t k = 0; k < nc; ++k) { double d = b_in[k] - w[k]; s += d * d; }
    *resid = std::sqrt(s);
    return reason;
  }
  double A_val_diag(int64_t r) const {
    for (int64_t k = A_off[r]; k < A_off[r + 1]; ++k)
      if (A_col[k] == r) return A_val[k];
    return 1.0;
  }

  // src/solver/mod_pressure_solver.f90:638-806 + pressure_backend_petsc.c:648-1034
  int pressure_solve(double tol, double atol, bool ptot, int* its_out, double* res_out) {
    std::vector<double> rw(rhs_p), pw(p.begin(), p.end());
    for (int64_t i = 0; i < nc; ++i) {
      if (!finite(rw[i])) rw[i] = 0.0;
      if (!finite(pw[i])) pw[i] = 0.0;
    }
    if (ptot)
      for (size_t k = 0; k < dir_rows.size(); ++k) rw[dir_rows[k]] += dir_vals[k];
    int maxit = std::max(P.p_max_iter, 2000);
    int its;
    double res;
    if (record) {
      rec_rhs.push_back(rw);
      rec_x0.push_back(pw);
      rec_atol.push_back(atol);
    }
    int reason = cg(rw.data(), pw.data(), tol, atol, maxit, false, &its, &res);
    if (reason < 0) {
      reason = cg(rw.data(), pw.data(), tol, atol, 4 * maxit, true, &its, &res);
      if (reason < 0 && !(reason == -3 && (res < tol * 1.0e4 || res < atol * 1.0e3))) return -(1000 + reason);
    }
    for (int64_t i = 0; i < nc; ++i) p[i] = pw[i];
    *its_out = its;
    *res_out = res;
    return 0;
  }

  double atol_dynamic(double dt) const {
    double u1 = 0.0, u2 = 0.0;
    for (int64_t c = 0; c < nc; ++c) {
      u1 += std::sqrt(U[3 * c] * U[3 * c] + U[3 * c + 1] * U[3 * c + 1] + U[3 * c + 2] * U[3 * c + 2]) * m.volume[c];
      u2 += m.volume[c];
    }
    double us = u1 / std::max(u2, SMALL);
    return std::max(1.0e-12 * std::max(us, 1.0) * V_min / dt, p_atol_factor);
  }

  // ------------------------------------------------------------------ exact cell projection
  // src/solver/mod_fv_solver.f90:3163-3221 (build_cell_projection): the non-skipped pressure
  // faces with their interpolation weight (periodic weight on periodic faces) and the outlet faces.
  void build_cell_projection() {
    cp_on = P.cell_projection == DPM_CELL_PROJECTION_EXACT;
    cp_own.clear(); cp_nbr.clear(); cp_sf.clear(); cp_gc.clear(); cp_bcell.clear(); cp_bsf.clear();
    for (int64_t i = 0; i < nfp; ++i) {
      if (ps_skip[i]) continue;
      int o = ps_owner[i], n = ps_nb[i];
      int64_t fm = ps_mesh[i];
      if (o < 0 || o >= nc || n < 0 || n >= nc || fm < 0 || fm >= nf) continue;
      cp_own.push_back(o);
      cp_nbr.push_back(n);
      for (int k = 0; k < 3; ++k) cp_sf.push_back(m.sf[3 * fm + k]);
      cp_gc.push_back(fm >= nfi ? m.periodic_gc[fm - nfi] : m.gc[fm]);
    }
    for (int64_t fb : nper_bf) {
      int64_t fg = nfi + fb;
      if (bc_of_face(fg) != BC_OUTLET) continue;
      cp_bcell.push_back(m.owner[fg]);
      for (int k = 0; k < 3; ++k) cp_bsf.push_back(m.sf[3 * fg + k]);
    }
  }
  // src/numerics/mod_cell_projection.f90:84-127 (cp_divergence): outflow sum of the interpolated
  // flux, accumulated in face order.
  void cp_divergence(const double* u, double* out) const {
    std::fill(out, out + nc, 0.0);
    for (size_t f = 0; f < cp_own.size(); ++f) {
      int o = cp_own[f], n = cp_nbr[f];
      double w = cp_gc[f];
      const double* sf = &cp_sf[3 * f];
      double fl = (w * u[3 * o] + (1.0 - w) * u[3 * n]) * sf[0] + (w * u[3 * o + 1] + (1.0 - w) * u[3 * n + 1]) * sf[1] +
                  (w * u[3 * o + 2] + (1.0 - w) * u[3 * n + 2]) * sf[2];
      out[o] = out[o] + fl;
      out[n] = out[n] - fl;
    }
    for (size_t f = 0; f < cp_bcell.size(); ++f) {
      int o = cp_bcell[f];
      const double* bs = &cp_bsf[3 * f];
      out[o] = out[o] + (u[3 * o] * bs[0] + u[3 * o + 1] * bs[1] + u[3 * o + 2] * bs[2]);
    }
  }
  // src/numerics/mod_cell_projection.f90:129-189 (cp_adjoint_gradient): v = V^-1 B^T chi.
  void cp_adjoint(const double* chi, double* v) const {
    std::fill(v, v + 3 * nc, 0.0);
    for (size_t f = 0; f < cp_own.size(); ++f) {
      int o = cp_own[f], n = cp_nbr[f];
      double w = cp_gc[f], d = chi[o] - chi[n];
      const double* sf = &cp_sf[3 * f];
      for (int k = 0; k < 3; ++k) v[3 * o + k] = v[3 * o + k] + w * d * sf[k];
      for (int k = 0; k < 3; ++k) v[3 * n + k] = v[3 * n + k] + (1.0 - w) * d * sf[k];
    }
    for (size_t f = 0; f < cp_bcell.size(); ++f) {
      int o = cp_bcell[f];
      for (int k = 0; k < 3; ++k) v[3 * o + k] = v[3 * o + k] + chi[o] * cp_bsf[3 * f + k];
    }
    for (int64_t c = 0; c < nc; ++c) {
      double iv = 1.0 / m.volume[c];
      for (int k = 0; k < 3; ++k) v[3 * c + k] = v[3 * c + k] * iv;
    }
  }
  // The preconditioner of the projection (mod_fv_solver.f90:3277-3282): z = 0, then the pressure
  // solve to rtol 0.05 with at most 50 iterations, which the backend raises to its 2000 floor
  // (pressure_backend_petsc.c:844), with the backend's NaN scrub and retry.
  int cp_precond(const double* r, double* z, int* its_out) {
    std::vector<double> rw(r, r + nc);
    for (auto& x : rw)
      if (!finite(x)) x = 0.0;
    std::fill(z, z + nc, 0.0);
    const double tol = 0.05, atol = 1.0e-50;
    const int maxit = std::max(50, 2000);
    int its = 0;
    double res = 0.0;
    int reason = cg(rw.data(), z, tol, atol, maxit, false, &its, &res);
    if (reason < 0) {
      reason = cg(rw.data(), z, tol, atol, 4 * maxit, true, &its, &res);
      if (reason < 0 && !(reason == -3 && (res < tol * 1.0e4 || res < atol * 1.0e3))) return -(1000 + reason);
    }
    *its_out = its;
    return 0;
  }
  // src/numerics/mod_cell_projection.f90:192-303 (cp_project): u <- u - V^-1 B^T chi with
  // (B V^-1 B^T) chi = B u + bconst by flexible PCG. identity_pc replaces the pressure-solve
  // preconditioner by z = r (the reference's unit test does the same).
  int cp_project(double* u, const double* bconst, double tol, int max_it, bool identity_pc, int* n_it) {
    std::vector<double> b(nc, 0.0), x(nc, 0.0), r(nc, 0.0), z(nc, 0.0), pv(nc, 0.0), q(nc, 0.0), rold(nc, 0.0),
        chi(nc, 0.0), v(3 * nc, 0.0);
    auto precond = [&](int* its) -> int {
      if (identity_pc) { z = r; *its = 0; return 0; }
      return cp_precond(r.data(), z.data(), its);
    };
    cp_divergence(u, b.data());
    double smax = 0.0;
    for (int64_t c = 0; c < nc; ++c) {
      b[c] = b[c] + bconst[c];
      r[c] = b[c];
      smax = std::max(smax, std::fabs(r[c]));
    }
    *n_it = 0;
    const double bn = smax, tiny = std::numeric_limits<double>::min();
    if (!(bn > tiny)) return 0;
    int its = 0;
    int rc = precond(&its);
    if (rc) return rc;
    cp_precond_iters += its;
    double rz = 0.0;
    for (int64_t c = 0; c < nc; ++c) {
      pv[c] = z[c];
      rz = rz + r[c] * z[c];
    }
    double en_tot = 0.0;
    for (int it = 1; it <= max_it; ++it) {
      *n_it = it;
      chi = pv;
      cp_adjoint(chi.data(), v.data());
      cp_divergence(v.data(), q.data());
      double pq = 0.0;
      for (int64_t c = 0; c < nc; ++c) pq = pq + pv[c] * q[c];
      if (std::fabs(pq) <= tiny) break;
      double alpha = rz / pq;
      double en_new = alpha * alpha * pq;
      en_tot = en_tot + en_new;
      smax = 0.0;
      for (int64_t c = 0; c < nc; ++c) {
        rold[c] = r[c];
        x[c] = x[c] + alpha * pv[c];
        r[c] = r[c] - alpha * q[c];
        smax = std::max(smax, std::fabs(r[c]));
      }
      if (smax <= 1.0e-12 * bn || (it >= 2 && en_new <= tol * tol * en_tot)) break;
      std::fill(z.begin(), z.end(), 0.0);
      rc = precond(&its);
      if (rc) return rc;
      cp_precond_iters += its;
      double s1 = 0.0, s2 = 0.0;
      for (int64_t c = 0; c < nc; ++c) {
        s1 = s1 + (r[c] - rold[c]) * z[c];
        s2 = s2 + r[c] * z[c];
      }
      double beta = std::max(0.0, s1 / rz);
      rz = s2;
      for (int64_t c = 0; c < nc; ++c) pv[c] = z[c] + beta * pv[c];
    }
    chi = x;
    cp_adjoint(chi.data(), v.data());
    for (int64_t c = 0; c < nc; ++c)
      for (int k = 0; k < 3; ++k) u[3 * c + k] = u[3 * c + k] - v[3 * c + k];
    return 0;
  }
  double cp_tol() const {
    double t = P.cell_projection_tol > 0.0 ? P.cell_projection_tol : 0.1;
    return std::max(t, 1.0e-8);
  }
  // src/solver/mod_fv_solver.f90:3223-3283 (project_cells_exact): the outlet pressure acts on its
  // cell as the boundary force -p_b S_f / V; Dirichlet-velocity faces give the fixed outflow.
  int project_cells_exact(double dt) {
    std::vector<double> bconst(nc, 0.0);
    for (int64_t fb : nper_bf) {
      int64_t fg = nfi + fb;
      int o = m.owner[fg];
      int bc = bc_of_face(fg);
      if (is_wall(bc)) continue;
      const double* sf = &m.sf[3 * fg];
      if (bc == BC_OUTLET) {
        double fl = dt * pc[m.patch[fg]].p_val / m.volume[o];
        for (int k = 0; k < 3; ++k) U[3 * o + k] = U[3 * o + k] - fl * sf[k];
      } else {
        bconst[o] = bconst[o] + (U_bnd[3 * fb] * sf[0] + U_bnd[3 * fb + 1] * sf[1] + U_bnd[3 * fb + 2] * sf[2]);
      }
    }
    int n_it = 0;
    int rc = cp_project(U.data(), bconst.data(), cp_tol(), 100, false, &n_it);
    cp_iters += n_it;
    return rc;
  }

  // src/stats/mod_sampling.f90:520-562 (cache_object_owners, one rank) and :493-518
  // (sample_points_local) with the gradients of sampling_maybe_sample (:171-177): one
  // Green-Gauss pass with the boundary values of U, p and T, the owner's value for nu_sgs.
  void sample_points(int np, const double* xyz, double* payload, int* owner) {
    std::vector<double> gu(9 * nc), gpv(3 * nc), gt(3 * nc), gn(3 * nc), nub(nb);
    for (int64_t b = 0; b < nb; ++b) nub[b] = nu_sgs[m.owner[nfi + b]];
    gg_gradient_vector(U.data(), U_bnd.data(), gu.data(), nullptr);
    gg_gradient_scalar(p.data(), p_bnd.data(), gpv.data(), nullptr);
    gg_gradient_scalar(T.data(), T_bnd.data(), gt.data(), nullptr);
    gg_gradient_scalar(nu_sgs.data(), nub.data(), gn.data(), nullptr);
    for (int i = 0; i < np; ++i) {
      const double* x = xyz + 3 * i;
      double best = 1.7976931348623157e308;
      int c = -1;
      for (int64_t k = 0; k < nc; ++k) {
        const double* ck = &m.centroid[3 * k];
        double dx = ck[0] - x[0], dy = ck[1] - x[1], dz = ck[2] - x[2];
        double d2 = (dx * dx + dy * dy) + dz * dz;
        if (d2 < best) { best = d2; c = (int)k; }
      }
      if (owner) owner[i] = c;
      double* out = payload + 6 * (size_t)i;
      if (c < 0) { for (int k = 0; k < 6; ++k) out[k] = 0.0; continue; }
      double d[3];
      for (int k = 0; k < 3; ++k) d[k] = x[k] - m.centroid[3 * c + k];
      for (int j = 0; j < 3; ++j)
        out[j] = U[3 * c + j] + (gu[9 * c + 3 * j] * d[0] + gu[9 * c + 3 * j + 1] * d[1] + gu[9 * c + 3 * j + 2] * d[2]);
      out[3] = p[c] + (gpv[3 * c] * d[0] + gpv[3 * c + 1] * d[1] + gpv[3 * c + 2] * d[2]);
      out[4] = T[c] + (gt[3 * c] * d[0] + gt[3 * c + 1] * d[1] + gt[3 * c + 2] * d[2]);
      out[5] = nu_sgs[c] + (gn[3 * c] * d[0] + gn[3 * c + 1] * d[1] + gn[3 * c + 2] * d[2]);
    }
  }

  // src/solver/mod_fv_solver.f90:837-918
  int project_once(double dt) {
    std::fill(rhs_p.begin(), rhs_p.end(), 0.0);
    std::fill(phi_prev.begin(), phi_prev.end(), 0.0);
    std::fill(phi_prev_bnd.begin(), phi_prev_bnd.end(), 0.0);
    std::fill(gp_rc.begin(), gp_rc.end(), 0.0);
    refresh_halos_and_bc();
    face_fluxes_and_rhs(dt, false);
    if (P.p_max_iter > 0) {
      int its;
      double res;
      int rc = pressure_solve(P.p_tol, atol_dynamic(dt), true, &its, &res);
      if (rc) return rc;
    }
    anchor_pressure();
    correct_face_fluxes(dt, true);
    U_face = face_flux;
    u_face_ready = true;
    apply_pressure_bc(p.data(), -1, false, false);
    if (cp_on) {
      int rc = project_cells_exact(dt);
      if (rc) return rc;
    } else {
      correct_velocity(dt, true, true);
    }
    apply_velocity_bc(-1, false);
    if (P.use_rotational_projection) {
      for (int64_t c = 0; c < nc; ++c) p[c] = p[c] + (P.nu + nu_sgs[c]) * rhs_p[c] * dt * inv_vol[c];
      apply_pressure_bc(p.data(), -1, false, false);
    }
    p_old = p;
    phi_prev = p;
    phi_prev_bnd = p_bnd;
    apply_pressure_bc(p.data(), -1, false, false);
    compute_pressure_gradient();
    return 0;
  }

  // src/solver/mod_fv_solver.f90:3718-3871
  void cfl_rates(double& conv, double& diff) const {
    std::vector<double> fs(nc, 0.0), ds(nc, 0.0);
    for (int64_t f = 0; f < nf; ++f) {
      int o = m.owner[f], n = m.neighbour[f];
      const double* sf = &m.sf[3 * f];
      double area = std::sqrt(sf[0] * sf[0] + sf[1] * sf[1] + sf[2] * sf[2]);
      double uf = u_face_ready ? U_face[f] : dot3(&U[3 * o], sf);
      fs[o] += std::fabs(uf);
      if (n >= 0) fs[n] += std::fabs(uf);
      double w = area / std::max(m.d_cf[f], SMALL);
      if (n >= 0) {
        double g = m.gc[f];
        double ne = P.nu + g * std::max(0.0, nu_sgs[o]) + (1.0 - g) * std::max(0.0, nu_sgs[n]);
        ds[o] += ne * w;
        ds[n] += ne * w;
      } else if (bc_of_face(f) != BC_WALL_MODEL) {
        ds[o] += (P.nu + std::max(0.0, nu_sgs[o])) * w;
      }
    }
    conv = 0.0; diff = 0.0;
    for (int64_t c = 0; c < nc; ++c) {
      conv = std::max(conv, fs[c] / (m.volume[c] + SMALL));
      diff = std::max(diff, ds[c] / (m.volume[c] + SMALL));
    }
  }
  int compute_dt(double& dt) const {
    double cr, dr;
    cfl_rates(cr, dr);
    double dc = 1e308, dd = 1e308;
    if (cr > SMALL) dc = P.cfl_max / cr;
    if (dr > SMALL) dd = 1.0 / dr;
    dt = std::min(dc, dd);
    if (!(dt > 0.0)) dt = P.dt;
    dt = std::min(dt, P.dt);
    double dmin = 1.0e-6 * P.dt;
    if (!(dt > 0.0)) dt = P.dt;
    else if (dt < dmin) return DPM_ERR_DT_COLLAPSE;
    return 0;
  }

  // src/solver/mod_fv_solver.f90:920-958 + advance_rk3w :1180-1614
  int advance(double dt_in) {
    double dt = dt_in;
    if (!P.adapt_dt) {
      double ds;
      int rc = compute_dt(ds);
      if (rc) return rc;
      if (dt > ds) dt = ds;
    }
    if (P.constant_mass_flux_forcing) update_mass_flux_forcing(dt);
    last_dt = dt;
    last_solves = 0; last_iters = 0; last_resid = 0.0;
    cp_iters = 0; cp_precond_iters = 0;
    std::fill(H_U.begin(), H_U.end(), 0.0);
    std::fill(rhs_p.begin(), rhs_p.end(), 0.0);
    std::fill(H_U0.begin(), H_U0.end(), 0.0);
    std::fill(H_T.begin(), H_T.end(), 0.0);
    std::fill(H_T0.begin(), H_T0.end(), 0.0);
    std::fill(H_C.begin(), H_C.end(), 0.0);
    std::fill(H_C0.begin(), H_C0.end(), 0.0);
    double time_n = time;
    for (int k = 0; k < 3; ++k) {
      double gk_dt = RK3W_GAMMA[k] * dt;
      time = time_n + RK3W_C[k] * dt;
      refresh_halos_and_bc();
      compute_all_gradients();
      sgs_viscosity(gk_dt);
      if (P.wall_model == DPM_WM_NONE) std::fill(tau_w.begin(), tau_w.end(), 0.0);
      else if (P.wall_model == DPM_WM_MOST) most_wall_model(k == 0);
      else wall_model(k == 0 ? dt : 0.0);
      explicit_rhs();
      double a_k = RK3W_ALPHA[k], b_k = RK3W_BETA[k];
      for (int64_t c = 0; c < nc; ++c)
        for (int j = 0; j < 3; ++j) U[3 * c + j] = U[3 * c + j] + dt * (a_k * H_U[3 * c + j] + b_k * H_U0[3 * c + j]);
      for (int64_t c = 0; c < nc; ++c) T[c] = T[c] + dt * (a_k * H_T[c] + b_k * H_T0[c]);
      for (size_t i = 0; i < Cs.size(); ++i) Cs[i] = Cs[i] + dt * (a_k * H_C[i] + b_k * H_C0[i]);
      if (sem.initialized)  // the stage's end time, sampled upstream of the step-start eddies (:1350-1358)
        update_sem_inflow(time_n + (RK3W_C[k] + RK3W_GAMMA[k]) * dt, true, (RK3W_C[k] + RK3W_GAMMA[k]) * dt);
      velocity_bc_refresh();
      p_old = p;
      if (cp_on) std::fill(gp_cell.begin(), gp_cell.end(), 0.0);  // nothing to add back (mod_fv_solver.f90:1373-1377)
      else correct_velocity(gk_dt, false, true);
      gp_rc = gp_cell;
      velocity_bc_refresh();
      compute_all_gradients();
      phi_prev = p;
      phi_prev_bnd = p_bnd;
      // Poisson block with non-orthogonal correctors
      double atol = atol_dynamic(gk_dt);
      int n_max;
      double stag;
      if (diag_interface) { n_max = std::min(P.n_nonortho_corr, 8); stag = 0.99; }
      else { n_max = std::min(P.n_nonortho_corr, 3); stag = 0.9; }
      double dprev = 1e308, dphi_prev = 1e308;
      if (P.nonortho_check) {
        n_max = std::min(P.n_nonortho_corr, 8);
        std::fill(phi_it.begin(), phi_it.end(), 0.0);
      }
      for (int jno = 1; jno <= n_max; ++jno) {
        face_fluxes_and_rhs(gk_dt, jno > 1);
        double dcur = 0.0;
        for (int64_t c = 0; c < nc; ++c) dcur = std::max(dcur, std::fabs(rhs_p[c]));
        if (jno == 1) std::fill(p.begin(), p.end(), 0.0);
        int its;
        double res;
        int rc = pressure_solve(P.p_tol, atol, false, &its, &res);
        if (rc) return rc;
        last_solves++;
        last_iters += its;
        last_resid = std::max(last_resid, res);
        apply_pressure_bc(p.data(), 0, !skip_grad_p, true);
        apply_pressure_bc(p.data(), 1, false, false);
        if (P.nonortho_check) {
          double dd = 0.0, dpp = 0.0;
          for (int64_t c = 0; c < nc; ++c) {
            dd = std::max(dd, std::fabs(p[c] - phi_it[c]));
            dpp = std::max(dpp, std::fabs(p[c]));
            phi_it[c] = p[c];
          }
          if (jno > 1 && (dd < NONORTHO_PHI_TOL * dpp || dd > dphi_prev * stag)) break;
          dphi_prev = dd;
        } else if (jno > 1 && (dcur < atol || dcur > dprev * stag)) {
          break;
        }
        dprev = dcur;
      }
      correct_face_fluxes(gk_dt, false);
      U_face = face_flux;
      u_face_ready = true;
      if (cp_on) {
        int rc2 = project_cells_exact(gk_dt);
        if (rc2) return rc2;
      } else {
        correct_velocity(gk_dt, true, false);
      }
      velocity_bc_refresh();
      if (P.use_rotational_projection) {
        for (int64_t c = 0; c < nc; ++c) p[c] = p[c] + (P.nu + nu_sgs[c]) * rhs_p[c] * gk_dt * inv_vol[c];
        apply_pressure_bc_o2(true);
        apply_pressure_bc(p.data(), 1, false, false);
      }
      for (int64_t c = 0; c < nc; ++c) p[c] = p[c] + p_old[c];
      anchor_pressure();
      apply_pressure_bc_o2(false);
      apply_pressure_bc(p.data(), 1, false, false);
      compute_pressure_gradient();
      H_U0 = H_U;
      H_T0 = H_T;
      H_C0 = H_C;
    }
    sem_advance(dt);  // mod_fv_solver.f90:1606-1610
    apply_scalar_bcs_all();
    time = time_n + dt;
    step++;
    return 0;
  }

  // src/stats/mod_stats.f90:271-336 + mod_fv_solver.f90:3643-3716
  void stats(dpm_stats_t* s) {
    double sums[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, umax = 0.0;
    for (int64_t c = 0; c < nc; ++c) {
      double v = m.volume[c];
      const double* u = &U[3 * c];
      const double* g = &grad_U[9 * c];
      sums[0] += 0.5 * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]) * v;
      sums[1] += v;
      double S11 = g[0], S22 = g[4], S33 = g[8];
      double S12 = 0.5 * (g[1] + g[3]), S13 = 0.5 * (g[2] + g[6]), S23 = 0.5 * (g[5] + g[7]);
      double SS = S11 * S11 + S22 * S22 + S33 * S33 + 2.0 * (S12 * S12 + S13 * S13 + S23 * S23);
      sums[2] += (P.nu + nu_sgs[c]) * SS * v;
      for (int k = 0; k < 3; ++k) sums[3 + k] += u[k] * v;
      sums[6] += nu_sgs[c] * v;
      umax = std::max(umax, std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]));
    }
    for (int q = 0; q < m.n_patches; ++q) {
      if (pc[q].bc_id != BC_WALL_MODEL) continue;
      for (int64_t f = 0; f < m.patch_nfaces[q]; ++f) {
        int64_t fb = m.patch_start[q] + f;
        const double* t = &tau_w[3 * fb];
        sums[7] += std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]) * m.area[nfi + fb];
        sums[8] += m.area[nfi + fb];
      }
    }
    s->time = time;
    s->E = sums[0] / sums[1];
    s->eps = 2.0 * sums[2] / sums[1];
    double mb[3] = {sums[3] / sums[1], sums[4] / sums[1], sums[5] / sums[1]};
    s->Ub = std::sqrt(mb[0] * mb[0] + mb[1] * mb[1] + mb[2] * mb[2]);
    s->nu_sgs_mean = sums[6] / sums[1];
    s->tauw_mean = sums[8] > SMALL ? sums[7] / sums[8] : 0.0;
    s->Umax = umax;
    // face-flux divergence
    std::vector<double> div(nc, 0.0);
    for (int64_t i = 0; i < nfp; ++i) {
      if (ps_skip[i]) continue;
      int o = ps_owner[i], n = ps_nb[i];
      double fl = face_flux[ps_mesh[i]];
      div[o] += fl * inv_vol[o];
      div[n] -= fl * inv_vol[n];
    }
    for (int64_t fb : nper_bf) {
      int o = m.owner[nfi + fb];
      div[o] += face_flux[nfi + fb] * inv_vol[o];
    }
    double mx = 0.0, as = 0.0, vs = 0.0;
    for (int64_t c = 0; c < nc; ++c) {
      mx = std::max(mx, std::fabs(div[c]));
      as += std::fabs(div[c]) * m.volume[c];
      vs += m.volume[c];
    }
    s->max_abs_divU = mx;
    s->volavg_abs_divU = as / vs;
    s->dt_used = last_dt;
    s->p_solves = last_solves;
    s->p_iters = last_iters;
    s->p_resid_max = last_resid;
    s->p_fallbacks = 0;
    s->p_solver_used = DPM_PSOLVER_JACOBI_PCG;
    s->p_bytes_per_iteration = 0.0;  // no device traffic on the CPU
    s->cp_iters = cp_iters;
    s->cp_precond_iters = cp_precond_iters;
    apply_velocity_bc(-1, false);  // solver_divergence_metrics refreshes U_bnd without gradients
    // cell_velocity_divergence (mod_fv_solver.f90:3582-3607): every mesh face in order, the
    // gc-interpolated velocity inside, the boundary velocity on boundary (periodic too) faces
    std::fill(div.begin(), div.end(), 0.0);
    for (int64_t f = 0; f < nf; ++f) {
      int o = m.owner[f], n = m.neighbour[f];
      double uf[3];
      if (n >= 0) {
        double g = m.gc[f];
        for (int k = 0; k < 3; ++k) uf[k] = g * U[3 * o + k] + (1.0 - g) * U[3 * n + k];
      } else {
        for (int k = 0; k < 3; ++k) uf[k] = U_bnd[3 * (f - nfi) + k];
      }
      double fl = dot3(uf, &m.sf[3 * f]);
      div[o] += fl * inv_vol[o];
      if (n >= 0) div[n] -= fl * inv_vol[n];
    }
    mx = 0.0; as = 0.0;
    for (int64_t c = 0; c < nc; ++c) {
      mx = std::max(mx, std::fabs(div[c]));
      as += std::fabs(div[c]) * m.volume[c];
    }
    s->max_abs_divU_cell = mx;
    s->volavg_abs_divU_cell = as / vs;
  }
};

}  // namespace orc

// ------------------------------------------------------------------------------------------
// C entry points used by the tests (ctypes) and by the CPU-baseline leg of bench.py.
extern "C" {

void* orc_create(const dpm_raw_mesh_t* raw, const dpm_patch_cfg_t* patches, const dpm_params_t* prm, int nthreads) {
  auto* s = new orc::Solver();
  s->nthreads = nthreads > 0 ? nthreads : 1;
  std::string err;
  if (s->init(raw, patches, prm, &err)) {
    std::fprintf(stderr, "orc_create: %s\n", err.c_str());
    delete s;
    return nullptr;
  }
  return s;
}
void orc_destroy(void* h) { delete static_cast<orc::Solver*>(h); }
void orc_sizes(void* h, int64_t* out) {
  auto* s = static_cast<orc::Solver*>(h);
  out[0] = s->nc; out[1] = s->nf; out[2] = s->nfi; out[3] = s->nb; out[4] = s->nfp;
  out[5] = s->skip_nonortho; out[6] = s->skip_grad_p; out[7] = s->diag_interface;
}
void orc_geometry(void* h, double* centroid, double* volume) {
  auto* s = static_cast<orc::Solver*>(h);
  if (centroid) std::memcpy(centroid, s->m.centroid.data(), sizeof(double) * 3 * s->nc);
  if (volume) std::memcpy(volume, s->m.volume.data(), sizeof(double) * s->nc);
}
void orc_face_centres(void* h, double* fc) {
  auto* s = static_cast<orc::Solver*>(h);
  std::memcpy(fc, s->m.centre.data(), sizeof(double) * 3 * s->nf);
}
void orc_vertex_bounds(void* h, double* lo, double* hi) {
  auto* s = static_cast<orc::Solver*>(h);
  for (int k = 0; k < 3; ++k) { lo[k] = 1e308; hi[k] = -1e308; }
  for (int64_t v = 0; v < s->m.n_vertices; ++v)
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], s->m.vertices[3 * v + k]);
      hi[k] = std::max(hi[k], s->m.vertices[3 * v + k]);
    }
}
void orc_set_state(void* h, const double* U, const double* p, const double* T) {
  auto* s = static_cast<orc::Solver*>(h);
  if (U) std::memcpy(s->U.data(), U, sizeof(double) * 3 * s->nc);
  if (p) std::memcpy(s->p.data(), p, sizeof(double) * s->nc);
  if (T) std::memcpy(s->T.data(), T, sizeof(double) * s->nc);
}
void orc_get_state(void* h, double* U, double* p, double* nu_sgs, double* grad_U, double* face_flux) {
  auto* s = static_cast<orc::Solver*>(h);
  if (U) std::memcpy(U, s->U.data(), sizeof(double) * 3 * s->nc);
  if (p) std::memcpy(p, s->p.data(), sizeof(double) * s->nc);
  if (nu_sgs) std::memcpy(nu_sgs, s->nu_sgs.data(), sizeof(double) * s->nc);
  if (grad_U) std::memcpy(grad_U, s->grad_U.data(), sizeof(double) * 9 * s->nc);
  if (face_flux) std::memcpy(face_flux, s->U_face.data(), sizeof(double) * s->nf);
}
// ------------------------------------------------------------------------------------------
// Learned term of the two-level preconditioner: loss and gradient in double, restating the
// device network (dopamine_b200/csrc/cuda/learn.cuh) with its bf16 rounding points, for the
// gradient check.  Network per cell: in = [bf16(f) ; bf16(sum_j a~_ij f_j)],
// h1 = relu(W1b in + b1), h2 = relu(W2b bf16(h1) + b2), omega = 0.25 softplus(w3 . h2 + b3);
// loss = mean_k 1 - (z.r)^2 / ((z.Az)(e.r)), z = zb + omega .* u.
namespace {
float orc_bf16(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);
  u &= 0xFFFF0000u;
  float y;
  std::memcpy(&y, &u, 4);
  return y;
}
}  // namespace
int orc_lp_loss_grad(int n, int C, int WL, const uint32_t* lpk, const float* feat, int WA, const int* col,
                     const double* val, int S, const double* R, const double* Z, const double* U, const double* E,
                     const float* prm, double* loss, double* grad) {
  const int F = 8, H = 16, W1 = 0, B1 = 256, W2 = 272, B2 = 528, W3 = 544, B3 = 560, NP = 561;
  std::vector<double> wb(NP);
  for (int j = 0; j < NP; ++j)
    wb[j] = (j < B1 || (j >= W2 && j < B2)) ? (double)orc_bf16(prm[j]) : (double)prm[j];
  std::vector<double> in((size_t)n * 16), h1((size_t)n * H), h2((size_t)n * H), pre(n), om(n);
  for (int i = 0; i < n; ++i) {
    const int base = (i / C) * C;
    float agg[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int s2 = 0; s2 < WL; ++s2) {
      const uint32_t e = lpk[(size_t)s2 * n + i];
      uint32_t hb = e & 0xFFFF0000u;
      float w;
      std::memcpy(&w, &hb, 4);
      if (w == 0.0f) continue;
      const int j = base + (int)(e & 0xFFFFu);
      for (int k = 0; k < F; ++k) agg[k] = std::fmaf(w, feat[(size_t)k * n + j], agg[k]);
    }
    for (int k = 0; k < F; ++k) {
      in[(size_t)i * 16 + k] = orc_bf16(feat[(size_t)k * n + i]);
      in[(size_t)i * 16 + F + k] = orc_bf16(agg[k]);
    }
    for (int o = 0; o < H; ++o) {
      double t = wb[B1 + o];
      for (int k = 0; k < 16; ++k) t += wb[W1 + o * 16 + k] * in[(size_t)i * 16 + k];
      h1[(size_t)i * H + o] = std::max(t, 0.0);
    }
    for (int o = 0; o < H; ++o) {
      double t = wb[B2 + o];
      for (int k = 0; k < H; ++k) t += wb[W2 + o * 16 + k] * (double)orc_bf16((float)h1[(size_t)i * H + k]);
      h2[(size_t)i * H + o] = std::max(t, 0.0);
    }
    double p = wb[B3];
    for (int k = 0; k < H; ++k) p += wb[W3 + k] * h2[(size_t)i * H + k];
    pre[i] = p;
    om[i] = 0.25 * (p > 20.0 ? p : std::log1p(std::exp(p)));
  }
  auto spmv = [&](const std::vector<double>& x, std::vector<double>& y) {
    for (int i = 0; i < n; ++i) {
      double t = 0.0;
      for (int w = 0; w < WA; ++w) t += val[(size_t)w * n + i] * x[col[(size_t)w * n + i]];
      y[i] = t;
    }
  };
  std::vector<double> z(n), Az(n), dom(n, 0.0);
  double L = 0.0;
  for (int k = 0; k < S; ++k) {
    const double *r = R + (size_t)k * n, *zb = Z + (size_t)k * n, *u = U + (size_t)k * n, *e = E + (size_t)k * n;
    for (int i = 0; i < n; ++i) z[i] = zb[i] + om[i] * u[i];
    spmv(z, Az);
    double a = 0.0, b = 0.0, c = 0.0;
    for (int i = 0; i < n; ++i) { a += z[i] * r[i]; b += z[i] * Az[i]; c += e[i] * r[i]; }
    const double bc = std::max(b * c, 1e-300);
    L += 1.0 - a * a / bc;
    const double c0 = 2.0 * a / bc, c1 = 2.0 * a * a / (bc * std::max(b, 1e-300));
    for (int i = 0; i < n; ++i) dom[i] += -(c0 * r[i] - c1 * Az[i]) / S * u[i];
  }
  *loss = L / S;
  if (!grad) return 0;
  for (int j = 0; j < NP; ++j) grad[j] = 0.0;
  for (int i = 0; i < n; ++i) {
    const double p = pre[i];
    const double dpre = dom[i] * 0.25 / (1.0 + std::exp(-p));
    double d2[16], d1[16];
    for (int k = 0; k < H; ++k) {
      const double x2 = h2[(size_t)i * H + k];
      grad[W3 + k] += dpre * x2;
      d2[k] = x2 > 0.0 ? dpre * wb[W3 + k] : 0.0;
    }
    grad[B3] += dpre;
    for (int o = 0; o < H; ++o) {
      grad[B2 + o] += d2[o];
      for (int k = 0; k < H; ++k) grad[W2 + o * 16 + k] += d2[o] * (double)orc_bf16((float)h1[(size_t)i * H + k]);
    }
    for (int k = 0; k < H; ++k) {
      double t = 0.0;
      for (int o = 0; o < H; ++o) t += d2[o] * wb[W2 + o * 16 + k];
      d1[k] = h1[(size_t)i * H + k] > 0.0 ? t : 0.0;
    }
    for (int o = 0; o < H; ++o) {
      grad[B1 + o] += d1[o];
      for (int k = 0; k < 16; ++k) grad[W1 + o * 16 + k] += d1[o] * in[(size_t)i * 16 + k];
    }
  }
  return 0;
}

// Temperature [nc] and passive scalars [n_scalars][nc] (scalar-major), either may be NULL.
void orc_get_scalars(void* h, double* T, double* C) {
  auto* s = static_cast<orc::Solver*>(h);
  if (T) std::memcpy(T, s->T.data(), sizeof(double) * s->nc);
  if (C && !s->Cs.empty()) std::memcpy(C, s->Cs.data(), sizeof(double) * s->Cs.size());
}
void orc_set_scalars(void* h, const double* T, const double* C) {
  auto* s = static_cast<orc::Solver*>(h);
  if (T) std::memcpy(s->T.data(), T, sizeof(double) * s->nc);
  if (C && !s->Cs.empty()) std::memcpy(s->Cs.data(), C, sizeof(double) * s->Cs.size());
}
int orc_project_once(void* h, double dt) { return static_cast<orc::Solver*>(h)->project_once(dt); }
int orc_advance(void* h, double dt) { return static_cast<orc::Solver*>(h)->advance(dt); }
void orc_stats(void* h, dpm_stats_t* out) { static_cast<orc::Solver*>(h)->stats(out); }
double orc_time(void* h) { return static_cast<orc::Solver*>(h)->time; }
int orc_compute_dt(void* h, double* dt) { return static_cast<orc::Solver*>(h)->compute_dt(*dt); }

// Single-operator checks on arbitrary inputs (same arguments as the product's dpm_* operators).
void orc_ls_gradient_vector(void* h, const double* U, const double* U_bnd, double* g) {
  static_cast<orc::Solver*>(h)->ls_gradient_vector(U, U_bnd, g);
}
// Green-Gauss gradient of a cell scalar (cell-major g[3c + i]) with `sweeps` sweeps.
void orc_gg_gradient_scalar(void* h, const double* phi, const double* pb, double* g, int sweeps) {
  auto* s = static_cast<orc::Solver*>(h);
  s->gg_gradient_scalar(phi, pb, g, nullptr);
  std::vector<double> prev;
  for (int it = 2; it <= sweeps; ++it) {
    prev.assign(g, g + 3 * s->nc);
    s->gg_gradient_scalar(phi, pb, g, prev.data());
  }
}
void orc_advection(void* h, int scheme, const double* U, const double* U_bnd, const double* flux, const double* gU,
                   double* rhs) {
  auto* s = static_cast<orc::Solver*>(h);
  std::memcpy(s->U.data(), U, sizeof(double) * 3 * s->nc);
  std::memcpy(s->U_bnd.data(), U_bnd, sizeof(double) * 3 * s->nb);
  std::memcpy(s->U_face.data(), flux, sizeof(double) * s->nf);
  std::memcpy(s->grad_U.data(), gU, sizeof(double) * 9 * s->nc);
  int keep = s->P.scheme;
  s->P.scheme = scheme;
  s->advection(rhs);
  s->P.scheme = keep;
}
// Scalar operators: phi [nc], phi_bnd [nb], grad_phi (3, nc) AoS.
void orc_advection_scalar(void* h, int scheme, const double* phi, const double* phi_bnd, const double* flux,
                          const double* gphi, double* rhs) {
  auto* s = static_cast<orc::Solver*>(h);
  std::memcpy(s->U_face.data(), flux, sizeof(double) * s->nf);
  s->advection_scalar(scheme, phi, phi_bnd, gphi, rhs);
}
void orc_viscous_scalar(void* h, const double* phi, double alpha, const double* nu_sgs, double prt, const double* gphi,
                        const double* phi_bnd, double* rhs) {
  auto* s = static_cast<orc::Solver*>(h);
  std::memcpy(s->nu_sgs.data(), nu_sgs, sizeof(double) * s->nc);
  s->viscous_scalar(phi, alpha, prt, gphi, phi_bnd, rhs);
}
void orc_viscous(void* h, const double* U, const double* nu_sgs, const double* gU, const double* U_bnd, double* rhs) {
  auto* s = static_cast<orc::Solver*>(h);
  std::memcpy(s->U.data(), U, sizeof(double) * 3 * s->nc);
  std::memcpy(s->nu_sgs.data(), nu_sgs, sizeof(double) * s->nc);
  std::memcpy(s->grad_U.data(), gU, sizeof(double) * 9 * s->nc);
  std::memcpy(s->U_bnd.data(), U_bnd, sizeof(double) * 3 * s->nb);
  s->viscous(rhs);
}
void orc_sgs(void* h, int model, const double* gU, const double* U, double dt_stab, double* nu) {
  auto* s = static_cast<orc::Solver*>(h);
  std::memcpy(s->grad_U.data(), gU, sizeof(double) * 9 * s->nc);
  std::memcpy(s->U.data(), U, sizeof(double) * 3 * s->nc);
  int keep = s->P.sgs_model;
  s->P.sgs_model = model;
  s->sgs_viscosity(dt_stab);
  s->P.sgs_model = keep;
  std::memcpy(nu, s->nu_sgs.data(), sizeof(double) * s->nc);
}
void orc_wall_model(void* h, const double* U, double* tau) {
  auto* s = static_cast<orc::Solver*>(h);
  std::memcpy(s->U.data(), U, sizeof(double) * 3 * s->nc);
  s->wall_model(0.0);
  std::memcpy(tau, s->tau_w.data(), sizeof(double) * 3 * s->nb);
}
double orc_amd_point(const double* alpha, const double* G, double c_amd) { return orc::amd_point(alpha, G, c_amd); }
// exact cell projection operators (src/numerics/mod_cell_projection.f90), u and v as (3, nc)
void orc_cp_divergence(void* h, const double* u, double* out) { static_cast<orc::Solver*>(h)->cp_divergence(u, out); }
void orc_cp_adjoint(void* h, const double* chi, double* v) { static_cast<orc::Solver*>(h)->cp_adjoint(chi, v); }
int orc_cp_project(void* h, double* u, const double* bconst, double tol, int max_it, int identity, int* n_it) {
  return static_cast<orc::Solver*>(h)->cp_project(u, bconst, tol, max_it, identity != 0, n_it);
}
void orc_set_nudging_profiles(void* h, int nt, int nz, const double* times, const double* z, const double* Up,
                              const double* Tp) {
  auto* s = static_cast<orc::Solver*>(h);
  s->nd_nt = nt; s->nd_nz = nz;
  s->nd_times.assign(times, times + nt);
  s->nd_z.assign(z, z + nz);
  s->nd_U.assign(Up, Up + 3 * (size_t)nz * nt);
  s->nd_T.assign(Tp, Tp + (size_t)nz * nt);
}
void orc_set_scalar_sources(void* h, int n, const dpm_scalar_source_t* src) {
  auto* s = static_cast<orc::Solver*>(h);
  s->srcs.clear();
  for (int i = 0; i < n; ++i) {
    orc::Solver::Src q;
    q.d = src[i];
    if (src[i].n_tag_points > 0 && src[i].tag_points) q.tags.assign(src[i].tag_points, src[i].tag_points + 3 * (size_t)src[i].n_tag_points);
    q.d.tag_points = nullptr;
    s->srcs.push_back(q);
  }
}
void orc_sample_points(void* h, int np, const double* xyz, double* payload, int* owner) {
  static_cast<orc::Solver*>(h)->sample_points(np, xyz, payload, owner);
}
void orc_kfactor_limited(const double* sf, const double* d_on, double min_cos, double* k) {
  orc::kfactor_limited(sf, d_on, min_cos, k);
}
void orc_wall_stress_newton(double u_par, double y_w, double nu, double* u_tau, double* tau) {
  bool capped;
  orc::wall_stress_newton(u_par, y_w, nu, *u_tau, *tau, capped);
}
// Plain PETSc-semantics CG on the handle's assembled Poisson operator.
int orc_poisson_solve(void* h, const double* rhs, double* x, double rtol, double atol, int maxit, int* its, double* res) {
  auto* s = static_cast<orc::Solver*>(h);
  return s->cg(rhs, x, rtol, atol, maxit, false, its, res);
}
void orc_poisson_matvec(void* h, const double* x, double* y) { static_cast<orc::Solver*>(h)->matvec(x, y); }
// Poisson operator as CSR (nnz first with null arrays, then filled).
int64_t orc_poisson_csr(void* h, int64_t* off, int* col, double* val) {
  auto* s = static_cast<orc::Solver*>(h);
  if (off) std::memcpy(off, s->A_off.data(), sizeof(int64_t) * s->A_off.size());
  if (col) std::memcpy(col, s->A_col.data(), sizeof(int) * s->A_col.size());
  if (val) std::memcpy(val, s->A_val.data(), sizeof(double) * s->A_val.size());
  return (int64_t)s->A_col.size();
}
void orc_record_poisson(void* h, int on) {
  auto* s = static_cast<orc::Solver*>(h);
  s->record = on != 0;
  s->rec_rhs.clear();
  s->rec_x0.clear();
  s->rec_atol.clear();
}
// k-th recorded system; returns the number recorded.
int orc_recorded_poisson(void* h, int k, double* rhs, double* x0, double* atol) {
  auto* s = static_cast<orc::Solver*>(h);
  if (k >= 0 && k < (int)s->rec_rhs.size()) {
    std::memcpy(rhs, s->rec_rhs[k].data(), sizeof(double) * s->nc);
    std::memcpy(x0, s->rec_x0[k].data(), sizeof(double) * s->nc);
    *atol = s->rec_atol[k];
  }
  return (int)s->rec_rhs.size();
}
}
