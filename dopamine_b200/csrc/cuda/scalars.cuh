// Temperature and passive-scalar transport: boundary values, face fluxes and the per-cell
// gather with the RK3W update.  Same structure as the momentum path (per-face fluxes, then a
// gather in ascending face order per cell, so no atomics and the reference's summation order).
#pragma once
#include "kernels.cuh"

namespace dpm {
namespace gpu {

// Boundary values of a cell scalar (src/bc/mod_bc.f90:489-588 apply_temperature_bc, :591-680
// apply_passive_scalar_bc).  kind 0 = temperature: inlet / fixed-temperature faces take bval,
// periodic faces the gc-weighted partner value, every other face the owner value extrapolated
// with the cell gradient g ([3][nc]).  kind 1 = passive scalar: periodic as above, else the
// face's mode (0 zero gradient, 1 Dirichlet bsval, 2 Neumann flux bsval with the face
// diffusivity alpha + nu_t / prt).  filt: -1 all faces, 0 non-periodic, 1 periodic.
__global__ void k_scalar_bc(Dev d, int kind, const double* __restrict__ phi, const double* __restrict__ g,
                            double* __restrict__ pb, int filt, const double* __restrict__ bval,
                            const int* __restrict__ bmode, const double* __restrict__ bsval, double alpha,
                            double prt, const double* __restrict__ nus) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.nb) return;
  const int nc = d.nc, nf = d.nf;
  const int f = d.nfi + b, bc = d.bbc[b];
  if (filt == 1 && bc != BC_PERIODIC) return;
  if (filt == 0 && bc == BC_PERIODIC) return;
  const int o = d.fo[f];
  double v;
  if (bc == BC_PERIODIC) {
    const int pn = d.bpnb[b];
    v = pn >= 0 ? d.bpgc[b] * phi[o] + (1.0 - d.bpgc[b]) * phi[pn] : phi[o];
  } else if (kind == 0) {
    if (bc == BC_INLET || bc == BC_FIXEDTEMP || (bc == BC_ABL_INLET && kind == 0)) {
      v = bval[b];
    } else {
      double d0 = d.fcen[f] - d.cen[o], d1 = d.fcen[nf + f] - d.cen[nc + o], d2 = d.fcen[2 * nf + f] - d.cen[2 * nc + o];
      v = phi[o] + g[o] * d0 + g[nc + o] * d1 + g[2 * nc + o] * d2;
    }
  } else {
    const int mode = bmode[b];
    if (mode == 1) {
      v = bsval[b];
    } else if (mode == 2) {
      const double a = alpha + nus[o] / prt;
      const double dd = fmax(d.dcf[f], SMALLD);
      v = a > SMALLD ? phi[o] + bsval[b] * dd / a : phi[o];
    } else {
      v = phi[o];
    }
  }
  pb[b] = v;
}

// Per-face advective flux Fn * phi_f (src/numerics/mod_advection.f90:267-675: CDS with the eps
// correction, QUICK, van Leer, Koren; Fn is the projected U_face, zero on walls) and diffusive
// flux (src/numerics/mod_viscous.f90:286-507: alpha_eff = alpha + nu_t / prt, clamped
// orthogonality weight, gc-mean gradient on the transverse part, Jasak split on boundaries).
__global__ void __launch_bounds__(TPB) k_face_scalar(Dev d, int scheme, const double* __restrict__ phi,
                                                     const double* __restrict__ pb, const double* __restrict__ g,
                                                     const double* __restrict__ nus, double alpha, double prt,
                                                     const double* __restrict__ Uface, double* __restrict__ fadv,
                                                     double* __restrict__ fdif) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= d.nf) return;
  const int nc = d.nc, nf = d.nf;
  const int o = d.fo[f], n = d.fn[f];
  const int b = f - d.nfi;
  const int bc = n >= 0 ? -1 : d.bbc[b];
  double Fn = (n < 0 && is_wall_bc(bc)) ? 0.0 : Uface[f];
  double ph;
  if (scheme == 3) {  // CDS
    int npr = -1;
    bool rec = n >= 0;
    if (!rec && bc == BC_PERIODIC) { npr = d.bpnb[b]; rec = npr >= 0; }
    if (rec) {
      const int ns = n >= 0 ? n : npr;
      const double w = f >= d.nfi ? d.bpgc[b] : d.gc[f];
      const double plain = w * phi[o] + (1.0 - w) * phi[ns];
      if (f < d.nfi) {
        double gm0 = w * g[o] + (1.0 - w) * g[ns];
        double gm1 = w * g[nc + o] + (1.0 - w) * g[nc + ns];
        double gm2 = w * g[2 * nc + o] + (1.0 - w) * g[2 * nc + ns];
        double pe = plain + (gm0 * d.eps[f] + gm1 * d.eps[nf + f] + gm2 * d.eps[2 * nf + f]);
        const double wb = d.wbl[f];
        if (wb < 1.0) pe = plain + wb * (pe - plain);
        ph = pe;
      } else {
        ph = plain;
      }
      if (!finite_d(ph)) ph = (Fn >= 0.0 || n < 0) ? phi[o] : phi[n];
    } else {
      ph = pb[b];
    }
  } else {  // QUICK (5), van Leer (1), Koren (2)
    ReconCtx ctx;
    const bool ok = recon_context_d(d, f, Fn, ctx);
    if (ok) {
      if (scheme == 5) quick_d<1>(d, ctx, phi, g, &ph);
      else ph = tvd_d(d, scheme, phi, ctx, far_upwind_d(d, ctx));
      if (!finite_d(ph)) ph = (Fn >= 0.0 || n < 0) ? phi[o] : phi[n];
    } else {
      ph = pb[b];
    }
  }
  if (!finite_d(Fn)) Fn = 0.0;
  if (!finite_d(ph)) ph = 0.0;
  fadv[f] = Fn * ph;

  // ---- diffusion (owner orientation)
  const double sf0 = d.sf[f], sf1 = d.sf[nf + f], sf2 = d.sf[2 * nf + f];
  const double area = d.area[f];
  auto pair_flux = [&](int nbc, double w, double aeff, const double* dn_, double dl) {
    const double sdd = (sf0 * dn_[0] + sf1 * dn_[1] + sf2 * dn_[2]) / dl;
    const double dp0 = sf0 - (sdd / dl) * dn_[0], dp1 = sf1 - (sdd / dl) * dn_[1], dp2 = sf2 - (sdd / dl) * dn_[2];
    const double wo = area * fmax(0.0, fmin(1.0, sdd / (area + SMALLD)));
    const double gf0 = w * g[o] + (1.0 - w) * g[nbc];
    const double gf1 = w * g[nc + o] + (1.0 - w) * g[nc + nbc];
    const double gf2 = w * g[2 * nc + o] + (1.0 - w) * g[2 * nc + nbc];
    const double dphi = (phi[nbc] - phi[o]) * wo / dl + (gf0 * dp0 + gf1 * dp1 + gf2 * dp2);
    return aeff * dphi;
  };
  auto bnd_flux = [&]() {
    const double aeff = alpha + nus[o] / prt;
    const double dn_[3] = {d.fcen[f] - d.cen[o], d.fcen[nf + f] - d.cen[nc + o], d.fcen[2 * nf + f] - d.cen[2 * nc + o]};
    const double dl = sqrt(dn_[0] * dn_[0] + dn_[1] * dn_[1] + dn_[2] * dn_[2]) + SMALLD;
    const double sdd = (sf0 * dn_[0] + sf1 * dn_[1] + sf2 * dn_[2]) / dl;
    const double dp0 = sf0 - (sdd / dl) * dn_[0], dp1 = sf1 - (sdd / dl) * dn_[1], dp2 = sf2 - (sdd / dl) * dn_[2];
    const double wo = area * fmax(0.0, fmin(1.0, sdd / (area + SMALLD)));
    const double dphi = (pb[b] - phi[o]) * wo / dl + (g[o] * dp0 + g[nc + o] * dp1 + g[2 * nc + o] * dp2);
    return aeff * dphi;
  };
  double flux;
  if (n >= 0) {
    const double w = d.gc[f];
    const double aeff = alpha + (w * nus[o] + (1.0 - w) * nus[n]) / prt;
    const double dn_[3] = {d.cen[n] - d.cen[o], d.cen[nc + n] - d.cen[nc + o], d.cen[2 * nc + n] - d.cen[2 * nc + o]};
    flux = pair_flux(n, w, aeff, dn_, sqrt(dn_[0] * dn_[0] + dn_[1] * dn_[1] + dn_[2] * dn_[2]) + SMALLD);
  } else if (bc == BC_PERIODIC && d.bpnb[b] >= 0) {
    const int npr = d.bpnb[b];
    const int pr = d.bpair[b];
    const int pf = pr >= 0 ? d.nfi + pr : -1;
    double dper, gcp;
    if (pf >= 0) { dper = d.dcf[f] + d.dcf[pf]; gcp = d.dcf[pf] / (dper + SMALLD); }
    else if (d.bpdcf[b] > SMALLD) { dper = d.dcf[f] + d.bpdcf[b]; gcp = d.bpdcf[b] / (dper + SMALLD); }
    else { dper = 2.0 * d.dcf[f]; gcp = 0.5; }
    const double aeff = alpha + (gcp * nus[o] + (1.0 - gcp) * nus[npr]) / prt;
    const double dn_[3] = {dper * d.nrm[f], dper * d.nrm[nf + f], dper * d.nrm[2 * nf + f]};
    flux = pair_flux(npr, gcp, aeff, dn_, dper + SMALLD);
  } else {
    flux = bnd_flux();
  }
  fdif[f] = flux;
}

// The same face fluxes for several fields at once (temperature and the passive scalars): the
// face geometry, the upwind context and the far-upwind search are formed once per face and
// shared; each field's arithmetic is that of k_face_scalar, expression for expression.
struct ScalarFaceSet {
  int n;
  int scheme[LS_SET];
  const double* phi[LS_SET];
  const double* pb[LS_SET];
  const double* g[LS_SET];
  double alpha[LS_SET], prt[LS_SET];
  double* fadv[LS_SET];
  double* fdif[LS_SET];
};
__global__ void __launch_bounds__(TPB) k_face_scalars(Dev d, ScalarFaceSet q, const double* __restrict__ nus,
                                                      const double* __restrict__ Uface) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= d.nf) return;
  const int nc = d.nc, nf = d.nf;
  const int o = d.fo[f], n = d.fn[f];
  const int b = f - d.nfi;
  const int bc = n >= 0 ? -1 : d.bbc[b];
  double Fn = (n < 0 && is_wall_bc(bc)) ? 0.0 : Uface[f];
  bool need_ctx = false, need_far = false, need_quick = false;
#pragma unroll
  for (int k = 0; k < LS_SET; ++k)
    if (k < q.n && q.scheme[k] != 3) {
      need_ctx = true;
      if (q.scheme[k] != 5) need_far = true;
      else need_quick = true;
    }
  ReconCtx ctx;
  bool ok = false;
  int far = -1, sg = 0, up = -1, down = -1;
  const bool pre = need_ctx && !need_quick && d.tvd_far;  // van Leer / Koren only: precomputed context
  if (pre) {
    sg = Fn >= 0.0 ? 0 : 1;
    far = d.tvd_far[sg * nf + f];
    ok = far != -2 && tvd_cells_d(d, f, sg, up, down);
  } else if (need_ctx) {
    ok = recon_context_d(d, f, Fn, ctx);
    if (ok && need_far) far = far_upwind_d(d, ctx);
  }
  // CDS interpolation partner and weight
  int npr = -1;
  bool rec = n >= 0;
  if (!rec && bc == BC_PERIODIC) { npr = d.bpnb[b]; rec = npr >= 0; }
  const int nsx = n >= 0 ? n : npr;
  const double wcds = f >= d.nfi ? (rec ? d.bpgc[b] : 0.0) : d.gc[f];
  // diffusion geometry (owner orientation)
  const double sf0 = d.sf[f], sf1 = d.sf[nf + f], sf2 = d.sf[2 * nf + f];
  const double area = d.area[f];
  int kind, nbc = -1;
  double w = 0.0, dn_[3], dl;
  if (n >= 0) {
    kind = 0;
    nbc = n;
    w = d.gc[f];
    dn_[0] = d.cen[n] - d.cen[o]; dn_[1] = d.cen[nc + n] - d.cen[nc + o]; dn_[2] = d.cen[2 * nc + n] - d.cen[2 * nc + o];
    dl = sqrt(dn_[0] * dn_[0] + dn_[1] * dn_[1] + dn_[2] * dn_[2]) + SMALLD;
  } else if (bc == BC_PERIODIC && d.bpnb[b] >= 0) {
    kind = 1;
    nbc = d.bpnb[b];
    const int pr = d.bpair[b];
    const int pf = pr >= 0 ? d.nfi + pr : -1;
    double dper;
    if (pf >= 0) { dper = d.dcf[f] + d.dcf[pf]; w = d.dcf[pf] / (dper + SMALLD); }
    else if (d.bpdcf[b] > SMALLD) { dper = d.dcf[f] + d.bpdcf[b]; w = d.bpdcf[b] / (dper + SMALLD); }
    else { dper = 2.0 * d.dcf[f]; w = 0.5; }
    dn_[0] = dper * d.nrm[f]; dn_[1] = dper * d.nrm[nf + f]; dn_[2] = dper * d.nrm[2 * nf + f];
    dl = dper + SMALLD;
  } else {
    kind = 2;
    dn_[0] = d.fcen[f] - d.cen[o]; dn_[1] = d.fcen[nf + f] - d.cen[nc + o]; dn_[2] = d.fcen[2 * nf + f] - d.cen[2 * nc + o];
    dl = sqrt(dn_[0] * dn_[0] + dn_[1] * dn_[1] + dn_[2] * dn_[2]) + SMALLD;
  }
  const double sdd = (sf0 * dn_[0] + sf1 * dn_[1] + sf2 * dn_[2]) / dl;
  const double dp0 = sf0 - (sdd / dl) * dn_[0], dp1 = sf1 - (sdd / dl) * dn_[1], dp2 = sf2 - (sdd / dl) * dn_[2];
  const double wo = area * fmax(0.0, fmin(1.0, sdd / (area + SMALLD)));
  const double nuf = kind == 2 ? nus[o] : (w * nus[o] + (1.0 - w) * nus[nbc]);
  const double Fc = finite_d(Fn) ? Fn : 0.0;
#pragma unroll
  for (int k = 0; k < LS_SET; ++k) {
    if (k >= q.n) break;
    const double* phi = q.phi[k];
    const double* g = q.g[k];
    double ph;
    if (q.scheme[k] == 3) {  // CDS
      if (rec) {
        const double plain = wcds * phi[o] + (1.0 - wcds) * phi[nsx];
        if (f < d.nfi) {
          double gm0 = wcds * g[o] + (1.0 - wcds) * g[nsx];
          double gm1 = wcds * g[nc + o] + (1.0 - wcds) * g[nc + nsx];
          double gm2 = wcds * g[2 * nc + o] + (1.0 - wcds) * g[2 * nc + nsx];
          double pe = plain + (gm0 * d.eps[f] + gm1 * d.eps[nf + f] + gm2 * d.eps[2 * nf + f]);
          const double wb = d.wbl[f];
          if (wb < 1.0) pe = plain + wb * (pe - plain);
          ph = pe;
        } else {
          ph = plain;
        }
        if (!finite_d(ph)) ph = (Fn >= 0.0 || n < 0) ? phi[o] : phi[n];
      } else {
        ph = q.pb[k][b];
      }
    } else if (ok) {  // QUICK (5), van Leer (1), Koren (2)
      if (q.scheme[k] == 5) quick_d<1>(d, ctx, phi, g, &ph);
      else ph = pre ? tvd_pre_d(d, q.scheme[k], phi, f, sg, up, down, far) : tvd_d(d, q.scheme[k], phi, ctx, far);
      if (!finite_d(ph)) ph = (Fn >= 0.0 || n < 0) ? phi[o] : phi[n];
    } else {
      ph = q.pb[k][b];
    }
    if (!finite_d(ph)) ph = 0.0;
    q.fadv[k][f] = Fc * ph;
    const double aeff = q.alpha[k] + nuf / q.prt[k];
    double dphi;
    if (kind == 2) {
      dphi = (q.pb[k][b] - phi[o]) * wo / dl + (g[o] * dp0 + g[nc + o] * dp1 + g[2 * nc + o] * dp2);
    } else {
      const double gf0 = w * g[o] + (1.0 - w) * g[nbc];
      const double gf1 = w * g[nc + o] + (1.0 - w) * g[nc + nbc];
      const double gf2 = w * g[2 * nc + o] + (1.0 - w) * g[2 * nc + nbc];
      dphi = (phi[nbc] - phi[o]) * wo / dl + (gf0 * dp0 + gf1 * dp1 + gf2 * dp2);
    }
    q.fdif[k][f] = aeff * dphi;
  }
}

// Per-cell gather: H = conv + diff in ascending face order, plus the MOST wall heat flux qw
// (kinematic, per area) of wall-model faces when qw is given (src/solver/mod_fv_solver.f90:
// 2279-2313); with predict, the RK3W update phi += dt (a_k H + b_k H0) in place (:1322-1350).
__global__ void __launch_bounds__(TPB) k_cell_scalar(Dev d, const double* __restrict__ fadv,
                                                     const double* __restrict__ fdif, double* __restrict__ H,
                                                     const double* __restrict__ H0, double* __restrict__ phi,
                                                     double* __restrict__ conv_out, double* __restrict__ dif_out,
                                                     double dt, double a_k, double b_k, int predict,
                                                     const double* __restrict__ qw) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.nc) return;
  const int nc = d.nc;
  const double iv = d.ivol[c];
  double cv = 0.0, vs = 0.0;
  for (int s = 0; s < d.S; ++s) {
    const int f = d.cf[s * nc + c];
    if (f == PADI) break;
    if (d.fo[f] == c) { cv -= fadv[f] * iv; vs += fdif[f] * iv; }
    else { cv += fadv[f] * iv; vs -= fdif[f] * iv; }
  }
  double h = cv + vs;
  if (qw)
    for (int s = 0; s < d.SB; ++s) {
      const int b = d.cbn[s * nc + c];
      if (b == PADI) break;
      if (d.bbc[b] == BC_WALL_MODEL) h = h + qw[b] * d.area[d.nfi + b] / d.vol[c];
    }
  H[c] = h;
  if (conv_out) conv_out[c] = cv;
  if (dif_out) dif_out[c] = vs;
  if (predict) phi[c] = phi[c] + dt * (a_k * h + b_k * H0[c]);
}

// ------------------------------------------------------------------------------------------
// MOST surface layer (src/abl/mod_abl_wall.f90, src/abl/mod_abl_profiles.f90:51-86): per
// wall-model face, u* and T* from the owner cell's tangential speed and temperature at its
// wall-normal distance, by relaxed Newton with a finite-difference Jacobian; wall stress
// -u*^2 t_hat, kinematic heat flux -u* T*, per-face Obukhov length carried to the next call.
__device__ __forceinline__ double most_psi_m_d(double z) {
  if (fabs(z) < 1.0e-6) return 0.0;
  if (z > 0.0) return -5.0 * z;
  const double x = pow(1.0 - 16.0 * z, 0.25);
  return 2.0 * log((1.0 + x) / 2.0) + log((1.0 + x * x) / 2.0) - 2.0 * atan(x) + 1.5707963267948966;
}
__device__ __forceinline__ double most_psi_h_d(double z) {
  if (fabs(z) < 1.0e-6) return 0.0;
  if (z > 0.0) return -5.0 * z;
  const double y = sqrt(1.0 - 16.0 * z);
  return 2.0 * log((1.0 + y) / 2.0);
}
constexpr double MOST_KAPPA_D = 0.41, MOST_G_D = 9.81, MOST_L_CLIP_D = 5000.0;
__device__ __forceinline__ double fsign_d(double a, double b) { return b >= 0.0 ? fabs(a) : -fabs(a); }
__device__ __forceinline__ double most_L_from_d(double us, double ts, double tref) {
  if (fabs(ts) > SMALLD) {
    double L = us * us * tref / (MOST_KAPPA_D * MOST_G_D * ts);
    L = fsign_d(fmax(fabs(L), 0.001), L);
    if (fabs(L) > MOST_L_CLIP_D) L = fsign_d(MOST_L_CLIP_D, L);
    return L;
  }
  return MOST_L_CLIP_D;
}
__device__ __forceinline__ void most_res_d(double us, double ts, double L, double up, double To, double Ts, double yw,
                                           double z0m, double z0h, double& Fu, double& FT) {
  double dm = log(yw / z0m) - most_psi_m_d(yw / L) + most_psi_m_d(z0m / L);
  double dh = log(yw / z0h) - most_psi_h_d(yw / L) + most_psi_h_d(z0h / L);
  if (fabs(dm) < SMALLD) dm = fsign_d(SMALLD, dm);
  if (fabs(dh) < SMALLD) dh = fsign_d(SMALLD, dh);
  Fu = us - MOST_KAPPA_D * up / dm;
  FT = ts - MOST_KAPPA_D * (To - Ts) / dh;
}
__global__ void k_most(Dev d, const double* __restrict__ U, const double* __restrict__ T, double* __restrict__ tau,
                       double* __restrict__ qw, double* __restrict__ Lb, double L_cfg, double Ts,
                       const double* __restrict__ bz0m, const double* __restrict__ bz0h) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.nb || d.bbc[b] != BC_WALL_MODEL) return;
  const double z0m = bz0m[b], z0h = bz0h[b];  // per-face roughness (patch value or the global one)
  const int nc = d.nc, nf = d.nf, nb = d.nb;
  const int f = d.nfi + b, o = d.fo[f];
  const double n0 = d.nrm[f], n1 = d.nrm[nf + f], n2 = d.nrm[2 * nf + f];
  const double yw = fabs((d.fcen[f] - d.cen[o]) * n0 + (d.fcen[nf + f] - d.cen[nc + o]) * n1 +
                         (d.fcen[2 * nf + f] - d.cen[2 * nc + o]) * n2) + SMALLD;
  const double u0 = U[o], u1 = U[nc + o], u2 = U[2 * nc + o];
  const double un = u0 * n0 + u1 * n1 + u2 * n2;
  double t0 = u0 - un * n0, t1 = u1 - un * n1, t2 = u2 - un * n2;
  const double up = sqrt(t0 * t0 + t1 * t1 + t2 * t2);
  if (up > SMALLD) { t0 /= up; t1 /= up; t2 /= up; }
  else { t0 = t1 = t2 = 0.0; }
  double Lg = Lb[b];
  if (fabs(Lg) < SMALLD) Lg = L_cfg;
  const double To = T[o], tref = To;
  double us = fmax(SMALLD, MOST_KAPPA_D * up / fmax(SMALLD, log(yw / z0m)));
  double ts = 0.1 * (To - Ts);
  double L = fabs(Lg) < SMALLD ? MOST_L_CLIP_D : Lg;
  for (int it = 1; it <= 20; ++it) {
    L = fsign_d(fmax(fabs(L), 0.001), L);
    if (fabs(L) > MOST_L_CLIP_D) L = fsign_d(MOST_L_CLIP_D, L);
    double Fu, FT, Fu_p, FT_p;
    most_res_d(us, ts, L, up, To, Ts, yw, z0m, z0h, Fu, FT);
    if (fabs(Fu) < 1.0e-8 && fabs(FT) < 1.0e-8) break;
    const double due = fmax(1.0e-6, 1.0e-6 * fabs(us)), dte = fmax(1.0e-6, 1.0e-6 * fabs(ts));
    most_res_d(us + due, ts, most_L_from_d(us + due, ts, tref), up, To, Ts, yw, z0m, z0h, Fu_p, FT_p);
    const double dFu_du = (Fu_p - Fu) / due, dFT_du = (FT_p - FT) / due;
    most_res_d(us, ts + dte, most_L_from_d(us, ts + dte, tref), up, To, Ts, yw, z0m, z0h, Fu_p, FT_p);
    const double dFu_dT = (Fu_p - Fu) / dte, dFT_dT = (FT_p - FT) / dte;
    const double den = dFu_du * dFT_dT - dFu_dT * dFT_du;
    if (fabs(den) < SMALLD) break;
    us = us + 0.5 * (-(dFT_dT * Fu - dFu_dT * FT) / den);
    ts = ts + 0.5 * (-(dFu_du * FT - dFT_du * Fu) / den);
    us = fmax(SMALLD, fmin(us, 0.5 * up));
    L = most_L_from_d(us, ts, tref);
  }
  Lb[b] = L;
  tau[b] = -us * us * t0;
  tau[nb + b] = -us * us * t1;
  tau[2 * nb + b] = -us * us * t2;
  qw[b] = -us * ts;
}

}  // namespace gpu
}  // namespace dpm
