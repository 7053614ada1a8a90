// The explicit half of the precision form (dpm_params_t.form = DPM_FORM_MIXED) in FP32.
//
// The north star's precision form keeps FP64 for the state, the outer defect-correction
// residual of the Poisson solve, the global CG reductions, the face mass-flux projection and the
// wall-model Newton update, and runs flux assembly, SGS and the inner Krylov iterations in FP32.
// Here: the first gradient pass of each stage (the one that feeds SGS and the explicit fluxes),
// the SGS closures, the momentum flux assembly with the RK3W right-hand side, and the scalar
// (temperature, passive scalars) face fluxes and gathers read FP32 copies of the static geometry
// and LS weights, hold their gradients in FP32 and compute in FP32.  Differences of the FP64 state
// (phi_nb - phi_c) are formed in FP64 and then rounded, so a field of large mean and small
// variations (a temperature near 300 K) keeps its relative resolution; sums, products and the
// gradient algebra are FP32.  The right-hand side H and the predictor U += dt (a H + b H0) are
// FP64.  The second gradient pass of a stage (it feeds the face mass flux of the projection and the
// boundary values) stays FP64.  Schemes: KEP, CDS, van Leer and Koren (the TVD schemes on the
// precomputed upwind context); QUICK is not provided in FP32.
//
// Each function restates, in single precision, the FP64 routine named beside it (kernels.cuh,
// scalars.cuh), which follows the reference routine cited there.
#pragma once
#include "kernels.cuh"
#include "scalars.cuh"

namespace dpm {
namespace gpu {

constexpr float SMALLF = 1.0e-30f;

// FP32 copies of the static geometry the explicit kernels read (null members when unused)
struct Geo32 {
  const float *vol, *ivol, *cen, *G, *ls_w;  // cells: [nc], [nc], [3][nc], [9][nc], [3][W][nc]
  const float *sf, *nrm, *fcen, *eps;        // faces [3][nf]
  const float *area, *gc, *wbl, *dcf;        // faces [nf]
  const float *bpgc, *bpdcf;                 // boundary faces [nb]
  const float *tvd_sf, *tvd_sd, *tvd_su;     // [2][nf]
};

__device__ __forceinline__ bool finite_f(float x) { return fabsf(x) <= 3.40282347e38f; }
__device__ __forceinline__ float clampv_f(float x, float lo, float hi) {
  const float l = fminf(lo, hi), h = fmaxf(lo, hi);
  return fminf(fmaxf(x, l), h);
}

// ---- least-squares gradients of U and NS scalars (k_ls_gradient_all)
struct LsScalarSet32 {
  int n;
  const double* phi[LS_SET];
  const double* pb[LS_SET];
  float* g[LS_SET];
};
constexpr int LS32_CHUNK = 2;  // stencil slots gathered together by k_ls32_gradient_all
template <int NS>
__global__ void __launch_bounds__(TPB) k_ls32_gradient_all(Dev d, Geo32 g, const double* __restrict__ U,
                                                           const double* __restrict__ Ub, float* __restrict__ gU,
                                                           LsScalarSet32 q) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.nc) return;
  const int nc = d.nc, nb = d.nb, W = d.W;
  const double uc0 = U[c], uc1 = U[nc + c], uc2 = U[2 * nc + c];
  float a[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  double pc[NS > 0 ? NS : 1];
  float a0[NS > 0 ? NS : 1], a1[NS > 0 ? NS : 1], a2[NS > 0 ? NS : 1];
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    pc[k] = q.phi[k][c];
    a0[k] = a1[k] = a2[k] = 0.0f;
  }
  // LS32_CHUNK slots at a time: all their loads are issued before the sums (slot order kept)
  constexpr int CH = LS32_CHUNK;
  for (int s0 = 0; s0 < W; s0 += CH) {
    int v[CH];
#pragma unroll
    for (int u = 0; u < CH; ++u) v[u] = s0 + u < W ? __ldg(&d.ls_idx[(s0 + u) * nc + c]) : PADI;
    if (v[0] == PADI) break;
    float w0[CH], w1[CH], w2[CH];
    double un0[CH], un1[CH], un2[CH], pv[CH][NS > 0 ? NS : 1];
#pragma unroll
    for (int u = 0; u < CH; ++u) {
      const int s = s0 + u;
      const bool on = v[u] != PADI;
      w0[u] = on ? __ldg(&g.ls_w[(0 * W + s) * nc + c]) : 0.0f;
      w1[u] = on ? __ldg(&g.ls_w[(1 * W + s) * nc + c]) : 0.0f;
      w2[u] = on ? __ldg(&g.ls_w[(2 * W + s) * nc + c]) : 0.0f;
      const int vv = v[u];
      if (vv >= 0) {
        un0[u] = U[vv]; un1[u] = U[nc + vv]; un2[u] = U[2 * nc + vv];
#pragma unroll
        for (int k = 0; k < NS; ++k) pv[u][k] = q.phi[k][vv];
      } else {
        const int b = on ? -vv - 1 : nb;  // a padding slot reads nothing
        if (b < nb) {
          un0[u] = Ub[b]; un1[u] = Ub[nb + b]; un2[u] = Ub[2 * nb + b];
#pragma unroll
          for (int k = 0; k < NS; ++k) pv[u][k] = q.pb[k][b];
        } else {
          un0[u] = uc0; un1[u] = uc1; un2[u] = uc2;
#pragma unroll
          for (int k = 0; k < NS; ++k) pv[u][k] = pc[k];
        }
      }
    }
#pragma unroll
    for (int u = 0; u < CH; ++u) {
      if (v[u] == PADI) break;
      const float du0 = (float)(un0[u] - uc0), du1 = (float)(un1[u] - uc1), du2 = (float)(un2[u] - uc2);
      a[0] = fmaf(w0[u], du0, a[0]); a[1] = fmaf(w1[u], du0, a[1]); a[2] = fmaf(w2[u], du0, a[2]);
      a[3] = fmaf(w0[u], du1, a[3]); a[4] = fmaf(w1[u], du1, a[4]); a[5] = fmaf(w2[u], du1, a[5]);
      a[6] = fmaf(w0[u], du2, a[6]); a[7] = fmaf(w1[u], du2, a[7]); a[8] = fmaf(w2[u], du2, a[8]);
#pragma unroll
      for (int k = 0; k < NS; ++k) {
        const float dd = (float)(pv[u][k] - pc[k]);
        a0[k] = fmaf(w0[u], dd, a0[k]);
        a1[k] = fmaf(w1[u], dd, a1[k]);
        a2[k] = fmaf(w2[u], dd, a2[k]);
      }
    }
  }
#pragma unroll
  for (int j = 0; j < 9; ++j) gU[j * nc + c] = a[j];
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    q.g[k][c] = a0[k];
    q.g[k][nc + c] = a1[k];
    q.g[k][2 * nc + c] = a2[k];
  }
}

// FP32 gradient into the FP64 array at the owner cells of outlet / zero-gradient boundary faces,
// the only places the boundary refresh after the predictor reads it (k_velocity_bc)
__global__ void k_grad32_to_bnd(Dev d, const float* __restrict__ gU32, double* __restrict__ gU) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.nb) return;
  const int bc = d.bbc[b];
  if (bc != BC_OUTLET && bc != BC_ZEROGRADIENT) return;
  const int o = d.fo[d.nfi + b], nc = d.nc;
#pragma unroll
  for (int j = 0; j < 9; ++j) gU[j * nc + o] = (double)gU32[j * nc + o];
}

// ---- SGS eddy viscosity (k_sgs): Vreman, Smagorinsky, AMD
__device__ __forceinline__ float amd_point_f(const float* a, const float* G, float c_amd) {
  float asq = 0.0f;
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) asq += a[i + 3 * j] * a[i + 3 * j];
  float num = 0.0f;
  for (int n = 0; n < 3; ++n)
    for (int m = 0; m < 3; ++m) {
      float beta = 0.0f;
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) beta += G[i + 3 * j] * a[i + 3 * m] * a[j + 3 * n];
      num -= beta * a[m + 3 * n];
    }
  const float trg = G[0] + G[4] + G[8];
  if (asq > 1.0e-20f && num > 1.0e-12f * trg * asq * sqrtf(asq)) return c_amd * num / asq;
  return 0.0f;
}
__device__ __forceinline__ float det3_f(const float* A) {
  return A[0] * (A[4] * A[8] - A[7] * A[5]) - A[3] * (A[1] * A[8] - A[7] * A[2]) + A[6] * (A[1] * A[5] - A[4] * A[2]);
}
__global__ void __launch_bounds__(TPB) k_sgs32(Dev d, Geo32 g, int model, const float* __restrict__ gU,
                                               double* __restrict__ nu, float dt_stab, float c_amd) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.nc) return;
  const int nc = d.nc;
  float a[9], G[9];
#pragma unroll
  for (int j = 0; j < 9; ++j) { a[j] = gU[j * nc + c]; G[j] = g.G[j * nc + c]; }
  float res = 0.0f;
  if (model == 1) {
    float beta[9];
    for (int j = 0; j < 3; ++j)
      for (int i = 0; i <= j; ++i) {
        float s = 0.0f;
        for (int n = 0; n < 3; ++n)
          for (int m = 0; m < 3; ++m) s += G[m + 3 * n] * a[m + 3 * i] * a[n + 3 * j];
        beta[i + 3 * j] = s;
      }
    const float asq = a[0] * a[0] + a[3] * a[3] + a[6] * a[6] + a[1] * a[1] + a[4] * a[4] + a[7] * a[7] +
                      a[2] * a[2] + a[5] * a[5] + a[8] * a[8];
    const float B = beta[0] * beta[4] - beta[3] * beta[3] + beta[0] * beta[8] - beta[6] * beta[6] +
                    beta[4] * beta[8] - beta[7] * beta[7];
    const float nuc = (asq > SMALLF && B > 0.0f) ? 0.025f * sqrtf(B / asq) : 0.0f;
    const float cap = 0.4f * powf(g.vol[c], 2.0f / 3.0f) / fmaxf(dt_stab, SMALLF);
    res = fminf(nuc, cap);
  } else if (model == 2) {
    float SS = 0.0f;
    for (int j = 0; j < 3; ++j)
      for (int i = 0; i < 3; ++i) {
        const float s = 0.5f * (a[i + 3 * j] + a[j + 3 * i]);
        SS += s * s;
      }
    const float Sn = sqrtf(2.0f * SS);
    const float delta = fmaxf(powf(fmaxf(det3_f(G), 0.0f), 1.0f / 6.0f), SMALLF);
    const float nuc = (0.1f * delta) * (0.1f * delta) * Sn;
    res = fminf(nuc, 0.4f * delta * delta / fmaxf(dt_stab, SMALLF));
  } else if (model == 3) {
    const float nuc = amd_point_f(a, G, c_amd);
    res = fminf(nuc, 0.4f * powf(g.vol[c], 2.0f / 3.0f) / fmaxf(dt_stab, SMALLF));
  }
  nu[c] = (double)res;
}
// AMD with the log-law gradient at wall-model cells (k_amd_wall): the Newton solve for u_tau in
// FP64 (wall_newton_d), the closure in FP32
__global__ void k_amd_wall32(Dev d, Geo32 g, const double* __restrict__ U, const float* __restrict__ gU,
                             double* nu_sgs, double nu, float c_amd, float dt_stab) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.nc) return;
  const int nc = d.nc, nf = d.nf;
  for (int s = 0; s < d.SB; ++s) {
    int b = d.cbn[s * nc + c];
    if (b == PADI) break;
    if (d.bbc[b] != BC_WALL_MODEL) continue;
    int f = d.nfi + b;
    double nr[3] = {-d.nrm[f], -d.nrm[nf + f], -d.nrm[2 * nf + f]};
    double dd[3] = {d.fcen[f] - d.cen[c], d.fcen[nf + f] - d.cen[nc + c], d.fcen[2 * nf + f] - d.cen[2 * nc + c]};
    double yw = fabs(dd[0] * nr[0] + dd[1] * nr[1] + dd[2] * nr[2]);
    double u[3] = {U[c], U[nc + c], U[2 * nc + c]};
    double un = u[0] * nr[0] + u[1] * nr[1] + u[2] * nr[2];
    double ut[3] = {u[0] - un * nr[0], u[1] - un * nr[1], u[2] - un * nr[2]};
    double utm = sqrt(ut[0] * ut[0] + ut[1] * ut[1] + ut[2] * ut[2]);
    if (utm <= 1.0e-14 || yw <= SMALLD) continue;
    double utau, tm;
    wall_newton_d(utm, yw, nu, utau, tm);
    const float gw = (float)(utau / (0.41 * yw));
    float a[9], G[9];
    for (int j = 0; j < 9; ++j) { a[j] = gU[j * nc + c]; G[j] = g.G[j * nc + c]; }
    float dold[3], dt_[3];
    const float nf3[3] = {(float)nr[0], (float)nr[1], (float)nr[2]};
    for (int j = 0; j < 3; ++j) dold[j] = nf3[0] * a[0 + 3 * j] + nf3[1] * a[1 + 3 * j] + nf3[2] * a[2 + 3 * j];
    const float dn = dold[0] * nf3[0] + dold[1] * nf3[1] + dold[2] * nf3[2];
    for (int j = 0; j < 3; ++j) dt_[j] = gw * (float)(ut[j] / utm) - (dold[j] - dn * nf3[j]);
    for (int j = 0; j < 3; ++j)
      for (int i = 0; i < 3; ++i) a[i + 3 * j] += nf3[i] * dt_[j];
    const float nuc = amd_point_f(a, G, c_amd);
    nu_sgs[c] = (double)fminf(nuc, 0.4f * powf(g.vol[c], 2.0f / 3.0f) / fmaxf(dt_stab, SMALLF));
  }
}

// ---- TVD face value on the precomputed context (tvd_pre_d): the limiter algebra in FP32, the
// face value added to the FP64 upwind value
__device__ __forceinline__ double tvd_pre_f(const Dev& d, const Geo32& g, int scheme, const double* phi, int f,
                                            int sg, int up, int down, int far) {
  const int nf = d.nf;
  const double pU = phi[up], pD = phi[down];
  const float sdn = (float)(pD - pU) / g.tvd_sd[sg * nf + f];
  float psi = 0.0f;
  if (far >= 0 && fabsf(sdn) > SMALLF) {
    const float r = ((float)(pU - phi[far]) / g.tvd_su[sg * nf + f]) / sdn;
    if (scheme == 1) {
      psi = (r + fabsf(r)) / (1.0f + fabsf(r));
      psi = fmaxf(0.0f, fminf(psi, 2.0f));
    } else {
      psi = fmaxf(0.0f, fminf(fminf(2.0f * r, (1.0f + 2.0f * r) / 3.0f), 2.0f));
    }
  }
  return clampv_d(pU + (double)(psi * sdn * g.tvd_sf[sg * nf + f]), fmin(pU, pD), fmax(pU, pD));
}

// ---- momentum face flux of face f (face_explicit_d): advective F phi_f and viscous stress
__device__ __forceinline__ void face_explicit_f(const Dev& d, const Geo32& g, int scheme, float nu,
                                                const double* __restrict__ U, const double* __restrict__ Ub,
                                                const float* __restrict__ gU, const double* __restrict__ nus,
                                                const double* __restrict__ Uface, int f, float* adv, float* vis,
                                                float& div) {
  div = 0.0f;
  const int nc = d.nc, nf = d.nf, nb = d.nb;
  const int o = d.fo[f], n = d.fn[f];
  const float sf0 = g.sf[f], sf1 = g.sf[nf + f], sf2 = g.sf[2 * nf + f];
  const int b = f - d.nfi;
  const int bc = n >= 0 ? -1 : d.bbc[b];
  float phi[3], Fn;
  // ---- advection
  if (scheme == 4) {  // KEP
    int npr = -1;
    if (n >= 0) {
      Fn = (float)Uface[f];
      for (int k = 0; k < 3; ++k) phi[k] = (float)(0.5 * (U[k * nc + o] + U[k * nc + n]));
    } else {
      double Ufv[3];
      if (bc == BC_PERIODIC) npr = d.bpnb[b];
      if (bc == BC_PERIODIC && npr >= 0) {
        const double w = (double)g.bpgc[b];
        for (int k = 0; k < 3; ++k) Ufv[k] = w * U[k * nc + o] + (1.0 - w) * U[k * nc + npr];
      } else {
        for (int k = 0; k < 3; ++k) Ufv[k] = Ub[k * nb + b];
      }
      if (bc == BC_PERIODIC || bc == BC_OUTLET) Fn = (float)Uface[f];
      else if (is_wall_bc(bc)) Fn = 0.0f;
      else Fn = (float)Ufv[0] * sf0 + (float)Ufv[1] * sf1 + (float)Ufv[2] * sf2;
      for (int k = 0; k < 3; ++k) phi[k] = (float)(npr >= 0 ? 0.5 * (U[k * nc + o] + U[k * nc + npr]) : Ufv[k]);
    }
    div = Fn;
  } else if (scheme == 3) {  // CDS
    int npr = -1;
    if (n >= 0) Fn = (float)Uface[f];
    else if (bc == BC_PERIODIC || bc == BC_OUTLET) Fn = (float)Uface[f];
    else if (is_wall_bc(bc)) Fn = 0.0f;
    else Fn = (float)Ub[b] * sf0 + (float)Ub[nb + b] * sf1 + (float)Ub[2 * nb + b] * sf2;
    bool rec = n >= 0;
    if (!rec && bc == BC_PERIODIC) { npr = d.bpnb[b]; rec = npr >= 0; }
    const int ns = rec ? (n >= 0 ? n : npr) : -1;
    for (int k = 0; k < 3; ++k) {
      float ph;
      if (rec) {
        const float gw = f >= d.nfi ? g.bpgc[b] : g.gc[f];
        const float plain = (float)(gw * U[k * nc + o] + (1.0 - gw) * U[k * nc + ns]);
        if (f < d.nfi) {
          const float gm0 = gw * gU[(3 * k + 0) * nc + o] + (1.0f - gw) * gU[(3 * k + 0) * nc + ns];
          const float gm1 = gw * gU[(3 * k + 1) * nc + o] + (1.0f - gw) * gU[(3 * k + 1) * nc + ns];
          const float gm2 = gw * gU[(3 * k + 2) * nc + o] + (1.0f - gw) * gU[(3 * k + 2) * nc + ns];
          float pe = plain + (gm0 * g.eps[f] + gm1 * g.eps[nf + f] + gm2 * g.eps[2 * nf + f]);
          const float wb = g.wbl[f];
          if (wb < 1.0f) pe = plain + wb * (pe - plain);
          ph = pe;
        } else {
          ph = plain;
        }
      } else {
        ph = (float)Ub[k * nb + b];
      }
      if (!finite_f(ph)) ph = 0.0f;
      phi[k] = ph;
    }
  } else {  // van Leer (1), Koren (2) on the precomputed context
    if (n >= 0) Fn = (float)Uface[f];
    else Fn = is_wall_bc(bc) ? 0.0f : (float)Uface[f];
    const int sg = Fn >= 0.0f ? 0 : 1;
    int up = -1, down = -1;
    const int far = d.tvd_far[sg * nf + f];
    const bool ok = far != -2 && tvd_cells_d(d, f, sg, up, down);
    if (!finite_f(Fn)) Fn = 0.0f;
    for (int k = 0; k < 3; ++k) {
      float ph;
      if (ok) {
        double pd = tvd_pre_f(d, g, scheme, U + (size_t)k * nc, f, sg, up, down, far);
        if (!finite_d(pd)) pd = (Fn >= 0.0f || n < 0) ? U[k * nc + o] : U[k * nc + n];
        ph = (float)pd;
      } else {
        ph = (float)Ub[k * nb + b];
      }
      if (!finite_f(ph)) ph = 0.0f;
      phi[k] = ph;
    }
  }
  for (int k = 0; k < 3; ++k) adv[k] = Fn * phi[k];

  // ---- viscous stress (owner orientation)
  float st[3] = {0, 0, 0};
  const float area = g.area[f];
  auto stress = [&](int nbc, float gw, float nu_eff, const float* dn_, float dl) {
    const float sdd = (sf0 * dn_[0] + sf1 * dn_[1] + sf2 * dn_[2]) / dl;
    const float dp0 = sf0 - (sdd / dl) * dn_[0], dp1 = sf1 - (sdd / dl) * dn_[1], dp2 = sf2 - (sdd / dl) * dn_[2];
    const float wo = area * fmaxf(0.0f, fminf(1.0f, sdd / (area + SMALLF)));
    float gf[9];
    for (int j = 0; j < 9; ++j) gf[j] = gw * gU[j * nc + o] + (1.0f - gw) * gU[j * nc + nbc];
    for (int k = 0; k < 3; ++k) {
      const float t1 = (float)(U[k * nc + nbc] - U[k * nc + o]) * wo / dl;
      const float t2 = gf[3 * k + 0] * dp0 + gf[3 * k + 1] * dp1 + gf[3 * k + 2] * dp2;
      const float t3 = gf[k] * sf0 + gf[3 + k] * sf1 + gf[6 + k] * sf2;
      st[k] = nu_eff * (t1 + t2 + t3);
    }
  };
  if (n >= 0) {
    const float gw = g.gc[f];
    const float ne = nu + gw * (float)nus[o] + (1.0f - gw) * (float)nus[n];
    const float dn_[3] = {g.cen[n] - g.cen[o], g.cen[nc + n] - g.cen[nc + o], g.cen[2 * nc + n] - g.cen[2 * nc + o]};
    const float dl = sqrtf(dn_[0] * dn_[0] + dn_[1] * dn_[1] + dn_[2] * dn_[2]) + SMALLF;
    stress(n, gw, ne, dn_, dl);
  } else if (bc == BC_PERIODIC) {
    const int npr = d.bpnb[b];
    const int pb = d.bpair[b];
    const int pf = pb >= 0 ? d.nfi + pb : -1;
    if (npr >= 0) {
      float dper, gcp;
      if (pf >= 0) { dper = g.dcf[f] + g.dcf[pf]; gcp = g.dcf[pf] / (dper + SMALLF); }
      else if (g.bpdcf[b] > SMALLF) { dper = g.dcf[f] + g.bpdcf[b]; gcp = g.bpdcf[b] / (dper + SMALLF); }
      else { dper = 2.0f * g.dcf[f]; gcp = 0.5f; }
      const float ne = nu + gcp * (float)nus[o] + (1.0f - gcp) * (float)nus[npr];
      const float dn_[3] = {dper * g.nrm[f], dper * g.nrm[nf + f], dper * g.nrm[2 * nf + f]};
      stress(npr, gcp, ne, dn_, dper + SMALLF);
    } else {
      const float ne = nu + (float)nus[o];
      for (int k = 0; k < 3; ++k) st[k] = ne * ((float)(Ub[k * nb + b] - U[k * nc + o]) / (g.dcf[f] + SMALLF)) * area;
    }
  } else if (bc != BC_WALL_MODEL) {
    const float ne = nu + (float)nus[o];
    const float dn_[3] = {g.fcen[f] - g.cen[o], g.fcen[nf + f] - g.cen[nc + o], g.fcen[2 * nf + f] - g.cen[2 * nc + o]};
    const float dl = sqrtf(dn_[0] * dn_[0] + dn_[1] * dn_[1] + dn_[2] * dn_[2]) + SMALLF;
    const float sdd = (sf0 * dn_[0] + sf1 * dn_[1] + sf2 * dn_[2]) / dl;
    const float dp0 = sf0 - (sdd / dl) * dn_[0], dp1 = sf1 - (sdd / dl) * dn_[1], dp2 = sf2 - (sdd / dl) * dn_[2];
    const float wo = area * fmaxf(0.0f, fminf(1.0f, sdd / (area + SMALLF)));
    for (int k = 0; k < 3; ++k) {
      const float t1 = (float)(Ub[k * nb + b] - U[k * nc + o]) * wo / dl;
      const float t2 = gU[(3 * k + 0) * nc + o] * dp0 + gU[(3 * k + 1) * nc + o] * dp1 + gU[(3 * k + 2) * nc + o] * dp2;
      const float t3 = gU[k * nc + o] * sf0 + gU[(3 + k) * nc + o] * sf1 + gU[(6 + k) * nc + o] * sf2;
      st[k] = ne * (t1 + t2 + t3);
    }
  }
  for (int k = 0; k < 3; ++k) vis[k] = st[k];
}

// ---- cell-owned momentum right-hand side and predictor (k_cell_momentum): face sums in FP32 in
// ascending face order, H and the update in FP64, the prediction into Unew
__global__ void __launch_bounds__(TPB) k_cell_momentum32(Dev d, Geo32 g, ExplicitArgs a, float nu,
                                                         const double* __restrict__ U, const double* __restrict__ Ub,
                                                         const float* __restrict__ gU, const double* __restrict__ nus,
                                                         const double* __restrict__ Uface, const double* __restrict__ T,
                                                         const double* __restrict__ tau, double* __restrict__ H,
                                                         const double* __restrict__ H0, double* __restrict__ Unew) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.nc) return;
  const int nc = d.nc, nb = d.nb;
  const float iv = g.ivol[c];
  float cv[3] = {0, 0, 0}, vs[3] = {0, 0, 0}, dv = 0.0f;
  for (int s = 0; s < d.S; ++s) {
    int f = d.cf[s * nc + c];
    if (f == PADI) break;
    float adv[3], vis[3], div;
    face_explicit_f(d, g, a.scheme, nu, U, Ub, gU, nus, Uface, f, adv, vis, div);
    const bool own = d.fo[f] == c;
    for (int k = 0; k < 3; ++k) {
      if (own) { cv[k] -= adv[k] * iv; vs[k] += vis[k] * iv; }
      else { cv[k] += adv[k] * iv; vs[k] -= vis[k] * iv; }
    }
    if (a.scheme == 4) dv = own ? dv + div : dv - div;
  }
  const double u[3] = {U[c], U[nc + c], U[2 * nc + c]};
  if (a.scheme == 4)
    for (int k = 0; k < 3; ++k) cv[k] += 0.5f * (float)u[k] * dv * iv;
  const double fb[3] = {a.f0, a.f1, a.f2}, gv[3] = {a.g0, a.g1, a.g2};
  double h[3];
  for (int k = 0; k < 3; ++k) h[k] = (double)(cv[k] + vs[k]) + fb[k];
  if (a.rot) {  // Coriolis, -2 Omega x U (mod_fv_solver.f90:1688-1692)
    h[0] = h[0] - 2.0 * (a.om1 * u[2] - a.om2 * u[1]);
    h[1] = h[1] - 2.0 * (a.om2 * u[0] - a.om0 * u[2]);
    h[2] = h[2] - 2.0 * (a.om0 * u[1] - a.om1 * u[0]);
  }
  if (a.bous)
    for (int k = 0; k < 3; ++k) h[k] = h[k] - a.beta * (T[c] - a.T_ref) * gv[k];
  for (int s = 0; s < d.SB; ++s) {
    int b = d.cbn[s * nc + c];
    if (b == PADI) break;
    if (d.bbc[b] != BC_WALL_MODEL) continue;
    double w = d.area[d.nfi + b] / d.vol[c];
    for (int k = 0; k < 3; ++k) h[k] = h[k] + tau[k * nb + b] * w;
  }
  for (int k = 0; k < 3; ++k) {
    H[k * nc + c] = h[k];
    Unew[k * nc + c] = u[k] + a.dt * (a.a_k * h[k] + a.b_k * H0[k * nc + c]);
  }
}

// ---- scalar face fluxes (k_face_scalars): CDS and the TVD schemes, FP32 face values and fluxes
struct ScalarFaceSet32 {
  int n;
  int scheme[LS_SET];
  const double* phi[LS_SET];
  const double* pb[LS_SET];
  const float* g[LS_SET];
  float alpha[LS_SET], prt[LS_SET];
  float* fadv[LS_SET];
  float* fdif[LS_SET];
};
__global__ void __launch_bounds__(TPB) k_face_scalars32(Dev d, Geo32 gg, ScalarFaceSet32 q, const double* __restrict__ nus,
                                                        const double* __restrict__ Uface) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= d.nf) return;
  const int nc = d.nc, nf = d.nf;
  const int o = d.fo[f], n = d.fn[f];
  const int b = f - d.nfi;
  const int bc = n >= 0 ? -1 : d.bbc[b];
  const double Fnd = (n < 0 && is_wall_bc(bc)) ? 0.0 : Uface[f];
  bool need_ctx = false;
#pragma unroll
  for (int k = 0; k < LS_SET; ++k)
    if (k < q.n && q.scheme[k] != 3) need_ctx = true;
  int far = -1, sg = 0, up = -1, down = -1;
  bool ok = false;
  if (need_ctx) {
    sg = Fnd >= 0.0 ? 0 : 1;
    far = d.tvd_far[sg * nf + f];
    ok = far != -2 && tvd_cells_d(d, f, sg, up, down);
  }
  int npr = -1;
  bool rec = n >= 0;
  if (!rec && bc == BC_PERIODIC) { npr = d.bpnb[b]; rec = npr >= 0; }
  const int nsx = n >= 0 ? n : npr;
  const float wcds = f >= d.nfi ? (rec ? gg.bpgc[b] : 0.0f) : gg.gc[f];
  const float sf0 = gg.sf[f], sf1 = gg.sf[nf + f], sf2 = gg.sf[2 * nf + f];
  const float area = gg.area[f];
  int kind, nbc = -1;
  float w = 0.0f, dn_[3], dl;
  if (n >= 0) {
    kind = 0;
    nbc = n;
    w = gg.gc[f];
    dn_[0] = gg.cen[n] - gg.cen[o]; dn_[1] = gg.cen[nc + n] - gg.cen[nc + o]; dn_[2] = gg.cen[2 * nc + n] - gg.cen[2 * nc + o];
    dl = sqrtf(dn_[0] * dn_[0] + dn_[1] * dn_[1] + dn_[2] * dn_[2]) + SMALLF;
  } else if (bc == BC_PERIODIC && d.bpnb[b] >= 0) {
    kind = 1;
    nbc = d.bpnb[b];
    const int pr = d.bpair[b];
    const int pf = pr >= 0 ? d.nfi + pr : -1;
    float dper;
    if (pf >= 0) { dper = gg.dcf[f] + gg.dcf[pf]; w = gg.dcf[pf] / (dper + SMALLF); }
    else if (gg.bpdcf[b] > SMALLF) { dper = gg.dcf[f] + gg.bpdcf[b]; w = gg.bpdcf[b] / (dper + SMALLF); }
    else { dper = 2.0f * gg.dcf[f]; w = 0.5f; }
    dn_[0] = dper * gg.nrm[f]; dn_[1] = dper * gg.nrm[nf + f]; dn_[2] = dper * gg.nrm[2 * nf + f];
    dl = dper + SMALLF;
  } else {
    kind = 2;
    dn_[0] = gg.fcen[f] - gg.cen[o]; dn_[1] = gg.fcen[nf + f] - gg.cen[nc + o]; dn_[2] = gg.fcen[2 * nf + f] - gg.cen[2 * nc + o];
    dl = sqrtf(dn_[0] * dn_[0] + dn_[1] * dn_[1] + dn_[2] * dn_[2]) + SMALLF;
  }
  const float sdd = (sf0 * dn_[0] + sf1 * dn_[1] + sf2 * dn_[2]) / dl;
  const float dp0 = sf0 - (sdd / dl) * dn_[0], dp1 = sf1 - (sdd / dl) * dn_[1], dp2 = sf2 - (sdd / dl) * dn_[2];
  const float wo = area * fmaxf(0.0f, fminf(1.0f, sdd / (area + SMALLF)));
  const float nuf = kind == 2 ? (float)nus[o] : (w * (float)nus[o] + (1.0f - w) * (float)nus[nbc]);
  const float Fc = finite_d(Fnd) ? (float)Fnd : 0.0f;
#pragma unroll
  for (int k = 0; k < LS_SET; ++k) {
    if (k >= q.n) break;
    const double* phi = q.phi[k];
    const float* g = q.g[k];
    double ph;
    if (q.scheme[k] == 3) {  // CDS
      if (rec) {
        const double plain = (double)wcds * phi[o] + (1.0 - (double)wcds) * phi[nsx];
        if (f < d.nfi) {
          const float gm0 = wcds * g[o] + (1.0f - wcds) * g[nsx];
          const float gm1 = wcds * g[nc + o] + (1.0f - wcds) * g[nc + nsx];
          const float gm2 = wcds * g[2 * nc + o] + (1.0f - wcds) * g[2 * nc + nsx];
          float corr = gm0 * gg.eps[f] + gm1 * gg.eps[nf + f] + gm2 * gg.eps[2 * nf + f];
          const float wb = gg.wbl[f];
          if (wb < 1.0f) corr = wb * corr;
          ph = plain + (double)corr;
        } else {
          ph = plain;
        }
        if (!finite_d(ph)) ph = (Fnd >= 0.0 || n < 0) ? phi[o] : phi[n];
      } else {
        ph = q.pb[k][b];
      }
    } else if (ok) {  // van Leer (1), Koren (2)
      ph = tvd_pre_f(d, gg, q.scheme[k], phi, f, sg, up, down, far);
      if (!finite_d(ph)) ph = (Fnd >= 0.0 || n < 0) ? phi[o] : phi[n];
    } else {
      ph = q.pb[k][b];
    }
    if (!finite_d(ph)) ph = 0.0;
    q.fadv[k][f] = Fc * (float)ph;
    const float aeff = q.alpha[k] + nuf / q.prt[k];
    float dphi;
    if (kind == 2) {
      dphi = (float)(q.pb[k][b] - phi[o]) * wo / dl + (g[o] * dp0 + g[nc + o] * dp1 + g[2 * nc + o] * dp2);
    } else {
      const float gf0 = w * g[o] + (1.0f - w) * g[nbc];
      const float gf1 = w * g[nc + o] + (1.0f - w) * g[nc + nbc];
      const float gf2 = w * g[2 * nc + o] + (1.0f - w) * g[2 * nc + nbc];
      dphi = (float)(phi[nbc] - phi[o]) * wo / dl + (gf0 * dp0 + gf1 * dp1 + gf2 * dp2);
    }
    q.fdif[k][f] = aeff * dphi;
  }
}
// per-cell gather of the FP32 scalar face fluxes (k_cell_scalar): sums in FP32 in ascending face
// order, + the MOST wall heat flux, H and the RK3W update in FP64
__global__ void __launch_bounds__(TPB) k_cell_scalar32(Dev d, Geo32 g, const float* __restrict__ fadv,
                                                       const float* __restrict__ fdif, double* __restrict__ H,
                                                       const double* __restrict__ H0, double* __restrict__ phi,
                                                       double dt, double a_k, double b_k,
                                                       const double* __restrict__ qw) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.nc) return;
  const int nc = d.nc;
  const float iv = g.ivol[c];
  float cv = 0.0f, vs = 0.0f;
  for (int s = 0; s < d.S; ++s) {
    const int f = d.cf[s * nc + c];
    if (f == PADI) break;
    if (d.fo[f] == c) { cv -= fadv[f] * iv; vs += fdif[f] * iv; }
    else { cv += fadv[f] * iv; vs -= fdif[f] * iv; }
  }
  double h = (double)(cv + vs);
  if (qw)
    for (int s = 0; s < d.SB; ++s) {
      const int b = d.cbn[s * nc + c];
      if (b == PADI) break;
      if (d.bbc[b] == BC_WALL_MODEL) h = h + qw[b] * d.area[d.nfi + b] / d.vol[c];
    }
  H[c] = h;
  phi[c] = phi[c] + dt * (a_k * h + b_k * H0[c]);
}

__global__ void k_to_f32(int64_t n, const double* __restrict__ in, float* __restrict__ out) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (float)in[i];
}

}  // namespace gpu
}  // namespace dpm
