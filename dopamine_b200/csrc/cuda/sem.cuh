// ABL inflow on the device: the synthetic-eddy method of src/abl/mod_sem_inflow.f90 (Jarrin
// tent eddies and the divergence-free eddies of Poletto et al.), feeding the BC_ABL_INLET faces.
//
// Set-up (frame of the inlet plane, eddy scales, seeding) runs once on the host; from then on the
// eddies live on the device: each stage derives every eddy's principal frame and intensities from
// the target stress at its height (k_sem_prepare), evaluates the fluctuation at every inlet face
// (k_sem_faces, one thread per face, every eddy in index order: the reference visits the same
// eddies through spatial bins) and removes the net inflow it adds (k_sem_finish); at the end of a
// step one thread convects the eddies and recycles, with the xorshift64 generator, those that
// left the box (k_sem_advance), so the random sequence is the reference's.
#pragma once

#include <cstdint>
#include <vector>

#include "common.cuh"

namespace dpm {
namespace gpu {

constexpr double SEM_SMALL = 1.0e-16;  // mod_sem_inflow.f90:16
constexpr double SEM_PI = 3.14159265358979323846;
constexpr int SEM_FACE_BLOCKS_MAX = 1024;

struct SemCfg {  // the ABLConfig fields the eddies read (src/abl/mod_abl_types.f90)
  double u_ref, z_ref, z0_m, wind_dir_deg, alpha, Iu_ref, Iv_ratio, Iw_ratio, rho_uw;
  int power_law;
};

struct SemState {  // SEMState (mod_abl_types.f90) with device arrays
  int dfsem, per1, per2, n;
  double n_in[3], x_inlet[3], t1[3], t2[3];
  double t1_min, t1_max, t2_min, t2_max, period1, period2, per1_lo, per2_lo;
  double sigma, rsup, box_volume, u_convect, lam_ref;
  unsigned long long rng;
  double *pos, *amp, *frame, *sig, *ampl;  // (3|9, n)
};

__host__ __device__ inline double sem_rand(unsigned long long& s) {  // :50-55
  s ^= s << 13;
  s ^= s >> 7;
  s ^= s << 17;
  return (double)(s & 4503599627370495ULL) / 4503599627370496.0;
}

__host__ __device__ inline double sem_ustar(double u_ref, double z_ref, double z0) {  // mod_abl_profiles.f90
  return (z_ref > z0 && z0 > 1.0e-30 && u_ref > 1.0e-30) ? 0.41 * u_ref / log(z_ref / z0) : 0.05 * u_ref;
}
__host__ __device__ inline double sem_log_u(double z, double u_star, double z0) {
  if (z <= z0 || u_star <= 1.0e-30 || z0 <= 1.0e-30) return 0.0;
  return (u_star / 0.41) * log(z / z0);
}

// sem_target_at (:663-711) without a table: the target stresses R = [uu,vv,ww,uv,uw,vw]
__host__ __device__ inline void sem_target(const SemCfg& c, double z, double R[6]) {
  const double zf = fmax(c.z0_m, 1.0e-6);
  const double us = sem_ustar(c.u_ref, c.z_ref, c.z0_m);
  for (int k = 0; k < 6; ++k) R[k] = 0.0;
  if (c.Iu_ref > 0.0) {
    const double zi = fmax(z, 10.0 * c.z0_m);
    const double Iu = c.Iu_ref * log(fmax(c.z_ref, 1.0001 * c.z0_m) / c.z0_m) / log(zi / c.z0_m);
    const double umag = c.power_law ? c.u_ref * pow(fmax(zi, zf) / fmax(c.z_ref, SEM_SMALL), c.alpha)
                                    : sem_log_u(zi, us, c.z0_m);
    const double su = Iu * umag, sv = c.Iv_ratio * su, sw = c.Iw_ratio * su;
    R[0] = su * su; R[1] = sv * sv; R[2] = sw * sw;
    R[4] = c.rho_uw * su * sw;
  } else {  // Panofsky & Dutton neutral surface layer
    R[0] = (2.4 * us) * (2.4 * us);
    R[1] = (1.9 * us) * (1.9 * us);
    R[2] = (1.25 * us) * (1.25 * us);
    R[4] = -(us * us);
  }
}
// sem_stress_at (:725-748): Rm and the frame axes Wr (row-major; columns e_s, e_n, e_z)
__host__ __device__ inline void sem_stress(const SemCfg& c, double z, double Rm[9], double Wr[9]) {
  double R[6];
  sem_target(c, z, R);
  Rm[0] = R[0]; Rm[4] = R[1]; Rm[8] = R[2];
  Rm[1] = R[3]; Rm[3] = R[3];
  Rm[2] = R[4]; Rm[6] = R[4];
  Rm[5] = R[5]; Rm[7] = R[5];
  const double w = c.wind_dir_deg * SEM_PI / 180.0;
  Wr[0] = -sin(w); Wr[1] = cos(w);  Wr[2] = 0.0;
  Wr[3] = -cos(w); Wr[4] = -sin(w); Wr[5] = 0.0;
  Wr[6] = 0.0;     Wr[7] = 0.0;     Wr[8] = 1.0;
}
// sem_eigen3 (:752-792): cyclic Jacobi; V row-major, its columns the eigenvectors
__host__ __device__ inline void sem_eigen3(const double Ain[9], double lam[3], double V[9]) {
  double A[9];
  for (int k = 0; k < 9; ++k) { A[k] = Ain[k]; V[k] = (k % 4 == 0) ? 1.0 : 0.0; }
  for (int sweep = 0; sweep < 30; ++sweep) {
    const double off = fabs(A[1]) + fabs(A[2]) + fabs(A[5]);
    if (off <= 1.0e-15 * (fabs(A[0]) + fabs(A[4]) + fabs(A[8]) + SEM_SMALL)) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        const double apq = A[3 * p + q];
        if (fabs(apq) <= SEM_SMALL) continue;
        const double th = (A[3 * q + q] - A[3 * p + p]) / (2.0 * apq);
        const double t = copysign(1.0, th) / (fabs(th) + sqrt(th * th + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), sn = t * c, tau = sn / (1.0 + c);
        A[3 * p + p] = A[3 * p + p] - t * apq;
        A[3 * q + q] = A[3 * q + q] + t * apq;
        A[3 * p + q] = 0.0; A[3 * q + p] = 0.0;
        for (int k = 0; k < 3; ++k) {
          if (k != p && k != q) {
            const double akp = A[3 * k + p], akq = A[3 * k + q];
            A[3 * k + p] = akp - sn * (akq + tau * akp); A[3 * p + k] = A[3 * k + p];
            A[3 * k + q] = akq + sn * (akp - tau * akq); A[3 * q + k] = A[3 * k + q];
          }
          const double vkp = V[3 * k + p], vkq = V[3 * k + q];
          V[3 * k + p] = vkp - sn * (vkq + tau * vkp);
          V[3 * k + q] = vkq + sn * (vkp - tau * vkq);
        }
      }
  }
  lam[0] = A[0]; lam[1] = A[4]; lam[2] = A[8];
}

// sem_place_eddy (:320-338)
__host__ __device__ inline void sem_place(SemState& s, double* pos, double* amp, int i, double sv, bool new_amp) {
  const double a = s.t1_min + (s.t1_max - s.t1_min) * sem_rand(s.rng);
  const double b = s.t2_min + (s.t2_max - s.t2_min) * sem_rand(s.rng);
  for (int k = 0; k < 3; ++k) pos[3 * i + k] = s.x_inlet[k] + sv * s.n_in[k] + a * s.t1[k] + b * s.t2[k];
  if (new_amp)
    for (int k = 0; k < 3; ++k) amp[3 * i + k] = copysign(1.0, sem_rand(s.rng) - 0.5);
}

// sem_prepare (:867-892): per eddy, the principal frame, half-extents and intensities
__global__ void k_sem_prepare(SemCfg c, SemState s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n || !s.dfsem) return;
  const double DF_I = 32.0 * SEM_PI / 945.0;
  double Rm[9], Wr[9], lam[3], V[9], sg[3];
  sem_stress(c, s.pos[3 * i + 2], Rm, Wr);
  sem_eigen3(Rm, lam, V);
  for (int j = 0; j < 3; ++j) {
    for (int r = 0; r < 3; ++r) {  // Vg = Wr V, column j
      double acc = 0.0;
      for (int k = 0; k < 3; ++k) acc = acc + Wr[3 * r + k] * V[3 * k + j];
      s.frame[9 * i + 3 * j + r] = acc;
    }
    sg[j] = s.sigma * fmax(0.2, sqrt(fmax(lam[j], 0.0) / s.lam_ref));
    s.sig[3 * i + j] = sg[j];
  }
  const double K = (double)s.n * sg[0] * sg[1] * sg[2] * DF_I / s.box_volume;
  double b[3], A[3];
  for (int j = 0; j < 3; ++j) b[j] = fmax(lam[j], 0.0) / (K * (sg[j] * sg[j]));
  A[0] = 0.5 * (b[1] + b[2] - b[0]);
  A[1] = 0.5 * (b[0] + b[2] - b[1]);
  A[2] = 0.5 * (b[0] + b[1] - b[2]);
  for (int j = 0; j < 3; ++j) s.ampl[3 * i + j] = sqrt(fmax(A[j], 0.0)) * s.amp[3 * i + j];
}

__device__ inline void sem_wrap(const SemState& s, double d[3]) {
  if (s.per1) {
    const double k = round((d[0] * s.t1[0] + d[1] * s.t1[1] + d[2] * s.t1[2]) / s.period1);
    for (int j = 0; j < 3; ++j) d[j] = d[j] - s.period1 * k * s.t1[j];
  }
  if (s.per2) {
    const double k = round((d[0] * s.t2[0] + d[1] * s.t2[1] + d[2] * s.t2[2]) / s.period2);
    for (int j = 0; j < 3; ++j) d[j] = d[j] - s.period2 * k * s.t2[j];
  }
}

// sem_velocity_at_face / sem_velocity_jarrin (:933-1039) at every ABL-inlet face; block partials
// of sum(u'.S_f) and sum(area) for the net-inflow removal
__global__ void __launch_bounds__(TPB) k_sem_faces(Dev d, SemCfg c, SemState s, int n_in_faces,
                                                   const int* __restrict__ faces, int look_ahead, double tau,
                                                   double* __restrict__ fluc, double* __restrict__ part) {
  const int nb = d.nb, nf = d.nf;
  double b1 = 0.0, b2 = 0.0;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n_in_faces; q += gridDim.x * blockDim.x) {
    const int b = faces[q], f = d.nfi + b;
    const double ctr[3] = {d.fcen[f], d.fcen[nf + f], d.fcen[2 * nf + f]};
    double xs[3], uf[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k < 3; ++k) xs[k] = look_ahead ? ctr[k] - s.u_convect * tau * s.n_in[k] : ctr[k];
    if (s.dfsem) {
      const double rs2 = s.rsup * s.rsup;
      for (int e = 0; e < s.n; ++e) {
        double dv[3];
        for (int k = 0; k < 3; ++k) dv[k] = xs[k] - s.pos[3 * e + k];
        sem_wrap(s, dv);
        if (dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2] >= rs2) continue;
        const double* fr = s.frame + 9 * e;
        const double* sg = s.sig + 3 * e;
        const double* al = s.ampl + 3 * e;
        double r[3], d2 = 0.0;
        for (int j = 0; j < 3; ++j) {
          r[j] = (dv[0] * fr[3 * j] + dv[1] * fr[3 * j + 1] + dv[2] * fr[3 * j + 2]) / sg[j];
          d2 = d2 + r[j] * r[j];
        }
        if (d2 >= 1.0) continue;
        const double g = 1.0 - d2;
        const double up0 = sg[0] * g * (r[1] * al[2] - r[2] * al[1]);
        const double up1 = sg[1] * g * (r[2] * al[0] - r[0] * al[2]);
        const double up2 = sg[2] * g * (r[0] * al[1] - r[1] * al[0]);
        for (int k = 0; k < 3; ++k) uf[k] = uf[k] + (up0 * fr[k] + up1 * fr[3 + k] + up2 * fr[6 + k]);
      }
    } else {
      double R[6];
      sem_target(c, ctr[2], R);
      const double w = c.wind_dir_deg * SEM_PI / 180.0;
      const double sgm = fmax(s.sigma, SEM_SMALL);
      const double norm = 1.5450968080927583 * sqrt(s.box_volume / (sgm * sgm * sgm)) / sqrt((double)s.n);
      double iso[3] = {0.0, 0.0, 0.0};
      for (int e = 0; e < s.n; ++e) {
        double dv[3];
        for (int k = 0; k < 3; ++k) dv[k] = xs[k] - s.pos[3 * e + k];
        sem_wrap(s, dv);
        if (fabs(dv[0]) >= sgm || fabs(dv[1]) >= sgm || fabs(dv[2]) >= sgm) continue;
        const double tent = fmax(0.0, 1.0 - sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]) / sgm);
        if (tent <= 0.0) continue;
        for (int k = 0; k < 3; ++k) iso[k] = iso[k] + norm * tent * s.amp[3 * e + k];
      }
      // sem_cholesky (:651-661) of the target stresses
      const double L11 = sqrt(fmax(R[0], SEM_SMALL)), L21 = R[3] / L11, L31 = R[4] / L11;
      const double L22 = sqrt(fmax(R[1] - L21 * L21, SEM_SMALL)), L32 = (R[5] - L31 * L21) / L22;
      const double L33 = sqrt(fmax(R[2] - L31 * L31 - L32 * L32, SEM_SMALL));
      const double a0 = L11 * iso[0], a1 = L21 * iso[0] + L22 * iso[1], a2 = L31 * iso[0] + L32 * iso[1] + L33 * iso[2];
      uf[0] = -a0 * sin(w) + a1 * cos(w);
      uf[1] = -a0 * cos(w) - a1 * sin(w);
      uf[2] = a2;
    }
    for (int k = 0; k < 3; ++k) fluc[k * nb + b] = uf[k];
    b1 = b1 + (uf[0] * d.sf[f] + uf[1] * d.sf[nf + f] + uf[2] * d.sf[2 * nf + f]);
    b2 = b2 + d.area[f];
  }
  __shared__ double sh[2][TPB / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int off = 16; off > 0; off >>= 1) {
    b1 += __shfl_down_sync(0xffffffffu, b1, off);
    b2 += __shfl_down_sync(0xffffffffu, b2, off);
  }
  if (lane == 0) { sh[0][wid] = b1; sh[1][wid] = b2; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t1 = 0.0, t2 = 0.0;
    for (int w = 0; w < TPB / 32; ++w) { t1 += sh[0][w]; t2 += sh[1][w]; }
    part[2 * blockIdx.x] = t1;
    part[2 * blockIdx.x + 1] = t2;
  }
}

// update_sem_inflow's tail (mod_fv_solver.f90:2106-2118): u' -= (sum u'.S / sum A) n_f
__global__ void __launch_bounds__(TPB) k_sem_finish(Dev d, int n_in_faces, const int* __restrict__ faces,
                                                    int nparts, const double* __restrict__ part,
                                                    double* __restrict__ fluc) {
  __shared__ double delta;
  if (threadIdx.x == 0) {
    double t1 = 0.0, t2 = 0.0;
    for (int j = 0; j < nparts; ++j) { t1 += part[2 * j]; t2 += part[2 * j + 1]; }
    delta = t2 <= 1.0e-30 ? 0.0 : t1 / t2;
  }
  __syncthreads();
  const int nb = d.nb, nf = d.nf;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n_in_faces; q += gridDim.x * blockDim.x) {
    const int b = faces[q], f = d.nfi + b;
    for (int k = 0; k < 3; ++k) fluc[k * nb + b] = fluc[k * nb + b] - delta * d.nrm[k * nf + f];
  }
}

// sem_advance (:341-358), one thread: convect along the inward normal, recycle what left the box
__global__ void k_sem_advance(SemState* st, double dt) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  SemState s = *st;
  const double disp = s.u_convect * dt;
  for (int i = 0; i < s.n; ++i) {
    for (int k = 0; k < 3; ++k) s.pos[3 * i + k] = s.pos[3 * i + k] + disp * s.n_in[k];
    const double dd = (s.pos[3 * i] - s.x_inlet[0]) * s.n_in[0] + (s.pos[3 * i + 1] - s.x_inlet[1]) * s.n_in[1] +
                      (s.pos[3 * i + 2] - s.x_inlet[2]) * s.n_in[2];
    if (dd > s.rsup) sem_place(s, s.pos, s.amp, i, -s.rsup, false);
  }
  st->rng = s.rng;
}

}  // namespace gpu
}  // namespace dpm
