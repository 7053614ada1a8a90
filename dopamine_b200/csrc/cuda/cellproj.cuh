// Exact cell projection (src/numerics/mod_cell_projection.f90, driven by
// src/solver/mod_fv_solver.f90:3223-3283 project_cells_exact): the cell velocity is projected
// V-orthogonally onto zero divergence of its gc-interpolated face flux,
//
//   u <- u - V^-1 B^T chi,   (B V^-1 B^T) chi = B u + bconst,
//
// B the outflow divergence over the pressure faces (interior faces and one face per periodic pair)
// plus the outlet faces.  The reference scatters per face with atomics; here each operator is a
// per-cell gather over the cell's pressure-face list, whose entries are in face order, so a cell
// accumulates its terms in the order the reference's face loop adds them.  Reductions are block
// partials over a fixed grid folded by one block in a fixed order (run to run deterministic); the
// Krylov scalars live on the device and the host reads one stop flag per iteration.
#pragma once

#include "common.cuh"

namespace dpm {
namespace gpu {

constexpr int CP_RED_BLOCKS = 1184;  // 8 blocks per SM on 148 SMs
constexpr int CP_NPART = 2;

// Device-resident scalars of the flexible CG (mod_cell_projection.f90:201-205).
struct CpState {
  double bn, rz, pq, alpha, en_new, en_tot, rn, beta;
  int stop;   // 0 running, 1 |pq| <= tiny, 2 converged, 3 right-hand side below tiny
  int it;
};

__device__ __forceinline__ double cp_dbl_min() { return 2.2250738585072014e-308; }  // tiny(1.0_rp)

// outflow divergence of u (SoA [3][nc]) at cell c (cp_divergence, :84-127)
__device__ __forceinline__ double cp_div_cell(const Dev& d, const double* __restrict__ u, int c) {
  const int nc = d.nc, nf = d.nf, nb = d.nb;
  double out = 0.0;
  for (int s = 0; s < d.SP; ++s) {
    int e = d.cps[s * nc + c];
    if (e == PADI) break;
    int i = e >= 0 ? e : ~e;
    int o = d.pso[i], n = d.psn[i], fm = d.psf[i];
    double w = d.psgcf[i];
    double fl = (w * u[o] + (1.0 - w) * u[n]) * d.sf[fm] + (w * u[nc + o] + (1.0 - w) * u[nc + n]) * d.sf[nf + fm] +
                (w * u[2 * nc + o] + (1.0 - w) * u[2 * nc + n]) * d.sf[2 * nf + fm];
    out = e >= 0 ? out + fl : out - fl;
  }
  for (int s = 0; s < d.SB; ++s) {
    int b = d.cbn[s * nc + c];
    if (b == PADI) break;
    if (d.bbc[b] != BC_OUTLET) continue;
    int f = d.nfi + b;
    out = out + (u[c] * d.sf[f] + u[nc + c] * d.sf[nf + f] + u[2 * nc + c] * d.sf[2 * nf + f]);
  }
  (void)nb;
  return out;
}

// block reduction of NV values (sums, or maxima where mx[k]) into part[blockIdx.x * CP_NPART + k]
template <int NV>
__device__ __forceinline__ void cp_block_partials(double (&v)[NV], const bool (&mx)[NV], double* __restrict__ part) {
  __shared__ double sh[TPB / 32][NV];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int k = 0; k < NV; ++k) {
    double t = v[k];
    for (int off = 16; off > 0; off >>= 1) {
      double o = __shfl_down_sync(0xffffffffu, t, off);
      t = mx[k] ? fmax(t, o) : t + o;
    }
    if (lane == 0) sh[wid][k] = t;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    const int k = threadIdx.x;
    double t = sh[0][k];
    for (int w = 1; w < TPB / 32; ++w) t = mx[k] ? fmax(t, sh[w][k]) : t + sh[w][k];
    part[blockIdx.x * CP_NPART + k] = t;
  }
}

// fold of the partials by one block of 32 threads: lane-strided, then a fixed shuffle tree
__device__ __forceinline__ double cp_fold(const double* __restrict__ part, int nparts, int k, bool mx) {
  double t = 0.0;
  for (int j = threadIdx.x; j < nparts; j += 32) t = mx ? fmax(t, part[j * CP_NPART + k]) : t + part[j * CP_NPART + k];
  for (int off = 16; off > 0; off >>= 1) {
    double o = __shfl_down_sync(0xffffffffu, t, off);
    t = mx ? fmax(t, o) : t + o;
  }
  return __shfl_sync(0xffffffffu, t, 0);
}

// project_cells_exact's boundary loop (mod_fv_solver.f90:3244-3270): the outlet pressure pushes
// its cell by -dt p_b S_f / V; inlet-type faces give the fixed outflow bconst.
__global__ void __launch_bounds__(TPB) k_cp_boundary(Dev d, double dt, double* __restrict__ U,
                                                     const double* __restrict__ Ub, double* __restrict__ bconst) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.nc) return;
  const int nc = d.nc, nf = d.nf, nb = d.nb;
  double bsum = 0.0;
  for (int s = 0; s < d.SB; ++s) {
    int b = d.cbn[s * nc + c];
    if (b == PADI) break;
    int bc = d.bbc[b];
    if (bc == BC_PERIODIC || is_wall_bc(bc)) continue;
    int f = d.nfi + b;
    if (bc == BC_OUTLET) {
      double fl = dt * d.bpval[b] / d.vol[c];
      for (int k = 0; k < 3; ++k) U[k * nc + c] = U[k * nc + c] - fl * d.sf[k * nf + f];
    } else {
      bsum = bsum + (Ub[b] * d.sf[f] + Ub[nb + b] * d.sf[nf + f] + Ub[2 * nb + b] * d.sf[2 * nf + f]);
    }
  }
  bconst[c] = bsum;
}

// b = B u + bconst, r = b; partial max|r| (:213-224)
__global__ void __launch_bounds__(TPB) k_cp_rhs(Dev d, const double* __restrict__ u, const double* __restrict__ bconst,
                                                double* __restrict__ r, double* __restrict__ part) {
  double v[1] = {0.0};
  const bool mx[1] = {true};
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < d.nc; c += gridDim.x * blockDim.x) {
    double b = cp_div_cell(d, u, c);
    if (bconst) b = b + bconst[c];
    r[c] = b;
    v[0] = fmax(v[0], fabs(b));
  }
  cp_block_partials<1>(v, mx, part);
}

// B u alone (the per-operator entry point)
__global__ void __launch_bounds__(TPB) k_cp_divergence(Dev d, const double* __restrict__ u, double* __restrict__ out) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < d.nc) out[c] = cp_div_cell(d, u, c);
}

// v = V^-1 B^T chi, SoA [3][nc] (cp_adjoint_gradient, :129-189)
__global__ void __launch_bounds__(TPB) k_cp_adjoint(Dev d, const double* __restrict__ chi, double* __restrict__ v) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.nc) return;
  const int nc = d.nc, nf = d.nf;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  for (int s = 0; s < d.SP; ++s) {
    int e = d.cps[s * nc + c];
    if (e == PADI) break;
    int i = e >= 0 ? e : ~e;
    int fm = d.psf[i];
    double w = d.psgcf[i], dd = chi[d.pso[i]] - chi[d.psn[i]];
    double ww = e >= 0 ? w : 1.0 - w;
    a0 = a0 + ww * dd * d.sf[fm];
    a1 = a1 + ww * dd * d.sf[nf + fm];
    a2 = a2 + ww * dd * d.sf[2 * nf + fm];
  }
  for (int s = 0; s < d.SB; ++s) {
    int b = d.cbn[s * nc + c];
    if (b == PADI) break;
    if (d.bbc[b] != BC_OUTLET) continue;
    int f = d.nfi + b;
    a0 = a0 + chi[c] * d.sf[f];
    a1 = a1 + chi[c] * d.sf[nf + f];
    a2 = a2 + chi[c] * d.sf[2 * nf + f];
  }
  double iv = 1.0 / d.vol[c];
  v[c] = a0 * iv;
  v[nc + c] = a1 * iv;
  v[2 * nc + c] = a2 * iv;
}

// q = B v; partial p.q (:243-252)
__global__ void __launch_bounds__(TPB) k_cp_div_dot(Dev d, const double* __restrict__ v, const double* __restrict__ p,
                                                    double* __restrict__ q, double* __restrict__ part) {
  double a[1] = {0.0};
  const bool mx[1] = {false};
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < d.nc; c += gridDim.x * blockDim.x) {
    double qc = cp_div_cell(d, v, c);
    q[c] = qc;
    a[0] = a[0] + p[c] * qc;
  }
  cp_block_partials<1>(a, mx, part);
}

// the scalar rules, one block of 32 threads
// mode 0: bn = max|b|; stop = 3 when bn <= tiny
// mode 1: rz = sum r.z (the first direction)
// mode 2: pq; stop = 1 when |pq| <= tiny, else alpha, en_new, en_tot
// mode 3: rn = max|r|; stop = 2 on rn <= 1e-12 bn or (it >= 2 and en_new <= tol^2 en_tot)
// mode 4: beta = max(0, sum (r - rold).z / rz), rz = sum r.z
__global__ void k_cp_rule(int mode, int nparts, const double* __restrict__ part, double tol, CpState* st) {
  double s0 = cp_fold(part, nparts, 0, mode == 0 || mode == 3);
  double s1 = mode == 4 ? cp_fold(part, nparts, 1, false) : 0.0;
  if (threadIdx.x != 0) return;
  const double tiny = cp_dbl_min();
  switch (mode) {
    case 0:
      st->bn = s0;
      st->stop = s0 > tiny ? 0 : 3;
      st->en_tot = 0.0;
      st->it = 0;
      break;
    case 1: st->rz = s0; break;
    case 2:
      st->it += 1;
      st->pq = s0;
      if (fabs(s0) <= tiny) {
        st->stop = 1;
      } else {
        double alpha = st->rz / s0;
        st->alpha = alpha;
        st->en_new = alpha * alpha * s0;
        st->en_tot = st->en_tot + st->en_new;
      }
      break;
    case 3:
      if (st->stop) break;
      st->rn = s0;
      if (s0 <= 1.0e-12 * st->bn || (st->it >= 2 && st->en_new <= tol * tol * st->en_tot)) st->stop = 2;
      break;
    case 4:
      st->beta = fmax(0.0, s0 / st->rz);
      st->rz = s1;
      break;
  }
}

// rold = r, x += alpha p, r -= alpha q; partial max|r| (:258-266); nothing when the pq rule stopped
__global__ void __launch_bounds__(TPB) k_cp_update(int n, const CpState* __restrict__ st, const double* __restrict__ p,
                                                   const double* __restrict__ q, double* __restrict__ x,
                                                   double* __restrict__ r, double* __restrict__ rold,
                                                   double* __restrict__ part) {
  double a[1] = {0.0};
  const bool mx[1] = {true};
  const bool run = st->stop == 0;
  const double alpha = st->alpha;
  if (run)
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
      double rc = r[c];
      rold[c] = rc;
      x[c] = x[c] + alpha * p[c];
      rc = rc - alpha * q[c];
      r[c] = rc;
      a[0] = fmax(a[0], fabs(rc));
    }
  cp_block_partials<1>(a, mx, part);
}

// partial sums of r.z (mode 1, with p = z) or of (r - rold).z and r.z (mode 4)
__global__ void __launch_bounds__(TPB) k_cp_dots(int n, int first, const double* __restrict__ r,
                                                 const double* __restrict__ rold, const double* __restrict__ z,
                                                 double* __restrict__ p, double* __restrict__ part) {
  double a[2] = {0.0, 0.0};
  const bool mx[2] = {false, false};
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    double zc = z[c], rc = r[c];
    if (first) {
      p[c] = zc;
      a[0] = a[0] + rc * zc;
    } else {
      a[0] = a[0] + (rc - rold[c]) * zc;
      a[1] = a[1] + rc * zc;
    }
  }
  cp_block_partials<2>(a, mx, part);
}

// p = z + beta p (:289-292)
__global__ void __launch_bounds__(TPB) k_cp_direction(int n, const CpState* __restrict__ st,
                                                      const double* __restrict__ z, double* __restrict__ p) {
  const double beta = st->beta;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) p[c] = z[c] + beta * p[c];
}

// u -= v (:296-300), both SoA [3][nc]
__global__ void __launch_bounds__(TPB) k_cp_apply(int n3, const double* __restrict__ v, double* __restrict__ u) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) u[i] = u[i] - v[i];
}

}  // namespace gpu
}  // namespace dpm
