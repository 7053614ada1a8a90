// Point sampling on the device (src/stats/mod_sampling.f90): the owner of each sample point is the
// cell with the nearest centroid (cache_object_owners, :520-562: the first cell in index order at
// the smallest squared distance), and a sample is the owner's value extrapolated with its
// Green-Gauss gradient, u + grad(u) . (x - x_c), for U, p, T and nu_sgs (sample_points_local,
// :493-518; gradients as sampling_maybe_sample takes them, :171-177: one Green-Gauss pass with
// the boundary values of U, p and T, the owner's value on every boundary face for nu_sgs).  Only
// the (6, n_points) payload leaves the device.
#pragma once

#include "common.cuh"

namespace dpm {
namespace gpu {

constexpr int SAMPLE_TILE = 256;

// One thread per point; the block walks the centroids in tiles staged in shared memory, so every
// thread scans the cells in index order and keeps the first strict minimum, as the reference does.
__global__ void __launch_bounds__(SAMPLE_TILE) k_sample_owner(Dev d, int np, const double* __restrict__ pts,
                                                              int* __restrict__ owner) {
  __shared__ double cx[SAMPLE_TILE], cy[SAMPLE_TILE], cz[SAMPLE_TILE];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = d.nc;
  double px = 0.0, py = 0.0, pz = 0.0;
  if (i < np) { px = pts[3 * i]; py = pts[3 * i + 1]; pz = pts[3 * i + 2]; }
  double best = 1.7976931348623157e308;  // huge(1.0_rp)
  int arg = -1;
  for (int base = 0; base < nc; base += SAMPLE_TILE) {
    const int c = base + threadIdx.x;
    if (c < nc) { cx[threadIdx.x] = d.cen[c]; cy[threadIdx.x] = d.cen[nc + c]; cz[threadIdx.x] = d.cen[2 * nc + c]; }
    __syncthreads();
    const int m = min(SAMPLE_TILE, nc - base);
    for (int k = 0; k < m; ++k) {
      const double dx = cx[k] - px, dy = cy[k] - py, dz = cz[k] - pz;
      const double d2 = (dx * dx + dy * dy) + dz * dz;
      if (d2 < best) { best = d2; arg = base + k; }
    }
    __syncthreads();
  }
  if (i < np) owner[i] = arg;
}

// Green-Gauss gradient of the velocity (grad[i + 3 j] = dU_j/dx_i) and of p, T, nu_sgs at cell c.
__device__ void sample_gradients(const Dev& d, int c, const double* __restrict__ U, const double* __restrict__ Ub,
                                 const double* __restrict__ p, const double* __restrict__ pb,
                                 const double* __restrict__ T, const double* __restrict__ Tb,
                                 const double* __restrict__ nu, double (&gu)[9], double (&gs)[3][3]) {
  const int nc = d.nc, nf = d.nf, nfi = d.nfi, nb = d.nb;
  for (int k = 0; k < 9; ++k) gu[k] = 0.0;
  for (int q = 0; q < 3; ++q) gs[q][0] = gs[q][1] = gs[q][2] = 0.0;
  for (int s = 0; s < d.S; ++s) {
    const int f = d.cf[s * nc + c];
    if (f == PADI) break;
    const double sf[3] = {d.sf[f], d.sf[nf + f], d.sf[2 * nf + f]};
    double uf[3], sv[3];
    bool own = true;
    if (f < nfi) {
      const int o = d.fo[f], n = d.fn[f];
      const double w = d.gc[f];
      own = o == c;
      for (int j = 0; j < 3; ++j) uf[j] = w * U[j * nc + o] + (1.0 - w) * U[j * nc + n];
      sv[0] = w * p[o] + (1.0 - w) * p[n];
      sv[1] = w * T[o] + (1.0 - w) * T[n];
      sv[2] = w * nu[o] + (1.0 - w) * nu[n];
    } else {
      const int b = f - nfi;
      for (int j = 0; j < 3; ++j) uf[j] = Ub[j * nb + b];
      sv[0] = pb[b];
      sv[1] = Tb[b];
      sv[2] = nu[c];  // no boundary values: the owner's own
    }
    for (int j = 0; j < 3; ++j)
      for (int i = 0; i < 3; ++i) gu[i + 3 * j] = own ? gu[i + 3 * j] + uf[j] * sf[i] : gu[i + 3 * j] - uf[j] * sf[i];
    for (int q = 0; q < 3; ++q)
      for (int i = 0; i < 3; ++i) gs[q][i] = own ? gs[q][i] + sv[q] * sf[i] : gs[q][i] - sv[q] * sf[i];
  }
  const double v = d.vol[c];
  if (v > 1.0e-30) {
    const double iv = 1.0 / v;
    for (int k = 0; k < 9; ++k) gu[k] = gu[k] * iv;
    for (int q = 0; q < 3; ++q)
      for (int i = 0; i < 3; ++i) gs[q][i] = gs[q][i] * iv;
  }
}

// payload(6, np): U(3), p, T, nu_sgs at each point; zero where a point has no owner
__global__ void __launch_bounds__(TPB) k_sample_points(Dev d, int np, const double* __restrict__ pts,
                                                       const int* __restrict__ owner, const double* __restrict__ U,
                                                       const double* __restrict__ Ub, const double* __restrict__ p,
                                                       const double* __restrict__ pb, const double* __restrict__ T,
                                                       const double* __restrict__ Tb, const double* __restrict__ nu,
                                                       double* __restrict__ payload) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  double* out = payload + 6 * (size_t)i;
  const int c = owner[i];
  if (c < 0 || c >= d.nc) {
    for (int k = 0; k < 6; ++k) out[k] = 0.0;
    return;
  }
  const int nc = d.nc;
  double gu[9], gs[3][3];
  sample_gradients(d, c, U, Ub, p, pb, T, Tb, nu, gu, gs);
  const double dx[3] = {pts[3 * i] - d.cen[c], pts[3 * i + 1] - d.cen[nc + c], pts[3 * i + 2] - d.cen[2 * nc + c]};
  for (int j = 0; j < 3; ++j) out[j] = U[j * nc + c] + (gu[3 * j] * dx[0] + gu[3 * j + 1] * dx[1] + gu[3 * j + 2] * dx[2]);
  out[3] = p[c] + (gs[0][0] * dx[0] + gs[0][1] * dx[1] + gs[0][2] * dx[2]);
  out[4] = T[c] + (gs[1][0] * dx[0] + gs[1][1] * dx[1] + gs[1][2] * dx[2]);
  out[5] = nu[c] + (gs[2][0] * dx[0] + gs[2][1] * dx[1] + gs[2][2] * dx[2]);
}

}  // namespace gpu
}  // namespace dpm
