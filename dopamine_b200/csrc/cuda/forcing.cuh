// Right-hand-side sources outside transport, on the device: Davies nudging of U and T towards
// reference profiles (src/abl/mod_abl_weather.f90:233-366) and passive-scalar sources
// (src/mod_scalar.f90:133-229, applied as mod_fv_solver.f90:1764-1784 applies them).  Both run
// after the right-hand sides are assembled and before the RK3W predictor, as in
// compute_explicit_rhs (mod_fv_solver.f90:1741-1760).
#pragma once

#include "common.cuh"

namespace dpm {
namespace gpu {

constexpr double NUDGE_SMALL = 1.0e-16;  // mod_abl_weather.f90:8

// interp_find_indices (:335-366), 0-based
__host__ __device__ inline void interp_find(const double* a, int n, double v, int& i1, int& i2, double& w) {
  i1 = 0;
  i2 = n - 1;
  for (int i = 0; i < n - 1; ++i)
    if (v >= a[i] && v <= a[i + 1]) {
      i1 = i;
      i2 = i + 1;
      break;
    }
  const double den = a[i2] - a[i1];
  if (fabs(den) < NUDGE_SMALL) w = 0.0;
  else w = fmax(0.0, fmin(1.0, (v - a[i1]) / den));
}

struct NudgeArgs {
  int it1, it2, nz, horiz;
  double wt, coeff, zs, zt;
  const double *z, *Up, *Tp;  // levels (nz); U (3, nz, nt) and T (nz, nt) in the Fortran layout
};

// nudging_apply_rhs (:233-287) with nudging_interpolate (:289-333); the time bracket is the same for
// every cell and comes from the host
__global__ void __launch_bounds__(TPB) k_nudging(Dev d, NudgeArgs a, const double* __restrict__ U,
                                                 const double* __restrict__ T, double* __restrict__ H,
                                                 double* __restrict__ HT) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.nc) return;
  const int nc = d.nc;
  const double z = d.cen[2 * nc + c];
  if (z < a.zs) return;
  const double ramp = a.zt > a.zs ? fmin(1.0, (z - a.zs) / (a.zt - a.zs)) : 1.0;
  int iz1, iz2;
  double wz;
  interp_find(a.z, a.nz, z, iz1, iz2, wz);
  const double wt = a.wt;
  auto up = [&](int j, int iz, int it) { return a.Up[j + 3 * (iz + a.nz * it)]; };
  auto tp = [&](int iz, int it) { return a.Tp[iz + a.nz * it]; };
  double ur[3];
  for (int j = 0; j < 3; ++j)
    ur[j] = (1.0 - wt) * (1.0 - wz) * up(j, iz1, a.it1) + wt * (1.0 - wz) * up(j, iz1, a.it2) +
            (1.0 - wt) * wz * up(j, iz2, a.it1) + wt * wz * up(j, iz2, a.it2);
  const double tr = (1.0 - wt) * (1.0 - wz) * tp(iz1, a.it1) + wt * (1.0 - wz) * tp(iz1, a.it2) +
                    (1.0 - wt) * wz * tp(iz2, a.it1) + wt * wz * tp(iz2, a.it2);
  H[c] = H[c] - ramp * a.coeff * (U[c] - ur[0]);
  H[nc + c] = H[nc + c] - ramp * a.coeff * (U[nc + c] - ur[1]);
  if (!a.horiz) H[2 * nc + c] = H[2 * nc + c] - ramp * a.coeff * (U[2 * nc + c] - ur[2]);
  HT[c] = HT[c] - ramp * a.coeff * (T[c] - tr);
}

// scalar_source_value_at (mod_scalar.f90:133-183) at x; tags is the source's tag points on the
// device, (3, n_tag_points)
__device__ double scalar_source_value(const dpm_scalar_source_t& s, const double* tags, const double x[3], double t) {
  const double small = 1.0e-30;  // src/mod_parameters.f90:29
  if (!s.enabled) return 0.0;
  auto dist2 = [](const double* p, const double* q) {
    double r = 0.0;
    for (int k = 0; k < 3; ++k) r = r + (p[k] - q[k]) * (p[k] - q[k]);
    return r;
  };
  auto slab = [&](double half) {
    const double nn = sqrt(s.normal[0] * s.normal[0] + s.normal[1] * s.normal[1] + s.normal[2] * s.normal[2]);
    double u[3] = {0.0, 0.0, 1.0};
    if (nn > small)
      for (int k = 0; k < 3; ++k) u[k] = s.normal[k] / nn;
    const double r0 = x[0] - s.center[0], r1 = x[1] - s.center[1], r2 = x[2] - s.center[2];
    return fabs(r0 * u[0] + r1 * u[1] + r2 * u[2]) <= fmax(half, small);
  };
  double w = 0.0;
  switch (s.src_kind) {
    case DPM_SCALAR_SRC_POINT:
      if (dist2(x, s.center) <= fmax(s.radius, small) * fmax(s.radius, small)) w = 1.0;
      break;
    case DPM_SCALAR_SRC_LINE: {  // point_segment_distance (:185-200)
      double ab[3], den = 0.0, tt = 0.0, pr[3], dd;
      for (int k = 0; k < 3; ++k) {
        ab[k] = s.p1[k] - s.p0[k];
        den = den + ab[k] * ab[k];
      }
      if (den <= small) {
        dd = sqrt(dist2(x, s.p0));
      } else {
        for (int k = 0; k < 3; ++k) tt = tt + (x[k] - s.p0[k]) * ab[k];
        tt = fmax(0.0, fmin(1.0, tt / den));
        for (int k = 0; k < 3; ++k) pr[k] = s.p0[k] + tt * ab[k];
        dd = sqrt(dist2(x, pr));
      }
      if (dd <= fmax(s.radius, small)) w = 1.0;
      break;
    }
    case DPM_SCALAR_SRC_SURFACE:
      if (slab(s.half_thickness)) {
        if (s.radius > 0.0) {
          if (dist2(x, s.center) <= s.radius * s.radius) w = 1.0;
        } else {
          w = 1.0;
        }
      }
      break;
    case DPM_SCALAR_SRC_OBJ:  // min_distance_to_points (:202-213)
      if (tags && s.n_tag_points > 0) {
        double dm = 1.7976931348623157e308;
        for (int i = 0; i < s.n_tag_points; ++i) {
          const double di = sqrt(dist2(x, tags + 3 * (size_t)i));
          if (di < dm) dm = di;
        }
        if (dm <= fmax(s.tag_radius, small)) w = 1.0;
      }
      break;
    default:
      if (s.shape == DPM_SCALAR_SHAPE_BOX) {
        if (x[0] >= s.box_min[0] && x[1] >= s.box_min[1] && x[2] >= s.box_min[2] && x[0] <= s.box_max[0] &&
            x[1] <= s.box_max[1] && x[2] <= s.box_max[2])
          w = 1.0;
      } else if (s.shape == DPM_SCALAR_SHAPE_PLANE) {
        if (slab(s.half_thickness)) w = 1.0;
      } else if (dist2(x, s.center) <= fmax(s.radius, small) * fmax(s.radius, small)) {
        w = 1.0;
      }
  }
  const double ts = s.time_mode == DPM_SCALAR_TIME_HARMONIC ? cos(s.omega * t + s.phase) : 1.0;
  return s.magnitude * ts * w;
}

// one source added to its scalar's right-hand side Hc (nc), the sources launched in order
__global__ void __launch_bounds__(TPB) k_scalar_source(Dev d, dpm_scalar_source_t s, const double* __restrict__ tags,
                                                       double t, double* __restrict__ Hc) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.nc) return;
  const int nc = d.nc;
  const double x[3] = {d.cen[c], d.cen[nc + c], d.cen[2 * nc + c]};
  const double v = scalar_source_value(s, tags, x, t);
  if (fabs(v) > 1.0e-30) Hc[c] = Hc[c] + v;
}

// the RK3W predictor phi += dt (a_k H + b_k H0) for a right-hand side assembled in parts
__global__ void __launch_bounds__(TPB) k_rk_predict(int64_t n, double dt, double a_k, double b_k,
                                                    const double* __restrict__ H, const double* __restrict__ H0,
                                                    double* __restrict__ phi) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) phi[i] = phi[i] + dt * (a_k * H[i] + b_k * H0[i]);
}

}  // namespace gpu
}  // namespace dpm
