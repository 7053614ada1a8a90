// Jacobi-preconditioned conjugate gradients as one persistent, cooperatively launched kernel.
//
// The reference solves A phi = rhs with PETSc KSPCG: unpreconditioned residual norm, convergence
// when ||r|| <= max(rtol ||b||, atol), nonzero initial guess, constant null space removed from the
// right-hand side and from every preconditioned residual when no Dirichlet row exists
// (src/solver/pressure_backend_petsc.c:381-463, 816-876).  This kernel runs the same recurrence
// with the whole solve on the device: every iteration is two grid-wide phases separated by a
// grid barrier, each phase reduces its dot products per block, and every block then sums the
// per-block partials in the same fixed order, so all blocks take identical convergence decisions
// and the result does not depend on scheduling.
//
// Phase A: p = (z - mean z) + beta/beta_old p_old (built on the fly for neighbours, ping-pong
//          buffers), q = A p, partial p.q
// Phase B: x += a p, r -= a q, z = D^-1 r, partials r.r, z.r, sum z, sum r
//
// The grid barrier is a counter plus generation word; waits are bounded (DPM_BARRIER_SPIN_LIMIT)
// and a timeout sets an error status instead of hanging.  The launch is cooperative, which
// guarantees that all blocks are co-resident.
#pragma once
#include "common.cuh"

namespace dpm {
namespace gpu {

#ifndef DPM_BARRIER_SPIN_LIMIT
#define DPM_BARRIER_SPIN_LIMIT (1u << 26)
#endif

template <class V>
struct PcgArgs {
  int n, WA;
  const int* col;      // [WA][n] sorted columns, PADI padded
  const V* val;        // [WA][n]
  const V* dinv;       // 1 / diag
  const V* b;          // right-hand side
  V* x;                // initial guess in, solution out
  V *r, *z, *p0, *p1, *q, *bp;
  double* partials;    // [2][nblocks][4]
  unsigned* bar;       // [0] arrival counter, [1] generation
  int* status;         // [0] reason, [1] iterations, [2] barrier timeout
  double* dout;        // [0] true residual ||b - A x||, [1] last ||r||, [2] ||b'||
  double rtol, atol;
  int maxit, nullsp, guess_zero;
};

__device__ __forceinline__ double ld_cg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ float ld_cg(const float* p) { return __ldcg(p); }

// Bounded grid barrier.  Returns false on timeout.
__device__ __forceinline__ bool grid_sync(unsigned* bar, unsigned nblocks, unsigned& gen, int* status) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    unsigned g = gen;
    __threadfence();
    unsigned arrived = atomicAdd(&bar[0], 1u);
    if (arrived == nblocks - 1) {
      atomicExch(&bar[0], 0u);
      __threadfence();
      atomicExch(&bar[1], g + 1u);
    } else {
      unsigned spins = 0;
      while (atomicAdd(&bar[1], 0u) == g) {
        if (++spins > DPM_BARRIER_SPIN_LIMIT) { ok = 0; atomicExch(&status[2], 1); break; }
        __nanosleep(64);
      }
    }
    __threadfence();
    gen = g + 1u;
    s_ok = ok && (atomicAdd(&status[2], 0) == 0);
  }
  __syncthreads();
  return s_ok != 0;
}

template <int NV>
__device__ __forceinline__ void block_partial(double (&v)[NV], double* out) {
  __shared__ double sh[32][NV];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) sh[w][k] = v[k];
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double t = lane < nw ? sh[lane][k] : 0.0;
      for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
      if (lane == 0) out[k] = t;
    }
  }
  __syncthreads();
}

// Every block sums the per-block partials in the same order.
template <int NV>
__device__ __forceinline__ void grid_total(const double* partials, int nblocks, double (&res)[NV]) {
  __shared__ double tot[NV];
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    double v[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = 0.0;
    for (int b = lane; b < nblocks; b += 32)
#pragma unroll
      for (int k = 0; k < NV; ++k) v[k] += __ldcg(&partials[b * 4 + k]);
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
      if (lane == 0) tot[k] = v[k];
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NV; ++k) res[k] = tot[k];
  __syncthreads();
}

template <class V>
__global__ void __launch_bounds__(TPB) k_pcg(PcgArgs<V> a) {
  const int n = a.n, WA = a.WA;
  const unsigned nblk = gridDim.x;
  const int stride = gridDim.x * blockDim.x;
  const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned gen = 0;
  if (i0 == 0) { /* generation word is reset by the host before launch */ }
  double* part0 = a.partials;
  double* part1 = a.partials + 4 * nblk;
  int ph = 0;
  auto part = [&]() { double* p = ph ? part1 : part0; ph ^= 1; return p; };

  // ---- b' = b - mean(b) (null space), r = b' - A x, ||r||, ||b'||
  double mb = 0.0;
  if (a.nullsp) {
    double v[1] = {0.0};
    for (int i = i0; i < n; i += stride) v[0] += (double)a.b[i];
    double* P = part();
    block_partial<1>(v, P + 4 * blockIdx.x);
    if (!grid_sync(a.bar, nblk, gen, a.status)) return;
    double t[1];
    grid_total<1>(P, nblk, t);
    mb = t[0] / (double)n;
  }
  if (a.guess_zero)
    for (int i = i0; i < n; i += stride) a.x[i] = (V)0;
  {
    double v[2] = {0.0, 0.0};
    for (int i = i0; i < n; i += stride) {
      V bi = a.b[i];
      V bpi = a.nullsp ? (V)((double)bi - mb) : bi;
      a.bp[i] = bpi;
      double s = 0.0;
      for (int w = 0; w < WA; ++w) {
        int j = __ldg(&a.col[w * n + i]);
        if (j == PADI) break;
        s += (double)__ldg(&a.val[w * n + i]) * (double)ld_cg(&a.x[j]);
      }
      double ri = (double)bpi - s;
      a.r[i] = (V)ri;
      v[0] += ri * ri;
      v[1] += (double)bpi * (double)bpi;
    }
    double* P = part();
    block_partial<2>(v, P + 4 * blockIdx.x);
    if (!grid_sync(a.bar, nblk, gen, a.status)) return;
    double t[2];
    grid_total<2>(P, nblk, t);
    double dp = sqrt(t[0]), sn = sqrt(t[1]);
    double rnorm0 = a.guess_zero ? dp : (sn == 0.0 ? dp : sn);
    a.dout[2] = sn;
    // stash scalars in registers of every thread
    a.dout[1] = dp;
    double ttol = fmax(a.rtol * rnorm0, a.atol);
    int reason = 0;
    if (!(fabs(dp) <= 1.7976931348623157e308)) reason = -9;
    else if (dp <= ttol) reason = dp < a.atol ? 3 : 2;
    else if (dp >= 1.0e5 * rnorm0) reason = -4;
    int its = 0;
    if (!reason) {
      // z = D^-1 r ; sums for the null-space projection and beta
      double v4[4] = {0, 0, 0, 0};
      for (int i = i0; i < n; i += stride) {
        double ri = (double)a.r[i];
        double zi = (double)(V)(ri * (double)a.dinv[i]);
        a.z[i] = (V)zi;
        v4[0] += zi;
        v4[1] += ri;
        v4[2] += zi * ri;
      }
      double* P = part();
      block_partial<4>(v4, P + 4 * blockIdx.x);
      if (!grid_sync(a.bar, nblk, gen, a.status)) return;
      double t4[4];
      grid_total<4>(P, nblk, t4);
      double mz = a.nullsp ? t4[0] / (double)n : 0.0;
      double beta = a.nullsp ? t4[2] - mz * t4[1] : t4[2];
      double betaold = 0.0, dpi = 0.0, dpiold = 0.0;
      V* pold = a.p0;
      V* pnew = a.p1;
      int it = 0;
      do {
        its = it + 1;
        if (beta == 0.0) { reason = 3; break; }
        if (it > 0 && beta * betaold < 0.0) { reason = -8; break; }
        const double bb = it == 0 ? 0.0 : beta / betaold;
        // ---- phase A
        {
          double v1[1] = {0.0};
          for (int i = i0; i < n; i += stride) {
            double s = 0.0;
            for (int w = 0; w < WA; ++w) {
              int j = __ldg(&a.col[w * n + i]);
              if (j == PADI) break;
              double pj = (double)ld_cg(&a.z[j]) - mz;
              if (it > 0) pj = pj + bb * (double)ld_cg(&pold[j]);
              s += (double)__ldg(&a.val[w * n + i]) * (double)(V)pj;
            }
            double pi = (double)a.z[i] - mz;
            if (it > 0) pi = pi + bb * (double)pold[i];
            pnew[i] = (V)pi;
            a.q[i] = (V)s;
            v1[0] += (double)(V)pi * (double)(V)s;
          }
          double* P = part();
          block_partial<1>(v1, P + 4 * blockIdx.x);
          if (!grid_sync(a.bar, nblk, gen, a.status)) return;
          double t1[1];
          grid_total<1>(P, nblk, t1);
          dpiold = dpi;
          dpi = t1[0];
        }
        betaold = beta;
        if (dpi == 0.0 || (it > 0 && ((dpi > 0) - (dpi < 0)) * ((dpiold > 0) - (dpiold < 0)) < 0)) {
          reason = dpi == 0.0 ? 3 : -10;
          break;
        }
        const double al = beta / dpi;
        // ---- phase B
        {
          double v4b[4] = {0, 0, 0, 0};
          for (int i = i0; i < n; i += stride) {
            double pi = (double)pnew[i];
            a.x[i] = (V)((double)a.x[i] + al * pi);
            double ri = (double)a.r[i] - al * (double)a.q[i];
            V rv = (V)ri;
            a.r[i] = rv;
            double rr = (double)rv;
            double zi = (double)(V)(rr * (double)a.dinv[i]);
            a.z[i] = (V)zi;
            v4b[0] += rr * rr;
            v4b[1] += zi;
            v4b[2] += rr;
            v4b[3] += zi * rr;
          }
          double* P = part();
          block_partial<4>(v4b, P + 4 * blockIdx.x);
          if (!grid_sync(a.bar, nblk, gen, a.status)) return;
          double t4b[4];
          grid_total<4>(P, nblk, t4b);
          dp = sqrt(t4b[0]);
          if (!(fabs(dp) <= 1.7976931348623157e308)) reason = -9;
          else if (dp <= ttol) reason = dp < a.atol ? 3 : 2;
          else if (dp >= 1.0e5 * rnorm0) reason = -4;
          if (reason) break;
          mz = a.nullsp ? t4b[1] / (double)n : 0.0;
          beta = a.nullsp ? t4b[3] - mz * t4b[2] : t4b[3];
        }
        V* t = pold; pold = pnew; pnew = t;
        it++;
      } while (it < a.maxit);
      if (!reason && it >= a.maxit) reason = -3;
      a.dout[1] = dp;
    }
    // ---- true residual ||b - A x|| with the caller's right-hand side (KSPBuildResidual)
    {
      if (!grid_sync(a.bar, nblk, gen, a.status)) return;  // x complete everywhere
      double v1[1] = {0.0};
      for (int i = i0; i < n; i += stride) {
        double s = 0.0;
        for (int w = 0; w < WA; ++w) {
          int j = __ldg(&a.col[w * n + i]);
          if (j == PADI) break;
          s += (double)__ldg(&a.val[w * n + i]) * (double)ld_cg(&a.x[j]);
        }
        double d = (double)a.b[i] - s;
        v1[0] += d * d;
      }
      double* P = part();
      block_partial<1>(v1, P + 4 * blockIdx.x);
      if (!grid_sync(a.bar, nblk, gen, a.status)) return;
      double t1[1];
      grid_total<1>(P, nblk, t1);
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.dout[0] = sqrt(t1[0]);
        a.status[0] = reason;
        a.status[1] = its;
      }
    }
  }
}

}  // namespace gpu
}  // namespace dpm
