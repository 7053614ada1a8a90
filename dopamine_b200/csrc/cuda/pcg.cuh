// Jacobi-preconditioned conjugate gradients as one persistent, cooperatively launched kernel.
//
// The reference solves A phi = rhs with PETSc KSPCG: unpreconditioned residual norm, convergence
// when ||r|| <= max(rtol ||b||, atol), nonzero initial guess, constant null space removed from the
// right-hand side and from every preconditioned residual when no Dirichlet row exists
// (src/solver/pressure_backend_petsc.c:381-463, 816-876).  This kernel runs the same recurrence
// with the whole solve on the device:
//
//   phase A: p = (z - mean z) + (beta/beta_old) p_old, built on the fly for neighbour cells
//            (ping-pong p buffers), q = A p, partial p.q            -> grid all-reduce
//   phase B: x += a p, r -= a q, z = D^-1 r, partials r.r, sum z, sum r, z.r  -> grid all-reduce
//
// Rows of A are stored ELL [width][n] with sorted columns and padded to a fixed width with
// (self, 0) entries, so each row is a fully unrolled set of independent loads.  A and 1/diag are
// read through the read-only path and stay L1-resident across iterations; the vectors that
// neighbours read (z, p) go through L2 (ld.cg), which is where other SMs' writes are visible.
// Each thread keeps its own cells' x, r, z and p in registers when the mesh fits (CPT cells per
// thread).  Grid all-reduces are deterministic (see grid_allreduce).  The launch is cooperative,
// which guarantees co-residency of all blocks; every wait is bounded.
#pragma once
#include "common.cuh"

namespace dpm {
namespace gpu {

#ifndef DPM_BARRIER_SPIN_LIMIT
#define DPM_BARRIER_SPIN_LIMIT (1u << 26)
#endif

constexpr int PCG_TPB = 1024;

// Poll limit of a grid-wide wait: status[3] when the host set it (a failure-detection test makes
// the wait run out this way), else DPM_BARRIER_SPIN_LIMIT.  Read by the waiting thread before it
// arrives, so the load overlaps the arrival.
__device__ __forceinline__ unsigned spin_limit(const int* status) {
  const unsigned o = (unsigned)__ldcg(&status[3]);
  return o ? o : (unsigned)DPM_BARRIER_SPIN_LIMIT;
}

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
  unsigned* bar;       // [0] monotonic arrival counter
  int* status;         // [0] reason, [1] iterations, [2] barrier timeout, [3] poll limit (0: default)
  double* dout;        // [0] true residual ||b - A x||, [1] last ||r||, [2] ||b'||
  double rtol, atol;
  int maxit, nullsp, guess_zero;
};

__device__ __forceinline__ double ld_cg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ float ld_cg(const float* p) { return __ldcg(p); }

// Grid-wide deterministic all-reduce + barrier.  Each block reduces its NV values (fixed shuffle
// trees; warp k takes value k), writes them into the partial buffer of this barrier (two buffers
// alternate) and thread 0 arrives on a monotonic counter; once all blocks have arrived, warp k of
// every block reads value k of all partials with a fixed lane-to-block mapping, all of a lane's
// loads of a round issued together, and reduces them with the same shuffle tree, so all blocks
// hold bit-identical totals.  The wait is bounded and returns false on timeout.
template <int NV>
__device__ __forceinline__ bool grid_allreduce(double (&v)[NV], double* partials, unsigned* bar, unsigned& gen,
                                               int* status, double (&res)[NV]) {
  constexpr int RB = 5;  // blocks per lane per round of the post-barrier read (one round up to 160 blocks)
  __shared__ double sh[32][4];
  __shared__ double shr[4];
  __shared__ int s_ok;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int P = gridDim.x;
  double* buf = partials + (size_t)(gen & 1u) * 4 * gridDim.x;
#pragma unroll
  for (int k = 0; k < NV; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) sh[w][k] = v[k];
  __syncthreads();
  if (w < NV) {  // warp w: value w over the block's warps
    double t = lane < nw ? sh[lane][w] : 0.0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (lane == 0) buf[blockIdx.x * 4 + w] = t;
  }
  __syncthreads();  // the partial stores precede thread 0's release below
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned target = (gen + 1u) * gridDim.x;
    const unsigned lim = spin_limit(status);
    __threadfence();
    atomicAdd(&bar[0], 1u);
    unsigned spins = 0;
    for (;;) {
      unsigned cur;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(cur) : "l"(&bar[0]) : "memory");
      if ((int)(cur - target) >= 0) break;
      if (++spins > lim) { ok = 0; atomicExch(&status[2], 1); break; }
      if (spins > 32) __nanosleep(20);
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  if (s_ok && w < NV) {  // warp w: value w over the blocks, lane l sums blocks l, l + 32, ... in order
    double u = 0.0;
    for (int b0 = lane; b0 < P; b0 += 32 * RB) {
      double pv[RB];
#pragma unroll
      for (int h = 0; h < RB; ++h) pv[h] = b0 + 32 * h < P ? __ldcg(&buf[(b0 + 32 * h) * 4 + w]) : 0.0;
#pragma unroll
      for (int h = 0; h < RB; ++h) u += pv[h];
    }
    for (int o = 16; o > 0; o >>= 1) u += __shfl_down_sync(0xffffffffu, u, o);
    if (lane == 0) shr[w] = u;
  }
  __syncthreads();
  gen = gen + 1u;
#pragma unroll
  for (int k = 0; k < NV; ++k) res[k] = s_ok ? shr[k] : 0.0;
  return s_ok != 0;
}

__device__ __forceinline__ int classify(double dp, double ttol, double atol, double rnorm0) {
  if (!(fabs(dp) <= 1.7976931348623157e308)) return -9;   // KSP_DIVERGED_NANORINF
  if (dp <= ttol) return dp < atol ? 3 : 2;               // KSP_CONVERGED_ATOL / _RTOL
  if (dp >= 1.0e5 * rnorm0) return -4;                    // KSP_DIVERGED_DTOL
  return 0;
}

// Row i of A times the vector v (ELL, padded rows: no early exit, all loads independent).
template <class V, int WT>
__device__ __forceinline__ double spmv_row(const PcgArgs<V>& a, int i, const V* v) {
  const int n = a.n;
  constexpr int W = WT > 0 ? WT : 16;
  const int WA = WT > 0 ? WT : a.WA;
  int c[W];
#pragma unroll
  for (int w = 0; w < W; ++w)
    if (w < WA) c[w] = __ldg(&a.col[w * n + i]);
  double x[W];
#pragma unroll
  for (int w = 0; w < W; ++w)
    if (w < WA) x[w] = (double)ld_cg(&v[c[w]]);
  double s = 0.0;
#pragma unroll
  for (int w = 0; w < W; ++w)
    if (w < WA) s += (double)__ldcg(&a.val[w * n + i]) * x[w];
  return s;
}

// Row i of A times p = (z - mz) + bb p_old (first iteration: p = z - mz), p formed on the fly.
template <class V, int WT>
__device__ __forceinline__ double spmv_row_p(const PcgArgs<V>& a, int i, const V* pold, double mz, double bb,
                                             bool first) {
  const int n = a.n;
  constexpr int W = WT > 0 ? WT : 16;
  const int WA = WT > 0 ? WT : a.WA;
  int c[W];
#pragma unroll
  for (int w = 0; w < W; ++w)
    if (w < WA) c[w] = __ldg(&a.col[w * n + i]);
  double zz[W], pp[W];
#pragma unroll
  for (int w = 0; w < W; ++w)
    if (w < WA) {
      zz[w] = (double)ld_cg(&a.z[c[w]]);
      pp[w] = first ? 0.0 : (double)ld_cg(&pold[c[w]]);
    }
  double s = 0.0;
#pragma unroll
  for (int w = 0; w < W; ++w)
    if (w < WA) {
      double pj = zz[w] - mz;
      if (!first) pj = pj + bb * pp[w];
      s += (double)__ldcg(&a.val[w * n + i]) * (double)(V)pj;
    }
  return s;
}

// CPT > 0: exactly CPT cells per thread, own x, r, z, p held in registers
//          (requires n <= grid * blockDim * CPT).
// CPT == 0: grid-stride loops with the own-cell vectors in global memory (any n).
// WT: fixed padded row width (7 on hexahedral meshes), 0 = runtime width <= 16.
template <class V, int CPT, int WT>
__global__ void __launch_bounds__(PCG_TPB, 1) k_pcg(PcgArgs<V> a) {
  const int n = a.n;
  const int stride = gridDim.x * blockDim.x;
  const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned gen = 0;
  constexpr int NR = CPT > 0 ? CPT : 1;
  double rx[NR], rr_[NR], rz[NR], rp[NR], rq[NR], rd[NR];

  // ---- b' = b - mean(b) when the constant null space is active
  double mb = 0.0;
  if (a.nullsp) {
    double v[1] = {0.0}, t[1];
    for (int i = i0; i < n; i += stride) v[0] += (double)a.b[i];
    if (!grid_allreduce<1>(v, a.partials, a.bar, gen, a.status, t)) return;
    mb = t[0] / (double)n;
  }
  if (a.guess_zero) {
    for (int i = i0; i < n; i += stride) a.x[i] = (V)0;
    double v[1] = {0.0}, t[1];
    if (!grid_allreduce<1>(v, a.partials, a.bar, gen, a.status, t)) return;
  }
  // ---- r = b' - A x
  double v2[2] = {0.0, 0.0}, t2[2];
  if (CPT > 0) {
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      int i = i0 + k * stride;
      if (i < n) {
        double bi = (double)a.b[i];
        double bpi = (double)(V)(a.nullsp ? bi - mb : bi);
        double ri = bpi - spmv_row<V, WT>(a, i, a.x);
        rx[k] = (double)a.x[i];
        rr_[k] = (double)(V)ri;
        rd[k] = (double)__ldg(&a.dinv[i]);
        v2[0] += rr_[k] * rr_[k];
        v2[1] += bpi * bpi;
      }
    }
  } else {
    for (int i = i0; i < n; i += stride) {
      double bi = (double)a.b[i];
      double bpi = (double)(V)(a.nullsp ? bi - mb : bi);
      double ri = (double)(V)(bpi - spmv_row<V, WT>(a, i, a.x));
      a.r[i] = (V)ri;
      v2[0] += ri * ri;
      v2[1] += bpi * bpi;
    }
  }
  if (!grid_allreduce<2>(v2, a.partials, a.bar, gen, a.status, t2)) return;
  double dp = sqrt(t2[0]);
  const double sn = sqrt(t2[1]);
  const double rnorm0 = a.guess_zero ? dp : (sn == 0.0 ? dp : sn);
  const double ttol = fmax(a.rtol * rnorm0, a.atol);
  int reason = classify(dp, ttol, a.atol, rnorm0);
  int its = 0;
  if (!reason) {
    // ---- z = D^-1 r
    double v4[4] = {0, 0, 0, 0}, t4[4];
    if (CPT > 0) {
#pragma unroll
      for (int k = 0; k < NR; ++k) {
        int i = i0 + k * stride;
        if (i < n) {
          rz[k] = (double)(V)(rr_[k] * rd[k]);
          a.z[i] = (V)rz[k];
          v4[0] += rz[k]; v4[1] += rr_[k]; v4[2] += rz[k] * rr_[k];
        }
      }
    } else {
      for (int i = i0; i < n; i += stride) {
        double ri = (double)a.r[i];
        double zi = (double)(V)(ri * (double)__ldg(&a.dinv[i]));
        a.z[i] = (V)zi;
        v4[0] += zi; v4[1] += ri; v4[2] += zi * ri;
      }
    }
    if (!grid_allreduce<4>(v4, a.partials, a.bar, gen, a.status, t4)) return;
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
      const bool first = it == 0;
      // ---- phase A: p, q = A p, p.q
      double v1[1] = {0.0}, t1[1];
      if (CPT > 0) {
#pragma unroll
        for (int k = 0; k < NR; ++k) {
          int i = i0 + k * stride;
          if (i < n) {
            double pi = rz[k] - mz;
            if (!first) pi = pi + bb * rp[k];
            rp[k] = (double)(V)pi;
            pnew[i] = (V)rp[k];
            rq[k] = (double)(V)spmv_row_p<V, WT>(a, i, pold, mz, bb, first);
            v1[0] += rp[k] * rq[k];
          }
        }
      } else {
        for (int i = i0; i < n; i += stride) {
          double pi = (double)a.z[i] - mz;
          if (!first) pi = pi + bb * (double)pold[i];
          pi = (double)(V)pi;
          pnew[i] = (V)pi;
          double qi = (double)(V)spmv_row_p<V, WT>(a, i, pold, mz, bb, first);
          a.q[i] = (V)qi;
          v1[0] += pi * qi;
        }
      }
      if (!grid_allreduce<1>(v1, a.partials, a.bar, gen, a.status, t1)) return;
      dpiold = dpi;
      dpi = t1[0];
      betaold = beta;
      if (dpi == 0.0 || (it > 0 && ((dpi > 0) - (dpi < 0)) * ((dpiold > 0) - (dpiold < 0)) < 0)) {
        reason = dpi == 0.0 ? 3 : -10;
        break;
      }
      const double al = beta / dpi;
      // ---- phase B: x, r, z and the four sums
      double w4[4] = {0, 0, 0, 0}, s4[4];
      if (CPT > 0) {
#pragma unroll
        for (int k = 0; k < NR; ++k) {
          int i = i0 + k * stride;
          if (i < n) {
            rx[k] = (double)(V)(rx[k] + al * rp[k]);
            rr_[k] = (double)(V)(rr_[k] - al * rq[k]);
            rz[k] = (double)(V)(rr_[k] * rd[k]);
            a.z[i] = (V)rz[k];
            w4[0] += rr_[k] * rr_[k]; w4[1] += rz[k]; w4[2] += rr_[k]; w4[3] += rz[k] * rr_[k];
          }
        }
      } else {
        for (int i = i0; i < n; i += stride) {
          double pi = (double)pnew[i];
          a.x[i] = (V)((double)a.x[i] + al * pi);
          double ri = (double)(V)((double)a.r[i] - al * (double)a.q[i]);
          a.r[i] = (V)ri;
          double zi = (double)(V)(ri * (double)__ldg(&a.dinv[i]));
          a.z[i] = (V)zi;
          w4[0] += ri * ri; w4[1] += zi; w4[2] += ri; w4[3] += zi * ri;
        }
      }
      if (!grid_allreduce<4>(w4, a.partials, a.bar, gen, a.status, s4)) return;
      dp = sqrt(s4[0]);
      reason = classify(dp, ttol, a.atol, rnorm0);
      if (reason) break;
      mz = a.nullsp ? s4[1] / (double)n : 0.0;
      beta = a.nullsp ? s4[3] - mz * s4[2] : s4[3];
      V* t = pold; pold = pnew; pnew = t;
      it++;
    } while (it < a.maxit);
    if (!reason && it >= a.maxit) reason = -3;
  }
  // ---- write back x, then the true residual ||b - A x|| with the caller's b (KSPBuildResidual)
  if (CPT > 0) {
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      int i = i0 + k * stride;
      if (i < n) a.x[i] = (V)rx[k];
    }
  }
  double v1[1] = {0.0}, t1[1];
  if (!grid_allreduce<1>(v1, a.partials, a.bar, gen, a.status, t1)) return;
  for (int i = i0; i < n; i += stride) {
    double d = (double)a.b[i] - spmv_row<V, WT>(a, i, a.x);
    v1[0] += d * d;
  }
  if (!grid_allreduce<1>(v1, a.partials, a.bar, gen, a.status, t1)) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.dout[0] = sqrt(t1[0]);
    a.dout[1] = dp;
    a.dout[2] = sn;
    a.status[0] = reason;
    a.status[1] = its;
  }
}

// Host helper: picks the instantiation for the mesh size (register-resident when it fits) and
// row width (fixed 7 for hexahedral meshes).
template <class V>
inline void* pcg_kernel_for(int n, int grid, int width, int* cpt_out) {
  const long cap = (long)grid * PCG_TPB;
  int cpt = n <= cap ? 1 : n <= 2 * cap ? 2 : n <= 3 * cap ? 3 : n <= 4 * cap ? 4 : 0;
  *cpt_out = cpt;
  if (width == 7) {
    switch (cpt) {
      case 1: return (void*)k_pcg<V, 1, 7>;
      case 2: return (void*)k_pcg<V, 2, 7>;
      case 3: return (void*)k_pcg<V, 3, 7>;
      case 4: return (void*)k_pcg<V, 4, 7>;
      default: return (void*)k_pcg<V, 0, 7>;
    }
  }
  switch (cpt) {
    case 1: return (void*)k_pcg<V, 1, 0>;
    case 2: return (void*)k_pcg<V, 2, 0>;
    case 3: return (void*)k_pcg<V, 3, 0>;
    case 4: return (void*)k_pcg<V, 4, 0>;
    default: return (void*)k_pcg<V, 0, 0>;
  }
}

}  // namespace gpu
}  // namespace dpm
