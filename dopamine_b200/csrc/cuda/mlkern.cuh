// The multilevel flexible-CG solve as a sequence of standalone kernels, for large meshes.
//
// k_mlcg keeps the whole solve in one persistent cooperative kernel: no launch gaps, but every
// phase runs at two 512-thread blocks per SM under a 64-register cap, and on a fine level of
// millions of rows its sweeps reach ~40 % of HBM bandwidth (long-scoreboard stalls; more rows per
// lane, a register software pipeline and shared-memory staging of the row data were all measured
// slower).  The same sweep as a standalone kernel - one row per thread, 32 registers, full
// occupancy - streams a 19.3M-row, 6-neighbour level at the measured copy bandwidth (0.21 ms,
// 6.6 TB/s).  So on large meshes each phase is its own kernel: Chebyshev sweep, residual,
// restriction (aggregate sums of the member rows' residuals, fixed order), dense coarse solve,
// prolongation, w = A z with per-block partial sums, the FCG scalars (one block reduces the
// partials in a fixed order and applies the stopping rule), and the vector update.  The Krylov
// state lives in device memory (MlkState); once a solve has stopped, every kernel returns at its
// first instruction, so the host can enqueue iterations ahead of the stopping test it reads back.
// The recurrences, the null-space handling, the stall guard and the stopping rule are those of
// k_mlcg and k_fcg (src/solver/pressure_backend_petsc.c:816-876 for the rule itself); only the
// order of the reductions' sums differs.
#pragma once
#include "mlcg.cuh"

namespace dpm {
namespace gpu {

constexpr int MLK_TPB = 256;
constexpr int MLK_NV = 8;            // sums reduced per iteration
constexpr int MLK_RED_BLOCKS = 2368; // grid of the reducing kernels (16 blocks per SM)

struct MlkState {
  double mb, rnorm0, ttol, rtol, atol, dp, sn, dp_mark, pq_old, alpha, beta, m, true_res;
  int its, reason, done, maxit, nullsp, guess_zero, stall_window;
  double stall_ratio;
};

// Block sum of NV values per thread into part[block][NV] (fixed shuffle tree, then warps in order).
template <int NV>
__device__ __forceinline__ void mlk_block_partials(double (&v)[NV], double* part) {
  __shared__ double sh[MLK_TPB / 32][NV];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double t = v[k];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (lane == 0) sh[w][k] = t;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double t = 0.0;
    for (int j = 0; j < MLK_TPB / 32; ++j) t += sh[j][threadIdx.x];
    part[(size_t)blockIdx.x * NV + threadIdx.x] = t;
  }
}

// Totals of the per-block partials (one block of 32 * NV threads: warp k sums value k over the
// blocks, lane l taking blocks l, l + 32, ... in order, then a fixed shuffle tree).
template <int NV>
__device__ __forceinline__ void mlk_totals(int nparts, const double* part, double (&tot)[NV]) {
  __shared__ double s_t[NV];
  const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (k < NV) {
    double t = 0.0;
    for (int j = lane; j < nparts; j += 32) t += part[(size_t)j * NV + k];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (lane == 0) s_t[k] = t;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NV; ++q) tot[q] = s_t[q];
}

// First Chebyshev step of level 0 from the residual (or the coarse right-hand side)
__device__ __forceinline__ void mlk_start0(const MlDevLevel* L0, float* bC, int i, double ri) {
  if (L0) {
    const float bi = (float)ri * __ldg(&L0->dinv[i]);
    const float di = L0->inv_theta * bi;
    L0->b[i] = bi;
    L0->d[i] = di;
    L0->x0[i] = di;
  } else {
    bC[i] = (float)ri;
  }
}

// ---- start: b' = b - mean(b) (null space), r = b' - A x
static __global__ void __launch_bounds__(MLK_TPB) k_mlk_init_sum(int n, const double* __restrict__ b, double* x,
                                                          int guess_zero, double* part) {
  double v[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (guess_zero) x[i] = 0.0;
    v[0] += b[i];
  }
  mlk_block_partials<1>(v, part);
}
static __global__ void k_mlk_init_mean(int n, int nparts, const double* part, MlkState* S) {
  double t[1];
  mlk_totals<1>(nparts, part, t);
  if (threadIdx.x == 0) S->mb = S->nullsp ? t[0] / (double)n : 0.0;
}
static __global__ void __launch_bounds__(MLK_TPB) k_mlk_init_resid(MlArgs a, const MlDevLevel* L0, const MlkState* S,
                                                            double* part) {
  const double mb = S->mb;
  double v[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
    const double bp = a.b[i] - mb;
    const double ri = bp - ml_row64(a, i, (const double*)a.x);
    a.r[i] = ri;
    a.p[i] = 0.0;
    a.q[i] = 0.0;
    v[0] += ri * ri;
    v[1] += bp * bp;
    mlk_start0(L0, a.bC, i, ri);
  }
  mlk_block_partials<2>(v, part);
}
static __global__ void k_mlk_init_rule(int nparts, const double* part, MlkState* S) {
  double t[2];
  mlk_totals<2>(nparts, part, t);
  if (threadIdx.x == 0) {
    const double dp = sqrt(t[0]), sn = sqrt(t[1]);
    S->dp = dp;
    S->sn = sn;
    S->rnorm0 = S->guess_zero ? dp : (sn == 0.0 ? dp : sn);
    S->ttol = fmax(S->rtol * S->rnorm0, S->atol);
    int reason = classify(dp, S->ttol, S->atol, S->rnorm0);
    if (!reason && S->maxit <= 0) reason = -3;
    S->reason = reason;
    S->its = 0;
    S->pq_old = 1.0;
    S->dp_mark = dp;
    S->done = reason != 0;
  }
}

// ---- V-cycle phases (one row per thread)
template <class SV>
static __global__ void __launch_bounds__(MLK_TPB) k_mlk_sweep(MlDevLevel L, float c1, float c2, int first,
                                                       const float* __restrict__ xi, float* __restrict__ xo,
                                                       const float* __restrict__ om, float gam, const MlkState* S) {
  if (S->done) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= L.n) return;
  const float acc = ml_part<SV, false>(L, i, xi, nullptr, 0.0f, 1, 0);
  const float b = __ldcg(&L.b[i]), x = __ldcg(&xi[i]);
  const float rs = b - fmaf(__ldg(&L.g[i]), x, acc);
  const float d = first ? L.inv_theta * rs : fmaf(c1, __ldcg(&L.d[i]), c2 * rs);
  L.d[i] = d;
  xo[i] = x + d + (om ? gam * __ldg(&om[i]) * b : 0.0f);
}
// residual in unscaled form, r_i = a_ii (b_i - g_i x_i - (S x)_i)
template <class SV>
static __global__ void __launch_bounds__(MLK_TPB) k_mlk_resid(MlDevLevel L, const float* __restrict__ x,
                                                       float* __restrict__ r, const MlkState* S) {
  if (S->done) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= L.n) return;
  const float acc = ml_part<SV, false>(L, i, x, nullptr, 0.0f, 1, 0);
  r[i] = __ldg(&L.diag[i]) * (__ldcg(&L.b[i]) - fmaf(__ldg(&L.g[i]), __ldcg(&x[i]), acc));
}
// restriction: each aggregate sums its members' residuals in member order, then the next level's
// first Chebyshev step (or the coarse right-hand side)
static __global__ void __launch_bounds__(MLK_TPB) k_mlk_restrict(MlDevLevel L, const float* __restrict__ r, MlDevLevel N,
                                                          int last, float* __restrict__ bC, const MlkState* S) {
  if (S->done) return;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= L.n_next) return;
  float sres = 0.0f;
  for (int m = 0; m < L.M; ++m) {
    const int i = __ldg(&L.mem[(size_t)m * L.n_next + c]);
    if (i >= 0) sres += __ldcg(&r[i]);
  }
  if (last) {
    bC[c] = sres;
  } else {
    const float bs = sres * __ldg(&N.dinv[c]);
    const float di = N.inv_theta * bs;
    N.b[c] = bs;
    N.d[c] = di;
    N.x0[c] = di;
  }
}
// coarsest level: x_C = A_C^-1 b_C, one warp per row
static __global__ void __launch_bounds__(MLK_TPB) k_mlk_coarse(int nC, const float* __restrict__ cinv,
                                                        const float* __restrict__ bC, float* __restrict__ xC,
                                                        const MlkState* S) {
  if (S->done) return;
  const int lane = threadIdx.x & 31;
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (row >= nC) return;
  float s = 0.0f;
  for (int k = lane; k < nC; k += 32) s = fmaf(__ldg(&cinv[(size_t)row * nC + k]), __ldcg(&bC[k]), s);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) xC[row] = s;
}
// prolongation in place: x_i += oc x_c(agg i)
static __global__ void __launch_bounds__(MLK_TPB) k_mlk_prolong(MlDevLevel L, float* __restrict__ x,
                                                         const float* __restrict__ xc, float oc, const MlkState* S) {
  if (S->done) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= L.n) return;
  x[i] = fmaf(oc, __ldcg(&xc[__ldg(&L.agg[i])]), x[i]);
}

// training-sample recording of the learned term (as in k_mlcg): every rec_stride-th iteration
static __global__ void __launch_bounds__(MLK_TPB) k_mlk_record(MlArgs a, const float* __restrict__ z, const float* b0,
                                                        const MlkState* S) {
  if (S->done) return;
  const int its = S->its;
  if (a.rec_stride <= 0 || its % a.rec_stride != 0 || a.rec_base + its / a.rec_stride >= a.rec_max) return;
  const size_t off = (size_t)(a.rec_base + its / a.rec_stride) * a.n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
    const size_t o = off + __ldg(&a.pinv[i]);
    a.rec_r[o] = __ldcg(&a.r[i]);
    a.rec_z[o] = (double)__ldcg(&z[i]);
    a.rec_u[o] = (double)__ldcg(&b0[i]);
    a.rec_x[o] = __ldcg(&a.x[i]);
  }
}

// ---- w = A z (FP64 operator) and the eight sums of the iteration: one row per thread (as the
// sweeps; a grid-stride loop over ~32 rows per thread ran at half the bandwidth), per-block
// partials folded by k_mlk_fold before the scalar kernel
template <class ZT>
static __global__ void __launch_bounds__(MLK_TPB) k_mlk_wz(MlArgs a, const ZT* __restrict__ z, double* part,
                                                    const MlkState* S) {
  if (S->done) return;
  double v[MLK_NV];
#pragma unroll
  for (int k = 0; k < MLK_NV; ++k) v[k] = 0.0;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.n) {
    const double wi = ml_row64(a, i, z);
    const double zi = (double)__ldcg(&z[i]), qi = __ldcg(&a.q[i]), ri = __ldcg(&a.r[i]);
    a.w[i] = wi;
    v[0] += zi * ri;
    v[1] += zi * qi;
    v[2] += zi * wi;
    v[3] += zi;
    v[4] += ri * ri;
    v[5] += ri;
    v[6] += qi;
    v[7] += wi;
  }
  mlk_block_partials<MLK_NV>(v, part);
}
// block b sums partials b*256 .. b*256+255 (fixed order), NV values each
template <int NV>
static __global__ void __launch_bounds__(MLK_TPB) k_mlk_fold(int nparts, const double* __restrict__ in, double* out,
                                                      const MlkState* S) {
  if (S->done) return;
  double v[NV];
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = j < nparts ? in[(size_t)j * NV + k] : 0.0;
  mlk_block_partials<NV>(v, out);
}
// the FCG scalars and the stopping rule (k_mlcg's, after its reduce-and-gather)
static __global__ void k_mlk_rule(int n, int nparts, const double* part, MlkState* S) {
  if (S->done) return;
  double t[MLK_NV];
  mlk_totals<MLK_NV>(nparts, part, t);
  if (threadIdx.x != 0) return;
  const double dp = sqrt(t[4]);
  S->dp = dp;
  int reason = classify(dp, S->ttol, S->atol, S->rnorm0);
  const int its = S->its;
  if (!reason && S->stall_window > 0 && its > 0 && its % S->stall_window == 0) {
    if (dp > S->stall_ratio * S->dp_mark) reason = -20;
    else S->dp_mark = dp;
  }
  if (!reason) {
    const double m = S->nullsp ? t[3] / (double)n : 0.0;
    const double zr = t[0] - m * t[5], zq = t[1] - m * t[6], zw = t[2] - m * t[7];
    const double beta = its == 0 ? 0.0 : -zq / S->pq_old;
    const double pq = zw + 2.0 * beta * zq + beta * beta * S->pq_old;
    if (!(pq > 0.0)) {
      reason = pq == 0.0 ? 3 : -10;
    } else {
      S->m = m;
      S->beta = beta;
      S->alpha = zr / pq;
      S->pq_old = pq;
    }
  }
  if (reason) {
    S->reason = reason;
    S->done = 1;
  }
}
// p = (z - m) + beta p, q = w + beta q, x += alpha p, r -= alpha q, then level 0's first step
template <class ZT>
static __global__ void __launch_bounds__(MLK_TPB) k_mlk_update(MlArgs a, const ZT* __restrict__ z, const MlDevLevel* L0,
                                                        const MlkState* S) {
  if (S->done) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const double m = S->m, beta = S->beta, al = S->alpha;
  const double pi = ((double)__ldcg(&z[i]) - m) + beta * __ldcg(&a.p[i]);
  const double qi = __ldcg(&a.w[i]) + beta * __ldcg(&a.q[i]);
  const double ri = __ldcg(&a.r[i]) - al * qi;
  a.p[i] = pi;
  a.q[i] = qi;
  a.x[i] = __ldcg(&a.x[i]) + al * pi;
  a.r[i] = ri;
  mlk_start0(L0, a.bC, i, ri);
}
// end of an iteration: its += 1; the iteration cap stops the solve (KSP_DIVERGED_ITS)
static __global__ void k_mlk_next(MlkState* S) {
  if (S->done) return;
  S->its += 1;
  if (S->its >= S->maxit) {
    S->reason = -3;
    S->done = 1;
  }
}

// ---- true residual ||b - A x|| and the outcome in the status / result words
static __global__ void __launch_bounds__(MLK_TPB) k_mlk_true_resid(MlArgs a, double* part) {
  double v[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
    const double di = a.b[i] - ml_row64(a, i, (const double*)a.x);
    v[0] += di * di;
  }
  mlk_block_partials<1>(v, part);
}
static __global__ void k_mlk_finish(int nparts, const double* part, const MlkState* S, int* status, double* dout) {
  double t[1];
  mlk_totals<1>(nparts, part, t);
  if (threadIdx.x == 0) {
    dout[0] = sqrt(t[0]);
    dout[1] = S->dp;
    dout[2] = S->sn;
    status[0] = S->reason;
    status[1] = S->its;
  }
}

}  // namespace gpu
}  // namespace dpm
