// Flexible conjugate gradients preconditioned by one aggregation-multigrid V-cycle, as one
// persistent cooperative kernel: the multilevel form of the pressure solve.
//
// Krylov vectors, the operator used for w = A z, and all reductions are FP64; the V-cycle runs
// in FP32 on the hierarchy of dopamine_b200/csrc/host/multilevel.cpp (it is preconditioner work
// only, so its rounding changes the Krylov path, not the solution the stopping rule accepts).
// V-cycle, for levels l = 0 .. nlev-1 and the directly solved coarsest level C:
//
//   down:  x_l = Cheb_k(A_l, b_l, 0);  b_{l+1} = T^T (b_l - A_l x_l)
//   C:     x_C = A_C^-1 b_C            (dense FP32 inverse, one warp per row)
//   up:    x_l = Cheb_k(A_l, b_l, x_l + oc T x_{l+1})
//
// Cheb_k: k steps of Chebyshev iteration on D^-1 A_l over [lmax/10, lmax] (Saad, Iterative
// Methods, alg. 12.1), T the piecewise-constant prolongation of the aggregates, oc the
// over-correction of the unsmoothed-aggregation coarse correction.  The smoother reads each
// level as D^-1 A = G + S: off-diagonal entries only, scaled by the row's diagonal and stored in
// FP32 or in binary16 (SV = unsigned short: the half's bits), with the diagonal term g_i chosen
// so that every stored row keeps the exact row sum; the level's right-hand side is kept scaled
// (b / a_ii).  A sweep then reads columns, scaled values, g, b, x and d - no diagonal entry and
// no 1/diagonal - and the restriction multiplies a member row's scaled residual back by a_ii.  Every smoothing step reads
// neighbour values written by the step before, so each step ends at a grid barrier; the first
// step of each down-smoothing is fused into the restriction that produces its right-hand side,
// and the prolongation into the first up-smoothing step, so a V-cycle costs 2 k nlev + 1
// barriers.  The FCG(1) recurrences, null-space handling and stopping rule are those of the
// two-level kernel (fcg.cuh); the stopping rule is the reference's, src/solver/
// pressure_backend_petsc.c:816-876.
#pragma once
#include <cuda_fp16.h>

#include "fcg.cuh"

namespace dpm {
namespace gpu {

constexpr int ML_TPB = 512;
constexpr int ML_RB = 10;                  // blocks per lane in the reduce-gather: grids up to 320 blocks
constexpr int ML_MAX_GRID = 32 * ML_RB;
constexpr int ML_LEVELS = 12;
constexpr int ML_DEG = 8;

struct MlDevLevel {
  int n, W, M, n_next;
  int MP;            // power of two >= M, <= 32
  int lgMP;          // log2 MP
  int lgG;           // log2 of the lanes that share one row of a smoothing step
  int lgGR;          // log2 of the lanes that share one member row of the restriction
  int rows_per_pass; // lgG == 0: rows a lane takes per pass (1..2)
  const int* col;    // [W][n] off-diagonal columns, padded with the own row (W = off-diagonal width)
  const void* sv;    // [W][n] s_ij = a_ij / a_ii, FP32 or binary16 bits (padding 0)
  const float* g;    // [n] diagonal term of the scaled row (1 up to the stored entries' rounding)
  const float* diag; // [n] a_ii
  const float* dinv; // [n] 1 / a_ii
  const int* agg;    // [n]
  const int* mem;    // [M][n_next], -1 padded
  float* b;          // [n] scaled right-hand side b / a_ii of this level
  float* x0;         // [n] iterate, two buffers
  float* x1;
  float* d;          // [n] Chebyshev direction
  float inv_theta;   // first Chebyshev step: d = D^-1 r / theta
  float c1[ML_DEG];  // step j >= 1: d = c1[j] d + c2[j] D^-1 r
  float c2[ML_DEG];
};

struct MlArgs {
  int n, WA, maxit, nullsp, guess_zero, nlev, degree, nC;
  const int* col;         // FP64 fine operator [WA][n]
  const double* val;
  const MlDevLevel* lv;   // [nlev]
  const float* cinv;      // [nC][nC]
  float* bC;              // [nC]
  float* xC;              // [nC]
  float oc;
  const double* b;
  double* x;
  double *r, *p, *q, *w;  // [n]
  double* partials;       // [2][grid][FCG_SLOT]
  unsigned* bar;
  int* status;            // [0] reason, [1] iterations, [2] barrier timeout, [3] poll limit (0: default)
  double* dout;           // [0] true residual, [1] last ||r||, [2] ||b'||
  double rtol, atol;
  int stall_window;        // > 0: stop with reason -20 when ||r|| > stall_ratio * ||r|| of a window earlier
  double stall_ratio;
  // learned term: gamma * omega .* D^-1 r added to the last fine-level smoothing step
  // (omega [n] in this numbering; gamma = 0: off)
  const float* omega;
  float gamma;
  // training-sample recording, as the two-level kernel does it: every rec_stride-th iteration,
  // slot rec_base + its / rec_stride (< rec_max) receives r, z, u = D^-1 r and x at position
  // pinv[i] (the learned term's part numbering).  rec_stride = 0: off.
  int rec_stride, rec_base, rec_max;
  const int* pinv;
  double *rec_r, *rec_z, *rec_u, *rec_x;
};

// Row products over padded ELL rows of runtime width, in chunks of ML_CHUNK entries: all column
// indices of a chunk are loaded, then all gathered values, then the products are summed in
// column-slot order (the same order as a plain loop), so the loads of a chunk are in flight
// together instead of one dependent load pair per entry.
constexpr int ML_CHUNK = 8;

__device__ __forceinline__ float ml_sval(const float* p) { return __ldg(p); }
__device__ __forceinline__ float ml_sval(const unsigned short* p) { return __half2float(__ushort_as_half(__ldg(p))); }

// Partial sum of s_ij x_j over the off-diagonal entries k = sub, sub + G, sub + 2G, ... of row i
// (G lanes share a row; G = 1: the whole row).  PRO: the iterate is the prolonged x + oc T x_c,
// formed on the fly.
template <class SV, bool PRO>
__device__ __forceinline__ float ml_part(const MlDevLevel& L, int i, const float* x, const float* xc, float oc,
                                         int G, int sub) {
  const SV* sv = static_cast<const SV*>(L.sv);
  float s = 0.0f;
  for (int k0 = sub; k0 < L.W; k0 += G * ML_CHUNK) {
    int c[ML_CHUNK];
    float v[ML_CHUNK], xv[ML_CHUNK];
#pragma unroll
    for (int u = 0; u < ML_CHUNK; ++u) {
      const int k = k0 + u * G;
      const size_t e = (size_t)k * L.n + i;
      c[u] = k < L.W ? __ldg(&L.col[e]) : i;
      v[u] = k < L.W ? ml_sval(&sv[e]) : 0.0f;
    }
    if (PRO) {
      int g[ML_CHUNK];
#pragma unroll
      for (int u = 0; u < ML_CHUNK; ++u) {
        g[u] = __ldg(&L.agg[c[u]]);
        xv[u] = __ldcg(&x[c[u]]);
      }
#pragma unroll
      for (int u = 0; u < ML_CHUNK; ++u) xv[u] = fmaf(oc, __ldcg(&xc[g[u]]), xv[u]);
    } else {
#pragma unroll
      for (int u = 0; u < ML_CHUNK; ++u) xv[u] = __ldcg(&x[c[u]]);
    }
#pragma unroll
    for (int u = 0; u < ML_CHUNK; ++u) s = fmaf(v[u], xv[u], s);
  }
  return s;
}

// One Chebyshev step on level L for every row, in the scaled form: rs = b - g x_in - S x_in
// (= D^-1 (b - A x_in)), d = c1 d + c2 rs, x_out = x_in + d.  PRO: the first step after the coarse
// correction, on the prolonged iterate x_in + oc T x_c, with d = rs / theta.  On large levels
// each lane takes R rows per pass so that their loads are in flight together.  om: the learned
// term gam * omega_i * b_i (b scaled) added to x_out.
template <class SV, bool PRO, int R>
__device__ __forceinline__ void ml_sweep_rows(const MlDevLevel& L, float c1, float c2, const float* xi, float* xo,
                                              const float* xc, float oc, int g0, int T, const float* om, float gam) {
  for (int i0 = g0; i0 < L.n; i0 += R * T) {
    int ii[R];
    float acc[R], b[R], gg[R], x[R], dd[R];
#pragma unroll
    for (int h = 0; h < R; ++h) {
      const int i = i0 + h * T;
      ii[h] = i < L.n ? i : i0;  // an absent row repeats row i0 (loads in bounds, no store)
    }
#pragma unroll
    for (int h = 0; h < R; ++h) acc[h] = ml_part<SV, PRO>(L, ii[h], xi, xc, oc, 1, 0);
#pragma unroll
    for (int h = 0; h < R; ++h) {
      b[h] = __ldcg(&L.b[ii[h]]);
      gg[h] = __ldg(&L.g[ii[h]]);
      x[h] = __ldcg(&xi[ii[h]]);
      dd[h] = PRO ? 0.0f : __ldcg(&L.d[ii[h]]);
      if (PRO) x[h] = fmaf(oc, __ldcg(&xc[__ldg(&L.agg[ii[h]])]), x[h]);
    }
#pragma unroll
    for (int h = 0; h < R; ++h) {
      const float rs = b[h] - fmaf(gg[h], x[h], acc[h]);
      const float d = PRO ? L.inv_theta * rs : fmaf(c1, dd[h], c2 * rs);
      if (i0 + h * T < L.n) {
        L.d[ii[h]] = d;
        xo[ii[h]] = x[h] + d + (om ? gam * __ldg(&om[ii[h]]) * b[h] : 0.0f);
      }
    }
  }
}

// One Chebyshev step on level L for every row (see ml_sweep_rows).  Rows are spread over 2^lgG
// lanes on small levels (partial sums combined by shuffles); on large levels each lane takes up
// to 4 rows per pass (rows_per_pass).
template <class SV, bool PRO>
__device__ __forceinline__ void ml_sweep(const MlDevLevel& L, float c1, float c2, const float* xi, float* xo,
                                         const float* xc, float oc, int g0, int T, const float* om = nullptr,
                                         float gam = 0.0f) {
  if (L.lgG == 0) {
    switch (L.rows_per_pass) {
      case 1: ml_sweep_rows<SV, PRO, 1>(L, c1, c2, xi, xo, xc, oc, g0, T, om, gam); return;
      case 2: ml_sweep_rows<SV, PRO, 2>(L, c1, c2, xi, xo, xc, oc, g0, T, om, gam); return;
      case 3: ml_sweep_rows<SV, PRO, 3>(L, c1, c2, xi, xo, xc, oc, g0, T, om, gam); return;
      default: ml_sweep_rows<SV, PRO, 4>(L, c1, c2, xi, xo, xc, oc, g0, T, om, gam); return;
    }
  }
  const int lane = threadIdx.x & 31;
  const int G = 1 << L.lgG, total = L.n << L.lgG;
  for (int u0 = g0 - lane; u0 < total; u0 += T) {
    const int u = u0 + lane;
    const bool ok = u < total;
    const int i = ok ? u >> L.lgG : 0, sub = u & (G - 1);
    float acc = ok ? ml_part<SV, PRO>(L, i, xi, xc, oc, G, sub) : 0.0f;
    for (int o = G >> 1; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (ok && sub == 0) {
      const float b = __ldcg(&L.b[i]);
      float x = __ldcg(&xi[i]);
      if (PRO) x = fmaf(oc, __ldcg(&xc[__ldg(&L.agg[i])]), x);
      const float rs = b - fmaf(__ldg(&L.g[i]), x, acc);
      const float d = PRO ? L.inv_theta * rs : fmaf(c1, __ldcg(&L.d[i]), c2 * rs);
      L.d[i] = d;
      xo[i] = x + d + (om ? gam * __ldg(&om[i]) * b : 0.0f);
    }
  }
}

template <class V>
__device__ __forceinline__ double ml_row64(const MlArgs& a, int i, const V* x) {
  double s = 0.0;
  for (int k0 = 0; k0 < a.WA; k0 += ML_CHUNK) {
    int c[ML_CHUNK];
    double v[ML_CHUNK], xv[ML_CHUNK];
#pragma unroll
    for (int u = 0; u < ML_CHUNK; ++u) {
      const size_t e = (size_t)(k0 + u) * a.n + i;
      c[u] = k0 + u < a.WA ? __ldg(&a.col[e]) : i;
      v[u] = k0 + u < a.WA ? __ldg(&a.val[e]) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < ML_CHUNK; ++u) xv[u] = (double)__ldcg(&x[c[u]]);
#pragma unroll
    for (int u = 0; u < ML_CHUNK; ++u) s = fma(v[u], xv[u], s);
  }
  return s;
}

// SV: value type of the smoother's scaled off-diagonals, float or unsigned short (binary16 bits)
template <class SV>
__global__ void __launch_bounds__(ML_TPB, 2) k_mlcg(MlArgs a) {
  __shared__ MlDevLevel s_lv[ML_LEVELS];
  __shared__ double s_gat[1];
  {
    const int words = (int)(sizeof(MlDevLevel) / sizeof(int)) * a.nlev;
    const int* src = reinterpret_cast<const int*>(a.lv);
    int* dst = reinterpret_cast<int*>(s_lv);
    for (int k = threadIdx.x; k < words; k += blockDim.x) dst[k] = src[k];
  }
  __syncthreads();
  const int g0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int T = gridDim.x * blockDim.x;
  const int n = a.n, nlev = a.nlev, deg = a.degree;
  unsigned gen = 0;

  // first Chebyshev step of level 0 from the residual r (or the coarse right-hand side when
  // the fine level is itself the coarsest)
  auto start_level0 = [&](int i, double ri) {
    if (nlev > 0) {
      const MlDevLevel& L = s_lv[0];
      const float bi = (float)ri * __ldg(&L.dinv[i]);  // scaled right-hand side
      const float di = L.inv_theta * bi;
      L.b[i] = bi;
      L.d[i] = di;
      L.x0[i] = di;
    } else {
      a.bC[i] = (float)ri;
    }
  };

  // ---- b' = b - mean(b), r = b' - A x
  double mb = 0.0;
  {
    double v[1] = {0.0}, t[1];
    for (int i = g0; i < n; i += T) {
      if (a.guess_zero) a.x[i] = 0.0;
      v[0] += a.b[i];
    }
    if (!grid_reduce_gather<1, 0, ML_RB>(v, a.partials, a.bar, gen, a.status, t, s_gat)) return;  // publishes x
    mb = a.nullsp ? t[0] / (double)n : 0.0;
  }
  double dp, sn;
  {
    double v[2] = {0.0, 0.0}, t[2];
    for (int i = g0; i < n; i += T) {
      const double bp = a.b[i] - mb;
      const double ri = bp - ml_row64(a, i, (const double*)a.x);
      a.r[i] = ri;
      a.p[i] = 0.0;
      a.q[i] = 0.0;
      v[0] += ri * ri;
      v[1] += bp * bp;
      start_level0(i, ri);
    }
    if (!grid_reduce_gather<2, 0, ML_RB>(v, a.partials, a.bar, gen, a.status, t, s_gat)) return;
    dp = sqrt(t[0]);
    sn = sqrt(t[1]);
  }
  const double rnorm0 = a.guess_zero ? dp : (sn == 0.0 ? dp : sn);
  const double ttol = fmax(a.rtol * rnorm0, a.atol);
  int reason = classify(dp, ttol, a.atol, rnorm0);
  int its = 0;
  double pq_old = 1.0, dp_mark = dp;
  unsigned cur_mask = 0;  // bit l: level l's down-smoothed iterate is in x1
  while (!reason) {
    if (its >= a.maxit) { reason = -3; break; }
    // ---- V-cycle, down: the remaining k-1 smoothing steps, then restriction (+ the next
    // level's first step)
    for (int l = 0; l < nlev; ++l) {
      const MlDevLevel& L = s_lv[l];
      int cur = 0;
      for (int j = 1; j < deg; ++j) {
        const float* xi = cur ? L.x1 : L.x0;
        float* xo = cur ? L.x0 : L.x1;
        ml_sweep<SV, false>(L, L.c1[j], L.c2[j], xi, xo, nullptr, 0.0f, g0, T);
        cur ^= 1;
        if (!grid_barrier(a.bar, gen, a.status)) return;
      }
      cur_mask = (cur_mask & ~(1u << l)) | ((unsigned)cur << l);
      const float* xf = cur ? L.x1 : L.x0;
      const bool last = l + 1 == nlev;
      // lanes [aggregate][member slot][2^lgGR lanes per member row]: a lane forms its share of a
      // member row's residual a_ii (b_i - g_i x_i - (S x)_i) (scaled form times the diagonal),
      // the butterfly over the aggregate's 2^(lgMP + lgGR) lanes adds up sum_i r_i in a fixed order
      const int lgR = L.lgMP + L.lgGR, span = 1 << lgR, GR = 1 << L.lgGR;
      const int total = L.n_next << lgR;
      const int lane = threadIdx.x & 31;
      for (int u0 = g0 - lane; u0 < total; u0 += T) {
        const int u = u0 + lane;
        const bool ok = u < total;
        const int c = u >> lgR, m = (u >> L.lgGR) & (L.MP - 1), sub = u & (GR - 1);
        float sres = 0.0f;
        if (ok && m < L.M) {
          const int i = __ldg(&L.mem[(size_t)m * L.n_next + c]);
          if (i >= 0) {
            sres = -ml_part<SV, false>(L, i, xf, nullptr, 0.0f, GR, sub);
            if (sub == 0) sres += __ldcg(&L.b[i]) - __ldg(&L.g[i]) * __ldcg(&xf[i]);
            sres *= __ldg(&L.diag[i]);
          }
        }
        for (int o = span >> 1; o > 0; o >>= 1) sres += __shfl_xor_sync(0xffffffffu, sres, o);
        if (ok && (u & (span - 1)) == 0) {
          if (last) {
            a.bC[c] = sres;
          } else {
            const MlDevLevel& N = s_lv[l + 1];
            const float bs = sres * __ldg(&N.dinv[c]);
            const float di = N.inv_theta * bs;
            N.b[c] = bs;
            N.d[c] = di;
            N.x0[c] = di;
          }
        }
      }
      if (!grid_barrier(a.bar, gen, a.status)) return;
    }
    // ---- coarsest level: x_C = A_C^-1 b_C, one warp per row
    {
      const int lane = threadIdx.x & 31;
      const int gw = g0 >> 5, nw = T >> 5;
      for (int row = gw; row < a.nC; row += nw) {
        float s = 0.0f;
        for (int k0 = lane; k0 < a.nC; k0 += 32 * ML_CHUNK) {
          float cv[ML_CHUNK], bv[ML_CHUNK];
#pragma unroll
          for (int u = 0; u < ML_CHUNK; ++u) {
            const int k = k0 + 32 * u;
            cv[u] = k < a.nC ? __ldg(&a.cinv[(size_t)row * a.nC + k]) : 0.0f;
            bv[u] = k < a.nC ? __ldcg(&a.bC[k]) : 0.0f;
          }
#pragma unroll
          for (int u = 0; u < ML_CHUNK; ++u) s = fmaf(cv[u], bv[u], s);
        }
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) a.xC[row] = s;
      }
      if (!grid_barrier(a.bar, gen, a.status)) return;
    }
    // ---- up: prolongation fused into the first of k smoothing steps
    const float* xcoarse = a.xC;
    for (int l = nlev - 1; l >= 0; --l) {
      const MlDevLevel& L = s_lv[l];
      int cur = (cur_mask >> l) & 1u;
      const float* om = (l == 0 && a.gamma != 0.0f) ? a.omega : nullptr;  // learned term: last fine step
      ml_sweep<SV, true>(L, 0.0f, 0.0f, cur ? L.x1 : L.x0, cur ? L.x0 : L.x1, xcoarse, a.oc, g0, T,
                         deg == 1 ? om : nullptr, a.gamma);
      cur ^= 1;
      if (!grid_barrier(a.bar, gen, a.status)) return;
      for (int j = 1; j < deg; ++j) {
        ml_sweep<SV, false>(L, L.c1[j], L.c2[j], cur ? L.x1 : L.x0, cur ? L.x0 : L.x1, nullptr, 0.0f, g0, T,
                            j == deg - 1 ? om : nullptr, a.gamma);
        cur ^= 1;
        if (!grid_barrier(a.bar, gen, a.status)) return;
      }
      xcoarse = cur ? L.x1 : L.x0;
    }
    const float* z = xcoarse;  // level 0's smoothed iterate (x_C when there is no smoothed level)
    // ---- w = A z and the sums
    double v[FCG_NV], t[FCG_NV];
#pragma unroll
    for (int k = 0; k < FCG_NV; ++k) v[k] = 0.0;
    if (a.rec_stride > 0 && its % a.rec_stride == 0 && a.rec_base + its / a.rec_stride < a.rec_max && nlev > 0) {
      const size_t off = (size_t)(a.rec_base + its / a.rec_stride) * n;
      const MlDevLevel& L0 = s_lv[0];
      for (int i = g0; i < n; i += T) {
        const size_t o = off + __ldg(&a.pinv[i]);
        a.rec_r[o] = __ldcg(&a.r[i]);
        a.rec_z[o] = (double)__ldcg(&z[i]);
        a.rec_u[o] = (double)__ldcg(&L0.b[i]);  // D^-1 r: the level's scaled right-hand side
        a.rec_x[o] = __ldcg(&a.x[i]);
      }
    }
    for (int i0 = g0; i0 < n; i0 += 2 * T) {  // two rows per pass: their loads in flight together
      const int i1 = i0 + T;
      const bool h1 = i1 < n;
      const int j1 = h1 ? i1 : i0;
      const double w0 = ml_row64(a, i0, z), w1 = ml_row64(a, j1, z);
      const double z0 = (double)__ldcg(&z[i0]), z1 = (double)__ldcg(&z[j1]);
      const double q0 = __ldcg(&a.q[i0]), q1 = __ldcg(&a.q[j1]);
      const double r0 = __ldcg(&a.r[i0]), r1 = __ldcg(&a.r[j1]);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (h == 1 && !h1) break;
        const double zi = h ? z1 : z0, wi = h ? w1 : w0, qi = h ? q1 : q0, ri = h ? r1 : r0;
        a.w[h ? i1 : i0] = wi;
        v[0] += zi * ri;
        v[1] += zi * qi;
        v[2] += zi * wi;
        v[3] += zi;
        v[4] += ri * ri;
        v[5] += ri;
        v[6] += qi;
        v[7] += wi;
      }
    }
    if (!grid_reduce_gather<FCG_NV, 0, ML_RB>(v, a.partials, a.bar, gen, a.status, t, s_gat)) return;
    dp = sqrt(t[4]);
    reason = classify(dp, ttol, a.atol, rnorm0);
    if (reason) break;
    if (a.stall_window > 0 && its > 0 && its % a.stall_window == 0) {
      if (dp > a.stall_ratio * dp_mark) { reason = -20; break; }
      dp_mark = dp;
    }
    const double m = a.nullsp ? t[3] / (double)n : 0.0;
    const double zr = t[0] - m * t[5], zq = t[1] - m * t[6], zw = t[2] - m * t[7];
    const double beta = its == 0 ? 0.0 : -zq / pq_old;
    const double pq = zw + 2.0 * beta * zq + beta * beta * pq_old;
    if (!(pq > 0.0)) { reason = pq == 0.0 ? 3 : -10; break; }
    const double al = zr / pq;
    for (int i = g0; i < n; i += T) {
      const double pi = ((double)__ldcg(&z[i]) - m) + beta * __ldcg(&a.p[i]);
      const double qi = __ldcg(&a.w[i]) + beta * __ldcg(&a.q[i]);
      const double ri = __ldcg(&a.r[i]) - al * qi;
      a.p[i] = pi;
      a.q[i] = qi;
      a.x[i] = __ldcg(&a.x[i]) + al * pi;
      a.r[i] = ri;
      start_level0(i, ri);
    }
    pq_old = pq;
    ++its;
    if (!grid_barrier(a.bar, gen, a.status)) return;
  }
  // ---- true residual ||b - A x||
  if (!grid_barrier(a.bar, gen, a.status)) return;
  double v1[1] = {0.0}, t1[1];
  for (int i = g0; i < n; i += T) {
    const double di = a.b[i] - ml_row64(a, i, (const double*)a.x);
    v1[0] += di * di;
  }
  if (!grid_reduce_gather<1, 0, ML_RB>(v1, a.partials, a.bar, gen, a.status, t1, s_gat)) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.dout[0] = sqrt(t1[0]);
    a.dout[1] = dp;
    a.dout[2] = sn;
    a.status[0] = reason;
    a.status[1] = its;
  }
}

}  // namespace gpu
}  // namespace dpm
