// Flexible conjugate gradients with a two-level (part-local Chebyshev + coarse) preconditioner,
// as one persistent cooperative kernel: the "chosen form" pressure solve.
//
// Cells are renumbered into P compact parts, one per thread block (dopamine_b200/csrc/host/
// twolevel.cpp); part b owns rows [b*C, b*C + size_b).  Per iteration (FCG(1), Notay 2000):
//
//   z  = y_b + S_b(r - A Z y)  y = E^-1 c, c = Z^T r (one value per part, all-gathered);
//                              S_b: `degree` Chebyshev steps on D^-1 A_bb in shared memory (FP32);
//                              A Z y needs y of the neighbouring parts only at part-boundary
//                              rows (deflated two-level form; without `deflate`: S_b(r))
//   grid barrier               (z is read by neighbour parts)
//   w  = A z                   FP64, global ELL
//   all-reduce                 z.r, z.q, z.w, r.r and the null-space sums; all-gather per part
//                              sum r, sum w, sum q
//   beta = -z'.q / (p.q)_old,  p.q = z'.w + 2 beta z'.q + beta^2 (p.q)_old,  alpha = z'.r / p.q
//   p = z' + beta p,  q = w + beta q,  x += alpha p,  r -= alpha q,  c = sum r - alpha (sum w + beta sum q)
//
// so an iteration has one barrier and one all-reduce, like the Jacobi-PCG kernel, while the
// preconditioner works without any grid-wide wait.  The stopping rule is the reference's
// (unpreconditioned ||r|| <= max(rtol ||b'||, atol), src/solver/pressure_backend_petsc.c:816-876),
// tested on the current residual at the top of each iteration.  Krylov vectors and reductions
// are FP64; the part-local smoother runs in FP32 and the coarse solve uses FP32 rows of E^-1
// with FP64 sums (both are preconditioner work only).
#pragma once
#include "pcg.cuh"

namespace dpm {
namespace gpu {

constexpr int FCG_TPB = 1024;
constexpr int FCG_SLOT = 16;  // doubles per block in the reduce/gather buffer
constexpr int FCG_NV = 8;     // reduced sums
constexpr int FCG_NG = 3;     // gathered per-part values
constexpr int FCG_MAX_GRID = 160;  // largest grid of the two-level kernel's reduce-gather (5 blocks per lane)

struct FcgArgs {
  int n, P, C, WL, maxit, nullsp, guess_zero, degree;
  const int* perm;        // perm[new] = old
  const int* col;         // [WA][n] new numbering, padded (self, 0)
  const double* val;      // [WA][n]
  const double* dinv;     // [n] new numbering
  const unsigned* lpk;    // [WL][n] local column (low 16 bits) | bf16 a_ij / a_ii (high 16 bits)
  const double* einv_nb;  // [P][NB][P] E^-1 rows of each part's slots (slot 0 = the part)
  int NB, deflate;        // slots per part; 1 = smooth r - A Z y instead of r (deflated form)
  const float* srow;      // [n] intra-part row sum
  const int* xoff;        // [n+1] cross-part couplings of each row
  const unsigned char* xslot;
  const float* xval;
  const double* b;        // right-hand side, original numbering
  double* x;              // guess in / solution out, original numbering
  double* xs;             // [n] scratch, new numbering
  double* zs;             // [n] scratch, new numbering
  double* partials;       // [2][P][FCG_SLOT]
  unsigned* bar;          // [0] arrival counter
  int* status;            // [0] reason, [1] iterations, [2] barrier timeout, [3] poll limit (0: default)
  double* dout;           // [0] true residual, [1] last ||r||, [2] ||b'||
  double rtol, atol;
  float theta, delta;     // Chebyshev interval [theta - delta, theta + delta] of D^-1 A_bb
  // learned term gamma * omega .* D^-1 rho0 added to the smoother output (omega [n], new numbering)
  const float* omega;
  float gamma;
  // training-sample recording: every rec_stride-th iteration, slot rec_base + its / rec_stride
  // (< rec_max) receives r, the preconditioned residual z, u = D^-1 rho0 and x ([slot][n], new
  // numbering).  rec_stride = 0: off.
  int rec_stride, rec_base, rec_max;
  double *rec_r, *rec_z, *rec_u, *rec_x;
  int stall_window;       // > 0: stop with reason -20 when ||r|| > stall_ratio * ||r|| of a window earlier
  double stall_ratio;     // default 0.9 (less than 10 % reduction over the window)
  // precision form: FP32 copy of the operator values and FP32 z for w = A z (products summed in
  // FP64); the initial and the final residual stay FP64.  inner_rel > 0: also stop once
  // ||r|| <= inner_rel * ||r_0|| (one pass of the outer FP64 defect correction).
  const float* val32;
  float* zs32;
  double inner_rel;
  // diagnostics: non-null = block 0 adds the globaltimer nanoseconds of each phase of an iteration
  // to phase[0..5] (coarse values, smoother, z published + barrier, w = A z and the sums, reduce and
  // gather, update) and counts the iterations in phase[7]
  double* phase;
};

__device__ __forceinline__ unsigned long long fcg_clock() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded grid barrier on the same monotonic counter as grid_allreduce (one arrival per block).
__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned& gen, int* status) {
  __shared__ int s_okb;
  __syncthreads();
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
    s_okb = ok;
  }
  __syncthreads();
  gen = gen + 1u;
  return s_okb != 0;
}

// All-reduce of the first NV of v (deterministic, as grid_allreduce) plus an all-gather of the
// block totals of the last NG into gat[k*P + block] (shared memory: every block gets every
// block's values).  v holds per-thread partials of all NV + NG values.  All reductions of the
// FCG kernels go through here so that every generation uses the same slot layout of the
// double-buffered partials.  Warp k reduces value k, both over the block's warps before the
// barrier and over the blocks after it, with all of a lane's loads issued together; the order
// of every sum is fixed (lane-ordered partials, then a shuffle tree), so results do not depend
// on timing.  Supports up to 32 * RB blocks (RB: blocks per lane in the post-barrier read).
template <int NV, int NG, int RB = FCG_MAX_GRID / 32>
__device__ __forceinline__ bool grid_reduce_gather(double (&v)[NV + NG], double* partials, unsigned* bar,
                                                   unsigned& gen, int* status, double (&res)[NV], double* gat) {
  constexpr int NT = NV + NG;
  static_assert(NT <= FCG_SLOT, "slot too small");
  __shared__ double sh[32][NT];
  __shared__ double shr[NV > 0 ? NV : 1];
  __shared__ int s_ok;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int P = gridDim.x;
  double* buf = partials + (size_t)(gen & 1u) * FCG_SLOT * P;
#pragma unroll
  for (int k = 0; k < NT; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NT; ++k) sh[w][k] = v[k];
  __syncthreads();
  if (w < NT) {  // warp w: value w over the block's warps
    double t = lane < nw ? sh[lane][w] : 0.0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (lane == 0) buf[blockIdx.x * FCG_SLOT + w] = t;
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
    s_ok = ok && P <= 32 * RB;
    if (P > 32 * RB) atomicExch(&status[2], 2);
  }
  __syncthreads();
  const bool ok = s_ok != 0;
  if (ok) {
    if (w < NV) {  // warp w: value w over the blocks, lane l sums blocks l, l + 32, ... in order
      double pv[RB];
#pragma unroll
      for (int h = 0; h < RB; ++h) pv[h] = lane + 32 * h < P ? __ldcg(&buf[(lane + 32 * h) * FCG_SLOT + w]) : 0.0;
      double u = 0.0;
#pragma unroll
      for (int h = 0; h < RB; ++h) u += pv[h];
      for (int o = 16; o > 0; o >>= 1) u += __shfl_down_sync(0xffffffffu, u, o);
      if (lane == 0) shr[w] = u;
    }
    if (NG > 0) {  // the per-block values, read by the threads after the first NV warps
      const int t0 = NV * 32 < (int)blockDim.x ? NV * 32 : 0;
      for (int idx = (int)threadIdx.x - t0; idx >= 0 && idx < NG * P; idx += blockDim.x - t0) {
        const int k = idx / P, b = idx - k * P;
        gat[idx] = __ldcg(&buf[b * FCG_SLOT + NV + k]);
      }
    }
  }
  __syncthreads();
  gen = gen + 1u;
#pragma unroll
  for (int k = 0; k < NV; ++k) res[k] = ok ? shr[k] : 0.0;
  return ok;
}

// Row i (new numbering) of A times v, global ELL with fixed width WT (0: runtime width <= 16);
// VA / VV: value types of the operator and of the vector (double, or float in the precision form).
template <int WT, class VA, class VV>
__device__ __forceinline__ double fcg_row(const FcgArgs& a, const VA* val, int WA, int i, const VV* v) {
  const int n = a.n;
  constexpr int W = WT > 0 ? WT : 16;
  const int wa = WT > 0 ? WT : WA;
  int c[W];
#pragma unroll
  for (int w = 0; w < W; ++w)
    if (w < wa) c[w] = __ldg(&a.col[w * n + i]);
  double x[W];
#pragma unroll
  for (int w = 0; w < W; ++w)
    if (w < wa) x[w] = (double)__ldcg(&v[c[w]]);
  double s = 0.0;
#pragma unroll
  for (int w = 0; w < W; ++w)
    if (w < wa) s += (double)__ldcg(&val[w * n + i]) * x[w];
  return s;
}

// Dynamic shared memory of the kernel for a given set-up.
inline size_t fcg_smem_bytes(int P, int C, int WL, int NB) {
  return (size_t)P * sizeof(double)                     // gathered sums r
         + (size_t)NB * P * sizeof(float)                // E^-1 rows of the slots (FP32)
         + (size_t)FCG_NG * P * sizeof(double)           // gather landing area
         + (size_t)3 * C * sizeof(double)                // own x, p, q
         + (size_t)C * sizeof(float)                     // own 1/diag (FP32, smoother)
         + (size_t)WL * C * sizeof(unsigned)             // packed local rows
         + (size_t)2 * C * sizeof(float);                // Chebyshev direction, double-buffered
}

// CPT: cells per thread (C <= CPT * FCG_TPB); WT: global row width (7 for hexahedra, 0 = runtime).
template <int CPT, int WT, bool MIXED>
__global__ void __launch_bounds__(FCG_TPB, 1) k_fcg(FcgArgs a, int WA) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int P = a.P, C = a.C, WL = a.WL, n = a.n;
  double* s_c = reinterpret_cast<double*>(smem);          // [P] c = Z^T r
  double* s_gat = s_c + P;                                 // [NG][P]
  double* s_x = s_gat + FCG_NG * P;                        // [C] own x
  double* s_p = s_x + C;                                   // [C] own p
  double* s_q = s_p + C;                                   // [C] own q
  float* s_dinv = reinterpret_cast<float*>(s_q + C);       // [C]
  unsigned* s_lpk = reinterpret_cast<unsigned*>(s_dinv + C);  // [WL][C]
  float* s_d0 = reinterpret_cast<float*>(s_lpk + (size_t)WL * C);  // [C]
  float* s_d1 = s_d0 + C;                                  // [C]
  float* s_er = s_d1 + C;                                  // [NB][P] E^-1 rows of this part's slots (FP32)
  __shared__ double s_yn[32];  // coarse values of this part's slots (slot 0 = own part)

  constexpr int LW = WT > 0 ? WT - 1 : 16;  // unrolled bound of the local row width
  const int b = blockIdx.x;
  const int base = b * C;
  const int size = min(C, n - base);
  unsigned gen = 0;

  // ---- stage the part's local operator and E^-1 row
  for (int s = 0; s < WL; ++s)
    for (int l = threadIdx.x; l < size; l += blockDim.x) s_lpk[s * C + l] = a.lpk[(size_t)s * n + base + l];
  for (int j = threadIdx.x; j < a.NB * P; j += blockDim.x) s_er[j] = (float)a.einv_nb[(size_t)b * a.NB * P + j];

  // own-cell state: r in registers; x, p, q and the FP32 1/diag in shared memory
  double rr[CPT];
#define OWN(k) (threadIdx.x + (k) * FCG_TPB < size)
#pragma unroll
  for (int k = 0; k < CPT; ++k) {
    const int l = threadIdx.x + k * FCG_TPB;
    rr[k] = 0.0;
    if (OWN(k)) {
      s_p[l] = 0.0;
      s_q[l] = 0.0;
      const int i = base + l;
      const int o = __ldg(&a.perm[i]);
      const double x0 = a.guess_zero ? 0.0 : a.x[o];
      s_x[l] = x0;
      rr[k] = a.b[o];  // b for now
      s_dinv[l] = (float)__ldg(&a.dinv[i]);
      a.xs[i] = x0;
    }
  }
  // ---- b' = b - mean(b) (null space), r = b' - A x, c = Z^T r
  double mb = 0.0;
  {
    double v[1] = {0.0}, t[1];
#pragma unroll
    for (int k = 0; k < CPT; ++k)
      if (OWN(k)) v[0] += rr[k];
    if (!grid_reduce_gather<1, 0>(v, a.partials, a.bar, gen, a.status, t, s_gat)) return;  // publishes xs
    mb = a.nullsp ? t[0] / (double)n : 0.0;
  }
  double v2[2 + 1], t2[2];
#pragma unroll
  for (int k = 0; k < 3; ++k) v2[k] = 0.0;
#pragma unroll
  for (int k = 0; k < CPT; ++k)
    if (OWN(k)) {
      const int i = base + threadIdx.x + k * FCG_TPB;
      const double bp = rr[k] - mb;
      rr[k] = bp - fcg_row<WT>(a, a.val, WA, i, a.xs);
      v2[0] += rr[k] * rr[k];
      v2[1] += bp * bp;
      v2[2] += rr[k];  // gathered: part sum of r
    }
  if (!grid_reduce_gather<2, 1>(v2, a.partials, a.bar, gen, a.status, t2, s_gat)) return;
  for (int j = threadIdx.x; j < P; j += blockDim.x) s_c[j] = s_gat[j];
  double dp = sqrt(t2[0]);
  const double sn = sqrt(t2[1]);
  const double rnorm0 = a.guess_zero ? dp : (sn == 0.0 ? dp : sn);
  const double ttol = fmax(fmax(a.rtol * rnorm0, a.atol), a.inner_rel > 0.0 ? a.inner_rel * dp : 0.0);
  int reason = classify(dp, ttol, a.atol, rnorm0);
  int its = 0;
  double pq_old = 1.0;
  double dp_mark = dp;
  const float th = a.theta, de = a.delta;
  const float sig = th / de;
  const bool timed = a.phase != nullptr && blockIdx.x == 0 && threadIdx.x == 0;
  unsigned long long tph = 0;
#define FCG_PHASE(k)                                    \
  if (timed) {                                          \
    const unsigned long long t_ = fcg_clock();          \
    a.phase[k] += (double)(t_ - tph);                   \
    tph = t_;                                           \
  }
  while (!reason) {
    if (its >= a.maxit) { reason = -3; break; }
    if (timed) {
      tph = fcg_clock();
      a.phase[7] += 1.0;
    }
    __syncthreads();  // s_c complete
    // ---- coarse values y = E^-1 c of this part and its neighbour parts (warp w: slot w)
    {
      const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
      if (w < a.NB) {
        double s = 0.0;
        for (int j = lane; j < P; j += 32) s += (double)s_er[(size_t)w * P + j] * s_c[j];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) s_yn[w] = s;
      }
    }
    __syncthreads();
    FCG_PHASE(0)
    const double yb = s_yn[0];
    // ---- part-local Chebyshev on D^-1 A_bb z = D^-1 r (FP32, shared memory).  With the
    // scaled residual s = D^-1 (r - A_bb z):  z += d;  s -= D^-1 A_bb d = d + sum a~_ij d_j;
    // d = c1 d + c2 s  (Saad, Iterative Methods, alg. 12.1, on the Jacobi-scaled operator).
    float zc[CPT], sc[CPT], dc[CPT];
    const bool rec_now = a.rec_stride > 0 && its % a.rec_stride == 0 && a.rec_base + its / a.rec_stride < a.rec_max;
    const size_t rec_off = rec_now ? (size_t)(a.rec_base + its / a.rec_stride) * n : 0;
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
      double rk = rr[k];
      if (a.deflate && OWN(k)) {  // r - (A Z y)_i
        const int i = base + threadIdx.x + k * FCG_TPB;
        double azy = yb * (double)__ldg(&a.srow[i]);
        const int e1 = __ldg(&a.xoff[i + 1]);
        for (int e = __ldg(&a.xoff[i]); e < e1; ++e) azy += (double)__ldg(&a.xval[e]) * s_yn[__ldg(&a.xslot[e])];
        rk -= azy;
      }
      sc[k] = OWN(k) ? s_dinv[threadIdx.x + k * FCG_TPB] * (float)rk : 0.0f;
      dc[k] = sc[k] / th;
      zc[k] = 0.0f;
      if (OWN(k)) {
        const int i = base + threadIdx.x + k * FCG_TPB;
        if (a.gamma != 0.0f) zc[k] = a.gamma * __ldg(&a.omega[i]) * sc[k];
        if (rec_now) {
          a.rec_r[rec_off + i] = rr[k];
          a.rec_u[rec_off + i] = (double)sc[k];
          a.rec_x[rec_off + i] = s_x[threadIdx.x + k * FCG_TPB];
        }
      }
    }
    float rho = 1.0f / sig;
    float* dcur = s_d0;
    float* dnext = s_d1;
    for (int j = 0; j < a.degree; ++j) {
#pragma unroll
      for (int k = 0; k < CPT; ++k) {
        zc[k] += dc[k];
        if (OWN(k)) dcur[threadIdx.x + k * FCG_TPB] = dc[k];
      }
      if (j == a.degree - 1) break;
      __syncthreads();
      const float rhon = 1.0f / (2.0f * sig - rho);
      const float c1 = rhon * rho, c2 = 2.0f * rhon / de;
#pragma unroll
      for (int k = 0; k < CPT; ++k)
        if (OWN(k)) {
          const int l = threadIdx.x + k * FCG_TPB;
          float ad = dc[k];
#pragma unroll
          for (int s = 0; s < LW; ++s)
            if (s < WL) {
              const unsigned e = s_lpk[s * C + l];
              ad = fmaf(__uint_as_float(e & 0xFFFF0000u), dcur[e & 0xFFFFu], ad);
            }
          sc[k] -= ad;
          dc[k] = c1 * dc[k] + c2 * sc[k];
        }
      rho = rhon;
      float* t = dcur; dcur = dnext; dnext = t;
    }
    __syncthreads();
    FCG_PHASE(1)
    // ---- z to global, barrier, w = A z and the sums
    double rz[CPT];
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
      rz[k] = (double)zc[k] + yb;
      if (OWN(k)) {
        if (MIXED) {
          const float zf = (float)rz[k];
          a.zs32[base + threadIdx.x + k * FCG_TPB] = zf;
          rz[k] = (double)zf;  // the z that A z is taken of
        } else {
          a.zs[base + threadIdx.x + k * FCG_TPB] = rz[k];
        }
        if (rec_now) a.rec_z[rec_off + base + threadIdx.x + k * FCG_TPB] = rz[k];
      }
    }
    if (!grid_barrier(a.bar, gen, a.status)) return;
    FCG_PHASE(2)
    double v[FCG_NV + FCG_NG], t[FCG_NV];
#pragma unroll
    for (int k = 0; k < FCG_NV + FCG_NG; ++k) v[k] = 0.0;
    double rw[CPT];
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
      rw[k] = 0.0;
      if (OWN(k)) {
        const int i = base + threadIdx.x + k * FCG_TPB;
        rw[k] = MIXED ? fcg_row<WT>(a, a.val32, WA, i, (const float*)a.zs32) : fcg_row<WT>(a, a.val, WA, i, a.zs);
        const double qk = s_q[threadIdx.x + k * FCG_TPB];
        v[0] += rz[k] * rr[k];
        v[1] += rz[k] * qk;
        v[2] += rz[k] * rw[k];
        v[3] += rz[k];
        v[4] += rr[k] * rr[k];
        v[5] += rr[k];
        v[6] += qk;
        v[7] += rw[k];
        v[8] += rr[k];   // gathered: part sums of r, w, q
        v[9] += rw[k];
        v[10] += qk;
      }
    }
    FCG_PHASE(3)
    if (!grid_reduce_gather<FCG_NV, FCG_NG>(v, a.partials, a.bar, gen, a.status, t, s_gat)) return;
    FCG_PHASE(4)
    dp = sqrt(t[4]);
    reason = classify(dp, ttol, a.atol, rnorm0);
    if (reason) break;
    if (a.stall_window > 0 && its > 0 && its % a.stall_window == 0) {  // automatic fallback trigger
      if (dp > a.stall_ratio * dp_mark) { reason = -20; break; }
      dp_mark = dp;
    }
    const double m = a.nullsp ? t[3] / (double)n : 0.0;
    const double zr = t[0] - m * t[5], zq = t[1] - m * t[6], zw = t[2] - m * t[7];
    const double beta = its == 0 ? 0.0 : -zq / pq_old;
    const double pq = zw + 2.0 * beta * zq + beta * beta * pq_old;
    if (!(pq > 0.0)) { reason = pq == 0.0 ? 3 : -10; break; }
    const double al = zr / pq;
#pragma unroll
    for (int k = 0; k < CPT; ++k)
      if (OWN(k)) {
        const int l = threadIdx.x + k * FCG_TPB;
        const double pk = (rz[k] - m) + beta * s_p[l];
        const double qk = rw[k] + beta * s_q[l];
        s_p[l] = pk;
        s_q[l] = qk;
        s_x[l] += al * pk;
        rr[k] -= al * qk;
      }
    for (int j = threadIdx.x; j < P; j += blockDim.x)
      s_c[j] = s_gat[j] - al * (s_gat[P + j] + beta * s_gat[2 * P + j]);
    pq_old = pq;
    FCG_PHASE(5)
    ++its;
  }
#undef FCG_PHASE
  // ---- write back x (original numbering) and the true residual ||b - A x||
  double v1[1] = {0.0}, t1[1];
#pragma unroll
  for (int k = 0; k < CPT; ++k)
    if (OWN(k)) {
      const int i = base + threadIdx.x + k * FCG_TPB;
      const double xi = s_x[threadIdx.x + k * FCG_TPB];
      a.xs[i] = xi;
      a.x[__ldg(&a.perm[i])] = xi;
    }
  if (!grid_barrier(a.bar, gen, a.status)) return;
#pragma unroll
  for (int k = 0; k < CPT; ++k)
    if (OWN(k)) {
      const int i = base + threadIdx.x + k * FCG_TPB;
      const double d = a.b[__ldg(&a.perm[i])] - fcg_row<WT>(a, a.val, WA, i, a.xs);
      v1[0] += d * d;
    }
  if (!grid_reduce_gather<1, 0>(v1, a.partials, a.bar, gen, a.status, t1, s_gat)) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.dout[0] = sqrt(t1[0]);
    a.dout[1] = dp;
    a.dout[2] = sn;
    a.status[0] = reason;
    a.status[1] = its;
  }
#undef OWN
}

template <bool MIXED>
inline void* fcg_kernel_sel(int cpt, int width) {
  if (width == 7) {
    switch (cpt) {
      case 1: return (void*)k_fcg<1, 7, MIXED>;
      case 2: return (void*)k_fcg<2, 7, MIXED>;
      case 3: return (void*)k_fcg<3, 7, MIXED>;
      case 4: return (void*)k_fcg<4, 7, MIXED>;
      default: return nullptr;
    }
  }
  switch (cpt) {
    case 1: return (void*)k_fcg<1, 0, MIXED>;
    case 2: return (void*)k_fcg<2, 0, MIXED>;
    case 3: return (void*)k_fcg<3, 0, MIXED>;
    case 4: return (void*)k_fcg<4, 0, MIXED>;
    default: return nullptr;
  }
}
inline void* fcg_kernel_for(int C, int width, bool mixed, int* cpt_out) {
  const int cpt = (C + FCG_TPB - 1) / FCG_TPB;
  *cpt_out = cpt;
  return mixed ? fcg_kernel_sel<true>(cpt, width) : fcg_kernel_sel<false>(cpt, width);
}

}  // namespace gpu
}  // namespace dpm
