// Learned term of the two-level preconditioner: a one-ring message-passing network that maps
// static per-cell features of the pressure operator to a non-negative weight omega_i; inside the
// flexible CG the preconditioned residual becomes
//
//     z = y_b + S_b(rho0) + gamma * omega .* D^-1 rho0,      rho0 = r - A Z y   (deflated residual)
//
// (gamma: a global scale chosen on held-out solves, 0 disables the term).  No counterpart in the
// reference.  Network (per cell, BF16 weights, FP32 accumulate):
//
//     a_i  = sum_j a~_ij f_j                 one-ring aggregation over the part-local couplings
//     h1_i = relu(W1 [f_i ; a_i] + b1)       16 -> 16, tensor cores (mma.sync m16n8k16 bf16)
//     h2_i = relu(W2 h1_i + b2)              16 -> 16, tensor cores
//     omega_i = OMEGA_SCALE * softplus(w3 . h2_i + b3)
//
// Training minimises, over solver-recorded samples k (r_k, its error e_k = x* - x_k, the base
// preconditioned residual zb_k and u_k = D^-1 rho0_k), the A-angle loss
//     L = mean_k (1 - (z_k.r_k)^2 / ((z_k.A z_k)(e_k.r_k))),   z_k = zb_k + omega .* u_k,
// with forward, loss, backward and Adam steps all in the kernels below.
#pragma once
#include "common.cuh"

namespace dpm {
namespace gpu {

constexpr int LP_F = 8;     // static features per cell
constexpr int LP_H = 16;    // hidden width
constexpr float LP_OMEGA_SCALE = 0.25f;
// parameter vector layout (FP32 masters): W1 [16 out][16 in], b1 [16], W2 [16][16], b2 [16], w3 [16], b3
constexpr int LP_W1 = 0, LP_B1 = 256, LP_W2 = 272, LP_B2 = 528, LP_W3 = 544, LP_B3 = 560, LP_NP = 561;

__device__ __forceinline__ unsigned short f2bf(float x) {  // round to nearest even (finite x)
  unsigned u = __float_as_uint(x);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return (unsigned short)(u >> 16);
}
__device__ __forceinline__ float bf2f(unsigned short h) { return __uint_as_float((unsigned)h << 16); }
__device__ __forceinline__ unsigned pack2(float lo, float hi) {
  return (unsigned)f2bf(lo) | ((unsigned)f2bf(hi) << 16);
}

// D[16x8] += A[16x16] * B[16x8], bf16 inputs, fp32 accumulate (PTX mma.sync.m16n8k16).
// Fragments (g = lane/4, t = lane%4): a0 = A[g][2t..2t+1], a1 = A[g+8][2t..], a2 = A[g][2t+8..],
// a3 = A[g+8][2t+8..]; b0 = B[2t..2t+1][g], b1 = B[2t+8..2t+9][g]; d0,d1 = D[g][2t..2t+1],
// d2,d3 = D[g+8][2t..2t+1].
__device__ __forceinline__ void mma16816(float (&d)[4], const unsigned (&a)[4], const unsigned (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// One-ring aggregation of the features over the part-local couplings (packed rows:
// local column | bf16 a_ij / a_ii), in the renumbered (part-contiguous) order.
__device__ __forceinline__ void lp_aggregate(int i, int n, int C, int WL, const unsigned* __restrict__ lpk,
                                             const float* __restrict__ feat, float (&agg)[LP_F]) {
  const int base = (i / C) * C;
#pragma unroll
  for (int k = 0; k < LP_F; ++k) agg[k] = 0.0f;
  for (int s = 0; s < WL; ++s) {
    const unsigned e = __ldg(&lpk[(size_t)s * n + i]);
    const float w = __uint_as_float(e & 0xFFFF0000u);
    if (w == 0.0f) continue;
    const int j = base + (int)(e & 0xFFFFu);
#pragma unroll
    for (int k = 0; k < LP_F; ++k) agg[k] = fmaf(w, __ldg(&feat[(size_t)k * n + j]), agg[k]);
  }
}

// Forward: one warp per 16 cells.  Writes omega [n] and, for the backward pass, the layer inputs
// h1, h2 [16][n] (after relu) and the output pre-activation.  Weights: bf16 copies wb [LP_NP].
__global__ void __launch_bounds__(256) k_lp_forward(int n, int C, int WL, const unsigned* __restrict__ lpk,
                                                    const float* __restrict__ feat,
                                                    const unsigned short* __restrict__ wb,
                                                    const float* __restrict__ prm, float* __restrict__ omega,
                                                    float* __restrict__ h1o, float* __restrict__ h2o,
                                                    float* __restrict__ preo) {
  __shared__ float s_in[8][16][17];  // per warp: 16 cells x 16 inputs (padded)
  __shared__ float s_h[8][16][17];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const int c0 = (blockIdx.x * 8 + warp) * 16;
  if (c0 >= n) return;
  // inputs [f ; agg] for the warp's 16 cells: lanes 0..15 one cell each
  if (lane < 16) {
    const int i = c0 + lane;
    float agg[LP_F];
    if (i < n) {
      lp_aggregate(i, n, C, WL, lpk, feat, agg);
#pragma unroll
      for (int k = 0; k < LP_F; ++k) {
        s_in[warp][lane][k] = __ldg(&feat[(size_t)k * n + i]);
        s_in[warp][lane][LP_F + k] = agg[k];
      }
    } else {
#pragma unroll
      for (int k = 0; k < 16; ++k) s_in[warp][lane][k] = 0.0f;
    }
  }
  __syncwarp();
  // layer 1: A = inputs [16 cells x 16], B = W1^T [16 in x 16 out] as two n8 tiles
  unsigned a[4];
  a[0] = pack2(s_in[warp][g][2 * t], s_in[warp][g][2 * t + 1]);
  a[1] = pack2(s_in[warp][g + 8][2 * t], s_in[warp][g + 8][2 * t + 1]);
  a[2] = pack2(s_in[warp][g][2 * t + 8], s_in[warp][g][2 * t + 9]);
  a[3] = pack2(s_in[warp][g + 8][2 * t + 8], s_in[warp][g + 8][2 * t + 9]);
  for (int nt = 0; nt < 2; ++nt) {
    const int o = nt * 8 + g;  // output column owned by this lane in the B fragment
    unsigned b[2];
    b[0] = (unsigned)wb[LP_W1 + o * 16 + 2 * t] | ((unsigned)wb[LP_W1 + o * 16 + 2 * t + 1] << 16);
    b[1] = (unsigned)wb[LP_W1 + o * 16 + 2 * t + 8] | ((unsigned)wb[LP_W1 + o * 16 + 2 * t + 9] << 16);
    float d[4] = {0.f, 0.f, 0.f, 0.f};
    mma16816(d, a, b);
    const int col = nt * 8 + 2 * t;
    s_h[warp][g][col] = fmaxf(d[0] + prm[LP_B1 + col], 0.0f);
    s_h[warp][g][col + 1] = fmaxf(d[1] + prm[LP_B1 + col + 1], 0.0f);
    s_h[warp][g + 8][col] = fmaxf(d[2] + prm[LP_B1 + col], 0.0f);
    s_h[warp][g + 8][col + 1] = fmaxf(d[3] + prm[LP_B1 + col + 1], 0.0f);
  }
  __syncwarp();
  // layer 2 (inputs h1 rounded to bf16 by the fragment packing)
  a[0] = pack2(s_h[warp][g][2 * t], s_h[warp][g][2 * t + 1]);
  a[1] = pack2(s_h[warp][g + 8][2 * t], s_h[warp][g + 8][2 * t + 1]);
  a[2] = pack2(s_h[warp][g][2 * t + 8], s_h[warp][g][2 * t + 9]);
  a[3] = pack2(s_h[warp][g + 8][2 * t + 8], s_h[warp][g + 8][2 * t + 9]);
  if (lane < 16 && c0 + lane < n)
    for (int k = 0; k < LP_H; ++k) h1o[(size_t)k * n + c0 + lane] = s_h[warp][lane][k];
  __syncwarp();
  for (int nt = 0; nt < 2; ++nt) {
    const int o = nt * 8 + g;
    unsigned b[2];
    b[0] = (unsigned)wb[LP_W2 + o * 16 + 2 * t] | ((unsigned)wb[LP_W2 + o * 16 + 2 * t + 1] << 16);
    b[1] = (unsigned)wb[LP_W2 + o * 16 + 2 * t + 8] | ((unsigned)wb[LP_W2 + o * 16 + 2 * t + 9] << 16);
    float d[4] = {0.f, 0.f, 0.f, 0.f};
    mma16816(d, a, b);
    const int col = nt * 8 + 2 * t;
    s_in[warp][g][col] = fmaxf(d[0] + prm[LP_B2 + col], 0.0f);
    s_in[warp][g][col + 1] = fmaxf(d[1] + prm[LP_B2 + col + 1], 0.0f);
    s_in[warp][g + 8][col] = fmaxf(d[2] + prm[LP_B2 + col], 0.0f);
    s_in[warp][g + 8][col + 1] = fmaxf(d[3] + prm[LP_B2 + col + 1], 0.0f);
  }
  __syncwarp();
  // output layer on CUDA cores (16 -> 1), FP32
  if (lane < 16 && c0 + lane < n) {
    const int i = c0 + lane;
    float pre = prm[LP_B3];
    for (int k = 0; k < LP_H; ++k) {
      const float h = s_in[warp][lane][k];
      h2o[(size_t)k * n + i] = h;
      pre = fmaf(prm[LP_W3 + k], h, pre);
    }
    preo[i] = pre;
    const float sp = pre > 20.0f ? pre : log1pf(expf(pre));
    omega[i] = LP_OMEGA_SCALE * sp;
  }
}

// Loss terms per sample k (deterministic block partials; final sums by k_lp_sum):
//   v = omega .* u_k:  q1 = v.r,  q2 = v.(A zb),  q3 = v.(A v)    (A v given as av_k)
__global__ void __launch_bounds__(256) k_lp_dots(int n, int S, const float* __restrict__ omega,
                                                 const double* __restrict__ U, const double* __restrict__ R,
                                                 const double* __restrict__ AZB, const double* __restrict__ AV,
                                                 double* __restrict__ part) {
  const int k = blockIdx.y;
  double q[3] = {0.0, 0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const size_t o = (size_t)k * n + i;
    const double v = (double)omega[i] * U[o];
    q[0] += v * R[o];
    q[1] += v * AZB[o];
    q[2] += v * AV[o];
  }
  __shared__ double sh[8][3];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    for (int o = 16; o > 0; o >>= 1) q[m] += __shfl_down_sync(0xffffffffu, q[m], o);
    if (lane == 0) sh[w][m] = q[m];
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double t = 0.0;
    for (int j = 0; j < (int)(blockDim.x >> 5); ++j) t += sh[j][threadIdx.x];
    part[((size_t)k * gridDim.x + blockIdx.x) * 3 + threadIdx.x] = t;
  }
}

// v_k = omega .* u_k, then A v_k with the renumbered ELL operator (one thread per row, per sample)
__global__ void __launch_bounds__(256) k_lp_av(int n, int WA, int S, const int* __restrict__ col,
                                               const double* __restrict__ val, const float* __restrict__ omega,
                                               const double* __restrict__ U, double* __restrict__ AV) {
  const int k = blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* u = U + (size_t)k * n;
  double s = 0.0;
  for (int w = 0; w < WA; ++w) {
    const int j = __ldg(&col[(size_t)w * n + i]);
    s += __ldg(&val[(size_t)w * n + i]) * ((double)omega[j] * u[j]);
  }
  AV[(size_t)k * n + i] = s;
}

// dL/domega_i = sum_k g_k,i u_k,i with g_k = dL/dz_k = -(1/S)[2a/(bc) r - 2a^2/(b^2 c) A z],
// a = z.r, b = z.A z, c = e.r, z = zb + v, A z = A zb + A v; coef[k] = {2a/(bc), 2a^2/(b^2 c)}.
__global__ void __launch_bounds__(256) k_lp_domega(int n, int S, const double* __restrict__ coef,
                                                   const double* __restrict__ U, const double* __restrict__ R,
                                                   const double* __restrict__ AZB, const double* __restrict__ AV,
                                                   float* __restrict__ domega) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double g = 0.0;
  for (int k = 0; k < S; ++k) {
    const size_t o = (size_t)k * n + i;
    const double gz = -(coef[2 * k] * R[o] - coef[2 * k + 1] * (AZB[o] + AV[o])) / (double)S;
    g += gz * U[o];
  }
  domega[i] = (float)g;
}

// Backward through the network, per cell; parameter gradients are reduced over each warp's 32
// cells by shuffles into that warp's own shared-memory row, then summed over the block's warps
// in a fixed order into part[block][LP_NP] (no atomics: deterministic).  The gradients are taken
// at the bf16-rounded weights and layer inputs that the forward pass used.
__device__ __forceinline__ float warp_sum_f(float v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__global__ void __launch_bounds__(128) k_lp_backward(int n, int C, int WL, const unsigned* __restrict__ lpk,
                                                     const float* __restrict__ feat,
                                                     const unsigned short* __restrict__ wb,
                                                     const float* __restrict__ prm, const float* __restrict__ h1,
                                                     const float* __restrict__ h2, const float* __restrict__ pre,
                                                     const float* __restrict__ domega, float* __restrict__ part) {
  __shared__ float s_g[4][LP_NP];
  __shared__ float s_w[LP_NP];  // bf16-rounded W1, W2 and FP32 w3 as used by the forward pass
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int j = threadIdx.x; j < LP_NP; j += blockDim.x) {
    s_w[j] = (j < LP_B1 || (j >= LP_W2 && j < LP_B2)) ? bf2f(wb[j]) : prm[j];
    for (int q = 0; q < 4; ++q) s_g[q][j] = 0.0f;
  }
  __syncthreads();
  for (int i0 = (blockIdx.x * 4 + w) * 32; i0 < n; i0 += gridDim.x * 4 * 32) {
    const int i = i0 + lane;
    const bool ok = i < n;
    float in[16], x1[16], d1[16], d2[16];
    float dpre = 0.0f;
    if (ok) {
      float agg[LP_F];
      lp_aggregate(i, n, C, WL, lpk, feat, agg);
#pragma unroll
      for (int k = 0; k < LP_F; ++k) {
        in[k] = bf2f(f2bf(__ldg(&feat[(size_t)k * n + i])));
        in[LP_F + k] = bf2f(f2bf(agg[k]));
      }
#pragma unroll
      for (int k = 0; k < 16; ++k) x1[k] = h1[(size_t)k * n + i];
      const float p = pre[i];
      dpre = domega[i] * LP_OMEGA_SCALE * (1.0f / (1.0f + expf(-p)));
    } else {
#pragma unroll
      for (int k = 0; k < 16; ++k) in[k] = x1[k] = 0.0f;
    }
    // output layer: pre = w3 . h2 + b3
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const float x2 = ok ? h2[(size_t)k * n + i] : 0.0f;
      const float gk = warp_sum_f(dpre * x2);
      if (lane == 0) s_g[w][LP_W3 + k] += gk;
      d2[k] = x2 > 0.0f ? dpre * s_w[LP_W3 + k] : 0.0f;  // d pre2
    }
    {
      const float gb = warp_sum_f(dpre);
      if (lane == 0) s_g[w][LP_B3] += gb;
    }
    // layer 2: pre2[o] = sum_k W2[o][k] bf16(h1[k]) + b2[o]
    float xb[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) xb[k] = bf2f(f2bf(x1[k]));
#pragma unroll
    for (int o = 0; o < 16; ++o) {
      const float gb = warp_sum_f(d2[o]);
      if (lane == 0) s_g[w][LP_B2 + o] += gb;
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const float g = warp_sum_f(d2[o] * xb[k]);
        if (lane == 0) s_g[w][LP_W2 + o * 16 + k] += g;
      }
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      float t = 0.0f;
#pragma unroll
      for (int o = 0; o < 16; ++o) t = fmaf(d2[o], s_w[LP_W2 + o * 16 + k], t);
      d1[k] = x1[k] > 0.0f ? t : 0.0f;  // d pre1
    }
    // layer 1: pre1[o] = sum_k W1[o][k] in[k] + b1[o]
#pragma unroll
    for (int o = 0; o < 16; ++o) {
      const float gb = warp_sum_f(d1[o]);
      if (lane == 0) s_g[w][LP_B1 + o] += gb;
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const float g = warp_sum_f(d1[o] * in[k]);
        if (lane == 0) s_g[w][LP_W1 + o * 16 + k] += g;
      }
    }
  }
  __syncthreads();
  for (int j = threadIdx.x; j < LP_NP; j += blockDim.x)
    part[(size_t)blockIdx.x * LP_NP + j] = ((s_g[0][j] + s_g[1][j]) + s_g[2][j]) + s_g[3][j];
}

// dst[perm[i]] = src[i]: renumbered (part-contiguous) order back to the mesh order
__global__ void k_perm_scatter(int n, const int* __restrict__ perm, const double* __restrict__ src,
                               double* __restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[perm[i]] = src[i];
}
__global__ void k_perm_gather(int n, const int* __restrict__ perm, const double* __restrict__ src,
                              double* __restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[perm[i]];
}
__global__ void k_perm_scatter_f(int n, const int* __restrict__ perm, const float* __restrict__ src,
                                 float* __restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[perm[i]] = src[i];
}
__global__ void k_fill_f(int n, float* p, float v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}
// e_k = x* - x_k for the recorded slots k = blockIdx.y (X holds x_k on entry, e_k on exit)
__global__ void k_lp_err(int n, const double* __restrict__ xs, double* __restrict__ X) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const size_t o = (size_t)blockIdx.y * n + i;
  X[o] = xs[i] - X[o];
}
// Y_k = A X_k (renumbered ELL), k = blockIdx.y
__global__ void __launch_bounds__(256) k_lp_spmv(int n, int WA, const int* __restrict__ col,
                                                 const double* __restrict__ val, const double* __restrict__ X,
                                                 double* __restrict__ Y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* x = X + (size_t)blockIdx.y * n;
  double s = 0.0;
  for (int w = 0; w < WA; ++w) s += __ldg(&val[(size_t)w * n + i]) * x[__ldg(&col[(size_t)w * n + i])];
  Y[(size_t)blockIdx.y * n + i] = s;
}
// per sample k: {a1.b1, a2.b2, a3.b3} as block partials part[(k * gridDim.x + block) * 3 + m]
__global__ void __launch_bounds__(256) k_lp_dots3(int n, const double* __restrict__ A1, const double* __restrict__ B1,
                                                  const double* __restrict__ A2, const double* __restrict__ B2,
                                                  const double* __restrict__ A3, const double* __restrict__ B3,
                                                  double* __restrict__ part) {
  const size_t off = (size_t)blockIdx.y * n;
  double q[3] = {0.0, 0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    q[0] += A1[off + i] * B1[off + i];
    q[1] += A2[off + i] * B2[off + i];
    q[2] += A3[off + i] * B3[off + i];
  }
  __shared__ double sh[8][3];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    for (int o = 16; o > 0; o >>= 1) q[m] += __shfl_down_sync(0xffffffffu, q[m], o);
    if (lane == 0) sh[w][m] = q[m];
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double t = 0.0;
    for (int j = 0; j < (int)(blockDim.x >> 5); ++j) t += sh[j][threadIdx.x];
    part[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * 3 + threadIdx.x] = t;
  }
}

// Fixed-order sums of per-block partials: out[j] = sum_b part[b][j] (one thread per j).
__global__ void k_lp_sum_f(int nb, int m, const float* __restrict__ part, float* __restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  float t = 0.0f;
  for (int b = 0; b < nb; ++b) t += part[(size_t)b * m + j];
  out[j] = t;
}
__global__ void k_lp_sum_d(int nb, int m, const double* __restrict__ part, double* __restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  double t = 0.0;
  for (int b = 0; b < nb; ++b) t += part[(size_t)b * m + j];
  out[j] = t;
}

// out[k*3 + m] = sum_b part[(k*nbk + b)*3 + m]  (fixed order)
__global__ void k_lp_sum_samples(int S, int nbk, const double* __restrict__ part, double* __restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= 3 * S) return;
  const int k = j / 3, m = j - 3 * k;
  double t = 0.0;
  for (int b = 0; b < nbk; ++b) t += part[((size_t)k * nbk + b) * 3 + m];
  out[j] = t;
}

// Adam on the FP32 master parameters, then the bf16 copies the forward pass reads.
__global__ void k_lp_adam(int np, float* __restrict__ prm, float* __restrict__ m1, float* __restrict__ m2,
                          const float* __restrict__ g, float lr, float b1, float b2, float eps, int step,
                          unsigned short* __restrict__ wb) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= np) return;
  const float gj = g[j];
  m1[j] = b1 * m1[j] + (1.0f - b1) * gj;
  m2[j] = b2 * m2[j] + (1.0f - b2) * gj * gj;
  const float mh = m1[j] / (1.0f - powf(b1, (float)step));
  const float vh = m2[j] / (1.0f - powf(b2, (float)step));
  prm[j] -= lr * mh / (sqrtf(vh) + eps);
  wb[j] = f2bf(prm[j]);
}
__global__ void k_lp_round(int np, const float* __restrict__ prm, unsigned short* __restrict__ wb) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < np) wb[j] = f2bf(prm[j]);
}

}  // namespace gpu
}  // namespace dpm
