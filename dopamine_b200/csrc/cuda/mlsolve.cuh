// Host side of the multilevel flexible-CG solve (k_mlcg), shared by the solver object and the
// drop-in pressure ABI: builds the aggregation hierarchy (csrc/host/multilevel.cpp), uploads the
// FP32 levels, sets the Chebyshev coefficients, sizes the cooperative grid and launches.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <vector>

#include "../../../include/dopamine_b200.h"
#include "../host/multilevel.hpp"
#include "mlcg.cuh"

namespace dpm {
namespace gpu {

struct MlSolver {
  MlArgs base{};
  int grid = 0;
  std::vector<int> sizes;      // rows per level, coarsest last
  std::vector<void*> owned;    // device allocations of this object
  int spin_limit_override = 0;  // > 0: poll limit of the kernel's grid-wide waits (status[3])
  bool half_values = false;     // smoother off-diagonals in binary16 (else FP32)
  void* kernel() const { return half_values ? (void*)k_mlcg<unsigned short> : (void*)k_mlcg<float>; }

  MlSolver() = default;
  MlSolver(const MlSolver&) = delete;
  MlSolver& operator=(const MlSolver&) = delete;
  ~MlSolver() { release(); }

  void release() {
    for (void* p : owned) cudaFree(p);
    owned.clear();
    base = MlArgs{};
    grid = 0;
    sizes.clear();
  }
  bool ready() const { return grid > 0; }

  template <class T>
  T* alloc(size_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return nullptr;
    owned.push_back(p);
    return static_cast<T*>(p);
  }
  template <class T>
  T* upload(const std::vector<T>& v) {
    T* p = alloc<T>(v.size());
    if (p && !v.empty() && cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
      return nullptr;
    return p;
  }

  // h_col / h_val: the FP64 operator in padded ELL [WA][n] on the host; d_col / d_val: the same
  // on the device (used for w = A z and the residuals).  bar / status / dout: the caller's
  // barrier counter [2], status [4] and result [4] buffers.  Returns 0 or a DPM_ERR_* code.
  int setup(int n, int WA, const int* h_col, const double* h_val, const int* d_col, const double* d_val, bool nullsp,
            int passes, int degree, double oc, int dev_sms, unsigned* bar, int* status, double* dout,
            int value_bits = 0) {
    release();
    if (value_bits != 0 && value_bits != 16 && value_bits != 32) return DPM_ERR_ARG;
    half_values = value_bits == 16;
    Multilevel M;
    if (build_multilevel(n, WA, h_col, h_val, nullsp, passes > 0 ? passes : 3, 0.25, 300, 1024, M))
      return DPM_ERR_UNSUPPORTED;
    const int nlev = (int)M.lv.size();
    const int deg = degree > 0 ? degree : 3;
    if (nlev > ML_LEVELS || deg > ML_DEG) return DPM_ERR_ARG;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel(), ML_TPB, 0) != cudaSuccess || per_sm < 1)
      return DPM_ERR_UNSUPPORTED;
    const int g = std::min(dev_sms * std::min(per_sm, 2), ML_MAX_GRID);
    const int64_t threads = (int64_t)g * ML_TPB;
    std::vector<MlDevLevel> hl(nlev);
    for (int l = 0; l < nlev; ++l) {
      const MlLevel& L = M.lv[l];
      MlDevLevel& D = hl[l];
      D = MlDevLevel{};
      D.n = L.n; D.W = L.Wo; D.M = L.M;
      D.n_next = l + 1 < nlev ? M.lv[l + 1].n : M.nC;
      D.MP = 1;
      D.lgMP = 0;
      while (D.MP < L.M) { D.MP *= 2; D.lgMP++; }
      if (D.MP > 32) return DPM_ERR_UNSUPPORTED;
      // lanes per row: spread small levels over up to 32 lanes (no more lanes than entries)
      int gl = 1;
      D.lgG = 0;
      while (gl < 32 && (int64_t)L.n * gl * 2 <= threads && 2 * gl <= L.Wo) { gl *= 2; D.lgG++; }
      // up to 2 rows per lane and pass: more rows do not keep more loads in flight within the
      // kernel's 64 registers (measured: 2 rows 4.5 % faster than 4 on a 2.4M-row fine level)
      D.rows_per_pass = (int)std::min<int64_t>(2, std::max<int64_t>(1, (L.n + threads - 1) / threads));
      gl = 1;
      D.lgGR = 0;
      while (D.MP * gl * 2 <= 32 && (int64_t)D.n_next * D.MP * gl * 2 <= threads && 2 * gl <= L.Wo) { gl *= 2; D.lgGR++; }
      D.col = upload(L.ocol);
      D.sv = half_values ? (const void*)upload(L.sv16) : (const void*)upload(L.sv32);
      D.g = upload(half_values ? L.g16 : L.g32);
      D.diag = upload(L.diag);
      D.dinv = upload(L.dinv);
      D.agg = upload(L.agg); D.mem = upload(L.mem);
      D.b = alloc<float>(L.n); D.x0 = alloc<float>(L.n); D.x1 = alloc<float>(L.n);
      D.d = alloc<float>(L.n);
      if (!D.col || !D.sv || !D.g || !D.diag || !D.dinv || !D.agg || !D.mem || !D.b || !D.x0 || !D.x1 || !D.d)
        return DPM_ERR_CUDA;
      // Chebyshev on [lmax/10, lmax], lmax = 1.1 x the power-iteration estimate
      const double lmax = 1.1 * L.lmax, lmin = 0.1 * lmax;
      const double th = 0.5 * (lmax + lmin), de = 0.5 * (lmax - lmin), sig = th / de;
      D.inv_theta = (float)(1.0 / th);
      double rho = 1.0 / sig;
      for (int j = 1; j < ML_DEG; ++j) {
        const double rhon = 1.0 / (2.0 * sig - rho);
        D.c1[j] = (float)(rhon * rho);
        D.c2[j] = (float)(2.0 * rhon / de);
        rho = rhon;
      }
    }
    MlArgs a{};
    a.n = n; a.WA = WA; a.nlev = nlev; a.degree = deg; a.nC = M.nC;
    a.col = d_col; a.val = d_val;
    if (nlev > 0) {
      a.lv = upload(hl);
      if (!a.lv) return DPM_ERR_CUDA;
    }
    a.cinv = upload(M.cinv);
    a.bC = alloc<float>(M.nC); a.xC = alloc<float>(M.nC);
    a.oc = (float)(oc > 0.0 ? oc : 1.6);
    a.r = alloc<double>(n); a.p = alloc<double>(n); a.q = alloc<double>(n); a.w = alloc<double>(n);
    a.partials = alloc<double>((size_t)2 * FCG_SLOT * g);
    a.bar = bar; a.status = status; a.dout = dout;
    a.nullsp = nullsp ? 1 : 0;
    a.stall_window = 50;
    a.stall_ratio = 0.9;
    if (!a.cinv || !a.bC || !a.xC || !a.r || !a.p || !a.q || !a.w || !a.partials) return DPM_ERR_CUDA;
    base = a;
    sizes = M.sizes;
    grid = g;
    return 0;
  }

  // One solve on stream st; reason / its / resid as the Krylov kernels report them.  extra: the
  // learned-term and recording fields (omega, gamma, rec_*, pinv), or null.
  int launch(const double* b, double* x, double rtol, double atol, int maxit, int guess_zero, cudaStream_t st,
             int* reason, int* its, double* resid, const MlArgs* extra = nullptr) {
    if (!ready()) return DPM_ERR_ARG;
    MlArgs a = base;
    if (extra) {
      a.omega = extra->omega; a.gamma = extra->gamma;
      a.rec_stride = extra->rec_stride; a.rec_base = extra->rec_base; a.rec_max = extra->rec_max;
      a.pinv = extra->pinv;
      a.rec_r = extra->rec_r; a.rec_z = extra->rec_z; a.rec_u = extra->rec_u; a.rec_x = extra->rec_x;
    }
    a.b = b; a.x = x; a.rtol = rtol; a.atol = atol; a.maxit = maxit; a.guess_zero = guess_zero;
    if (cudaMemsetAsync(a.bar, 0, 2 * sizeof(unsigned), st) != cudaSuccess) return DPM_ERR_CUDA;
    if (cudaMemsetAsync(a.status, 0, 4 * sizeof(int), st) != cudaSuccess) return DPM_ERR_CUDA;
    if (spin_limit_override &&
        cudaMemcpyAsync(a.status + 3, &spin_limit_override, sizeof(int), cudaMemcpyHostToDevice, st) != cudaSuccess)
      return DPM_ERR_CUDA;
    void* args[] = {&a};
    if (cudaLaunchCooperativeKernel(kernel(), dim3(grid), dim3(ML_TPB), args, 0, st) != cudaSuccess)
      return DPM_ERR_CUDA;
    int h_st[4];
    double h_d[4];
    if (cudaMemcpyAsync(h_st, a.status, 4 * sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return DPM_ERR_CUDA;
    if (cudaMemcpyAsync(h_d, a.dout, 4 * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess) return DPM_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return DPM_ERR_CUDA;
    if (h_st[2]) {
      std::fprintf(stderr, "dopamine_b200: multilevel FCG grid barrier timed out\n");
      return DPM_ERR_BARRIER_TIMEOUT;
    }
    *reason = h_st[0];
    *its = h_st[1];
    *resid = h_d[0];
    return 0;
  }
};

}  // namespace gpu
}  // namespace dpm
