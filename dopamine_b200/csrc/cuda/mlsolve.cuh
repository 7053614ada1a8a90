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
#include "mlkern.cuh"

namespace dpm {
namespace gpu {

struct MlSolver {
  MlArgs base{};
  int grid = 0;
  std::vector<int> sizes;      // rows per level, coarsest last
  std::vector<void*> owned;    // device allocations of this object
  int spin_limit_override = 0;  // > 0: poll limit of the kernel's grid-wide waits (status[3])
  // Multi-kernel form (mlkern.cuh) for fine levels of at least kernels_min_rows rows: the levels
  // on the host for by-value launches, the Krylov state, partial sums, a residual scratch vector,
  // and a pinned stop flag per batch of iterations with its event.
  static constexpr int kernels_min_rows = 1 << 20;
  static constexpr int iters_per_batch = 2;
  bool multi = false;
  double bytes_per_iteration = 0.0;  // algorithmic bytes of one Krylov iteration (roofline numerator)
  std::vector<MlDevLevel> hlv;
  MlkState* dS = nullptr;
  double* kpart = nullptr;
  double* kpart2 = nullptr;  // per-block partials of w = A z (one block per 256 rows)
  float* kres = nullptr;
  int* h_flag = nullptr;  // pinned, 2 entries
  cudaEvent_t kev[2] = {nullptr, nullptr};
  bool half_values = false;     // smoother off-diagonals in binary16 (else FP32)
  void* kernel() const { return half_values ? (void*)k_mlcg<unsigned short> : (void*)k_mlcg<float>; }

  MlSolver() = default;
  MlSolver(const MlSolver&) = delete;
  MlSolver& operator=(const MlSolver&) = delete;
  ~MlSolver() { release(); }

  void release() {
    for (void* p : owned) cudaFree(p);
    owned.clear();
    if (h_flag) cudaFreeHost(h_flag);
    h_flag = nullptr;
    for (auto& e : kev)
      if (e) { cudaEventDestroy(e); e = nullptr; }
    multi = false;
    hlv.clear();
    dS = nullptr; kpart = nullptr; kpart2 = nullptr; kres = nullptr;
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
    // Chebyshev steps per smoothing: 3 for the persistent kernel (each step costs a grid-wide
    // barrier there), 2 for the multi-kernel form of large meshes, where the sweeps are bandwidth-
    // bound (measured on the 19.3M-cell urban mesh: 294 vs 322 ms of Poisson solve per step,
    // 113 vs 96 iterations)
    const bool multi_form = n >= kernels_min_rows;
    const int deg = degree > 0 ? degree : (multi_form ? 2 : 3);
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
    multi = multi_form && nlev > 0;
    // algorithmic bytes of one iteration (each array touched once per pass): per level and V-cycle
    // deg - 1 down sweeps, the residual, the restriction, the prolongation and deg up sweeps (the
    // first without the old direction); the coarse solve; the FP64 w = A z pass with the sums;
    // the vector update with level 0's first step
    {
      const double svb = half_values ? 2.0 : 4.0;
      double bytes = 0.0;
      for (int l = 0; l < nlev; ++l) {
        const MlLevel& L = M.lv[l];
        const double nl = L.n, row = L.Wo * (4.0 + svb);
        const double nn = l + 1 < nlev ? M.lv[l + 1].n : M.nC;
        const double sweep = nl * (row + 24.0), first = nl * (row + 20.0), resid = nl * (row + 20.0);
        const double restrict_ = nn * (L.M * 4.0 + 16.0) + nl * 4.0, prolong = nl * 12.0;
        bytes += (2.0 * deg - 2.0) * sweep + first + resid + restrict_ + prolong;
      }
      bytes += (double)M.nC * M.nC * 4.0 + 8.0 * M.nC;
      bytes += (double)n * (WA * 12.0 + 28.0) + (double)n * 92.0;
      bytes_per_iteration = bytes;
    }
    if (multi) {
      hlv = hl;
      dS = alloc<MlkState>(1);
      const int64_t nfold = (((int64_t)n + MLK_TPB - 1) / MLK_TPB + MLK_TPB - 1) / MLK_TPB;  // fold blocks of w = A z
      kpart = alloc<double>((size_t)std::max<int64_t>(MLK_RED_BLOCKS, nfold) * MLK_NV);
      kres = alloc<float>(hl[0].n);
      kpart2 = alloc<double>((size_t)((n + MLK_TPB - 1) / MLK_TPB) * MLK_NV);
      if (!dS || !kpart || !kres || !kpart2) return DPM_ERR_CUDA;
      if (cudaHostAlloc(&h_flag, 2 * sizeof(int), cudaHostAllocDefault) != cudaSuccess) return DPM_ERR_CUDA;
      for (auto& e : kev)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return DPM_ERR_CUDA;
    }
    return 0;
  }

  template <class SV>
  void enqueue_iteration(const MlArgs& a, int G, cudaStream_t st) {
    const int nlev = a.nlev, deg = a.degree;
    auto nb = [](int64_t m) { return (int)((m + MLK_TPB - 1) / MLK_TPB); };
    unsigned curmask = 0;
    for (int l = 0; l < nlev; ++l) {
      const MlDevLevel& L = hlv[l];
      int cur = 0;
      for (int j = 1; j < deg; ++j) {
        k_mlk_sweep<SV><<<nb(L.n), MLK_TPB, 0, st>>>(L, L.c1[j], L.c2[j], 0, cur ? L.x1 : L.x0, cur ? L.x0 : L.x1,
                                                     nullptr, 0.0f, dS);
        cur ^= 1;
      }
      curmask |= (unsigned)cur << l;
      const bool last = l + 1 == nlev;
      k_mlk_resid<SV><<<nb(L.n), MLK_TPB, 0, st>>>(L, cur ? L.x1 : L.x0, kres, dS);
      k_mlk_restrict<<<nb(L.n_next), MLK_TPB, 0, st>>>(L, kres, last ? L : hlv[l + 1], last ? 1 : 0, a.bC, dS);
    }
    k_mlk_coarse<<<nb((int64_t)a.nC * 32), MLK_TPB, 0, st>>>(a.nC, a.cinv, a.bC, a.xC, dS);
    const float* xcoarse = a.xC;
    for (int l = nlev - 1; l >= 0; --l) {
      const MlDevLevel& L = hlv[l];
      int cur = (curmask >> l) & 1u;
      k_mlk_prolong<<<nb(L.n), MLK_TPB, 0, st>>>(L, cur ? L.x1 : L.x0, xcoarse, a.oc, dS);
      for (int j = 0; j < deg; ++j) {
        const float* om = (l == 0 && j == deg - 1 && a.gamma != 0.0f) ? a.omega : nullptr;
        k_mlk_sweep<SV><<<nb(L.n), MLK_TPB, 0, st>>>(L, L.c1[j], L.c2[j], j == 0 ? 1 : 0, cur ? L.x1 : L.x0,
                                                     cur ? L.x0 : L.x1, om, a.gamma, dS);
        cur ^= 1;
      }
      xcoarse = cur ? L.x1 : L.x0;
    }
    const float* z = xcoarse;
    if (a.rec_stride > 0) k_mlk_record<<<G, MLK_TPB, 0, st>>>(a, z, hlv[0].b, dS);
    const int nw = nb(a.n), nf = (nw + MLK_TPB - 1) / MLK_TPB;
    k_mlk_wz<float><<<nw, MLK_TPB, 0, st>>>(a, z, kpart2, dS);
    k_mlk_fold<MLK_NV><<<nf, MLK_TPB, 0, st>>>(nw, kpart2, kpart, dS);
    k_mlk_rule<<<1, 32 * MLK_NV, 0, st>>>(a.n, nf, kpart, dS);
    k_mlk_update<float><<<nb(a.n), MLK_TPB, 0, st>>>(a, z, a.lv, dS);
    k_mlk_next<<<1, 1, 0, st>>>(dS);
  }

  // The solve as standalone kernels: start, then batches of iters_per_batch iterations with the
  // stop flag of each batch read back while the next batch runs, then the true residual.
  int launch_multi(MlArgs& a, cudaStream_t st, int* reason, int* its, double* resid) {
    MlkState h{};
    h.rtol = a.rtol; h.atol = a.atol; h.maxit = a.maxit; h.nullsp = a.nullsp; h.guess_zero = a.guess_zero;
    h.stall_window = a.stall_window; h.stall_ratio = a.stall_ratio;
    if (cudaMemcpyAsync(dS, &h, sizeof(h), cudaMemcpyHostToDevice, st) != cudaSuccess) return DPM_ERR_CUDA;
    const int G = std::min((a.n + MLK_TPB - 1) / MLK_TPB, MLK_RED_BLOCKS);
    k_mlk_init_sum<<<G, MLK_TPB, 0, st>>>(a.n, a.b, a.x, a.guess_zero, kpart);
    k_mlk_init_mean<<<1, 32, 0, st>>>(a.n, G, kpart, dS);
    k_mlk_init_resid<<<G, MLK_TPB, 0, st>>>(a, a.lv, dS, kpart);
    k_mlk_init_rule<<<1, 64, 0, st>>>(G, kpart, dS);
    const int max_batches = (std::max(a.maxit, 0) + iters_per_batch - 1) / iters_per_batch + 1;
    for (int bt = 0; bt < max_batches; ++bt) {
      for (int k = 0; k < iters_per_batch; ++k) {
        if (half_values) enqueue_iteration<unsigned short>(a, G, st);
        else enqueue_iteration<float>(a, G, st);
      }
      if (cudaMemcpyAsync(&h_flag[bt & 1], &dS->done, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          cudaEventRecord(kev[bt & 1], st) != cudaSuccess)
        return DPM_ERR_CUDA;
      if (bt > 0) {  // the previous batch's flag, read while this batch runs
        if (cudaEventSynchronize(kev[(bt - 1) & 1]) != cudaSuccess) return DPM_ERR_CUDA;
        if (h_flag[(bt - 1) & 1]) break;
      }
    }
    if (cudaGetLastError() != cudaSuccess) return DPM_ERR_CUDA;
    k_mlk_true_resid<<<G, MLK_TPB, 0, st>>>(a, kpart);
    k_mlk_finish<<<1, 32, 0, st>>>(G, kpart, dS, a.status, a.dout);
    int h_st[4];
    double h_d[4];
    if (cudaMemcpyAsync(h_st, a.status, 4 * sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return DPM_ERR_CUDA;
    if (cudaMemcpyAsync(h_d, a.dout, 4 * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess) return DPM_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return DPM_ERR_CUDA;
    *reason = h_st[0];
    *its = h_st[1];
    *resid = h_d[0];
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
    if (multi) return launch_multi(a, st, reason, its, resid);
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
