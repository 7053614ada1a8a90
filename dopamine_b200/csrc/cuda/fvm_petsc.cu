// Drop-in replacement of the reference's pressure-solve C ABI (src/solver/pressure_backend_petsc.c).
//
// Same symbols, arguments and status codes as the PETSc backend.  The preconditioner names of
// fvm_petsc_set_pressure_solver select the Krylov kernel: "boomeramg" and "gamg" (the
// reference's algebraic-multigrid choices, pressure_backend_petsc.c:10, :533-537) run flexible CG
// with the FP32 aggregation-multigrid V-cycle of mlcg.cuh; "jacobi" (or -pc_type jacobi through
// fvm_petsc_insert_option), and the state before any selection, run the Jacobi-PCG of pcg.cuh.
// Conventions kept from the reference:
//  * indices are 1-based, face_neighbor_global <= 0 or skip_face != 0 drops a face;
//  * the operator is assembled once and cached; it is rebuilt when n_cells, n_faces or the
//    reference cell change (pressure_backend_petsc.c:687-715), coefficients are not re-read;
//  * the constant null space is used when no rank has Dirichlet rows (:770-800);
//  * non-finite rhs / guess entries are zeroed (:770-777);
//  * on Krylov failure the solve is retried from a zero guess with 4x the iteration cap, and a
//    DIVERGED_ITS result within 1e4 rtol or 1e3 atol is accepted (:878-961); otherwise the
//    status is -(1000 + reason);
//  * with fvm_petsc_set_io_on_device(1), rhs and solution are device pointers.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../../include/dopamine_b200.h"
#include "common.cuh"
#include "pcg.cuh"
#include "mlsolve.cuh"

namespace {
using namespace dpm::gpu;

struct Ctx {
  bool ready = false;
  int device = 0;
  cudaStream_t st = nullptr;
  int n = 0, nfaces = 0, ref_row = 0, WA = 0, grid = 0;
  int n_dir = 0;
  int *col = nullptr, *status = nullptr;
  unsigned* bar = nullptr;
  double *val = nullptr, *dinv = nullptr, *b = nullptr, *x = nullptr, *r = nullptr, *z = nullptr, *p0 = nullptr,
         *p1 = nullptr, *q = nullptr, *bp = nullptr, *part = nullptr, *dout = nullptr, *tot = nullptr;
  void* kernel = nullptr;
  dpm::gpu::MlSolver* ml = nullptr;  // multilevel solve of the current operator (AMG names)
  int ml_nullsp = -1;
  std::vector<int> hcol;             // host copy of the operator, kept for the multilevel set-up
  std::vector<double> hval;
  void release() {
    delete ml;
    ml = nullptr;
    ml_nullsp = -1;
    void* ps[] = {col, status, bar, val, dinv, b, x, r, z, p0, p1, q, bp, part, dout, tot};
    for (void* p : ps)
      if (p) cudaFree(p);
    col = status = nullptr;
    bar = nullptr;
    val = dinv = b = x = r = z = p0 = p1 = q = bp = part = dout = tot = nullptr;
    ready = false;
  }
};

Ctx g_ctx;
bool g_initialized = false;
int g_io_on_device = 0;
int g_local_rank = 0;
int g_force_maxit = 0;
int g_multilevel = 0;  // 1: the AMG names were selected
double g_force_rtol = -1.0;

template <class T>
int dalloc(T** p, size_t n) {
  return cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T)) == cudaSuccess ? 0 : -1;
}

int build(int n, int nfaces, const int* l2g, const int* fo, const int* fnl, const int* fng, const int* skip,
          const double* diag, const double* coeff, int ref_row) {
  g_ctx.release();
  std::vector<std::vector<std::pair<int, double>>> rows(n);
  for (int i = 0; i < n; ++i) {
    double dv = diag[i];
    if (!std::isfinite(dv) || std::fabs(dv) < 1.0e-20) dv = 1.0;
    rows[l2g[i] - 1].push_back({l2g[i] - 1, dv});
  }
  for (int f = 0; f < nfaces; ++f) {
    if (skip[f] != 0 || fng[f] <= 0) continue;
    int ol = fo[f] - 1;
    if (ol < 0 || ol >= n) continue;
    double c = coeff[f];
    if (!std::isfinite(c) || c == 0.0) continue;
    int og = l2g[ol] - 1, ng = fng[f] - 1;
    if (ng < 0 || ng >= n) return -16;  // single-rank operator: every neighbour is local
    rows[og].push_back({ng, -c});
    if (fnl[f] > 0) rows[ng].push_back({og, -c});
  }
  int WA = 0;
  std::vector<std::vector<int>> cols(n);
  std::vector<std::vector<double>> vals(n);
  for (int i = 0; i < n; ++i) {
    auto& r = rows[i];
    std::stable_sort(r.begin(), r.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    for (auto& e : r) {
      if (!cols[i].empty() && cols[i].back() == e.first) vals[i].back() += e.second;
      else { cols[i].push_back(e.first); vals[i].push_back(e.second); }
    }
    WA = std::max<int>(WA, (int)cols[i].size());
  }
  if (WA > 16) return -12;
  std::vector<int> hc((size_t)WA * n);
  for (int w = 0; w < WA; ++w)
    for (int i = 0; i < n; ++i) hc[(size_t)w * n + i] = i;  // padding (self, 0)
  std::vector<double> hv((size_t)WA * n, 0.0), hd(n, 1.0);
  for (int i = 0; i < n; ++i)
    for (size_t s = 0; s < cols[i].size(); ++s) {
      hc[s * n + i] = cols[i][s];
      hv[s * n + i] = vals[i][s];
      if (cols[i][s] == i) hd[i] = 1.0 / vals[i][s];
    }
  if (!g_ctx.st && cudaStreamCreateWithFlags(&g_ctx.st, cudaStreamNonBlocking) != cudaSuccess) return -10;
  if (dalloc(&g_ctx.col, hc.size()) || dalloc(&g_ctx.val, hv.size()) || dalloc(&g_ctx.dinv, n) ||
      dalloc(&g_ctx.b, n) || dalloc(&g_ctx.x, n) || dalloc(&g_ctx.r, n) || dalloc(&g_ctx.z, n) ||
      dalloc(&g_ctx.p0, n) || dalloc(&g_ctx.p1, n) || dalloc(&g_ctx.q, n) || dalloc(&g_ctx.bp, n) ||
      dalloc(&g_ctx.bar, 2) || dalloc(&g_ctx.status, 4) || dalloc(&g_ctx.dout, 4))
    return -11;
  cudaMemcpy(g_ctx.col, hc.data(), hc.size() * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(g_ctx.val, hv.data(), hv.size() * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(g_ctx.dinv, hd.data(), n * sizeof(double), cudaMemcpyHostToDevice);
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g_ctx.device);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg<double, 0, 0>, PCG_TPB, 0) != cudaSuccess || per_sm < 1)
    return -26;
  g_ctx.grid = std::min(sms * per_sm, (n + PCG_TPB - 1) / PCG_TPB);
  if (g_ctx.grid < 1) g_ctx.grid = 1;
  int cpt = 0;
  g_ctx.kernel = pcg_kernel_for<double>(n, g_ctx.grid, WA, &cpt);
  int per_sm2 = 0;
  cudaFuncSetAttribute(g_ctx.kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 5);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm2, g_ctx.kernel, PCG_TPB, 0) != cudaSuccess || per_sm2 < 1)
    return -26;
  if (sms * per_sm2 < g_ctx.grid) {
    g_ctx.grid = sms * per_sm2;
    g_ctx.kernel = pcg_kernel_for<double>(n, g_ctx.grid, WA, &cpt);
    cudaFuncSetAttribute(g_ctx.kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 5);
  }
  if (dalloc(&g_ctx.part, 8 * (size_t)g_ctx.grid)) return -11;
  g_ctx.n = n;
  g_ctx.nfaces = nfaces;
  g_ctx.ref_row = ref_row;
  g_ctx.WA = WA;
  g_ctx.hcol = std::move(hc);
  g_ctx.hval = std::move(hv);
  g_ctx.ready = true;
  return 0;
}

// Multilevel solve of the cached operator; its hierarchy is built on first use and again when
// the null-space setting changes.
int run_ml(double rtol, double atol, int maxit, int* reason, int* its, double* resid) {
  const int nullsp = g_ctx.n_dir > 0 ? 0 : 1;
  if (!g_ctx.ml || g_ctx.ml_nullsp != nullsp) {
    delete g_ctx.ml;
    g_ctx.ml = new dpm::gpu::MlSolver();
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g_ctx.device);
    if (g_ctx.ml->setup(g_ctx.n, g_ctx.WA, g_ctx.hcol.data(), g_ctx.hval.data(), g_ctx.col, g_ctx.val, nullsp != 0, 0,
                        0, 0.0, sms, g_ctx.bar, g_ctx.status, g_ctx.dout)) {
      delete g_ctx.ml;
      g_ctx.ml = nullptr;
      return -26;
    }
    g_ctx.ml_nullsp = nullsp;
  }
  int rc = g_ctx.ml->launch(g_ctx.b, g_ctx.x, rtol, atol, maxit, 0, g_ctx.st, reason, its, resid);
  return rc ? -33 : 0;
}

int run_pcg(double rtol, double atol, int maxit, int guess_zero, int* reason, int* its, double* resid) {
  PcgArgs<double> a{};
  a.n = g_ctx.n; a.WA = g_ctx.WA; a.col = g_ctx.col; a.val = g_ctx.val; a.dinv = g_ctx.dinv;
  a.b = g_ctx.b; a.x = g_ctx.x; a.r = g_ctx.r; a.z = g_ctx.z; a.p0 = g_ctx.p0; a.p1 = g_ctx.p1; a.q = g_ctx.q;
  a.bp = g_ctx.bp; a.partials = g_ctx.part; a.bar = g_ctx.bar; a.status = g_ctx.status;
  a.dout = g_ctx.dout;
  a.rtol = rtol; a.atol = atol; a.maxit = maxit; a.nullsp = g_ctx.n_dir > 0 ? 0 : 1; a.guess_zero = guess_zero;
  cudaMemsetAsync(g_ctx.bar, 0, 2 * sizeof(unsigned), g_ctx.st);
  cudaMemsetAsync(g_ctx.status, 0, 4 * sizeof(int), g_ctx.st);
  void* args[] = {&a};
  if (cudaLaunchCooperativeKernel(g_ctx.kernel, dim3(g_ctx.grid), dim3(PCG_TPB), args, 0, g_ctx.st) != cudaSuccess)
    return -33;
  int hs[4];
  double hd[4];
  cudaMemcpyAsync(hs, g_ctx.status, sizeof(hs), cudaMemcpyDeviceToHost, g_ctx.st);
  cudaMemcpyAsync(hd, g_ctx.dout, sizeof(hd), cudaMemcpyDeviceToHost, g_ctx.st);
  if (cudaStreamSynchronize(g_ctx.st) != cudaSuccess) return -33;
  if (hs[2]) return -34;  // barrier timeout
  *reason = hs[0];
  *its = hs[1];
  *resid = hd[0];
  return 0;
}

__global__ void k_scrub(int n, double* v) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && !(fabs(v[i]) <= 1.7976931348623157e308)) v[i] = 0.0;
}

}  // namespace

extern "C" {

int fvm_petsc_backend_available(void) {
  int n = 0;
  return (cudaGetDeviceCount(&n) == cudaSuccess && n > 0) ? 1 : 0;
}

int fvm_petsc_backend_initialize(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return -1;
  g_ctx.device = n > 0 ? g_local_rank % n : 0;
  if (cudaSetDevice(g_ctx.device) != cudaSuccess) return -1;
  g_initialized = true;
  return 0;
}

int fvm_petsc_backend_finalize(void) {
  g_ctx.release();
  if (g_ctx.st) {
    cudaStreamDestroy(g_ctx.st);
    g_ctx.st = nullptr;
  }
  g_initialized = false;
  return 0;
}

void fvm_petsc_set_pressure_solver(const char* solver_name) {
  if (!solver_name) return;
  if (std::strncmp(solver_name, "boomeramg", 9) == 0 || std::strncmp(solver_name, "gamg", 4) == 0) g_multilevel = 1;
  else if (std::strncmp(solver_name, "jacobi", 6) == 0) g_multilevel = 0;
}

int fvm_petsc_device_io_supported(void) { return 1; }

void fvm_petsc_set_io_on_device(int on) { g_io_on_device = on ? 1 : 0; }

void fvm_petsc_insert_option(const char* opt) {
  if (!opt) return;
  std::string s(opt);
  auto val = [&](const char* key) -> const char* {
    size_t k = s.find(key);
    if (k == std::string::npos) return nullptr;
    size_t v = s.find_first_not_of(" =", k + std::strlen(key));
    return v == std::string::npos ? nullptr : s.c_str() + v;
  };
  if (const char* v = val("-ksp_max_it")) g_force_maxit = std::atoi(v);
  if (const char* v = val("-ksp_rtol")) g_force_rtol = std::atof(v);
  if (const char* v = val("-pc_type")) {
    if (std::strncmp(v, "jacobi", 6) == 0) g_multilevel = 0;
    else if (std::strncmp(v, "hypre", 5) == 0 || std::strncmp(v, "gamg", 4) == 0) g_multilevel = 1;
  }
}

void fvm_petsc_set_device_local_rank(int local_rank) { g_local_rank = local_rank; }

int fvm_petsc_solve_pressure(int n_cells_local, int n_cells_global, int n_faces, const int* local_to_global,
                             const int* face_owner, const int* face_neighbor_local, const int* face_neighbor_global,
                             const int* skip_face, const double* diagonal, const double* rhs, const double* face_coeff,
                             int reference_cell, int max_iterations, double rtol, double atol, const int* dirichlet_rows,
                             const double* dirichlet_values, int n_dirichlet_rows, double* solution,
                             int* iteration_count, double* residual_norm) {
  (void)dirichlet_rows;
  (void)dirichlet_values;
  if (n_cells_local != n_cells_global) return -1;  // one rank per GPU, whole mesh on this GPU
  if (!g_initialized && fvm_petsc_backend_initialize() != 0) return -1;
  cudaSetDevice(g_ctx.device);
  int ref = reference_cell - 1;
  if (ref < 0 || ref >= n_cells_global) ref = 0;
  if (!g_ctx.ready || g_ctx.n != n_cells_local || g_ctx.nfaces != n_faces || g_ctx.ref_row != ref) {
    int rc = build(n_cells_local, n_faces, local_to_global, face_owner, face_neighbor_local, face_neighbor_global,
                   skip_face, diagonal, face_coeff, ref);
    if (rc) {
      g_ctx.release();
      return rc;
    }
  }
  g_ctx.n_dir = n_dirichlet_rows > 0 ? n_dirichlet_rows : 0;
  const size_t nbytes = (size_t)n_cells_local * sizeof(double);
  cudaMemcpyKind kin = g_io_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  if (cudaMemcpyAsync(g_ctx.b, rhs, nbytes, kin, g_ctx.st) != cudaSuccess) return -15;
  if (cudaMemcpyAsync(g_ctx.x, solution, nbytes, kin, g_ctx.st) != cudaSuccess) return -25;
  int nb = (n_cells_local + TPB - 1) / TPB;
  k_scrub<<<nb, TPB, 0, g_ctx.st>>>(n_cells_local, g_ctx.b);
  k_scrub<<<nb, TPB, 0, g_ctx.st>>>(n_cells_local, g_ctx.x);
  int maxit = std::max(max_iterations, 2000);
  if (g_force_maxit > 0) maxit = g_force_maxit;
  if (g_force_rtol > 0.0) rtol = g_force_rtol;
  int reason = 0, its = 0;
  double res = 0.0;
  int rc = g_multilevel ? run_ml(rtol, atol, maxit, &reason, &its, &res) : run_pcg(rtol, atol, maxit, 0, &reason, &its, &res);
  if (rc) return rc;
  int status = 0;
  if (reason < 0) {  // retry as the reference does after a failed solve: from zero, 4x the cap, Jacobi
    rc = run_pcg(rtol, atol, 4 * maxit, 1, &reason, &its, &res);
    if (rc) return rc;
    if (reason < 0 && !(reason == -3 && (res < rtol * 1.0e4 || res < atol * 1.0e3))) status = -(1000 + reason);
  }
  *iteration_count = its;
  *residual_norm = res;
  cudaMemcpyKind kout = g_io_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  if (cudaMemcpyAsync(solution, g_ctx.x, nbytes, kout, g_ctx.st) != cudaSuccess) return -43;
  if (cudaStreamSynchronize(g_ctx.st) != cudaSuccess) return -43;
  return status;
}

}  // extern "C"
