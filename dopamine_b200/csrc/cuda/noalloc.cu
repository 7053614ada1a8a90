// Allocation-free Jacobi-PCG solve: dpm_pcg_solve_noalloc (include/dopamine_b200.h).
//
// Some callers cannot allocate device memory at the point where they need a pressure solve:
// hosts whose device memory is entirely owned by their own pool allocator (for example a
// framework's caching allocator, or a Fortran host that reserves all memory at start-up), and
// code paths where cudaMalloc is not acceptable because it can synchronize the device (tight
// time-stepping loops with latency budgets).  For them this entry point takes the operator,
// right-hand side and solution as caller-owned device buffers and keeps every work vector of
// the solve in one file-scope __device__ array of fixed size, so it calls no cudaMalloc,
// cudaFree or allocating library routine.
//
// Limits and behaviour a caller must know:
//  * at most DPM_NOALLOC_MAX_CELLS cells and rows of at most 16 entries; larger problems are
//    rejected with DPM_ERR_ARG and a message on stderr;
//  * the scratch array (about 5.3 MB) belongs to this library's device module.  The CUDA runtime
//    loads modules lazily, so the array (and the solve kernels' code) is created on a device by
//    the first call on that device, not when the library is loaded; from then on it is held
//    until the process exits.  That first call can fail with DPM_ERR_CUDA when the device has no
//    free memory left.  A call with max_iterations == 0 does only this per-device set-up (module
//    load, every solve kernel variant, the array's address) and returns 0 without touching any
//    array argument: make it before the host's pool reserves the device's memory;
//  * all calls share that one array and it keeps the last call's contents; each call clears
//    the parts that must start at zero (barrier counter, status words) itself;
//  * calls that overlap on the GPU (two streams, or two host threads) race on the array and must
//    be serialized by the caller;
//  * the array's device address is looked up (cudaGetSymbolAddress) on every call, so a device
//    reset that reloads the module is followed correctly.
#include <cuda_runtime.h>

#include <cstdio>

#include "../../../include/dopamine_b200.h"
#include "common.cuh"
#include "pcg.cuh"

namespace {
using namespace dpm::gpu;

constexpr int kMaxCells = DPM_NOALLOC_MAX_CELLS;
constexpr int kMaxBlocks = 1024;
// doubles: r, z, p0, p1, q (5 x kMaxCells), partials (2 x 4 x kMaxBlocks), dout (4);
// then unsigned bar (4) and int status (4)
constexpr size_t kVecOff = 0;
constexpr size_t kPartOff = 5ull * kMaxCells;
constexpr size_t kDoutOff = kPartOff + 8ull * kMaxBlocks;
constexpr size_t kNumDoubles = kDoutOff + 4;
constexpr size_t kScratchBytes = kNumDoubles * sizeof(double) + 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// The array's device address on the current device.  The symbol name itself is only a host
// stand-in: a kernel handed it would read the wrong memory.  Loads the module on first use.
int scratch_address(void** ptr) {
  *ptr = nullptr;
  cudaError_t e = cudaGetSymbolAddress(ptr, g_noalloc_scratch);
  if (e != cudaSuccess || !*ptr) {
    std::fprintf(stderr, "dpm_pcg_solve_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
    return DPM_ERR_CUDA;
  }
  return 0;
}

// Every k_pcg instantiation the solve can pick (cells per thread 0..4, row width 7 or runtime):
// querying their attributes makes the runtime load them now rather than at a later launch.
int preload_kernels() {
  const void* ks[] = {(const void*)k_pcg<double, 0, 7>, (const void*)k_pcg<double, 1, 7>,
                      (const void*)k_pcg<double, 2, 7>, (const void*)k_pcg<double, 3, 7>,
                      (const void*)k_pcg<double, 4, 7>, (const void*)k_pcg<double, 0, 0>,
                      (const void*)k_pcg<double, 1, 0>, (const void*)k_pcg<double, 2, 0>,
                      (const void*)k_pcg<double, 3, 0>, (const void*)k_pcg<double, 4, 0>};
  for (const void* k : ks) {
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, k) != cudaSuccess) return DPM_ERR_CUDA;
    if (cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 5) != cudaSuccess) return DPM_ERR_CUDA;
  }
  return 0;
}

}  // namespace

extern "C" int dpm_pcg_solve_noalloc(int n_cells, int row_width, const int* col, const double* val,
                                     const double* inv_diag, const double* rhs, double* x, double rtol, double atol,
                                     int max_iterations, int null_space, void* stream, int* iteration_count,
                                     double* residual_norm) {
  if (n_cells < 1 || n_cells > kMaxCells || row_width < 1 || row_width > 16) {
    std::fprintf(stderr,
                 "dpm_pcg_solve_noalloc: n_cells=%d row_width=%d outside the supported range "
                 "(1..%d cells, rows of 1..16 entries); use fvm_petsc_solve_pressure for larger systems\n",
                 n_cells, row_width, kMaxCells);
    return DPM_ERR_ARG;
  }
  if (!iteration_count || !residual_norm || max_iterations < 0) return DPM_ERR_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return DPM_ERR_CUDA;
  void* scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc) return rc;
  if (max_iterations == 0) {  // per-device set-up only: no array argument is read
    rc = preload_kernels();
    if (rc) return rc;
    *iteration_count = 0;
    *residual_norm = 0.0;
    return DPM_OK;
  }
  if (!col || !val || !inv_diag || !rhs || !x) return DPM_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  int sms = 0, per_sm = 0, cpt = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return DPM_ERR_CUDA;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg<double, 0, 0>, PCG_TPB, 0) != cudaSuccess ||
      per_sm < 1)
    return DPM_ERR_CUDA;
  int grid = sms * per_sm;
  if (grid > (n_cells + PCG_TPB - 1) / PCG_TPB) grid = (n_cells + PCG_TPB - 1) / PCG_TPB;
  if (grid > kMaxBlocks) grid = kMaxBlocks;
  if (grid < 1) grid = 1;
  void* kernel = pcg_kernel_for<double>(n_cells, grid, row_width, &cpt);
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 5) != cudaSuccess) return DPM_ERR_CUDA;
  int per_sm2 = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm2, kernel, PCG_TPB, 0) != cudaSuccess || per_sm2 < 1)
    return DPM_ERR_CUDA;
  if (grid > sms * per_sm2) {
    grid = sms * per_sm2;
    kernel = pcg_kernel_for<double>(n_cells, grid, row_width, &cpt);
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 5) != cudaSuccess)
      return DPM_ERR_CUDA;
  }

  double* base = static_cast<double*>(scratch);
  unsigned* bar = reinterpret_cast<unsigned*>(base + kNumDoubles);
  int* status = reinterpret_cast<int*>(bar + 4);
  // barrier counter and status words must start at zero; the rest is overwritten by the solve
  if (cudaMemsetAsync(bar, 0, 4 * sizeof(unsigned) + 4 * sizeof(int), st) != cudaSuccess) return DPM_ERR_CUDA;

  PcgArgs<double> a{};
  a.n = n_cells;
  a.WA = row_width;
  a.col = col;
  a.val = val;
  a.dinv = inv_diag;
  a.b = rhs;
  a.x = x;
  a.r = base + kVecOff;
  a.z = base + kVecOff + 1ull * kMaxCells;
  a.p0 = base + kVecOff + 2ull * kMaxCells;
  a.p1 = base + kVecOff + 3ull * kMaxCells;
  a.q = base + kVecOff + 4ull * kMaxCells;
  a.bp = a.r;
  a.partials = base + kPartOff;
  a.bar = bar;
  a.status = status;
  a.dout = base + kDoutOff;
  a.rtol = rtol;
  a.atol = atol;
  a.maxit = max_iterations;
  a.nullsp = null_space ? 1 : 0;
  a.guess_zero = 0;
  void* args[] = {&a};
  if (cudaLaunchCooperativeKernel(kernel, dim3(grid), dim3(PCG_TPB), args, 0, st) != cudaSuccess) return DPM_ERR_CUDA;
  int hs[4];
  double hd[4];
  if (cudaMemcpyAsync(hs, status, sizeof(hs), cudaMemcpyDeviceToHost, st) != cudaSuccess) return DPM_ERR_CUDA;
  if (cudaMemcpyAsync(hd, a.dout, sizeof(hd), cudaMemcpyDeviceToHost, st) != cudaSuccess) return DPM_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return DPM_ERR_CUDA;
  if (hs[2]) {
    std::fprintf(stderr, "dpm_pcg_solve_noalloc: grid barrier timed out\n");
    return DPM_ERR_CUDA;
  }
  *iteration_count = hs[1];
  *residual_norm = hd[0];
  return hs[0] < 0 ? -(1000 + hs[0]) : DPM_OK;
}
