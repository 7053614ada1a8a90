// Device-resident RK3W fractional-step solver and its C ABI (include/dopamine_b200.h).
//
// The stage sequence mirrors advance_rk3w (src/solver/mod_fv_solver.f90:1180-1614): BC refresh,
// velocity gradients, SGS viscosity, wall model, explicit right-hand side and predictor,
// pre-correction with the old pressure, second gradient pass, Poisson block with Jasak
// correctors, flux and velocity projection, rotational pressure correction, pressure update.
// All fields stay in HBM; the host only launches kernels and reads back the few scalars that
// steer the control flow (CFL-clamped dt, corrector exit test, Krylov status).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <memory>
#include <string>
#include <vector>

#include "../../../include/dopamine_b200.h"
#include "../host/mesh.hpp"
#include "../host/fortran_records.hpp"
#include "../host/ops.hpp"
#include "../host/twolevel.hpp"
#include "../host/multilevel.hpp"
#include "cellproj.cuh"
#include "common.cuh"
#include "explicit32.cuh"
#include "fcg.cuh"
#include "forcing.cuh"
#include "kernels.cuh"
#include "learn.cuh"
#include "mlsolve.cuh"
#include "pcg.cuh"
#include "sampling.cuh"
#include "sem.cuh"
#include "scalars.cuh"
#include "setup_gpu.hpp"

namespace dpm {
namespace gpu {

const double RK3W_ALPHA[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};  // src/mod_parameters.f90:64-71
const double RK3W_BETA[3] = {0.0, -17.0 / 60.0, -5.0 / 12.0};
const double RK3W_GAMMA[3] = {8.0 / 15.0, 2.0 / 15.0, 1.0 / 3.0};
const double RK3W_C[3] = {0.0, 8.0 / 15.0, 2.0 / 3.0};

#define CK(x)                                                                                      \
  do {                                                                                             \
    cudaError_t e_ = (x);                                                                          \
    if (e_ != cudaSuccess) {                                                                       \
      std::fprintf(stderr, "dopamine_b200: CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, \
                   __LINE__);                                                                      \
      return DPM_ERR_CUDA;                                                                         \
    }                                                                                              \
  } while (0)

struct DMem {
  std::vector<void*> ptrs;
  ~DMem() {
    for (void* p : ptrs) cudaFree(p);
  }
  template <class T>
  T* alloc(size_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return nullptr;
    cudaMemset(p, 0, std::max<size_t>(n, 1) * sizeof(T));
    ptrs.push_back(p);
    return static_cast<T*>(p);
  }
  template <class T>
  T* upload(const std::vector<T>& v) {
    T* p = alloc<T>(v.size());
    if (p && !v.empty()) cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    return p;
  }
};

inline int nblk(int64_t n) { return (int)((n + TPB - 1) / TPB); }

// ---- deterministic reductions: per-block partials, then one block sums them in order --------
enum RedMode { RED_MAXABS = 0, RED_SUM2 = 1, RED_UBULK = 2, RED_STATS = 3, RED_MAX2 = 4, RED_DIVSTAT = 5 };
constexpr int RED_NV = 10;

struct RedArgs {
  int mode, n;
  const double *a, *b, *c, *vol, *gU, *nus;
  double nu;
};

__global__ void __launch_bounds__(TPB) k_reduce_partial(RedArgs r, double* partials) {
  double v[RED_NV];
  for (int k = 0; k < RED_NV; ++k) v[k] = 0.0;
  const int n = r.n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    switch (r.mode) {
      case RED_MAXABS: v[0] = fmax(v[0], fabs(r.a[i])); break;
      case RED_SUM2: v[0] += r.a[i] * r.b[i]; v[1] += r.b[i]; break;
      case RED_UBULK: {
        double u0 = r.a[i], u1 = r.a[n + i], u2 = r.a[2 * n + i];
        v[0] += sqrt(u0 * u0 + u1 * u1 + u2 * u2) * r.vol[i];
        v[1] += r.vol[i];
        break;
      }
      case RED_MAX2: v[0] = fmax(v[0], r.a[i]); v[1] = fmax(v[1], r.b[i]); break;
      case RED_STATS: {
        double vv = r.vol[i];
        double u0 = r.a[i], u1 = r.a[n + i], u2 = r.a[2 * n + i];
        const double* g = r.gU;
        double S11 = g[0 * n + i], S22 = g[4 * n + i], S33 = g[8 * n + i];
        double S12 = 0.5 * (g[1 * n + i] + g[3 * n + i]), S13 = 0.5 * (g[2 * n + i] + g[6 * n + i]);
        double S23 = 0.5 * (g[5 * n + i] + g[7 * n + i]);
        double SS = S11 * S11 + S22 * S22 + S33 * S33 + 2.0 * (S12 * S12 + S13 * S13 + S23 * S23);
        v[0] += 0.5 * (u0 * u0 + u1 * u1 + u2 * u2) * vv;
        v[1] += vv;
        v[2] += (r.nu + r.nus[i]) * SS * vv;
        v[3] += u0 * vv; v[4] += u1 * vv; v[5] += u2 * vv;
        v[6] += r.nus[i] * vv;
        v[7] = fmax(v[7], sqrt(u0 * u0 + u1 * u1 + u2 * u2));
        break;
      }
      case RED_DIVSTAT: v[0] = fmax(v[0], fabs(r.a[i])); v[1] += fabs(r.a[i]) * r.vol[i]; v[2] += r.vol[i]; break;
    }
  }
  __shared__ double sh[TPB / 32][RED_NV];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int k = 0; k < RED_NV; ++k) {
    bool mx = (r.mode == RED_MAXABS && k == 0) || (r.mode == RED_MAX2 && k < 2) || (r.mode == RED_STATS && k == 7) ||
              (r.mode == RED_DIVSTAT && k == 0);
    double t = v[k];
    for (int o = 16; o > 0; o >>= 1) {
      double u = __shfl_down_sync(0xffffffffu, t, o);
      t = mx ? fmax(t, u) : t + u;
    }
    if (lane == 0) sh[w][k] = t;
  }
  __syncthreads();
  if (threadIdx.x < RED_NV) {
    int k = threadIdx.x;
    bool mx = (r.mode == RED_MAXABS && k == 0) || (r.mode == RED_MAX2 && k < 2) || (r.mode == RED_STATS && k == 7) ||
              (r.mode == RED_DIVSTAT && k == 0);
    double t = sh[0][k];
    for (int j = 1; j < TPB / 32; ++j) t = mx ? fmax(t, sh[j][k]) : t + sh[j][k];
    partials[blockIdx.x * RED_NV + k] = t;
  }
}

// One warp per component: lane l folds partials l, l+32, ... in order, then a fixed shuffle tree,
// so the result does not depend on scheduling.
__global__ void __launch_bounds__(32 * RED_NV) k_reduce_final(int mode, int nparts, const double* partials, double* out) {
  const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (k >= RED_NV) return;
  bool mx = (mode == RED_MAXABS && k == 0) || (mode == RED_MAX2 && k < 2) || (mode == RED_STATS && k == 7) ||
            (mode == RED_DIVSTAT && k == 0);
  double t = 0.0;
  for (int j = lane; j < nparts; j += 32) t = mx ? fmax(t, partials[j * RED_NV + k]) : t + partials[j * RED_NV + k];
  for (int o = 16; o > 0; o >>= 1) {
    double u = __shfl_down_sync(0xffffffffu, t, o);
    t = mx ? fmax(t, u) : t + u;
  }
  if (lane == 0) out[k] = t;
}

// anchor_pressure_to_outlet (mod_fv_solver.f90:3610-3641): shift = sum(p V) / V_total.
__global__ void k_anchor_shift(const double* sums, double vtot, double* shift) { *shift = vtot > 0.0 ? sums[0] / vtot : 0.0; }

// ------------------------------------------------------------------------------------------
struct Solver {
  int device = 0;
  cudaStream_t st = nullptr;
  Mesh m;
  StaticOps S;
  dpm_params_t P{};
  std::vector<dpm_patch_cfg_t> pc;
  DMem mem;
  Dev d{};
  Fld F{};
  int nc = 0, nf = 0, nb = 0, nfp = 0;
  // scratch
  double *red_part = nullptr, *red_out = nullptr, *scratch_c = nullptr, *scratch_c2 = nullptr;
  double *aos_buf = nullptr;
  double *conv_tmp = nullptr, *visc_tmp = nullptr;
  double* U_spare = nullptr;  // second velocity buffer: the fused explicit pass writes the prediction here
  // precision form, explicit half in FP32 (explicit32.cuh): FP32 geometry, first-pass gradients,
  // scalar face fluxes
  bool x32 = false;
  Geo32 g32{};
  float *gU32 = nullptr, *gS32 = nullptr, *sc_fadv32 = nullptr, *sc_fdif32 = nullptr;
  // synthetic-eddy inflow (sem.cuh): configuration, state (device arrays; the generator state
  // advances in the device copy), ABL-inlet faces, their fluctuation and reduction partials
  bool sem_on = false;
  SemCfg sem_cfg{};
  SemState sem_h{};
  SemState* sem_d = nullptr;
  int* sem_faces = nullptr;
  int sem_nfaces = 0, sem_grid = 1;
  double *sem_fluc = nullptr, *sem_part = nullptr;
  // mass-flux forcing of the current step; Davies nudging profiles; passive-scalar sources
  double mass_flux_force[3] = {0.0, 0.0, 0.0};
  int nd_nt = 0, nd_nz = 0;
  std::vector<double> nd_times_h, nd_z_h;
  double *nd_z = nullptr, *nd_U = nullptr, *nd_T = nullptr;
  std::vector<dpm_scalar_source_t> srcs;
  std::vector<double*> src_tags;  // device tag points per source (null when none)
  // sample points (sampling.cuh): coordinates (3, n), owner cells, payload (6, n)
  int samp_n = 0;
  double *samp_pts = nullptr, *samp_payload = nullptr;
  int* samp_owner = nullptr;
  // exact cell projection (cellproj.cuh): work vectors, partials and device scalars, allocated
  // on first use; outer and preconditioner iterations of the current step
  bool cp_on = false;
  double *cp_x = nullptr, *cp_r = nullptr, *cp_z = nullptr, *cp_p = nullptr, *cp_q = nullptr, *cp_rold = nullptr,
         *cp_v = nullptr, *cp_bconst = nullptr, *cp_part = nullptr;
  CpState* cp_st = nullptr;
  int cp_iters = 0, cp_precond_iters = 0;
  // PCG workspace
  double *cg_r, *cg_z, *cg_p0, *cg_p1, *cg_q, *cg_bp, *cg_x, *cg_part, *cg_dout;
  void* cg_kernel = nullptr;
  int cg_cpt = 0;
  unsigned* cg_bar;
  int* cg_status;
  int cg_grid = 0;
  bool cg_coop = true;
  // temperature (transported when Boussinesq is on) and passive scalars, scalar-major
  double *Tb = nullptr, *gT = nullptr, *HT = nullptr, *HT0 = nullptr;
  int ns = 0;
  double *Cs = nullptr, *Cb = nullptr, *gC = nullptr, *HC = nullptr, *HC0 = nullptr;
  double *sc_fadv = nullptr, *sc_fdif = nullptr, *bTval = nullptr, *bsval = nullptr;
  int* bsmode = nullptr;
  double *most_L = nullptr, *most_qw = nullptr;  // MOST per-face Obukhov length and heat flux
  double *most_z0m = nullptr, *most_z0h = nullptr;  // MOST per-face roughness lengths
  // learned term of the two-level preconditioner (learn.cuh)
  int lp_S = 32, lp_count = 0, lp_stride = 10, lp_val_lo = 0;
  bool lp_recording = false, lp_ready = false;
  float lp_gamma = 0.0f;
  float *lp_feat = nullptr, *lp_omega = nullptr, *lp_h1 = nullptr, *lp_h2 = nullptr, *lp_pre = nullptr,
        *lp_dom = nullptr, *lp_prm = nullptr, *lp_m1 = nullptr, *lp_m2 = nullptr, *lp_grad = nullptr,
        *lp_gpart = nullptr;
  unsigned short* lp_wb = nullptr;
  double *lp_r = nullptr, *lp_z = nullptr, *lp_u = nullptr, *lp_x = nullptr, *lp_azb = nullptr, *lp_av = nullptr,
         *lp_dpart = nullptr, *lp_dsum = nullptr, *lp_coef = nullptr;
  std::vector<int> lp_solve_of;  // solve index of each recorded slot
  int lp_solves = 0, p_fallbacks = 0;
  // two-level flexible CG (p_solver == DPM_PSOLVER_TWOLEVEL_FCG)
  bool use_fcg = false;
  FcgArgs fa{};
  int fcg_WA = 0;
  void* fcg_kernel = nullptr;
  bool fcg_mixed = false;
  bool inner_rel_is_first_ = true;
  size_t fcg_smem = 0;
  // multilevel flexible CG (p_solver == DPM_PSOLVER_MULTILEVEL_FCG)
  bool use_ml = false;
  MlSolver ml;
  bool ml_learn_ready = false;   // the learned term's partition and buffers exist for the multilevel form
  int* ml_pinv = nullptr;        // [n] position of each cell in the learned term's numbering
  float* ml_omega = nullptr;     // [n] omega in the mesh numbering
  int dev_sms_ = 0;
  double *gg_prevU = nullptr, *gg_prevS = nullptr;  // Green-Gauss previous-sweep gradients
  // state
  double time = 0.0;
  int64_t step = 0;
  bool u_face_ready = false;
  bool filt_ready = false;
  int64_t launches = 0;
  dpm_stats_t last{};
  double last_step_ms = 0.0, last_poisson_ms = 0.0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, evp0 = nullptr, evp1 = nullptr;
  double poisson_ms_acc = 0.0;
  int spin_limit = 0;  // > 0: poll limit of the Krylov kernels' grid-wide waits (failure-detection tests)
  bool force_plain = false;  // dpm_select_pressure_solver: plain Jacobi-PCG although a flexible form is set up
  SetupTimes setup_t;        // set-up stage times of init
  double* fcg_phase = nullptr;  // dpm_fcg_phase_times: per-phase ns of the two-level kernel, [8]
  double setup_upload_ms = 0.0, setup_total_ms = 0.0, setup_psolver_ms = 0.0;
  bool flexible() const { return (use_fcg || use_ml) && !force_plain; }

  ~Solver() {
    free_samples();
    free_sources();
    for (double* p : {nd_z, nd_U, nd_T})
      if (p) cudaFree(p);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (evp0) cudaEventDestroy(evp0);
    if (evp1) cudaEventDestroy(evp1);
    if (st) cudaStreamDestroy(st);
  }

  int init(const dpm_raw_mesh_t* raw, const dpm_patch_cfg_t* patches, const dpm_params_t* prm, int dev) {
    device = dev;
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    CK(cudaEventCreate(&ev0)); CK(cudaEventCreate(&ev1)); CK(cudaEventCreate(&evp0)); CK(cudaEventCreate(&evp1));
    RawMesh r;
    r.n_nodes = raw->n_nodes; r.xyz = raw->xyz; r.n_cells = raw->n_cells; r.cell_type = raw->cell_type;
    r.cell_off = raw->cell_off; r.cell_nodes = raw->cell_nodes; r.n_bfaces = raw->n_bfaces;
    r.bface_off = raw->bface_off; r.bface_nodes = raw->bface_nodes; r.bface_patch = raw->bface_patch;
    r.n_patches = raw->n_patches;
    std::vector<int> pbc(raw->n_patches);
    for (int i = 0; i < raw->n_patches; ++i) pbc[i] = patches[i].bc_id;
    std::string err;
    using Clk = std::chrono::steady_clock;
    auto ms_between = [](Clk::time_point a, Clk::time_point b) {
      return std::chrono::duration<double, std::milli>(b - a).count();
    };
    const auto t_begin = Clk::now();
    P = *prm;
    if (P.cell_projection != DPM_CELL_PROJECTION_LS && P.cell_projection != DPM_CELL_PROJECTION_EXACT) return DPM_ERR_ARG;
    cp_on = P.cell_projection == DPM_CELL_PROJECTION_EXACT;
    pc.assign(patches, patches + raw->n_patches);
    if (P.host_setup) {
      if (build_mesh(r, pbc.data(), m, &err)) {
        std::fprintf(stderr, "dopamine_b200: mesh set-up failed: %s\n", err.c_str());
        return DPM_ERR_MESH;
      }
      const auto t_mesh = Clk::now();
      {
          const int rs = build_static_ops(m, pc.data(), P, S);  // rows wider than 16: unsupported
          if (rs) return rs == DPM_ERR_UNSUPPORTED ? rs : DPM_ERR_MESH;
        }
      setup_t.mesh_ms = ms_between(t_begin, t_mesh);
      setup_t.ops_ms = ms_between(t_mesh, Clk::now());
    }
    SetupDeviceArrays da;
    if (!P.host_setup) {
      int rc = build_setup_device(r, pc.data(), P, device, m, S, &err, &setup_t, &da);
      if (rc == SETUP_DEVICE_LIMIT) {  // beyond the device builder's per-cell limits: the host builder
        std::fprintf(stderr, "dopamine_b200: %s; building the mesh on the host\n", err.c_str());
        P.host_setup = 1;
        const auto t_h = Clk::now();
        if (build_mesh(r, pbc.data(), m, &err)) {
          std::fprintf(stderr, "dopamine_b200: mesh set-up failed: %s\n", err.c_str());
          return DPM_ERR_MESH;
        }
        const auto t_mesh = Clk::now();
        {
          const int rs = build_static_ops(m, pc.data(), P, S);  // rows wider than 16: unsupported
          if (rs) return rs == DPM_ERR_UNSUPPORTED ? rs : DPM_ERR_MESH;
        }
        setup_t = SetupTimes();
        setup_t.mesh_ms = ms_between(t_h, t_mesh);
        setup_t.ops_ms = ms_between(t_mesh, Clk::now());
      } else if (rc) {
        std::fprintf(stderr, "dopamine_b200: device set-up failed: %s\n", err.c_str());
        return (rc < 0 && rc >= -4) ? DPM_ERR_MESH : rc;  // build_mesh's codes -1..-4
      }
    }
    if (m.n_cells > 2000000000LL || m.n_faces > 2000000000LL) return DPM_ERR_UNSUPPORTED;
    nc = (int)m.n_cells; nf = (int)m.n_faces; nb = (int)m.n_bnd_faces; nfp = (int)S.nfp;
    const auto t_up = Clk::now();
    int rc = upload(P.host_setup ? nullptr : &da);
    setup_upload_ms = ms_between(t_up, Clk::now());
    setup_total_ms = ms_between(t_begin, Clk::now());
    return rc;
  }

  // Polyhedral mesh (dpm_create_poly): the device builder (or the host one with host_setup).
  int init_poly(const dpm_poly_mesh_t* pmsh, const dpm_patch_cfg_t* patches, const dpm_params_t* prm, int dev) {
    device = dev;
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    CK(cudaEventCreate(&ev0)); CK(cudaEventCreate(&ev1)); CK(cudaEventCreate(&evp0)); CK(cudaEventCreate(&evp1));
    PolyMesh pm;
    pm.n_points = pmsh->n_points; pm.xyz = pmsh->xyz; pm.n_faces = pmsh->n_faces; pm.face_off = pmsh->face_off;
    pm.face_nodes = pmsh->face_nodes; pm.owner = pmsh->owner; pm.n_int_faces = pmsh->n_int_faces;
    pm.neighbour = pmsh->neighbour; pm.n_patches = pmsh->n_patches; pm.patch_start = pmsh->patch_start;
    pm.patch_nfaces = pmsh->patch_nfaces;
    std::vector<int> pbc(pmsh->n_patches);
    for (int i = 0; i < pmsh->n_patches; ++i) pbc[i] = patches[i].bc_id;
    using Clk = std::chrono::steady_clock;
    auto ms_between = [](Clk::time_point a, Clk::time_point b) {
      return std::chrono::duration<double, std::milli>(b - a).count();
    };
    const auto t_begin = Clk::now();
    P = *prm;
    if (P.cell_projection != DPM_CELL_PROJECTION_LS && P.cell_projection != DPM_CELL_PROJECTION_EXACT) return DPM_ERR_ARG;
    cp_on = P.cell_projection == DPM_CELL_PROJECTION_EXACT;
    pc.assign(patches, patches + pmsh->n_patches);
    std::string err;
    SetupDeviceArrays da;
    if (P.host_setup) {
      if (build_mesh_poly(pm, pbc.data(), m, &err)) {
        std::fprintf(stderr, "dopamine_b200: polyhedral mesh set-up failed: %s\n", err.c_str());
        return DPM_ERR_MESH;
      }
      const auto t_mesh = Clk::now();
      {
          const int rs = build_static_ops(m, pc.data(), P, S);  // rows wider than 16: unsupported
          if (rs) return rs == DPM_ERR_UNSUPPORTED ? rs : DPM_ERR_MESH;
        }
      setup_t.mesh_ms = ms_between(t_begin, t_mesh);
      setup_t.ops_ms = ms_between(t_mesh, Clk::now());
    } else {
      int rc = build_setup_device_poly(pm, pc.data(), P, device, m, S, &err, &setup_t, &da);
      if (rc == SETUP_DEVICE_LIMIT) {  // cells beyond the device builder's limits: the host builder
        std::fprintf(stderr, "dopamine_b200: %s; building the mesh on the host\n", err.c_str());
        P.host_setup = 1;
        const auto t_h = Clk::now();
        if (build_mesh_poly(pm, pbc.data(), m, &err)) {
          std::fprintf(stderr, "dopamine_b200: polyhedral mesh set-up failed: %s\n", err.c_str());
          return DPM_ERR_MESH;
        }
        const auto t_mesh = Clk::now();
        {
          const int rs = build_static_ops(m, pc.data(), P, S);  // rows wider than 16: unsupported
          if (rs) return rs == DPM_ERR_UNSUPPORTED ? rs : DPM_ERR_MESH;
        }
        setup_t = SetupTimes();
        setup_t.mesh_ms = ms_between(t_h, t_mesh);
        setup_t.ops_ms = ms_between(t_mesh, Clk::now());
      } else if (rc) {
        std::fprintf(stderr, "dopamine_b200: polyhedral mesh set-up failed: %s\n", err.c_str());
        return (rc < 0 && rc >= -8) ? DPM_ERR_MESH : rc;  // build_mesh_poly's codes -5..-8
      }
    }
    if (m.n_cells > 2000000000LL || m.n_faces > 2000000000LL) return DPM_ERR_UNSUPPORTED;
    nc = (int)m.n_cells; nf = (int)m.n_faces; nb = (int)m.n_bnd_faces; nfp = (int)S.nfp;
    const auto t_up = Clk::now();
    int rc = upload(P.host_setup ? nullptr : &da);
    setup_upload_ms = ms_between(t_up, Clk::now());
    setup_total_ms = ms_between(t_begin, Clk::now());
    return rc;
  }

  template <class T>
  static std::vector<T> soa3(const std::vector<T>& aos, int64_t n) {
    std::vector<T> s(3 * n);
    for (int64_t i = 0; i < n; ++i)
      for (int k = 0; k < 3; ++k) s[k * n + i] = aos[3 * i + k];
    return s;
  }
  template <class T>
  static std::vector<T> soa9(const std::vector<T>& aos, int64_t n) {
    std::vector<T> s(9 * n);
    for (int64_t i = 0; i < n; ++i)
      for (int k = 0; k < 9; ++k) s[k * n + i] = aos[9 * i + k];
    return s;
  }

  // Static data to HBM: from the host builder's m and S, or (da) adopted from the device builder,
  // whose arrays are already in these layouts.
  int upload(SetupDeviceArrays* da) {
    const int64_t nfi = m.n_int_faces;
    d.nc = nc; d.nf = nf; d.nfi = (int)nfi; d.nb = nb; d.nfp = nfp;
    d.S = S.S; d.SP = S.SP; d.SB = S.SB; d.W = S.W; d.WA = S.WA;
    std::vector<int> bps(nb, -1), bcanon(nb, 0);
    if (da) {
      for (void* q : da->release()) mem.ptrs.push_back(q);
      d.vol = da->vol; d.ivol = da->ivol; d.cen = da->cen; d.Tinv = da->Tinv; d.G = da->G;
      d.cf = da->cf; d.cps = da->cps; d.cbn = da->cbn; d.ls_idx = da->ls_idx; d.ls_w = da->ls_w;
      d.fo = da->fo; d.fn = da->fn; d.sf = da->sf; d.nrm = da->nrm; d.fcen = da->fcen; d.eps = da->eps;
      d.area = da->area; d.gc = da->gc; d.wbl = da->wbl; d.dcf = da->dcf;
      d.pso = da->pso; d.psn = da->psn; d.psf = da->psf; d.psc = da->psc; d.psgcf = da->psgcf;
      d.psgcw = da->psgcw; d.psk = da->psk; d.pskrc = da->pskrc;
      d.Acol = da->Acol; d.Aval = da->Aval; d.Adinv = da->Adinv;
      bps = da->bps;
      bcanon = da->bcanon;
    } else {
      std::vector<double> ivol(nc);
      for (int c = 0; c < nc; ++c) ivol[c] = 1.0 / std::max(m.volume[c], SMALL);
      d.vol = mem.upload(m.volume);
      d.ivol = mem.upload(ivol);
      d.cen = mem.upload(soa3(m.centroid, nc));
      d.Tinv = mem.upload(soa9(S.Tinv, nc));
      d.G = mem.upload(soa9(S.G, nc));
      d.cf = mem.upload(S.cell_face);
      d.cps = mem.upload(S.cell_ps);
      d.cbn = mem.upload(S.cell_bnd);
      d.ls_idx = mem.upload(S.ls_idx);
      d.ls_w = mem.upload(S.ls_w);
      d.fo = mem.upload(m.owner);
      d.fn = mem.upload(m.neighbour);
      d.sf = mem.upload(soa3(m.sf, nf));
      d.nrm = mem.upload(soa3(m.normal, nf));
      d.fcen = mem.upload(soa3(m.centre, nf));
      d.eps = mem.upload(soa3(m.eps, nf));
      d.area = mem.upload(m.area);
      d.gc = mem.upload(m.gc);
      d.wbl = mem.upload(S.wblend);
      d.dcf = mem.upload(m.d_cf);
      d.pso = mem.upload(S.ps_o);
      d.psn = mem.upload(S.ps_n);
      d.psf = mem.upload(S.ps_f);
      d.psc = mem.upload(S.ps_coeff);
      d.psgcf = mem.upload(S.ps_gcf);
      d.psgcw = mem.upload(S.ps_gcw);
      d.psk = mem.upload(S.ps_k);
      d.pskrc = mem.upload(S.ps_krc);
      d.Acol = mem.upload(S.A_col);
      d.Aval = mem.upload(S.A_val);
      std::vector<double> dinv(nc);
      for (int c = 0; c < nc; ++c) dinv[c] = 1.0 / S.diag[c];
      d.Adinv = mem.upload(dinv);
      for (int i = (int)nfi; i < nfp; ++i) {
        int b = S.ps_f[i] - (int)nfi;
        bps[b] = i;
        bcanon[b] = 1;
        int pb = m.periodic_pair[b];
        if (pb >= 0) bps[pb] = i;
      }
    }
    std::vector<double> bU(3 * nb, 0.0), bp(nb, 0.0);
    const double wr = P.abl_wind_dir_deg * SEM_PI / 180.0;
    for (int b = 0; b < nb; ++b) {
      int p = m.patch[nfi + b];
      if (p < 0) continue;
      for (int k = 0; k < 3; ++k) bU[k * nb + b] = pc[p].U_val[k];
      bp[b] = pc[p].p_val;
      if (pc[p].bc_id == BC_ABL_INLET) {  // neutral log law along the wind (mod_bc.f90:352-372)
        const double z0 = pc[p].abl_z0_m > 0.0 ? pc[p].abl_z0_m : P.abl_z0_m;
        const double um = sem_log_u(m.centre[3 * (nfi + b) + 2], sem_ustar(P.abl_u_ref, P.abl_z_ref, z0), z0);
        bU[b] = -um * std::sin(wr);
        bU[nb + b] = -um * std::cos(wr);
        bU[2 * nb + b] = 0.0;
      }
    }
    d.bbc = mem.upload(S.bnd_bc);
    d.bpnb = mem.upload(S.bnd_pnb);
    d.bpair = mem.upload(m.periodic_pair);
    d.bps = mem.upload(bps);
    d.bcanon = mem.upload(bcanon);
    d.bpgc = mem.upload(m.periodic_gc);
    d.bpdcf = mem.upload(m.periodic_pair_dcf);
    d.bcb = mem.upload(S.bnd_cb);
    d.bkout = mem.upload(S.bnd_kout);
    d.yw = mem.upload(S.y_w);
    d.bUval = mem.upload(bU);
    d.bpval = mem.upload(bp);
    {  // TVD upwind context per face and flux sign, when a van Leer / Koren scheme is configured
      auto is_tvd = [](int sch) { return sch == DPM_SCHEME_VANLEER_TVD || sch == DPM_SCHEME_KOREN_TVD; };
      if (is_tvd(P.scheme) || (P.boussinesq && is_tvd(P.temperature_scheme)) ||
          (P.n_scalars > 0 && is_tvd(P.scalar_scheme))) {
        int* far2 = mem.alloc<int>(2 * (size_t)nf);
        double *sf2 = mem.alloc<double>(2 * (size_t)nf), *sd2 = mem.alloc<double>(2 * (size_t)nf),
               *su2 = mem.alloc<double>(2 * (size_t)nf);
        if (!far2 || !sf2 || !sd2 || !su2) return DPM_ERR_CUDA;
        k_tvd_context<<<nblk(nf), TPB, 0, st>>>(d, far2, sf2, sd2, su2);
        launches++;
        d.tvd_far = far2; d.tvd_sf = sf2; d.tvd_sd = sd2; d.tvd_su = su2;
      }
    }
    // fields
    F.U = mem.alloc<double>(3 * nc);
    F.p = mem.alloc<double>(nc); F.p_old = mem.alloc<double>(nc); F.phi_prev = mem.alloc<double>(nc);
    F.nu_sgs = mem.alloc<double>(nc); F.rhs = mem.alloc<double>(nc); F.T = mem.alloc<double>(nc);
    F.Ub = mem.alloc<double>(3 * nb); F.pb = mem.alloc<double>(nb); F.phi_prev_b = mem.alloc<double>(nb);
    F.tau = mem.alloc<double>(3 * nb); F.upf = mem.alloc<double>(3 * nb);
    F.gU = mem.alloc<double>(9 * nc); F.gp = mem.alloc<double>(3 * nc); F.gp_rc = mem.alloc<double>(3 * nc);
    F.gpc = mem.alloc<double>(3 * nc); F.H = mem.alloc<double>(3 * nc); F.H0 = mem.alloc<double>(3 * nc);
    F.ff = mem.alloc<double>(nf); F.Uf = mem.alloc<double>(nf);
    F.fadv = mem.alloc<double>(3 * nf); F.fvis = mem.alloc<double>(3 * nf); F.fdiv = mem.alloc<double>(nf);
    F.ps_cross = mem.alloc<double>(nfp);
    F.ptot = mem.alloc<double>(nc); F.ptot_b = mem.alloc<double>(nb); F.phi_it = mem.alloc<double>(nc);
    red_part = mem.alloc<double>(RED_NV * 2048);
    red_out = mem.alloc<double>(RED_NV);
    scratch_c = mem.alloc<double>(nc); scratch_c2 = mem.alloc<double>(nc);
    aos_buf = mem.alloc<double>(9 * (size_t)std::max(nc, nf));
    conv_tmp = mem.alloc<double>(3 * nc); visc_tmp = mem.alloc<double>(3 * nc);
    U_spare = mem.alloc<double>(3 * (size_t)nc);
    if (!U_spare) return DPM_ERR_CUDA;
    cg_r = mem.alloc<double>(nc); cg_z = mem.alloc<double>(nc); cg_p0 = mem.alloc<double>(nc);
    cg_p1 = mem.alloc<double>(nc); cg_q = mem.alloc<double>(nc); cg_bp = mem.alloc<double>(nc);
    cg_x = mem.alloc<double>(nc);
    cg_bar = mem.alloc<unsigned>(2); cg_status = mem.alloc<int>(4); cg_dout = mem.alloc<double>(4);
    if (P.gradient_scheme != DPM_GRAD_LEAST_SQUARES && P.gradient_scheme != DPM_GRAD_GREEN_GAUSS) return DPM_ERR_ARG;
    if (gg()) {
      gg_prevU = mem.alloc<double>((size_t)9 * nc);
      gg_prevS = mem.alloc<double>((size_t)3 * LS_SET * nc);
      if (!gg_prevU || !gg_prevS) return DPM_ERR_CUDA;
    }
    if (!cg_dout || !F.fadv || !aos_buf) return DPM_ERR_CUDA;
    if (cp_on && cp_alloc()) return DPM_ERR_CUDA;
    {
      int rc = setup_sem();
      if (rc) return rc;
    }
    // cooperative grid for the persistent PCG
    int dev_sms = 0, per_sm = 0, coop = 0;
    CK(cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, device));
    CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg<double, 0, 0>, PCG_TPB, 0));
    cg_coop = coop != 0 && per_sm > 0;
    if (!cg_coop) return DPM_ERR_UNSUPPORTED;
    cg_grid = std::min(dev_sms * per_sm, std::max(1, (nc + PCG_TPB - 1) / PCG_TPB));
    cg_kernel = pcg_kernel_for<double>(nc, cg_grid, S.WA, &cg_cpt);
    // A and 1/diag should stay in L1 across iterations: prefer the largest L1 carveout (set before
    // the occupancy query, which the cooperative launch check must agree with).
    CK(cudaFuncSetAttribute(cg_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 5));
    {
      int per_sm2 = 0;
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm2, cg_kernel, PCG_TPB, 0));
      if (per_sm2 < 1) return DPM_ERR_UNSUPPORTED;
      if (dev_sms * per_sm2 < cg_grid) {  // fewer co-resident blocks: re-pick with the smaller grid
        cg_grid = dev_sms * per_sm2;
        cg_kernel = pcg_kernel_for<double>(nc, cg_grid, S.WA, &cg_cpt);
        CK(cudaFuncSetAttribute(cg_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 5));
      }
    }
    cg_part = mem.alloc<double>(8 * (size_t)cg_grid);
    {
      int rc = setup_scalars();
      if (rc) return rc;
      rc = setup_x32();
      if (rc) return rc;
      if (x32 && P.use_nudging) return DPM_ERR_UNSUPPORTED;  // the FP32 explicit half fuses the predictor
    }
    const auto t_ps = std::chrono::steady_clock::now();
    if (P.p_solver == DPM_PSOLVER_TWOLEVEL_FCG) {
      int rc = setup_fcg(dev_sms);
      if (rc) return rc;
    } else if (P.p_solver == DPM_PSOLVER_MULTILEVEL_FCG) {
      int rc = setup_ml(dev_sms);
      if (rc) return rc;
    } else if (P.p_solver == DPM_PSOLVER_AUTO) {
      // the two-level kernel keeps a part of <= 4096 cells per block, one block per SM
      int rc = (nc + dev_sms - 1) / dev_sms <= 4096 ? setup_fcg(dev_sms) : DPM_ERR_UNSUPPORTED;
      if (rc == DPM_ERR_UNSUPPORTED) rc = setup_ml(dev_sms);
      if (rc) return rc;
    } else if (P.p_solver != DPM_PSOLVER_JACOBI_PCG) {
      return DPM_ERR_ARG;
    } else if (P.form == DPM_FORM_MIXED) {
      return DPM_ERR_UNSUPPORTED;  // the precision form is built on the flexible CG
    }
    setup_psolver_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_ps).count();
    // initial fields: T = T_ref, velocity from an inlet patch (initialize_velocity_from_bc)
    launch_fill(F.T, nc, P.T_ref);
    double u0[3] = {0, 0, 0};
    for (auto& q : pc)
      if (q.bc_id == BC_INLET) { for (int k = 0; k < 3; ++k) u0[k] = q.U_val[k]; break; }
    for (int k = 0; k < 3; ++k) launch_fill(F.U + (size_t)k * nc, nc, u0[k]);
    CK(cudaGetLastError());
    return 0;
  }

  void launch_fill(double* p, int64_t n, double v) {
    k_fill<<<nblk(n), TPB, 0, st>>>((int)n, p, v);
    launches++;
  }

  // ---------------------------------------------------------------- building blocks
  void velocity_bc(int filt, int have_grad) {
    if (nb == 0) return;
    k_velocity_bc<<<nblk(nb), TPB, 0, st>>>(d, F.U, F.gU, F.Ub, filt, have_grad);
    launches++;
  }
  void pressure_bc(const double* pf, int filt, int have_grad, int incr) {
    if (nb == 0) return;
    k_pressure_bc<<<nblk(nb), TPB, 0, st>>>(d, pf, F.gp, F.pb, filt, have_grad, incr);
    launches++;
  }
  void refresh_halos_and_bc() {
    velocity_bc(0, 1);
    pressure_bc(F.p, 0, !S.skip_grad_p, 0);
    scalar_bcs(0);
    velocity_bc(1, 1);
    pressure_bc(F.p, 1, 0, 0);
    scalar_bcs(1);
  }
  void velocity_bc_refresh() {
    velocity_bc(0, 1);
    velocity_bc(1, 1);
  }
  // Gradients: least squares, or Green-Gauss with gg_sweeps() sweeps (src/solver/
  // mod_fv_solver.f90:1003-1077, :2341-2369); the sweeps after the first read the previous
  // sweep's gradient, copied aside.
  bool gg() const { return P.gradient_scheme == DPM_GRAD_GREEN_GAUSS; }
  int gg_sweeps() const { return P.gg_iterations > 0 ? P.gg_iterations : 2; }
  void grad_U() {
    if (!gg()) {
      k_ls_gradient_vector<<<nblk(nc), TPB, 0, st>>>(d, F.U, F.Ub, F.gU);
      launches++;
      return;
    }
    k_gg_gradient_vector<<<nblk(nc), TPB, 0, st>>>(d, F.U, F.Ub, nullptr, F.gU);
    launches++;
    for (int it = 2; it <= gg_sweeps(); ++it) {
      copy(gg_prevU, F.gU, (size_t)9 * nc);
      k_gg_gradient_vector<<<nblk(nc), TPB, 0, st>>>(d, F.U, F.Ub, gg_prevU, F.gU);
      launches++;
    }
  }
  // Green-Gauss sweeps of a set of scalar fields (slot k of the previous-gradient scratch per field)
  void gg_scalars(GgScalarSet q) {
    for (int k = 0; k < LS_SET; ++k) q.gprev[k] = nullptr;
    k_gg_gradient_scalars<<<nblk(nc), TPB, 0, st>>>(d, q);
    launches++;
    for (int it = 2; it <= gg_sweeps(); ++it) {
      for (int k = 0; k < q.n; ++k) {
        double* prev = gg_prevS + (size_t)k * 3 * nc;
        copy(prev, q.g[k], (size_t)3 * nc);
        q.gprev[k] = prev;
      }
      k_gg_gradient_scalars<<<nblk(nc), TPB, 0, st>>>(d, q);
      launches++;
    }
  }
  void grad_scalar(const double* phi, const double* pb, double* g) {
    if (gg()) {
      GgScalarSet q{};
      q.n = 1; q.phi[0] = phi; q.pb[0] = pb; q.g[0] = g;
      gg_scalars(q);
      return;
    }
    k_ls_gradient_scalar<<<nblk(nc), TPB, 0, st>>>(d, phi, pb, g);
    launches++;
  }
  void pressure_gradient() {
    if (!S.skip_grad_p) grad_scalar(F.p, F.pb, F.gp);
  }
  void copy(double* dst, const double* src, size_t n) { cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToDevice, st); }

  int reduce(RedArgs r, double* host_out, int nv) {
    int g = std::min(nblk(r.n), 2048);
    if (g < 1) g = 1;
    k_reduce_partial<<<g, TPB, 0, st>>>(r, red_part);
    k_reduce_final<<<1, 32 * RED_NV, 0, st>>>(r.mode, g, red_part, red_out);
    launches += 2;
    if (host_out) {
      CK(cudaMemcpyAsync(host_out, red_out, nv * sizeof(double), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
    }
    return 0;
  }

  void anchor_pressure() {
    if (S.n_outlet > 0) return;
    RedArgs r{};
    r.mode = RED_SUM2; r.n = nc; r.a = F.p; r.b = d.vol;
    reduce(r, nullptr, 0);
    k_anchor_shift<<<1, 1, 0, st>>>(red_out, S.V_total, red_out + 8);
    k_shift<<<nblk(nc), TPB, 0, st>>>(nc, F.p, red_out + 8);
    launches += 2;
  }

  int atol_dynamic(double dt, double& atol) {
    RedArgs r{};
    r.mode = RED_UBULK; r.n = nc; r.a = F.U; r.vol = d.vol;
    double o[2];
    int rc = reduce(r, o, 2);
    if (rc) return rc;
    double us = o[0] / std::max(o[1], SMALL);
    atol = std::max(1.0e-12 * std::max(us, 1.0) * S.V_min / dt, 1.0e-15);
    return 0;
  }

  void sgs(double dt_stab) {
    if (P.sgs_model == DPM_SGS_NONE) {
      launch_fill(F.nu_sgs, nc, 0.0);
      return;
    }
    k_sgs<<<nblk(nc), TPB, 0, st>>>(d, P.sgs_model, F.gU, F.nu_sgs, dt_stab, P.c_amd);
    launches++;
    if (P.sgs_model == DPM_SGS_AMD && P.amd_wall_gradient && nb > 0) {
      k_amd_wall<<<nblk(nc), TPB, 0, st>>>(d, F.U, F.gU, F.nu_sgs, P.nu, P.c_amd, dt_stab);
      launches++;
    }
  }

  void wall_model(double dt_filter) {
    if (nb == 0) return;
    if (P.wall_model == DPM_WM_NONE) {
      launch_fill(F.tau, 3 * (int64_t)nb, 0.0);
      return;
    }
    if (P.wall_model == DPM_WM_MOST) {
      // The reference also refreshes a domain-mean Obukhov length at stage 1; it only seeds faces
      // whose own length is still zero, i.e. the first call, so the configured value is used.
      k_most<<<nblk(nb), TPB, 0, st>>>(d, F.U, F.T, F.tau, most_qw, most_L, P.abl_L_obukhov, P.abl_T_surface,
                                       most_z0m, most_z0h);
      launches++;
      return;
    }
    double t_use = P.wall_model_filter_time, tf = P.wall_model_filter_tf_fac;
    bool adaptive = tf > SMALL;
    int filter = adaptive ? 2 : (t_use > SMALL ? 1 : 0);
    double w_filt = (filter == 1) ? dt_filter / (t_use + dt_filter) : 0.0;
    k_wall_model<<<nblk(nb), TPB, 0, st>>>(d, F.U, F.tau, F.upf, P.nu, filter, filt_ready ? 0 : 1, w_filt, dt_filter, tf);
    launches++;
    if (filter) filt_ready = true;
  }

  // body_force_now (src/solver/mod_fv_solver.f90:2903-2922): constant or mass-flux forcing plus the
  // harmonic forcing at time t
  void body_force(double t, double f[3]) const {
    for (int k = 0; k < 3; ++k) f[k] = P.constant_mass_flux_forcing ? mass_flux_force[k] : P.f_const[k];
    if (P.use_harmonic_forcing) {
      const double* fd = P.forcing_dir;
      const double dn = std::sqrt(fd[0] * fd[0] + fd[1] * fd[1] + fd[2] * fd[2]);
      double hd[3] = {1.0, 0.0, 0.0};
      if (dn > SMALL)
        for (int k = 0; k < 3; ++k) hd[k] = fd[k] / dn;
      const double hs = P.forcing_amp * std::cos(P.forcing_omega * t + P.forcing_phase);
      for (int k = 0; k < 3; ++k) f[k] = f[k] + hs * hd[k];
    }
  }
  void set_forces(ExplicitArgs& a) const {
    double f[3];
    body_force(time, f);
    a.f0 = f[0]; a.f1 = f[1]; a.f2 = f[2];
    a.rot = P.use_rotation ? 1 : 0;
    a.om0 = P.omega_rot[0]; a.om1 = P.omega_rot[1]; a.om2 = P.omega_rot[2];
  }
  // update_mass_flux_forcing (mod_fv_solver.f90:959-983): (U_bulk_target - <U>) / dt
  int update_mass_flux_forcing(double dt) {
    RedArgs r{};
    r.mode = RED_STATS; r.n = nc; r.a = F.U; r.vol = d.vol; r.gU = F.gU; r.nus = F.nu_sgs; r.nu = P.nu;
    double o[RED_NV];
    int rc = reduce(r, o, RED_NV);
    if (rc) return rc;
    for (int k = 0; k < 3; ++k) mass_flux_force[k] = (P.U_bulk_target[k] - o[3 + k] / std::max(S.V_total, SMALL)) / dt;
    return 0;
  }

  void explicit_rhs(double dt, double a_k, double b_k, int predict) {
    ExplicitArgs a{};
    a.scheme = P.scheme;
    set_forces(a);
    a.bous = P.boussinesq; a.beta = P.beta; a.T_ref = P.T_ref; a.g0 = P.g[0]; a.g1 = P.g[1]; a.g2 = P.g[2];
    a.dt = dt; a.a_k = a_k; a.b_k = b_k; a.predict = predict;
    if (predict) {  // cell-owned fused pass, predicted velocity into the spare buffer
      k_cell_momentum<<<nblk(nc), TPB, 0, st>>>(d, a, P.nu, F.U, F.Ub, F.gU, F.nu_sgs, F.Uf, F.T, F.tau, F.H, F.H0,
                                                U_spare);
      launches++;
      std::swap(F.U, U_spare);
      return;
    }
    k_face_explicit<<<nblk(nf), TPB, 0, st>>>(d, P.scheme, P.nu, F.U, F.Ub, F.gU, F.nu_sgs, F.Uf, F.fadv, F.fvis, F.fdiv);
    k_cell_explicit<<<nblk(nc), TPB, 0, st>>>(d, a, F.U, F.T, F.fadv, F.fvis, F.fdiv, F.tau, F.H, F.H0, conv_tmp,
                                                visc_tmp);
    launches += 2;
  }

  void correct_velocity(double dt, bool with_cross, bool ptot) {
    CorrArgs a{};
    a.dt = dt;
    a.do_cross = with_cross && !S.skip_nonortho;
    a.ptot = ptot;
    double fb[3];
    body_force(time, fb);
    a.f0 = fb[0]; a.f1 = fb[1]; a.f2 = fb[2];
    a.bb = P.boussinesq ? P.beta : 0.0; a.T_ref = P.T_ref; a.g0 = P.g[0]; a.g1 = P.g[1]; a.g2 = P.g[2];
    k_correct_velocity<<<nblk(nc), TPB, 0, st>>>(d, a, F.p, F.gp, F.T, F.U, F.gpc);
    launches++;
  }

  void face_fluxes_and_rhs(double dt, bool incr) {
    if (!S.skip_grad_p) {
      if (incr) {
        copy(F.ptot, F.phi_prev, nc);
        copy(F.ptot_b, F.phi_prev_b, nb);
        k_add<<<nblk(nc), TPB, 0, st>>>(nc, F.ptot, F.p);
        if (nb) k_add<<<nblk(nb), TPB, 0, st>>>(nb, F.ptot_b, F.pb);
        launches += 2;
        grad_scalar(F.ptot, F.ptot_b, F.gp);
      } else {
        grad_scalar(F.p, F.pb, F.gp);
      }
    }
    int wc = !S.skip_nonortho;
    k_face_flux<<<nblk(nf), TPB, 0, st>>>(d, dt, F.U, F.gU, F.gp_rc, F.phi_prev, F.Ub, F.gp, wc, cp_on ? 1 : 0, F.ff,
                                          F.ps_cross);
    k_rhs_gather<<<nblk(nc), TPB, 0, st>>>(d, 1.0 / std::max(dt, SMALL), wc, F.ff, F.ps_cross, F.gp, F.rhs);
    launches += 2;
  }

  void correct_face_fluxes(double dt, bool ptot) {
    k_correct_face_flux<<<nblk(nf), TPB, 0, st>>>(d, dt, ptot, !S.skip_nonortho, F.p, F.gp, F.ff, F.Uf);
    launches++;
  }

  // Temperature and passive scalars: fields, per-face boundary data (fixed temperature, scalar
  // mode and value per boundary face) and flux scratch.
  int setup_scalars() {
    auto ok_scheme = [](int sch) {
      return sch == DPM_SCHEME_CDS || sch == DPM_SCHEME_QUICK || sch == DPM_SCHEME_VANLEER_TVD ||
             sch == DPM_SCHEME_KOREN_TVD;
    };
    ns = std::max(0, std::min(P.n_scalars, 4));
    if ((P.boussinesq && !ok_scheme(P.temperature_scheme)) || (ns > 0 && !ok_scheme(P.scalar_scheme)))
      return DPM_ERR_UNSUPPORTED;
    Tb = mem.alloc<double>(std::max(nb, 1)); gT = mem.alloc<double>(3 * (size_t)nc);
    HT = mem.alloc<double>(nc); HT0 = mem.alloc<double>(nc);
    // face fluxes per transported field (temperature, then the passive scalars)
    sc_fadv = mem.alloc<double>((size_t)(ns + 1) * nf); sc_fdif = mem.alloc<double>((size_t)(ns + 1) * nf);
    std::vector<double> tv(std::max(nb, 1), P.T_ref), sv((size_t)std::max(ns, 1) * std::max(nb, 1), 0.0);
    std::vector<int> sm((size_t)std::max(ns, 1) * std::max(nb, 1), 0);
    for (int b = 0; b < nb; ++b) {
      const int q = m.patch[nfi_() + b];
      if (q < 0) continue;
      tv[b] = pc[q].T_val;
      if (pc[q].bc_id == BC_ABL_INLET) {  // MOST neutral temperature profile (mod_bc.f90:557-562)
        const double z0h = pc[q].abl_z0_h > 0.0 ? pc[q].abl_z0_h : P.abl_z0_h, z = m.centre[3 * (nfi_() + b) + 2];
        const double ts = (P.abl_z_ref > z0h && z0h > SMALL)
                              ? 0.41 * (P.abl_T_ref - P.abl_T_surface) / std::log(P.abl_z_ref / z0h) : 0.0;
        tv[b] = (z <= z0h || std::fabs(ts) <= SMALL || z0h <= SMALL) ? P.abl_T_surface
                                                                    : P.abl_T_surface + (ts / 0.41) * std::log(z / z0h);
      }
      for (int k = 0; k < ns; ++k) {
        sm[(size_t)k * nb + b] = pc[q].scalar_mode[k];
        sv[(size_t)k * nb + b] = pc[q].scalar_value[k];
      }
    }
    bTval = mem.upload(tv);
    bsmode = mem.upload(sm);
    bsval = mem.upload(sv);
    if (!Tb || !gT || !HT || !HT0 || !sc_fadv || !sc_fdif || !bTval || !bsmode || !bsval) return DPM_ERR_CUDA;
    launch_fill(Tb, std::max(nb, 1), P.T_ref);
    most_L = mem.alloc<double>(std::max(nb, 1));
    most_qw = mem.alloc<double>(std::max(nb, 1));
    {  // per-face roughness: the patch's value when positive, else the global one
      std::vector<double> z0m(std::max(nb, 1), std::max(P.abl_z0_m, SMALL)), z0h(std::max(nb, 1), std::max(P.abl_z0_h, SMALL));
      for (int b = 0; b < nb; ++b) {
        const int q = m.patch[nfi_() + b];
        if (q < 0) continue;
        if (pc[q].abl_z0_m > 0.0) z0m[b] = std::max(pc[q].abl_z0_m, SMALL);
        if (pc[q].abl_z0_h > 0.0) z0h[b] = std::max(pc[q].abl_z0_h, SMALL);
      }
      most_z0m = mem.upload(z0m);
      most_z0h = mem.upload(z0h);
    }
    if (!most_L || !most_qw || !most_z0m || !most_z0h) return DPM_ERR_CUDA;
    launch_fill(most_L, std::max(nb, 1), 0.0);
    launch_fill(most_qw, std::max(nb, 1), 0.0);
    launch_fill(gT, 3 * (int64_t)nc, 0.0);
    if (ns > 0) {
      Cs = mem.alloc<double>((size_t)ns * nc); Cb = mem.alloc<double>((size_t)ns * std::max(nb, 1));
      gC = mem.alloc<double>((size_t)ns * 3 * nc);
      HC = mem.alloc<double>((size_t)ns * nc); HC0 = mem.alloc<double>((size_t)ns * nc);
      if (!Cs || !Cb || !gC || !HC || !HC0) return DPM_ERR_CUDA;
      launch_fill(Cs, (int64_t)ns * nc, 0.0);
      launch_fill(Cb, (int64_t)ns * std::max(nb, 1), 0.0);
      launch_fill(gC, (int64_t)ns * 3 * nc, 0.0);
    }
    return 0;
  }
  int nfi_() const { return (int)m.n_int_faces; }

  // The precision form's FP32 explicit half: FP32 copies of the static geometry and LS weights
  // (made on the device from the FP64 arrays), FP32 first-pass gradients and scalar face fluxes.
  // Schemes it provides: KEP, CDS, van Leer, Koren; least-squares gradients.
  int setup_x32() {
    if (P.form != DPM_FORM_MIXED) return 0;
    auto ok_mom = [](int s) {
      return s == DPM_SCHEME_KEP || s == DPM_SCHEME_CDS || s == DPM_SCHEME_VANLEER_TVD || s == DPM_SCHEME_KOREN_TVD;
    };
    auto ok_sc = [](int s) { return s == DPM_SCHEME_CDS || s == DPM_SCHEME_VANLEER_TVD || s == DPM_SCHEME_KOREN_TVD; };
    if (!ok_mom(P.scheme) || (P.boussinesq && !ok_sc(P.temperature_scheme)) || (ns > 0 && !ok_sc(P.scalar_scheme)) ||
        gg())
      return DPM_ERR_UNSUPPORTED;
    auto f32 = [&](const double* src, size_t n) -> const float* {
      float* dst = mem.alloc<float>(n);
      if (!dst || !src) return dst;
      k_to_f32<<<(unsigned)((n + TPB - 1) / TPB), TPB, 0, st>>>((int64_t)n, src, dst);
      launches++;
      return dst;
    };
    g32.vol = f32(d.vol, nc); g32.ivol = f32(d.ivol, nc); g32.cen = f32(d.cen, 3 * (size_t)nc);
    g32.G = f32(d.G, 9 * (size_t)nc); g32.ls_w = f32(d.ls_w, 3 * (size_t)d.W * nc);
    g32.sf = f32(d.sf, 3 * (size_t)nf); g32.nrm = f32(d.nrm, 3 * (size_t)nf); g32.fcen = f32(d.fcen, 3 * (size_t)nf);
    g32.eps = f32(d.eps, 3 * (size_t)nf); g32.area = f32(d.area, nf); g32.gc = f32(d.gc, nf);
    g32.wbl = f32(d.wbl, nf); g32.dcf = f32(d.dcf, nf);
    g32.bpgc = f32(d.bpgc, std::max(nb, 1)); g32.bpdcf = f32(d.bpdcf, std::max(nb, 1));
    if (d.tvd_far) {
      g32.tvd_sf = f32(d.tvd_sf, 2 * (size_t)nf); g32.tvd_sd = f32(d.tvd_sd, 2 * (size_t)nf);
      g32.tvd_su = f32(d.tvd_su, 2 * (size_t)nf);
    }
    gU32 = mem.alloc<float>(9 * (size_t)nc);
    gS32 = mem.alloc<float>(3 * (size_t)(ns + 1) * nc);
    sc_fadv32 = mem.alloc<float>((size_t)(ns + 1) * nf);
    sc_fdif32 = mem.alloc<float>((size_t)(ns + 1) * nf);
    if (!g32.vol || !g32.ls_w || !g32.sf || !g32.eps || !g32.dcf || !gU32 || !gS32 || !sc_fadv32 || !sc_fdif32)
      return DPM_ERR_CUDA;
    x32 = true;
    return 0;
  }
  // first gradient pass of a stage in FP32 (U, T when transported, the scalars: one pass over the
  // FP32 weights), and the FP64 gradient at the cells whose boundary values extrapolate with it
  void grad_all32() {
    LsScalarSet32 q{};
    if (P.boussinesq) { q.phi[q.n] = F.T; q.pb[q.n] = Tb; q.g[q.n] = gS32; q.n++; }
    for (int k = 0; k < ns; ++k) {
      q.phi[q.n] = Cs + (size_t)k * nc; q.pb[q.n] = Cb + (size_t)k * nb; q.g[q.n] = gS32 + (size_t)q.n * 3 * nc; q.n++;
    }
    switch (q.n) {
      case 0: k_ls32_gradient_all<0><<<nblk(nc), TPB, 0, st>>>(d, g32, F.U, F.Ub, gU32, q); break;
      case 1: k_ls32_gradient_all<1><<<nblk(nc), TPB, 0, st>>>(d, g32, F.U, F.Ub, gU32, q); break;
      case 2: k_ls32_gradient_all<2><<<nblk(nc), TPB, 0, st>>>(d, g32, F.U, F.Ub, gU32, q); break;
      case 3: k_ls32_gradient_all<3><<<nblk(nc), TPB, 0, st>>>(d, g32, F.U, F.Ub, gU32, q); break;
      case 4: k_ls32_gradient_all<4><<<nblk(nc), TPB, 0, st>>>(d, g32, F.U, F.Ub, gU32, q); break;
      default: k_ls32_gradient_all<5><<<nblk(nc), TPB, 0, st>>>(d, g32, F.U, F.Ub, gU32, q); break;
    }
    launches++;
    if (nb) {
      k_grad32_to_bnd<<<nblk(nb), TPB, 0, st>>>(d, gU32, F.gU);
      launches++;
    }
  }
  void sgs32(double dt_stab) {
    if (P.sgs_model == DPM_SGS_NONE) {
      launch_fill(F.nu_sgs, nc, 0.0);
      return;
    }
    k_sgs32<<<nblk(nc), TPB, 0, st>>>(d, g32, P.sgs_model, gU32, F.nu_sgs, (float)dt_stab, (float)P.c_amd);
    launches++;
    if (P.sgs_model == DPM_SGS_AMD && P.amd_wall_gradient && nb > 0) {
      k_amd_wall32<<<nblk(nc), TPB, 0, st>>>(d, g32, F.U, gU32, F.nu_sgs, P.nu, (float)P.c_amd, (float)dt_stab);
      launches++;
    }
  }
  void explicit_rhs32(double dt, double a_k, double b_k) {
    ExplicitArgs a{};
    a.scheme = P.scheme;
    set_forces(a);
    a.bous = P.boussinesq; a.beta = P.beta; a.T_ref = P.T_ref; a.g0 = P.g[0]; a.g1 = P.g[1]; a.g2 = P.g[2];
    a.dt = dt; a.a_k = a_k; a.b_k = b_k; a.predict = 1;
    k_cell_momentum32<<<nblk(nc), TPB, 0, st>>>(d, g32, a, (float)P.nu, F.U, F.Ub, gU32, F.nu_sgs, F.Uf, F.T, F.tau,
                                                F.H, F.H0, U_spare);
    launches++;
    std::swap(F.U, U_spare);
  }
  void scalars_rhs32(double dt, double a_k, double b_k) {
    ScalarFaceSet32 q{};
    double* H[LS_SET];
    const double* H0[LS_SET];
    double* phi[LS_SET];
    const double* qw[LS_SET];
    auto add = [&](int scheme, double* f, const double* pbv, double alpha, double prt, double* h, const double* h0,
                   const double* w) {
      const int k = q.n++;
      q.scheme[k] = scheme; q.phi[k] = f; q.pb[k] = pbv; q.g[k] = gS32 + (size_t)k * 3 * nc;
      q.alpha[k] = (float)alpha; q.prt[k] = (float)prt;
      q.fadv[k] = sc_fadv32 + (size_t)k * nf; q.fdif[k] = sc_fdif32 + (size_t)k * nf;
      H[k] = h; H0[k] = h0; phi[k] = f; qw[k] = w;
    };
    if (P.boussinesq)
      add(P.temperature_scheme, F.T, Tb, P.alpha_T, P.Pr_t, HT, HT0, P.wall_model == DPM_WM_MOST ? most_qw : nullptr);
    for (int k = 0; k < ns; ++k)
      add(P.scalar_scheme, Cs + (size_t)k * nc, Cb + (size_t)k * nb, P.scalar_diffusivity[k], P.scalar_pr_t[k],
          HC + (size_t)k * nc, HC0 + (size_t)k * nc, nullptr);
    if (q.n == 0) return;
    k_face_scalars32<<<nblk(nf), TPB, 0, st>>>(d, g32, q, F.nu_sgs, F.Uf);
    launches++;
    for (int k = 0; k < q.n; ++k) {
      k_cell_scalar32<<<nblk(nc), TPB, 0, st>>>(d, g32, q.fadv[k], q.fdif[k], H[k], H0[k], phi[k], dt, a_k, b_k, qw[k]);
      launches++;
    }
  }

  void temperature_bc(int filt) {
    if (nb == 0) return;
    k_scalar_bc<<<nblk(nb), TPB, 0, st>>>(d, 0, F.T, gT, Tb, filt, bTval, nullptr, nullptr, 0.0, 1.0, F.nu_sgs);
    launches++;
  }
  void scalar_bc(int k, int filt) {
    if (nb == 0) return;
    k_scalar_bc<<<nblk(nb), TPB, 0, st>>>(d, 1, Cs + (size_t)k * nc, nullptr, Cb + (size_t)k * nb, filt, nullptr,
                                          bsmode + (size_t)k * nb, bsval + (size_t)k * nb, P.scalar_diffusivity[k],
                                          P.Pr_t, F.nu_sgs);
    launches++;
  }
  void scalar_bcs(int filt) {
    if (P.boussinesq) temperature_bc(filt);  // T_bnd is only read when T is transported
    for (int k = 0; k < ns; ++k) scalar_bc(k, filt);
  }
  // cell gradients of U, of T when it is transported, and of every passive scalar
  void grad_all() {
    LsScalarSet q{};  // temperature and passive scalars: one pass over the LS weights
    if (P.boussinesq) {
      q.phi[q.n] = F.T; q.pb[q.n] = Tb; q.g[q.n] = gT; q.n++;
    }
    for (int k = 0; k < ns; ++k) {
      q.phi[q.n] = Cs + (size_t)k * nc; q.pb[q.n] = Cb + (size_t)k * nb; q.g[q.n] = gC + (size_t)k * 3 * nc; q.n++;
    }
    if (gg() || q.n == 0) {
      grad_U();
      if (q.n > 0) {
        GgScalarSet h{};
        h.n = q.n;
        for (int k = 0; k < q.n; ++k) { h.phi[k] = q.phi[k]; h.pb[k] = q.pb[k]; h.g[k] = q.g[k]; }
        gg_scalars(h);
      }
      return;
    }
    // least squares: U, T and the scalars in one pass over the stencil weights
    switch (q.n) {
      case 1: k_ls_gradient_all<1><<<nblk(nc), TPB, 0, st>>>(d, F.U, F.Ub, F.gU, q); break;
      case 2: k_ls_gradient_all<2><<<nblk(nc), TPB, 0, st>>>(d, F.U, F.Ub, F.gU, q); break;
      case 3: k_ls_gradient_all<3><<<nblk(nc), TPB, 0, st>>>(d, F.U, F.Ub, F.gU, q); break;
      case 4: k_ls_gradient_all<4><<<nblk(nc), TPB, 0, st>>>(d, F.U, F.Ub, F.gU, q); break;
      default: k_ls_gradient_all<5><<<nblk(nc), TPB, 0, st>>>(d, F.U, F.Ub, F.gU, q); break;
    }
    launches++;
  }
  // explicit right-hand side and RK3W update of T and the scalars (after the momentum predictor,
  // which reads the old T for the buoyancy term)
  void scalar_transport(int scheme, double* phi, const double* pbv, const double* g, double alpha, double prt,
                        double* H, const double* H0, double dt, double a_k, double b_k, int predict,
                        double* conv_out, double* dif_out, const double* qw = nullptr) {
    k_face_scalar<<<nblk(nf), TPB, 0, st>>>(d, scheme, phi, pbv, g, F.nu_sgs, alpha, prt, F.Uf, sc_fadv, sc_fdif);
    k_cell_scalar<<<nblk(nc), TPB, 0, st>>>(d, sc_fadv, sc_fdif, H, H0, phi, conv_out, dif_out, dt, a_k, b_k, predict,
                                            qw);
    launches += 2;
  }
  // All transported fields together: one face pass for every field (the fields do not read each
  // other), then each field's gather and RK3W update.
  void scalars_rhs(double dt, double a_k, double b_k, int predict = 1) {
    ScalarFaceSet q{};
    double* H[LS_SET];
    const double* H0[LS_SET];
    double* phi[LS_SET];
    const double* qw[LS_SET];
    auto add = [&](int scheme, double* f, const double* pbv, const double* g, double alpha, double prt, double* h,
                   const double* h0, const double* w) {
      const int k = q.n++;
      q.scheme[k] = scheme; q.phi[k] = f; q.pb[k] = pbv; q.g[k] = g; q.alpha[k] = alpha; q.prt[k] = prt;
      q.fadv[k] = sc_fadv + (size_t)k * nf; q.fdif[k] = sc_fdif + (size_t)k * nf;
      H[k] = h; H0[k] = h0; phi[k] = f; qw[k] = w;
    };
    if (P.boussinesq)
      add(P.temperature_scheme, F.T, Tb, gT, P.alpha_T, P.Pr_t, HT, HT0, P.wall_model == DPM_WM_MOST ? most_qw : nullptr);
    for (int k = 0; k < ns; ++k)
      add(P.scalar_scheme, Cs + (size_t)k * nc, Cb + (size_t)k * nb, gC + (size_t)k * 3 * nc, P.scalar_diffusivity[k],
          P.scalar_pr_t[k], HC + (size_t)k * nc, HC0 + (size_t)k * nc, nullptr);
    if (q.n == 0) return;
    k_face_scalars<<<nblk(nf), TPB, 0, st>>>(d, q, F.nu_sgs, F.Uf);
    launches++;
    for (int k = 0; k < q.n; ++k) {
      k_cell_scalar<<<nblk(nc), TPB, 0, st>>>(d, q.fadv[k], q.fdif[k], H[k], H0[k], phi[k], nullptr, nullptr, dt, a_k,
                                              b_k, predict, qw[k]);
      launches++;
    }
  }

  // Two-level FCG set-up: one part per SM (the kernel needs one co-resident block per part and
  // its part's local operator in shared memory).
  int setup_fcg(int dev_sms) {
    TwoLevel T;
    const bool nullsp = S.dir_rows.empty();
    int rc = build_two_level(nc, S.WA, S.A_col.data(), S.A_val.data(), m.centroid.data(), dev_sms, nullsp, T);
    if (rc) return DPM_ERR_UNSUPPORTED;
    int cpt = 0;
    fcg_mixed = P.form == DPM_FORM_MIXED;
    fcg_kernel = fcg_kernel_for(T.C, T.WA, fcg_mixed, &cpt);
    fcg_smem = fcg_smem_bytes(T.P, T.C, T.WL, T.NB);
    if (!fcg_kernel || fcg_smem > 219 * 1024) return DPM_ERR_UNSUPPORTED;
    CK(cudaFuncSetAttribute(fcg_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fcg_smem));
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fcg_kernel, FCG_TPB, fcg_smem));
    if (per_sm < 1 || T.P > dev_sms * per_sm || T.P > FCG_MAX_GRID) return DPM_ERR_UNSUPPORTED;
    fa = FcgArgs{};
    fa.n = nc; fa.P = T.P; fa.C = T.C; fa.WL = T.WL;
    fa.perm = mem.upload(T.perm);
    fa.col = mem.upload(T.col);
    fa.val = mem.upload(T.val);
    fa.dinv = mem.upload(T.dinv);
    fa.lpk = mem.upload(T.lpk);
    fa.einv_nb = mem.upload(T.einv_nb);
    fa.NB = T.NB;
    fa.deflate = T.deflate;
    fa.srow = mem.upload(T.srow);
    fa.xoff = mem.upload(T.xoff);
    fa.xslot = mem.upload(T.xslot);
    fa.xval = mem.upload(T.xval);
    fa.xs = mem.alloc<double>(nc);
    fa.zs = mem.alloc<double>(nc);
    if (fcg_mixed) {
      std::vector<float> v32(T.val.begin(), T.val.end());
      fa.val32 = mem.upload(v32);
      fa.zs32 = mem.alloc<float>(nc);
      if (!fa.val32 || !fa.zs32) return DPM_ERR_CUDA;
    }
    fa.partials = mem.alloc<double>((size_t)2 * FCG_SLOT * T.P);
    fa.bar = cg_bar; fa.status = cg_status; fa.dout = cg_dout;
    fa.nullsp = nullsp ? 1 : 0;
    fa.degree = P.p_smooth_degree > 0 ? P.p_smooth_degree : 7;
    const double lmin = P.p_smooth_lmin > 0.0 ? P.p_smooth_lmin : 0.05;
    const double lmax = P.p_smooth_lmax > 0.0 ? P.p_smooth_lmax : 2.0;
    if (!(lmax > lmin)) return DPM_ERR_ARG;
    fa.theta = (float)(0.5 * (lmax + lmin));
    fa.delta = (float)(0.5 * (lmax - lmin));
    fcg_WA = T.WA;
    if (!fa.partials || !fa.zs) return DPM_ERR_CUDA;
    fa.stall_window = P.p_stall_window > 0 ? P.p_stall_window : 50;
    fa.stall_ratio = P.p_stall_ratio > 0.0 ? P.p_stall_ratio : 0.9;
    use_fcg = true;
    return setup_learned(T);
  }

  // Multilevel FCG set-up (csrc/cuda/mlsolve.cuh): hierarchy on the host, FP32 levels on the
  // device, the FP64 operator shared with the plain solve.
  int setup_ml(int dev_sms) {
    dev_sms_ = dev_sms;
    const bool nullsp = S.dir_rows.empty();
    // an aggregate holds up to 3^passes rows and the restriction gives it at most 32 lanes
    if (P.p_ml_passes > 3) return DPM_ERR_ARG;
    int rc = ml.setup(nc, S.WA, S.A_col.data(), S.A_val.data(), d.Acol, d.Aval, nullsp, P.p_ml_passes, P.p_ml_degree,
                      P.p_ml_overcorrect, dev_sms, cg_bar, cg_status, cg_dout, P.p_ml_value_bits);
    if (rc) return rc;
    if (P.p_stall_window > 0) ml.base.stall_window = P.p_stall_window;
    if (P.p_stall_ratio > 0.0) ml.base.stall_ratio = P.p_stall_ratio;
    use_ml = true;
    return 0;
  }
  int ml_launch(const double* rhs, double* x, double rtol, double atol, int maxit, int guess_zero, int* its,
                double* resid, int* reason) {
    MlArgs e{};
    if (ml_learn_ready && lp_ready) {
      e.omega = ml_omega;
      e.gamma = lp_gamma;
    }
    const bool rec = ml_learn_ready && lp_recording && lp_count < lp_S;
    if (rec) {
      e.gamma = 0.0f;
      e.rec_stride = lp_stride; e.rec_base = lp_count; e.rec_max = lp_S; e.pinv = ml_pinv;
      e.rec_r = lp_r; e.rec_z = lp_z; e.rec_u = lp_u; e.rec_x = lp_x;
    }
    launches++;
    int rc = ml.launch(rhs, x, rtol, atol, maxit, guess_zero, st, reason, its, resid, &e);
    if (rc) return rc;
    if (rec) {  // errors of the recorded iterates, in the learned term's numbering: e = x* - x_k
      const int used = std::min(lp_S - lp_count, *its / lp_stride + 1);
      if (used > 0) {
        k_perm_gather<<<nblk(nc), TPB, 0, st>>>(nc, fa.perm, x, fa.xs);
        dim3 g(nblk(nc), used);
        k_lp_err<<<g, TPB, 0, st>>>(nc, fa.xs, lp_x + (size_t)lp_count * nc);
        launches += 2;
        for (int k = 0; k < used; ++k) lp_solve_of.push_back(lp_solves);
        lp_count += used;
      }
      lp_solves++;
    }
    return 0;
  }
  // The learned term on the multilevel form: an RCB partition into parts of <= 4096 cells gives
  // the one-ring network its local rows and features (no coarse data), built on first use.
  int ml_learn_setup() {
    if (ml_learn_ready) return 0;
    TwoLevel T;
    const int P = std::max(dev_sms_, (nc + 4095) / 4096);
    if (build_two_level(nc, S.WA, S.A_col.data(), S.A_val.data(), m.centroid.data(), P, S.dir_rows.empty(), T, false))
      return DPM_ERR_UNSUPPORTED;
    fa = FcgArgs{};
    fa.n = nc; fa.P = T.P; fa.C = T.C; fa.WL = T.WL;
    fa.perm = mem.upload(T.perm);
    fa.col = mem.upload(T.col);
    fa.val = mem.upload(T.val);
    fa.dinv = mem.upload(T.dinv);
    fa.lpk = mem.upload(T.lpk);
    fa.xs = mem.alloc<double>(nc);
    fcg_WA = T.WA;
    std::vector<int> pinv(nc);
    for (int i = 0; i < nc; ++i) pinv[T.perm[i]] = i;
    ml_pinv = mem.upload(pinv);
    ml_omega = mem.alloc<float>(nc);
    if (!fa.perm || !fa.col || !fa.val || !fa.dinv || !fa.lpk || !fa.xs || !ml_pinv || !ml_omega) return DPM_ERR_CUDA;
    launch_fill_f(ml_omega, nc, 0.0f);
    int rc = setup_learned(T);
    if (rc) return rc;
    ml_learn_ready = true;
    return 0;
  }
  void ml_sync_omega() {  // the trained omega into the mesh numbering
    if (!ml_learn_ready) return;
    k_perm_scatter_f<<<nblk(nc), TPB, 0, st>>>(nc, fa.perm, lp_omega, ml_omega);
    launches++;
  }

  // Static per-cell features of the learned term, in the renumbered order:
  // [1, intra-part coupling mass, cross-part coupling mass, max and min scaled coupling,
  //  intra row-sum ratio, log diagonal scale, intra neighbour count / 6].
  int setup_learned(const TwoLevel& T) {
    const int n = T.n;
    std::vector<float> f((size_t)LP_F * n, 0.0f);
    double lmean = 0.0;
    for (int i = 0; i < n; ++i) lmean += std::log(1.0 / T.dinv[i]);
    lmean /= std::max(n, 1);
    for (int i = 0; i < n; ++i) {
      const int b = i / T.C;
      double intra = 0.0, cross = 0.0, mx = 0.0, mn = 1e300;
      int cnt = 0;
      for (int w = 0; w < T.WA; ++w) {
        const double v = T.val[(size_t)w * n + i];
        const int j = T.col[(size_t)w * n + i];
        if (v == 0.0 || j == i) continue;
        const double sv = std::fabs(v) * T.dinv[i];
        if (j / T.C == b) { intra += sv; cnt++; } else { cross += sv; }
        mx = std::max(mx, sv);
        mn = std::min(mn, sv);
      }
      if (mn > 1e299) mn = 0.0;
      f[0 * (size_t)n + i] = 1.0f;
      f[1 * (size_t)n + i] = (float)intra;
      f[2 * (size_t)n + i] = (float)cross;
      f[3 * (size_t)n + i] = (float)mx;
      f[4 * (size_t)n + i] = (float)mn;
      f[5 * (size_t)n + i] = (float)(T.srow[i] * T.dinv[i]);
      f[6 * (size_t)n + i] = (float)((std::log(1.0 / T.dinv[i]) - lmean) / 5.0);
      f[7 * (size_t)n + i] = (float)(cnt / 6.0);
    }
    lp_feat = mem.upload(f);
    lp_omega = mem.alloc<float>(n);
    lp_h1 = mem.alloc<float>((size_t)LP_H * n); lp_h2 = mem.alloc<float>((size_t)LP_H * n);
    lp_pre = mem.alloc<float>(n); lp_dom = mem.alloc<float>(n);
    lp_prm = mem.alloc<float>(LP_NP); lp_m1 = mem.alloc<float>(LP_NP); lp_m2 = mem.alloc<float>(LP_NP);
    lp_grad = mem.alloc<float>(LP_NP);
    lp_wb = mem.alloc<unsigned short>(LP_NP);
    lp_gpart = mem.alloc<float>((size_t)LP_BWD_BLOCKS * LP_NP);
    if (!lp_feat || !lp_omega || !lp_h1 || !lp_h2 || !lp_pre || !lp_dom || !lp_prm || !lp_wb || !lp_gpart)
      return DPM_ERR_CUDA;
    std::vector<float> p0 = lp_initial_params();
    CK(cudaMemcpyAsync(lp_prm, p0.data(), sizeof(float) * LP_NP, cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(lp_m1, 0, sizeof(float) * LP_NP, st));
    CK(cudaMemsetAsync(lp_m2, 0, sizeof(float) * LP_NP, st));
    k_lp_round<<<(LP_NP + 255) / 256, 256, 0, st>>>(LP_NP, lp_prm, lp_wb);
    launch_fill_f(lp_omega, n, 0.0f);
    launches++;
    fa.omega = lp_omega;
    fa.gamma = 0.0f;
    return 0;
  }
  static constexpr int LP_BWD_BLOCKS = 296;
  // Deterministic initial parameters: uniform in +-1/sqrt(fan_in) from SplitMix64, output bias -4
  // so that omega starts near zero.
  static std::vector<float> lp_initial_params() {
    std::vector<float> p(LP_NP, 0.0f);
    uint64_t x = 0x5EEDULL;
    auto uni = [&]() {
      x += 0x9E3779B97F4A7C15ULL;
      uint64_t z = x;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
      z ^= z >> 31;
      return (double)(z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
    };
    for (int j = 0; j < 256; ++j) p[LP_W1 + j] = (float)(uni() * 0.25);
    for (int j = 0; j < 256; ++j) p[LP_W2 + j] = (float)(uni() * 0.25);
    for (int j = 0; j < 16; ++j) p[LP_W3 + j] = (float)(uni() * 0.25);
    p[LP_B3] = -4.0f;
    return p;
  }
  void launch_fill_f(float* q, int64_t m, float v) {
    k_fill_f<<<nblk(m), TPB, 0, st>>>((int)m, q, v);
    launches++;
  }

  // Precision form: FP32-operator inner solves, each ending at 1e-5 of its own FP64 initial
  // residual, restarted from the current x (whose residual every launch recomputes in FP64) until
  // a launch finds the FP64 residual already below the target.
  int fcg(const double* rhs, double* x, double rtol, double atol, int maxit, int guess_zero, int* its, double* resid,
          int* reason) {
    if (!fcg_mixed) return fcg_launch(rhs, x, rtol, atol, maxit, guess_zero, its, resid, reason, 0.0);
    int tot = 0;
    for (int outer = 0; outer < 8; ++outer) {
      int it = 0;
      inner_rel_is_first_ = outer == 0;  // samples are recorded in the first inner solve only
      int rc = fcg_launch(rhs, x, rtol, atol, std::max(maxit - tot, 1), outer == 0 ? guess_zero : 0, &it, resid,
                          reason, 1.0e-5);
      if (rc) return rc;
      tot += it;
      if (*reason < 0 || it == 0 || tot >= maxit) break;
    }
    inner_rel_is_first_ = true;
    *its = tot;
    return 0;
  }
  int fcg_launch(const double* rhs, double* x, double rtol, double atol, int maxit, int guess_zero, int* its,
                 double* resid, int* reason, double inner_rel) {
    FcgArgs a = fa;
    a.inner_rel = inner_rel;
    a.phase = fcg_phase;
    a.b = rhs; a.x = x; a.rtol = rtol; a.atol = atol; a.maxit = maxit; a.guess_zero = guess_zero;
    a.gamma = lp_ready ? lp_gamma : 0.0f;
    const bool rec = lp_recording && lp_count < lp_S && inner_rel_is_first_;
    if (rec) {
      a.gamma = 0.0f;
      a.rec_stride = lp_stride; a.rec_base = lp_count; a.rec_max = lp_S;
      a.rec_r = lp_r; a.rec_z = lp_z; a.rec_u = lp_u; a.rec_x = lp_x;
    }
    CK(cudaMemsetAsync(cg_bar, 0, 2 * sizeof(unsigned), st));
    CK(cudaMemsetAsync(cg_status, 0, 4 * sizeof(int), st));
    if (spin_limit) CK(cudaMemcpyAsync(cg_status + 3, &spin_limit, sizeof(int), cudaMemcpyHostToDevice, st));
    int wa = fcg_WA;
    void* args[] = {&a, &wa};
    CK(cudaLaunchCooperativeKernel(fcg_kernel, dim3(a.P), dim3(FCG_TPB), args, fcg_smem, st));
    launches++;
    int h_st[4];
    double h_d[4];
    CK(cudaMemcpyAsync(h_st, cg_status, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(h_d, cg_dout, 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (h_st[2]) {
      std::fprintf(stderr, "dopamine_b200: FCG grid barrier timed out\n");
      return DPM_ERR_BARRIER_TIMEOUT;
    }
    *reason = h_st[0];
    *its = h_st[1];
    *resid = h_d[0];
    if (rec) {  // errors of the recorded iterates: e = x* - x_k (x* = the solve's final xs)
      const int used = std::min(lp_S - lp_count, *its / lp_stride + 1);
      if (used > 0) {
        dim3 g(nblk(nc), used);
        k_lp_err<<<g, TPB, 0, st>>>(nc, fa.xs, lp_x + (size_t)lp_count * nc);
        launches++;
        for (int k = 0; k < used; ++k) lp_solve_of.push_back(lp_solves);
        lp_count += used;
      }
      lp_solves++;
    }
    return 0;
  }

  // ---------------------------------------------------------------- learned term: training
  static constexpr int LP_DOT_BLOCKS = 64;
  int learn_alloc() {
    if (lp_r) return 0;
    const size_t m = (size_t)lp_S * nc;
    lp_r = mem.alloc<double>(m); lp_z = mem.alloc<double>(m); lp_u = mem.alloc<double>(m);
    lp_x = mem.alloc<double>(m); lp_azb = mem.alloc<double>(m); lp_av = mem.alloc<double>(m);
    lp_dpart = mem.alloc<double>((size_t)lp_S * LP_DOT_BLOCKS * 3);
    lp_dsum = mem.alloc<double>((size_t)lp_S * 3);
    lp_coef = mem.alloc<double>((size_t)lp_S * 2);
    return (lp_r && lp_z && lp_u && lp_x && lp_azb && lp_av && lp_dpart && lp_dsum && lp_coef) ? 0 : DPM_ERR_CUDA;
  }
  // per-sample dot products {a.b} over the first S slots, to the host
  int lp_dots(int S, const double* A1, const double* B1, const double* A2, const double* B2, const double* A3,
              const double* B3, std::vector<double>& out) {
    k_lp_dots3<<<dim3(LP_DOT_BLOCKS, S), 256, 0, st>>>(nc, A1, B1, A2, B2, A3, B3, lp_dpart);
    k_lp_sum_samples<<<(3 * S + 127) / 128, 128, 0, st>>>(S, LP_DOT_BLOCKS, lp_dpart, lp_dsum);
    launches += 2;
    out.resize(3 * S);
    CK(cudaMemcpyAsync(out.data(), lp_dsum, sizeof(double) * 3 * S, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return 0;
  }
  void lp_forward() {
    k_lp_forward<<<(nc + 127) / 128, 256, 0, st>>>(nc, fa.C, fa.WL, fa.lpk, lp_feat, lp_wb, lp_prm, lp_omega, lp_h1,
                                                   lp_h2, lp_pre);
    launches++;
  }
  // Loss over the first S slots at the current parameters; with grad, the parameter gradient
  // (into lp_grad).  base = {z.r, z.A z, e.r} per slot.
  int lp_loss_grad(int S, const std::vector<double>& base, double* loss, bool grad) {
    lp_forward();
    k_lp_av<<<dim3(nblk(nc), S), 256, 0, st>>>(nc, fcg_WA, S, fa.col, fa.val, lp_omega, lp_u, lp_av);
    k_lp_dots<<<dim3(LP_DOT_BLOCKS, S), 256, 0, st>>>(nc, S, lp_omega, lp_u, lp_r, lp_azb, lp_av, lp_dpart);
    k_lp_sum_samples<<<(3 * S + 127) / 128, 128, 0, st>>>(S, LP_DOT_BLOCKS, lp_dpart, lp_dsum);
    launches += 3;
    std::vector<double> q(3 * S), coef(2 * S);
    CK(cudaMemcpyAsync(q.data(), lp_dsum, sizeof(double) * 3 * S, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    double L = 0.0;
    int used = 0;
    for (int k = 0; k < S; ++k) {
      const double a = base[3 * k] + q[3 * k];
      const double b = base[3 * k + 1] + 2.0 * q[3 * k + 1] + q[3 * k + 2];
      const double c = base[3 * k + 2];
      coef[2 * k] = coef[2 * k + 1] = 0.0;
      // a sample whose error energy e.r is not positive (an iterate already at round-off) carries
      // no information: it is left out of the loss
      if (!(c > 0.0) || !(b > 0.0) || !std::isfinite(a)) continue;
      const double bc = b * c;
      L += 1.0 - a * a / bc;
      coef[2 * k] = 2.0 * a / bc;
      coef[2 * k + 1] = 2.0 * a * a / (bc * b);
      used++;
    }
    *loss = used > 0 ? L / used : 0.0;
    const double scale = used > 0 ? (double)S / used : 0.0;  // k_lp_domega divides by S
    for (auto& c : coef) c *= scale;
    if (!grad) return 0;
    CK(cudaMemcpyAsync(lp_coef, coef.data(), sizeof(double) * 2 * S, cudaMemcpyHostToDevice, st));
    k_lp_domega<<<nblk(nc), 256, 0, st>>>(nc, S, lp_coef, lp_u, lp_r, lp_azb, lp_av, lp_dom);
    k_lp_backward<<<LP_BWD_BLOCKS, 128, 0, st>>>(nc, fa.C, fa.WL, fa.lpk, lp_feat, lp_wb, lp_prm, lp_h1, lp_h2, lp_pre,
                                                 lp_dom, lp_gpart);
    k_lp_sum_f<<<(LP_NP + 127) / 128, 128, 0, st>>>(LP_BWD_BLOCKS, LP_NP, lp_gpart, lp_grad);
    launches += 3;
    return 0;
  }
  int lp_train_slots() const {  // slots of all but the last recorded solve (that one is held out)
    if (lp_count == 0) return 0;
    const int last = lp_solve_of.back();
    int k = 0;
    while (k < lp_count && lp_solve_of[k] < last) ++k;
    return k > 0 ? k : lp_count;
  }
  int lp_prepare(int S, std::vector<double>& base) {
    k_lp_spmv<<<dim3(nblk(nc), S), 256, 0, st>>>(nc, fcg_WA, fa.col, fa.val, lp_z, lp_azb);
    launches++;
    return lp_dots(S, lp_z, lp_r, lp_z, lp_azb, lp_x, lp_r, base);  // lp_x holds e after recording
  }
  // Held-out solves: the right-hand side recorded at iteration 0 of each held-out solve (its x0 is
  // 0), solved again from zero with the learned term scaled by g; total iterations.
  int lp_validate(float g, int* its_total) {
    *its_total = 0;
    const float keep = lp_gamma;
    const bool keep_ready = lp_ready;
    lp_gamma = g;
    lp_ready = true;
    for (int k = lp_train_slots(); k < lp_count; ++k) {
      if (k > 0 && lp_solve_of[k] == lp_solve_of[k - 1]) continue;  // first slot of each held-out solve
      k_perm_scatter<<<nblk(nc), TPB, 0, st>>>(nc, fa.perm, lp_r + (size_t)k * nc, scratch_c);
      launch_fill(scratch_c2, nc, 0.0);
      launches++;
      int its = 0, reason = 0;
      double res = 0.0;
      int rc = pcg(scratch_c, scratch_c2, P.p_tol, 1e-300, 2000, 1, &its, &res, &reason);
      if (rc) return rc;
      *its_total += its + (reason < 0 ? 100000 : 0);
    }
    lp_gamma = keep;
    lp_ready = keep_ready;
    return 0;
  }
  int learn_collect(int n_steps, int* n_samples) {
    if (!flexible()) return DPM_ERR_UNSUPPORTED;
    int rc = use_ml ? ml_learn_setup() : 0;
    if (rc) return rc;
    rc = learn_alloc();
    if (rc) return rc;
    lp_count = 0;
    lp_solves = 0;
    lp_solve_of.clear();
    lp_recording = true;
    for (int k = 0; k < n_steps && rc == 0; ++k) rc = advance(P.dt);
    lp_recording = false;
    if (n_samples) *n_samples = lp_count;
    return rc;
  }
  int learn_train(int epochs, double lr, dpm_learn_report_t* rep) {
    if (!flexible() || lp_count == 0) return DPM_ERR_ARG;
    auto t0 = std::chrono::steady_clock::now();
    const int S = lp_train_slots();
    std::vector<double> base;
    int rc = lp_prepare(S, base);
    if (rc) return rc;
    double L0 = 0.0, L = 0.0;
    rc = lp_loss_grad(S, base, &L0, false);
    if (rc) return rc;
    for (int e = 1; e <= epochs; ++e) {
      rc = lp_loss_grad(S, base, &L, true);
      if (rc) return rc;
      k_lp_adam<<<(LP_NP + 127) / 128, 128, 0, st>>>(LP_NP, lp_prm, lp_m1, lp_m2, lp_grad, (float)lr, 0.9f, 0.999f,
                                                    1e-8f, e, lp_wb);
      launches++;
    }
    rc = lp_loss_grad(S, base, &L, false);  // final loss, omega of the trained network
    if (rc) return rc;
    if (use_ml) ml_sync_omega();
    // gate: the scale of the learned term that does best on the held-out solves (ties keep 0)
    const float cand[3] = {0.0f, 0.5f, 1.0f};
    int best_its = 0, its0 = 0;
    float best = 0.0f;
    for (int c = 0; c < 3; ++c) {
      int its = 0;
      rc = lp_validate(cand[c], &its);
      if (rc) return rc;
      if (c == 0) { its0 = its; best_its = its; }
      else if (its < best_its) { best_its = its; best = cand[c]; }
    }
    lp_gamma = best;
    lp_ready = true;
    auto t1 = std::chrono::steady_clock::now();
    if (rep) {
      rep->samples = S;
      rep->val_solves = 0;
      for (int k = S; k < lp_count; ++k)
        if (k == S || lp_solve_of[k] != lp_solve_of[k - 1]) rep->val_solves++;
      rep->loss_initial = L0;
      rep->loss_final = L;
      rep->gamma = best;
      rep->its_val_base = its0;
      rep->its_val_learned = best_its;
      rep->train_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    }
    return 0;
  }

  // ---------------------------------------------------------------- Poisson solve
  int pcg(const double* rhs, double* x, double rtol, double atol, int maxit, int guess_zero, int* its, double* resid,
          int* reason) {
    if (use_fcg && !force_plain) return fcg(rhs, x, rtol, atol, maxit, guess_zero, its, resid, reason);
    if (use_ml && !force_plain) return ml_launch(rhs, x, rtol, atol, maxit, guess_zero, its, resid, reason);
    return pcg_plain(rhs, x, rtol, atol, maxit, guess_zero, its, resid, reason);
  }
  int pcg_plain(const double* rhs, double* x, double rtol, double atol, int maxit, int guess_zero, int* its,
                double* resid, int* reason) {
    PcgArgs<double> a{};
    a.n = nc; a.WA = S.WA; a.col = d.Acol; a.val = d.Aval; a.dinv = d.Adinv;
    a.b = rhs; a.x = x; a.r = cg_r; a.z = cg_z; a.p0 = cg_p0; a.p1 = cg_p1; a.q = cg_q; a.bp = cg_bp;
    a.partials = cg_part; a.bar = cg_bar; a.status = cg_status; a.dout = cg_dout;
    a.rtol = rtol; a.atol = atol; a.maxit = maxit; a.nullsp = S.dir_rows.empty() ? 1 : 0; a.guess_zero = guess_zero;
    CK(cudaMemsetAsync(cg_bar, 0, 2 * sizeof(unsigned), st));
    CK(cudaMemsetAsync(cg_status, 0, 4 * sizeof(int), st));
    if (spin_limit) CK(cudaMemcpyAsync(cg_status + 3, &spin_limit, sizeof(int), cudaMemcpyHostToDevice, st));
    void* args[] = {&a};
    CK(cudaLaunchCooperativeKernel(cg_kernel, dim3(cg_grid), dim3(PCG_TPB), args, 0, st));
    launches++;
    int h_st[4];
    double h_d[4];
    CK(cudaMemcpyAsync(h_st, cg_status, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(h_d, cg_dout, 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (h_st[2]) {
      std::fprintf(stderr, "dopamine_b200: PCG grid barrier timed out\n");
      return DPM_ERR_BARRIER_TIMEOUT;
    }
    *reason = h_st[0];
    *its = h_st[1];
    *resid = h_d[0];
    return 0;
  }

  // pressure_solver_solve + fvm_petsc_solve_pressure: NaN scrub, Dirichlet rows when the
  // pressure is total, BJACOBI-style retry from a zero guess on failure.
  int pressure_solve(double tol, double atol, bool ptot, int* its_out, double* res_out) {
    const double* rhs = F.rhs;
    if (ptot && !S.dir_rows.empty()) {
      std::vector<double> add(nc, 0.0);
      for (size_t k = 0; k < S.dir_rows.size(); ++k) add[S.dir_rows[k]] += S.dir_vals[k];
      CK(cudaMemcpyAsync(scratch_c2, add.data(), nc * sizeof(double), cudaMemcpyHostToDevice, st));
      copy(scratch_c, F.rhs, nc);
      k_add<<<nblk(nc), TPB, 0, st>>>(nc, scratch_c, scratch_c2);
      launches++;
      rhs = scratch_c;
    }
    int maxit = std::max(P.p_max_iter, 2000), its = 0, reason = 0;
    double res = 0.0;
    cudaEventRecord(evp0, st);
    int rc = pcg(rhs, F.p, tol, atol, maxit, 0, &its, &res, &reason);
    if (rc) return rc;
    if (reason < 0 && flexible()) {  // flexible CG stalled or failed: plain Jacobi-PCG takes over from its x
      p_fallbacks++;
      int its2 = 0;
      rc = pcg_plain(rhs, F.p, tol, atol, maxit, 0, &its2, &res, &reason);
      if (rc) return rc;
      its += its2;
    }
    if (reason < 0) {
      rc = pcg_plain(rhs, F.p, tol, atol, 4 * maxit, 1, &its, &res, &reason);
      if (rc) return rc;
      if (reason < 0 && !(reason == -3 && (res < tol * 1.0e4 || res < atol * 1.0e3))) return -(1000 + reason);
    }
    cudaEventRecord(evp1, st);
    cudaEventSynchronize(evp1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, evp0, evp1);
    poisson_ms_acc += ms;
    *its_out = its;
    *res_out = res;
    return 0;
  }

  // ---------------------------------------------------------------- synthetic-eddy inflow (sem.cuh)
  // sem_init (src/abl/mod_sem_inflow.f90:59-316): the inlet frame and its periodic directions, the
  // eddy scales, the box and the seeded eddies; false (nothing to do) without an ABL inlet
  int setup_sem() {
    const int64_t nfi = m.n_int_faces;
    std::vector<int> fl;
    for (int b = 0; b < nb; ++b) {
      const int q = m.patch[nfi + b];
      if (q >= 0 && pc[q].bc_id == BC_ABL_INLET) fl.push_back(b);
    }
    if (!P.use_sem || fl.empty()) return 0;
    sem_cfg = SemCfg{P.abl_u_ref, P.abl_z_ref, P.abl_z0_m, P.abl_wind_dir_deg, P.sem_alpha, P.sem_Iu_ref, P.sem_Iv_ratio,
                     P.sem_Iw_ratio, P.sem_rho_uw, P.sem_mean_law == DPM_SEM_MEAN_POWER ? 1 : 0};
    SemState s{};
    auto dot = [](const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
    double ns[3] = {0, 0, 0}, xs[3] = {0, 0, 0}, asum = 0.0;
    for (int b : fl) {
      const int64_t f = nfi + b;
      for (int k = 0; k < 3; ++k) { ns[k] = ns[k] + m.area[f] * m.normal[3 * f + k]; xs[k] = xs[k] + m.area[f] * m.centre[3 * f + k]; }
      asum = asum + m.area[f];
    }
    const double nl = std::sqrt(ns[0] * ns[0] + ns[1] * ns[1] + ns[2] * ns[2]);
    if (!(asum > SEM_SMALL) || nl <= SEM_SMALL) return 0;
    for (int k = 0; k < 3; ++k) { s.n_in[k] = -ns[k] / nl; s.x_inlet[k] = xs[k] / asum; }
    const double seed_axis[3] = {std::fabs(s.n_in[2]) < 0.9 ? 0.0 : 1.0, 0.0, std::fabs(s.n_in[2]) < 0.9 ? 1.0 : 0.0};
    s.t1[0] = seed_axis[1] * s.n_in[2] - seed_axis[2] * s.n_in[1];
    s.t1[1] = seed_axis[2] * s.n_in[0] - seed_axis[0] * s.n_in[2];
    s.t1[2] = seed_axis[0] * s.n_in[1] - seed_axis[1] * s.n_in[0];
    const double tl = std::max(std::sqrt(dot(s.t1, s.t1)), SEM_SMALL);
    for (int k = 0; k < 3; ++k) s.t1[k] = s.t1[k] / tl;
    s.t2[0] = s.n_in[1] * s.t1[2] - s.n_in[2] * s.t1[1];
    s.t2[1] = s.n_in[2] * s.t1[0] - s.n_in[0] * s.t1[2];
    s.t2[2] = s.n_in[0] * s.t1[1] - s.n_in[1] * s.t1[0];
    const double HUGE_V = 1.7976931348623157e308;
    double lo[2] = {HUGE_V, HUGE_V}, hi[2] = {-HUGE_V, -HUGE_V};
    for (int b : fl) {
      const int64_t f = nfi + b;
      double dd[3];
      for (int k = 0; k < 3; ++k) dd[k] = m.centre[3 * f + k] - s.x_inlet[k];
      lo[0] = std::min(lo[0], dot(dd, s.t1)); hi[0] = std::max(hi[0], dot(dd, s.t1));
      lo[1] = std::min(lo[1], dot(dd, s.t2)); hi[1] = std::max(hi[1], dot(dd, s.t2));
    }
    s.t1_min = lo[0]; s.t1_max = hi[0]; s.t2_min = lo[1]; s.t2_max = hi[1];
    double plo[2] = {HUGE_V, HUGE_V}, phi[2] = {-HUGE_V, -HUGE_V};  // sem_detect_periodic (:131-165)
    for (int k = 0; k < 2; ++k) {
      const double* tk = k == 0 ? s.t1 : s.t2;
      for (int b = 0; b < nb; ++b) {
        const int q = m.patch[nfi + b];
        if (q < 0 || pc[q].bc_id != BC_PERIODIC) continue;
        const int64_t f = nfi + b;
        if (std::fabs(dot(&m.normal[3 * f], tk)) < 0.99) continue;
        double dd[3];
        for (int j = 0; j < 3; ++j) dd[j] = m.centre[3 * f + j] - s.x_inlet[j];
        plo[k] = std::min(plo[k], dot(dd, tk)); phi[k] = std::max(phi[k], dot(dd, tk));
      }
    }
    if (phi[0] - plo[0] > SEM_SMALL && plo[0] <= s.t1_min + SEM_SMALL && phi[0] >= s.t1_max - SEM_SMALL) {
      s.per1 = 1; s.period1 = phi[0] - plo[0]; s.per1_lo = plo[0];
    }
    if (phi[1] - plo[1] > SEM_SMALL && plo[1] <= s.t2_min + SEM_SMALL && phi[1] >= s.t2_max - SEM_SMALL) {
      s.per2 = 1; s.period2 = phi[1] - plo[1]; s.per2_lo = plo[1];
    }
    // sem_setup (:211-297)
    const int ne = std::max(1, P.sem_n_eddies);
    s.n = ne;
    s.sigma = P.sem_sigma <= SEM_SMALL ? 0.1 * std::min(s.t1_max - s.t1_min, s.t2_max - s.t2_min) : P.sem_sigma;
    if (s.sigma <= SEM_SMALL) s.sigma = 0.1 * P.abl_z_ref;
    s.dfsem = P.sem_type != DPM_SEM_JARRIN;
    s.rsup = s.sigma;
    if (s.dfsem) {  // sem_reference_scales (:795-841): the largest principal stress over the inlet heights
      const int nlv = 65;
      const double zlo = s.x_inlet[2] + s.t2_min, zhi = s.x_inlet[2] + s.t2_max;
      double lmax = SEM_SMALL, Rm[9], Wr[9], lam[3], V[9];
      for (int k = 1; k <= nlv; ++k) {
        const double z = k < nlv ? zlo + (zhi - zlo) * (double)(k - 1) / (double)(nlv - 2) : P.abl_z_ref;
        sem_stress(sem_cfg, z, Rm, Wr);
        sem_eigen3(Rm, lam, V);
        lmax = std::max(lmax, std::max(lam[0], std::max(lam[1], lam[2])));
      }
      s.lam_ref = lmax;
    }
    if ((s.per1 && s.rsup >= 0.5 * s.period1) || (s.per2 && s.rsup >= 0.5 * s.period2)) {
      std::fprintf(stderr, "dopamine_b200: the eddy support must be below half the periodic inlet width\n");
      return DPM_ERR_ARG;
    }
    if (s.per1) { s.t1_min = s.per1_lo; s.t1_max = s.per1_lo + s.period1; }
    else { s.t1_min = s.t1_min - s.rsup; s.t1_max = s.t1_max + s.rsup; }
    if (s.per2) { s.t2_min = s.per2_lo; s.t2_max = s.per2_lo + s.period2; }
    else { s.t2_min = s.t2_min - s.rsup; s.t2_max = s.t2_max + s.rsup; }
    s.box_volume = 2.0 * s.rsup * (s.t1_max - s.t1_min) * (s.t2_max - s.t2_min);
    s.u_convect = std::max(P.abl_u_ref, SEM_SMALL);
    s.rng = 88172645463325252ULL;
    if (P.sem_seed != 0) {
      s.rng = 88172645463325252ULL ^ ((unsigned long long)(long long)P.sem_seed * 2654435761ULL);
      if (s.rng == 0) s.rng = 88172645463325252ULL;
      for (int i = 0; i < 8; ++i) sem_rand(s.rng);
    }
    std::vector<double> pos(3 * (size_t)ne, 0.0), amp(3 * (size_t)ne, 0.0);
    for (int i = 0; i < ne; ++i) {
      const double sv = s.rsup * (2.0 * sem_rand(s.rng) - 1.0);
      sem_place(s, pos.data(), amp.data(), i, sv, true);
    }
    for (int k = 0; k < 3; ++k) {  // sem_balance_amplitudes (:300-316)
      double ssum = 0.0;
      for (int i = 0; i < ne; ++i) ssum = ssum + amp[3 * i + k];
      for (int i = 0; i < ne; ++i) {
        if (std::fabs(ssum) < 1.0) break;
        if (amp[3 * i + k] * ssum > 0.0) {
          amp[3 * i + k] = -amp[3 * i + k];
          ssum = ssum + 2.0 * amp[3 * i + k];
        }
      }
    }
    s.pos = mem.upload(pos);
    s.amp = mem.upload(amp);
    s.frame = mem.alloc<double>(9 * (size_t)ne);
    s.sig = mem.alloc<double>(3 * (size_t)ne);
    s.ampl = mem.alloc<double>(3 * (size_t)ne);
    sem_d = mem.alloc<SemState>(1);
    sem_faces = mem.upload(fl);
    sem_nfaces = (int)fl.size();
    sem_grid = std::max(1, std::min(nblk(sem_nfaces), SEM_FACE_BLOCKS_MAX));
    sem_part = mem.alloc<double>(2 * (size_t)sem_grid);
    sem_fluc = mem.alloc<double>(3 * (size_t)nb);
    if (!s.pos || !s.amp || !s.frame || !s.sig || !s.ampl || !sem_d || !sem_faces || !sem_part || !sem_fluc)
      return DPM_ERR_CUDA;
    CK(cudaMemcpy(sem_d, &s, sizeof(SemState), cudaMemcpyHostToDevice));
    sem_h = s;
    d.abl_fluc = sem_fluc;
    sem_on = true;
    return update_sem(false, 0.0);
  }
  // update_sem_inflow (mod_fv_solver.f90:2062-2119) for the eddies' current positions
  int update_sem(bool look_ahead, double tau) {
    if (!sem_on) return 0;
    if (sem_h.dfsem) {
      k_sem_prepare<<<(sem_h.n + 127) / 128, 128, 0, st>>>(sem_cfg, sem_h);
      launches++;
    }
    k_sem_faces<<<sem_grid, TPB, 0, st>>>(d, sem_cfg, sem_h, sem_nfaces, sem_faces, look_ahead ? 1 : 0, tau, sem_fluc,
                                          sem_part);
    k_sem_finish<<<sem_grid, TPB, 0, st>>>(d, sem_nfaces, sem_faces, sem_grid, sem_part, sem_fluc);
    launches += 2;
    return 0;
  }

  // ---------------------------------------------------------------- sources (forcing.cuh)
  bool split_rhs() const { return P.use_nudging || !srcs.empty(); }
  // compute_explicit_rhs's tail (mod_fv_solver.f90:1741-1760): scalar sources in their order, then
  // the nudging of U and T, at the stage time
  void add_sources_and_nudging() {
    for (size_t i = 0; i < srcs.size(); ++i) {
      const dpm_scalar_source_t& q = srcs[i];
      if (!q.enabled || q.scalar_id < 1 || q.scalar_id > ns) continue;
      k_scalar_source<<<nblk(nc), TPB, 0, st>>>(d, q, src_tags[i], time, HC + (size_t)(q.scalar_id - 1) * nc);
      launches++;
    }
    if (P.use_nudging && nd_nt > 0) {
      NudgeArgs a{};
      interp_find(nd_times_h.data(), nd_nt, time, a.it1, a.it2, a.wt);
      a.nz = nd_nz;
      a.horiz = P.nudging_horizontal_only ? 1 : 0;
      a.coeff = 1.0 / std::max(P.nudging_tau, NUDGE_SMALL);
      if (P.dt > NUDGE_SMALL) a.coeff = std::min(a.coeff, 0.5 / P.dt);
      a.zs = P.nudging_z_start;
      a.zt = P.nudging_z_full;
      a.z = nd_z; a.Up = nd_U; a.Tp = nd_T;
      k_nudging<<<nblk(nc), TPB, 0, st>>>(d, a, F.U, F.T, F.H, HT);
      launches++;
    }
  }
  template <class T>
  int dev_copy(T** dst, const T* src, size_t n) {
    if (*dst) cudaFree(*dst);
    *dst = nullptr;
    CK(cudaMalloc(dst, std::max<size_t>(n, 1) * sizeof(T)));
    if (n) CK(cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice));
    return 0;
  }
  int set_nudging(int nt, int nz, const double* times, const double* z, const double* Up, const double* Tp) {
    if (nt < 1 || nz < 1 || !times || !z || !Up || !Tp) return DPM_ERR_ARG;
    if (x32) return DPM_ERR_UNSUPPORTED;
    nd_nt = nt; nd_nz = nz;
    nd_times_h.assign(times, times + nt);
    nd_z_h.assign(z, z + nz);
    int rc = dev_copy(&nd_z, z, (size_t)nz);
    if (!rc) rc = dev_copy(&nd_U, Up, 3 * (size_t)nz * nt);
    if (!rc) rc = dev_copy(&nd_T, Tp, (size_t)nz * nt);
    return rc;
  }
  void free_sources() {
    for (double* p : src_tags)
      if (p) cudaFree(p);
    src_tags.clear();
    srcs.clear();
  }
  int set_sources(int n, const dpm_scalar_source_t* q) {
    if (n < 0 || (n > 0 && !q)) return DPM_ERR_ARG;
    if (n > 0 && x32) return DPM_ERR_UNSUPPORTED;
    free_sources();
    for (int i = 0; i < n; ++i) {
      dpm_scalar_source_t s = q[i];
      double* tags = nullptr;
      if (s.n_tag_points > 0 && s.tag_points) {
        int rc = dev_copy(&tags, s.tag_points, 3 * (size_t)s.n_tag_points);
        if (rc) return rc;
      }
      s.tag_points = nullptr;
      srcs.push_back(s);
      src_tags.push_back(tags);
    }
    return 0;
  }

  // ---------------------------------------------------------------- sampling (sampling.cuh)
  void free_samples() {
    if (samp_pts) cudaFree(samp_pts);
    if (samp_payload) cudaFree(samp_payload);
    if (samp_owner) cudaFree(samp_owner);
    samp_pts = samp_payload = nullptr;
    samp_owner = nullptr;
    samp_n = 0;
  }
  // cache_object_owners (src/stats/mod_sampling.f90:520-562) for the points xyz(3, n)
  int set_sample_points(int n, const double* xyz, int* owner_out) {
    free_samples();
    if (n <= 0) return 0;
    CK(cudaMalloc(&samp_pts, 3 * sizeof(double) * n));
    CK(cudaMalloc(&samp_payload, 6 * sizeof(double) * n));
    CK(cudaMalloc(&samp_owner, sizeof(int) * n));
    samp_n = n;
    CK(cudaMemcpyAsync(samp_pts, xyz, 3 * sizeof(double) * n, cudaMemcpyHostToDevice, st));
    k_sample_owner<<<(n + SAMPLE_TILE - 1) / SAMPLE_TILE, SAMPLE_TILE, 0, st>>>(d, n, samp_pts, samp_owner);
    launches++;
    if (owner_out) CK(cudaMemcpyAsync(owner_out, samp_owner, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    CK(cudaGetLastError());
    return 0;
  }
  // sample_points_local (:493-518) on the current state; payload(6, n) to the host
  int sample_points(double* payload) {
    if (samp_n <= 0) return DPM_ERR_ARG;
    k_sample_points<<<nblk(samp_n), TPB, 0, st>>>(d, samp_n, samp_pts, samp_owner, F.U, F.Ub, F.p, F.pb, F.T, Tb,
                                                  F.nu_sgs, samp_payload);
    launches++;
    CK(cudaMemcpyAsync(payload, samp_payload, 6 * sizeof(double) * samp_n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    CK(cudaGetLastError());
    return 0;
  }

  // ---------------------------------------------------------------- checkpoint (mod_checkpoint_io.f90)
  // A device array (SoA [k][n] when k > 1) in the Fortran layout (k, n) on the host.
  int fetch(const double* dev, int n, int k, std::vector<double>& h) {
    h.resize((size_t)n * k);
    if (n == 0) return 0;
    if (k == 1) {
      CK(cudaMemcpyAsync(h.data(), dev, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    } else {
      k_soa_to_aos_k<<<nblk(n), TPB, 0, st>>>(n, k, dev, aos_buf);
      launches++;
      CK(cudaMemcpyAsync(h.data(), aos_buf, sizeof(double) * (size_t)n * k, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    return 0;
  }
  int store(double* dev, int n, int k, const std::vector<char>& rec) {
    if ((int64_t)rec.size() != (int64_t)n * k * 8) return DPM_ERR_ARG;
    if (n == 0) return 0;
    if (k == 1) {
      CK(cudaMemcpyAsync(dev, rec.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st));
    } else {
      CK(cudaMemcpyAsync(aos_buf, rec.data(), sizeof(double) * (size_t)n * k, cudaMemcpyHostToDevice, st));
      k_aos_to_soa_k<<<nblk(n), TPB, 0, st>>>(n, k, aos_buf, dev);
      launches++;
    }
    CK(cudaStreamSynchronize(st));
    return 0;
  }
  // header(8): 1 tau_w_bnd, 2 q_w_bnd, 4 L_bnd (MOST), 8 the wall-stress filter state, 16 eddies
  int checkpoint_mask() const {
    int mask = 1;
    if (P.wall_model == DPM_WM_MOST) mask += 2 + 4;
    if (filt_ready && P.wall_model == DPM_WM_LOGLAW) mask += 8;
    if (sem_on) mask += 16;
    return mask;
  }
  static std::string checkpoint_file(const char* dir, int file_step) {
    char name[64];
    std::snprintf(name, sizeof name, "checkpoint_%08d.bin", file_step);
    return (std::filesystem::path(dir) / "processor0" / name).string();
  }
  // write_checkpoint (:15-138): <dir>/processor0/checkpoint_<step>.bin and <dir>/checkpoint_latest
  int write_checkpoint(const char* dir, int file_step) {
    std::error_code ec;
    std::filesystem::create_directories(std::filesystem::path(dir) / "processor0", ec);
    if (ec) return DPM_ERR_ARG;
    const std::string fname = checkpoint_file(dir, file_step);
    std::FILE* f = std::fopen(fname.c_str(), "wb");
    if (!f) return DPM_ERR_ARG;
    bool ok = true;
    int rc = 0;
    const int mask = checkpoint_mask();
    int32_t hdr[8] = {(int32_t)nc, (int32_t)ns, 0, (int32_t)step, ns > 0 ? 1 : 0, 0, u_face_ready ? 1 : 0, mask};
    ok = ok && frec::write_record(f, hdr, sizeof hdr);
    ok = ok && frec::write_record(f, &time, sizeof time);
    {
      std::vector<int64_t> gid(nc);
      for (int c = 0; c < nc; ++c) gid[c] = c + 1;
      ok = ok && (nc == 0 || frec::write_record(f, gid.data(), 8 * (int64_t)nc));
    }
    std::vector<double> h;
    auto put = [&](const double* dev, int n, int k) {
      if (!ok || rc) return;
      rc = fetch(dev, n, k, h);
      if (!rc) ok = frec::write_record(f, h.data(), 8 * (int64_t)n * k);
    };
    if (nc > 0) {
      put(F.U, nc, 3);
      put(F.p, nc, 1);
      put(F.T, nc, 1);
      put(F.nu_sgs, nc, 1);
      if (ns > 0) put(Cs, nc, ns);
    }
    if (u_face_ready) put(F.Uf, nf, 1);
    put(F.tau, nb, 3);
    if (mask & 2) put(most_qw, nb, 1);
    if (mask & 4) put(most_L, nb, 1);
    if (mask & 8) put(F.upf, nb, 3);
    if ((mask & 16) && ok && !rc) {  // eddy count and generator state, positions, signs (:127-131)
      SemState cur{};
      if (cudaMemcpy(&cur, sem_d, sizeof(SemState), cudaMemcpyDeviceToHost) != cudaSuccess) rc = DPM_ERR_CUDA;
      char head[12];
      const int32_t n32 = sem_h.n;
      const int64_t r64 = (int64_t)cur.rng;
      std::memcpy(head, &n32, 4);
      std::memcpy(head + 4, &r64, 8);
      ok = !rc && frec::write_record(f, head, 12);
      std::vector<double> hv(3 * (size_t)sem_h.n);
      for (double* dv : {sem_h.pos, sem_h.amp}) {
        if (!ok || cudaMemcpy(hv.data(), dv, hv.size() * 8, cudaMemcpyDeviceToHost) != cudaSuccess) { ok = false; break; }
        ok = frec::write_record(f, hv.data(), 8 * (int64_t)hv.size());
      }
    }
    ok = (std::fclose(f) == 0) && ok;
    if (rc) return rc;
    if (!ok) return DPM_ERR_ARG;
    std::FILE* l = std::fopen((std::filesystem::path(dir) / "checkpoint_latest").string().c_str(), "w");
    if (!l) return DPM_ERR_ARG;
    std::fprintf(l, "%d\n", file_step);
    return std::fclose(l) == 0 ? 0 : DPM_ERR_ARG;
  }
  // read_checkpoint (:143-282) and refresh_after_restart (mod_fv_solver.f90:601-609); file_step
  // < 0 reads the step that <dir>/checkpoint_latest names
  int read_checkpoint(const char* dir, int file_step) {
    if (file_step < 0) {
      std::FILE* l = std::fopen((std::filesystem::path(dir) / "checkpoint_latest").string().c_str(), "r");
      if (!l) return DPM_ERR_ARG;
      int k = -1;
      const int got = std::fscanf(l, "%d", &k);
      std::fclose(l);
      if (got != 1 || k < 0) return DPM_ERR_ARG;
      file_step = k;
    }
    std::FILE* f = std::fopen(checkpoint_file(dir, file_step).c_str(), "rb");
    if (!f) return DPM_ERR_ARG;
    std::vector<char> rec;
    auto next = [&]() { return frec::read_record(f, rec); };
    int32_t hdr[8];
    double t = 0.0;
    int rc = DPM_ERR_ARG;
    do {
      if (!next() || rec.size() != sizeof hdr) break;
      std::memcpy(hdr, rec.data(), sizeof hdr);
      if (hdr[0] != nc || hdr[1] != ns) {
        std::fprintf(stderr, "dopamine_b200: checkpoint has %d cells / %d scalars, this handle %d / %d\n", hdr[0],
                     hdr[1], nc, ns);
        rc = DPM_ERR_MESH;
        break;
      }
      if (!frec::read_record_into(f, &t, sizeof t)) break;
      if (nc > 0) {
        if (!next() || (int64_t)rec.size() != 8 * (int64_t)nc) break;
        const int64_t* gid = reinterpret_cast<const int64_t*>(rec.data());
        bool same = true;
        for (int c = 0; c < nc && same; ++c) same = gid[c] == c + 1;
        if (!same) {  // the reference stops on a different partition (:205-206)
          rc = DPM_ERR_MESH;
          break;
        }
        if (!next() || store(F.U, nc, 3, rec)) break;
        if (!next() || store(F.p, nc, 1, rec)) break;
        if (!next() || store(F.T, nc, 1, rec)) break;
        if (!next() || store(F.nu_sgs, nc, 1, rec)) break;
        if (hdr[1] > 0 && (!next() || store(Cs, nc, ns, rec))) break;
      }
      if (hdr[6] == 1) {
        if (!next() || store(F.Uf, nf, 1, rec)) break;
        u_face_ready = true;
      } else {
        std::fprintf(stderr, "dopamine_b200: checkpoint has no face flux; it is rebuilt from the restored velocity\n");
      }
      const int mask = hdr[7];
      bool bad = false;
      if (mask & 1) bad = bad || !next() || store(F.tau, nb, 3, rec);
      if (mask & 2) bad = bad || !next() || (P.wall_model == DPM_WM_MOST && store(most_qw, nb, 1, rec));
      if (mask & 4) bad = bad || !next() || (P.wall_model == DPM_WM_MOST && store(most_L, nb, 1, rec));
      if (mask & 8) {
        bad = bad || !next() || store(F.upf, nb, 3, rec);
        if (!bad) filt_ready = true;
      }
      if (mask & 16) {  // synthetic-eddy state, adopted when this run has the same eddy count
        std::vector<char> head, rp, ra;
        bad = bad || !frec::read_record(f, head) || !frec::read_record(f, rp) || !frec::read_record(f, ra);
        if (!bad && head.size() == 12) {
          int32_t n32;
          int64_t r64;
          std::memcpy(&n32, head.data(), 4);
          std::memcpy(&r64, head.data() + 4, 8);
          if (sem_on && n32 == sem_h.n && rp.size() == 24 * (size_t)n32 && ra.size() == rp.size()) {
            CK(cudaMemcpy(sem_h.pos, rp.data(), rp.size(), cudaMemcpyHostToDevice));
            CK(cudaMemcpy(sem_h.amp, ra.data(), ra.size(), cudaMemcpyHostToDevice));
            sem_h.rng = (unsigned long long)r64;
            CK(cudaMemcpy(sem_d, &sem_h, sizeof(SemState), cudaMemcpyHostToDevice));
          } else {
            std::fprintf(stderr, "dopamine_b200: checkpoint synthetic-eddy state does not match this run\n");
          }
        }
      }
      if (bad) break;
      rc = 0;
    } while (false);
    std::fclose(f);
    if (rc) return rc;
    time = t;
    step = hdr[3];
    if (sem_on) update_sem(false, 0.0);  // inlet fluctuation of the restored eddies (:262-263)
    refresh_halos_and_bc();
    grad_all();
    pressure_gradient();
    refresh_halos_and_bc();
    grad_all();
    if (!u_face_ready) {
      rc = rebuild_face_flux();
      if (rc) return rc;
    }
    CK(cudaStreamSynchronize(st));
    CK(cudaGetLastError());
    return 0;
  }
  // solver_rebuild_face_flux (mod_fv_solver.f90:612-654): one projection whose face flux is kept,
  // everything else put back
  int rebuild_face_flux() {
    const size_t n3 = 3 * (size_t)nc;
    std::vector<double> U0(n3), p0(nc), pb0(nb), Ub0(3 * (size_t)nb), ff0(nf), pold0(nc), pp0(nc), ppb0(nb), gp0(n3),
        gprc0(n3);
    auto down = [&](std::vector<double>& h, const double* dv) {
      if (!h.empty()) cudaMemcpyAsync(h.data(), dv, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st);
    };
    auto up = [&](double* dv, const std::vector<double>& h) {
      if (!h.empty()) cudaMemcpyAsync(dv, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, st);
    };
    down(U0, F.U); down(p0, F.p); down(pb0, F.pb); down(Ub0, F.Ub); down(ff0, F.ff); down(pold0, F.p_old);
    down(pp0, F.phi_prev); down(ppb0, F.phi_prev_b); down(gp0, F.gp); down(gprc0, F.gp_rc);
    CK(cudaStreamSynchronize(st));
    int rc = project_once(P.dt);
    if (rc) return rc;
    up(F.U, U0); up(F.p, p0); up(F.pb, pb0); up(F.Ub, Ub0); up(F.ff, ff0); up(F.p_old, pold0);
    up(F.phi_prev, pp0); up(F.phi_prev_b, ppb0); up(F.gp, gp0); up(F.gp_rc, gprc0);
    CK(cudaStreamSynchronize(st));
    u_face_ready = true;
    return 0;
  }

  // ---------------------------------------------------------------- exact cell projection
  int cp_alloc() {
    if (cp_st) return 0;
    cp_x = mem.alloc<double>(nc); cp_r = mem.alloc<double>(nc); cp_z = mem.alloc<double>(nc);
    cp_p = mem.alloc<double>(nc); cp_q = mem.alloc<double>(nc); cp_rold = mem.alloc<double>(nc);
    cp_bconst = mem.alloc<double>(nc); cp_v = mem.alloc<double>(3 * (size_t)nc);
    cp_part = mem.alloc<double>((size_t)CP_RED_BLOCKS * CP_NPART);
    cp_st = mem.alloc<CpState>(1);
    return (cp_x && cp_r && cp_z && cp_p && cp_q && cp_rold && cp_bconst && cp_v && cp_part && cp_st) ? 0 : DPM_ERR_CUDA;
  }
  int cp_grid() const { return std::max(1, std::min(nblk(nc), CP_RED_BLOCKS)); }
  double cp_tol() const { return std::max(P.cell_projection_tol > 0.0 ? P.cell_projection_tol : 0.1, 1.0e-8); }
  // The projection's preconditioner (mod_fv_solver.f90:3277-3282): z = 0, then the handle's
  // pressure solve to rtol 0.05 with at most 50 iterations, which the backend raises to its 2000
  // floor (pressure_backend_petsc.c:844); a failed solve is retried from zero like pressure_solve.
  int cp_precond(int* its_out) {
    launch_fill(cp_z, nc, 0.0);
    const double tol = 0.05, atol = 1.0e-50;
    const int maxit = std::max(50, 2000);
    int its = 0, reason = 0;
    double res = 0.0;
    int rc = pcg(cp_r, cp_z, tol, atol, maxit, 0, &its, &res, &reason);
    if (rc) return rc;
    if (reason < 0 && flexible()) {
      p_fallbacks++;
      int its2 = 0;
      rc = pcg_plain(cp_r, cp_z, tol, atol, maxit, 0, &its2, &res, &reason);
      if (rc) return rc;
      its += its2;
    }
    if (reason < 0) {
      rc = pcg_plain(cp_r, cp_z, tol, atol, 4 * maxit, 1, &its, &res, &reason);
      if (rc) return rc;
      if (reason < 0 && !(reason == -3 && (res < tol * 1.0e4 || res < atol * 1.0e3))) return -(1000 + reason);
    }
    *its_out = its;
    return 0;
  }
  // cp_project (src/numerics/mod_cell_projection.f90:192-303) on the SoA velocity u; identity_pc
  // replaces the pressure-solve preconditioner by z = r (the reference's unit test does so).
  int cp_project(double* u, const double* bconst, double tol, int max_it, bool identity_pc, int* n_it) {
    int rc = cp_alloc();
    if (rc) return rc;
    const int g = cp_grid();
    launch_fill(cp_x, nc, 0.0);
    k_cp_rhs<<<g, TPB, 0, st>>>(d, u, bconst, cp_r, cp_part);
    k_cp_rule<<<1, 32, 0, st>>>(0, g, cp_part, tol, cp_st);
    launches += 2;
    CpState h{};
    CK(cudaMemcpyAsync(&h, cp_st, sizeof(CpState), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    *n_it = 0;
    if (h.stop) return 0;
    auto precond = [&]() -> int {
      if (identity_pc) {
        copy(cp_z, cp_r, nc);
        return 0;
      }
      int its = 0;
      int rc2 = cp_precond(&its);
      cp_precond_iters += its;
      return rc2;
    };
    rc = precond();
    if (rc) return rc;
    k_cp_dots<<<g, TPB, 0, st>>>(nc, 1, cp_r, cp_rold, cp_z, cp_p, cp_part);
    k_cp_rule<<<1, 32, 0, st>>>(1, g, cp_part, tol, cp_st);
    launches += 2;
    for (int it = 1; it <= max_it; ++it) {
      *n_it = it;
      k_cp_adjoint<<<nblk(nc), TPB, 0, st>>>(d, cp_p, cp_v);
      k_cp_div_dot<<<g, TPB, 0, st>>>(d, cp_v, cp_p, cp_q, cp_part);
      k_cp_rule<<<1, 32, 0, st>>>(2, g, cp_part, tol, cp_st);
      k_cp_update<<<g, TPB, 0, st>>>(nc, cp_st, cp_p, cp_q, cp_x, cp_r, cp_rold, cp_part);
      k_cp_rule<<<1, 32, 0, st>>>(3, g, cp_part, tol, cp_st);
      launches += 5;
      int stop = 0;
      CK(cudaMemcpyAsync(&stop, &cp_st->stop, sizeof(int), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      if (stop) break;
      rc = precond();
      if (rc) return rc;
      k_cp_dots<<<g, TPB, 0, st>>>(nc, 0, cp_r, cp_rold, cp_z, cp_p, cp_part);
      k_cp_rule<<<1, 32, 0, st>>>(4, g, cp_part, tol, cp_st);
      k_cp_direction<<<g, TPB, 0, st>>>(nc, cp_st, cp_z, cp_p);
      launches += 3;
    }
    k_cp_adjoint<<<nblk(nc), TPB, 0, st>>>(d, cp_x, cp_v);
    k_cp_apply<<<nblk(3 * (int64_t)nc), TPB, 0, st>>>(3 * nc, cp_v, u);
    launches += 2;
    CK(cudaGetLastError());
    return 0;
  }
  // project_cells_exact (mod_fv_solver.f90:3223-3283)
  int project_cells_exact(double dt) {
    int rc = cp_alloc();
    if (rc) return rc;
    k_cp_boundary<<<nblk(nc), TPB, 0, st>>>(d, dt, F.U, F.Ub, cp_bconst);
    launches++;
    int n_it = 0;
    rc = cp_project(F.U, cp_bconst, cp_tol(), 100, false, &n_it);
    cp_iters += n_it;
    return rc;
  }

  // ---------------------------------------------------------------- solver_project_once
  int project_once(double dt) {
    launch_fill(F.rhs, nc, 0.0);
    launch_fill(F.phi_prev, nc, 0.0);
    if (nb) launch_fill(F.phi_prev_b, nb, 0.0);
    launch_fill(F.gp_rc, 3 * (int64_t)nc, 0.0);
    refresh_halos_and_bc();
    face_fluxes_and_rhs(dt, false);
    if (P.p_max_iter > 0) {
      double atol;
      int rc = atol_dynamic(dt, atol);
      if (rc) return rc;
      int its;
      double res;
      rc = pressure_solve(P.p_tol, atol, true, &its, &res);
      if (rc) return rc;
    }
    anchor_pressure();
    correct_face_fluxes(dt, true);
    copy(F.ff, F.Uf, nf);
    u_face_ready = true;
    pressure_bc(F.p, -1, 0, 0);
    if (cp_on) {
      int rc = project_cells_exact(dt);
      if (rc) return rc;
    } else {
      correct_velocity(dt, true, true);
    }
    velocity_bc(-1, 0);
    if (P.use_rotational_projection) {
      k_rotational<<<nblk(nc), TPB, 0, st>>>(nc, F.p, F.nu_sgs, F.rhs, d.ivol, P.nu, dt);
      launches++;
      pressure_bc(F.p, -1, 0, 0);
    }
    copy(F.p_old, F.p, nc);
    copy(F.phi_prev, F.p, nc);
    copy(F.phi_prev_b, F.pb, nb);
    pressure_bc(F.p, -1, 0, 0);
    pressure_gradient();
    CK(cudaStreamSynchronize(st));
    CK(cudaGetLastError());
    return 0;
  }

  // ---------------------------------------------------------------- CFL (solver_compute_dt)
  int compute_dt(double& dt) {
    k_cfl_cell<<<nblk(nc), TPB, 0, st>>>(d, P.nu, u_face_ready, F.U, F.Uf, F.nu_sgs, scratch_c, scratch_c2);
    launches++;
    RedArgs r{};
    r.mode = RED_MAX2; r.n = nc; r.a = scratch_c; r.b = scratch_c2;
    double o[2];
    int rc = reduce(r, o, 2);
    if (rc) return rc;
    double dc = 1e308, dd = 1e308;
    if (o[0] > SMALL) dc = P.cfl_max / o[0];
    if (o[1] > SMALL) dd = 1.0 / o[1];
    dt = std::min(dc, dd);
    if (!(dt > 0.0)) dt = P.dt;
    dt = std::min(dt, P.dt);
    if (!(dt > 0.0)) dt = P.dt;
    else if (dt < 1.0e-6 * P.dt) return DPM_ERR_DT_COLLAPSE;
    return 0;
  }

  // ---------------------------------------------------------------- solver_advance
  int advance(double dt_in) {
    double dt = dt_in;
    if (!P.adapt_dt) {
      double ds;
      int rc = compute_dt(ds);
      if (rc) return rc;
      if (dt > ds) dt = ds;
    }
    if (P.constant_mass_flux_forcing) {
      int rc = update_mass_flux_forcing(dt);
      if (rc) return rc;
    }
    poisson_ms_acc = 0.0;
    cudaEventRecord(ev0, st);
    last.dt_used = dt;
    last.p_solves = 0; last.p_iters = 0; last.p_resid_max = 0.0;
    cp_iters = 0; cp_precond_iters = 0;
    launch_fill(F.H, 3 * (int64_t)nc, 0.0);
    launch_fill(F.H0, 3 * (int64_t)nc, 0.0);
    launch_fill(F.rhs, nc, 0.0);
    if (P.boussinesq || P.use_nudging) {
      launch_fill(HT, nc, 0.0);
      launch_fill(HT0, nc, 0.0);
    }
    if (ns > 0) {
      launch_fill(HC, (int64_t)ns * nc, 0.0);
      launch_fill(HC0, (int64_t)ns * nc, 0.0);
    }
    double time_n = time;
    for (int k = 0; k < 3; ++k) {
      double gk_dt = RK3W_GAMMA[k] * dt;
      time = time_n + RK3W_C[k] * dt;
      refresh_halos_and_bc();
      if (x32) {  // precision form: gradients, SGS and flux assembly in FP32
        grad_all32();
        sgs32(gk_dt);
        wall_model(k == 0 ? dt : 0.0);
        explicit_rhs32(dt, RK3W_ALPHA[k], RK3W_BETA[k]);
        scalars_rhs32(dt, RK3W_ALPHA[k], RK3W_BETA[k]);
      } else if (split_rhs()) {  // sources or nudging: assemble H, add them, then predict
        grad_all();
        sgs(gk_dt);
        wall_model(k == 0 ? dt : 0.0);
        explicit_rhs(dt, RK3W_ALPHA[k], RK3W_BETA[k], 0);
        if (!P.boussinesq) launch_fill(HT, nc, 0.0);
        scalars_rhs(dt, RK3W_ALPHA[k], RK3W_BETA[k], 0);
        add_sources_and_nudging();
        const double a_k = RK3W_ALPHA[k], b_k = RK3W_BETA[k];
        k_rk_predict<<<nblk(3 * (int64_t)nc), TPB, 0, st>>>(3 * (int64_t)nc, dt, a_k, b_k, F.H, F.H0, F.U);
        launches++;
        if (P.boussinesq || P.use_nudging) {
          k_rk_predict<<<nblk(nc), TPB, 0, st>>>(nc, dt, a_k, b_k, HT, HT0, F.T);
          launches++;
        }
        if (ns > 0) {
          k_rk_predict<<<nblk((int64_t)ns * nc), TPB, 0, st>>>((int64_t)ns * nc, dt, a_k, b_k, HC, HC0, Cs);
          launches++;
        }
      } else {
        grad_all();
        sgs(gk_dt);
        wall_model(k == 0 ? dt : 0.0);
        explicit_rhs(dt, RK3W_ALPHA[k], RK3W_BETA[k], 1);
        scalars_rhs(dt, RK3W_ALPHA[k], RK3W_BETA[k]);
      }
      if (sem_on) update_sem(true, (RK3W_C[k] + RK3W_GAMMA[k]) * dt);  // the stage's end (mod_fv_solver.f90:1350-1358)
      velocity_bc_refresh();
      copy(F.p_old, F.p, nc);
      if (cp_on) launch_fill(F.gpc, 3 * (int64_t)nc, 0.0);  // nothing to add back (mod_fv_solver.f90:1373-1377)
      else correct_velocity(gk_dt, false, true);
      copy(F.gp_rc, F.gpc, 3 * (size_t)nc);
      velocity_bc_refresh();
      grad_all();
      copy(F.phi_prev, F.p, nc);
      copy(F.phi_prev_b, F.pb, nb);
      double atol;
      int rc = atol_dynamic(gk_dt, atol);
      if (rc) return rc;
      int n_max;
      double stag;
      if (S.diag_interface) { n_max = std::min(S.n_nonortho_corr, 8); stag = 0.99; }
      else { n_max = std::min(S.n_nonortho_corr, 3); stag = 0.9; }
      if (P.nonortho_check) {
        n_max = std::min(S.n_nonortho_corr, 8);
        launch_fill(F.phi_it, nc, 0.0);
      }
      double dprev = 1e308, dphi_prev = 1e308;
      for (int jno = 1; jno <= n_max; ++jno) {
        face_fluxes_and_rhs(gk_dt, jno > 1);
        double dcur = 0.0;
        if (n_max > 1 && !P.nonortho_check) {
          RedArgs r{};
          r.mode = RED_MAXABS; r.n = nc; r.a = F.rhs;
          rc = reduce(r, &dcur, 1);
          if (rc) return rc;
        }
        if (jno == 1) launch_fill(F.p, nc, 0.0);
        int its;
        double res;
        rc = pressure_solve(P.p_tol, atol, false, &its, &res);
        if (rc) return rc;
        last.p_solves++;
        last.p_iters += its;
        last.p_resid_max = std::max(last.p_resid_max, res);
        pressure_bc(F.p, 0, !S.skip_grad_p, 1);
        pressure_bc(F.p, 1, 0, 0);
        if (P.nonortho_check) {
          // |p - phi_it|_max and |p|_max, then phi_it = p
          RedArgs r{};
          copy(scratch_c, F.p, nc);
          k_shift_vec(F.phi_it);
          r.mode = RED_MAXABS; r.n = nc; r.a = scratch_c;
          double dd;
          rc = reduce(r, &dd, 1);
          if (rc) return rc;
          r.a = F.p;
          double dpp;
          rc = reduce(r, &dpp, 1);
          if (rc) return rc;
          copy(F.phi_it, F.p, nc);
          if (jno > 1 && (dd < 1.0e-3 * dpp || dd > dphi_prev * stag)) break;
          dphi_prev = dd;
        } else if (jno > 1 && (dcur < atol || dcur > dprev * stag)) {
          break;
        }
        dprev = dcur;
      }
      correct_face_fluxes(gk_dt, false);
      copy(F.ff, F.Uf, nf);
      u_face_ready = true;
      if (cp_on) {
        rc = project_cells_exact(gk_dt);
        if (rc) return rc;
      } else {
        correct_velocity(gk_dt, true, false);
      }
      velocity_bc_refresh();
      if (P.use_rotational_projection) {
        k_rotational<<<nblk(nc), TPB, 0, st>>>(nc, F.p, F.nu_sgs, F.rhs, d.ivol, P.nu, gk_dt);
        launches++;
        pressure_bc(F.p, 0, !S.skip_grad_p, 1);
        pressure_bc(F.p, 1, 0, 0);
      }
      k_add<<<nblk(nc), TPB, 0, st>>>(nc, F.p, F.p_old);
      launches++;
      anchor_pressure();
      pressure_bc(F.p, 0, !S.skip_grad_p, 0);
      pressure_bc(F.p, 1, 0, 0);
      pressure_gradient();
      std::swap(F.H, F.H0);
      std::swap(HT, HT0);
      std::swap(HC, HC0);
    }
    if (sem_on) {  // sem_advance (mod_fv_solver.f90:1606-1610)
      k_sem_advance<<<1, 1, 0, st>>>(sem_d, dt);
      launches++;
    }
    scalar_bcs(-1);
    time = time_n + dt;
    step++;
    cudaEventRecord(ev1, st);
    CK(cudaEventSynchronize(ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    last_step_ms = ms;
    last_poisson_ms = poisson_ms_acc;
    CK(cudaGetLastError());
    return 0;
  }

  // scratch_c = scratch_c - v (used for the increment norm of nonortho_check)
  void k_shift_vec(const double* v) {
    k_sub<<<nblk(nc), TPB, 0, st>>>(nc, scratch_c, v);
    launches++;
  }

  // ---------------------------------------------------------------- statistics
  int stats(dpm_stats_t* s) {
    RedArgs r{};
    r.mode = RED_STATS; r.n = nc; r.a = F.U; r.vol = d.vol; r.gU = F.gU; r.nus = F.nu_sgs; r.nu = P.nu;
    double o[RED_NV];
    int rc = reduce(r, o, RED_NV);
    if (rc) return rc;
    s->time = time;
    s->E = o[0] / o[1];
    s->eps = 2.0 * o[2] / o[1];
    double mb0 = o[3] / o[1], mb1 = o[4] / o[1], mb2 = o[5] / o[1];
    s->Ub = std::sqrt(mb0 * mb0 + mb1 * mb1 + mb2 * mb2);
    s->nu_sgs_mean = o[6] / o[1];
    s->Umax = o[7];
    // wall shear (host: small)
    s->tauw_mean = 0.0;
    if (nb) {
      std::vector<double> tau(3 * (size_t)nb);
      CK(cudaMemcpyAsync(tau.data(), F.tau, tau.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      double num = 0.0, den = 0.0;
      for (int q = 0; q < m.n_patches; ++q) {
        if (pc[q].bc_id != BC_WALL_MODEL) continue;
        for (int64_t k = 0; k < m.patch_nfaces[q]; ++k) {
          int64_t b = m.patch_start[q] + k;
          double t0 = tau[b], t1 = tau[nb + b], t2 = tau[2 * (size_t)nb + b];
          num += std::sqrt(t0 * t0 + t1 * t1 + t2 * t2) * m.area[m.n_int_faces + b];
          den += m.area[m.n_int_faces + b];
        }
      }
      s->tauw_mean = den > SMALL ? num / den : 0.0;
    }
    k_flux_divergence<<<nblk(nc), TPB, 0, st>>>(d, F.Uf, scratch_c);
    launches++;
    RedArgs r2{};
    r2.mode = RED_DIVSTAT; r2.n = nc; r2.a = scratch_c; r2.vol = d.vol;
    double o2[3];
    rc = reduce(r2, o2, 3);
    if (rc) return rc;
    s->max_abs_divU = o2[0];
    s->volavg_abs_divU = o2[1] / o2[2];
    s->dt_used = last.dt_used;
    s->p_fallbacks = p_fallbacks;
    s->cp_iters = cp_iters;
    s->cp_precond_iters = cp_precond_iters;
    s->p_solver_used = force_plain ? DPM_PSOLVER_JACOBI_PCG
                                   : (use_fcg ? DPM_PSOLVER_TWOLEVEL_FCG
                                              : (use_ml ? DPM_PSOLVER_MULTILEVEL_FCG : DPM_PSOLVER_JACOBI_PCG));
    // algorithmic bytes per Krylov iteration: Jacobi-PCG phase A (row of A, z gathered, p old /
    // new, q) and phase B (x, p, r, q, 1/diag in; x, r, z out); two-level FCG w = A z (row of A, z
    // gathered and written, deflation row data: the smoother runs in shared memory and registers);
    // multilevel from its hierarchy
    {
      const double n = nc, wa = S.WA;
      if (s->p_solver_used == DPM_PSOLVER_MULTILEVEL_FCG) s->p_bytes_per_iteration = ml.bytes_per_iteration;
      else if (s->p_solver_used == DPM_PSOLVER_TWOLEVEL_FCG) s->p_bytes_per_iteration = n * (wa * 12.0 + 24.0);
      else s->p_bytes_per_iteration = n * (wa * 12.0 + 32.0) + n * 64.0;
    }
    s->p_solves = last.p_solves;
    s->p_iters = last.p_iters;
    s->p_resid_max = last.p_resid_max;
    velocity_bc(-1, 0);  // solver_divergence_metrics refreshes U_bnd without gradients
    k_cell_velocity_divergence<<<nblk(nc), TPB, 0, st>>>(d, F.U, F.Ub, scratch_c);
    launches++;
    rc = reduce(r2, o2, 3);
    if (rc) return rc;
    s->max_abs_divU_cell = o2[0];
    s->volavg_abs_divU_cell = o2[1] / o2[2];
    CK(cudaStreamSynchronize(st));
    return 0;
  }
};

}  // namespace gpu
}  // namespace dpm

using dpm::gpu::Solver;
struct dpm_solver {
  std::unique_ptr<Solver> s;
};

// ------------------------------------------------------------------------------------------
extern "C" {

int dpm_create(const dpm_raw_mesh_t* mesh, const dpm_patch_cfg_t* patches, const dpm_params_t* params, int device,
               dpm_solver_t** out) {
  if (!mesh || !patches || !params || !out) return DPM_ERR_ARG;
  auto* h = new dpm_solver();
  h->s = std::make_unique<Solver>();
  int rc = h->s->init(mesh, patches, params, device);
  if (rc) {
    delete h;
    *out = nullptr;
    return rc;
  }
  *out = h;
  return DPM_OK;
}

int dpm_create_poly(const dpm_poly_mesh_t* mesh, const dpm_patch_cfg_t* patches, const dpm_params_t* params,
                    int device, dpm_solver_t** out) {
  if (!mesh || !patches || !params || !out) return DPM_ERR_ARG;
  auto* h = new dpm_solver();
  h->s = std::make_unique<Solver>();
  int rc = h->s->init_poly(mesh, patches, params, device);
  if (rc) {
    delete h;
    *out = nullptr;
    return rc;
  }
  *out = h;
  return DPM_OK;
}

int dpm_destroy(dpm_solver_t* s) {
  if (!s) return DPM_ERR_ARG;
  cudaSetDevice(s->s->device);
  delete s;
  return DPM_OK;
}

int dpm_n_cells(const dpm_solver_t* s, int64_t* n_cells, int64_t* n_faces, int64_t* n_bnd_faces) {
  if (!s) return DPM_ERR_ARG;
  if (n_cells) *n_cells = s->s->nc;
  if (n_faces) *n_faces = s->s->nf;
  if (n_bnd_faces) *n_bnd_faces = s->s->nb;
  return DPM_OK;
}

int dpm_cell_geometry(const dpm_solver_t* s, double* centroid, double* volume) {
  if (!s) return DPM_ERR_ARG;
  const auto& m = s->s->m;
  if (centroid) std::memcpy(centroid, m.centroid.data(), sizeof(double) * 3 * m.n_cells);
  if (volume) std::memcpy(volume, m.volume.data(), sizeof(double) * m.n_cells);
  return DPM_OK;
}

int dpm_upload_state(dpm_solver_t* h, const double* U, const double* p, const double* T) {
  if (!h) return DPM_ERR_ARG;
  Solver& s = *h->s;
  CK(cudaSetDevice(s.device));
  if (U) {
    CK(cudaMemcpyAsync(s.aos_buf, U, 3 * sizeof(double) * s.nc, cudaMemcpyHostToDevice, s.st));
    dpm::gpu::k_aos_to_soa<<<dpm::gpu::nblk(s.nc), dpm::gpu::TPB, 0, s.st>>>(s.nc, s.aos_buf, s.F.U);
    s.launches++;
  }
  if (p) CK(cudaMemcpyAsync(s.F.p, p, sizeof(double) * s.nc, cudaMemcpyHostToDevice, s.st));
  if (T) CK(cudaMemcpyAsync(s.F.T, T, sizeof(double) * s.nc, cudaMemcpyHostToDevice, s.st));
  CK(cudaStreamSynchronize(s.st));
  return DPM_OK;
}

int dpm_download_state(dpm_solver_t* h, double* U, double* p, double* T, double* nu_sgs) {
  if (!h) return DPM_ERR_ARG;
  Solver& s = *h->s;
  CK(cudaSetDevice(s.device));
  if (U) {
    dpm::gpu::k_soa_to_aos<<<dpm::gpu::nblk(s.nc), dpm::gpu::TPB, 0, s.st>>>(s.nc, s.F.U, s.aos_buf);
    s.launches++;
    CK(cudaMemcpyAsync(U, s.aos_buf, 3 * sizeof(double) * s.nc, cudaMemcpyDeviceToHost, s.st));
  }
  if (p) CK(cudaMemcpyAsync(p, s.F.p, sizeof(double) * s.nc, cudaMemcpyDeviceToHost, s.st));
  if (T) CK(cudaMemcpyAsync(T, s.F.T, sizeof(double) * s.nc, cudaMemcpyDeviceToHost, s.st));
  if (nu_sgs) CK(cudaMemcpyAsync(nu_sgs, s.F.nu_sgs, sizeof(double) * s.nc, cudaMemcpyDeviceToHost, s.st));
  CK(cudaStreamSynchronize(s.st));
  return DPM_OK;
}

int dpm_learn_collect(dpm_solver_t* h, int n_steps, int* n_samples) {
  if (!h || n_steps < 1) return DPM_ERR_ARG;
  CK(cudaSetDevice(h->s->device));
  return h->s->learn_collect(n_steps, n_samples);
}

int dpm_learn_train(dpm_solver_t* h, int epochs, double lr, dpm_learn_report_t* report) {
  if (!h || epochs < 0 || !(lr > 0.0)) return DPM_ERR_ARG;
  CK(cudaSetDevice(h->s->device));
  return h->s->learn_train(epochs, lr, report);
}

int dpm_learn_set_gamma(dpm_solver_t* h, double gamma) {
  if (!h || !(gamma >= 0.0)) return DPM_ERR_ARG;
  Solver& s = *h->s;
  if (!s.use_fcg && !(s.use_ml && s.ml_learn_ready)) return DPM_ERR_UNSUPPORTED;
  s.lp_gamma = (float)gamma;
  s.lp_ready = true;
  return DPM_OK;
}

int dpm_multilevel_hierarchy(int n, int width, const int* col, const double* val, int nullsp, int passes,
                             int* sizes, long long* nnz, int max_levels) {
  if (n < 1 || width < 1 || !col || !val || !sizes || max_levels < 1) return DPM_ERR_ARG;
  dpm::Multilevel M;
  int rc = dpm::build_multilevel(n, width, col, val, nullsp != 0, passes > 0 ? passes : 3, 0.25, 300, 1024, M);
  if (rc) return rc;
  const int L = std::min<int>((int)M.sizes.size(), max_levels);
  for (int l = 0; l < L; ++l) {
    sizes[l] = M.sizes[l];
    if (nnz) nnz[l] = (long long)M.nnz[l];
  }
  return (int)M.sizes.size();
}

int dpm_multilevel_digest(int n, int width, const int* col, const double* val, int nullsp, int passes,
                          unsigned long long* digest) {
  if (n < 1 || width < 1 || !col || !val || !digest) return DPM_ERR_ARG;
  dpm::Multilevel M;
  int rc = dpm::build_multilevel(n, width, col, val, nullsp != 0, passes > 0 ? passes : 3, 0.25, 300, 1024, M);
  if (rc) return rc;
  // 64-bit FNV-1a over every array of every level, each preceded by its element count
  uint64_t h = 1469598103934665603ull;
  auto mix = [&](const void* p, size_t bytes) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < bytes; ++i) { h ^= b[i]; h *= 1099511628211ull; }
  };
  auto vec = [&](const auto& v) {
    const int64_t k = (int64_t)v.size();
    mix(&k, sizeof(k));
    if (k) mix(v.data(), v.size() * sizeof(v[0]));
  };
  for (const dpm::MlLevel& L : M.lv) {
    const int hdr[4] = {L.n, L.W, L.M, L.Wo};
    mix(hdr, sizeof(hdr));
    vec(L.dinv); vec(L.ocol); vec(L.sv32); vec(L.sv16); vec(L.g32); vec(L.g16); vec(L.diag); vec(L.agg);
    vec(L.mem);
    mix(&L.lmax, sizeof(L.lmax));
  }
  mix(&M.nC, sizeof(M.nC));
  vec(M.cinv); vec(M.sizes); vec(M.nnz);
  *digest = (unsigned long long)h;
  return (int)M.sizes.size();
}

int dpm_learn_sizes(dpm_solver_t* h, int* sizes) {
  if (!h || !sizes) return DPM_ERR_ARG;
  Solver& s = *h->s;
  if (!s.use_fcg && !(s.use_ml && s.ml_learn_ready)) return DPM_ERR_UNSUPPORTED;
  sizes[0] = s.nc; sizes[1] = s.fa.C; sizes[2] = s.fa.WL; sizes[3] = s.fcg_WA;
  sizes[4] = s.lp_train_slots(); sizes[5] = dpm::gpu::LP_F; sizes[6] = dpm::gpu::LP_NP;
  return DPM_OK;
}

int dpm_learn_export(dpm_solver_t* h, float* feat, unsigned* lpk, int* col, double* val, double* R, double* Z,
                     double* U, double* E, float* params) {
  if (!h) return DPM_ERR_ARG;
  Solver& s = *h->s;
  if (!s.use_fcg && !(s.use_ml && s.ml_learn_ready)) return DPM_ERR_UNSUPPORTED;
  CK(cudaSetDevice(s.device));
  const size_t n = s.nc, S = s.lp_train_slots();
  auto cp = [&](void* dst, const void* src, size_t bytes) -> int {
    if (dst && src && bytes) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s.st));
    return 0;
  };
  cp(feat, s.lp_feat, sizeof(float) * dpm::gpu::LP_F * n);
  cp(lpk, s.fa.lpk, sizeof(unsigned) * s.fa.WL * n);
  cp(col, s.fa.col, sizeof(int) * s.fcg_WA * n);
  cp(val, s.fa.val, sizeof(double) * s.fcg_WA * n);
  cp(R, s.lp_r, sizeof(double) * S * n);
  cp(Z, s.lp_z, sizeof(double) * S * n);
  cp(U, s.lp_u, sizeof(double) * S * n);
  cp(E, s.lp_x, sizeof(double) * S * n);
  cp(params, s.lp_prm, sizeof(float) * dpm::gpu::LP_NP);
  CK(cudaStreamSynchronize(s.st));
  return DPM_OK;
}

int dpm_learn_loss_grad(dpm_solver_t* h, const float* params, double* loss, float* grad) {
  if (!h || !loss) return DPM_ERR_ARG;
  Solver& s = *h->s;
  if ((!s.use_fcg && !s.use_ml) || s.lp_count == 0) return DPM_ERR_ARG;
  CK(cudaSetDevice(s.device));
  const int S = s.lp_train_slots();
  std::vector<float> keep(dpm::gpu::LP_NP);
  CK(cudaMemcpyAsync(keep.data(), s.lp_prm, sizeof(float) * keep.size(), cudaMemcpyDeviceToHost, s.st));
  if (params) {
    CK(cudaMemcpyAsync(s.lp_prm, params, sizeof(float) * dpm::gpu::LP_NP, cudaMemcpyHostToDevice, s.st));
    dpm::gpu::k_lp_round<<<(dpm::gpu::LP_NP + 255) / 256, 256, 0, s.st>>>(dpm::gpu::LP_NP, s.lp_prm, s.lp_wb);
  }
  std::vector<double> base;
  int rc = s.lp_prepare(S, base);
  if (!rc) rc = s.lp_loss_grad(S, base, loss, grad != nullptr);
  if (!rc && grad) CK(cudaMemcpyAsync(grad, s.lp_grad, sizeof(float) * dpm::gpu::LP_NP, cudaMemcpyDeviceToHost, s.st));
  if (params) {  // leave the trained parameters as they were
    CK(cudaMemcpyAsync(s.lp_prm, keep.data(), sizeof(float) * keep.size(), cudaMemcpyHostToDevice, s.st));
    dpm::gpu::k_lp_round<<<(dpm::gpu::LP_NP + 255) / 256, 256, 0, s.st>>>(dpm::gpu::LP_NP, s.lp_prm, s.lp_wb);
    s.lp_forward();
  }
  CK(cudaStreamSynchronize(s.st));
  return rc;
}

int dpm_upload_scalars(dpm_solver_t* h, const double* C) {
  if (!h || !C) return DPM_ERR_ARG;
  Solver& s = *h->s;
  if (s.ns == 0) return DPM_OK;
  CK(cudaSetDevice(s.device));
  if (s.ns == 1) {  // C(1, n) is already one contiguous field
    CK(cudaMemcpyAsync(s.Cs, C, sizeof(double) * s.nc, cudaMemcpyHostToDevice, s.st));
  } else {  // C(ns, n), scalar index fastest: transposed on the device (aos_buf holds >= 9 n)
    CK(cudaMemcpyAsync(s.aos_buf, C, sizeof(double) * s.ns * s.nc, cudaMemcpyHostToDevice, s.st));
    dpm::gpu::k_aos_to_soa_k<<<dpm::gpu::nblk(s.nc), dpm::gpu::TPB, 0, s.st>>>(s.nc, s.ns, s.aos_buf, s.Cs);
    s.launches++;
  }
  CK(cudaStreamSynchronize(s.st));
  return DPM_OK;
}

int dpm_download_scalars(dpm_solver_t* h, double* C) {
  if (!h || !C) return DPM_ERR_ARG;
  Solver& s = *h->s;
  if (s.ns == 0) return DPM_OK;
  CK(cudaSetDevice(s.device));
  if (s.ns == 1) {
    CK(cudaMemcpyAsync(C, s.Cs, sizeof(double) * s.nc, cudaMemcpyDeviceToHost, s.st));
  } else {
    dpm::gpu::k_soa_to_aos_k<<<dpm::gpu::nblk(s.nc), dpm::gpu::TPB, 0, s.st>>>(s.nc, s.ns, s.Cs, s.aos_buf);
    s.launches++;
    CK(cudaMemcpyAsync(C, s.aos_buf, sizeof(double) * s.ns * s.nc, cudaMemcpyDeviceToHost, s.st));
  }
  CK(cudaStreamSynchronize(s.st));
  return DPM_OK;
}

int dpm_download_face_flux(dpm_solver_t* h, double* face_flux) {
  if (!h || !face_flux) return DPM_ERR_ARG;
  Solver& s = *h->s;
  CK(cudaMemcpyAsync(face_flux, s.F.Uf, sizeof(double) * s.nf, cudaMemcpyDeviceToHost, s.st));
  CK(cudaStreamSynchronize(s.st));
  return DPM_OK;
}

int dpm_download_gradient(dpm_solver_t* h, double* grad_U) {
  if (!h || !grad_U) return DPM_ERR_ARG;
  Solver& s = *h->s;
  dpm::gpu::k_grad_soa_to_aos<<<dpm::gpu::nblk(s.nc), dpm::gpu::TPB, 0, s.st>>>(s.nc, s.F.gU, s.aos_buf);
  s.launches++;
  CK(cudaMemcpyAsync(grad_U, s.aos_buf, 9 * sizeof(double) * s.nc, cudaMemcpyDeviceToHost, s.st));
  CK(cudaStreamSynchronize(s.st));
  return DPM_OK;
}

int dpm_project_once(dpm_solver_t* h, double dt) {
  if (!h) return DPM_ERR_ARG;
  CK(cudaSetDevice(h->s->device));
  return h->s->project_once(dt);
}

int dpm_advance(dpm_solver_t* h, double dt) {
  if (!h) return DPM_ERR_ARG;
  CK(cudaSetDevice(h->s->device));
  return h->s->advance(dt);
}

int dpm_advance_n(dpm_solver_t* h, double dt, int n_steps) {
  if (!h || n_steps < 0) return DPM_ERR_ARG;
  CK(cudaSetDevice(h->s->device));
  for (int i = 0; i < n_steps; ++i) {
    int rc = h->s->advance(dt);
    if (rc) return rc;
  }
  return DPM_OK;
}

int dpm_stats(dpm_solver_t* h, dpm_stats_t* out) {
  if (!h || !out) return DPM_ERR_ARG;
  CK(cudaSetDevice(h->s->device));
  return h->s->stats(out);
}

int dpm_state_is_finite(dpm_solver_t* h, int* ok) {
  if (!h || !ok) return DPM_ERR_ARG;
  Solver& s = *h->s;
  dpm::gpu::RedArgs r{};
  r.mode = dpm::gpu::RED_SUM2;
  r.n = 3 * s.nc;
  r.a = s.F.U;
  r.b = s.F.U;
  double o[2];
  int rc = s.reduce(r, o, 2);
  if (rc) return rc;
  r.n = s.nc; r.a = s.F.p; r.b = s.F.p;
  double o2[2];
  rc = s.reduce(r, o2, 2);
  if (rc) return rc;
  double t = o[1] + o2[1];
  *ok = std::fabs(t) <= 1.7976931348623157e308 ? 1 : 0;
  return DPM_OK;
}

int dpm_compute_dt(dpm_solver_t* h, double* dt) {
  if (!h || !dt) return DPM_ERR_ARG;
  return h->s->compute_dt(*dt);
}

int dpm_get_time(const dpm_solver_t* h, double* time) {
  if (!h || !time) return DPM_ERR_ARG;
  *time = h->s->time;
  return DPM_OK;
}

int dpm_set_time(dpm_solver_t* h, double time) {
  if (!h) return DPM_ERR_ARG;
  h->s->time = time;
  return DPM_OK;
}

int dpm_last_timing(const dpm_solver_t* h, double* step_ms, double* poisson_ms) {
  if (!h) return DPM_ERR_ARG;
  if (step_ms) *step_ms = h->s->last_step_ms;
  if (poisson_ms) *poisson_ms = h->s->last_poisson_ms;
  return DPM_OK;
}

int dpm_kernel_launches(const dpm_solver_t* h, int64_t* n) {
  if (!h || !n) return DPM_ERR_ARG;
  *n = h->s->launches;
  return DPM_OK;
}

int dpm_fcg_phase_times(dpm_solver_t* h, int enable, double* us) {
  if (!h) return DPM_ERR_ARG;
  Solver& s = *h->s;
  CK(cudaSetDevice(s.device));
  if (us) {
    double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (s.fcg_phase) {
      CK(cudaStreamSynchronize(s.st));
      CK(cudaMemcpy(v, s.fcg_phase, sizeof(v), cudaMemcpyDeviceToHost));
    }
    const double n = v[7] > 0.0 ? v[7] : 1.0;
    for (int k = 0; k < 6; ++k) us[k] = v[k] / n * 1e-3;
    us[6] = 0.0;
    us[7] = v[7];
  }
  if (enable) {
    if (!s.fcg_phase) {
      s.fcg_phase = s.mem.alloc<double>(8);
      if (!s.fcg_phase) return DPM_ERR_CUDA;
    }
    CK(cudaMemsetAsync(s.fcg_phase, 0, 8 * sizeof(double), s.st));
  } else {
    s.fcg_phase = nullptr;  // the buffer stays with the handle's allocations
  }
  return DPM_OK;
}

int dpm_setup_times(const dpm_solver_t* h, double* ms) {
  if (!h || !ms) return DPM_ERR_ARG;
  const Solver& s = *h->s;
  ms[0] = s.setup_t.mesh_ms;
  ms[1] = s.setup_t.ops_ms;
  ms[2] = s.setup_upload_ms;
  ms[3] = s.setup_total_ms;
  for (int k = 0; k < 7; ++k) ms[4 + k] = s.setup_t.stage_ms[k];
  ms[11] = s.setup_psolver_ms;
  return DPM_OK;
}

int dpm_select_pressure_solver(dpm_solver_t* h, int p_solver) {
  if (!h) return DPM_ERR_ARG;
  Solver& s = *h->s;
  if (p_solver == DPM_PSOLVER_JACOBI_PCG) { s.force_plain = true; return DPM_OK; }
  const bool ok = (p_solver == DPM_PSOLVER_TWOLEVEL_FCG && s.use_fcg) ||
                  (p_solver == DPM_PSOLVER_MULTILEVEL_FCG && s.use_ml) ||
                  (p_solver == DPM_PSOLVER_AUTO && (s.use_fcg || s.use_ml));
  if (!ok) return DPM_ERR_UNSUPPORTED;
  s.force_plain = false;
  return DPM_OK;
}

int dpm_set_barrier_spin_limit(dpm_solver_t* h, long long spins) {
  if (!h || spins < 0 || spins > 0x7fffffffLL) return DPM_ERR_ARG;
  h->s->spin_limit = (int)spins;
  h->s->ml.spin_limit_override = (int)spins;
  return DPM_OK;
}

// ---- per-operator entry points --------------------------------------------------------------
static int upload_vec3(Solver& s, const double* host_aos, double* dev_soa, int n) {
  CK(cudaMemcpyAsync(s.aos_buf, host_aos, 3 * sizeof(double) * n, cudaMemcpyHostToDevice, s.st));
  dpm::gpu::k_aos_to_soa<<<dpm::gpu::nblk(n), dpm::gpu::TPB, 0, s.st>>>(n, s.aos_buf, dev_soa);
  s.launches++;
  CK(cudaStreamSynchronize(s.st));
  return 0;
}
static int download_vec3(Solver& s, const double* dev_soa, double* host_aos, int n) {
  dpm::gpu::k_soa_to_aos<<<dpm::gpu::nblk(n), dpm::gpu::TPB, 0, s.st>>>(n, dev_soa, s.aos_buf);
  s.launches++;
  CK(cudaMemcpyAsync(host_aos, s.aos_buf, 3 * sizeof(double) * n, cudaMemcpyDeviceToHost, s.st));
  CK(cudaStreamSynchronize(s.st));
  return 0;
}
static int upload_grad(Solver& s, const double* host_aos) {
  CK(cudaMemcpyAsync(s.aos_buf, host_aos, 9 * sizeof(double) * s.nc, cudaMemcpyHostToDevice, s.st));
  dpm::gpu::k_grad_aos_to_soa<<<dpm::gpu::nblk(s.nc), dpm::gpu::TPB, 0, s.st>>>(s.nc, s.aos_buf, s.F.gU);
  s.launches++;
  CK(cudaStreamSynchronize(s.st));
  return 0;
}

int dpm_ls_gradient_vector(dpm_solver_t* h, const double* U, const double* U_bnd, double* grad_U) {
  if (!h || !U || !U_bnd || !grad_U) return DPM_ERR_ARG;
  Solver& s = *h->s;
  int rc = upload_vec3(s, U, s.F.U, s.nc);
  if (!rc && s.nb) rc = upload_vec3(s, U_bnd, s.F.Ub, s.nb);
  if (rc) return rc;
  s.grad_U();
  return dpm_download_gradient(h, grad_U);
}

int dpm_advection_rhs_vector(dpm_solver_t* h, int scheme, const double* U, const double* U_bnd,
                             const double* face_flux, const double* grad_U, double* rhs) {
  if (!h || !U || !U_bnd || !face_flux || !grad_U || !rhs) return DPM_ERR_ARG;
  Solver& s = *h->s;
  int rc = upload_vec3(s, U, s.F.U, s.nc);
  if (!rc && s.nb) rc = upload_vec3(s, U_bnd, s.F.Ub, s.nb);
  if (!rc) rc = upload_grad(s, grad_U);
  if (rc) return rc;
  CK(cudaMemcpyAsync(s.F.Uf, face_flux, sizeof(double) * s.nf, cudaMemcpyHostToDevice, s.st));
  int keep = s.P.scheme;
  double keep_nu = s.P.nu;
  s.P.scheme = scheme;
  // advection only: zero viscosity, zero SGS, zero body force -> H = conv
  s.launch_fill(s.F.nu_sgs, s.nc, 0.0);
  s.P.nu = 0.0;
  dpm::gpu::k_face_explicit<<<dpm::gpu::nblk(s.nf), dpm::gpu::TPB, 0, s.st>>>(
      s.d, scheme, 0.0, s.F.U, s.F.Ub, s.F.gU, s.F.nu_sgs, s.F.Uf, s.F.fadv, s.F.fvis, s.F.fdiv);
  dpm::gpu::ExplicitArgs a{};
  a.scheme = scheme;
  dpm::gpu::k_cell_explicit<<<dpm::gpu::nblk(s.nc), dpm::gpu::TPB, 0, s.st>>>(
      s.d, a, s.F.U, s.F.T, s.F.fadv, s.F.fvis, s.F.fdiv, s.F.tau, s.F.H, s.F.H0, s.conv_tmp, s.visc_tmp);
  s.launches += 2;
  s.P.scheme = keep;
  s.P.nu = keep_nu;
  return download_vec3(s, s.conv_tmp, rhs, s.nc);
}

// Scalar operators on caller data: phi [n], phi_bnd [n_bnd], grad_phi (3, n) Fortran layout.
static int scalar_operator(Solver& s, int scheme, const double* phi, const double* phi_bnd, const double* face_flux,
                           const double* grad_phi, const double* nu_sgs, double alpha, double prt, double* conv,
                           double* dif) {
  CK(cudaSetDevice(s.device));
  double* ph = s.scratch_c;
  CK(cudaMemcpyAsync(ph, phi, sizeof(double) * s.nc, cudaMemcpyHostToDevice, s.st));
  if (s.nb) CK(cudaMemcpyAsync(s.Tb, phi_bnd, sizeof(double) * s.nb, cudaMemcpyHostToDevice, s.st));
  CK(cudaMemcpyAsync(s.aos_buf, grad_phi, 3 * sizeof(double) * s.nc, cudaMemcpyHostToDevice, s.st));
  dpm::gpu::k_aos_to_soa<<<dpm::gpu::nblk(s.nc), dpm::gpu::TPB, 0, s.st>>>(s.nc, s.aos_buf, s.gT);
  if (face_flux) CK(cudaMemcpyAsync(s.F.Uf, face_flux, sizeof(double) * s.nf, cudaMemcpyHostToDevice, s.st));
  else s.launch_fill(s.F.Uf, s.nf, 0.0);
  if (nu_sgs) CK(cudaMemcpyAsync(s.F.nu_sgs, nu_sgs, sizeof(double) * s.nc, cudaMemcpyHostToDevice, s.st));
  else s.launch_fill(s.F.nu_sgs, s.nc, 0.0);
  s.scalar_transport(scheme, ph, s.Tb, s.gT, alpha, prt, s.HT, s.HT0, 0.0, 0.0, 0.0, 0, s.conv_tmp, s.visc_tmp);
  s.launches++;
  if (conv) CK(cudaMemcpyAsync(conv, s.conv_tmp, sizeof(double) * s.nc, cudaMemcpyDeviceToHost, s.st));
  if (dif) CK(cudaMemcpyAsync(dif, s.visc_tmp, sizeof(double) * s.nc, cudaMemcpyDeviceToHost, s.st));
  CK(cudaStreamSynchronize(s.st));
  return DPM_OK;
}

int dpm_advection_rhs_scalar(dpm_solver_t* h, int scheme, const double* phi, const double* phi_bnd,
                             const double* face_flux, const double* grad_phi, double* rhs) {
  if (!h || !phi || !phi_bnd || !face_flux || !grad_phi || !rhs) return DPM_ERR_ARG;
  if (scheme != DPM_SCHEME_CDS && scheme != DPM_SCHEME_QUICK && scheme != DPM_SCHEME_VANLEER_TVD &&
      scheme != DPM_SCHEME_KOREN_TVD)
    return DPM_ERR_UNSUPPORTED;
  return scalar_operator(*h->s, scheme, phi, phi_bnd, face_flux, grad_phi, nullptr, 0.0, 1.0, rhs, nullptr);
}

int dpm_viscous_rhs_scalar(dpm_solver_t* h, const double* phi, double alpha, const double* nu_sgs, double Pr_t,
                           const double* grad_phi, const double* phi_bnd, double* rhs) {
  if (!h || !phi || !nu_sgs || !grad_phi || !phi_bnd || !rhs || !(Pr_t > 0.0)) return DPM_ERR_ARG;
  return scalar_operator(*h->s, DPM_SCHEME_CDS, phi, phi_bnd, nullptr, grad_phi, nu_sgs, alpha, Pr_t, nullptr, rhs);
}

int dpm_viscous_rhs_vector(dpm_solver_t* h, const double* U, double nu, const double* nu_sgs, const double* grad_U,
                           const double* U_bnd, double* rhs) {
  if (!h || !U || !nu_sgs || !grad_U || !U_bnd || !rhs) return DPM_ERR_ARG;
  Solver& s = *h->s;
  int rc = upload_vec3(s, U, s.F.U, s.nc);
  if (!rc && s.nb) rc = upload_vec3(s, U_bnd, s.F.Ub, s.nb);
  if (!rc) rc = upload_grad(s, grad_U);
  if (rc) return rc;
  CK(cudaMemcpyAsync(s.F.nu_sgs, nu_sgs, sizeof(double) * s.nc, cudaMemcpyHostToDevice, s.st));
  s.launch_fill(s.F.Uf, s.nf, 0.0);
  dpm::gpu::k_face_explicit<<<dpm::gpu::nblk(s.nf), dpm::gpu::TPB, 0, s.st>>>(
      s.d, DPM_SCHEME_CDS, nu, s.F.U, s.F.Ub, s.F.gU, s.F.nu_sgs, s.F.Uf, s.F.fadv, s.F.fvis, s.F.fdiv);
  dpm::gpu::ExplicitArgs a{};
  a.scheme = DPM_SCHEME_CDS;
  dpm::gpu::k_cell_explicit<<<dpm::gpu::nblk(s.nc), dpm::gpu::TPB, 0, s.st>>>(
      s.d, a, s.F.U, s.F.T, s.F.fadv, s.F.fvis, s.F.fdiv, s.F.tau, s.F.H, s.F.H0, s.conv_tmp, s.visc_tmp);
  s.launches += 2;
  return download_vec3(s, s.visc_tmp, rhs, s.nc);
}

int dpm_sgs_viscosity(dpm_solver_t* h, int model, const double* U, const double* U_bnd, const double* grad_U,
                      double dt_stab, double* nu_sgs) {
  if (!h || !U || !grad_U || !nu_sgs) return DPM_ERR_ARG;
  (void)U_bnd;
  Solver& s = *h->s;
  int rc = upload_vec3(s, U, s.F.U, s.nc);
  if (!rc) rc = upload_grad(s, grad_U);
  if (rc) return rc;
  int keep = s.P.sgs_model;
  s.P.sgs_model = model;
  s.sgs(dt_stab);
  s.P.sgs_model = keep;
  CK(cudaMemcpyAsync(nu_sgs, s.F.nu_sgs, sizeof(double) * s.nc, cudaMemcpyDeviceToHost, s.st));
  CK(cudaStreamSynchronize(s.st));
  return DPM_OK;
}

int dpm_wall_model(dpm_solver_t* h, const double* U, double nu, double* tau_w) {
  if (!h || !U || !tau_w) return DPM_ERR_ARG;
  Solver& s = *h->s;
  int rc = upload_vec3(s, U, s.F.U, s.nc);
  if (rc) return rc;
  double keep = s.P.nu;
  s.P.nu = nu;
  s.wall_model(0.0);
  s.P.nu = keep;
  if (s.nb) return download_vec3(s, s.F.tau, tau_w, s.nb);
  return DPM_OK;
}

int dpm_write_checkpoint(dpm_solver_t* h, const char* checkpoint_dir, int step) {
  if (!h || !checkpoint_dir || step < 0) return DPM_ERR_ARG;
  CK(cudaSetDevice(h->s->device));
  return h->s->write_checkpoint(checkpoint_dir, step);
}

int dpm_read_checkpoint(dpm_solver_t* h, const char* checkpoint_dir, int step) {
  if (!h || !checkpoint_dir) return DPM_ERR_ARG;
  CK(cudaSetDevice(h->s->device));
  return h->s->read_checkpoint(checkpoint_dir, step);
}

int dpm_sampling_set_points(dpm_solver_t* h, int n_points, const double* xyz, int* owner_cell) {
  if (!h || n_points < 0 || (n_points > 0 && !xyz)) return DPM_ERR_ARG;
  CK(cudaSetDevice(h->s->device));
  return h->s->set_sample_points(n_points, xyz, owner_cell);
}

int dpm_sample_points(dpm_solver_t* h, double* payload) {
  if (!h || !payload) return DPM_ERR_ARG;
  CK(cudaSetDevice(h->s->device));
  return h->s->sample_points(payload);
}

int dpm_set_nudging_profiles(dpm_solver_t* h, int n_times, int n_levels, const double* times, const double* z_levels,
                             const double* U_profile, const double* T_profile) {
  if (!h) return DPM_ERR_ARG;
  CK(cudaSetDevice(h->s->device));
  return h->s->set_nudging(n_times, n_levels, times, z_levels, U_profile, T_profile);
}

int dpm_set_scalar_sources(dpm_solver_t* h, int n_sources, const dpm_scalar_source_t* sources) {
  if (!h) return DPM_ERR_ARG;
  CK(cudaSetDevice(h->s->device));
  return h->s->set_sources(n_sources, sources);
}

int dpm_cell_divergence(dpm_solver_t* h, const double* u, double* out) {
  if (!h || !u || !out) return DPM_ERR_ARG;
  Solver& s = *h->s;
  int rc = s.cp_alloc();
  if (!rc) rc = upload_vec3(s, u, s.cp_v, s.nc);
  if (rc) return rc;
  dpm::gpu::k_cp_divergence<<<dpm::gpu::nblk(s.nc), dpm::gpu::TPB, 0, s.st>>>(s.d, s.cp_v, s.cp_q);
  s.launches++;
  CK(cudaMemcpyAsync(out, s.cp_q, sizeof(double) * s.nc, cudaMemcpyDeviceToHost, s.st));
  CK(cudaStreamSynchronize(s.st));
  return DPM_OK;
}

int dpm_cell_adjoint_gradient(dpm_solver_t* h, const double* chi, double* v) {
  if (!h || !chi || !v) return DPM_ERR_ARG;
  Solver& s = *h->s;
  int rc = s.cp_alloc();
  if (rc) return rc;
  CK(cudaMemcpyAsync(s.cp_p, chi, sizeof(double) * s.nc, cudaMemcpyHostToDevice, s.st));
  dpm::gpu::k_cp_adjoint<<<dpm::gpu::nblk(s.nc), dpm::gpu::TPB, 0, s.st>>>(s.d, s.cp_p, s.cp_v);
  s.launches++;
  return download_vec3(s, s.cp_v, v, s.nc);
}

int dpm_cell_project(dpm_solver_t* h, double* u, const double* bconst, double tol, int max_it, int identity_precond,
                     int* n_it) {
  if (!h || !u || !bconst || !n_it || max_it < 0 || !(tol >= 0.0)) return DPM_ERR_ARG;
  Solver& s = *h->s;
  int rc = s.cp_alloc();
  if (!rc) rc = upload_vec3(s, u, s.U_spare, s.nc);
  if (rc) return rc;
  CK(cudaMemcpyAsync(s.cp_bconst, bconst, sizeof(double) * s.nc, cudaMemcpyHostToDevice, s.st));
  rc = s.cp_project(s.U_spare, s.cp_bconst, tol, max_it, identity_precond != 0, n_it);
  if (rc) return rc;
  return download_vec3(s, s.U_spare, u, s.nc);
}

}  // extern "C"
