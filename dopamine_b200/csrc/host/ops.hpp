// Static operator data the time step consumes, derived once from the mesh and the boundary
// configuration (the reference computes these in solver_init, src/solver/mod_fv_solver.f90:302-508,
// and pressure_solver_init, src/solver/mod_pressure_solver.f90:100-452).  Laid out for the GPU:
// per-cell lists are ELLPACK ([slot][cell], padded) so that one thread per cell reads them with
// coalesced loads, and every per-cell list keeps the reference's accumulation order.
#pragma once
#include <cstdint>
#include <vector>

#include "../../../include/dopamine_b200.h"
#include "mesh.hpp"

namespace dpm {

constexpr int PAD = -2147483647 - 1;  // INT_MIN: unused ELL slot

struct StaticOps {
  int64_t nc = 0, nf = 0, nfi = 0, nb = 0, nfp = 0;
  // pressure-solver face list: interior faces (idx == face id), then one canonical face per periodic pair
  std::vector<int> ps_o, ps_n, ps_f;
  std::vector<double> ps_coeff;   // |S| / (d . n)  (periodic: mean area / (d_o + d_partner))
  std::vector<double> ps_gcf;     // owner weight of the face-velocity interpolation
  std::vector<double> ps_gcw;     // owner weight of the deferred cross term
  std::vector<double> ps_k;       // [3][nfp] Jasak k-vector, 0 where inactive
  std::vector<double> ps_krc;     // [3][nfp] k used by Rhie-Chow (0 when rhie_chow_dual)
  std::vector<double> diag;       // operator diagonal
  std::vector<double> bnd_kout;   // [3][nb] k-vector of outlet faces, 0 elsewhere
  std::vector<double> bnd_cb;     // area / d_orth of outlet faces (0 elsewhere)
  std::vector<int> bnd_bc;        // bc id per boundary face
  std::vector<int> bnd_pnb;       // periodic partner cell (-1)
  std::vector<int> dir_rows;      // outlet owner rows
  std::vector<double> dir_vals;   // c_b * p_val
  bool skip_nonortho = false, skip_grad_p = false, diag_interface = false;
  int n_nonortho_corr = 1;
  int64_t n_outlet = 0;
  double V_min = 0.0, V_total = 0.0;
  // assembled matrix rows, columns sorted, diagonal in place: ELL [WA][nc]
  int WA = 0;
  std::vector<int> A_col;
  std::vector<double> A_val;
  // per-cell ELL lists
  int S = 0;                      // max faces per cell
  std::vector<int> cell_face;     // [S][nc] face ids ascending
  int SP = 0;                     // max pressure-solver faces per cell
  std::vector<int> cell_ps;       // [SP][nc] ps idx (owner) or ~idx (neighbour), ascending idx
  int SB = 0;                     // max boundary faces per cell
  std::vector<int> cell_bnd;      // [SB][nc] boundary-face index b, ascending
  int W = 0;                      // max LS stencil width
  std::vector<int> ls_idx;        // [W][nc] cell >= 0, boundary entry -(b+1), PAD
  std::vector<double> ls_w;       // [3][W][nc]
  // cell operators
  std::vector<double> Tinv;       // [9][nc] inverse of sum |S| n n^T (column-major 3x3)
  std::vector<double> G;          // [9][nc] SGS filter tensor
  std::vector<double> y_w;        // wall-model sampling distance per boundary face
  std::vector<double> wblend;     // refine_blend_weight(skew) per face
};

int build_static_ops(const Mesh& m, const dpm_patch_cfg_t* pc, const dpm_params_t& P, StaticOps& S);

}  // namespace dpm
