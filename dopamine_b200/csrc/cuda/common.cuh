// Shared device-side definitions for the sm_100a RK3W hot path.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace dpm {
namespace gpu {

constexpr double SMALLD = 1.0e-30;
constexpr int PADI = -2147483647 - 1;
constexpr int TPB = 256;

// Boundary-condition ids (src/mod_parameters.f90:41-51)
constexpr int BC_INLET = 1, BC_OUTLET = 2, BC_WALL_NOSLIP = 3, BC_WALL_MODEL = 4, BC_SLIP = 5, BC_PERIODIC = 6,
              BC_SYMMETRY = 7, BC_FIXEDTEMP = 8, BC_ZEROGRADIENT = 9, BC_WALL_VELOCITY = 10,
              BC_ABL_INLET = 11;

__host__ __device__ inline bool is_wall_bc(int bc) {
  return bc == BC_WALL_NOSLIP || bc == BC_WALL_MODEL || bc == BC_WALL_VELOCITY || bc == BC_SLIP || bc == BC_SYMMETRY;
}

// Static mesh and operator data resident in HBM.  Cell and face vectors are SoA: component k
// of cell c is at [k * nc + c]; ELL lists are [slot * nc + c].
struct Dev {
  int nc, nf, nfi, nb, nfp;
  int S, SP, SB, W, WA;
  // cells
  const double *vol, *ivol, *cen;   // cen [3][nc]
  const double *Tinv, *G;           // [9][nc], column-major 3x3 per cell
  const int *cf, *cps, *cbn;        // ELL: faces, pressure faces (~idx = neighbour side), boundary faces
  const int* ls_idx;                // [W][nc]: cell, -(b+1) boundary entry, PADI
  const double* ls_w;               // [3][W][nc]
  // faces
  const int *fo, *fn;
  const double *sf, *nrm, *fcen, *eps;  // [3][nf]
  const double *area, *gc, *wbl, *dcf;
  // boundary faces (b = f - nfi)
  const int *bbc, *bpnb, *bpair, *bps, *bcanon;  // bc id, periodic partner cell, pair b, canonical ps idx, is canonical
  const double *bpgc, *bpdcf, *bcb, *bkout, *yw, *bUval, *bpval;  // bkout, bUval [3][nb]
  const double* abl_fluc;  // [3][nb] synthetic fluctuation of the ABL-inlet faces, null without one
  // pressure-solver faces
  const int *pso, *psn, *psf;
  const double *psc, *psgcf, *psgcw, *psk, *pskrc;  // psk, pskrc [3][nfp]
  // matrix (ELL, sorted columns)
  const int* Acol;
  const double *Aval, *Adinv;
  // TVD upwind context per face and flux sign (slot 0: F >= 0, slot 1: F < 0), [2][nf]; null when
  // no TVD scheme is in use: far-upwind cell (-1: none, -2: no reconstruction context), the face
  // and downwind distances along the upwind direction (the latter floored at 1e-30) and the
  // far-upwind cell's distance behind the upwind cell
  const int* tvd_far;
  const double *tvd_sf, *tvd_sd, *tvd_su;
};

// Fields and work arrays.
struct Fld {
  double *U, *p, *p_old, *phi_prev, *nu_sgs, *rhs, *T;
  double *Ub, *pb, *phi_prev_b, *tau;
  double *gU, *gp, *gp_rc, *gpc;
  double *H, *H0;
  double *ff, *Uf;
  double *fadv, *fvis, *fdiv, *ps_cross;
  double *ptot, *ptot_b, *phi_it;
  double* upf;  // wall-model filter state [3][nb]
};

}  // namespace gpu
}  // namespace dpm
