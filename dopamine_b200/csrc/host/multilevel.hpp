// Set-up of the aggregation multigrid preconditioner used by the multilevel flexible-CG
// pressure solve.
//
// Levels are built by pairwise aggregation along the strongest negative coupling (each pass
// pairs every still-unpaired row with its strongest unpaired neighbour, so a pass roughly
// halves the rows and follows the mesh anisotropy; `passes` passes make one level), with the
// Galerkin operator A_{l+1} = T^T A_l T of the piecewise-constant prolongation T.  Each
// smoothed level keeps its operator in FP32 padded ELL, 1/diagonal, the aggregate of every row
// and the member rows of every aggregate; the coarsest level keeps a dense FP32 inverse
// (regularised by the constant vector when the operator is singular).  No counterpart in the
// reference, whose pressure solve is PETSc CG with BoomerAMG or (block-)Jacobi
// (src/solver/pressure_backend_petsc.c:381-463); the Krylov stopping rule is kept identical.
#pragma once
#include <cstdint>
#include <vector>

namespace dpm {

constexpr int ML_MAX_LEVELS = 12;
constexpr int ML_MAX_DEGREE = 8;

struct MlLevel {
  int n = 0, W = 0, M = 0;        // rows, widest row (diagonal included), members per aggregate
  std::vector<float> dinv;        // [n]
  // The same operator as the smoother reads it: off-diagonal entries only, scaled by the row's
  // diagonal (D^-1 A = G + S), in ELL [Wo][n] padded with (own row, 0).  sv32 holds s_ij in FP32,
  // sv16 the IEEE binary16 bits of s_ij (round to nearest even); g32 / g16 the diagonal term of
  // the scaled row, 1 + sum_j (s_ij - stored s_ij), so that every stored row sums to the same
  // value as the exact one (a rounded off-diagonal would otherwise shift the near-null space).
  int Wo = 0;
  std::vector<int> ocol;          // [Wo][n]
  std::vector<float> sv32;        // [Wo][n]
  std::vector<unsigned short> sv16;  // [Wo][n]
  std::vector<float> g32, g16;    // [n]
  std::vector<float> diag;        // [n] a_ii
  std::vector<int> agg;           // [n] row of the next level this row belongs to
  std::vector<int> mem;           // [M][n_next] rows of this level in each aggregate, -1 padded
  double lmax = 0.0;              // estimate of the largest eigenvalue of D^-1 A
};

struct Multilevel {
  std::vector<MlLevel> lv;        // smoothed levels (level 0 = the fine operator)
  int nC = 0;                     // rows of the coarsest (directly solved) level
  std::vector<float> cinv;        // [nC][nC]
  std::vector<int> sizes;         // rows per level, coarsest last
  std::vector<int64_t> nnz;       // non-zeros per level, coarsest last
};

// A in padded ELL [WA][n] (padding = (own row, 0)); nullsp = the operator has the constant null
// space.  Coarsening stops at <= ncoarse rows; returns 0, or a negative code when the coarsening
// stalls above max_dense rows or a factorisation fails.
int build_multilevel(int n, int WA, const int* A_col, const double* A_val, bool nullsp, int passes, double beta,
                     int ncoarse, int max_dense, Multilevel& M);

}  // namespace dpm
