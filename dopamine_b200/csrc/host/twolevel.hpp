// Set-up of the two-level preconditioner used by the flexible-CG pressure solve.
//
// The cells are split into P spatially compact parts (recursive coordinate bisection of the
// cell centres), one part per thread block of the persistent solve, and renumbered so that
// part b owns the contiguous range [b*C, b*C + size_b).  The preconditioner is additive:
//   z = S_b(r) + y_b,   y = E^-1 Z^T r,   E = Z^T A Z,
// with S_b a few Chebyshev sweeps on the part's own rows (couplings to other parts dropped)
// and Z the part-indicator matrix.  No counterpart in the reference, whose pressure solve is
// PETSc CG with BoomerAMG or (block-)Jacobi (src/solver/pressure_backend_petsc.c:381-463);
// the Krylov stopping rule is kept identical.
#pragma once
#include <cstdint>
#include <vector>

namespace dpm {

struct TwoLevel {
  int n = 0, P = 0, C = 0;        // cells, parts, cells per part (last part may be shorter)
  int WA = 0, WL = 0;             // global and local (intra-part, off-diagonal) row widths
  std::vector<int> perm;          // perm[new] = old
  std::vector<int> col;           // [WA][n] permuted operator, columns in new numbering
  std::vector<double> val;        // [WA][n]
  std::vector<double> dinv;       // [n] 1 / diagonal, new numbering
  // local (intra-part) off-diagonal couplings, row-scaled by 1/diagonal and packed per entry as
  // (local column in the low 16 bits | bfloat16 of a_ij / a_ii in the high 16 bits); rows are
  // padded to WL entries with (own local index, 0)
  std::vector<unsigned> lpk;      // [WL][n]
  std::vector<double> einv;       // [P][P] inverse (or regularised inverse) of E
  // Deflation of the coarse correction before smoothing: z = y_b + S_b(r - A Z y).  (A Z y)_i
  // needs y of the parts next to i's part: NB slots per part (slot 0 = the part itself, then its
  // neighbour parts), the E^-1 rows of those slots, and per cell the intra-part row sum and the
  // cross-part couplings (slot, value).  deflate = 0 when a part has more than 31 neighbours.
  int deflate = 0, NB = 1;
  std::vector<int> nbr;           // [P][NB] part ids, -1 padded
  std::vector<double> einv_nb;    // [P][NB][P]
  std::vector<float> srow;        // [n] sum of the row's entries inside the part (diagonal included)
  std::vector<int> xoff;          // [n+1] cross-part couplings of row i: xoff[i] .. xoff[i+1]-1
  std::vector<unsigned char> xslot;  // slot of the coupled cell's part in its own part's list
  std::vector<float> xval;        // coupling value a_ij
};

// A in padded ELL [WA][n] (padding = (own row, 0)), cell centres xyz[3*n]; nullsp = the
// operator has the constant null space (no Dirichlet rows).  Returns 0 or a negative code.
// coarse = false: the partition, permuted operator, local rows and intra-part row sums only (the
// learned term's structures on meshes whose parts do not fit the two-level kernel).
int build_two_level(int n, int WA, const int* A_col, const double* A_val, const double* xyz, int P, bool nullsp,
                    TwoLevel& T, bool coarse = true);

}  // namespace dpm
