// lela_b200/csrc/echelon.h -- dense row-echelon form over Z/p (device).
#pragma once
#include <cstddef>
#include <cstdint>
#include <utility>
#include <vector>

#include "context.h"

namespace lela {

// Non-reduced row-echelon form of the m x n matrix D in place, with LELA's
// pivot rule (see echelon.cu): rank, det = product of the pivots, and the
// pivot columns in order (optional).  Synchronises the stream per block.
// Returns ST_PIVOT when a pivot is not invertible in Modular<uint32>.
// PLUQ bookkeeping (optional): every panel's multipliers kept in L (m x
// ldL, zeroed here; column k holds pivot k's multipliers, rows moved with
// the row transpositions), and the row transpositions (current row, pivot
// row) in order, those of equal rows included.
struct EchelonKeep {
  uint32_t *L = nullptr;
  size_t ldL = 0;
  std::vector<std::pair<int, int>> swaps;
};

int zp_echelon_dev(Ctx *c, int m, int n, uint32_t p, uint32_t *D, size_t ld, size_t *rank,
                   uint32_t *det, std::vector<int> *pivot_cols, EchelonKeep *keep = nullptr);

// PLUQ decomposition of D in place with LELA's Elimination::pluq semantics
// (see echelon.cu): U above and on the diagonal in the permuted column
// order, the multipliers of L below it; P and Q as transposition pairs in
// the reference's (reversed) order.  ST_PIVOT when a pivot is not
// invertible in Modular<uint32>.
int zp_pluq_dev(Ctx *c, int m, int n, uint32_t p, uint32_t *D, size_t ld,
                std::vector<std::pair<int, int>> *P, std::vector<std::pair<int, int>> *Q,
                size_t *rank, uint32_t *det);

// The standard method's reduced form (pivots 1) of D in place with its
// transform, as Elimination::echelonize_reduced (A, L, P, rank, det, true)
// leaves them: Lout (m x m, leading dimension ldl) with R = Lout P D_in, P
// the row transpositions in the order applied.  p < 2^31 (ST_ARG above);
// ST_PIVOT when a pivot is not invertible.
int zp_echelon_transform_dev(Ctx *c, int m, int n, uint32_t p, uint32_t *D, size_t ld,
                             uint32_t *Lout, size_t ldl, std::vector<std::pair<int, int>> *P,
                             size_t *rank, uint32_t *det);

// Reduced row-echelon form of D in place as LELA's GaussJordan::
// echelonize_reduced leaves it (pivots keep their values; zero above and
// below them), or with unit_pivots as Elimination::echelonize_reduced does
// (each pivot row divided by its pivot): the form above, then the pivot
// columns cleared upwards by one triangular solve.  Same rank, det and
// errors.  Defined in fl.cu, beside the column gather it shares with the
// reduced FL form.
int zp_echelon_reduced_dev(Ctx *c, int m, int n, uint32_t p, uint32_t *D, size_t ld,
                           bool unit_pivots, size_t *rank, uint32_t *det);

}  // namespace lela
