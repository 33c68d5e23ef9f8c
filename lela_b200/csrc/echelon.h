// lela_b200/csrc/echelon.h -- dense row-echelon form over Z/p (device).
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

#include "context.h"

namespace lela {

// Non-reduced row-echelon form of the m x n matrix D in place, with LELA's
// pivot rule (see echelon.cu): rank, det = product of the pivots, and the
// pivot columns in order (optional).  Synchronises the stream per block.
// Returns ST_PIVOT when a pivot is not invertible in Modular<uint32>.
int zp_echelon_dev(Ctx *c, int m, int n, uint32_t p, uint32_t *D, size_t ld, size_t *rank,
                   uint32_t *det, std::vector<int> *pivot_cols);

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
