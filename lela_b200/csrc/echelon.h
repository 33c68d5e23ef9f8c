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

}  // namespace lela
