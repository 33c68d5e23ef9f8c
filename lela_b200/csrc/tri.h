// lela_b200/csrc/tri.h -- triangular solves over Z/p (device pointers).
#pragma once
#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

#include "context.h"

namespace lela {

// B <- alpha * A^-1 * B (see tri.cu).  Synchronises once to read the
// diagonal check; returns ST_DIAG with *bad_idx on a singular diagonal.
// sparse: A may have many all-zero 64 x 64 tiles (read once more, with one
// more synchronisation, to trim the updates to the occupied tiles).
// row_kr (device, optional with sparse): per row r of A, a column range
// [x, y) outside which the row is zero (see zp_gemm_dev); the updates then
// also skip, per 128-row tile, the K blocks the tile cannot touch.
int zp_trsm_dev(Ctx *c, bool upper, bool unit, int m, int n, uint32_t p, uint32_t alpha,
                const uint32_t *A, size_t lda, uint32_t *B, size_t ldb, size_t *bad_idx,
                bool sparse = false, const int2 *row_kr = nullptr);

// B <- alpha * A^-1 * B for an n x n upper-triangular A in CSR form on the
// device (the sparse pivot block of Faugere-Lachartre); A is expanded into
// a dense scratch copy and solved by zp_trsm_dev.  Synchronises once to
// check the column indices.
int zp_trsm_csr_upper_dev(Ctx *c, bool unit, int n, int ncols, uint32_t p, uint32_t alpha,
                          const uint64_t *rowptr, const uint32_t *col, const uint32_t *val,
                          uint32_t *B, size_t ldb, size_t *bad_idx);

// Workspace bytes zp_trsm_dev asks ctx_workspace for (either solver), so a
// caller holding the workspace can size it once.
size_t zp_trsm_workspace_bytes(uint32_t p, int m, int n);

// One diagonal block (nb <= 64) solved on CUDA cores: B <- alpha*T^-1*B;
// dinv = inverted diagonal (nullptr for a unit diagonal).
int tri_left_block(Ctx *c, bool upper, int nb, const uint32_t *T, size_t ldt,
                   const uint32_t *dinv, uint32_t *B, size_t ldb, int ncols, uint32_t p,
                   uint32_t alpha);

}  // namespace lela
