// lela_b200/csrc/fl.h -- Faugere-Lachartre echelon form over Z/p (device).
#pragma once
#include <cstddef>
#include <cstdint>

#include "context.h"

namespace lela {

struct FlResult {
  size_t rank;
  uint32_t det;
  size_t out_rows;  // rows written to R
  size_t bad_row;   // WrongMatrixForm row, or the singular pivot index
};

// The result as CSR rows (the SparseMatrix layout: column indices strictly
// increasing in a row), built on the device in the handle's buffers
// BUF_FL_CSR_P (row pointers) and BUF_FL_CSR_V (column indices, then
// values): rowptr[out_rows + 1], colidx[nnz], vals[nnz].
struct FlCsr {
  uint64_t *rowptr = nullptr;
  uint32_t *colidx = nullptr, *vals = nullptr;
  size_t nnz = 0;
};

// X = CSR (device arrays) with its row pointers and row heads (first
// stored column and value of each non-empty row) also on the host.
// R: device, out_rows x n (row stride ldr), fully written -- or, with csr
// given (R may then be null), the result as CSR rows instead.
int zp_fl_echelonize_dev(Ctx *c, int m, int n, uint32_t p, const uint64_t *d_rowptr,
                         const uint32_t *d_colidx, const uint32_t *d_vals,
                         const uint64_t *h_rowptr, const uint32_t *h_heads,
                         const uint32_t *h_headvals, bool reduced, bool only_D, uint32_t *R,
                         size_t ldr, FlResult *res, FlCsr *csr = nullptr);

// Row heads of a device CSR: heads[r] = colidx[rowptr[r]], vals likewise
// (0 for empty rows).
int fl_row_heads_dev(Ctx *c, int m, const uint64_t *d_rowptr, const uint32_t *d_colidx,
                     const uint32_t *d_vals, uint32_t *d_heads, uint32_t *d_headvals);

}  // namespace lela
