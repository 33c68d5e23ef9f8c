// lela_b200/csrc/gf2.h -- dense GF(2) gemm and echelon form (device).
#pragma once
#include <cstddef>
#include <cstdint>

#include "context.h"

namespace lela {

// C <- alpha*A*B + beta*C over GF(2) on packed words (row strides in words).
// kernel: GF2_AUTO, GF2_TC (int8-expanded tensor cores) or GF2_M4RM.
int gf2_gemm_dev(Ctx *c, int kernel, int M, int N, int K, int alpha, const uint64_t *A,
                 size_t lda, const uint64_t *B, size_t ldb, int beta, uint64_t *C, size_t ldc);

// The bit-packed four-Russians product alone.
int gf2_m4rm_dev(Ctx *c, int M, int N, int K, int alpha, const uint64_t *A, size_t lda,
                 const uint64_t *B, size_t ldb, int beta, uint64_t *C, size_t ldc);

// Non-reduced row-echelon form in place (LELA's pivot rule); *rank.
int gf2_echelon_dev(Ctx *c, int m, int n, uint64_t *D, size_t ld, size_t *rank);

}  // namespace lela
