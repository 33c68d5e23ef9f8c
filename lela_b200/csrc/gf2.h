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

// Whether the host-pointer GF(2) gemm of this shape works in row blocks
// with its copies overlapped (tensor-core path, one K chunk, alpha = 1, at
// least two blocks of 512 rows).
bool gf2_gemm_pipelined(const Ctx *c, int M, int N, int K, int alpha);

// C <- A*B + beta*C over GF(2) with A, B, C in host memory (row strides in
// words) through the device buffers dA (M x words(K)), dB (K x words(N)),
// dC (M x words(N)), packed: B is copied and expanded to bytes once, then
// A's and C's rows block by block on the handle's copy stream, each block's
// product as soon as its rows are in, and its rows of C back on a second
// copy stream.  Asynchronous on the handle stream, which ends after the
// last copy back.  Only for shapes gf2_gemm_pipelined accepts.
int gf2_gemm_host_rows(Ctx *c, int M, int N, int K, const uint64_t *hA, size_t lda,
                       const uint64_t *hB, size_t ldb, int beta, uint64_t *hC, size_t ldc,
                       uint64_t *dA, uint64_t *dB, uint64_t *dC);

// The bit-packed four-Russians product alone.
int gf2_m4rm_dev(Ctx *c, int M, int N, int K, int alpha, const uint64_t *A, size_t lda,
                 const uint64_t *B, size_t ldb, int beta, uint64_t *C, size_t ldc);

// Non-reduced row-echelon form in place (LELA's pivot rule); *rank.
int gf2_echelon_dev(Ctx *c, int m, int n, uint64_t *D, size_t ld, size_t *rank);

}  // namespace lela
