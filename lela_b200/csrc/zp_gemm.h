// lela_b200/csrc/zp_gemm.h -- dense Z/p gemm entry points (device pointers).
#pragma once
#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

#include "context.h"

namespace lela {

// Largest K handled by one tensor-core launch: 32768 * 255^2 < 2^31.
constexpr int ZP_KCHUNK = 32768;

int zp_limbs_for(uint32_t p);
size_t zp_gemm_workspace_bytes(uint32_t p, int M, int N, int K);

// C <- alpha*A*B + beta*C mod p on the handle's stream (asynchronous).
// kernel: GEMM_AUTO, GEMM_PLAIN or GEMM_TC.  ws_override, when non-null,
// is used instead of the handle workspace for the limb planes and must hold
// zp_gemm_workspace_bytes(p, M, N, K) bytes.  kr (device, optional): per
// row r of A, a column range [kr[r].x, kr[r].y) of the whole matrix outside
// which row r is zero (y <= x: the row is zero), and kbase the whole
// matrix's column of A's column 0; the tensor-core kernel then multiplies,
// per 128-row tile, only the K blocks its rows can touch (the other
// kernels ignore it: the result is the same).
int zp_gemm_dev(Ctx *c, int kernel, int M, int N, int K, uint32_t p, uint32_t alpha,
                const uint32_t *A, size_t lda, const uint32_t *B, size_t ldb, uint32_t beta,
                uint32_t *C, size_t ldc, uint8_t *ws_override, const int2 *kr = nullptr,
                int kbase = 0);

// The kernel GEMM_AUTO resolves to for this shape (the handle's forced
// kernel, else the small-K crossover rule).
int zp_gemm_pick(const Ctx *c, int M, int N, int K, uint32_t p);
// The tensor-core tile variant (TcCfg<L, T>'s T: 0, 1, or 2 for one limb)
// for this K and modulus: the handle's forced shape (wide or
// double-buffered), else wide for two limbs at K >= 512 and four limbs,
// double-buffered otherwise; for one limb the number of epilogue warps
// follows K.
int zp_gemm_tile_pick(const Ctx *c, int K, uint32_t p);

// Whether the host-pointer gemm of this shape is done in row blocks with
// its copies overlapped (tensor-core path, one K chunk, at least two blocks
// of PIPE_MIN_ROWS rows).
constexpr int PIPE_MIN_ROWS = 512;
bool zp_gemm_pipelined(const Ctx *c, int M, int N, int K, uint32_t p, uint32_t alpha);

// C <- alpha*A*B + beta*C mod p with A, B, C in host memory (row strides
// lda, ldb, ldc) through the device buffers dA (M x K), dB (K x N), dC
// (M x N, packed): the row-block pipeline above.  Asynchronous on the
// handle stream, which ends after the last copy back; the caller
// synchronises it.  Only for shapes zp_gemm_pipelined accepts.
int zp_gemm_host_rows(Ctx *c, int M, int N, int K, uint32_t p, uint32_t alpha,
                      const uint32_t *hA, size_t lda, const uint32_t *hB, size_t ldb,
                      uint32_t beta, uint32_t *hC, size_t ldc, uint32_t *dA, uint32_t *dB,
                      uint32_t *dC);

}  // namespace lela

namespace lela {
// GF(2) product on the tensor cores from 0/1 byte planes (see zp_gemm.cu).
int gf2_gemm_tc_planes(Ctx *c, int M, int N, int K, const uint8_t *Ab, const uint8_t *Bb, int Kp,
                       uint32_t alpha, uint32_t beta, uint64_t *C, size_t ldc_words);
}  // namespace lela
