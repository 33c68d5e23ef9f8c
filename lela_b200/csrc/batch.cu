// lela_b200/csrc/batch.cu -- batched work: many independent dense Z/p echelon
// blocks and many Faugere-Lachartre matrices per call.
//
// Small dense blocks (m * n * 4 bytes fit in one CTA's shared memory) are
// processed by ONE persistent launch: every CTA takes the next block from a
// device work counter, loads it into shared memory, runs the reference's
// elimination (Elimination::echelonize, lela/algorithms/elimination.tcc:
// 47-139 with DensePivotStrategy, pivot-strategy.tcc:19-42) and writes the
// echelon form, rank and det back.  The launch has a fixed shape, so it can
// be captured in a CUDA graph and replayed.  Larger blocks go through the
// panel pipeline of echelon.cu; the kernel used for their trailing updates
// (tensor-core or CUDA-core gemm) is chosen per block by the caller's
// selector.  Faugere-Lachartre matrices are spread over worker threads, each
// with its own handle state and CUDA stream, so one matrix's host-side
// steps overlap another's GPU work.
#include <atomic>
#include <mutex>
#include <thread>
#include <vector>

#include "batch.h"
#include "common.cuh"
#include "context.h"
#include "echelon.h"
#include "fl.h"

namespace lela {

// Largest block the small kernel takes: 200 KB of shared memory.
constexpr int SMALL_SMEM = 200 * 1024;

__global__ void __launch_bounds__(512)
    echelon_small_batch_kernel(const SmallItem *__restrict__ items, int count,
                               unsigned *__restrict__ next, uint64_t *__restrict__ rank_out,
                               uint32_t *__restrict__ det_out, uint32_t *__restrict__ status) {
  extern __shared__ uint32_t S[];
  __shared__ int s_item;
  __shared__ unsigned s_piv;
  while (true) {
    if (threadIdx.x == 0) s_item = (int)atomicAdd(next, 1u);
    __syncthreads();
    const int it = s_item;
    if (it >= count) break;
    const SmallItem I = items[it];
    const int m = I.m, n = I.n;
    const Modulus mod = make_modulus(I.p);
    const uint32_t p = I.p;
    for (int e = threadIdx.x; e < m * n; e += blockDim.x)
      S[e] = I.A[(size_t)(e / n) * I.ld + (e % n)];
    __syncthreads();
    int i = 0;
    uint32_t det = 1u % p;
    bool bad = false;
    for (int col = 0; col < n && i < m; ++col) {
      if (threadIdx.x == 0) s_piv = 0xFFFFFFFFu;
      __syncthreads();
      for (int r = i + threadIdx.x; r < m; r += blockDim.x)
        if (S[r * n + col] != 0u) atomicMin(&s_piv, (unsigned)r);
      __syncthreads();
      const unsigned q = s_piv;
      __syncthreads();
      if (q == 0xFFFFFFFFu) continue;
      if ((int)q != i)
        for (int j = col + threadIdx.x; j < n; j += blockDim.x) {
          uint32_t t = S[i * n + j];
          S[i * n + j] = S[q * n + j];
          S[q * n + j] = t;
        }
      __syncthreads();
      const uint32_t x = S[i * n + col];
      const uint32_t xinv = lela_inv_u32(p, x);
      if (xinv == 0u) {
        bad = true;
        break;
      }
      det = mod_mul(det, x, mod);
      // rows below: row_r -= (a_r / x) * row_i on columns col..n-1
      const int rows = m - i - 1, cols = n - col;
      for (int e = threadIdx.x; e < rows * cols; e += blockDim.x) {
        const int r = i + 1 + e / cols, j = col + e % cols;
        const uint32_t a = S[r * n + col];
        if (a == 0u || j == col) continue;
        const uint32_t f = mod_mul(a, xinv, mod);
        const uint32_t v = S[r * n + j], pv = mod_mul(f, S[i * n + j], mod);
        S[r * n + j] = v >= pv ? v - pv : v + (p - pv);
      }
      __syncthreads();
      for (int r = i + 1 + threadIdx.x; r < m; r += blockDim.x) S[r * n + col] = 0u;
      __syncthreads();
      ++i;
    }
    for (int e = threadIdx.x; e < m * n; e += blockDim.x)
      I.A[(size_t)(e / n) * I.ld + (e % n)] = S[e];
    if (threadIdx.x == 0) {
      rank_out[it] = (uint64_t)i;
      det_out[it] = det;
      status[it] = bad ? (uint32_t)ST_PIVOT : 0u;
    }
    __syncthreads();
  }
}

bool small_echelon_fits(int m, int n) { return (size_t)m * n * 4 <= (size_t)SMALL_SMEM; }

int echelon_small_batch_prepare(Ctx *c) {
  static std::once_flag once;
  static cudaError_t attr_err = cudaSuccess;
  std::call_once(once, [] {
    attr_err = cudaFuncSetAttribute(echelon_small_batch_kernel,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, SMALL_SMEM);
  });
  return attr_err == cudaSuccess ? ST_OK
                                 : ctx_cuda(c, attr_err, "cudaFuncSetAttribute(small batch)");
}

int echelon_small_batch_dev(Ctx *c, int count, const SmallItem *d_items, unsigned *d_next,
                            uint64_t *d_rank, uint32_t *d_det, uint32_t *d_status) {
  cudaError_t e = cudaMemsetAsync(d_next, 0, sizeof(unsigned), c->stream);
  if (e != cudaSuccess) return ctx_cuda(c, e, "small batch: counter");
  const int grid = std::min(count, c->num_sms);
  int pi = prof_begin(c, "echelon_small_batch");
  echelon_small_batch_kernel<<<grid, 512, SMALL_SMEM, c->stream>>>(d_items, count, d_next, d_rank,
                                                                   d_det, d_status);
  prof_end(c, pi);
  ctx_launched(c);
  e = cudaGetLastError();
  return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "small batch launch");
}

}  // namespace lela
