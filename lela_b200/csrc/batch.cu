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
// panel pipeline of echelon.cu, spread over worker handles with their own
// streams while the persistent launch runs; the kernel used for their
// trailing updates (tensor-core or CUDA-core gemm) is chosen per block by the
// caller's selector.  Faugere-Lachartre matrices are spread over worker threads, each
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
constexpr int SB_THREADS = 512;
constexpr int SB_WARPS = SB_THREADS / 32;
constexpr int SB_MAXRANK = 256;  // min(m, n) <= 226 for any block that fits

// Field arithmetic for the small kernel: 32-bit Barrett when p < 2^16 (all
// products fit in 32 bits), 64-bit Barrett otherwise.
struct SbSmall {
  uint32_t p, mu;  // mu = floor(2^32 / p)
  __device__ explicit SbSmall(uint32_t p_) : p(p_), mu((uint32_t)((1ull << 32) / p_)) {}
  __device__ __forceinline__ uint32_t red(uint32_t x) const {
    const uint32_t r = x - __umulhi(x, mu) * p;
    return r >= p ? r - p : r;
  }
  __device__ __forceinline__ uint32_t mul(uint32_t a, uint32_t b) const { return red(a * b); }
  __device__ __forceinline__ uint32_t dot2(uint32_t a, uint32_t b, uint32_t c, uint32_t d) const {
    const uint32_t r = red(a * b) + red(c * d);
    return r >= p ? r - p : r;
  }
};
struct SbWide {
  Modulus mod;
  uint32_t p, two64;
  __device__ explicit SbWide(uint32_t p_) : mod(make_modulus(p_)), p(p_), two64(two64_mod(p_)) {}
  __device__ __forceinline__ uint32_t mul(uint32_t a, uint32_t b) const {
    return mod_mul(a, b, mod);
  }
  __device__ __forceinline__ uint32_t dot2(uint32_t a, uint32_t b, uint32_t c, uint32_t d) const {
    const uint64_t x = (uint64_t)a * b, y = (uint64_t)c * d;
    uint64_t s = x + y;
    if (s < y) s += two64;
    return mod_reduce(s, mod);
  }
};

// Exact inverse of a unit modulo p (extended Euclid, 64-bit coefficients);
// 0 when gcd(x, p) != 1.
__device__ __forceinline__ uint32_t sb_inv_exact(uint32_t p, uint32_t x) {
  uint32_t r0 = p, r1 = x;
  int64_t s0 = 0, s1 = 1;
  while (r1 != 0) {
    const uint32_t q = r0 / r1, r = r0 - q * r1;
    r0 = r1;
    r1 = r;
    const int64_t s = s0 - (int64_t)q * s1;
    s0 = s1;
    s1 = s;
  }
  if (r0 != 1) return 0;
  int64_t v = s0 % (int64_t)p;
  return (uint32_t)(v < 0 ? v + p : v);
}

struct SbShared {
  int pcol[SB_MAXRANK];
  uint32_t y[SB_MAXRANK], S[SB_MAXRANK], sinv[SB_MAXRANK], x[SB_MAXRANK];
  int first[SB_WARPS];
  int bad;
};

// The reference's elimination on the m x n block S (row-major in shared
// memory) without division: the pivot of a column is the first row at or
// below the current one with a nonzero there (swapped in), and each row r
// below becomes y row_r - row_r[col] row_i for pivot value y.  Row i then
// holds S_i U_i with S_i the product of the earlier pivot values; the
// entries left of the current column are not kept up to date.  At the end
// the S_i are inverted in parallel, pivot row i is scaled to U_i (zero left
// of its pivot column), rows below the rank are zero, det is the product of
// the pivots x_i = y_i / S_i, and a pivot that Modular<uint32>::inv cannot
// invert sets *bad (the reference's error).
template <class A>
__device__ void small_echelon(uint32_t *S, int m, int n, const A ar, SbShared &sh, int *rank_out,
                              uint32_t *det_out) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const uint32_t p = ar.p;
  int i = 0;
  uint32_t Sc = 1u % p;
  for (int col = 0; col < n && i < m; ++col) {
    int q = -1;
    for (int base = i; base < m; base += SB_THREADS) {
      const int r = base + tid;
      const unsigned b = __ballot_sync(0xffffffffu, r < m && S[(size_t)r * n + col] != 0u);
      if (lane == 0) sh.first[wid] = b ? base + wid * 32 + __ffs(b) - 1 : 0x7fffffff;
      __syncthreads();
      int f = 0x7fffffff;
      for (int k = 0; k < SB_WARPS; ++k) f = min(f, sh.first[k]);
      if (f != 0x7fffffff) {
        q = f;
        break;
      }
      __syncthreads();  // sh.first is rewritten by the next chunk or column
    }
    if (q < 0) continue;
    if (q != i) {
      for (int j = col + tid; j < n; j += SB_THREADS) {
        const uint32_t a = S[(size_t)i * n + j];
        S[(size_t)i * n + j] = S[(size_t)q * n + j];
        S[(size_t)q * n + j] = a;
      }
      __syncthreads();
    }
    const uint32_t *P = S + (size_t)i * n;
    const uint32_t y = P[col];
    for (int r = i + 1 + wid; r < m; r += SB_WARPS) {
      uint32_t *row = S + (size_t)r * n;
      const uint32_t a = row[col];
      const uint32_t na = a ? p - a : 0u;
      for (int j = col + 1 + lane; j < n; j += 32) row[j] = ar.dot2(y, row[j], na, P[j]);
    }
    if (tid == 0) {
      sh.pcol[i] = col;
      sh.y[i] = y;
      sh.S[i] = Sc;
    }
    __syncthreads();
    Sc = ar.mul(Sc, y);
    ++i;
  }
  const int rank = i;
  if (tid == 0) sh.bad = 0;
  __syncthreads();
  for (int k = tid; k < rank; k += SB_THREADS) {
    const uint32_t si = sb_inv_exact(p, sh.S[k]);
    const uint32_t x = ar.mul(sh.y[k], si);
    sh.sinv[k] = si;
    sh.x[k] = x;
    if (si == 0u || lela_inv_u32(p, x) == 0u) atomicOr(&sh.bad, 1);
  }
  __syncthreads();
  for (int r = wid; r < m; r += SB_WARPS) {
    uint32_t *row = S + (size_t)r * n;
    if (r < rank) {
      const int pc = sh.pcol[r];
      const uint32_t si = sh.sinv[r];
      for (int j = lane; j < n; j += 32) row[j] = j < pc ? 0u : ar.mul(row[j], si);
    } else {
      for (int j = lane; j < n; j += 32) row[j] = 0u;
    }
  }
  if (tid == 0) {
    uint32_t det = 1u % p;
    for (int k = 0; k < rank; ++k) det = ar.mul(det, sh.x[k]);
    *rank_out = rank;
    *det_out = det;
  }
  __syncthreads();
}

// Persistent launch: each CTA takes the next block from the work counter.
__global__ void __launch_bounds__(SB_THREADS)
    echelon_small_batch_kernel(const SmallItem *__restrict__ items, int count,
                               unsigned *__restrict__ next, uint64_t *__restrict__ rank_out,
                               uint32_t *__restrict__ det_out, uint32_t *__restrict__ status) {
  extern __shared__ uint32_t S[];
  __shared__ SbShared sh;
  __shared__ int s_item, s_rank;
  __shared__ uint32_t s_det;
  while (true) {
    if (threadIdx.x == 0) s_item = (int)atomicAdd(next, 1u);
    __syncthreads();
    const int it = s_item;
    if (it >= count) break;
    const SmallItem I = items[it];
    const int m = I.m, n = I.n;
    for (int e = threadIdx.x; e < m * n; e += SB_THREADS)
      S[e] = I.A[(size_t)(e / n) * I.ld + (e % n)];
    __syncthreads();
    if (I.p < (1u << 16))
      small_echelon(S, m, n, SbSmall(I.p), sh, &s_rank, &s_det);
    else
      small_echelon(S, m, n, SbWide(I.p), sh, &s_rank, &s_det);
    for (int e = threadIdx.x; e < m * n; e += SB_THREADS)
      I.A[(size_t)(e / n) * I.ld + (e % n)] = S[e];
    if (threadIdx.x == 0) {
      rank_out[it] = (uint64_t)s_rank;
      det_out[it] = s_det;
      status[it] = sh.bad ? (uint32_t)ST_PIVOT : 0u;
    }
    __syncthreads();
  }
}

bool small_echelon_fits(int m, int n) { return (size_t)m * n * 4 <= (size_t)SMALL_SMEM; }

int echelon_small_batch_prepare(Ctx *c) {
  return ctx_smem_attr(c, (const void *)echelon_small_batch_kernel, SMALL_SMEM,
                       "cudaFuncSetAttribute(small batch)");
}

int echelon_small_batch_dev(Ctx *c, int count, const SmallItem *d_items, unsigned *d_next,
                            uint64_t *d_rank, uint32_t *d_det, uint32_t *d_status) {
  cudaError_t e = cudaMemsetAsync(d_next, 0, sizeof(unsigned), c->stream);
  if (e != cudaSuccess) return ctx_cuda(c, e, "small batch: counter");
  const int grid = std::min(count, c->num_sms);
  int pi = prof_begin(c, "echelon_small_batch");
  echelon_small_batch_kernel<<<grid, SB_THREADS, SMALL_SMEM, c->stream>>>(d_items, count, d_next, d_rank,
                                                                   d_det, d_status);
  prof_end(c, pi);
  ctx_launched(c);
  e = cudaGetLastError();
  return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "small batch launch");
}

}  // namespace lela
