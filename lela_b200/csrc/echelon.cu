// lela_b200/csrc/echelon.cu -- non-reduced row-echelon form over Z/p with
// LELA's pivot rule, in place on a dense device matrix.
//
// Reference semantics (bit-exact target): Elimination::echelonize
// (lela/algorithms/elimination.tcc:47-139) with DensePivotStrategy
// (lela/algorithms/pivot-strategy.tcc:19-42), which EchelonForm's dense path
// (GaussJordan::echelonize + move_L, lela/solutions/echelon-form.h:103-134)
// reproduces (tests/test-gauss-jordan.C:91-99).  At current row i and column
// c the pivot is the first nonzero of column c at or below row i (columns
// without one are skipped); it is swapped into row i by a transposition,
// multiplies det, and every row below gets row_i * (-a/x) added.  Pivots
// are not normalised; entries below pivots end up zero.
//
// Blocked, speculative, exact.  Over a block of up to W = 64 columns the
// rule almost always picks "the next nonzero row" -- identically zero rows
// are never pivots and only move under the transpositions.  So:
//  1. the candidate rows are the next W rows at or below i that are not
//     known to be zero; one CTA computes the LU factorisation without
//     pivoting of their W x W block and stops at the first zero pivot t;
//  2. the first t pivots are exactly the reference's: the transpositions
//     they imply (each pivot swaps with the row at its target position) are
//     replayed on the host and applied to the matrix with one row gather;
//  3. right-looking update: L21 = A21 U11^-1 (CUDA cores), U12 = L11^-1 A12
//     (CUDA cores), A22 -= L21 U12 (limb-split tensor-core gemm, K = t);
//  4. at a zero pivot the now up-to-date column is searched for its first
//     nonzero at or below row i (one kernel); the row is transposed into
//     place, or the column is skipped; a row found identically zero from the
//     current column on is marked and never offered as a candidate again.
// Every pivot thus equals the reference's, so U, rank and det do too.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "context.h"
#include "echelon.h"
#include "tri.h"
#include "zp_gemm.h"

namespace lela {

constexpr int EW = 64;  // block width (columns / candidate rows)

// flags[r] = 1 if row r has a nonzero in columns [c0, n).
__global__ void row_nonzero_kernel(const uint32_t *__restrict__ D, size_t ld, int m, int c0, int n,
                                   uint8_t *__restrict__ flags) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int r = warp; r < m; r += nwarps) {
    const uint32_t *row = D + (size_t)r * ld;
    uint32_t any = 0;
    for (int j = c0 + lane; j < n; j += 32) any |= row[j];
    any = __any_sync(0xffffffffu, any != 0);
    if (lane == 0) flags[r] = any ? 1 : 0;
  }
}

// LU without pivoting of the w x w block D[rows[k], c + j] (k, j < w) in
// shared memory.  Writes the combined factors (L strictly below the
// diagonal, U on and above) to blk (64 x 64, row stride 64), the inverted
// pivots to pinv, and out[0] = t, the number of leading nonzero pivots;
// out[1] = 1 when a nonzero pivot is not invertible (LELA's LELAError).
__global__ void __launch_bounds__(1024)
    block_lu_kernel(const uint32_t *__restrict__ D, size_t ld, const int *__restrict__ rows, int c,
                    int w, Modulus mod, uint32_t *__restrict__ blk, uint32_t *__restrict__ pinv,
                    uint32_t *out) {
  __shared__ uint32_t S[EW][EW + 1];
  __shared__ uint32_t s_inv;
  __shared__ int s_stop;
  const uint32_t p = (uint32_t)mod.p;
  for (int e = threadIdx.x; e < EW * EW; e += blockDim.x) {
    int r = e / EW, j = e % EW;
    S[r][j] = (r < w && j < w) ? D[(size_t)rows[r] * ld + c + j] : 0u;
  }
  if (threadIdx.x == 0) s_stop = 0;
  __syncthreads();
  int t = w;
  for (int k = 0; k < w; ++k) {
    if (threadIdx.x == 0) {
      uint32_t piv = S[k][k];
      if (piv == 0) {
        s_stop = 1;
      } else {
        uint32_t inv = lela_inv_u32(p, piv);
        if (inv == 0) {
          s_stop = 2;
        } else {
          s_inv = inv;
          pinv[k] = inv;
        }
      }
    }
    __syncthreads();
    if (s_stop) {
      t = k;
      break;
    }
    const uint32_t inv = s_inv;
    const int rem = w - k - 1;
    // multipliers l_j = S[j][k] / pivot, then the rank-1 update
    for (int e = threadIdx.x; e < rem; e += blockDim.x) {
      int j = k + 1 + e;
      S[j][k] = mod_mul(S[j][k], inv, mod);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < rem * rem; e += blockDim.x) {
      int j = k + 1 + e / rem, q = k + 1 + e % rem;
      uint32_t l = S[j][k];
      if (l) {
        uint32_t prod = mod_mul(l, S[k][q], mod);
        uint32_t v = S[j][q];
        S[j][q] = v >= prod ? v - prod : v + (p - prod);
      }
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < EW * EW; e += blockDim.x) {
    int r = e / EW, j = e % EW;
    blk[e] = S[r][j];
  }
  if (threadIdx.x == 0) {
    out[0] = (uint32_t)t;
    out[1] = (s_stop == 2) ? 1u : 0u;
  }
}

// Row permutation through a temporary: tmp[k] = D[src[k]] (full rows),
// then D[dst[k]] = tmp[k].
__global__ void gather_rows_kernel(const uint32_t *__restrict__ D, size_t ld, int n,
                                   const int *__restrict__ src, int cnt, uint32_t *__restrict__ tmp) {
  for (int k = blockIdx.y; k < cnt; k += gridDim.y) {
    const uint32_t *s = D + (size_t)src[k] * ld;
    uint32_t *d = tmp + (size_t)k * n;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
      d[j] = s[j];
  }
}
__global__ void scatter_rows_kernel(uint32_t *__restrict__ D, size_t ld, int n,
                                    const int *__restrict__ dst, int cnt,
                                    const uint32_t *__restrict__ tmp) {
  for (int k = blockIdx.y; k < cnt; k += gridDim.y) {
    uint32_t *d = D + (size_t)dst[k] * ld;
    const uint32_t *s = tmp + (size_t)k * n;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
      d[j] = s[j];
  }
}

// Pivot rows i..i+t-1, columns c..c+t-1 <- U11 (zeros below the diagonal).
__global__ void write_u11_kernel(uint32_t *__restrict__ D, size_t ld, int i, int c, int t,
                                 const uint32_t *__restrict__ blk) {
  for (int e = threadIdx.x; e < t * t; e += blockDim.x) {
    int r = e / t, j = e % t;
    D[(size_t)(i + r) * ld + c + j] = (j >= r) ? blk[r * EW + j] : 0u;
  }
}

// Rows r0..m-1: L[r - r0][k] = (D[r][c..c+t) * U11^-1)_k, then the block of
// D is zeroed (those entries are eliminated).  One thread per row.
__global__ void __launch_bounds__(128)
    right_solve_kernel(uint32_t *__restrict__ D, size_t ld, int r0, int m, int c, int t,
                       const uint32_t *__restrict__ blk, const uint32_t *__restrict__ pinv,
                       uint32_t *__restrict__ L, Modulus mod, uint32_t two64) {
  __shared__ uint32_t U[EW][EW + 1];
  __shared__ uint32_t sI[EW];
  for (int e = threadIdx.x; e < EW * EW; e += blockDim.x) {
    int r = e / EW, j = e % EW;
    U[r][j] = (r < t && j < t && j >= r) ? blk[r * EW + j] : 0u;
  }
  for (int e = threadIdx.x; e < EW; e += blockDim.x) sI[e] = e < t ? pinv[e] : 0u;
  __syncthreads();
  const int r = r0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= m) return;
  const uint32_t p = (uint32_t)mod.p;
  uint32_t *row = D + (size_t)r * ld + c;
  uint32_t x[EW];
#pragma unroll
  for (int k = 0; k < EW; ++k) x[k] = k < t ? row[k] : 0u;
  // x U = a: x_k = (a_k - sum_{j<k} x_j U[j][k]) / U[k][k]
#pragma unroll
  for (int k = 0; k < EW; ++k) {
    uint64_t s = 0;
#pragma unroll
    for (int j = 0; j < k; ++j) {
      uint64_t q = (uint64_t)x[j] * U[j][k];
      s += q;
      if (s < q) s += two64;
    }
    uint32_t red = mod_reduce(s, mod);
    uint32_t v = x[k] >= red ? x[k] - red : x[k] + (p - red);
    x[k] = mod_mul(v, sI[k], mod);
  }
  uint32_t *lrow = L + (size_t)(r - r0) * t;
#pragma unroll
  for (int k = 0; k < EW; ++k)
    if (k < t) {
      lrow[k] = x[k];
      row[k] = 0u;
    }
}

// Slow path: out[2] = first row q >= i with D[q][c] != 0 (0xFFFFFFFF if
// none); out[3] = 1 if row i has a nonzero in columns [c, n).
__global__ void column_search_kernel(const uint32_t *__restrict__ D, size_t ld, int i, int m,
                                     int c, int n, uint32_t *out) {
  for (int r = i + blockIdx.x * blockDim.x + threadIdx.x; r < m; r += gridDim.x * blockDim.x)
    if (D[(size_t)r * ld + c] != 0) atomicMin(&out[2], (uint32_t)r);
  if (blockIdx.x == 0 && i < m) {
    uint32_t any = 0;
    const uint32_t *row = D + (size_t)i * ld;
    for (int j = c + threadIdx.x; j < n; j += blockDim.x) any |= row[j];
    if (any) atomicOr(&out[3], 1u);
  }
}

static int sync_read(Ctx *c, uint32_t *dev, uint32_t *host, int words, const char *what) {
  cudaError_t e = cudaMemcpyAsync(host, dev, words * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                  c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, what);
}

int zp_echelon_dev(Ctx *c, int m, int n, uint32_t p, uint32_t *D, size_t ld, size_t *rank_out,
                   uint32_t *det_out, std::vector<int> *pivot_cols) {
  if (p < 2) return ctx_fail(c, ST_ARG, "modulus must be at least 2");
  if (m < 0 || n < 0) return ctx_fail(c, ST_ARG, "negative dimension");
  if (m > 0 && n > 0 && ld < (size_t)n) return ctx_fail(c, ST_ARG, "leading dimension too small");
  if (pivot_cols) pivot_cols->clear();
  uint64_t det = 1 % p;
  size_t rank = 0;
  if (m == 0 || n == 0) {
    *rank_out = 0;
    *det_out = (uint32_t)det;
    return ST_OK;
  }
  const Modulus mod = make_modulus(p);
  const uint32_t t64 = two64_mod(p);

  // device scratch: [blk 64x64][pinv 64][idx 2*m ints][flags m][L m x 64][tmp rows]
  const size_t blk_bytes = EW * EW * 4, pinv_bytes = EW * 4;
  const size_t idx_bytes = (size_t)2 * (m + EW) * sizeof(int);
  const size_t flag_bytes = ((size_t)m + 255) & ~(size_t)255;
  const size_t l_bytes = (size_t)m * EW * 4;
  const size_t tmp_bytes = (size_t)2 * EW * n * 4;
  void *base = nullptr;
  int st = ctx_buffer(c, BUF_ECH_0,
                      blk_bytes + pinv_bytes + idx_bytes + flag_bytes + l_bytes + tmp_bytes + 1024,
                      &base);
  if (st) return st;
  uint8_t *b8 = static_cast<uint8_t *>(base);
  uint32_t *d_blk = reinterpret_cast<uint32_t *>(b8);
  uint32_t *d_pinv = reinterpret_cast<uint32_t *>(b8 + blk_bytes);
  int *d_idx = reinterpret_cast<int *>(b8 + blk_bytes + pinv_bytes);
  uint8_t *d_flags = b8 + blk_bytes + pinv_bytes + idx_bytes;
  uint32_t *d_L = reinterpret_cast<uint32_t *>(d_flags + flag_bytes);
  uint32_t *d_tmp = d_L + (size_t)m * EW;
  void *gws = nullptr;
  st = ctx_workspace(c, zp_gemm_workspace_bytes(p, m, n, EW), &gws);
  if (st) return st;

  // which rows are identically zero
  std::vector<uint8_t> nz(m);
  {
    int grid = std::min((m * 32 + 255) / 256, c->num_sms * 8);
    row_nonzero_kernel<<<grid, 256, 0, c->stream>>>(D, ld, m, 0, n, d_flags);
    ctx_launched(c);
    cudaError_t e = cudaMemcpyAsync(nz.data(), d_flags, m, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return ctx_cuda(c, e, "echelon: zero-row scan");
  }

  std::vector<int> cand, at, src, dst;
  int i = 0, col = 0;
  while (i < m && col < n) {
    // 1. candidates
    cand.clear();
    for (int r = i; r < m && (int)cand.size() < EW; ++r)
      if (nz[r]) cand.push_back(r);
    if (cand.empty()) break;  // every remaining row is zero
    const int w = std::min<int>({EW, n - col, (int)cand.size()});
    cudaError_t e = cudaMemcpyAsync(d_idx, cand.data(), w * sizeof(int), cudaMemcpyHostToDevice,
                                    c->stream);
    if (e != cudaSuccess) return ctx_cuda(c, e, "echelon: candidates");
    cudaMemsetAsync(c->dstatus + 4, 0, 4 * sizeof(uint32_t), c->stream);
    int pi = prof_begin(c, "ech_block_lu");
    block_lu_kernel<<<1, 1024, 0, c->stream>>>(D, ld, d_idx, col, w, mod, d_blk, d_pinv,
                                               c->dstatus + 4);
    prof_end(c, pi);
    ctx_launched(c);
    uint32_t hs[2];
    if ((st = sync_read(c, c->dstatus + 4, hs, 2, "echelon: block LU"))) return st;
    const int t = (int)hs[0];
    if (hs[1]) return ctx_fail(c, ST_PIVOT, "Could not invert pivot-element in the ring");

    if (t > 0) {
      // 2. replay the transpositions of the t accepted pivots
      const int hi = cand[t - 1];
      at.resize(hi - i + 1);
      for (int q = i; q <= hi; ++q) at[q - i] = q;
      for (int k = 0; k < t; ++k) std::swap(at[k], at[cand[k] - i]);
      src.clear();
      dst.clear();
      for (int q = i; q <= hi; ++q)
        if (at[q - i] != q) {
          dst.push_back(q);
          src.push_back(at[q - i]);
        }
      if (!src.empty()) {
        const int cnt = (int)src.size();
        std::vector<uint8_t> nz_new(cnt);
        for (int k = 0; k < cnt; ++k) nz_new[k] = nz[src[k]];
        for (int k = 0; k < cnt; ++k) nz[dst[k]] = nz_new[k];
        std::vector<int> both(src);
        both.insert(both.end(), dst.begin(), dst.end());
        e = cudaMemcpyAsync(d_idx + EW, both.data(), both.size() * sizeof(int),
                            cudaMemcpyHostToDevice, c->stream);
        if (e != cudaSuccess) return ctx_cuda(c, e, "echelon: permutation");
        // t transpositions move at most 2t <= 2*EW rows, all gathered into
        // the temporary before any is written back.
        if (cnt > 2 * EW) return ctx_fail(c, ST_ARG, "echelon: permutation larger than expected");
        dim3 grid((n + 255) / 256, cnt);
        gather_rows_kernel<<<grid, 256, 0, c->stream>>>(D, ld, n, d_idx + EW, cnt, d_tmp);
        scatter_rows_kernel<<<grid, 256, 0, c->stream>>>(D, ld, n, d_idx + EW + cnt, cnt, d_tmp);
        ctx_launched(c, 2);
      }
      // 3. finish the block and update the trailing matrix
      write_u11_kernel<<<1, 1024, 0, c->stream>>>(D, ld, i, col, t, d_blk);
      ctx_launched(c);
      const int below = m - (i + t);
      if (below > 0) {
        pi = prof_begin(c, "ech_right_solve");
        right_solve_kernel<<<(below + 127) / 128, 128, 0, c->stream>>>(
            D, ld, i + t, m, col, t, d_blk, d_pinv, d_L, mod, t64);
        prof_end(c, pi);
        ctx_launched(c);
      }
      const int rest = n - (col + t);
      if (rest > 0) {
        // U12 = L11^-1 A12 (unit lower, stored below blk's diagonal)
        if ((st = tri_left_block(c, false, t, d_blk, EW, nullptr, D + (size_t)i * ld + col + t, ld,
                                 rest, p, 1)))
          return st;
        if (below > 0 &&
            (st = zp_gemm_dev(c, GEMM_AUTO, below, rest, t, p, p - 1, d_L, (size_t)t,
                              D + (size_t)i * ld + col + t, ld, 1,
                              D + (size_t)(i + t) * ld + col + t, ld,
                              static_cast<uint8_t *>(gws))))
          return st;
      }
      // det and pivot columns
      std::vector<uint32_t> diag(EW * EW);
      if ((st = sync_read(c, d_blk, diag.data(), EW * EW, "echelon: pivots"))) return st;
      for (int k = 0; k < t; ++k) {
        det = (det * diag[k * EW + k]) % p;
        if (pivot_cols) pivot_cols->push_back(col + k);
      }
      rank += t;
      i += t;
      col += t;
    }
    if (t < w && i < m && col < n) {
      // 4. zero pivot at (i, col): exact search of the updated column
      cudaMemsetAsync(c->dstatus + 6, 0xFF, sizeof(uint32_t), c->stream);
      cudaMemsetAsync(c->dstatus + 7, 0, sizeof(uint32_t), c->stream);
      int grid = std::min((m - i + 255) / 256, c->num_sms * 4);
      column_search_kernel<<<std::max(grid, 1), 256, 0, c->stream>>>(D, ld, i, m, col, n,
                                                                     c->dstatus + 4);
      ctx_launched(c);
      uint32_t hs2[2];
      if ((st = sync_read(c, c->dstatus + 6, hs2, 2, "echelon: column search"))) return st;
      if (!hs2[1]) nz[i] = 0;  // row i is zero from here on
      if (hs2[0] == 0xFFFFFFFFu) {
        ++col;  // no pivot in this column
      } else {
        const int q = (int)hs2[0];
        if (q != i) {
          // the transposition (i, q): tmp = [row q, row i]; D[i] = tmp[0],
          // D[q] = tmp[1].  (Pageable host sources are staged by the copy
          // call itself, so the local array may go out of scope.)
          std::swap(nz[i], nz[q]);
          int idx4[4] = {q, i, i, q};
          e = cudaMemcpyAsync(d_idx + EW, idx4, sizeof idx4, cudaMemcpyHostToDevice, c->stream);
          if (e != cudaSuccess) return ctx_cuda(c, e, "echelon: swap");
          dim3 g2((n + 255) / 256, 2);
          gather_rows_kernel<<<g2, 256, 0, c->stream>>>(D, ld, n, d_idx + EW, 2, d_tmp);
          scatter_rows_kernel<<<g2, 256, 0, c->stream>>>(D, ld, n, d_idx + EW + 2, 2, d_tmp);
          ctx_launched(c, 2);
        }
        nz[i] = 1;
      }
    }
  }
  *rank_out = rank;
  *det_out = (uint32_t)det;
  return ST_OK;
}

}  // namespace lela
