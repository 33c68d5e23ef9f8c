// lela_b200/csrc/tri.cu -- triangular solves over Z/p (Modular<uint32>).
//
//   B <- alpha * A^-1 * B,  A m x m upper or lower triangular, unit or
//   non-unit diagonal, B m x n.
//
// Replaces _trsm<Ring, GenericModule::Tag>::trsm_impl (lela/blas/
// level3-generic.tcc:421-498) for dense operands.  The recursion is the
// reference's (split at l ~ m/2; lower: solve A11, B2 <- alpha*B2 - A21*B1,
// solve A22 with coefficient 1; upper: A22 first, then B1 <- alpha*B1 -
// A12*B2, then A11), with the off-diagonal updates on the limb-split
// tensor-core gemm.  The diagonal leaves are either 256-row blocks solved by
// substitution on CUDA cores, or (from 1024 rows) 512-row blocks whose
// inverses are built once and applied by the tensor-core gemm.
//
// Sparse operands.  When the caller says A may be sparse (Faugere-
// Lachartre's pivot block, the CSR entry point), the occupancy of A's 64 x 64
// tiles is read once (one kernel, one copy to the host), and every
// off-diagonal update of the recursion runs only over the bounding box of
// the occupied tiles of its block of A: the rows of B outside the box get
// no update (only the alpha scaling), and the columns outside it multiply
// zero.  The result is the same; for F4 pivot blocks, whose nonzeros lie in
// a band above the diagonal, the update work drops by about 3x at m = 20000.
//
// Error behaviour.  With alpha = 0 the reference returns alpha*B = 0
// without looking at A (:433-434); otherwise a diagonal entry that
// Modular<uint32>::inv cannot invert throws DiagonalEntryNotInvertible(idx)
// where idx is the first such entry in the recursion's visiting order: the
// smallest index for lower, the largest for upper.  Here all diagonal
// inverses are computed first (one kernel); on failure the same idx is
// reported and B is left unchanged (the reference leaves it partially
// solved, which callers such as Faugere-Lachartre discard).
#include <algorithm>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "context.h"
#include "tri.h"
#include "zp_gemm.h"

namespace lela {

constexpr int TRI_NB = 64;

// dinv[i] = inverse of A(i,i) (1 for a unit diagonal).  Failures record the
// smallest (status[1]) and largest + 1 (status[2]) failing index.
__global__ void diag_inverse_kernel(const uint32_t *__restrict__ A, size_t lda, int m, uint32_t p,
                                    uint32_t *__restrict__ dinv, uint32_t *status) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    uint32_t v = lela_inv_u32(p, A[(size_t)i * lda + i]);
    dinv[i] = v;
    if (v == 0) {
      atomicMin(&status[1], (uint32_t)i);
      atomicMax(&status[2], (uint32_t)i + 1);
    }
  }
}

// occ[bi * tn + bj] = 1 when tile (bi, bj) (TRI_NB x TRI_NB) of the m x m
// matrix A holds a nonzero entry.  Tiles on the other side of the diagonal
// than the triangle are not read (0).  One CTA of 256 threads per tile;
// warp w reads 8 of its rows, two 128-byte segments per row.
__global__ void __launch_bounds__(256)
    tile_occupancy_kernel(const uint32_t *__restrict__ A, size_t lda, int m, int tn, bool upper,
                          uint8_t *__restrict__ occ) {
  const int bi = blockIdx.y, bj = blockIdx.x;
  if (upper ? bj < bi : bj > bi) {
    if (threadIdx.x == 0) occ[(size_t)bi * tn + bj] = 0;
    return;
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int c0 = bj * TRI_NB + lane, c1 = c0 + 32;
  bool nz = false;
  for (int rr = 0; rr < TRI_NB / 8; ++rr) {
    const int r = bi * TRI_NB + w * (TRI_NB / 8) + rr;
    if (r >= m) break;
    const uint32_t *row = A + (size_t)r * lda;
    nz |= (c0 < m && row[c0] != 0u) || (c1 < m && row[c1] != 0u);
  }
  nz = __syncthreads_or(nz);
  if (threadIdx.x == 0) occ[(size_t)bi * tn + bj] = nz ? 1 : 0;
}

// Solve T x = x in place for one column held by a quad of threads: thread q
// holds the entries k = 4i + q (x[i]); T (nb x nb, nb <= 64, lower or upper
// triangular) is in shared memory with its inverted diagonal sD (unitd: 1).
// Right-looking: each thread keeps, per entry it holds, the 64-bit sum of
// the products T[j][k] x[k] of the entries already solved (the reference's
// wrap-around correction, +2^64 mod p, when NOWRAP is false; with p < 2^28
// the sums cannot wrap).  Step k: the owner of k reduces its sum and
// finishes x[k], one shuffle hands x[k] to the quad, and every thread adds
// T[j][k] x[k] into the sums of its entries j still to solve -- sixteen
// independent multiply-adds, so the sequential chain per step is one
// reduction, one shuffle and one multiply-add.  The entries of the current
// group of four (k / 4) sit in slot CUR: after each group the registers
// rotate by one, so no step needs a dynamic register index, and after the
// sixteen groups they are back in place.  Entries from nb on are zero and
// never solved.
template <bool UPPER, bool NOWRAP>
__device__ __forceinline__ void tri_quad_solve(const uint32_t (*sT)[TRI_NB + 1],
                                               const uint32_t *sD, bool unitd, int nb, int q,
                                               uint32_t (&x)[TRI_NB / 4], const Modulus &mod,
                                               uint32_t two64) {
  constexpr int NI = TRI_NB / 4;
  constexpr int CUR = UPPER ? NI - 1 : 0;  // slot s holds group (g + s - CUR) mod NI
  const uint32_t p = (uint32_t)mod.p;
  const int qbase = (threadIdx.x & 31) & ~3;
  const int last = (nb - 1) >> 2;  // last group with an entry
  uint64_t acc[NI];
#pragma unroll
  for (int i = 0; i < NI; ++i) acc[i] = 0ull;
#pragma unroll 1
  for (int gg = 0; gg < NI; ++gg) {
    const int g = UPPER ? NI - 1 - gg : gg;
    if (g <= last) {
#pragma unroll
      for (int rr = 0; rr < 4; ++rr) {
        const int r = UPPER ? 3 - rr : rr;
        const int k = 4 * g + r;
        if (k < nb) {
          // every lane forms its candidate; the owner's (q == r) is x[k]
          const uint32_t red = mod_reduce(acc[CUR], mod);
          uint32_t v = x[CUR] >= red ? x[CUR] - red : x[CUR] + (p - red);
          if (!unitd) v = mod_mul(v, sD[k], mod);
          if (q == r) x[CUR] = v;
          v = __shfl_sync(0xffffffffu, v, qbase + r);
#pragma unroll
          for (int sl = 0; sl < NI; ++sl) {
            const int j = 4 * ((g + sl - CUR) & (NI - 1)) + q;
            if (UPPER ? j < k : j > k) {
              const uint64_t t = (uint64_t)sT[j][k] * v;
              acc[sl] += t;
              if (!NOWRAP && acc[sl] < t) acc[sl] += two64;
            }
          }
        }
      }
    }
    // the next group into slot CUR
    if (UPPER) {
      const uint32_t xe = x[NI - 1];
      const uint64_t ae = acc[NI - 1];
#pragma unroll
      for (int sl = NI - 1; sl > 0; --sl) {
        x[sl] = x[sl - 1];
        acc[sl] = acc[sl - 1];
      }
      x[0] = xe;
      acc[0] = ae;
    } else {
      const uint32_t xe = x[0];
      const uint64_t ae = acc[0];
#pragma unroll
      for (int sl = 0; sl < NI - 1; ++sl) {
        x[sl] = x[sl + 1];
        acc[sl] = acc[sl + 1];
      }
      x[NI - 1] = xe;
      acc[NI - 1] = ae;
    }
  }
}

// Left solve of one diagonal block: for every column of B (a quad of
// threads each), x <- alpha * T^-1 x, T = nb x nb (nb <= 64) lower or upper
// triangular with inverted diagonal dinv (nullptr: unit diagonal).
template <bool UPPER, bool NOWRAP>
__global__ void __launch_bounds__(128)
    tri_left_kernel(const uint32_t *__restrict__ T, size_t ldt, int nb,
                    const uint32_t *__restrict__ dinv, uint32_t *__restrict__ B, size_t ldb,
                    int ncols, Modulus mod, uint32_t two64, uint32_t alpha) {
  __shared__ uint32_t sT[TRI_NB][TRI_NB + 1];
  __shared__ uint32_t sD[TRI_NB];
  // asynchronous copies, all in flight at once (entries outside nb x nb are
  // zero-filled)
  for (int e = threadIdx.x; e < TRI_NB * TRI_NB; e += blockDim.x) {
    const int r = e / TRI_NB, cc = e % TRI_NB;
    const bool in = r < nb && cc < nb;
    cp_async4(&sT[r][cc], in ? T + (size_t)r * ldt + cc : T, in);
  }
  for (int e = threadIdx.x; e < TRI_NB; e += blockDim.x) sD[e] = (e < nb && dinv) ? dinv[e] : 1u;
  cp_async_wait_all();
  __syncthreads();
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int col = gt >> 2, q = gt & 3;
  const bool ok = col < ncols;  // every lane stays for the quad's shuffles
  uint32_t x[TRI_NB / 4];
#pragma unroll
  for (int i = 0; i < TRI_NB / 4; ++i) {
    const int k = 4 * i + q;
    const uint32_t v = (ok && k < nb) ? B[(size_t)k * ldb + col] : 0u;
    x[i] = (alpha == 1u) ? v : mod_mul(v, alpha, mod);
  }
  tri_quad_solve<UPPER, NOWRAP>(sT, sD, dinv == nullptr, nb, q, x, mod, two64);
  if (ok)
#pragma unroll
    for (int i = 0; i < TRI_NB / 4; ++i) {
      const int k = 4 * i + q;
      if (k < nb) B[(size_t)k * ldb + col] = x[i];
    }
}

// Inverses of all diagonal blocks at once: block b (rows/cols 64b ..
// 64b+nb) of the triangular A; one CTA of 256 threads per block, a quad per
// column j solving T x = e_j.  Out: the 64 x 64 inverse (zero padded) at
// rows 64b.. of Tinv (row stride ldo), columns (64b mod cmod)..: ldo = cmod
// = 64 stores the blocks one after the other; ldo = cmod = NB places them
// on the diagonal of the NB-row block inverses.
template <bool UPPER>
__global__ void __launch_bounds__(256)
    tri_inv_blocks_kernel(const uint32_t *__restrict__ A, size_t lda, int m,
                          const uint32_t *__restrict__ dinv, uint32_t *__restrict__ Tinv,
                          size_t ldo, int cmod, Modulus mod, uint32_t two64) {
  __shared__ uint32_t sT[TRI_NB][TRI_NB + 1];
  __shared__ uint32_t sD[TRI_NB];
  const int b = blockIdx.x;
  const int r0 = b * TRI_NB;
  const int nb = min(TRI_NB, m - r0);
  const uint32_t *T = A + (size_t)r0 * lda + r0;
  for (int e = threadIdx.x; e < TRI_NB * TRI_NB; e += blockDim.x) {
    const int r = e / TRI_NB, cc = e % TRI_NB;
    const bool in = r < nb && cc < nb;
    cp_async4(&sT[r][cc], in ? T + (size_t)r * lda + cc : T, in);
  }
  for (int e = threadIdx.x; e < TRI_NB; e += blockDim.x) sD[e] = (e < nb && dinv) ? dinv[r0 + e] : 1u;
  cp_async_wait_all();
  __syncthreads();
  const int j = threadIdx.x >> 2, q = threadIdx.x & 3;
  uint32_t x[TRI_NB / 4];
#pragma unroll
  for (int i = 0; i < TRI_NB / 4; ++i) x[i] = (4 * i + q == j && j < nb) ? 1u : 0u;
  tri_quad_solve<UPPER, false>(sT, sD, dinv == nullptr, nb, q, x, mod, two64);
  uint32_t *out = Tinv + (size_t)r0 * ldo + r0 % cmod;
#pragma unroll
  for (int i = 0; i < TRI_NB / 4; ++i) out[(size_t)(4 * i + q) * ldo + j] = (j < nb) ? x[i] : 0u;
}

// ----------------------------------------------------------- inverse leaves
// For wide right-hand sides the diagonal blocks of TI_NB rows (aligned to
// multiples of TI_NB from the top-left) are inverted once, and each leaf of
// the recursion becomes B_leaf <- alpha * inv(A_leaf) * B_leaf on the
// tensor-core gemm.  The triangular system has a unique solution (every
// diagonal entry is a unit, checked first), so the result is the
// substitution's.  The inverses are assembled from the 64-row ones by
// doubling: for a block [[A11, A12], [0, A22]] with inverses I11, I22 of its
// halves, inv = [[I11, -I11 A12 I22], [0, I22]] (lower: the off-diagonal
// block is -I22 A21 I11).  W (rows x TI_NB) holds the inverse of leaf b in
// its rows TI_NB b .., columns 0 ..; every level writes its off-diagonal
// blocks in place.
constexpr int TI_NB = 512;
constexpr int MG_T = 64, MG_K = 32;

// One operand of a batched merge product: entry (i, j) of instance z sits at
// ptr[(z rs + ro + i) ld + (z cs + co) mod cmod + j].
struct MergeOp {
  const uint32_t *ptr;
  size_t ld;
  int rs, ro, cs, co, cmod;
  __host__ __device__ const uint32_t *at(int z) const {
    return ptr + (size_t)(z * rs + ro) * ld + (z * cs + co) % cmod;
  }
};

// C_z <- alpha X_z Y_z (M x N, inner dimension K) for the instances
// z = zbase + blockIdx.z; 64 x 64 tiles as the small-K gemm.  NOWRAP
// (p < 2^28): unchecked sums reduced every 256 terms.
template <bool NOWRAP>
__global__ void __launch_bounds__(256)
    tri_merge_kernel(MergeOp X, MergeOp Y, MergeOp Cop, int zbase, int M, int N, int K,
                     Modulus mod, uint32_t two64, uint32_t alpha) {
  __shared__ uint32_t Xs[MG_K][MG_T + 1];
  __shared__ uint32_t Ys[MG_K][MG_T + 1];
  const int z = zbase + blockIdx.z;
  const uint32_t *__restrict__ Xp = X.at(z);
  const uint32_t *__restrict__ Yp = Y.at(z);
  uint32_t *Cp = const_cast<uint32_t *>(Cop.at(z));
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int m0 = blockIdx.y * MG_T, n0 = blockIdx.x * MG_T;
  uint64_t acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0;
  for (int k0 = 0; k0 < K; k0 += MG_K) {
#pragma unroll
    for (int e = 0; e < (MG_T * MG_K) / 256; ++e) {
      const int idx = threadIdx.x + 256 * e;
      const int r = idx / MG_K, kk = idx % MG_K;
      const int gm = m0 + r, gk = k0 + kk;
      Xs[kk][r] = (gm < M && gk < K) ? Xp[(size_t)gm * X.ld + gk] : 0u;
      const int kr = idx / MG_T, cc = idx % MG_T;
      const int gk2 = k0 + kr, gn = n0 + cc;
      Ys[kr][cc] = (gk2 < K && gn < N) ? Yp[(size_t)gk2 * Y.ld + gn] : 0u;
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < MG_K; ++kk) {
      uint32_t a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = Xs[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Ys[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const uint64_t t = (uint64_t)a[i] * b[j];
          if (NOWRAP) {
            acc[i][j] += t;
          } else {
            const uint64_t s = acc[i][j] + t;
            acc[i][j] = (s < t) ? s + two64 : s;
          }
        }
    }
    if (NOWRAP && ((k0 / MG_K) & 7) == 7)
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = mod_reduce(acc[i][j], mod);
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int gm = m0 + ty + 16 * i;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gn = n0 + tx + 16 * j;
      if (gn < N) Cp[(size_t)gm * Cop.ld + gn] = mod_mul(mod_reduce(acc[i][j], mod), alpha, mod);
    }
  }
}

// C <- beta * C for an m x n block (beta in [0, p)).
__global__ void zp_scale2_kernel(uint32_t *C, size_t ldc, int M, int N, Modulus mod,
                                 uint32_t beta) {
  const size_t total = (size_t)M * N;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    size_t r = idx / N, cc = idx % N;
    uint32_t *x = C + r * ldc + cc;
    *x = beta ? mod_mul(*x, beta, mod) : 0u;
  }
}

int tri_left_block(Ctx *c, bool upper, int nb, const uint32_t *T, size_t ldt,
                   const uint32_t *dinv, uint32_t *B, size_t ldb, int ncols, uint32_t p,
                   uint32_t alpha) {
  if (nb <= 0 || ncols <= 0) return ST_OK;
  const Modulus mod = make_modulus(p);
  const uint32_t t64 = two64_mod(p);
  const int threads = 128;  // 32 columns, four threads each
  const int grid = (ncols * 4 + threads - 1) / threads;
  const bool nowrap = p < (1u << 28);
  int pi = prof_begin(c, "tri_left");
  if (upper && nowrap)
    tri_left_kernel<true, true><<<grid, threads, 0, c->stream>>>(T, ldt, nb, dinv, B, ldb, ncols,
                                                                 mod, t64, alpha);
  else if (upper)
    tri_left_kernel<true, false><<<grid, threads, 0, c->stream>>>(T, ldt, nb, dinv, B, ldb, ncols,
                                                                  mod, t64, alpha);
  else if (nowrap)
    tri_left_kernel<false, true><<<grid, threads, 0, c->stream>>>(T, ldt, nb, dinv, B, ldb, ncols,
                                                                  mod, t64, alpha);
  else
    tri_left_kernel<false, false><<<grid, threads, 0, c->stream>>>(T, ldt, nb, dinv, B, ldb, ncols,
                                                                   mod, t64, alpha);
  prof_end(c, pi);
  ctx_launched(c);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "tri_left launch");
}

// Inverted diagonal blocks of the whole system: the leaf whose top-left
// entry is A_base[off*(lda+1)] uses tinv + (off/64) * 64*64 (leaves start
// at multiples of 64 because every split point is one).
struct TriLeaves {
  const uint32_t *A_base;
  const uint32_t *tinv;
};

// Diagonal blocks of up to TB_NB rows in one launch: each CTA holds a
// CT-column slice of the block's B in shared memory and runs the whole
// block's substitution over its 64-row sub-blocks (upper: last first): the
// sub-block's rows minus A's off-diagonal 64 x 64 tiles times the solved
// sub-blocks, then times the inverted diagonal 64-block.  A thread owns a
// register tile of RPT rows x 4 columns.  NOWRAP (p < 2^28): 64-term sums
// cannot wrap, no per-term check.
constexpr int TB_NB = 256;
constexpr int TB_THREADS = 256;

template <bool UPPER, bool NOWRAP, int CT>
__global__ void __launch_bounds__(TB_THREADS)
    tri_block_kernel(const uint32_t *__restrict__ A, size_t lda, const uint32_t *__restrict__ Tinv,
                     int nb, uint32_t *__restrict__ B, size_t ldb, int ncols, Modulus mod,
                     uint32_t two64, uint32_t alpha) {
  constexpr int CG = CT / 4;              // column groups (4 columns each, stride CG)
  constexpr int RG = TB_THREADS / CG;     // row groups
  constexpr int RPT = TRI_NB / RG;        // rows per thread within a 64-row sub-block
  extern __shared__ uint32_t Xs[];        // nb x CT
  __shared__ uint32_t At[TRI_NB][TRI_NB + 1];
  const int tid = threadIdx.x, cg = tid % CG, rg = tid / CG;
  const int c0 = blockIdx.x * CT;
  const uint32_t p = (uint32_t)mod.p;
  // tiles come in through asynchronous copies (all in flight at once)
  for (int e = tid; e < nb * CT; e += TB_THREADS) {
    const int r = e / CT, cc = e % CT;
    const bool ok = c0 + cc < ncols;
    cp_async4(&Xs[e], ok ? B + (size_t)r * ldb + c0 + cc : B, ok);
  }
  cp_async_wait_all();
  if (alpha != 1u)
    for (int e = tid; e < nb * CT; e += TB_THREADS) Xs[e] = mod_mul(Xs[e], alpha, mod);
  const int nsb = (nb + TRI_NB - 1) / TRI_NB;
  for (int jj = 0; jj < nsb; ++jj) {
    const int j = UPPER ? nsb - 1 - jj : jj;
    const int r0 = j * TRI_NB, bj = min(TRI_NB, nb - r0);
    __syncthreads();  // Xs written by the previous sub-block (or the load)
    uint32_t y[RPT][4];
#pragma unroll
    for (int u = 0; u < RPT; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int r = rg * RPT + u;
        y[u][v] = r < bj ? Xs[(r0 + r) * CT + cg + CG * v] : 0u;
      }
    const int jlo = UPPER ? j + 1 : 0, jhi = UPPER ? nsb : j;
    for (int j2 = jlo; j2 <= jhi; ++j2) {
      // j2 < jhi (or > j for upper): an off-diagonal tile; the last pass
      // (j2 == jhi) applies the inverted diagonal block to y
      const bool diag = j2 == jhi;
      const int k0 = diag ? r0 : j2 * TRI_NB, bk = diag ? bj : min(TRI_NB, nb - k0);
      __syncthreads();  // At is free; for diag, every thread has read Xs below
      if (diag) {
#pragma unroll
        for (int u = 0; u < RPT; ++u)
#pragma unroll
          for (int v = 0; v < 4; ++v) {
            const int r = rg * RPT + u;
            if (r < bj) Xs[(r0 + r) * CT + cg + CG * v] = y[u][v];
          }
        const uint32_t *T = Tinv + (size_t)j * TRI_NB * TRI_NB;
        for (int e = tid; e < TRI_NB * TRI_NB; e += TB_THREADS)
          cp_async4(&At[e / TRI_NB][e % TRI_NB], T + e, true);
      } else {
        for (int e = tid; e < TRI_NB * TRI_NB; e += TB_THREADS) {
          const int rr = e / TRI_NB, kk = e % TRI_NB;
          const bool ok = rr < bj && kk < bk;
          cp_async4(&At[rr][kk], ok ? A + (size_t)(r0 + rr) * lda + k0 + kk : A, ok);
        }
      }
      cp_async_wait_all();
      __syncthreads();
      uint64_t s[RPT][4];
#pragma unroll
      for (int u = 0; u < RPT; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) s[u][v] = 0;
      for (int k = 0; k < bk; ++k) {
        uint32_t xv[4], av[RPT];
#pragma unroll
        for (int v = 0; v < 4; ++v) xv[v] = Xs[(k0 + k) * CT + cg + CG * v];
#pragma unroll
        for (int u = 0; u < RPT; ++u) av[u] = At[rg * RPT + u][k];
#pragma unroll
        for (int u = 0; u < RPT; ++u)
#pragma unroll
          for (int v = 0; v < 4; ++v) {
            const uint64_t t = (uint64_t)av[u] * xv[v];
            s[u][v] += t;
            if (!NOWRAP && s[u][v] < t) s[u][v] += two64;
          }
      }
#pragma unroll
      for (int u = 0; u < RPT; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const uint32_t w = mod_reduce(s[u][v], mod);
          y[u][v] = diag ? w : (y[u][v] >= w ? y[u][v] - w : y[u][v] + (p - w));
        }
    }
    __syncthreads();  // every thread has read the sub-block's right-hand sides
#pragma unroll
    for (int u = 0; u < RPT; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int r = rg * RPT + u;
        if (r < bj) Xs[(r0 + r) * CT + cg + CG * v] = y[u][v];
      }
  }
  __syncthreads();
  for (int e = tid; e < nb * CT; e += TB_THREADS) {
    const int r = e / CT, cc = e % CT;
    if (c0 + cc < ncols) B[(size_t)r * ldb + c0 + cc] = Xs[e];
  }
}

static int tri_block(Ctx *c, const TriLeaves &L, bool upper, int m, const uint32_t *A, size_t lda,
                     uint32_t *B, size_t ldb, int n, uint32_t p, uint32_t alpha) {
  if (n <= 0) return ST_OK;
  {
    const void *fns[8] = {
        (const void *)tri_block_kernel<true, true, 64>, (const void *)tri_block_kernel<true, false, 64>,
        (const void *)tri_block_kernel<false, true, 64>, (const void *)tri_block_kernel<false, false, 64>,
        (const void *)tri_block_kernel<true, true, 32>, (const void *)tri_block_kernel<true, false, 32>,
        (const void *)tri_block_kernel<false, true, 32>, (const void *)tri_block_kernel<false, false, 32>};
    for (int k = 0; k < 8; ++k)
      if (int st = ctx_smem_attr(c, fns[k], TB_NB * (k < 4 ? 64 : 32) * 4,
                                 "cudaFuncSetAttribute(tri_block)"))
        return st;
  }
  const size_t off = (size_t)(A - L.A_base) / (lda + 1);
  const uint32_t *T = L.tinv + (off / TRI_NB) * TRI_NB * TRI_NB;
  const Modulus mod = make_modulus(p);
  const uint32_t t64 = two64_mod(p);
  // 64-column slices when they still give every SM a CTA, else 32
  const bool wide = n >= 64 * c->num_sms;
  const int ct = wide ? 64 : 32;
  const int grid = (n + ct - 1) / ct;
  const size_t smem = (size_t)m * ct * 4;
  const bool nowrap = p < (1u << 28);
  int pi = prof_begin(c, "tri_block");
#define TB_LAUNCH(U, W, C)                                                              \
  tri_block_kernel<U, W, C><<<grid, TB_THREADS, smem, c->stream>>>(A, lda, T, m, B, ldb, n, \
                                                                   mod, t64, alpha)
  if (wide) {
    if (upper && nowrap) TB_LAUNCH(true, true, 64);
    else if (upper) TB_LAUNCH(true, false, 64);
    else if (nowrap) TB_LAUNCH(false, true, 64);
    else TB_LAUNCH(false, false, 64);
  } else {
    if (upper && nowrap) TB_LAUNCH(true, true, 32);
    else if (upper) TB_LAUNCH(true, false, 32);
    else if (nowrap) TB_LAUNCH(false, true, 32);
    else TB_LAUNCH(false, false, 32);
  }
#undef TB_LAUNCH
  prof_end(c, pi);
  ctx_launched(c);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "tri_block launch");
}

// Occupied TRI_NB-tiles of A (host copy): a summed-area table over the
// tile grid answers "which rows / columns of this block hold nonzeros".
struct TileMap {
  int tn = 0;
  std::vector<int> S;            // (tn + 1)^2 prefix counts
  const int2 *kr = nullptr;      // per-row column ranges of A (device), or null
  int count(int i0, int i1, int j0, int j1) const {
    const int w = tn + 1;
    return S[(size_t)i1 * w + j1] - S[(size_t)i0 * w + j1] - S[(size_t)i1 * w + j0] +
           S[(size_t)i0 * w + j0];
  }
  // Bounding box, in entries, of the occupied tiles of rows [r0, r1) x
  // columns [c0, c1) of A (r0, c0 multiples of TRI_NB); false when empty.
  bool box(int r0, int r1, int c0, int c1, int &br0, int &br1, int &bc0, int &bc1) const {
    const int i0 = r0 / TRI_NB, i1 = (r1 + TRI_NB - 1) / TRI_NB;
    const int j0 = c0 / TRI_NB, j1 = (c1 + TRI_NB - 1) / TRI_NB;
    if (count(i0, i1, j0, j1) == 0) return false;
    int a = i0, b = i1, x = j0, y = j1;
    while (count(a, a + 1, j0, j1) == 0) ++a;
    while (count(b - 1, b, j0, j1) == 0) --b;
    while (count(i0, i1, x, x + 1) == 0) ++x;
    while (count(i0, i1, y - 1, y) == 0) --y;
    br0 = a * TRI_NB;
    br1 = std::min(r1, b * TRI_NB);
    bc0 = x * TRI_NB;
    bc1 = std::min(c1, y * TRI_NB);
    return true;
  }
};

static int build_tile_map(Ctx *c, bool upper, int m, const uint32_t *A, size_t lda, TileMap *tm) {
  const int tn = (m + TRI_NB - 1) / TRI_NB;
  void *buf = nullptr;
  int st = ctx_buffer(c, BUF_TRI_OCC, (size_t)tn * tn, &buf);
  if (st) return st;
  uint8_t *d_occ = static_cast<uint8_t *>(buf);
  tile_occupancy_kernel<<<dim3(tn, tn), 256, 0, c->stream>>>(A, lda, m, tn, upper, d_occ);
  ctx_launched(c);
  std::vector<uint8_t> occ((size_t)tn * tn);
  cudaError_t e = cudaMemcpyAsync(occ.data(), d_occ, occ.size(), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return ctx_cuda(c, e, "trsm: tile occupancy");
  tm->tn = tn;
  const int w = tn + 1;
  tm->S.assign((size_t)w * w, 0);
  for (int i = 0; i < tn; ++i)
    for (int j = 0; j < tn; ++j)
      tm->S[(size_t)(i + 1) * w + j + 1] = occ[(size_t)i * tn + j] + tm->S[(size_t)i * w + j + 1] +
                                           tm->S[(size_t)(i + 1) * w + j] - tm->S[(size_t)i * w + j];
  return ST_OK;
}

// The off-diagonal update of the recursion, Bd <- alpha Bd - Ablk Bs, where
// Ablk (rows x cols) is the block of A at rows ar, columns ac of the whole
// matrix.  With a tile map only its occupied bounding box is multiplied; the
// other rows of Bd are scaled by alpha (nothing to do for alpha = 1).
static int tri_update(Ctx *c, const TileMap *tm, int ar, int ac, int rows, int cols, int n,
                      uint32_t p, uint32_t alpha, const uint32_t *Ablk, size_t lda,
                      const uint32_t *Bs, uint32_t *Bd, size_t ldb, uint8_t *gemm_ws) {
  if (!tm)
    return zp_gemm_dev(c, GEMM_AUTO, rows, n, cols, p, p - 1, Ablk, lda, Bs, ldb, alpha, Bd, ldb,
                       gemm_ws);
  int r0, r1, c0, c1;
  const bool any = tm->box(ar, ar + rows, ac, ac + cols, r0, r1, c0, c1);
  if (!any) {
    r0 = r1 = ar;
    c0 = c1 = ac;
  }
  const int lo = r0 - ar, hi = r1 - ar;  // rows of Bd that get a product
  if (alpha != 1u && n > 0) {
    const Modulus mod = make_modulus(p);
    auto scale = [&](int a, int b) {
      if (b <= a) return;
      const size_t total = (size_t)(b - a) * n;
      const int grid = (int)std::min<size_t>((total + 255) / 256, (size_t)c->num_sms * 8);
      zp_scale2_kernel<<<grid, 256, 0, c->stream>>>(Bd + (size_t)a * ldb, ldb, b - a, n, mod, alpha);
      ctx_launched(c);
    };
    scale(0, lo);
    scale(hi, rows);
  }
  if (!any) return ST_OK;
  return zp_gemm_dev(c, GEMM_AUTO, hi - lo, n, c1 - c0, p, p - 1,
                     Ablk + (size_t)lo * lda + (c0 - ac), lda, Bs + (size_t)(c0 - ac) * ldb, ldb,
                     alpha, Bd + (size_t)lo * ldb, ldb, gemm_ws,
                     tm->kr ? tm->kr + (ar + lo) : nullptr, c0);
}

// Recursive solve (dinv is the inverted diagonal of the current sub-system,
// whose top-left entry is A's entry (off, off)).
static int trsm_rec(Ctx *c, const TriLeaves &TL, const TileMap *tm, int off, bool upper, int m,
                    int n, uint32_t p, uint32_t alpha, const uint32_t *A, size_t lda,
                    const uint32_t *dinv, uint32_t *B, size_t ldb, uint8_t *gemm_ws) {
  if (m <= 0) return ST_OK;
  if (m <= TB_NB) return tri_block(c, TL, upper, m, A, lda, B, ldb, n, p, alpha);
  // split at a multiple of the leaf size, near the middle
  int l = ((m / 2 + TRI_NB - 1) / TRI_NB) * TRI_NB;
  if (l >= m) l = m - TRI_NB;
  const uint32_t *A11 = A, *A12 = A + l, *A21 = A + (size_t)l * lda, *A22 = A21 + l;
  uint32_t *B1 = B, *B2 = B + (size_t)l * ldb;
  int st;
  if (!upper) {
    if ((st = trsm_rec(c, TL, tm, off, upper, l, n, p, alpha, A11, lda, dinv, B1, ldb, gemm_ws)))
      return st;
    if ((st = tri_update(c, tm, off + l, off, m - l, l, n, p, alpha, A21, lda, B1, B2, ldb,
                         gemm_ws)))
      return st;
    return trsm_rec(c, TL, tm, off + l, upper, m - l, n, p, 1, A22, lda,
                    dinv ? dinv + l : nullptr, B2, ldb, gemm_ws);
  } else {
    if ((st = trsm_rec(c, TL, tm, off + l, upper, m - l, n, p, alpha, A22, lda,
                       dinv ? dinv + l : nullptr, B2, ldb, gemm_ws)))
      return st;
    if ((st = tri_update(c, tm, off, off + l, l, m - l, n, p, alpha, A12, lda, B2, B1, ldb,
                         gemm_ws)))
      return st;
    return trsm_rec(c, TL, tm, off, upper, l, n, p, 1, A11, lda, dinv, B1, ldb, gemm_ws);
  }
}

// Off-diagonal blocks of the TI_NB-row diagonal block inverses, level by
// level (block size s = 128, 256, .., TI_NB), on W whose diagonal 64-blocks
// hold the 64-row inverses and whose other entries are zero.  T: scratch of
// (m / TI_NB + 1) * (TI_NB / 2)^2 entries (the largest level's need).
static int tri_inverse_levels(Ctx *c, bool upper, int m, uint32_t p, const uint32_t *A,
                              size_t lda, uint32_t *W, uint32_t *T) {
  const Modulus mod = make_modulus(p);
  const uint32_t t64 = two64_mod(p);
  const bool nowrap = p < (1u << 28);
  constexpr int NOMOD = 1 << 30;
  for (int s = 2 * TRI_NB; s <= TI_NB && s / 2 < m; s *= 2) {
    const int h = s / 2;
    const int nfull = m / s;
    const int h2p = m - nfull * s - h;  // second half of the last, partial block
    for (int pass = 0; pass < 2; ++pass) {
      const int zbase = pass ? nfull : 0, nz = pass ? 1 : nfull, h2 = pass ? h2p : h;
      if (nz <= 0 || h2 <= 0) continue;
      const MergeOp Tz{T, (size_t)h, h, 0, 0, 0, NOMOD};
      MergeOp X1, Y1, X2, C2;
      int M1, N1, K1, M2, N2, K2;
      if (upper) {
        // T = A12 I22 (h x h2); W12 = -I11 T
        X1 = {A, lda, s, 0, s, h, NOMOD};
        Y1 = {W, (size_t)TI_NB, s, h, s, h, TI_NB};
        X2 = {W, (size_t)TI_NB, s, 0, s, 0, TI_NB};
        C2 = {W, (size_t)TI_NB, s, 0, s, h, TI_NB};
        M1 = h, N1 = h2, K1 = h2, M2 = h, N2 = h2, K2 = h;
      } else {
        // T = A21 I11 (h2 x h); W21 = -I22 T
        X1 = {A, lda, s, h, s, 0, NOMOD};
        Y1 = {W, (size_t)TI_NB, s, 0, s, 0, TI_NB};
        X2 = {W, (size_t)TI_NB, s, h, s, h, TI_NB};
        C2 = {W, (size_t)TI_NB, s, h, s, 0, TI_NB};
        M1 = h2, N1 = h, K1 = h, M2 = h2, N2 = h, K2 = h2;
      }
      const dim3 g1((N1 + MG_T - 1) / MG_T, (M1 + MG_T - 1) / MG_T, nz);
      const dim3 g2((N2 + MG_T - 1) / MG_T, (M2 + MG_T - 1) / MG_T, nz);
      if (nowrap) {
        tri_merge_kernel<true><<<g1, 256, 0, c->stream>>>(X1, Y1, Tz, zbase, M1, N1, K1, mod, t64, 1u);
        tri_merge_kernel<true><<<g2, 256, 0, c->stream>>>(X2, Tz, C2, zbase, M2, N2, K2, mod, t64, p - 1);
      } else {
        tri_merge_kernel<false><<<g1, 256, 0, c->stream>>>(X1, Y1, Tz, zbase, M1, N1, K1, mod, t64, 1u);
        tri_merge_kernel<false><<<g2, 256, 0, c->stream>>>(X2, Tz, C2, zbase, M2, N2, K2, mod, t64, p - 1);
      }
      ctx_launched(c, 2);
    }
  }
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "tri_merge launch");
}

// Recursion with inverse leaves: splits at multiples of TI_NB (so every leaf
// is one of W's blocks; W points at the rows of A's top-left entry, which is
// A's entry (off, off)).
static int trsm_rec_inv(Ctx *c, const TileMap *tm, int off, bool upper, int m, int n, uint32_t p,
                        uint32_t alpha, const uint32_t *A, size_t lda, const uint32_t *W,
                        uint32_t *B, size_t ldb, uint8_t *gemm_ws) {
  if (m <= 0) return ST_OK;
  if (m <= TI_NB) {
    // in place: the tensor-core path converts B to limbs in the workspace
    // before its first product, and with one K chunk (m <= TI_NB) each
    // output tile is written once, after every product that reads B
    return zp_gemm_dev(c, GEMM_TC, m, n, m, p, alpha, W, TI_NB, B, ldb, 0, B, ldb, gemm_ws);
  }
  const int l = ((m / 2 + TI_NB - 1) / TI_NB) * TI_NB;  // TI_NB <= l < m
  const uint32_t *A12 = A + l, *A21 = A + (size_t)l * lda, *A22 = A21 + l;
  const uint32_t *W2 = W + (size_t)l * TI_NB;
  uint32_t *B1 = B, *B2 = B + (size_t)l * ldb;
  int st;
  if (!upper) {
    if ((st = trsm_rec_inv(c, tm, off, upper, l, n, p, alpha, A, lda, W, B1, ldb, gemm_ws)))
      return st;
    if ((st = tri_update(c, tm, off + l, off, m - l, l, n, p, alpha, A21, lda, B1, B2, ldb,
                         gemm_ws)))
      return st;
    return trsm_rec_inv(c, tm, off + l, upper, m - l, n, p, 1, A22, lda, W2, B2, ldb, gemm_ws);
  } else {
    if ((st = trsm_rec_inv(c, tm, off + l, upper, m - l, n, p, alpha, A22, lda, W2, B2, ldb,
                           gemm_ws)))
      return st;
    if ((st = tri_update(c, tm, off, off + l, l, m - l, n, p, alpha, A12, lda, B2, B1, ldb,
                         gemm_ws)))
      return st;
    return trsm_rec_inv(c, tm, off, upper, l, n, p, 1, A, lda, W, B1, ldb, gemm_ws);
  }
}

size_t zp_trsm_workspace_bytes(uint32_t p, int m, int n) {
  // the largest update is about (m/2 + leaf) x n x (m/2 + leaf)
  return zp_gemm_workspace_bytes(p, m, n, (m + 1) / 2 + std::max(TI_NB, TRI_NB));
}

int zp_trsm_dev(Ctx *c, bool upper, bool unit, int m, int n, uint32_t p, uint32_t alpha,
                const uint32_t *A, size_t lda, uint32_t *B, size_t ldb, size_t *bad_idx,
                bool sparse, const int2 *row_kr) {
  if (p < 2) return ctx_fail(c, ST_ARG, "modulus must be at least 2");
  if (m < 0 || n < 0) return ctx_fail(c, ST_ARG, "negative dimension");
  if (m == 0) return ST_OK;
  if (lda < (size_t)m || (n > 0 && ldb < (size_t)n))
    return ctx_fail(c, ST_ARG, "leading dimension smaller than the row length");
  alpha %= p;
  const Modulus mod = make_modulus(p);
  if (alpha == 0) {
    if (n == 0) return ST_OK;
    const size_t total = (size_t)m * n;
    int grid = (int)std::min<size_t>((total + 255) / 256, (size_t)c->num_sms * 8);
    zp_scale2_kernel<<<grid, 256, 0, c->stream>>>(B, ldb, m, n, mod, 0);
    ctx_launched(c);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "scale launch");
  }
  void *buf = nullptr;
  int st = ctx_buffer(c, BUF_DINV, (size_t)m * sizeof(uint32_t), &buf);
  if (st) return st;
  uint32_t *dinv = static_cast<uint32_t *>(buf);
  if (!unit) {
    // status[1] = min failing index (init all ones), status[2] = max + 1
    cudaError_t e = cudaMemsetAsync(c->dstatus + 1, 0xFF, sizeof(uint32_t), c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->dstatus + 2, 0, sizeof(uint32_t), c->stream);
    if (e != cudaSuccess) return ctx_cuda(c, e, "cudaMemsetAsync");
    int grid = std::min((m + 255) / 256, c->num_sms * 4);
    diag_inverse_kernel<<<grid, 256, 0, c->stream>>>(A, lda, m, p, dinv, c->dstatus);
    ctx_launched(c);
    e = cudaMemcpyAsync(c->hstatus, c->dstatus, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                        c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return ctx_cuda(c, e, "diagonal inverses");
    if (c->hstatus[2] != 0) {
      size_t idx = upper ? (size_t)c->hstatus[2] - 1 : (size_t)c->hstatus[1];
      if (bad_idx) *bad_idx = idx;
      return ctx_fail(c, ST_DIAG, "diagonal entry not invertible");
    }
  }
  if (n == 0) return ST_OK;
  int kind = c->trsm_kernel;
  if (kind == TRSM_AUTO) {
    // inverse leaves from two leaves up (measured faster there for every
    // width from 64 columns; a single leaf's set-up costs more than the
    // substitution), and not when the caller forced a CUDA-core gemm
    const bool tc = c->gemm_kernel == GEMM_AUTO || c->gemm_kernel == GEMM_TC;
    kind = (tc && m >= 2 * TI_NB) ? TRSM_INVERSE : TRSM_BLOCKS;
  }
  // occupied tiles of a possibly sparse A (bounding boxes of the updates)
  TileMap map;
  const TileMap *tm = nullptr;
  if (sparse && m > TRI_NB) {
    if ((st = build_tile_map(c, upper, m, A, lda, &map))) return st;
    map.kr = row_kr;
    tm = &map;
  }
  // inverses of all 64 x 64 diagonal blocks, in one launch: one after the
  // other for the block substitution, on the diagonal of W for the inverse
  // leaves
  const int nblk = (m + TRI_NB - 1) / TRI_NB;
  const uint32_t *dv = unit ? nullptr : dinv;
  if (kind == TRSM_INVERSE) {
    const int nleaf = (m + TI_NB - 1) / TI_NB;
    void *wb = nullptr, *tb = nullptr;
    if ((st = ctx_buffer(c, BUF_TRI_W, (size_t)nleaf * TI_NB * TI_NB * 4, &wb))) return st;
    // T holds one (s/2)^2 product per block of a level: at most at s = TI_NB
    const size_t tent = (size_t)(m / TI_NB + 1) * (TI_NB / 2) * (TI_NB / 2);
    if ((st = ctx_buffer(c, BUF_TRI_T, tent * 4, &tb))) return st;
    uint32_t *W = static_cast<uint32_t *>(wb);
    cudaError_t e = cudaMemsetAsync(W, 0, (size_t)nleaf * TI_NB * TI_NB * 4, c->stream);
    if (e != cudaSuccess) return ctx_cuda(c, e, "cudaMemsetAsync(trsm inverses)");
    if (upper)
      tri_inv_blocks_kernel<true><<<nblk, 256, 0, c->stream>>>(A, lda, m, dv, W, TI_NB, TI_NB,
                                                              mod, two64_mod(p));
    else
      tri_inv_blocks_kernel<false><<<nblk, 256, 0, c->stream>>>(A, lda, m, dv, W, TI_NB, TI_NB,
                                                               mod, two64_mod(p));
    ctx_launched(c);
    if ((st = tri_inverse_levels(c, upper, m, p, A, lda, W, static_cast<uint32_t *>(tb))))
      return st;
    void *w = nullptr;
    if ((st = ctx_workspace(c, zp_trsm_workspace_bytes(p, m, n), &w))) return st;
    return trsm_rec_inv(c, tm, 0, upper, m, n, p, alpha, A, lda, W, B, ldb,
                        static_cast<uint8_t *>(w));
  }
  void *tb = nullptr;
  if ((st = ctx_buffer(c, BUF_TINV, (size_t)nblk * TRI_NB * TRI_NB * 4, &tb))) return st;
  uint32_t *tinv = static_cast<uint32_t *>(tb);
  if (upper)
    tri_inv_blocks_kernel<true><<<nblk, 256, 0, c->stream>>>(A, lda, m, dv, tinv, TRI_NB, TRI_NB,
                                                            mod, two64_mod(p));
  else
    tri_inv_blocks_kernel<false><<<nblk, 256, 0, c->stream>>>(A, lda, m, dv, tinv, TRI_NB, TRI_NB,
                                                             mod, two64_mod(p));
  ctx_launched(c);
  void *w = nullptr;
  if ((st = ctx_workspace(c, zp_trsm_workspace_bytes(p, m, n), &w))) return st;
  TriLeaves TL{A, tinv};
  return trsm_rec(c, TL, tm, 0, upper, m, n, p, alpha, A, lda, unit ? nullptr : dinv, B, ldb,
                  static_cast<uint8_t *>(w));
}

}  // namespace lela

namespace lela {

// ------------------------------------------------------- sparse operand
// Upper-triangular A given as CSR (rowptr[n + 1], col, val) -> dense rows of
// the zeroed n x n matrix A (one warp per row), and per row the column range
// [first, last + 1) of its stored entries on or right of the diagonal (the
// solve's updates skip the K blocks outside it).  Entries left of the
// diagonal are not part of an upper-triangular operand (the reference's
// upper solve never reads them) and are skipped; values are taken mod p; a
// column index >= n sets *bad.
__global__ void csr_upper_to_dense_kernel(const uint64_t *__restrict__ rowptr,
                                          const uint32_t *__restrict__ col,
                                          const uint32_t *__restrict__ val, int n, uint32_t p,
                                          uint32_t *__restrict__ A, size_t lda, uint32_t *bad,
                                          int2 *__restrict__ kr) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += warps) {
    const uint64_t e0 = rowptr[r], e1 = rowptr[r + 1];
    int lo = 0x7fffffff, hi = -1;
    for (uint64_t e = e0 + lane; e < e1; e += 32) {
      const uint32_t j = col[e];
      if (j >= (uint32_t)n) {
        atomicOr(bad, 1u);
      } else if ((int)j >= r) {
        A[(size_t)r * lda + j] = val[e] % p;
        lo = min(lo, (int)j);
        hi = max(hi, (int)j);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if (lane == 0) kr[r] = hi >= 0 ? make_int2(lo, hi + 1) : make_int2(0, 0);
  }
}

int zp_trsm_csr_upper_dev(Ctx *c, bool unit, int n, int ncols, uint32_t p, uint32_t alpha,
                          const uint64_t *rowptr, const uint32_t *col, const uint32_t *val,
                          uint32_t *B, size_t ldb, size_t *bad_idx) {
  if (p < 2) return ctx_fail(c, ST_ARG, "modulus must be at least 2");
  if (n < 0 || ncols < 0) return ctx_fail(c, ST_ARG, "negative dimension");
  if (n == 0) return ST_OK;
  if (ncols > 0 && ldb < (size_t)ncols)
    return ctx_fail(c, ST_ARG, "leading dimension smaller than the row length");
  void *buf = nullptr;
  const size_t abytes = ((size_t)n * n * 4 + 255) & ~(size_t)255;
  int st = ctx_buffer(c, BUF_TRI_A, abytes + (size_t)n * sizeof(int2), &buf);
  if (st) return st;
  uint32_t *A = static_cast<uint32_t *>(buf);
  int2 *kr = reinterpret_cast<int2 *>(static_cast<uint8_t *>(buf) + abytes);
  cudaError_t e = cudaMemsetAsync(A, 0, (size_t)n * n * 4, c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->dstatus + 3, 0, sizeof(uint32_t), c->stream);
  if (e != cudaSuccess) return ctx_cuda(c, e, "trsm csr: scratch");
  const int grid = std::max(1, std::min((n + 7) / 8, c->num_sms * 8));
  csr_upper_to_dense_kernel<<<grid, 256, 0, c->stream>>>(rowptr, col, val, n, p, A, (size_t)n,
                                                         c->dstatus + 3, kr);
  ctx_launched(c);
  // the index check is read before the solve (one synchronisation)
  e = cudaMemcpyAsync(c->hstatus + 3, c->dstatus + 3, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                      c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return ctx_cuda(c, e, "trsm csr: conversion");
  if (c->hstatus[3]) return ctx_fail(c, ST_ARG, "column index out of range");
  return zp_trsm_dev(c, true, unit, n, ncols, p, alpha, A, (size_t)n, B, ldb, bad_idx, true, kr);
}

}  // namespace lela
