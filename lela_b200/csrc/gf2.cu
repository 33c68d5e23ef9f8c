// lela_b200/csrc/gf2.cu -- dense GF(2) kernels on bit-packed matrices.
//
// Layout: LELA's DenseMatrix<bool> rows are BitVector<LittleEndian<uint64>>
// (lela/ring/gf2.h:311; bit j of word w = column 64w + j,
// lela/vector/bit-iterator.h:249-296), row stride in words.  Bits beyond the
// last column of a row are zero on input and kept zero on output.
//
// gemm  C <- a*A*B + b*C (a, b in {0, 1}).  Replaces the generic
// Row*Row*Row gemm over GF2 (lela/blas/level3-generic.tcc:243-263 ->
// _gemv<GF2> lela/blas/level2-gf2.tcc:132-155: row i of C is the XOR of the
// rows of B selected by row i of A) and M4RI's mzd_mul/mzd_addmul
// (lela/blas/level3-m4ri.tcc:78-80).  Two kernels:
//  * gf2_m4rm_kernel: bit-packed, "method of four Russians": per group of
//    8 rows of B a 256-entry table of all their XOR combinations is built in
//    shared memory, and each row of A then needs one table lookup per byte
//    instead of eight row XORs;
//  * the int8-expanded tensor-core variant (gf2_gemm_tc_planes in
//    zp_gemm.cu): bits become 0/1 bytes, tcgen05 .kind::i8 counts the
//    products exactly, and the parity of the count is the GF(2) entry.
//
// echelon  Non-reduced row-echelon form with LELA's pivot rule (first row
// at or below the current one with a 1 in the column, swapped in by a
// transposition; rows below with a 1 get the pivot row XOR-ed in), i.e.
// Elimination::echelonize on a Dense01 matrix (lela/algorithms/
// elimination.tcc:47-139, pivot-strategy.tcc:44-66), which the dense
// EchelonForm path (GaussJordan + move_L) reproduces.  Same exact panel
// scheme as the Z/p version (echelon.cu) with 64-column panels = one word
// per row; the trailing update is an M4RM product.
#include <algorithm>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "context.h"
#include "gf2.h"
#include "zp_gemm.h"

namespace lela {

// ------------------------------------------------------------------ M4RM
constexpr int M4_BW = 8;      // words of C per CTA
constexpr int M4_ROWS = 4;    // rows of C per thread
constexpr int M4_THREADS = 256;
constexpr int M4_KC = 32;     // rows of B per table round (4 tables of 8)

// C[r, w0 .. w0+8) for the CTA's rows; tables T[g][w][s] in shared memory.
__global__ void __launch_bounds__(M4_THREADS)
    gf2_m4rm_kernel(const uint64_t *__restrict__ A, size_t lda, const uint64_t *__restrict__ B,
                    size_t ldb, uint64_t *__restrict__ C, size_t ldc, int M, int Nw, int K,
                    uint64_t tail_mask, int alpha, int beta) {
  extern __shared__ uint64_t m4_smem[];
  uint64_t(*T)[M4_BW][256] = reinterpret_cast<uint64_t(*)[M4_BW][256]>(m4_smem);
  uint64_t(*Bk)[M4_BW] = reinterpret_cast<uint64_t(*)[M4_BW]>(m4_smem + 4 * M4_BW * 256);
  const int w0 = blockIdx.x * M4_BW;
  const int r0 = blockIdx.y * (M4_THREADS * M4_ROWS);
  uint64_t acc[M4_ROWS][M4_BW];
#pragma unroll
  for (int i = 0; i < M4_ROWS; ++i)
#pragma unroll
    for (int w = 0; w < M4_BW; ++w) acc[i][w] = 0;

  for (int k0 = 0; k0 < K; k0 += M4_KC) {
    __syncthreads();
    for (int e = threadIdx.x; e < M4_KC * M4_BW; e += blockDim.x) {
      const int kk = e / M4_BW, w = e % M4_BW;
      Bk[kk][w] = (k0 + kk < K && w0 + w < Nw) ? B[(size_t)(k0 + kk) * ldb + w0 + w] : 0ull;
    }
    if (threadIdx.x < 4 * M4_BW) T[threadIdx.x / M4_BW][threadIdx.x % M4_BW][0] = 0ull;
    __syncthreads();
    // T[g][w][s + 2^j] = T[g][w][s] ^ B[8g + j][w] for s < 2^j
#pragma unroll 1
    for (int j = 0; j < 8; ++j) {
      const int half = 1 << j;
      for (int e = threadIdx.x; e < 4 * M4_BW * half; e += blockDim.x) {
        const int s = e % half, w = (e / half) % M4_BW, g = e / (half * M4_BW);
        T[g][w][s + half] = T[g][w][s] ^ Bk[8 * g + j][w];
      }
      __syncthreads();
    }
    const int wk = k0 >> 6, sh = k0 & 63;  // the 32 bits of A for k0 .. k0+31
#pragma unroll
    for (int i = 0; i < M4_ROWS; ++i) {
      const int r = r0 + i * M4_THREADS + threadIdx.x;
      uint32_t bits = 0;
      if (r < M) {
        bits = (uint32_t)(A[(size_t)r * lda + wk] >> sh);
        if (K - k0 < 32) bits &= (1u << (K - k0)) - 1u;
      }
      const uint32_t b0 = bits & 255u, b1 = (bits >> 8) & 255u, b2 = (bits >> 16) & 255u,
                     b3 = bits >> 24;
#pragma unroll
      for (int w = 0; w < M4_BW; ++w)
        acc[i][w] ^= T[0][w][b0] ^ T[1][w][b1] ^ T[2][w][b2] ^ T[3][w][b3];
    }
  }
#pragma unroll
  for (int i = 0; i < M4_ROWS; ++i) {
    const int r = r0 + i * M4_THREADS + threadIdx.x;
    if (r >= M) continue;
    uint64_t *crow = C + (size_t)r * ldc;
#pragma unroll
    for (int w = 0; w < M4_BW; ++w) {
      const int gw = w0 + w;
      if (gw >= Nw) break;
      uint64_t v = (beta ? crow[gw] : 0ull) ^ (alpha ? acc[i][w] : 0ull);
      if (gw == Nw - 1) v &= tail_mask;
      crow[gw] = v;
    }
  }
}

int gf2_m4rm_dev(Ctx *c, int M, int N, int K, int alpha, const uint64_t *A, size_t lda,
                 const uint64_t *B, size_t ldb, int beta, uint64_t *C, size_t ldc) {
  if (M <= 0 || N <= 0) return ST_OK;
  const int Nw = (N + 63) / 64;
  const uint64_t tail = (N & 63) ? ((1ull << (N & 63)) - 1ull) : ~0ull;
  dim3 grid((Nw + M4_BW - 1) / M4_BW, (M + M4_THREADS * M4_ROWS - 1) / (M4_THREADS * M4_ROWS));
  constexpr int smem = (4 * M4_BW * 256 + M4_KC * M4_BW) * 8;
  static std::once_flag once;
  static cudaError_t attr_err = cudaSuccess;
  std::call_once(once, [] {
    attr_err = cudaFuncSetAttribute(gf2_m4rm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)((4 * M4_BW * 256 + M4_KC * M4_BW) * 8));
  });
  if (attr_err != cudaSuccess) return ctx_cuda(c, attr_err, "cudaFuncSetAttribute(gf2_m4rm)");
  int pi = prof_begin(c, "gf2_m4rm");
  gf2_m4rm_kernel<<<grid, M4_THREADS, smem, c->stream>>>(A, lda, B, ldb, C, ldc, M, Nw, K, tail,
                                                         alpha, beta);
  prof_end(c, pi);
  ctx_launched(c);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "gf2_m4rm launch");
}

// ------------------------------------------------- int8 expansion for TC
// Ab[r][k] = bit k0+k of row r of A (K-major bytes, row pitch Kp).
__global__ void gf2_unpack_rows_kernel(const uint64_t *__restrict__ A, size_t lda, int M, int k0,
                                       int kc, uint8_t *__restrict__ out, int Kp) {
  const int kq = (kc + 3) >> 2;
  const size_t total = (size_t)M * kq;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(idx / kq), k = (int)(idx % kq) * 4;
    const int gk = k0 + k;  // k0 is a multiple of 64, so 4 bits never straddle words
    const uint64_t wv = A[(size_t)r * lda + (gk >> 6)] >> (gk & 63);
    uint32_t v = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i)
      if (k + i < kc) v |= (uint32_t)((wv >> i) & 1ull) << (8 * i);
    *reinterpret_cast<uint32_t *>(out + (size_t)r * Kp + k) = v;
  }
}

// Bb[n][k] = bit n of row k0+k of B: one CTA of 64 threads per 64 rows of B
// and one word (64 columns).
__global__ void gf2_unpack_cols_kernel(const uint64_t *__restrict__ B, size_t ldb, int k0, int kc,
                                       int N, uint8_t *__restrict__ out, int Kp) {
  __shared__ uint64_t rows[64];
  const int w = blockIdx.x, kb = blockIdx.y * 64;
  const int t = threadIdx.x;
  rows[t] = (kb + t < kc) ? B[(size_t)(k0 + kb + t) * ldb + w] : 0ull;
  __syncthreads();
  const int n = w * 64 + t;
  if (n >= N) return;
  uint8_t *dst = out + (size_t)n * Kp + kb;
  for (int q = 0; q < 64 && kb + q < Kp; q += 4) {
    uint32_t v = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) v |= (uint32_t)((rows[q + i] >> t) & 1ull) << (8 * i);
    *reinterpret_cast<uint32_t *>(dst + q) = v;
  }
}

int gf2_gemm_dev(Ctx *c, int kernel, int M, int N, int K, int alpha, const uint64_t *A,
                 size_t lda, const uint64_t *B, size_t ldb, int beta, uint64_t *C, size_t ldc) {
  if (M < 0 || N < 0 || K < 0) return ctx_fail(c, ST_ARG, "negative dimension");
  if (M == 0 || N == 0) return ST_OK;
  const int Nw = (N + 63) / 64, Kw = (K + 63) / 64;
  if (ldc < (size_t)Nw || (K > 0 && (lda < (size_t)Kw || ldb < (size_t)Nw)))
    return ctx_fail(c, ST_ARG, "leading dimension smaller than the row length");
  alpha &= 1;
  beta &= 1;
  if (kernel == GF2_AUTO) kernel = c->gf2_kernel == GF2_AUTO ? GF2_TC : c->gf2_kernel;
  if (K == 0 || alpha == 0 || kernel == GF2_M4RM)
    return gf2_m4rm_dev(c, M, N, (alpha && K > 0) ? K : 0, alpha, A, lda, B, ldb, beta, C, ldc);
  // tensor cores on 0/1 bytes, K in chunks of 32768 (the counts stay exact)
  const int kcmax = std::min(K, ZP_KCHUNK);
  const int Kpmax = (kcmax + 63) & ~63;
  void *w = nullptr;
  int st = ctx_workspace(c, (size_t)(M + N) * Kpmax + 256, &w);
  if (st) return st;
  uint8_t *Ab = static_cast<uint8_t *>(w);
  uint32_t b = (uint32_t)beta;
  for (int k0 = 0; k0 < K; k0 += ZP_KCHUNK) {
    const int kc = std::min(ZP_KCHUNK, K - k0);
    const int Kp = (kc + 63) & ~63;
    uint8_t *Bb = Ab + (size_t)M * Kp;
    const size_t total = (size_t)M * ((kc + 3) / 4);
    int grid = (int)std::min<size_t>((total + 255) / 256, (size_t)c->num_sms * 16);
    int pi = prof_begin(c, "gf2_unpack");
    gf2_unpack_rows_kernel<<<grid, 256, 0, c->stream>>>(A, lda, M, k0, kc, Ab, Kp);
    dim3 g2(Nw, Kp / 64);
    gf2_unpack_cols_kernel<<<g2, 64, 0, c->stream>>>(B, ldb, k0, kc, N, Bb, Kp);
    prof_end(c, pi);
    ctx_launched(c, 2);
    if ((st = gf2_gemm_tc_planes(c, M, N, kc, Ab, Bb, Kp, 1u, b, C, ldc))) return st;
    b = 1;
  }
  return ST_OK;
}

// --------------------------------------------------------------- echelon
constexpr int GW = 64;

struct Gf2PanelOut {
  uint32_t t, nact, last_pos, pad;
  uint32_t ti[GW], tq[GW], pcol[GW];
};

__device__ __forceinline__ int gf2_block_scan(int flag, int *warp_sums, int *total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  unsigned b = __ballot_sync(0xffffffffu, flag);
  int in_warp = __popc(b & ((1u << lane) - 1u));
  if (lane == 0) warp_sums[wid] = __popc(b);
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int w = 0; w < nw; ++w) {
      int v = warp_sums[w];
      warp_sums[w] = s;
      s += v;
    }
    *total = s;
  }
  __syncthreads();
  int r = warp_sums[wid] + in_warp;
  __syncthreads();
  return r;
}

// The reference's steps restricted to panel word `wc` (w valid bits) on the
// rows at or below i0 that have a bit set there (see echelon.cu).
__global__ void __launch_bounds__(1024)
    gf2_panel_kernel(const uint64_t *__restrict__ D, size_t ld, int i0, int m, int wc, int w,
                     int *__restrict__ act_row, int *__restrict__ act_pos,
                     uint64_t *__restrict__ vals, uint64_t *__restrict__ mult, Gf2PanelOut *out) {
  __shared__ int warp_sums[32];
  __shared__ int s_total, s_nact;
  __shared__ unsigned long long s_key;
  __shared__ int s_at_i;
  const uint64_t mask = (w == 64) ? ~0ull : ((1ull << w) - 1ull);
  if (threadIdx.x == 0) s_nact = 0;
  __syncthreads();
  for (int base = i0; base < m; base += blockDim.x) {
    const int r = base + threadIdx.x;
    const int flag = (r < m) && (D[(size_t)r * ld + wc] & mask) != 0ull;
    int off = gf2_block_scan(flag, warp_sums, &s_total);
    if (flag) act_row[s_nact + off] = r;
    __syncthreads();
    if (threadIdx.x == 0) s_nact += s_total;
    __syncthreads();
  }
  const int nact = s_nact;
  for (int a = threadIdx.x; a < nact; a += blockDim.x) {
    act_pos[a] = act_row[a];
    vals[a] = D[(size_t)act_row[a] * ld + wc] & mask;
    mult[a] = 0ull;
  }
  __syncthreads();
  int i = i0, t = 0;
  for (int col = 0; col < w && i < m; ++col) {
    if (threadIdx.x == 0) {
      s_key = ~0ull;
      s_at_i = -1;
    }
    __syncthreads();
    for (int a = threadIdx.x; a < nact; a += blockDim.x) {
      const int pos = act_pos[a];
      if (pos >= i && ((vals[a] >> col) & 1ull))
        atomicMin(&s_key, ((unsigned long long)(unsigned)pos << 32) | (unsigned)a);
      if (pos == i) s_at_i = a;
    }
    __syncthreads();
    const unsigned long long key = s_key;
    const int ai = s_at_i;
    __syncthreads();
    if (key == ~0ull) continue;
    const int ap = (int)(key & 0xffffffffu), q = (int)(key >> 32);
    const uint64_t pw = vals[ap];
    if (threadIdx.x == 0) {
      out->ti[t] = (uint32_t)i;
      out->tq[t] = (uint32_t)q;
      out->pcol[t] = (uint32_t)col;
      if (ai >= 0 && ai != ap) act_pos[ai] = q;
      act_pos[ap] = i;
    }
    __syncthreads();
    for (int a = threadIdx.x; a < nact; a += blockDim.x) {
      if (act_pos[a] <= i) continue;
      if ((vals[a] >> col) & 1ull) {
        vals[a] ^= pw;
        mult[a] |= 1ull << t;
      }
    }
    __syncthreads();
    ++i;
    ++t;
  }
  if (threadIdx.x == 0) s_key = 0;
  __syncthreads();
  for (int a = threadIdx.x; a < nact; a += blockDim.x)
    if (act_pos[a] >= i) atomicMax(&s_key, (unsigned long long)(unsigned)act_pos[a]);
  __syncthreads();
  if (threadIdx.x == 0) {
    out->t = (uint32_t)t;
    out->nact = (uint32_t)nact;
    out->last_pos = (uint32_t)s_key;
  }
}

__global__ void gf2_gather_rows_kernel(const uint64_t *__restrict__ D, size_t ld, int nw,
                                       const int *__restrict__ src, int cnt,
                                       uint64_t *__restrict__ tmp) {
  for (int k = blockIdx.y; k < cnt; k += gridDim.y)
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nw; j += gridDim.x * blockDim.x)
      tmp[(size_t)k * nw + j] = D[(size_t)src[k] * ld + j];
}
__global__ void gf2_scatter_rows_kernel(uint64_t *__restrict__ D, size_t ld, int nw,
                                        const int *__restrict__ dst, int cnt,
                                        const uint64_t *__restrict__ tmp) {
  for (int k = blockIdx.y; k < cnt; k += gridDim.y)
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nw; j += gridDim.x * blockDim.x)
      D[(size_t)dst[k] * ld + j] = tmp[(size_t)k * nw + j];
}

// Panel words back into D; L11 rows (pivot k: its multiplier bits) and the
// L21 word of every row in r0..r1 (zero when the row was not eliminated).
__global__ void gf2_panel_writeback_kernel(uint64_t *__restrict__ D, size_t ld, int wc,
                                           uint64_t keep_mask, int nact,
                                           const int *__restrict__ act_pos,
                                           const uint64_t *__restrict__ vals,
                                           const uint64_t *__restrict__ mult, int i0, int t,
                                           uint64_t *__restrict__ L11, uint64_t *__restrict__ L21,
                                           int r0) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nact; a += gridDim.x * blockDim.x) {
    const int pos = act_pos[a];
    uint64_t *x = D + (size_t)pos * ld + wc;
    *x = (*x & keep_mask) | vals[a];
    if (pos < i0 + t)
      L11[pos - i0] = mult[a];
    else if (pos >= r0)
      L21[pos - r0] = mult[a];
  }
}

// U12 = L11^-1 A12 over GF(2): pivot rows i0..i0+t-1, words from w1; row k
// gets the XOR of the earlier pivot rows j whose bit is set in L11[k].
// One thread per word with the t words of the column in registers.
__global__ void gf2_l11_solve_kernel(uint64_t *__restrict__ D, size_t ld, int i0, int t, int w1,
                                     int nw, const uint64_t *__restrict__ L11) {
  __shared__ uint64_t sL[GW];
  if (threadIdx.x < GW) sL[threadIdx.x] = threadIdx.x < t ? L11[threadIdx.x] : 0ull;
  __syncthreads();
  const int w = w1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= nw) return;
  uint64_t x[GW];
#pragma unroll
  for (int k = 0; k < GW; ++k) x[k] = k < t ? D[(size_t)(i0 + k) * ld + w] : 0ull;
#pragma unroll
  for (int k = 1; k < GW; ++k) {
    const uint64_t lk = sL[k];
#pragma unroll
    for (int j = 0; j < k; ++j)
      if ((lk >> j) & 1ull) x[k] ^= x[j];
  }
#pragma unroll
  for (int k = 0; k < GW; ++k)
    if (k < t) D[(size_t)(i0 + k) * ld + w] = x[k];
}

__global__ void gf2_zero_kernel(uint64_t *x, size_t n) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x)
    x[k] = 0ull;
}

int gf2_echelon_dev(Ctx *c, int m, int n, uint64_t *D, size_t ld, size_t *rank_out) {
  if (m < 0 || n < 0) return ctx_fail(c, ST_ARG, "negative dimension");
  const int nw = (n + 63) / 64;
  if (m > 0 && n > 0 && ld < (size_t)nw) return ctx_fail(c, ST_ARG, "leading dimension too small");
  size_t rank = 0;
  if (m == 0 || n == 0) {
    *rank_out = 0;
    return ST_OK;
  }
  const size_t out_bytes = (sizeof(Gf2PanelOut) + 255) & ~(size_t)255;
  const size_t i_bytes = (((size_t)2 * m + 4 * GW) * sizeof(int) + 255) & ~(size_t)255;
  const size_t v_bytes = (size_t)m * 8;
  void *base = nullptr;
  int st = ctx_buffer(c, BUF_GF2_0,
                      out_bytes + i_bytes + 3 * v_bytes + GW * 8 + (size_t)2 * GW * nw * 8 + 1024,
                      &base);
  if (st) return st;
  uint8_t *b8 = static_cast<uint8_t *>(base);
  Gf2PanelOut *d_out = reinterpret_cast<Gf2PanelOut *>(b8);
  int *d_act_row = reinterpret_cast<int *>(b8 + out_bytes);
  int *d_act_pos = d_act_row + m;
  int *d_perm = d_act_pos + m;
  uint64_t *d_vals = reinterpret_cast<uint64_t *>(b8 + out_bytes + i_bytes);
  uint64_t *d_mult = d_vals + m;
  uint64_t *d_L21 = d_mult + m;
  uint64_t *d_L11 = d_L21 + m;
  uint64_t *d_tmp = d_L11 + GW;

  Gf2PanelOut h;
  std::vector<int> at, src, dst;
  int i = 0;
  for (int wc = 0; wc < nw && i < m; ++wc) {
    const int w = std::min(64, n - 64 * wc);
    int pi = prof_begin(c, "gf2_panel");
    gf2_panel_kernel<<<1, 1024, 0, c->stream>>>(D, ld, i, m, wc, w, d_act_row, d_act_pos, d_vals,
                                                d_mult, d_out);
    prof_end(c, pi);
    ctx_launched(c);
    cudaError_t e = cudaMemcpyAsync(&h, d_out, sizeof h, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return ctx_cuda(c, e, "gf2 echelon: panel");
    const int t = (int)h.t;
    if (t == 0) continue;
    int hi = i;
    for (int k = 0; k < t; ++k) hi = std::max(hi, (int)h.tq[k]);
    at.resize(hi - i + 1);
    for (int q = i; q <= hi; ++q) at[q - i] = q;
    for (int k = 0; k < t; ++k) std::swap(at[h.ti[k] - i], at[h.tq[k] - i]);
    src.clear();
    dst.clear();
    for (int q = i; q <= hi; ++q)
      if (at[q - i] != q) {
        dst.push_back(q);
        src.push_back(at[q - i]);
      }
    const int cnt = (int)src.size();
    if (cnt > 2 * GW) return ctx_fail(c, ST_ARG, "gf2 echelon: permutation larger than expected");
    if (cnt > 0) {
      std::vector<int> both(src);
      both.insert(both.end(), dst.begin(), dst.end());
      e = cudaMemcpyAsync(d_perm, both.data(), both.size() * sizeof(int), cudaMemcpyHostToDevice,
                          c->stream);
      if (e != cudaSuccess) return ctx_cuda(c, e, "gf2 echelon: permutation");
      dim3 grid((nw + 255) / 256, cnt);
      gf2_gather_rows_kernel<<<grid, 256, 0, c->stream>>>(D, ld, nw, d_perm, cnt, d_tmp);
      gf2_scatter_rows_kernel<<<grid, 256, 0, c->stream>>>(D, ld, nw, d_perm + cnt, cnt, d_tmp);
      ctx_launched(c, 2);
    }
    const int r0 = i + t;
    const int r1 = (h.last_pos >= (uint32_t)r0) ? (int)h.last_pos : r0 - 1;
    const int below = r1 - r0 + 1;
    if (below > 0) {
      gf2_zero_kernel<<<std::min((below + 255) / 256, c->num_sms * 8), 256, 0, c->stream>>>(
          d_L21, (size_t)below);
      ctx_launched(c);
    }
    const uint64_t pmask = (w == 64) ? ~0ull : ((1ull << w) - 1ull);
    const int nact = (int)h.nact;
    gf2_panel_writeback_kernel<<<std::max(1, std::min((nact + 255) / 256, c->num_sms * 4)), 256,
                                 0, c->stream>>>(D, ld, wc, ~pmask, nact, d_act_pos, d_vals,
                                                 d_mult, i, t, d_L11, d_L21, r0);
    ctx_launched(c);
    const int w1 = wc + 1;
    if (w1 < nw) {
      gf2_l11_solve_kernel<<<(nw - w1 + 127) / 128, 128, 0, c->stream>>>(D, ld, i, t, w1, nw,
                                                                          d_L11);
      ctx_launched(c);
      if (below > 0) {
        // rows r0..r1, trailing words: C ^= L21 (one word of t bits per row) * U12
        pi = prof_begin(c, "gf2_update");
        st = gf2_m4rm_dev(c, below, n - 64 * w1, t, 1, d_L21, 1, D + (size_t)i * ld + w1, ld, 1,
                          D + (size_t)r0 * ld + w1, ld);
        prof_end(c, pi);
        if (st) return st;
      }
    }
    rank += t;
    i += t;
  }
  *rank_out = rank;
  return ST_OK;
}

}  // namespace lela
