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
#include <cstddef>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "context.h"
#include "gf2.h"
#include "zp_gemm.h"

namespace lela {

// ------------------------------------------------------------------ M4RM
constexpr int M4_THREADS = 256;
constexpr int M4_KC = 32;     // rows of B per table round (4 tables of 8)

// C[r, w0 .. w0+M4_BW) for the CTA's rows (M4_ROWS per thread); tables
// T[g][w][s] in shared memory.
template <int M4_ROWS, int M4_BW>
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
      // bits of the last word at columns >= N keep their old values (they
      // may belong to the next columns of a strided view)
      const bool part = gw == Nw - 1 && tail_mask != ~0ull;
      const uint64_t old = (beta || part) ? crow[gw] : 0ull;
      uint64_t v = (beta ? old : 0ull) ^ (alpha ? acc[i][w] : 0ull);
      if (part) v = (v & tail_mask) | (old & ~tail_mask);
      crow[gw] = v;
    }
  }
}

int gf2_m4rm_dev(Ctx *c, int M, int N, int K, int alpha, const uint64_t *A, size_t lda,
                 const uint64_t *B, size_t ldb, int beta, uint64_t *C, size_t ldc) {
  if (M <= 0 || N <= 0) return ST_OK;
  const int Nw = (N + 63) / 64;
  const uint64_t tail = (N & 63) ? ((1ull << (N & 63)) - 1ull) : ~0ull;
  // Eight words and four rows per thread per CTA; one row when that leaves
  // fewer than two CTAs per SM; two words as well when even that does (few
  // rows, e.g. a panel's 64 pivot rows against a wide B: the tables, which
  // dominate there, are then built by four times as many CTAs, each a
  // quarter of them).
  auto smem_for = [](int bw) { return (4 * bw * 256 + M4_KC * bw) * 8; };
  if (int st = ctx_smem_attr(c, (const void *)gf2_m4rm_kernel<4, 8>, smem_for(8),
                             "cudaFuncSetAttribute(gf2_m4rm)"))
    return st;
  if (int st = ctx_smem_attr(c, (const void *)gf2_m4rm_kernel<1, 8>, smem_for(8),
                             "cudaFuncSetAttribute(gf2_m4rm)"))
    return st;
  const size_t enough = 2u * c->num_sms;
  const int gx8 = (Nw + 7) / 8, gx2 = (Nw + 1) / 2;
  const int gy4 = (M + M4_THREADS * 4 - 1) / (M4_THREADS * 4), gy1 = (M + M4_THREADS - 1) / M4_THREADS;
  int pi = prof_begin(c, "gf2_m4rm");
  if ((size_t)gx8 * gy4 >= enough)
    gf2_m4rm_kernel<4, 8><<<dim3(gx8, gy4), M4_THREADS, smem_for(8), c->stream>>>(
        A, lda, B, ldb, C, ldc, M, Nw, K, tail, alpha, beta);
  else if ((size_t)gx8 * gy1 >= enough)
    gf2_m4rm_kernel<1, 8><<<dim3(gx8, gy1), M4_THREADS, smem_for(8), c->stream>>>(
        A, lda, B, ldb, C, ldc, M, Nw, K, tail, alpha, beta);
  else
    gf2_m4rm_kernel<1, 2><<<dim3(gx2, gy1), M4_THREADS, smem_for(2), c->stream>>>(
        A, lda, B, ldb, C, ldc, M, Nw, K, tail, alpha, beta);
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

// ---------------------------------------------- host-pointer row blocks
constexpr int GF2_PIPE_MIN_ROWS = 512;

bool gf2_gemm_pipelined(const Ctx *c, int M, int N, int K, int alpha) {
  const int kernel = c->gf2_kernel == GF2_AUTO ? GF2_TC : c->gf2_kernel;
  return kernel == GF2_TC && (alpha & 1) && K > 0 && K <= ZP_KCHUNK && N > 0 &&
         M >= 2 * GF2_PIPE_MIN_ROWS;
}

int gf2_gemm_host_rows(Ctx *c, int M, int N, int K, const uint64_t *hA, size_t lda,
                       const uint64_t *hB, size_t ldb, int beta, uint64_t *hC, size_t ldc,
                       uint64_t *dA, uint64_t *dB, uint64_t *dC) {
  if (!gf2_gemm_pipelined(c, M, N, K, 1)) return ctx_fail(c, ST_ARG, "not a pipelined gemm");
  if (int st = ctx_pipe(c)) return st;
  const int Kp = (K + 63) & ~63;
  const int Kw = (K + 63) / 64, Nw = (N + 63) / 64;
  void *w = nullptr;
  if (int st = ctx_workspace(c, (size_t)(M + N) * Kp + 256, &w)) return st;
  uint8_t *Ab = static_cast<uint8_t *>(w), *Bb = Ab + (size_t)M * Kp;
  // row blocks: a multiple of 128 rows (the tensor-core tile), at most
  // PIPE_MAX_BLOCKS of them
  const int per = (M + PIPE_MAX_BLOCKS - 1) / PIPE_MAX_BLOCKS;
  const int rb = std::max(GF2_PIPE_MIN_ROWS, (per + 127) / 128 * 128);
  const int nblk = (M + rb - 1) / rb;
  cudaEvent_t *ready = c->pipe_ev, *done = c->pipe_ev + PIPE_MAX_BLOCKS;
  cudaEvent_t ev_start = c->pipe_ev[2 * PIPE_MAX_BLOCKS], ev_b = c->pipe_ev[2 * PIPE_MAX_BLOCKS + 1],
              ev_out = c->pipe_ev[2 * PIPE_MAX_BLOCKS + 2];
  const size_t rowA = (size_t)Kw * 8, rowB = (size_t)Nw * 8;
  // C's rows come in when b = 1, and for the bits past column N of each
  // row's last word, which the product leaves as they were
  const bool cin = (beta & 1) || (N & 63);
  cudaError_t e = cudaEventRecord(ev_start, c->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(c->copy_in, ev_start, 0);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(c->copy_out, ev_start, 0);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(dB, rowB, hB, ldb * 8, rowB, (size_t)K, cudaMemcpyHostToDevice,
                          c->copy_in);
  if (e == cudaSuccess) e = cudaEventRecord(ev_b, c->copy_in);
  for (int j = 0; e == cudaSuccess && j < nblk; ++j) {
    const int r0 = j * rb, rows = std::min(rb, M - r0);
    e = cudaMemcpy2DAsync(dA + (size_t)r0 * Kw, rowA, hA + (size_t)r0 * lda, lda * 8, rowA,
                          (size_t)rows, cudaMemcpyHostToDevice, c->copy_in);
    if (e == cudaSuccess && cin)
      e = cudaMemcpy2DAsync(dC + (size_t)r0 * Nw, rowB, hC + (size_t)r0 * ldc, ldc * 8, rowB,
                            (size_t)rows, cudaMemcpyHostToDevice, c->copy_in);
    if (e == cudaSuccess) e = cudaEventRecord(ready[j], c->copy_in);
  }
  // B's bytes once; each block's A bytes in its own part of the workspace
  int st = ST_OK;
  if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, ev_b, 0);
  if (e == cudaSuccess) {
    int pi = prof_begin(c, "gf2_unpack");
    gf2_unpack_cols_kernel<<<dim3(Nw, Kp / 64), 64, 0, c->stream>>>(dB, (size_t)Nw, 0, K, N, Bb, Kp);
    prof_end(c, pi);
    ctx_launched(c);
    e = cudaGetLastError();
  }
  for (int j = 0; e == cudaSuccess && !st && j < nblk; ++j) {
    const int r0 = j * rb, rows = std::min(rb, M - r0);
    uint8_t *Aj = Ab + (size_t)r0 * Kp;
    e = cudaStreamWaitEvent(c->stream, ready[j], 0);
    if (e != cudaSuccess) break;
    const size_t total = (size_t)rows * ((K + 3) / 4);
    const int grid = (int)std::min<size_t>((total + 255) / 256, (size_t)c->num_sms * 16);
    int pi = prof_begin(c, "gf2_unpack");
    gf2_unpack_rows_kernel<<<grid, 256, 0, c->stream>>>(dA + (size_t)r0 * Kw, (size_t)Kw, rows, 0,
                                                        K, Aj, Kp);
    prof_end(c, pi);
    ctx_launched(c);
    st = gf2_gemm_tc_planes(c, rows, N, K, Aj, Bb, Kp, 1u, (uint32_t)(beta & 1),
                            dC + (size_t)r0 * Nw, (size_t)Nw);
    if (st) break;
    e = cudaEventRecord(done[j], c->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->copy_out, done[j], 0);
    if (e == cudaSuccess)
      e = cudaMemcpy2DAsync(hC + (size_t)r0 * ldc, ldc * 8, dC + (size_t)r0 * Nw, rowB, rowB,
                            (size_t)rows, cudaMemcpyDeviceToHost, c->copy_out);
  }
  // the handle stream ends after the last copy out
  if (e == cudaSuccess && !st) e = cudaEventRecord(ev_out, c->copy_out);
  if (e == cudaSuccess && !st) e = cudaStreamWaitEvent(c->stream, ev_out, 0);
  if (e != cudaSuccess || st) {
    // copies already queued may still use the caller's buffers
    cudaStreamSynchronize(c->copy_in);
    cudaStreamSynchronize(c->copy_out);
    return st ? st : ctx_cuda(c, e, "pipelined gf2 gemm");
  }
  return ST_OK;
}

// --------------------------------------------------------------- echelon
//
// Per 64-column panel (one word per row), the Z/p panel scheme of
// echelon.cu with GF(2) arithmetic:
//  * gf2_heads_kernel: first set bit of each row's panel word, the head
//    histogram and the last row with a nonzero word;
//  * gf2_search_kernel: the reference's pivot choice, lazily.  The pivot
//    rows are kept as a reduced basis g_k (bit pcol_j of g_k is delta_kj)
//    and, per column c, the mask M[c] = (1 << c) | sum_k g_k[c] << pcol_k,
//    so bit c of a row reduced by all pivots so far is parity(v & M[c]):
//    32 positions are tested per ballot;
//  * the host replays the transpositions and moves the rows;
//  * gf2_solve_kernel: per row from the first pivot down to the last
//    possibly nonzero row, the reference's elimination steps on the word
//    (pivot k XOR-ed in when bit pcol_k is set) give the multipliers; pivot
//    rows become U_k, rows below become zero;
//  * U12 = L11^-1 A12 and the M4RM trailing update C ^= L21 U12.
constexpr int GW = 64;
constexpr uint8_t GF2_HEAD_NONE = 64;

struct Gf2PanelOut {
  uint32_t t, pad0, last_pos, pad;
  uint32_t ti[GW], tq[GW], pcol[GW];
};

__device__ __forceinline__ int gf2_row_at(int pos, const int *p2r, const int *stamp, int epoch) {
  return stamp[pos] == epoch ? p2r[pos] : pos;
}

constexpr int GF2_HEADS_THREADS = 256;
// hist counts only the rows from position hist0 on (those the search reads
// lazily, past its register window).
__global__ void __launch_bounds__(GF2_HEADS_THREADS)
    gf2_heads_kernel(const uint64_t *__restrict__ D, size_t ld, int i0, int m, int wc,
                     uint64_t pmask, uint8_t *__restrict__ head, uint8_t *__restrict__ act,
                     int *hist, int *last, int hist0) {
  __shared__ int s_last;
  __shared__ int s_hist[GW + 1];
  if (threadIdx.x == 0) s_last = -1;
  if (threadIdx.x <= GW) s_hist[threadIdx.x] = 0;
  __syncthreads();
  int my_last = -1;
  for (int r = i0 + blockIdx.x * blockDim.x + threadIdx.x; r < m; r += gridDim.x * blockDim.x) {
    const uint64_t v = D[(size_t)r * ld + wc] & pmask;
    const int h = v ? __ffsll((long long)v) - 1 : GF2_HEAD_NONE;
    head[r] = (uint8_t)h;
    act[r] = v != 0ull;
    if (r >= hist0) atomicAdd(&s_hist[h], 1);
    if (v) my_last = r;
  }
  if (my_last >= 0) atomicMax(&s_last, my_last);
  __syncthreads();
  if (threadIdx.x == 0 && s_last >= 0) atomicMax(last, s_last);
  if (threadIdx.x <= GW && s_hist[threadIdx.x]) atomicAdd(&hist[threadIdx.x], s_hist[threadIdx.x]);
}

// One warp.  The words of positions i0 .. i0 + GF2_WR - 1 (the window) sit
// in registers, lane l holding positions i0 + l + 32 u, and are eliminated
// eagerly: when the pivot of column c is chosen, every other window row at
// or below the current position with bit c set gets the pivot word XOR-ed
// in, so the pivot of a column is the first window position at or below
// the current one with the bit set (one ballot per 32 positions), and a
// pivot row's word is its final U_k (reduced by the pivots before it, as the
// reference's elimination leaves it).  Rows past the window are tested
// lazily: the pivot rows are also kept as a reduced basis g_k (bit pcol_j of
// g_k is delta_kj) with, per column c, the mask M[c] = (1 << c) | sum_k
// g_k[c] << pcol_k, so bit c of a row reduced by all pivots so far is
// parity(v & M[c]); head[] holds a lower bound of the first set bit of each
// such row's reduced word and cnt[h] counts them by that bound, so the scan
// past the window runs only when a row there may hold the pivot.  Outputs:
// Gf2PanelOut, U (the pivot rows' final words).  Resets *last_act and
// hist[] for the next panel.
constexpr int GF2_WR = 128;               // window positions (registers)
constexpr int GF2_WU = GF2_WR / 32;       // per lane
__global__ void __launch_bounds__(32)
    gf2_search_kernel(const uint64_t *__restrict__ D, size_t ld, int i0, int m, int wc, int w,
                      uint64_t pmask, uint8_t *__restrict__ head, const uint8_t *__restrict__ act,
                      int *__restrict__ hist, int *__restrict__ last_act, int *__restrict__ p2r,
                      int *__restrict__ stamp, int epoch, uint64_t *__restrict__ Uout,
                      Gf2PanelOut *out, Gf2PanelOut *hout, volatile uint32_t *hflag,
                      uint32_t seq) {
  __shared__ uint64_t G[GW], M[GW], s_U[GW];
  __shared__ int s_pcol[GW], s_ti[GW], s_tq[GW];
  __shared__ int s_cnt[GW + 1];
  const int lane = threadIdx.x;
  const int wend = min(i0 + GF2_WR, m);  // positions past the window start here
  // cnt: the rows from wend on (the heads kernel counted only those)
  for (int h = lane; h <= GW; h += 32) {
    s_cnt[h] = hist[h];
    hist[h] = 0;
  }
  __syncwarp();
  uint64_t wv[GF2_WU];
  int wr[GF2_WU];  // row index at the position (-1: past the matrix)
#pragma unroll
  for (int u = 0; u < GF2_WU; ++u) {
    const int pos = i0 + lane + 32 * u;
    wr[u] = pos < m ? pos : -1;  // no transposition has touched this panel yet
    wv[u] = pos < m ? D[(size_t)pos * ld + wc] & pmask : 0ull;
  }
  M[lane] = 1ull << lane;
  M[lane + 32] = 1ull << (lane + 32);
  __syncwarp();
  auto pick64 = [&](int g) -> uint64_t {
    uint64_t v = wv[0];
#pragma unroll
    for (int u = 1; u < GF2_WU; ++u)
      if (g == u) v = wv[u];
    return v;
  };
  auto pickr = [&](int g) -> int {
    int v = wr[0];
#pragma unroll
    for (int u = 1; u < GF2_WU; ++u)
      if (g == u) v = wr[u];
    return v;
  };
  // The basis g_k and masks M: pivot U at column c makes g_k ^= U where g_k
  // has bit c, and M[c'] ^= M[c] for the columns c' > c where U has a bit.
  // Only the scan past the window uses them, so they are built when it first
  // runs (replaying the pivots so far) and kept from then on.
  auto basis_add = [&](uint64_t U, int c, int k) {
    const uint64_t mcol = M[c], b = 1ull << c;
    __syncwarp();
    if (lane < k && (G[lane] & b)) G[lane] ^= U;
    if (lane + 32 < k && (G[lane + 32] & b)) G[lane + 32] ^= U;
    for (int cc = lane; cc < w; cc += 32)
      if (cc > c && ((U >> cc) & 1ull)) M[cc] ^= mcol;
    __syncwarp();
    if (lane == 0) G[k] = U;
    __syncwarp();
  };
  bool basis = false;
  int i = i0, t = 0;
  for (int col = 0; col < w && i < m; ++col) {
    const uint64_t bit = 1ull << col;
    // first window position at or below i with bit col set
    int qi = -1;
#pragma unroll
    for (int u = 0; u < GF2_WU; ++u) {
      const int pos = i0 + lane + 32 * u;
      const unsigned b = __ballot_sync(0xffffffffu, pos >= i && (wv[u] & bit) != 0ull);
      if (qi < 0 && b) qi = 32 * u + __ffs(b) - 1;
    }
    int q;
    uint64_t U;
    if (qi >= 0) {
      q = i0 + qi;
      U = __shfl_sync(0xffffffffu, pick64(qi >> 5), qi & 31);
      // eliminate the other window rows at or below i
#pragma unroll
      for (int u = 0; u < GF2_WU; ++u) {
        const int e = lane + 32 * u;
        if (i0 + e >= i && e != qi && (wv[u] & bit)) wv[u] ^= U;
      }
      // transposition (i, q) inside the window: the row at i (bit col clear,
      // so not changed above) and the pivot row trade places
      if (q != i) {
        const int ei = i - i0;
        const uint64_t vi = __shfl_sync(0xffffffffu, pick64(ei >> 5), ei & 31);
        const int ri = __shfl_sync(0xffffffffu, pickr(ei >> 5), ei & 31);
        const int rq = __shfl_sync(0xffffffffu, pickr(qi >> 5), qi & 31);
#pragma unroll
        for (int u = 0; u < GF2_WU; ++u) {
          const int e = lane + 32 * u;
          if (e == ei) {
            wv[u] = U;
            wr[u] = rq;
          } else if (e == qi) {
            wv[u] = vi;
            wr[u] = ri;
          }
        }
      }
    } else {
      // none in the window: rows past it whose bound allows a pivot here
      int cand = 0;
      for (int h = lane; h <= col; h += 32) cand += s_cnt[h];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) cand += __shfl_xor_sync(0xffffffffu, cand, o);
      if (cand == 0) continue;  // no pivot in this column
      if (!basis) {
        for (int k = 0; k < t; ++k) basis_add(s_U[k], s_pcol[k], k);
        basis = true;
      }
      q = -1;
      uint64_t v = 0ull;
      for (int base = wend; base < m && cand > 0; base += 32) {
        const int pos = base + lane;
        int is_cand = 0, hit = 0;
        uint64_t pv = 0ull;
        if (pos < m) {
          const int r = gf2_row_at(pos, p2r, stamp, epoch);
          const int hr = head[r];
          if (hr <= col) {
            is_cand = 1;
            pv = D[(size_t)r * ld + wc] & pmask;
            int c = col;
            while (c < w && !(__popcll(pv & M[c]) & 1)) ++c;
            const int hn = c < w ? c : GF2_HEAD_NONE;
            if (hn != hr) {
              head[r] = (uint8_t)hn;
              atomicSub(&s_cnt[hr], 1);
              atomicAdd(&s_cnt[hn], 1);
            }
            hit = c == col;
          }
        }
        cand -= __popc(__ballot_sync(0xffffffffu, is_cand));
        const unsigned hb = __ballot_sync(0xffffffffu, hit);
        if (hb) {
          const int l = __ffs(hb) - 1;
          q = base + l;
          v = __shfl_sync(0xffffffffu, pv, l);
          break;
        }
      }
      __syncwarp();
      if (q < 0) continue;  // no pivot in this column
      // the pivot row reduced by the pivots so far: U = v ^ sum_{k: v bit pcol_k} g_k
      uint64_t x = 0;
      if (lane < t && ((v >> s_pcol[lane]) & 1ull)) x ^= G[lane];
      if (lane + 32 < t && ((v >> s_pcol[lane + 32]) & 1ull)) x ^= G[lane + 32];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x ^= __shfl_xor_sync(0xffffffffu, x, o);
      U = v ^ x;
      // transposition (i, q): the pivot row takes position i; the window row
      // there (bit col clear, reduced by every pivot) goes to position q, with
      // the bound of its reduced word
      const int ei = i - i0;
      const uint64_t vi = __shfl_sync(0xffffffffu, pick64(ei >> 5), ei & 31);
      const int ri = __shfl_sync(0xffffffffu, pickr(ei >> 5), ei & 31);
      const int ap = gf2_row_at(q, p2r, stamp, epoch);  // before the maps change
      __syncwarp();
      if (lane == 0) {
        const int hv = vi ? __ffsll((long long)vi) - 1 : GF2_HEAD_NONE;
        atomicSub(&s_cnt[head[ap]], 1);  // the pivot row leaves the counts
        head[ri] = (uint8_t)hv;
        atomicAdd(&s_cnt[hv], 1);
        p2r[q] = ri;
        stamp[q] = epoch;
      }
#pragma unroll
      for (int u = 0; u < GF2_WU; ++u)
        if (lane + 32 * u == ei) {
          wv[u] = U;
          wr[u] = ap;
        }
    }
    if (basis) basis_add(U, col, t);
    if (lane == 0) {
      s_U[t] = U;
      s_pcol[t] = col;
      s_ti[t] = i;
      s_tq[t] = q;
    }
    __syncwarp();
    ++i;
    ++t;
  }
  // last final position of a non-pivot row with a nonzero word
  int hi = i - 1;
  for (int k = lane; k < t; k += 32) hi = max(hi, s_tq[k]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  int last = -1;
#pragma unroll
  for (int u = 0; u < GF2_WU; ++u) {
    const int pos = i0 + lane + 32 * u;
    if (pos >= i && pos <= hi && wr[u] >= 0 && act[wr[u]]) last = max(last, pos);
  }
  for (int pos = max(i, wend) + lane; pos <= hi && pos < m; pos += 32)
    if (act[gf2_row_at(pos, p2r, stamp, epoch)]) last = max(last, pos);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) last = max(last, __shfl_xor_sync(0xffffffffu, last, o));
  if (lane == 0) {
    const int la = *last_act;
    if (la > hi) last = la;
    out->t = (uint32_t)t;
    out->last_pos = (uint32_t)(last >= 0 ? last : 0);
    *last_act = -1;
    hout->t = (uint32_t)t;
    hout->last_pos = (uint32_t)(last >= 0 ? last : 0);
  }
  // the outputs; the result also goes to mapped host memory, then the
  // sequence flag
  __syncwarp();
  for (int k = lane; k < t; k += 32) {
    Uout[k] = s_U[k];
    out->ti[k] = hout->ti[k] = (uint32_t)s_ti[k];
    out->tq[k] = hout->tq[k] = (uint32_t)s_tq[k];
    out->pcol[k] = hout->pcol[k] = (uint32_t)s_pcol[k];
  }
  __threadfence_system();
  __syncwarp();
  if (lane == 0) *hflag = seq;
}

// Rows i0..r1 at their final positions: the reference's elimination steps
// on the panel word give the multipliers (L11 row of pivot row k over the
// pivots before it; L21 row of the rows below over all t) and the final
// word (U_k; zero below).  One thread per row.
__global__ void gf2_solve_kernel(uint64_t *__restrict__ D, size_t ld, int i0, int r1, int wc,
                                 uint64_t pmask, int t, const uint32_t *__restrict__ pcol,
                                 const uint64_t *__restrict__ Uin, uint64_t *__restrict__ L11,
                                 uint64_t *__restrict__ L21) {
  __shared__ uint64_t sU[GW];
  __shared__ int sP[GW];
  if (threadIdx.x < GW) {
    sU[threadIdx.x] = threadIdx.x < t ? Uin[threadIdx.x] : 0ull;
    sP[threadIdx.x] = threadIdx.x < t ? (int)pcol[threadIdx.x] : 0;
  }
  __syncthreads();
  const int r0 = i0 + t;
  for (int pos = i0 + blockIdx.x * blockDim.x + threadIdx.x; pos <= r1;
       pos += gridDim.x * blockDim.x) {
    uint64_t *x = D + (size_t)pos * ld + wc;
    uint64_t v = *x & pmask;
    const int kk = pos - i0, lim = kk < t ? kk : t;
    uint64_t l = 0;
    for (int k = 0; k < lim; ++k)
      if ((v >> sP[k]) & 1ull) {
        v ^= sU[k];
        l |= 1ull << k;
      }
    *x = (*x & ~pmask) | v;
    if (kk < t)
      L11[kk] = l;
    else
      L21[pos - r0] = l;
  }
}

// Row permutation in one launch: each CTA takes GF2_PERM_WORDS words of
// every moved row.  Its threads load all their words of the source rows at
// once (at most GF2_PERM_PER each, into registers), wait at the barrier,
// then store them to the destination rows; the CTAs own disjoint words, so
// no grid-wide ordering is needed.  cnt <= 2 * GW rows.
constexpr int GF2_PERM_THREADS = 256, GF2_PERM_WORDS = 16;
constexpr int GF2_PERM_PER = 2 * GW * GF2_PERM_WORDS / GF2_PERM_THREADS;
__global__ void __launch_bounds__(GF2_PERM_THREADS)
    gf2_permute_rows_kernel(uint64_t *__restrict__ D, size_t ld, int nw,
                            const int *__restrict__ src, const int *__restrict__ dst, int cnt) {
  const int w0 = blockIdx.x * GF2_PERM_WORDS, total = cnt * GF2_PERM_WORDS;
  uint64_t v[GF2_PERM_PER];
#pragma unroll
  for (int u = 0; u < GF2_PERM_PER; ++u) {
    const int e = threadIdx.x + u * GF2_PERM_THREADS, w = w0 + e % GF2_PERM_WORDS;
    v[u] = (e < total && w < nw) ? D[(size_t)src[e / GF2_PERM_WORDS] * ld + w] : 0ull;
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < GF2_PERM_PER; ++u) {
    const int e = threadIdx.x + u * GF2_PERM_THREADS, w = w0 + e % GF2_PERM_WORDS;
    if (e < total && w < nw) D[(size_t)dst[e / GF2_PERM_WORDS] * ld + w] = v[u];
  }
}

// U12 = L11^-1 A12 over GF(2): pivot rows i0..i0+t-1, words w1 .. nw-1;
// row k gets the XOR of the earlier pivot rows j whose bit is set in
// L11[k].  One warp per word, lane l holding rows l and l + 32: step k hands
// the finished row k to the warp (one shuffle) and the later rows whose
// L11 row has bit k XOR it in (right-looking, 64 short steps per word
// instead of a thread's 2016 dependent XORs).
constexpr int GF2_L11_THREADS = 256;
__global__ void __launch_bounds__(GF2_L11_THREADS)
    gf2_l11_solve_kernel(uint64_t *__restrict__ D, size_t ld, int i0, int t, int w1, int nw,
                         const uint64_t *__restrict__ L11) {
  const int lane = threadIdx.x & 31;
  const int w = w1 + (int)((blockIdx.x * (size_t)GF2_L11_THREADS + threadIdx.x) >> 5);
  if (w >= nw) return;  // whole warps
  const uint64_t l0 = lane < t ? L11[lane] : 0ull, l1 = lane + 32 < t ? L11[lane + 32] : 0ull;
  uint64_t x0 = lane < t ? D[(size_t)(i0 + lane) * ld + w] : 0ull;
  uint64_t x1 = lane + 32 < t ? D[(size_t)(i0 + lane + 32) * ld + w] : 0ull;
  for (int k = 0; k < t - 1; ++k) {
    const uint64_t xk = __shfl_sync(0xffffffffu, k < 32 ? x0 : x1, k & 31);
    if (lane > k && ((l0 >> k) & 1ull)) x0 ^= xk;
    if ((l1 >> k) & 1ull) x1 ^= xk;  // L11 is strictly lower: bit k set means k < the row
  }
  if (lane < t) D[(size_t)(i0 + lane) * ld + w] = x0;
  if (lane + 32 < t) D[(size_t)(i0 + lane + 32) * ld + w] = x1;
}

// The panel's multipliers into the block's rows of bits: rows i0..r1, the
// t bits of L11 (pivot rows) or L21 (rows below) at bit offset off of the
// row's GB words (the caller zeroed the block's rows).
constexpr int GB = 8;  // panels (words) per block of delayed updates
__global__ void gf2_deposit_kernel(uint64_t *__restrict__ Lb, int i0, int r1, int t, int off,
                                   const uint64_t *__restrict__ L11,
                                   const uint64_t *__restrict__ L21) {
  const int r0 = i0 + t;
  for (int pos = i0 + blockIdx.x * blockDim.x + threadIdx.x; pos <= r1;
       pos += gridDim.x * blockDim.x) {
    const uint64_t l = pos < r0 ? L11[pos - i0] : L21[pos - r0];
    uint64_t *row = Lb + (size_t)pos * GB;
    const int wq = off >> 6, sh = off & 63;
    row[wq] |= l << sh;
    if (sh && sh + t > 64) row[wq + 1] |= l >> (64 - sh);
  }
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
  // p2r, stamp (m each); permutation lists (4 GW); last row (1); histogram (GW + 1)
  const size_t i_bytes =
      (((size_t)2 * m + 4 * GW + 1 + GW + 1) * sizeof(int) + 255) & ~(size_t)255;
  const size_t h_bytes = ((size_t)2 * m + 255) & ~(size_t)255;
  void *base = nullptr;
  const size_t lb_bytes = (size_t)m * GB * 8 + (size_t)GB * GW * 8;  // block bits, panel L11s
  int st = ctx_buffer(c, BUF_GF2_0,
                      out_bytes + i_bytes + h_bytes + (size_t)m * 8 + 2 * GW * 8 + lb_bytes + 1024,
                      &base);
  if (st) return st;
  uint8_t *b8 = static_cast<uint8_t *>(base);
  Gf2PanelOut *d_out = reinterpret_cast<Gf2PanelOut *>(b8);
  int *d_p2r = reinterpret_cast<int *>(b8 + out_bytes);
  int *d_stamp = d_p2r + m;
  int *d_perm = d_stamp + m;      // 4*GW ints
  int *d_last = d_perm + 4 * GW;  // largest row with a nonzero word
  int *d_hist = d_last + 1;       // GW + 1 head counts
  uint8_t *d_head = b8 + out_bytes + i_bytes;
  uint8_t *d_act = d_head + m;
  uint64_t *d_L21 = reinterpret_cast<uint64_t *>(b8 + out_bytes + i_bytes + h_bytes);
  uint64_t *d_L11 = d_L21 + m;
  uint64_t *d_U = d_L11 + GW;
  uint64_t *d_Lb = d_U + GW;                 // m x GB words
  uint64_t *d_L11s = d_Lb + (size_t)m * GB;                       // GB x GW words
  const uint32_t *d_pcol = reinterpret_cast<const uint32_t *>(b8 + offsetof(Gf2PanelOut, pcol));
  static_assert(sizeof(Gf2PanelOut) <= PANEL_FLAG_OFF, "panel result and flag share the mapped page");
  void *mh = nullptr, *md = nullptr;
  if ((st = ctx_panel_map(c, &mh, &md))) return st;
  const Gf2PanelOut *hmap = static_cast<const Gf2PanelOut *>(mh);
  int *hperm = reinterpret_cast<int *>(static_cast<char *>(mh) + PANEL_PERM_OFF);
  static_assert(sizeof(Gf2PanelOut) <= PANEL_PERM_OFF && 2 * (2 * GW) <= (int)PANEL_PERM_INTS, "staging layout");
  volatile uint32_t *hflag = reinterpret_cast<volatile uint32_t *>(static_cast<char *>(mh) + PANEL_FLAG_OFF);
  Gf2PanelOut *hmap_dev = static_cast<Gf2PanelOut *>(md);
  uint32_t *hflag_dev = reinterpret_cast<uint32_t *>(static_cast<char *>(md) + PANEL_FLAG_OFF);
  cudaError_t e = cudaMemsetAsync(d_stamp, 0xff, (size_t)m * sizeof(int), c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_last, 0xff, sizeof(int), c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_hist, 0, (GW + 1) * sizeof(int), c->stream);
  if (e != cudaSuccess) return ctx_cuda(c, e, "gf2 echelon: scratch");

  Gf2PanelOut h;
  std::vector<int> at, src, dst;
  int i = 0, epoch = 0;
  const int head_grid = std::max(1, std::min((m + GF2_HEADS_THREADS - 1) / GF2_HEADS_THREADS,
                                             c->num_sms * 2));
  // Blocks of GB words (delayed updates), as in the Z/p form: when the
  // block's first panel with pivots has at least DELAY_ROWS rows below it,
  // the block's panels update only the block's words; the words right of it
  // get, per block, U12 = L11^-1 A12 on the block's pivot rows (panel by
  // panel: the earlier panels' part by a gemm, then the panel's own L11) and
  // one C ^= L21 U12 with K = the block's pivots (up to 64 GB bits) on the rows
  // below.  d_Lb row q (GB words) holds the multipliers of the row at
  // position q, panel k of the block at bits Tb_k .. Tb_k + t_k - 1; later
  // panels' transpositions move d_Lb's rows with D's.
  constexpr int DELAY_ROWS = 512;
  int ib = 0, Tb = 0, R = -1, bw1 = 0, delayed = 0, np = 0;
  int pan_i[GB], pan_t[GB], pan_off[GB];
  auto flush = [&]() -> int {
    if (Tb == 0 || bw1 >= nw) return ST_OK;
    const int nrest = n - 64 * bw1;  // bits right of the block
    for (int j = 0; j < np; ++j) {
      if (pan_off[j] > 0) {
        // M = this panel's pivots (<= 64 rows): the four-Russians kernel,
        // which needs no byte expansion of the wide B
        int s = gf2_gemm_dev(c, GF2_M4RM, pan_t[j], nrest, pan_off[j], 1,
                             d_Lb + (size_t)pan_i[j] * GB, GB, D + (size_t)ib * ld + bw1, ld, 1,
                             D + (size_t)pan_i[j] * ld + bw1, ld);
        if (s) return s;
      }
      gf2_l11_solve_kernel<<<(nw - bw1 + GF2_L11_THREADS / 32 - 1) / (GF2_L11_THREADS / 32),
                             GF2_L11_THREADS, 0, c->stream>>>(D, ld, pan_i[j], pan_t[j], bw1, nw,
                                                              d_L11s + (size_t)j * GW);
      ctx_launched(c);
    }
    const int rb = ib + Tb;
    if (R < rb) return ST_OK;
    int pi = prof_begin(c, "gf2_block_update");
    int s = gf2_gemm_dev(c, GF2_AUTO, R - rb + 1, nrest, Tb, 1, d_Lb + (size_t)rb * GB, GB,
                         D + (size_t)ib * ld + bw1, ld, 1, D + (size_t)rb * ld + bw1, ld);
    prof_end(c, pi);
    return s;
  };
  for (int wc = 0; wc < nw && i < m; ++wc) {
    const int w = std::min(64, n - 64 * wc);
    if (wc % GB == 0) {
      if ((st = flush())) return st;
      ib = i;
      Tb = 0;
      R = -1;
      np = 0;
      bw1 = std::min(nw, wc + GB);
      delayed = -1;  // decided at the block's first panel with pivots
    }
    const uint64_t pmask = (w == 64) ? ~0ull : ((1ull << w) - 1ull);
    int pi = prof_begin(c, "gf2_heads");
    gf2_heads_kernel<<<head_grid, GF2_HEADS_THREADS, 0, c->stream>>>(
        D, ld, i, m, wc, pmask, d_head, d_act, d_hist, d_last, i + GF2_WR);
    prof_end(c, pi);
    const uint32_t seq = ++c->panel_seq;
    pi = prof_begin(c, "gf2_search");
    gf2_search_kernel<<<1, 32, 0, c->stream>>>(
        D, ld, i, m, wc, w, pmask, d_head, d_act, d_hist, d_last, d_p2r, d_stamp, epoch++, d_U,
        d_out, hmap_dev, hflag_dev, seq);
    prof_end(c, pi);
    ctx_launched(c, 2);
    if ((st = ctx_wait_flag(c, hflag, seq, "gf2 echelon: panel"))) return st;
    h.t = hmap->t;
    h.last_pos = hmap->last_pos;
    for (uint32_t k = 0; k < h.t && k < (uint32_t)GW; ++k) {
      h.ti[k] = hmap->ti[k];
      h.tq[k] = hmap->tq[k];
      h.pcol[k] = hmap->pcol[k];
    }
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
      for (int k = 0; k < cnt; ++k) {
        hperm[k] = src[k];
        hperm[cnt + k] = dst[k];
      }
      e = cudaMemcpyAsync(d_perm, hperm, (size_t)2 * cnt * sizeof(int), cudaMemcpyHostToDevice,
                          c->stream);
      if (e != cudaSuccess) return ctx_cuda(c, e, "gf2 echelon: permutation");
      gf2_permute_rows_kernel<<<(nw + GF2_PERM_WORDS - 1) / GF2_PERM_WORDS, GF2_PERM_THREADS, 0,
                                c->stream>>>(D, ld, nw, d_perm, d_perm + cnt, cnt);
      ctx_launched(c);
      if (Tb > 0) {  // the block's earlier multipliers move with their rows
        gf2_permute_rows_kernel<<<(GB + GF2_PERM_WORDS - 1) / GF2_PERM_WORDS, GF2_PERM_THREADS,
                                  0, c->stream>>>(d_Lb, GB, GB, d_perm, d_perm + cnt, cnt);
        ctx_launched(c);
      }
    }
    const int r0 = i + t;
    const int r1 = (h.last_pos >= (uint32_t)r0) ? (int)h.last_pos : r0 - 1;
    const int below = r1 - r0 + 1;
    if (delayed < 0) {
      delayed = below >= DELAY_ROWS && bw1 < nw;
      if (delayed) {  // rows the panels' solves do not reach hold zero multipliers
        e = cudaMemsetAsync(d_Lb + (size_t)i * GB, 0, (size_t)(m - i) * GB * 8, c->stream);
        if (e != cudaSuccess) return ctx_cuda(c, e, "gf2 echelon: multipliers");
      }
    }
    {
      const int rows = r1 - i + 1;
      pi = prof_begin(c, "gf2_solve");
      gf2_solve_kernel<<<std::max(1, std::min((rows + 255) / 256, c->num_sms * 4)), 256, 0,
                         c->stream>>>(D, ld, i, r1, wc, pmask, t, d_pcol, d_U, d_L11, d_L21);
      prof_end(c, pi);
      ctx_launched(c);
    }
    if (delayed) {
      const int rows = r1 - i + 1;
      gf2_deposit_kernel<<<std::max(1, std::min((rows + 255) / 256, c->num_sms * 4)), 256, 0,
                           c->stream>>>(d_Lb, i, r1, t, Tb, d_L11, d_L21);
      e = cudaMemcpyAsync(d_L11s + (size_t)np * GW, d_L11, (size_t)t * 8, cudaMemcpyDeviceToDevice,
                          c->stream);
      if (e != cudaSuccess) return ctx_cuda(c, e, "gf2 echelon: panel multipliers");
      ctx_launched(c);
    }
    // the rest of the block's words (delayed), or of all words
    const int w1 = wc + 1, wend = delayed ? bw1 : nw;
    if (w1 < wend) {
      gf2_l11_solve_kernel<<<(wend - w1 + GF2_L11_THREADS / 32 - 1) / (GF2_L11_THREADS / 32),
                             GF2_L11_THREADS, 0, c->stream>>>(D, ld, i, t, w1, wend, d_L11);
      ctx_launched(c);
      if (below > 0) {
        // rows r0..r1, those words: C ^= L21 (one word of t bits per row) * U12
        pi = prof_begin(c, "gf2_update");
        st = gf2_m4rm_dev(c, below, std::min(n, 64 * wend) - 64 * w1, t, 1, d_L21, 1,
                          D + (size_t)i * ld + w1, ld, 1, D + (size_t)r0 * ld + w1, ld);
        prof_end(c, pi);
        if (st) return st;
      }
    }
    if (delayed) {
      pan_i[np] = i;
      pan_t[np] = t;
      pan_off[np] = Tb;
      ++np;
      R = std::max(R, std::max(r1, hi));
      Tb += t;
    }
    rank += t;
    i += t;
  }
  if ((st = flush())) return st;
  *rank_out = rank;
  return ST_OK;
}

}  // namespace lela
