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
// multiplies det, and every row below with a nonzero a in column c gets
// row_i * (-a/x) added.  Pivots are not normalised.
//
// Blocked right-looking form, exact.  The columns are taken in panels of
// W = 64.  Facts the design rests on, for one panel:
//  * the value of a row after elimination by the panel's pivot rows
//    U_0..U_{t-1} is the unique vector of v + span(U) that is zero in the
//    pivot columns, whatever order the eliminations take, and so are the
//    multipliers l (v = l U + reduced);
//  * after the whole panel every row below the pivots is zero in all W
//    columns (a skipped column was zero in every row at or below the
//    current row, and every later pivot row is zero there as well);
//  * the pivot of column c is the first row at or below the current row
//    whose reduced entry in c is nonzero, and that entry only involves the
//    row's entries in the pivot columns found so far and in c.
// So per panel:
//  1. panel_heads_kernel: each row at or below the current row records the
//     first nonzero column of its panel part (64: none), with a histogram;
//  2. panel_search_kernel (one CTA) replays the reference's pivot choice on
//     a window of the first rows, held in shared memory and eliminated
//     eagerly without division (a row W becomes y W - W[c] P for pivot row
//     P with pivot value y), so no inverse is on this sequential path; rows
//     below the window are reduced only when the head histogram says one of
//     them may hold a pivot the window lacks.  The pivot inverses and the
//     pivot rows U_k come out of parallel inversions at the end, and, after
//     the host has been signalled and when many rows are to be solved, the
//     inverse of the pivot block U_P (the pivot rows at the pivot columns);
//  3. the host replays the recorded transpositions and moves the affected
//     rows (at most two per pivot) with one gather;
//  4. panel_solve_inv_kernel / panel_solve_kernel (all SMs, one warp per
//     row): for every row from the first pivot to the last possibly nonzero
//     row, its multipliers (the L11 row of a pivot row, the L21 row
//     otherwise): a_P U_P^-1 from its entries a_P at the pivot columns, or
//     the reference's elimination steps on its panel part; the panel becomes
//     U_k in pivot row k and zero below;
//  5. U12 = L11^-1 A12 on CUDA cores and A22 -= L21 U12 on the limb-split
//     tensor-core gemm over the rows down to the last possibly nonzero row,
//     for the columns of the panel's block of EB columns; the columns right
//     of the block get one such update per block, with the multipliers of
//     all its panels (K up to EB = 16 W instead of W: a sixteenth of the
//     passes over the trailing matrix).
// F4 Schur complements are staircase-shaped (rows sorted by head), so few
// rows are touched per panel; dense matrices make every row active and the
// scheme becomes ordinary blocked LU with LELA's pivot choice.
#include <algorithm>
#include <cstddef>
#include <mutex>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "context.h"
#include "echelon.h"
#include "tri.h"
#include "zp_gemm.h"

namespace lela {

constexpr int EW = 64;                     // panel width
constexpr int EB = 16 * EW;                // block of panels sharing one trailing update
constexpr int PS_THREADS = 512;            // panel search CTA
constexpr int PS_FAST = PS_THREADS / 32;   // positions tested per column by whole warps
constexpr uint8_t HEAD_NONE = 64;

struct PanelOut {
  uint32_t t;         // pivots found in the panel
  uint32_t err;       // 1: a pivot is not invertible in Modular<uint32>
  uint32_t uinv;      // 1: U_P^-1 written (the rows to solve take panel_solve_inv_kernel)
  uint32_t last_pos;  // largest final position of a non-pivot row with a nonzero panel (or 0)
  uint32_t det;       // product of the panel's pivots
  uint32_t pad[3];
  uint32_t pcol[EW];  // pivot columns (relative to c0)
  uint32_t ti[EW];    // transposition k: (ti[k], tq[k])
  uint32_t tq[EW];
};

// Exact inverse of a unit x modulo p (any p < 2^32): extended Euclid on
// unsigned remainders with 64-bit signed coefficients.  0 when gcd != 1.
__device__ __forceinline__ uint32_t inv_exact_u32(uint32_t p, uint32_t x) {
  uint32_t r0 = p, r1 = x;
  int64_t s0 = 0, s1 = 1;
  while (r1 != 0) {
    const uint32_t q = r0 / r1;
    const uint32_t r = r0 - q * r1;
    r0 = r1;
    r1 = r;
    const int64_t s = s0 - (int64_t)q * s1;
    s0 = s1;
    s1 = s;
  }
  if (r0 != 1) return 0;
  int64_t v = s0 % (int64_t)p;
  if (v < 0) v += p;
  return (uint32_t)v;
}

// Row index currently at position pos: positions touched by this panel's
// transpositions carry the panel's epoch stamp.
__device__ __forceinline__ int row_at(int pos, const int *p2r, const int *stamp, int epoch) {
  return stamp[pos] == epoch ? p2r[pos] : pos;
}

// sum of two products a*b + c*d modulo p (a, b, c, d < p < 2^32)
__device__ __forceinline__ uint32_t mod_dot2(uint32_t a, uint32_t b, uint32_t c, uint32_t d,
                                             const Modulus &mod, uint32_t two64) {
  const uint64_t x = (uint64_t)a * b, y = (uint64_t)c * d;
  uint64_t s = x + y;
  if (s < y) s += two64;
  return mod_reduce(s, mod);
}

// Field arithmetic for the panel kernels, in two forms chosen by the host:
// ArithSmall for p < 2^16 (every product fits in 32 bits; Barrett reduction
// with a 32-bit reciprocal, one correction) and ArithWide for any p < 2^32
// (64-bit products and Barrett reduction).  Both return canonical residues.
struct ArithSmall {
  uint32_t p, mu;  // mu = floor(2^32 / p)
  __host__ static ArithSmall make(uint32_t p) {
    ArithSmall a;
    a.p = p;
    a.mu = (uint32_t)((1ull << 32) / p);
    return a;
  }
  __device__ __forceinline__ uint32_t red(uint32_t x) const {
    const uint32_t r = x - __umulhi(x, mu) * p;
    return r >= p ? r - p : r;
  }
  __device__ __forceinline__ uint32_t mul(uint32_t a, uint32_t b) const { return red(a * b); }
  // a*b + c*d
  __device__ __forceinline__ uint32_t dot2(uint32_t a, uint32_t b, uint32_t c, uint32_t d) const {
    const uint32_t r = red(a * b) + red(c * d);
    return r >= p ? r - p : r;
  }
  // s += a*b for a sum of products reduced once at the end (red64): each
  // product is below 2^32, so up to 2^16 of them fit
  __device__ __forceinline__ void acc(uint64_t &s, uint32_t a, uint32_t b) const {
    s += (uint64_t)a * b;
  }
  // s mod p for s < 2^48: (s mod 2^32 reduced) + (s / 2^32) (2^32 mod p)
  __device__ __forceinline__ uint32_t red64(uint64_t s) const {
    const uint32_t c32 = 0u - mu * p;
    return red(red((uint32_t)s) + (uint32_t)(s >> 32) * c32);
  }
};
struct ArithWide {
  Modulus mod;
  uint32_t p, two64;
  __host__ static ArithWide make(uint32_t p) {
    ArithWide a;
    a.mod = make_modulus(p);
    a.p = p;
    a.two64 = two64_mod(p);
    return a;
  }
  __device__ __forceinline__ uint32_t mul(uint32_t a, uint32_t b) const {
    return mod_mul(a, b, mod);
  }
  __device__ __forceinline__ uint32_t dot2(uint32_t a, uint32_t b, uint32_t c, uint32_t d) const {
    return mod_dot2(a, b, c, d, mod, two64);
  }
  // s += a*b modulo p: on a wrap past 2^64 the lost 2^64 comes back as
  // 2^64 mod p (the sum then stays below 2^64: it is below the product)
  __device__ __forceinline__ void acc(uint64_t &s, uint32_t a, uint32_t b) const {
    const uint64_t x = (uint64_t)a * b;
    s += x;
    if (s < x) s += two64;
  }
  __device__ __forceinline__ uint32_t red64(uint64_t s) const { return mod_reduce(s, mod); }
};

// Inverse of a 64 x 64 triangular matrix X (row stride LD, shared memory)
// in place by doubling: the inverse of [[A, B], [0, C]] is [[A^-1, -A^-1 B
// C^-1], [0, C^-1]] (lower: [[A^-1, 0], [-C^-1 B A^-1, C^-1]]), so the
// diagonal blocks of sizes 1, 2, 4, .., 32 are inverted level by level,
// each level two products of b x b blocks (through T, 32 b entries) over
// all pairs at once.  On entry the diagonal holds the inverses of the
// diagonal entries and the rest of the triangle the matrix's entries, the
// other triangle zero (the products run over whole blocks, zeros included).
// Every thread of the CTA calls it (12 barriers).  A
// triangular matrix with unit diagonal entries has one inverse over Z/p,
// so the result is the one any substitution gives.
template <class A, bool UPPER, int LD, int B>
__device__ __forceinline__ void tri64_invert_level(uint32_t (*X)[LD], uint32_t *T, const A &ar,
                                                   int tid, int nthreads) {
  // products over whole b x b blocks (the zero triangle included): fixed
  // trip counts, unrolled
  constexpr int n = (EW / (2 * B)) * B * B;
  const uint32_t p = ar.p;
  for (int e = tid; e < n; e += nthreads) {
    const int q = e / (B * B), ii = (e / B) % B, jj = e % B, r = 2 * B * q;
    uint64_t acc = 0;
#pragma unroll
    for (int kk = 0; kk < B; ++kk) {
      if constexpr (UPPER) ar.acc(acc, X[r + ii][r + B + kk], X[r + B + kk][r + B + jj]);  // B C^-1
      else ar.acc(acc, X[r + B + ii][r + kk], X[r + kk][r + jj]);                          // B A^-1
    }
    T[e] = ar.red64(acc);
  }
  __syncthreads();
  for (int e = tid; e < n; e += nthreads) {
    const int q = e / (B * B), ii = (e / B) % B, jj = e % B, r = 2 * B * q;
    const uint32_t *Tq = T + q * B * B;
    uint64_t acc = 0;
#pragma unroll
    for (int kk = 0; kk < B; ++kk) {
      if constexpr (UPPER) ar.acc(acc, X[r + ii][r + kk], Tq[kk * B + jj]);  // -A^-1 (B C^-1)
      else ar.acc(acc, X[r + B + ii][r + B + kk], Tq[kk * B + jj]);         // -C^-1 (B A^-1)
    }
    const uint32_t v = ar.red64(acc);
    if constexpr (UPPER) X[r + ii][r + B + jj] = v ? p - v : 0u;
    else X[r + B + ii][r + jj] = v ? p - v : 0u;
  }
  __syncthreads();
}

template <class A, bool UPPER, int LD>
__device__ void tri64_invert(uint32_t (*X)[LD], uint32_t *T, const A &ar, int tid,
                             int nthreads) {
  static_assert(EW == 64, "six levels");
  tri64_invert_level<A, UPPER, LD, 1>(X, T, ar, tid, nthreads);
  tri64_invert_level<A, UPPER, LD, 2>(X, T, ar, tid, nthreads);
  tri64_invert_level<A, UPPER, LD, 4>(X, T, ar, tid, nthreads);
  tri64_invert_level<A, UPPER, LD, 8>(X, T, ar, tid, nthreads);
  tri64_invert_level<A, UPPER, LD, 16>(X, T, ar, tid, nthreads);
  tri64_invert_level<A, UPPER, LD, 32>(X, T, ar, tid, nthreads);
}

// 1. First nonzero column of each row's panel part, rows i0..m-1 (one warp
// per row); the histogram of these heads (hist[0..64], which the caller
// has zeroed) and the largest row index with a nonzero panel (*last, which
// the caller has set to -1).
constexpr int HEADS_THREADS = 256;
__global__ void __launch_bounds__(HEADS_THREADS)
    panel_heads_kernel(const uint32_t *__restrict__ D, size_t ld, int i0, int m, int c0, int w,
                       uint8_t *__restrict__ head, uint8_t *__restrict__ act, int *hist,
                       int *last) {
  __shared__ int s_last;
  __shared__ int s_hist[EW + 1];
  if (threadIdx.x == 0) s_last = -1;
  if (threadIdx.x <= EW) s_hist[threadIdx.x] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  int my_last = -1;
  for (int r = i0 + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); r < m; r += warps) {
    const uint32_t *row = D + (size_t)r * ld + c0;
    const uint32_t a = lane < w ? row[lane] : 0u;
    const uint32_t b = lane + 32 < w ? row[lane + 32] : 0u;
    const unsigned ba = __ballot_sync(0xffffffffu, a != 0u);
    const unsigned bb = __ballot_sync(0xffffffffu, b != 0u);
    const int h = ba ? __ffs(ba) - 1 : (bb ? 32 + __ffs(bb) - 1 : HEAD_NONE);
    if (lane == 0) {
      head[r] = (uint8_t)h;
      act[r] = h < HEAD_NONE;
      atomicAdd(&s_hist[h], 1);
    }
    if (h < HEAD_NONE) my_last = r;
  }
  if (lane == 0 && my_last >= 0) atomicMax(&s_last, my_last);
  __syncthreads();
  if (threadIdx.x == 0 && s_last >= 0) atomicMax(last, s_last);
  if (threadIdx.x <= EW && s_hist[threadIdx.x]) atomicAdd(&hist[threadIdx.x], s_hist[threadIdx.x]);
}

// 2. The reference's pivot choice on the panel (see the file comment).
// The window: the first wcap <= PW_R rows at or below i0, by position, with a nonzero
// in the panel, kept in shared memory and eliminated eagerly without
// division: when pivot row P (pivot value y) is chosen, every window row W
// becomes y W - W[col] P.  So a window row holds S_t times its row reduced
// by the t pivots so far (S_t = y_0 ... y_{t-1}); pivot rows move to PV,
// holding S_k U_k.  Rows between window rows are zero in the panel and can
// never hold a pivot.  The pivot of a column is the first window row, by
// position, with a nonzero there; rows past the last window position are
// reached only when no window row has one and the head histogram says one
// of them may: they are then reduced by the same recurrence, in position
// order.  At the end the S_k and the pivots x_k = y_k / S_k are inverted in
// parallel.  Outputs: PanelOut; U (t x EW, row stride EW: the pivot rows'
// final panel values) and the pivot inverses.  Resets *last_act to -1 and
// hist[] to zero for the next panel.
//
// Bookkeeping: the window is a list of entries sorted by position, entry ->
// shared-memory slot (perm) and position (ppos), double-buffered and
// rewritten each column (or, when only its first entry leaves, read from one
// entry further on); wrow[slot] is the row index in D.  A transposition
// (i, q) moves the row at position i to q: a window row keeps its entry
// (with position q); a row outside the window (zero in the panel) is
// recorded in p2r / stamp.  Rows past the window carry in head[] a lower
// bound of the first nonzero column of their reduced panel part; cnt[h]
// counts them by that bound.
constexpr int PW_R = 80;                   // window rows
// window rows padded to EW + 1 words: a column read across rows (the pivot
// test, the multipliers) then touches every bank once
constexpr int PW_LD = EW + 1;
constexpr size_t PW_SMEM = (size_t)PW_R * PW_LD * 4;  // dynamic shared memory: the window rows
constexpr int PW_EU = (PW_R + 31) / 32;  // window list entries per lane
// rows to solve from which the panel's multipliers come from U_P^-1
constexpr int SOLVE_INV_ROWS = 768;

template <class A>
__global__ void __launch_bounds__(PS_THREADS, 1)
    panel_search_kernel(const uint32_t *__restrict__ D, size_t ld, int i0, int m, int c0, int w,
                        A ar, uint8_t *__restrict__ head, const uint8_t *__restrict__ act,
                        int *__restrict__ hist, int *__restrict__ last_act, int *__restrict__ p2r,
                        int *__restrict__ stamp, int epoch, uint32_t *__restrict__ Uout,
                        uint32_t *__restrict__ xinv_out, uint32_t *__restrict__ Uinv_out,
                        PanelOut *out, PanelOut *hout, volatile uint32_t *hflag, uint32_t seq,
                        int wcap) {
  extern __shared__ __align__(16) uint32_t dyn_w[];
  uint32_t(*Wv)[PW_LD] = reinterpret_cast<uint32_t(*)[PW_LD]>(dyn_w);  // PW_R rows
  __shared__ uint32_t PV[EW][EW];
  __shared__ int perm[2][PW_R], ppos[2][PW_R];
  __shared__ int wrow[PW_R];
  __shared__ uint32_t s_red[PS_FAST][EW];  // rows past the window, reduced (one per warp)
  __shared__ int s_pcol[EW];
  __shared__ uint32_t s_y[EW], s_S[EW], s_x[EW], s_sinv[EW], s_yinv[EW], s_xi[EW];
  __shared__ int s_cnt[EW + 1];
  __shared__ int s_first[PS_FAST], s_wcnt[PS_FAST];
  __shared__ int s_list[PS_THREADS], s_lrow[PS_THREADS], s_lhead[PS_THREADS];
  __shared__ int s_err, s_last, s_hi, s_wlast, s_uinv;
  const uint32_t p = ar.p;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;

  // the window: ordered compaction of the rows with a nonzero panel
  int nl = 0;
  if (tid == 0) s_wlast = m - 1;
  if (tid <= EW) {
    s_cnt[tid] = hist[tid];
    hist[tid] = 0;
  }
  for (int base = i0; base < m && nl < wcap; base += PS_THREADS) {
    const int pos = base + tid;
    const bool a = pos < m && act[pos];
    const unsigned bal = __ballot_sync(0xffffffffu, a);
    if (lane == 0) s_wcnt[wid] = __popc(bal);
    __syncthreads();
    int off = 0, cnt = 0;
    for (int k = 0; k < PS_FAST; ++k) {
      const int v = s_wcnt[k];
      off += k < wid ? v : 0;
      cnt += v;
    }
    off += __popc(bal & ((1u << lane) - 1u));
    const int take = min(cnt, wcap - nl);
    if (a && off < take) {
      const int slot = nl + off;
      perm[0][slot] = slot;
      ppos[0][slot] = pos;
      wrow[slot] = pos;
      atomicSub(&s_cnt[head[pos]], 1);  // the window's rows leave the counts
      if (off == wcap - 1 - nl) s_wlast = pos;
    }
    nl += take;
    __syncthreads();  // s_wcnt is rewritten by the next pass
  }
  // the window rows' panel values: all threads, consecutive lanes on
  // consecutive columns of a row (coalesced reads)
  for (int e = tid; e < nl * EW; e += PS_THREADS) {
    const int slot = e / EW, c = e % EW;
    cp_async4(&Wv[slot][c], D + (size_t)wrow[slot] * ld + c0 + (c < w ? c : 0), c < w);
  }
  cp_async_wait_all();
  __syncthreads();
  const int wlast = s_wlast;  // rows past it are outside the window

  int cur = 0, off = 0, i = i0, t = 0;  // the entry list: perm[cur] / ppos[cur] from off
  uint32_t S = 1u % p;
  for (int col = 0; col < w && i < m; ++col) {
    const int *pm = perm[cur] + off, *pp = ppos[cur] + off;
    int *pn = perm[cur ^ 1], *ppn = ppos[cur ^ 1];
    // A. first window entry (by position) with a nonzero in col.  Every warp
    // finds it by itself: column col of the window and the entry list were
    // last written before the previous column's closing barrier, and the
    // work of this column (phase B) writes only columns right of col and the
    // other list buffer, so no barrier is needed here
    int qs = 0x7fffffff;
    for (int base = 0; base < nl; base += 32) {
      const int e = base + lane;
      const bool nz = e < nl && Wv[pm[e]][col] != 0u;
      const unsigned b = __ballot_sync(0xffffffffu, nz);
      if (b) {
        qs = base + __ffs(b) - 1;
        break;
      }
    }
    const bool z = nl > 0 && pp[0] == i;  // the row at position i is window entry 0
    const uint32_t *P;                    // the pivot row (S_t times reduced)
    int q, drop;                          // pivot position; window entry leaving (-1: none)
    bool relocate0 = false;               // entry 0 moves to position q, in place of qs
    if (qs == 0x7fffffff) {
      // none in the window: rows past it whose bound allows a pivot here
      // (a warp-wide sum; every warp computes the same count)
      int cand = 0;
      if (wlast < m - 1) {
        const int v = (lane <= col ? s_cnt[lane] : 0) + (lane + 32 <= col ? s_cnt[lane + 32] : 0);
        cand = __reduce_add_sync(0xffffffffu, v);
      }
      // no barrier when there is no candidate: nothing shared changes
      if (cand == 0) continue;
      __syncthreads();  // every thread has its count before s_cnt changes
      // per pass the CTA lists the candidates among PS_THREADS positions
      // (ordered compaction), then each warp reduces one of them by the t
      // pivots, W <- y_k W - W[pcol_k] (S_k U_k), and records its exact head
      int found = -1, fw = 0;
      for (int base = wlast + 1; base < m && cand > 0 && found < 0; base += PS_THREADS) {
        const int pos = base + tid;
        int r = -1, hr = HEAD_NONE;
        if (pos < m) {
          r = row_at(pos, p2r, stamp, epoch);
          hr = head[r];
        }
        const bool isc = hr <= col;
        const unsigned bal = __ballot_sync(0xffffffffu, isc);
        if (lane == 0) s_wcnt[wid] = __popc(bal);
        __syncthreads();
        int off = 0, ncand = 0;
        for (int k = 0; k < PS_FAST; ++k) {
          const int v = s_wcnt[k];
          off += k < wid ? v : 0;
          ncand += v;
        }
        if (isc) {
          const int o = off + __popc(bal & ((1u << lane) - 1u));
          s_list[o] = pos;
          s_lrow[o] = r;
          s_lhead[o] = hr;
        }
        __syncthreads();
        for (int j0 = 0; j0 < ncand && found < 0; j0 += PS_FAST) {
          const int j = j0 + wid;
          int hit_pos = 0x7fffffff;
          if (j < ncand) {
            const int rj = s_lrow[j], hrj = s_lhead[j];
            const uint32_t *v = D + (size_t)rj * ld + c0;
            uint32_t a0 = lane < w ? v[lane] : 0u, a1 = lane + 32 < w ? v[lane + 32] : 0u;
            for (int k = 0; k < t; ++k) {
              const int pc = s_pcol[k];
              const uint32_t f = __shfl_sync(0xffffffffu, pc < 32 ? a0 : a1, pc & 31);
              const uint32_t nf = f ? p - f : 0u;
              a0 = ar.dot2(s_y[k], a0, nf, PV[k][lane]);
              a1 = ar.dot2(s_y[k], a1, nf, PV[k][lane + 32]);
            }
            s_red[wid][lane] = a0;
            s_red[wid][lane + 32] = a1;
            const unsigned b0 = __ballot_sync(0xffffffffu, a0 != 0u && lane >= col);
            const unsigned b1 = __ballot_sync(0xffffffffu, a1 != 0u && lane + 32 >= col);
            const int hn = b0 ? __ffs(b0) - 1 : (b1 ? 32 + __ffs(b1) - 1 : HEAD_NONE);
            if (hn == col) hit_pos = s_list[j];
            if (lane == 0 && hn != hrj) {
              head[rj] = (uint8_t)hn;
              atomicSub(&s_cnt[hrj], 1);
              atomicAdd(&s_cnt[hn], 1);
            }
          }
          if (lane == 0) s_first[wid] = hit_pos;
          __syncthreads();
          for (int k = 0; k < PS_FAST; ++k)
            if (s_first[k] < (found < 0 ? 0x7fffffff : found)) {
              found = s_first[k];
              fw = k;
            }
          __syncthreads();  // s_first and s_red are rewritten by the next round
        }
        cand -= ncand;
      }
      if (found < 0) {
        __syncthreads();
        continue;
      }
      // the pivot comes from past the window; the row at position i goes to
      // position `found`: window entry 0 leaves the window (with the bound
      // of its values), a row outside it is recorded in p2r
      q = found;
      P = s_red[fw];
      drop = z ? 0 : -1;
      if (wid == 0) {
        int hd = HEAD_NONE;
        if (z) {
          const uint32_t *E = Wv[pm[0]];
          const unsigned b0 = __ballot_sync(0xffffffffu, E[lane] != 0u && lane > col);
          const unsigned b1 = __ballot_sync(0xffffffffu, E[lane + 32] != 0u && lane + 32 > col);
          hd = b0 ? __ffs(b0) - 1 : (b1 ? 32 + __ffs(b1) - 1 : HEAD_NONE);
        }
        if (lane == 0) {
          const int rq = row_at(q, p2r, stamp, epoch);
          atomicSub(&s_cnt[head[rq]], 1);
          int ri;
          if (z) {
            ri = wrow[pm[0]];
            head[ri] = (uint8_t)hd;
            atomicAdd(&s_cnt[hd], 1);
          } else {
            ri = row_at(i, p2r, stamp, epoch);
          }
          p2r[q] = ri;
          stamp[q] = epoch;
        }
      }
    } else {
      q = pp[qs];
      P = Wv[pm[qs]];
      drop = qs;
      relocate0 = z && qs > 0;
      if (!z && q != i && tid == 0) {  // the row at i is outside the window
        p2r[q] = row_at(i, p2r, stamp, epoch);
        stamp[q] = epoch;
      }
    }
    // B. eliminate the window rows that stay, keep the pivot row in PV, and
    // write the new entry list
    const uint32_t y = P[col];
    {
      // Warp wid takes the columns col + 1 + wid, col + 17 + wid, ..; lane
      // takes the list entries lane, lane + 32, lane + 64.  An entry's
      // multiplier W[col] is loaded once for all of the warp's columns, and
      // two columns are in flight at a time (their loads issued before
      // their stores).
      // NU groups of 32 entries, NU fixed per instantiation (the window
      // shrinks by one entry per pivot, so most columns need one or two)
      auto elim = [&](auto nu_c) {
        constexpr int NU = decltype(nu_c)::value;
        int pr[NU];
        uint32_t na[NU];
#pragma unroll
        for (int u = 0; u < NU; ++u) {
          const int s = lane + 32 * u;
          pr[u] = (s < nl && s != drop) ? pm[s] : -1;
          const uint32_t a = pr[u] >= 0 ? Wv[pr[u]][col] : 0u;
          na[u] = a ? p - a : 0u;
        }
        for (int c = col + 1 + wid; c < w; c += 2 * PS_FAST) {
          const int c2 = c + PS_FAST;
          const bool two = c2 < w;
          const uint32_t pc = P[c], pc2 = two ? P[c2] : 0u;
          uint32_t wv[NU], wv2[NU];
#pragma unroll
          for (int u = 0; u < NU; ++u) {
            wv[u] = pr[u] >= 0 ? Wv[pr[u]][c] : 0u;
            wv2[u] = (pr[u] >= 0 && two) ? Wv[pr[u]][c2] : 0u;
          }
#pragma unroll
          for (int u = 0; u < NU; ++u)
            if (pr[u] >= 0) {
              Wv[pr[u]][c] = ar.dot2(y, wv[u], na[u], pc);
              if (two) Wv[pr[u]][c2] = ar.dot2(y, wv2[u], na[u], pc2);
            }
        }
      };
      static_assert(PW_EU == 3, "the dispatch below covers three groups");
      const int nu = (nl + 31) >> 5;
      if (nu <= 1)
        elim(std::integral_constant<int, 1>{});
      else if (nu == 2)
        elim(std::integral_constant<int, 2>{});
      else
        elim(std::integral_constant<int, 3>{});
    }
    if (tid < EW) PV[t][tid] = P[tid];
    const int nn = drop >= 0 ? nl - 1 : nl;
    // the new entry list; when entry 0 leaves and nothing moves (a pivot at
    // the row at position i, the usual case) it is the old list from its
    // second entry, and nothing is copied
    const bool shift = drop == 0 && !relocate0;
    for (int s = tid; s < nn && !shift; s += PS_THREADS) {
      int src, pos;
      if (relocate0) {
        src = s < drop - 1 ? s + 1 : (s == drop - 1 ? 0 : s + 1);
        pos = s == drop - 1 ? q : pp[src];
      } else {
        src = (drop >= 0 && s >= drop) ? s + 1 : s;
        pos = pp[src];
      }
      pn[s] = pm[src];
      ppn[s] = pos;
    }
    if (tid == 0) {
      s_pcol[t] = col;
      s_y[t] = y;
      s_S[t] = S;
      out->pcol[t] = (uint32_t)col;
      out->ti[t] = (uint32_t)i;
      out->tq[t] = (uint32_t)q;
    }
    __syncthreads();
    if (shift) {
      ++off;
    } else {
      cur ^= 1;
      off = 0;
    }
    nl = nn;
    S = ar.mul(S, y);
    ++i;
    ++t;
  }

  // inverses in parallel: S_k^-1 (exact), the pivots x_k = y_k / S_k, and
  // the reference's inverse of each pivot (its failure is the reference's
  // error)
  if (tid == 0) {
    s_err = 0;
    s_last = -1;
    s_hi = i - 1;
  }
  __syncthreads();
  // For p < 2^31 the reference's inverse is the exact one, so x_k^-1 =
  // S_k y_k^-1, and the two inversions of pivot k run side by side (threads
  // k and 64 + k); for larger p the reference's inverse of x_k itself.
  const bool exact_inv = p < 0x80000000u;
  if (tid < t) {
    s_sinv[tid] = inv_exact_u32(p, s_S[tid]);
    atomicMax(&s_hi, (int)out->tq[tid]);
  } else if (exact_inv && tid >= EW && tid < EW + t) {
    s_yinv[tid - EW] = inv_exact_u32(p, s_y[tid - EW]);
  }
  __syncthreads();
  if (tid < t) {
    const uint32_t si = s_sinv[tid];
    const uint32_t x = ar.mul(s_y[tid], si);
    const uint32_t xi = exact_inv ? ar.mul(s_S[tid], s_yinv[tid]) : lela_inv_u32(p, x);
    s_x[tid] = x;
    s_xi[tid] = xi;
    xinv_out[tid] = xi;
    if (si == 0u || xi == 0u) atomicOr(&s_err, 1);
  }
  __syncthreads();
  // U_k = (S_k U_k) / S_k; entries left of the pivot column are not kept up
  // to date, and U_k is zero there
  for (int e = tid; e < t * EW; e += PS_THREADS) {
    const int k = e / EW, c = e % EW;
    Uout[e] = c < s_pcol[k] ? 0u : ar.mul(PV[k][c], s_sinv[k]);
  }
  // last final position of a non-pivot row with a nonzero panel: the window
  // entries, positions past the window up to the largest transposition target
  // through p2r; beyond that rows have not moved
  const int hi = s_hi;
  for (int s = tid; s < nl; s += PS_THREADS)
    if (act[wrow[perm[cur][off + s]]]) atomicMax(&s_last, ppos[cur][off + s]);
  for (int pos = max(wlast + 1, i) + tid; pos <= hi && pos < m; pos += PS_THREADS)
    if (act[row_at(pos, p2r, stamp, epoch)]) atomicMax(&s_last, pos);
  __syncthreads();
  // the panel's determinant factor: product of the x_k, by warp 0
  uint32_t det = 1u % p;
  if (wid == 0) {
    uint32_t v = lane < t ? s_x[lane] : 1u % p;
    if (lane + 32 < t) v = ar.mul(v, s_x[lane + 32]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = ar.mul(v, __shfl_xor_sync(0xffffffffu, v, o));
    det = v;
  }
  if (tid == 0) {
    const int la = *last_act;
    int last = s_last;
    if (la > hi) last = max(last, la);
    // the rows the panel's solve takes: i0 .. max(last, i0 + t - 1)
    const int rows = max(last, i0 + t - 1) - i0 + 1;
    s_uinv = exact_inv && t > 0 && rows >= SOLVE_INV_ROWS;
    out->uinv = hout->uinv = (uint32_t)s_uinv;
    out->t = (uint32_t)t;
    out->err = (uint32_t)s_err;
    out->last_pos = (uint32_t)(last >= 0 ? last : 0);
    out->det = det;
    *last_act = -1;
    hout->t = (uint32_t)t;
    hout->err = (uint32_t)s_err;
    hout->last_pos = (uint32_t)(last >= 0 ? last : 0);
    hout->det = det;
  }
  // the result also goes to mapped host memory, then a sequence flag: the
  // host waits on the flag instead of a copy and a stream synchronisation
  __syncthreads();
  for (int k = tid; k < t; k += PS_THREADS) {
    hout->pcol[k] = out->pcol[k];
    hout->ti[k] = out->ti[k];
    hout->tq[k] = out->tq[k];
  }
  __threadfence_system();
  __syncthreads();
  if (tid == 0) *hflag = seq;
  // After the flag, so that it overlaps the host's handling of the result
  // (its only reader is the next kernel on the stream): for p < 2^31 (exact
  // pivot inverses), when at least SOLVE_INV_ROWS rows are to be solved (it
  // costs a few microseconds), the inverse of U_P, the t x t upper triangular matrix of
  // the pivot rows at the pivot columns (U_P[k][j] = U_k[pcol_j], diagonal
  // x_k), padded to 64 x 64 with the identity.  A row's multipliers are then
  // a_P U_P^-1 (a_P: its values at the pivot columns), all at once.  In the
  // window's shared memory, now free.
  if (s_uinv) {
    uint32_t(*X)[PW_LD] = Wv;
    uint32_t *T = dyn_w + EW * PW_LD;
    static_assert(EW * PW_LD + 32 * EW / 2 <= PW_R * PW_LD, "inverse scratch fits the window");
    for (int e = tid; e < EW * EW; e += PS_THREADS) {
      const int k = e / EW, j = e % EW;
      uint32_t v;
      if (k >= t || j >= t) v = k == j ? 1u : 0u;
      else if (j < k) v = 0u;
      else if (j == k) v = s_xi[k];
      else v = ar.mul(PV[k][s_pcol[j]], s_sinv[k]);
      X[k][j] = v;
    }
    __syncthreads();
    tri64_invert<A, true, PW_LD>(X, T, ar, tid, PS_THREADS);
    for (int e = tid; e < t * EW; e += PS_THREADS) Uinv_out[e] = X[e / EW][e % EW];
  }
}

// Row permutation in one launch: each CTA takes a slice of PERM_COLS
// columns of every moved row.  Its threads load all their elements of the
// source rows at once (at most PERM_PER each, into registers), wait at the
// barrier, then store them to the destination rows; the CTAs own disjoint
// columns, so no grid-wide ordering is needed.  cnt <= 2 * EW rows.
constexpr int PERM_THREADS = 256, PERM_COLS = 32;
constexpr int PERM_PER = 2 * EW * PERM_COLS / PERM_THREADS;
__global__ void __launch_bounds__(PERM_THREADS)
    permute_rows_kernel(uint32_t *__restrict__ D, size_t ld, int n, const int *__restrict__ src,
                        const int *__restrict__ dst, int cnt) {
  const int c0 = blockIdx.x * PERM_COLS, total = cnt * PERM_COLS;
  uint32_t v[PERM_PER];
#pragma unroll
  for (int u = 0; u < PERM_PER; ++u) {
    const int e = threadIdx.x + u * PERM_THREADS, c = c0 + e % PERM_COLS;
    v[u] = (e < total && c < n) ? D[(size_t)src[e / PERM_COLS] * ld + c] : 0u;
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < PERM_PER; ++u) {
    const int e = threadIdx.x + u * PERM_THREADS, c = c0 + e % PERM_COLS;
    if (e < total && c < n) D[(size_t)dst[e / PERM_COLS] * ld + c] = v[u];
  }
}

// 4. Rows i0..r1 at their final positions, one warp per row: the
// reference's elimination steps on the panel part, pivot k applied with
// multiplier l_k = v[pcol_k] / x_k (v: the row's current value) and
// v -= l_k U_k.  Pivot row k takes the pivots before it (its L11 row, unit
// lower; its panel becomes U_k); rows below take all t (their L21 row; their
// panel becomes zero).  Row i0 + r of L = [L11; L21] goes to
// Lout[r * ldl + 0 .. t-1].
constexpr int SOLVE_THREADS = 256;
template <class A>
__global__ void __launch_bounds__(SOLVE_THREADS)
    panel_solve_kernel(uint32_t *__restrict__ D, size_t ld, int i0, int r1, int c0, int w, int t,
                       const uint32_t *__restrict__ pcol, const uint32_t *__restrict__ Uin,
                       const uint32_t *__restrict__ xinv, A ar, uint32_t *__restrict__ Lout,
                       size_t ldl) {
  __shared__ uint32_t sU[EW][EW];
  __shared__ uint32_t sX[EW];
  __shared__ int sP[EW];
  const int tid = threadIdx.x, lane = tid & 31;
  for (int e = tid; e < t * EW; e += SOLVE_THREADS) cp_async4(&sU[e / EW][e % EW], Uin + e, true);
  if (tid < EW) {
    sX[tid] = tid < t ? xinv[tid] : 0u;
    sP[tid] = tid < t ? (int)pcol[tid] : 0;
  }
  cp_async_wait_all();
  __syncthreads();
  const uint32_t p = ar.p;
  const int warps = (gridDim.x * SOLVE_THREADS) >> 5;
  for (int pos = i0 + ((blockIdx.x * SOLVE_THREADS + tid) >> 5); pos <= r1; pos += warps) {
    uint32_t *row = D + (size_t)pos * ld + c0;
    uint32_t a0 = lane < w ? row[lane] : 0u, a1 = lane + 32 < w ? row[lane + 32] : 0u;
    const int kk = pos - i0, lim = kk < t ? kk : t;
    uint32_t l0 = 0u, l1 = 0u;  // multipliers k = lane, lane + 32
    if (__any_sync(0xffffffffu, (a0 | a1) != 0u)) {
      for (int k = 0; k < lim; ++k) {
        const int pc = sP[k];
        const uint32_t f = __shfl_sync(0xffffffffu, pc < 32 ? a0 : a1, pc & 31);
        const uint32_t l = ar.mul(f, sX[k]);
        if (k == lane) l0 = l;
        if (k == lane + 32) l1 = l;
        const uint32_t nl = l ? p - l : 0u;
        a0 = ar.dot2(1u, a0, nl, sU[k][lane]);
        a1 = ar.dot2(1u, a1, nl, sU[k][lane + 32]);
      }
    }
    if (lane < w) row[lane] = a0;
    if (lane + 32 < w) row[lane + 32] = a1;
    uint32_t *lr = Lout + (size_t)kk * ldl;
    if (kk < t) {
      if (lane < t) lr[lane] = lane < kk ? l0 : (lane == kk ? 1u : 0u);
      if (lane + 32 < t) lr[lane + 32] = lane + 32 < kk ? l1 : (lane + 32 == kk ? 1u : 0u);
    } else {
      if (lane < t) lr[lane] = l0;
      if (lane + 32 < t) lr[lane + 32] = l1;
    }
  }
}

// The same results for p < 2^31 from the inverse of U_P (the search's
// Uinv, t x EW): a row's multipliers are l = a_P U_P^-1 (a_P: the row's
// values at the pivot columns), one dot product of length t per lane
// instead of t dependent elimination steps.  A pivot row k (position i0 +
// k) keeps multipliers l_j for j < k and 1 at k (a_P = sum_{j<k} l_j U_P[j] +
// U_P[k]), and its panel becomes U_k; every other row's panel becomes zero
// (each panel column either holds a pivot, eliminated from all rows below
// it, or was zero at and below the pivot row when it was reached).
template <class A>
__global__ void __launch_bounds__(SOLVE_THREADS)
    panel_solve_inv_kernel(uint32_t *__restrict__ D, size_t ld, int i0, int r1, int c0, int w,
                           int t, const uint32_t *__restrict__ pcol,
                           const uint32_t *__restrict__ Uin, const uint32_t *__restrict__ Uinv,
                           A ar, uint32_t *__restrict__ Lout, size_t ldl) {
  __shared__ uint32_t sUi[EW][EW];
  __shared__ int sP[EW];
  const int tid = threadIdx.x, lane = tid & 31;
  for (int e = tid; e < t * EW; e += SOLVE_THREADS) cp_async4(&sUi[e / EW][e % EW], Uinv + e, true);
  if (tid < EW) sP[tid] = tid < t ? (int)pcol[tid] : 0;
  cp_async_wait_all();
  __syncthreads();
  const int pc0 = sP[lane], pc1 = sP[lane + 32];
  const int warps = (gridDim.x * SOLVE_THREADS) >> 5;
  for (int pos = i0 + ((blockIdx.x * SOLVE_THREADS + tid) >> 5); pos <= r1; pos += warps) {
    uint32_t *row = D + (size_t)pos * ld + c0;
    const uint32_t a0 = lane < w ? row[lane] : 0u, a1 = lane + 32 < w ? row[lane + 32] : 0u;
    // the row's values at the pivot columns: lane j holds a[pcol_j], a[pcol_{j+32}]
    const uint32_t x0 = __shfl_sync(0xffffffffu, a0, pc0 & 31);
    const uint32_t x1 = __shfl_sync(0xffffffffu, a1, pc0 & 31);
    const uint32_t y0 = __shfl_sync(0xffffffffu, a0, pc1 & 31);
    const uint32_t y1 = __shfl_sync(0xffffffffu, a1, pc1 & 31);
    const uint32_t ap0 = lane < t ? (pc0 < 32 ? x0 : x1) : 0u;
    const uint32_t ap1 = lane + 32 < t ? (pc1 < 32 ? y0 : y1) : 0u;
    uint32_t l0 = 0u, l1 = 0u;  // multipliers k = lane, lane + 32
    if (__any_sync(0xffffffffu, (ap0 | ap1) != 0u)) {
      uint64_t s0 = 0, s1 = 0;
      for (int j = 0; j < t; ++j) {
        const uint32_t f = __shfl_sync(0xffffffffu, j < 32 ? ap0 : ap1, j & 31);
        ar.acc(s0, f, sUi[j][lane]);
        ar.acc(s1, f, sUi[j][lane + 32]);
      }
      l0 = ar.red64(s0);
      l1 = ar.red64(s1);
    }
    const int kk = pos - i0;
    uint32_t *lr = Lout + (size_t)kk * ldl;
    if (kk < t) {
      if (lane < w) row[lane] = Uin[(size_t)kk * EW + lane];
      if (lane + 32 < w) row[lane + 32] = Uin[(size_t)kk * EW + lane + 32];
      if (lane < t) lr[lane] = lane < kk ? l0 : (lane == kk ? 1u : 0u);
      if (lane + 32 < t) lr[lane + 32] = lane + 32 < kk ? l1 : (lane + 32 == kk ? 1u : 0u);
    } else {
      if (lane < w) row[lane] = 0u;
      if (lane + 32 < w) row[lane + 32] = 0u;
      if (lane < t) lr[lane] = l0;
      if (lane + 32 < t) lr[lane + 32] = l1;
    }
  }
}

// U12 = L11^-1 A12 for one panel, in place: forward substitution x_k = a_k -
// sum_{j<k} L11[k][j] x_j with the unit lower L11 (the panel's multipliers of
// its pivot rows, row stride ldl) in shared memory.  Four lanes per column
// of A12, lane l holding the column's entries j = l mod 4 in registers (the
// loops fully unrolled, so every register index is a constant): per k each
// lane sums its share of the products, two shuffles add the four shares, and
// the owner of entry k updates it.  The same field operations as any
// substitution with a unit diagonal.
constexpr int U12_THREADS = 128;
constexpr int U12_COLS = U12_THREADS / 4;
template <class A>
__global__ void __launch_bounds__(U12_THREADS)
    panel_u12_kernel(const uint32_t *__restrict__ L, size_t ldl, int t, uint32_t *__restrict__ B,
                     size_t ldb, int ncols, A ar) {
  __shared__ __align__(16) uint32_t sL[EW][EW];
  {
    constexpr int PER = EW * EW / U12_THREADS;
    uint32_t v[PER];
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const int e = threadIdx.x + u * U12_THREADS, k = e / EW, j = e % EW;
      v[u] = (k < t && j < k) ? L[(size_t)k * ldl + j] : 0u;
    }
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const int e = threadIdx.x + u * U12_THREADS;
      sL[e / EW][e % EW] = v[u];
    }
  }
  __syncthreads();
  const int l4 = threadIdx.x & 3;
  const int c = blockIdx.x * U12_COLS + (threadIdx.x >> 2);
  const bool valid = c < ncols;  // every lane stays for the shuffles
  const uint32_t p = ar.p;
  uint32_t x[EW / 4];  // x[i]: entry 4 i + l4
#pragma unroll
  for (int i = 0; i < EW / 4; ++i) {
    const int j = 4 * i + l4;
    x[i] = (valid && j < t) ? B[(size_t)j * ldb + c] : 0u;
  }
#pragma unroll
  for (int k = 1; k < EW; ++k) {
    if (k < t) {
      // entries j >= k still hold a_j, but L11[k][j] is zero there
      uint64_t acc = 0;
#pragma unroll
      for (int i = 0; i <= (k - 1) / 4; ++i) ar.acc(acc, sL[k][4 * i + l4], x[i]);
      uint32_t v = ar.red64(acc);
#pragma unroll
      for (int o = 1; o <= 2; o <<= 1) {  // v + w mod p without overflow (any p < 2^32)
        const uint32_t nw = p - __shfl_xor_sync(0xffffffffu, v, o);
        v = v >= nw ? v - nw : v + (p - nw);
      }
      if (l4 == (k & 3)) {
        const uint32_t a = x[k >> 2];
        x[k >> 2] = a >= v ? a - v : a + (p - v);
      }
    }
  }
#pragma unroll
  for (int i = 0; i < EW / 4; ++i) {
    const int j = 4 * i + l4;
    if (valid && j >= 1 && j < t) B[(size_t)j * ldb + c] = x[i];
  }
}

int zp_echelon_dev(Ctx *c, int m, int n, uint32_t p, uint32_t *D, size_t ld, size_t *rank_out,
                   uint32_t *det_out, std::vector<int> *pivot_cols, EchelonKeep *keep) {
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

  // device scratch
  const size_t out_bytes = (sizeof(PanelOut) + 255) & ~(size_t)255;
  // p2r, stamp (m each); permutation lists (4 EW); last row (1); histogram (EW + 1)
  const size_t i_bytes =
      (((size_t)2 * m + 4 * EW + 1 + EW + 1) * sizeof(int) + 255) & ~(size_t)255;
  const size_t h_bytes = ((size_t)2 * m + 255) & ~(size_t)255;
  const size_t sq_bytes = (size_t)EW * EW * 4;
  const size_t l_bytes = (size_t)m * EB * 4;
  void *base = nullptr;
  int st = ctx_buffer(c, BUF_ECH_0,
                      out_bytes + i_bytes + h_bytes + 3 * sq_bytes + l_bytes + 1024,
                      &base);
  if (st) return st;
  uint8_t *b8 = static_cast<uint8_t *>(base);
  PanelOut *d_out = reinterpret_cast<PanelOut *>(b8);
  int *d_p2r = reinterpret_cast<int *>(b8 + out_bytes);
  int *d_stamp = d_p2r + m;
  int *d_perm = d_stamp + m;      // 4*EW ints: src list, dst list
  int *d_last = d_perm + 4 * EW;  // largest row with a nonzero panel
  int *d_hist = d_last + 1;       // EW + 1 head counts
  uint8_t *d_head = b8 + out_bytes + i_bytes;
  uint8_t *d_act = d_head + m;
  uint32_t *d_U = reinterpret_cast<uint32_t *>(b8 + out_bytes + i_bytes + h_bytes);
  uint32_t *d_xinv = d_U + EW * EW;  // pivot inverses (EW)
  uint32_t *d_Uinv = d_xinv + EW * EW;  // U_P^-1 (t x EW), p < 2^31
  uint32_t *d_L = d_Uinv + EW * EW;  // the block's multipliers (m x EB)
  const uint32_t *d_pcol = reinterpret_cast<const uint32_t *>(b8 + offsetof(PanelOut, pcol));
  void *gws = nullptr;
  // one size for the panel and block updates and the block's trsm (which
  // takes the same workspace, so it must not grow it)
  st = ctx_workspace(c, std::max(zp_gemm_workspace_bytes(p, m, n, EB),
                                 zp_trsm_workspace_bytes(p, EB, n)),
                     &gws);
  if (st) return st;
  const bool small = p < (1u << 16);
  if ((st = ctx_smem_attr(c, (const void *)panel_search_kernel<ArithSmall>, (int)PW_SMEM,
                          "echelon: panel search attributes")) ||
      (st = ctx_smem_attr(c, (const void *)panel_search_kernel<ArithWide>, (int)PW_SMEM,
                          "echelon: panel search attributes")))
    return st;
  const ArithSmall ars = ArithSmall::make(p);
  const ArithWide arw = ArithWide::make(p);
  static_assert(sizeof(PanelOut) <= PANEL_FLAG_OFF, "panel result and flag share the mapped page");
  void *mh = nullptr, *md = nullptr;
  if ((st = ctx_panel_map(c, &mh, &md))) return st;
  const PanelOut *hmap = static_cast<const PanelOut *>(mh);
  int *hperm = reinterpret_cast<int *>(static_cast<char *>(mh) + PANEL_PERM_OFF);
  static_assert(sizeof(PanelOut) <= PANEL_PERM_OFF && 2 * (2 * EW) <= (int)PANEL_PERM_INTS, "staging layout");
  volatile uint32_t *hflag = reinterpret_cast<volatile uint32_t *>(static_cast<char *>(mh) + PANEL_FLAG_OFF);
  PanelOut *hmap_dev = static_cast<PanelOut *>(md);
  uint32_t *hflag_dev = reinterpret_cast<uint32_t *>(static_cast<char *>(md) + PANEL_FLAG_OFF);
  cudaError_t e = cudaMemsetAsync(d_stamp, 0xff, (size_t)m * sizeof(int), c->stream);
  if (e == cudaSuccess && keep) {
    keep->swaps.clear();
    e = cudaMemsetAsync(keep->L, 0, (size_t)m * keep->ldL * 4, c->stream);
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(d_last, 0xff, sizeof(int), c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_hist, 0, (EW + 1) * sizeof(int), c->stream);
  if (e != cudaSuccess) return ctx_cuda(c, e, "echelon: scratch");

  PanelOut h;
  std::vector<int> at, src, dst;
  int i = 0, epoch = 0;
  const int head_grid = std::max(1, std::min((m + 7) / 8, c->num_sms * 2));
  // Blocks of EB columns (delayed updates): a block's panels update only the
  // block's columns; the columns right of it are updated once per block,
  // U12 = L11^-1 A12 on the block's Tb pivot rows (from row ib) and
  // A22 -= L21 U12 on the rows below, down to R.  L = [L11; L21] holds the
  // block's multipliers: d_L row q (stride EB) belongs to the row at position
  // q, panel k of the block fills columns Tb_k .. Tb_k + t_k - 1, and later
  // panels' transpositions move d_L's rows with D's.  The result is the
  // panel-by-panel one: the multipliers are the same, and the delayed update
  // is the same Schur complement.  A block is delayed when the first panel
  // with pivots has at least DELAY_ROWS rows to update below them (dense
  // matrices); otherwise (staircase Schur complements, where few rows are
  // touched) each panel updates all columns at once and the block solve is
  // not paid.
  constexpr int DELAY_ROWS = 512;
  int ib = 0, Tb = 0, R = -1, b1 = 0, delayed = 0;
  auto flush = [&]() -> int {
    if (Tb == 0 || b1 >= n) return ST_OK;
    int s = zp_trsm_dev(c, false, true, Tb, n - b1, p, 1, d_L + (size_t)ib * EB, EB,
                        D + (size_t)ib * ld + b1, ld, nullptr);
    if (s) return s;
    const int rb = ib + Tb;
    if (R < rb) return ST_OK;
    int pi = prof_begin(c, "ech_block_update");
    s = zp_gemm_dev(c, GEMM_AUTO, R - rb + 1, n - b1, Tb, p, p - 1, d_L + (size_t)rb * EB, EB,
                    D + (size_t)ib * ld + b1, ld, 1, D + (size_t)rb * ld + b1, ld,
                    static_cast<uint8_t *>(gws));
    prof_end(c, pi);
    return s;
  };
  // window rows of the search: the full PW_R, or 64 when the previous panel
  // had many rows below its pivots (dense matrices, where the first 64
  // active rows nearly always hold the panel's pivots; the rows past the
  // window stay reachable through the search's slower path)
  int wcap = PW_R;
  for (int c0 = 0; c0 < n && i < m; c0 += EW) {
    const int w = std::min(EW, n - c0);
    if (c0 % EB == 0) {
      if ((st = flush())) return st;
      ib = i;
      Tb = 0;
      R = -1;
      b1 = std::min(n, c0 + EB);
      delayed = -1;  // decided at the block's first panel with pivots
    }
    int pi = prof_begin(c, "ech_heads");
    panel_heads_kernel<<<head_grid, HEADS_THREADS, 0, c->stream>>>(D, ld, i, m, c0, w, d_head,
                                                                    d_act, d_hist, d_last);
    prof_end(c, pi);
    const uint32_t seq = ++c->panel_seq;
    pi = prof_begin(c, "ech_search");
    if (small)
      panel_search_kernel<<<1, PS_THREADS, PW_SMEM, c->stream>>>(
          D, ld, i, m, c0, w, ars, d_head, d_act, d_hist, d_last, d_p2r, d_stamp, epoch, d_U,
          d_xinv, d_Uinv, d_out, hmap_dev, hflag_dev, seq, wcap);
    else
      panel_search_kernel<<<1, PS_THREADS, PW_SMEM, c->stream>>>(
          D, ld, i, m, c0, w, arw, d_head, d_act, d_hist, d_last, d_p2r, d_stamp, epoch, d_U,
          d_xinv, d_Uinv, d_out, hmap_dev, hflag_dev, seq, wcap);
    ++epoch;
    prof_end(c, pi);
    ctx_launched(c, 2);
    if ((st = ctx_wait_flag(c, hflag, seq, "echelon: panel"))) return st;
    h.t = hmap->t;
    h.uinv = hmap->uinv;
    h.err = hmap->err;
    h.last_pos = hmap->last_pos;
    h.det = hmap->det;
    for (uint32_t k = 0; k < h.t && k < (uint32_t)EW; ++k) {
      h.pcol[k] = hmap->pcol[k];
      h.ti[k] = hmap->ti[k];
      h.tq[k] = hmap->tq[k];
    }
    if (h.err) return ctx_fail(c, ST_PIVOT, "Could not invert pivot-element in the ring");
    const int t = (int)h.t;
    if (t == 0) continue;
    // replay the transpositions on the positions they touch
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
    if (cnt > 2 * EW) return ctx_fail(c, ST_ARG, "echelon: permutation larger than expected");
    if (cnt > 0) {
      for (int k = 0; k < cnt; ++k) {
        hperm[k] = src[k];
        hperm[cnt + k] = dst[k];
      }
      e = cudaMemcpyAsync(d_perm, hperm, (size_t)2 * cnt * sizeof(int), cudaMemcpyHostToDevice,
                          c->stream);
      if (e != cudaSuccess) return ctx_cuda(c, e, "echelon: permutation");
      permute_rows_kernel<<<(n + PERM_COLS - 1) / PERM_COLS, PERM_THREADS, 0, c->stream>>>(
          D, ld, n, d_perm, d_perm + cnt, cnt);
      ctx_launched(c);
      if (Tb > 0) {  // the multipliers of the block's earlier panels move too
        permute_rows_kernel<<<(EB + PERM_COLS - 1) / PERM_COLS, PERM_THREADS, 0, c->stream>>>(
            d_L, EB, EB, d_perm, d_perm + cnt, cnt);
        ctx_launched(c);
      }
      if (keep && rank > 0) {  // and every earlier pivot's kept multipliers
        permute_rows_kernel<<<((int)rank + PERM_COLS - 1) / PERM_COLS, PERM_THREADS, 0,
                              c->stream>>>(keep->L, keep->ldL, (int)rank, d_perm, d_perm + cnt,
                                           cnt);
        ctx_launched(c);
      }
    }
    // L11 / L21 and the panel's final values
    const int r0 = i + t;
    const int r1 = (h.last_pos >= (uint32_t)r0) ? (int)h.last_pos : r0 - 1;
    const int below = r1 - r0 + 1;
    wcap = below >= DELAY_ROWS ? EW : PW_R;
    if (delayed < 0) {
      delayed = below >= DELAY_ROWS;
      if (delayed) {  // rows a panel's solve does not reach hold zero multipliers
        e = cudaMemsetAsync(d_L + (size_t)i * EB, 0, (size_t)(m - i) * EB * 4, c->stream);
        if (e != cudaSuccess) return ctx_cuda(c, e, "echelon: multipliers");
      }
    }
    uint32_t *Lp = d_L + (size_t)i * EB + Tb;  // this panel's columns of L, from row i
    {
      const int groups = (r1 - i + 1 + SOLVE_THREADS / 32 - 1) / (SOLVE_THREADS / 32);
      pi = prof_begin(c, "ech_solve");
      const int sgrid = std::max(1, std::min(groups, c->num_sms * 8));
      // U_P^-1 when the search wrote it (p < 2^31: exact pivot inverses, and
      // many rows), else the elimination steps
      if (h.uinv && small)
        panel_solve_inv_kernel<<<sgrid, SOLVE_THREADS, 0, c->stream>>>(
            D, ld, i, r1, c0, w, t, d_pcol, d_U, d_Uinv, ars, Lp, EB);
      else if (h.uinv)
        panel_solve_inv_kernel<<<sgrid, SOLVE_THREADS, 0, c->stream>>>(
            D, ld, i, r1, c0, w, t, d_pcol, d_U, d_Uinv, arw, Lp, EB);
      else if (small)
        panel_solve_kernel<<<sgrid, SOLVE_THREADS, 0, c->stream>>>(D, ld, i, r1, c0, w, t, d_pcol,
                                                                   d_U, d_xinv, ars, Lp, EB);
      else
        panel_solve_kernel<<<sgrid, SOLVE_THREADS, 0, c->stream>>>(D, ld, i, r1, c0, w, t, d_pcol,
                                                                   d_U, d_xinv, arw, Lp, EB);
      prof_end(c, pi);
      ctx_launched(c);
    }
    if (keep) {
      // this panel's multipliers (rows i..r1) into columns rank.. of L
      e = cudaMemcpy2DAsync(keep->L + (size_t)i * keep->ldL + rank, keep->ldL * 4, Lp, EB * 4,
                            (size_t)t * 4, (size_t)(r1 - i + 1), cudaMemcpyDeviceToDevice,
                            c->stream);
      if (e != cudaSuccess) return ctx_cuda(c, e, "pluq: multipliers");
      for (int k = 0; k < t; ++k) keep->swaps.emplace_back((int)h.ti[k], (int)h.tq[k]);
    }
    // the rest of the block's columns (delayed), or of all columns
    const int rest = (delayed ? b1 : n) - (c0 + w);
    if (rest > 0) {
      uint32_t *U12 = D + (size_t)i * ld + c0 + w;
      pi = prof_begin(c, "ech_u12");
      const int ugrid = (rest + U12_COLS - 1) / U12_COLS;
      if (small)
        panel_u12_kernel<<<ugrid, U12_THREADS, 0, c->stream>>>(Lp, EB, t, U12, ld, rest, ars);
      else
        panel_u12_kernel<<<ugrid, U12_THREADS, 0, c->stream>>>(Lp, EB, t, U12, ld, rest, arw);
      prof_end(c, pi);
      ctx_launched(c);
      if (below > 0) {
        pi = prof_begin(c, "ech_update");
        st = zp_gemm_dev(c, GEMM_AUTO, below, rest, t, p, p - 1, Lp + (size_t)t * EB, EB, U12,
                         ld, 1, D + (size_t)r0 * ld + c0 + w, ld, static_cast<uint8_t *>(gws));
        prof_end(c, pi);
        if (st) return st;
      }
    }
    if (delayed) {
      // rows with multipliers: down to r1, and wherever a transposition moved one
      R = std::max(R, std::max(r1, hi));
      Tb += t;
    }
    det = (det * h.det) % p;
    if (pivot_cols)
      for (int k = 0; k < t; ++k) pivot_cols->push_back(c0 + (int)h.pcol[k]);
    rank += t;
    i += t;
  }
  if ((st = flush())) return st;
  *rank_out = rank;
  *det_out = (uint32_t)det;
  return ST_OK;
}

// ---------------------------------------------------------------- PLUQ
//
// Elimination::pluq (lela/algorithms/elimination.tcc:266-370) with
// DensePivotStrategy: at step i the first column, in the current column
// order, with a nonzero at or below row i, and its first such row, are
// swapped into place (transpositions (i, row) and (i, column)); det is
// multiplied by the pivot x; every row j below gets row_j - (a / x) row_i
// right of the pivot and keeps a / x below the diagonal.  A column passed
// over at step i is zero at and below row i and stays so, so the pivots are
// those of the non-reduced echelon form: the same rows, transpositions and
// values (the eliminations are the same field operations).  The echelon
// pipeline therefore runs with its multipliers kept (EchelonKeep); Q
// follows on the host from the pivot columns, and one gather writes L
// below the diagonal and U, its columns in Q's order, on and above it.

__global__ void pluq_assemble_kernel(const uint32_t *__restrict__ U, size_t ldu,
                                     const uint32_t *__restrict__ L, size_t ldl,
                                     const int *__restrict__ qcol, int m, int n, int r,
                                     uint32_t *__restrict__ out) {
  const size_t total = (size_t)m * n;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int q = (int)(idx / n), j = (int)(idx % n);
    out[idx] = j < min(q, r) ? L[(size_t)q * ldl + j] : U[(size_t)q * ldu + qcol[j]];
  }
}

int zp_pluq_dev(Ctx *c, int m, int n, uint32_t p, uint32_t *D, size_t ld,
                std::vector<std::pair<int, int>> *P, std::vector<std::pair<int, int>> *Q,
                size_t *rank, uint32_t *det) {
  P->clear();
  Q->clear();
  if (p < 2) return ctx_fail(c, ST_ARG, "modulus must be at least 2");
  if (m < 0 || n < 0) return ctx_fail(c, ST_ARG, "negative dimension");
  if (m == 0 || n == 0) {
    *rank = 0;
    *det = 1 % p;
    return ST_OK;
  }
  const int rmax = std::min(m, n);
  const size_t l_bytes = ((size_t)m * rmax * 4 + 255) & ~(size_t)255;
  const size_t o_bytes = ((size_t)m * n * 4 + 255) & ~(size_t)255;
  void *buf = nullptr;
  int st = ctx_buffer(c, BUF_PLUQ, l_bytes + o_bytes + (size_t)n * sizeof(int) + 256, &buf);
  if (st) return st;
  uint8_t *b8 = static_cast<uint8_t *>(buf);
  EchelonKeep keep;
  keep.L = reinterpret_cast<uint32_t *>(b8);
  keep.ldL = (size_t)rmax;
  uint32_t *out = reinterpret_cast<uint32_t *>(b8 + l_bytes);
  int *d_qcol = reinterpret_cast<int *>(b8 + l_bytes + o_bytes);
  std::vector<int> piv;
  if ((st = zp_echelon_dev(c, m, n, p, D, ld, rank, det, &piv, &keep))) return st;
  const int r = (int)*rank;
  for (const auto &sw : keep.swaps)
    if (sw.first != sw.second) P->push_back(sw);
  std::vector<int> qcol(n), where(n);  // position -> column, column -> position
  for (int j = 0; j < n; ++j) qcol[j] = where[j] = j;
  for (int i = 0; i < r; ++i) {
    const int pos = where[piv[i]];
    if (pos != i) {
      std::swap(qcol[i], qcol[pos]);
      where[qcol[i]] = i;
      where[qcol[pos]] = pos;
      Q->emplace_back(i, pos);
    }
  }
  std::reverse(P->begin(), P->end());  // the reference returns them reversed (:362-363)
  std::reverse(Q->begin(), Q->end());
  cudaError_t e = cudaMemcpyAsync(d_qcol, qcol.data(), (size_t)n * sizeof(int),
                                  cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) return ctx_cuda(c, e, "pluq: column order");
  const size_t total = (size_t)m * n;
  const int grid = (int)std::min<size_t>((total + 255) / 256, (size_t)c->num_sms * 16);
  pluq_assemble_kernel<<<grid, 256, 0, c->stream>>>(D, ld, keep.L, keep.ldL, d_qcol, m, n, r, out);
  ctx_launched(c);
  e = cudaMemcpy2DAsync(D, ld * 4, out, (size_t)n * 4, (size_t)n * 4, (size_t)m,
                        cudaMemcpyDeviceToDevice, c->stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  // the host vector qcol must outlive the copy above
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "pluq: assembly");
}

// ---------------------------------------------------------------------------
// The standard method's reduced form with its transform:
// Elimination::echelonize_reduced (A, L, P, rank, det, true) (lela/
// algorithms/elimination.tcc:143-265).  There L starts as the identity and
// takes every row operation of A, with each transposition applied to its
// rows and columns, so that at the end R = L B with B = P A_in (the
// transpositions in the order they were applied).
//
// The pivots, the transpositions and the pivot values of that loop are those
// of the non-reduced form (the rows at and below the current one are the
// same in both loops), so the panel pipeline above gives them, together
// with the non-reduced rows U (r x n) and the multipliers Lk (m x r, unit
// lower trapezoidal) with B = Lk U.  Write Lk = [L1; L2] (r and m - r rows)
// and U_P for U at the pivot columns (upper triangular, the pivots on its
// diagonal).  Pivot rows only ever receive multiples of pivot rows, and the
// other rows keep their own unit entry, so L = [[X, 0], [Y, I]]; R's pivot
// rows have the identity at the pivot columns, and its other rows are zero.
// Hence X = U_P^-1 L1^-1, Y = -L2 L1^-1, and R's first r rows are
// U_P^-1 U:
//   1. Lout <- I (m x m), T <- L1 (unit lower), W <- U_P;
//   2. Lout[0:r, 0:r] <- T^-1             (trsm, unit lower: no inversions);
//   3. Lout[r:m, 0:r] <- -L2 Lout[0:r, 0:r]           (gemm, alpha = p - 1);
//   4. Lout[0:r, 0:r] <- W^-1 Lout[0:r, 0:r]      (trsm, upper: the pivots);
//   5. D[0:r, :] <- W^-1 D[0:r, :]; D's rows from r on are zero already.
// The only inversions are of the pivots, as in the reference, so a pivot it
// cannot invert fails here too (in the panel pipeline, before any solve).
// ---------------------------------------------------------------------------

// Step 1.  T (r x r) <- the unit lower triangle of Lk's first r rows; W
// (r x r) <- D's first r rows at the pivot columns piv (row i of D is zero
// left of piv[i], so W is upper triangular); Lout (m x m) <- the identity.
__global__ void transform_setup_kernel(const uint32_t *__restrict__ Lk, size_t ldk,
                                       const uint32_t *__restrict__ D, size_t ldd,
                                       const int *__restrict__ piv, int m, int r,
                                       uint32_t *__restrict__ T, uint32_t *__restrict__ W,
                                       uint32_t *__restrict__ Lout, size_t ldl) {
  const size_t mm = (size_t)m * m, rr = (size_t)r * r;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < mm + 2 * rr;
       idx += (size_t)gridDim.x * blockDim.x) {
    if (idx < mm) {
      const size_t i = idx / m, j = idx % m;
      Lout[i * ldl + j] = i == j ? 1u : 0u;
    } else if (idx < mm + rr) {
      const size_t e = idx - mm, i = e / r, j = e % r;
      T[e] = j < i ? Lk[i * ldk + j] : (i == j ? 1u : 0u);
    } else {
      const size_t e = idx - mm - rr, i = e / r, j = e % r;
      W[e] = D[i * ldd + piv[j]];
    }
  }
}

int zp_echelon_transform_dev(Ctx *c, int m, int n, uint32_t p, uint32_t *D, size_t ld,
                             uint32_t *Lout, size_t ldl, std::vector<std::pair<int, int>> *P,
                             size_t *rank, uint32_t *det) {
  P->clear();
  if (p < 2) return ctx_fail(c, ST_ARG, "modulus must be at least 2");
  if (p >= 0x80000000u)
    return ctx_fail(c, ST_ARG,
                    "modulus must be below 2^31 (Modular<uint32>'s inverse wraps above it)");
  if (m < 0 || n < 0) return ctx_fail(c, ST_ARG, "negative dimension");
  if (m > 0 && ldl < (size_t)m) return ctx_fail(c, ST_ARG, "transform leading dimension too small");
  *rank = 0;
  *det = 1 % p;
  if (m == 0) return ST_OK;
  const int rmax = std::max(1, std::min(m, n));
  const size_t k_bytes = ((size_t)m * rmax * 4 + 255) & ~(size_t)255;
  const size_t sq_bytes = ((size_t)rmax * rmax * 4 + 255) & ~(size_t)255;
  void *buf = nullptr;
  int st = ctx_buffer(c, BUF_TRANSFORM, k_bytes + 2 * sq_bytes + (size_t)rmax * sizeof(int) + 256,
                      &buf);
  if (st) return st;
  uint8_t *b8 = static_cast<uint8_t *>(buf);
  uint32_t *Lk = reinterpret_cast<uint32_t *>(b8);
  uint32_t *T = reinterpret_cast<uint32_t *>(b8 + k_bytes);
  uint32_t *W = reinterpret_cast<uint32_t *>(b8 + k_bytes + sq_bytes);
  int *d_piv = reinterpret_cast<int *>(b8 + k_bytes + 2 * sq_bytes);
  std::vector<int> piv;
  if (n > 0) {
    EchelonKeep keep;
    keep.L = Lk;
    keep.ldL = (size_t)rmax;
    if ((st = zp_echelon_dev(c, m, n, p, D, ld, rank, det, &piv, &keep))) return st;
    for (const auto &sw : keep.swaps)
      if (sw.first != sw.second) P->push_back(sw);  // in the order applied
  }
  const int r = (int)*rank;
  cudaError_t e = cudaSuccess;
  if (r > 0)
    e = cudaMemcpyAsync(d_piv, piv.data(), (size_t)r * sizeof(int), cudaMemcpyHostToDevice,
                        c->stream);
  if (e != cudaSuccess) return ctx_cuda(c, e, "transform: pivot columns");
  {
    const size_t total = (size_t)m * m + 2 * (size_t)r * r;
    const int grid = (int)std::min<size_t>((total + 255) / 256, (size_t)c->num_sms * 16);
    transform_setup_kernel<<<grid, 256, 0, c->stream>>>(Lk, (size_t)rmax, D, ld, d_piv, m, r, T,
                                                        W, Lout, ldl);
    ctx_launched(c);
    if ((e = cudaGetLastError()) != cudaSuccess) return ctx_cuda(c, e, "transform: set-up");
  }
  if (r > 0) {
    size_t bad = 0;
    if ((st = zp_trsm_dev(c, false, true, r, r, p, 1u, T, (size_t)r, Lout, ldl, &bad))) return st;
    if (m > r &&
        (st = zp_gemm_dev(c, GEMM_AUTO, m - r, r, r, p, p - 1, Lk + (size_t)r * rmax, (size_t)rmax,
                          Lout, ldl, 0u, Lout + (size_t)r * ldl, ldl, nullptr)))
      return st;
    if ((st = zp_trsm_dev(c, true, false, r, r, p, 1u, W, (size_t)r, Lout, ldl, &bad))) return st;
    if ((st = zp_trsm_dev(c, true, false, r, n, p, 1u, W, (size_t)r, D, ld, &bad))) return st;
  }
  // the host vector piv must outlive the copy above
  e = cudaStreamSynchronize(c->stream);
  return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "transform");
}

}  // namespace lela
