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
// W = 64.  For a panel [c0, c0+W):
//  1. panel_kernel (one CTA) collects the "active" rows -- rows at or below
//     the current row with a nonzero in the panel; no other row can be a
//     pivot of these columns or be changed by their elimination steps, so
//     the reference's steps restricted to the panel run on the active rows
//     alone: per column, the active row with the smallest current position
//     and a nonzero entry is the pivot, the transposition (i, q) is recorded
//     (tracking where active rows move), and the active rows below are
//     eliminated inside the panel, keeping their multipliers;
//  2. the host replays the recorded transpositions on the row positions and
//     moves the affected rows (at most two per pivot) with one gather;
//  3. the panel values are written back, U12 = L11^-1 A12 is solved on CUDA
//     cores, and A22 -= L21 U12 runs on the limb-split tensor-core gemm over
//     the rows from the first row below the pivots to the last active one.
// F4 Schur complements are staircase-shaped (rows sorted by head), so few
// rows are active per panel; dense matrices make every row active and the
// scheme becomes ordinary blocked LU with LELA's pivot choice.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "context.h"
#include "echelon.h"
#include "tri.h"
#include "zp_gemm.h"

namespace lela {

constexpr int EW = 64;  // panel width

struct PanelOut {
  uint32_t t;         // pivots found in the panel
  uint32_t err;       // 1: a pivot is not invertible in Modular<uint32>
  uint32_t nact;      // active rows
  uint32_t last_pos;  // largest final position of an active non-pivot row (or 0)
  uint32_t det;       // product of the panel's pivots
  uint32_t pad[3];
  uint32_t pcol[EW];  // pivot columns (relative to c0)
  uint32_t ti[EW];    // transposition k: (ti[k], tq[k])
  uint32_t tq[EW];
  uint32_t prow[EW];  // active index of pivot k
};

__device__ __forceinline__ uint32_t sub_mod(uint32_t a, uint32_t b, uint32_t p) {
  return a >= b ? a - b : a + (p - b);
}

// Block-wide ordered compaction helper: returns this thread's exclusive
// prefix of `flag` within the block and writes the block total to *total.
__device__ __forceinline__ int block_scan_flag(int flag, int *warp_sums, int *total) {
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

__global__ void __launch_bounds__(1024)
    panel_kernel(const uint32_t *__restrict__ D, size_t ld, int i0, int m, int c0, int w,
                 Modulus mod, int *__restrict__ act_row, int *__restrict__ act_pos,
                 uint32_t *__restrict__ vals, uint32_t *__restrict__ mult, PanelOut *out) {
  __shared__ int warp_sums[32];
  __shared__ int s_total, s_nact;
  __shared__ unsigned long long s_key;
  __shared__ int s_at_i;
  __shared__ uint32_t prow_vals[EW];
  __shared__ uint32_t s_xinv;
  __shared__ int s_stop;
  const uint32_t p = (uint32_t)mod.p;

  // 1. active rows, in position order
  if (threadIdx.x == 0) s_nact = 0;
  __syncthreads();
  for (int base = i0; base < m; base += blockDim.x) {
    const int r = base + threadIdx.x;
    int flag = 0;
    if (r < m) {
      const uint32_t *row = D + (size_t)r * ld + c0;
      uint32_t any = 0;
      for (int j = 0; j < w; ++j) any |= row[j];
      flag = any != 0;
    }
    int off = block_scan_flag(flag, warp_sums, &s_total);
    if (flag) act_row[s_nact + off] = r;
    __syncthreads();
    if (threadIdx.x == 0) s_nact += s_total;
    __syncthreads();
  }
  const int nact = s_nact;
  for (int a = threadIdx.x; a < nact; a += blockDim.x) {
    const int r = act_row[a];
    act_pos[a] = r;
    const uint32_t *row = D + (size_t)r * ld + c0;
    uint32_t *v = vals + (size_t)a * EW;
    uint32_t *mu = mult + (size_t)a * EW;
    for (int j = 0; j < EW; ++j) {
      v[j] = j < w ? row[j] : 0u;
      mu[j] = 0u;
    }
  }
  if (threadIdx.x == 0) s_stop = 0;
  __syncthreads();

  // 2. the reference's steps on the panel
  int i = i0, t = 0;
  uint32_t det = 1u % p;
  for (int col = 0; col < w && i < m; ++col) {
    if (threadIdx.x == 0) {
      s_key = ~0ull;
      s_at_i = -1;
    }
    __syncthreads();
    for (int a = threadIdx.x; a < nact; a += blockDim.x) {
      const int pos = act_pos[a];
      if (pos >= i && vals[(size_t)a * EW + col] != 0u)
        atomicMin(&s_key, ((unsigned long long)(unsigned)pos << 32) | (unsigned)a);
      if (pos == i) s_at_i = a;
    }
    __syncthreads();
    const unsigned long long key = s_key;
    const int ai = s_at_i;
    __syncthreads();  // every thread has read s_key / s_at_i before they change
    if (key == ~0ull) continue;  // no pivot in this column
    const int ap = (int)(key & 0xffffffffu), q = (int)(key >> 32);
    if (threadIdx.x == 0) {
      const uint32_t x = vals[(size_t)ap * EW + col];
      const uint32_t xinv = lela_inv_u32(p, x);
      if (xinv == 0) s_stop = 1;
      s_xinv = xinv;
      det = mod_mul(det, x, mod);
      out->pcol[t] = (uint32_t)col;
      out->ti[t] = (uint32_t)i;
      out->tq[t] = (uint32_t)q;
      out->prow[t] = (uint32_t)ap;
      if (ai >= 0 && ai != ap) act_pos[ai] = q;
      act_pos[ap] = i;
    }
    for (int j = threadIdx.x; j < EW; j += blockDim.x) prow_vals[j] = vals[(size_t)ap * EW + j];
    __syncthreads();
    if (s_stop) break;
    const uint32_t xinv = s_xinv;
    // eliminate the active rows below
    for (int a = threadIdx.x; a < nact; a += blockDim.x) {
      if (act_pos[a] <= i) continue;
      uint32_t *v = vals + (size_t)a * EW;
      const uint32_t av = v[col];
      if (av == 0u) continue;
      const uint32_t f = mod_mul(av, xinv, mod);
      mult[(size_t)a * EW + t] = f;
      v[col] = 0u;
      for (int j = col + 1; j < w; ++j) {
        const uint32_t pj = prow_vals[j];
        if (pj) v[j] = sub_mod(v[j], mod_mul(f, pj, mod), p);
      }
    }
    __syncthreads();
    ++i;
    ++t;
  }
  // 3. results
  if (threadIdx.x == 0) {
    s_key = 0;
  }
  __syncthreads();
  for (int a = threadIdx.x; a < nact; a += blockDim.x)
    if (act_pos[a] >= i) atomicMax(&s_key, (unsigned long long)(unsigned)act_pos[a]);
  __syncthreads();
  if (threadIdx.x == 0) {
    out->t = (uint32_t)t;
    out->err = (uint32_t)s_stop;
    out->nact = (uint32_t)nact;
    out->last_pos = (uint32_t)s_key;
    out->det = det;
  }
}

// Row permutation through a temporary: tmp[k] = D[src[k]], then
// D[dst[k]] = tmp[k] (full rows).
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

// After the permutation: panel values of the active rows go back to D at
// their final positions; L11 (t x t, unit lower, row stride EW) and L21
// (rows r0..r1 by position, t columns, zero for rows without multipliers)
// are laid out for the solve and the gemm.
__global__ void panel_writeback_kernel(uint32_t *__restrict__ D, size_t ld, int c0, int w,
                                       int nact, const int *__restrict__ act_pos,
                                       const uint32_t *__restrict__ vals,
                                       const uint32_t *__restrict__ mult, int i0, int t,
                                       uint32_t *__restrict__ L11, uint32_t *__restrict__ L21,
                                       int r0) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nact; a += gridDim.x * blockDim.x) {
    const int pos = act_pos[a];
    uint32_t *row = D + (size_t)pos * ld + c0;
    const uint32_t *v = vals + (size_t)a * EW;
    for (int j = 0; j < w; ++j) row[j] = v[j];
    const uint32_t *mu = mult + (size_t)a * EW;
    if (pos < i0 + t) {
      const int k = pos - i0;  // pivot index
      for (int j = 0; j < EW; ++j) L11[k * EW + j] = (j < k) ? mu[j] : (j == k ? 1u : 0u);
    } else if (pos >= r0) {
      uint32_t *l = L21 + (size_t)(pos - r0) * t;
      for (int j = 0; j < t; ++j) l[j] = mu[j];
    }
  }
}

// Speculative fast path for dense panels.  LU without pivoting of the
// w x w block D[i0 .. i0+w, c0 .. c0+w) (one CTA, shared memory).  When all
// w pivots are nonzero and invertible the reference's rule picks exactly
// these rows, in order, with no transposition: at step k row i0+k has a
// nonzero entry in column c0+k and is the first row at or below i0+k.
// out[0] = number of leading nonzero invertible pivots; blk = L\U (row
// stride EW); pinv = inverted pivots; out[1] = product of the pivots.
__global__ void __launch_bounds__(1024)
    spec_lu_kernel(const uint32_t *__restrict__ D, size_t ld, int i0, int c0, int w, Modulus mod,
                   uint32_t *__restrict__ blk, uint32_t *__restrict__ pinv, uint32_t *out) {
  __shared__ uint32_t S[EW][EW + 1];
  __shared__ uint32_t s_inv;
  __shared__ int s_stop;
  const uint32_t p = (uint32_t)mod.p;
  for (int e = threadIdx.x; e < EW * EW; e += blockDim.x) {
    int r = e / EW, j = e % EW;
    S[r][j] = (r < w && j < w) ? D[(size_t)(i0 + r) * ld + c0 + j] : 0u;
  }
  if (threadIdx.x == 0) s_stop = 0;
  __syncthreads();
  int t = w;
  uint32_t det = 1u % p;
  for (int k = 0; k < w; ++k) {
    if (threadIdx.x == 0) {
      const uint32_t piv = S[k][k];
      const uint32_t inv = piv ? lela_inv_u32(p, piv) : 0u;
      if (inv == 0u) s_stop = 1;
      s_inv = inv;
      pinv[k] = inv;
      det = mod_mul(det, piv, mod);
    }
    __syncthreads();
    if (s_stop) {
      t = k;
      break;
    }
    const uint32_t inv = s_inv;
    const int rem = w - k - 1;
    for (int e = threadIdx.x; e < rem; e += blockDim.x) S[k + 1 + e][k] = mod_mul(S[k + 1 + e][k], inv, mod);
    __syncthreads();
    for (int e = threadIdx.x; e < rem * rem; e += blockDim.x) {
      const int j = k + 1 + e / rem, q = k + 1 + e % rem;
      const uint32_t l = S[j][k];
      if (l) S[j][q] = sub_mod(S[j][q], mod_mul(l, S[k][q], mod), p);
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < EW * EW; e += blockDim.x) blk[e] = S[e / EW][e % EW];
  if (threadIdx.x == 0) {
    out[0] = (uint32_t)t;
    out[1] = det;
  }
}

// Rows r0..m-1: L[r - r0][k] = (D[r][c..c+t) * U11^-1)_k, and the eliminated
// block D[r][c..c+t) becomes zero.  One thread per row.
__global__ void __launch_bounds__(128)
    spec_right_solve_kernel(uint32_t *__restrict__ D, size_t ld, int r0, int m, int c, int t,
                            const uint32_t *__restrict__ blk, const uint32_t *__restrict__ pinv,
                            uint32_t *__restrict__ L, Modulus mod, uint32_t two64) {
  __shared__ uint32_t U[EW][EW + 1];
  __shared__ uint32_t sI[EW];
  for (int e = threadIdx.x; e < EW * EW; e += blockDim.x) {
    const int r = e / EW, j = e % EW;
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
#pragma unroll
  for (int k = 0; k < EW; ++k) {
    uint64_t s = 0;
#pragma unroll
    for (int j = 0; j < k; ++j) {
      const uint64_t q = (uint64_t)x[j] * U[j][k];
      s += q;
      if (s < q) s += two64;
    }
    x[k] = mod_mul(sub_mod(x[k], mod_reduce(s, mod), p), sI[k], mod);
  }
  uint32_t *lrow = L + (size_t)(r - r0) * t;
#pragma unroll
  for (int k = 0; k < EW; ++k)
    if (k < t) {
      lrow[k] = x[k];
      row[k] = 0u;
    }
}

// Pivot rows i..i+t-1, panel columns c..c+t-1 <- U11 (zeros below the
// diagonal); L11 (unit lower, row stride EW) for the U12 solve.
__global__ void spec_write_kernel(uint32_t *__restrict__ D, size_t ld, int i, int c, int t,
                                  const uint32_t *__restrict__ blk, uint32_t *__restrict__ L11) {
  for (int e = threadIdx.x; e < t * EW; e += blockDim.x) {
    const int r = e / EW, j = e % EW;
    if (j < t) D[(size_t)(i + r) * ld + c + j] = (j >= r) ? blk[r * EW + j] : 0u;
    L11[r * EW + j] = (j < r) ? blk[r * EW + j] : (j == r ? 1u : 0u);
  }
}

__global__ void zero_kernel(uint32_t *x, size_t n) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x)
    x[k] = 0u;
}

static int sync_read(Ctx *c, const void *dev, void *host, size_t bytes, const char *what) {
  cudaError_t e = cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, c->stream);
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

  // device scratch
  const size_t out_bytes = (sizeof(PanelOut) + 255) & ~(size_t)255;
  const size_t i_bytes = (((size_t)2 * m + 4 * EW) * sizeof(int) + 255) & ~(size_t)255;
  const size_t v_bytes = (size_t)m * EW * 4;
  const size_t l11_bytes = EW * EW * 4;
  const size_t tmp_bytes = (size_t)2 * EW * n * 4;
  void *base = nullptr;
  const size_t spec_bytes = (size_t)(EW * EW + EW + 4) * 4;
  int st = ctx_buffer(c, BUF_ECH_0,
                      out_bytes + i_bytes + 3 * v_bytes + l11_bytes + tmp_bytes + spec_bytes + 1024,
                      &base);
  if (st) return st;
  uint8_t *b8 = static_cast<uint8_t *>(base);
  PanelOut *d_out = reinterpret_cast<PanelOut *>(b8);
  int *d_act_row = reinterpret_cast<int *>(b8 + out_bytes);
  int *d_act_pos = d_act_row + m;
  int *d_perm = d_act_pos + m;  // 4*EW ints: src list, dst list
  uint32_t *d_vals = reinterpret_cast<uint32_t *>(b8 + out_bytes + i_bytes);
  uint32_t *d_mult = d_vals + (size_t)m * EW;
  uint32_t *d_L21 = d_mult + (size_t)m * EW;
  uint32_t *d_L11 = d_L21 + (size_t)m * EW;
  uint32_t *d_tmp = d_L11 + EW * EW;
  uint32_t *d_blk = d_tmp + (size_t)2 * EW * n;
  uint32_t *d_pinv = d_blk + EW * EW;
  uint32_t *d_spec = d_pinv + EW;
  void *gws = nullptr;
  st = ctx_workspace(c, zp_gemm_workspace_bytes(p, m, n, EW), &gws);
  if (st) return st;
  const uint32_t t64 = two64_mod(p);

  PanelOut h;
  std::vector<int> at, src, dst;
  int i = 0;
  int backoff = 1, skip = 0;  // speculation is retried less often after failures
  for (int c0 = 0; c0 < n && i < m; c0 += EW) {
    const int w = std::min(EW, n - c0);
    if (skip > 0) {
      --skip;
    } else if (m - i >= w) {
      // speculative dense panel: rows i .. i+w-1 are the pivots, in order
      int ps = prof_begin(c, "ech_spec_lu");
      spec_lu_kernel<<<1, 1024, 0, c->stream>>>(D, ld, i, c0, w, mod, d_blk, d_pinv, d_spec);
      prof_end(c, ps);
      ctx_launched(c);
      uint32_t hs[2];
      if ((st = sync_read(c, d_spec, hs, sizeof hs, "echelon: speculation"))) return st;
      if ((int)hs[0] == w) {
        backoff = 1;
        spec_write_kernel<<<1, 1024, 0, c->stream>>>(D, ld, i, c0, w, d_blk, d_L11);
        ctx_launched(c);
        const int r0 = i + w, below = m - r0, rest = n - (c0 + w);
        if (below > 0) {
          ps = prof_begin(c, "ech_spec_solve");
          spec_right_solve_kernel<<<(below + 127) / 128, 128, 0, c->stream>>>(
              D, ld, r0, m, c0, w, d_blk, d_pinv, d_L21, mod, t64);
          prof_end(c, ps);
          ctx_launched(c);
        }
        if (rest > 0) {
          uint32_t *U12 = D + (size_t)i * ld + c0 + w;
          if ((st = tri_left_block(c, false, w, d_L11, EW, nullptr, U12, ld, rest, p, 1)))
            return st;
          if (below > 0) {
            ps = prof_begin(c, "ech_update");
            st = zp_gemm_dev(c, GEMM_AUTO, below, rest, w, p, p - 1, d_L21, (size_t)w, U12, ld, 1,
                             D + (size_t)r0 * ld + c0 + w, ld, static_cast<uint8_t *>(gws));
            prof_end(c, ps);
            if (st) return st;
          }
        }
        det = (det * hs[1]) % p;
        if (pivot_cols)
          for (int k = 0; k < w; ++k) pivot_cols->push_back(c0 + k);
        rank += w;
        i += w;
        continue;
      }
      backoff = std::min(backoff * 2, 32);
      skip = backoff - 1;
    }
    int pi = prof_begin(c, "ech_panel");
    panel_kernel<<<1, 1024, 0, c->stream>>>(D, ld, i, m, c0, w, mod, d_act_row, d_act_pos, d_vals,
                                            d_mult, d_out);
    prof_end(c, pi);
    ctx_launched(c);
    if ((st = sync_read(c, d_out, &h, sizeof h, "echelon: panel"))) return st;
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
      std::vector<int> both(src);
      both.insert(both.end(), dst.begin(), dst.end());
      cudaError_t e = cudaMemcpyAsync(d_perm, both.data(), both.size() * sizeof(int),
                                      cudaMemcpyHostToDevice, c->stream);
      if (e != cudaSuccess) return ctx_cuda(c, e, "echelon: permutation");
      dim3 grid((n + 255) / 256, cnt);
      gather_rows_kernel<<<grid, 256, 0, c->stream>>>(D, ld, n, d_perm, cnt, d_tmp);
      scatter_rows_kernel<<<grid, 256, 0, c->stream>>>(D, ld, n, d_perm + cnt, cnt, d_tmp);
      ctx_launched(c, 2);
    }
    // write back, L11 / L21
    const int r0 = i + t;
    const int r1 = (h.last_pos >= (uint32_t)r0) ? (int)h.last_pos : r0 - 1;
    const int below = r1 - r0 + 1;
    if (below > 0) {
      const size_t words = (size_t)below * t;
      zero_kernel<<<(int)std::min<size_t>((words + 255) / 256, (size_t)c->num_sms * 8), 256, 0,
                    c->stream>>>(d_L21, words);
      ctx_launched(c);
    }
    const int nact = (int)h.nact;
    panel_writeback_kernel<<<std::max(1, std::min((nact + 127) / 128, c->num_sms * 4)), 128, 0,
                             c->stream>>>(D, ld, c0, w, nact, d_act_pos, d_vals, d_mult, i, t,
                                          d_L11, d_L21, r0);
    ctx_launched(c);
    const int rest = n - (c0 + w);
    if (rest > 0) {
      uint32_t *U12 = D + (size_t)i * ld + c0 + w;
      if ((st = tri_left_block(c, false, t, d_L11, EW, nullptr, U12, ld, rest, p, 1))) return st;
      if (below > 0) {
        pi = prof_begin(c, "ech_update");
        st = zp_gemm_dev(c, GEMM_AUTO, below, rest, t, p, p - 1, d_L21, (size_t)t, U12, ld, 1,
                         D + (size_t)r0 * ld + c0 + w, ld, static_cast<uint8_t *>(gws));
        prof_end(c, pi);
        if (st) return st;
      }
    }
    det = (det * h.det) % p;
    if (pivot_cols)
      for (int k = 0; k < t; ++k) pivot_cols->push_back(c0 + (int)h.pcol[k]);
    rank += t;
    i += t;
  }
  *rank_out = rank;
  *det_out = (uint32_t)det;
  return ST_OK;
}

}  // namespace lela
