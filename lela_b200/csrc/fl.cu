// lela_b200/csrc/fl.cu -- Faugere-Lachartre echelon form of an F4 matrix
// over Z/p on the GPU.
//
// Reference: FaugereLachartre::echelonize (lela/algorithms/
// faugere-lachartre.tcc:735-917).  Steps and their GPU form:
//
//  setup_splicer (:47-146)  The head of a sparse row is its first stored
//      entry (BLAS1::head on a sparse vector, lela/blas/level1-generic.tcc:
//      452-460).  Walking the rows: a head larger than the last pivot column
//      makes a pivot row (det *= head value), an equal head a non-pivot row,
//      a smaller head throws WrongMatrixForm(row), and the first empty row
//      ends the walk (every later row is a non-pivot row).  This O(m) walk
//      runs on the host over the row heads.
//  split (MatrixGrid1, :766)  One scatter kernel places every stored entry
//      into dense A (pivot rows x pivot columns, upper triangular), B, C, D.
//  B <- A^-1 B (:791)  Dense trsm (tri.cu): tensor-core updates, inverse
//      leaves; the updates skip A's empty tiles (its nonzeros lie in a band
//      above the diagonal), using the per-row column ranges the split
//      records.  A singular diagonal makes the reference return early
//      (:792-799); reported here as LELA_CUDA_DIAG_NOT_INVERTIBLE with rank
//      and det as the reference leaves them.
//  D <- D - C B (:805)  Limb-split INT8 tensor-core gemm (zp_gemm.cu),
//      each 128-row tile over the K blocks its rows of C can touch.
//  echelon(D) (:822, then setup_splicer on it, :833)  echelon.cu; its pivots
//      multiply det and add to the rank.
//  reduced (:851-902)  D1 | D2 split by D's pivot columns, D2 <- D1^-1 D2
//      (trsm), B2 <- B2 - B1 D2 (gemm), then the rows are assembled in
//      pivot-column order (the reduced row-echelon form is unique).
//  non-reduced / only_D (:867-874, :906-911)  as the reference's
//      MatrixGrid4/5 write them (see oracle/lela_oracle.c for the exact rows).
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "context.h"
#include "echelon.h"
#include "fl.h"
#include "tri.h"
#include "zp_gemm.h"

namespace lela {

// Row r of X: pos[r] = index of r among pivot rows (>= 0) or -(1 + index
// among non-pivot rows); column c: cpos likewise.  Also, per row of A (a
// pivot row) and of C (a non-pivot row), the range [first, last + 1) of its
// pivot columns holding entries ((0, 0) when none): the products with A
// and C skip the K blocks outside them.
__global__ void fl_split_kernel(const uint64_t *__restrict__ rowptr,
                                const uint32_t *__restrict__ colidx,
                                const uint32_t *__restrict__ vals, int m,
                                const int *__restrict__ rpos, const int *__restrict__ cpos,
                                uint32_t *A, size_t npiv, uint32_t *B, size_t nres, uint32_t *C,
                                uint32_t *D, int2 *krA, int2 *krC) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int r = warp; r < m; r += nwarps) {
    const int rp = rpos[r];
    int lo = 0x7fffffff, hi = -1;
    for (uint64_t e = rowptr[r] + lane; e < rowptr[r + 1]; e += 32) {
      const int cp = cpos[colidx[e]];
      const uint32_t v = vals[e];
      if (cp >= 0) {
        lo = min(lo, cp);
        hi = max(hi, cp);
      }
      if (rp >= 0) {
        if (cp >= 0) A[(size_t)rp * npiv + cp] = v;
        else B[(size_t)rp * nres + (-1 - cp)] = v;
      } else {
        if (cp >= 0) C[(size_t)(-1 - rp) * npiv + cp] = v;
        else D[(size_t)(-1 - rp) * nres + (-1 - cp)] = v;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if (lane == 0) {
      const int2 v = hi >= 0 ? make_int2(lo, hi + 1) : make_int2(0, 0);
      if (rp >= 0) krA[rp] = v;
      else krC[-1 - rp] = v;
    }
  }
}

// Gather columns: out[r][j] = in[r][cols[j]] for r < rows, j < ncols.
__global__ void gather_cols_kernel(const uint32_t *__restrict__ in, size_t ldi, int rows,
                                   const int *__restrict__ cols, int ncols,
                                   uint32_t *__restrict__ out, size_t ldo) {
  const size_t total = (size_t)rows * ncols;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    size_t r = idx / ncols, j = idx % ncols;
    out[r * ldo + j] = in[r * ldi + cols[j]];
  }
}

// Assemble output rows, one block per row.  For output row o: kind[o] =
// 0 (zero row), 1 (values from M1 row src_row[o]), 2 (values from M2 row
// src_row[o]), 4 (no values); unit_col[o] = column that gets a 1 (or -1).
// Values of a row are scattered to columns vcols[0..nv).
__global__ void fl_assemble_kernel(uint32_t *__restrict__ R, size_t ldr, int rows, int n,
                                   const int *__restrict__ kind, const int *__restrict__ src_row,
                                   const int *__restrict__ unit_col,
                                   const uint32_t *__restrict__ M1, size_t ld1,
                                   const uint32_t *__restrict__ M2, size_t ld2,
                                   const int *__restrict__ vcols, int nv) {
  for (int o = blockIdx.x; o < rows; o += gridDim.x) {
    uint32_t *out = R + (size_t)o * ldr;
    const int k = kind[o];
    for (int j = threadIdx.x; j < n; j += blockDim.x) out[j] = 0u;
    __syncthreads();
    if (k == 1 || k == 2) {
      const uint32_t *src = (k == 1 ? M1 + (size_t)src_row[o] * ld1 : M2 + (size_t)src_row[o] * ld2);
      for (int j = threadIdx.x; j < nv; j += blockDim.x) out[vcols[j]] = src[j];
    }
    if (k != 0 && threadIdx.x == 0 && unit_col[o] >= 0) out[unit_col[o]] = 1u;
    __syncthreads();
  }
}

// CSR form of the rows fl_assemble_kernel writes (same plan), one warp per
// row.  Count pass: cnt[o] = nonzero values of the row's source plus its
// unit entry.  Fill pass (row pointers = exclusive sums of the counts): the
// nonzero values in column order, the unit entry in its sorted place (the
// value columns vcols are increasing and never hold the unit column).
__global__ void fl_csr_count_kernel(int rows, const int *__restrict__ kind,
                                    const int *__restrict__ src_row,
                                    const int *__restrict__ unit_col,
                                    const uint32_t *__restrict__ M1, size_t ld1,
                                    const uint32_t *__restrict__ M2, size_t ld2, int nv,
                                    uint64_t *__restrict__ cnt) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int o = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; o < rows; o += warps) {
    const int k = kind[o];
    int c = 0;
    if (k == 1 || k == 2) {
      const uint32_t *src = k == 1 ? M1 + (size_t)src_row[o] * ld1 : M2 + (size_t)src_row[o] * ld2;
      for (int j = lane; j < nv; j += 32) c += src[j] != 0u;
      c = __reduce_add_sync(0xffffffffu, c);
    }
    if (lane == 0) cnt[o] = (uint64_t)c + ((k != 0 && unit_col[o] >= 0) ? 1u : 0u);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) cnt[rows] = 0;
}

__global__ void fl_csr_fill_kernel(int rows, const int *__restrict__ kind,
                                   const int *__restrict__ src_row,
                                   const int *__restrict__ unit_col,
                                   const uint32_t *__restrict__ M1, size_t ld1,
                                   const uint32_t *__restrict__ M2, size_t ld2,
                                   const int *__restrict__ vcols, int nv,
                                   const uint64_t *__restrict__ rowptr,
                                   uint32_t *__restrict__ colidx, uint32_t *__restrict__ vals) {
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int o = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; o < rows; o += warps) {
    const int k = kind[o];
    if (k == 0) continue;
    const uint64_t base = rowptr[o];
    const int u = unit_col[o];
    int before = 0;  // nonzero values left of the unit column
    if (k == 1 || k == 2) {
      const uint32_t *src = k == 1 ? M1 + (size_t)src_row[o] * ld1 : M2 + (size_t)src_row[o] * ld2;
      if (u >= 0) {
        for (int j = lane; j < nv; j += 32) before += (src[j] != 0u && vcols[j] < u);
        before = __reduce_add_sync(0xffffffffu, before);
      }
      uint64_t run = 0;
      for (int j0 = 0; j0 < nv; j0 += 32) {
        const int j = j0 + lane;
        const uint32_t v = j < nv ? src[j] : 0u;
        const unsigned bal = __ballot_sync(0xffffffffu, v != 0u);
        if (v != 0u) {
          const int col = vcols[j];
          const uint64_t at = base + run + __popc(bal & below) + ((u >= 0 && col > u) ? 1 : 0);
          colidx[at] = (uint32_t)col;
          vals[at] = v;
        }
        run += __popc(bal);
      }
    }
    if (lane == 0 && u >= 0) {
      colidx[base + before] = (uint32_t)u;
      vals[base + before] = 1u;
    }
  }
}

__global__ void fl_heads_kernel(int m, const uint64_t *__restrict__ rowptr,
                                const uint32_t *__restrict__ colidx,
                                const uint32_t *__restrict__ vals, uint32_t *heads,
                                uint32_t *headvals) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < m; r += gridDim.x * blockDim.x) {
    const uint64_t e = rowptr[r];
    const bool empty = rowptr[r + 1] == e;
    heads[r] = empty ? 0u : colidx[e];
    headvals[r] = empty ? 0u : vals[e];
  }
}

int fl_row_heads_dev(Ctx *c, int m, const uint64_t *d_rowptr, const uint32_t *d_colidx,
                     const uint32_t *d_vals, uint32_t *d_heads, uint32_t *d_headvals) {
  if (m <= 0) return ST_OK;
  int grid = std::min((m + 255) / 256, c->num_sms * 8);
  fl_heads_kernel<<<grid, 256, 0, c->stream>>>(m, d_rowptr, d_colidx, d_vals, d_heads, d_headvals);
  ctx_launched(c);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "fl heads launch");
}

// The output rows of an assembly plan (kind, src_row, unit_col, vcols as
// for fl_assemble_kernel, at d_plan) as CSR in the handle's buffers:
// counts, exclusive scan (CUB), one synchronisation to size the entries,
// fill.
static int fl_assemble_csr(Ctx *c, int rows, const int *d_plan, const uint32_t *M1, size_t ld1,
                           const uint32_t *M2, size_t ld2, int nv, FlCsr *csr) {
  size_t temp = 0;
  cudaError_t e = cub::DeviceScan::ExclusiveSum(nullptr, temp, (const uint64_t *)nullptr,
                                                (uint64_t *)nullptr, rows + 1, c->stream);
  if (e != cudaSuccess) return ctx_cuda(c, e, "fl: csr scan size");
  const size_t cnt_bytes = ((size_t)(rows + 1) * 8 + 255) & ~(size_t)255;
  void *vP = nullptr;
  int st = ctx_buffer(c, BUF_FL_CSR_P, 2 * cnt_bytes + temp + 256, &vP);
  if (st) return st;
  uint8_t *b = static_cast<uint8_t *>(vP);
  uint64_t *cnt = reinterpret_cast<uint64_t *>(b);
  uint64_t *rowptr = reinterpret_cast<uint64_t *>(b + cnt_bytes);
  void *d_temp = b + 2 * cnt_bytes;
  const int *kind = d_plan, *srow = d_plan + rows, *ucol = d_plan + 2 * rows, *vcols = d_plan + 3 * rows;
  const int grid = std::max(1, std::min((rows + 7) / 8, c->num_sms * 16));
  int pi = prof_begin(c, "fl_assemble");
  fl_csr_count_kernel<<<grid, 256, 0, c->stream>>>(rows, kind, srow, ucol, M1, ld1, M2, ld2, nv, cnt);
  ctx_launched(c);
  e = cub::DeviceScan::ExclusiveSum(d_temp, temp, cnt, rowptr, rows + 1, c->stream);
  if (e != cudaSuccess) return ctx_cuda(c, e, "fl: csr scan");
  uint64_t nnz = 0;
  e = cudaMemcpyAsync(&nnz, rowptr + rows, 8, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return ctx_cuda(c, e, "fl: csr size");
  void *vV = nullptr;
  const size_t col_bytes = ((size_t)nnz * 4 + 255) & ~(size_t)255;
  if ((st = ctx_buffer(c, BUF_FL_CSR_V, col_bytes + (size_t)nnz * 4 + 256, &vV))) return st;
  uint32_t *colidx = static_cast<uint32_t *>(vV);
  uint32_t *vals = reinterpret_cast<uint32_t *>(static_cast<uint8_t *>(vV) + col_bytes);
  fl_csr_fill_kernel<<<grid, 256, 0, c->stream>>>(rows, kind, srow, ucol, M1, ld1, M2, ld2, vcols,
                                                  nv, rowptr, colidx, vals);
  ctx_launched(c);
  prof_end(c, pi);
  e = cudaGetLastError();
  if (e != cudaSuccess) return ctx_cuda(c, e, "fl: csr fill");
  csr->rowptr = rowptr;
  csr->colidx = colidx;
  csr->vals = vals;
  csr->nnz = (size_t)nnz;
  c->fl_csr_nnz = (size_t)nnz;
  return ST_OK;
}

static int upload(Ctx *c, void *dst, const void *src, size_t bytes, const char *what) {
  if (!bytes) return ST_OK;
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream);
  return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, what);
}

int zp_fl_echelonize_dev(Ctx *c, int m, int n, uint32_t p, const uint64_t *d_rowptr,
                         const uint32_t *d_colidx, const uint32_t *d_vals,
                         const uint64_t *h_rowptr, const uint32_t *h_heads,
                         const uint32_t *h_headvals, bool reduced, bool only_D, uint32_t *R,
                         size_t ldr, FlResult *res, FlCsr *csr) {
  c->fl_csr_nnz = (size_t)-1;  // a kept CSR result is replaced by this call's
  res->rank = 0;
  res->det = 1 % p;
  res->out_rows = 0;
  res->bad_row = 0;
  if (p < 2) return ctx_fail(c, ST_ARG, "modulus must be at least 2");
  int st;
  uint64_t det = 1 % p;

  // ---- setup_splicer on the row heads
  std::vector<int> rpos(m), cpos(n, 0);
  std::vector<char> is_piv_col(n, 0);
  std::vector<int> piv_rows, res_rows, piv_cols, res_cols;
  long last_col = -1;
  bool walking = true;
  for (int r = 0; r < m; ++r) {
    bool piv = false;
    if (walking && h_rowptr[r] == h_rowptr[r + 1]) walking = false;  // first empty row
    if (walking) {
      long col = h_heads[r];
      if (col < last_col) {
        res->bad_row = (size_t)r;
        return ctx_fail(c, ST_WRONG_FORM, "Bad input-matrix for Faugere-Lachartre");
      }
      if (col > last_col) {
        piv = true;
        is_piv_col[col] = 1;
        last_col = col;
      }
      det = (det * h_headvals[r]) % p;
    }
    if (piv) {
      rpos[r] = (int)piv_rows.size();
      piv_rows.push_back(r);
    } else {
      rpos[r] = -1 - (int)res_rows.size();
      res_rows.push_back(r);
    }
  }
  const int npiv = (int)piv_rows.size();
  for (int col = 0; col < n; ++col) {
    if (is_piv_col[col]) {
      cpos[col] = (int)piv_cols.size();
      piv_cols.push_back(col);
    } else {
      cpos[col] = -1 - (int)res_cols.size();
      res_cols.push_back(col);
    }
  }
  const int mres = (int)res_rows.size(), nres = (int)res_cols.size();
  res->rank = (size_t)npiv;
  res->det = (uint32_t)det;

  // ---- device blocks
  void *vA, *vB, *vC, *vD, *vI;
  const size_t szA = (size_t)npiv * npiv, szB = (size_t)npiv * nres, szC = (size_t)mres * npiv,
               szD = (size_t)mres * nres;
  if ((st = ctx_buffer(c, BUF_FL_A, szA * 4 + 16, &vA))) return st;
  if ((st = ctx_buffer(c, BUF_FL_B, szB * 4 + 16, &vB))) return st;
  if ((st = ctx_buffer(c, BUF_FL_C, szC * 4 + 16, &vC))) return st;
  if ((st = ctx_buffer(c, BUF_FL_D, szD * 4 + 16, &vD))) return st;
  const size_t idx_words = (size_t)m + n + 4 * ((size_t)m + n) + 64;
  if ((st = ctx_buffer(c, BUF_FL_IDX, idx_words * sizeof(int), &vI))) return st;
  uint32_t *A = (uint32_t *)vA, *B = (uint32_t *)vB, *C = (uint32_t *)vC, *D = (uint32_t *)vD;
  int *d_rpos = (int *)vI, *d_cpos = d_rpos + m, *d_aux = d_cpos + n;
  void *vK = nullptr;
  if ((st = ctx_buffer(c, BUF_FL_KR, ((size_t)npiv + mres + 1) * sizeof(int2), &vK))) return st;
  int2 *krA = static_cast<int2 *>(vK), *krC = krA + npiv;
  cudaMemsetAsync(A, 0, szA * 4, c->stream);
  cudaMemsetAsync(B, 0, szB * 4, c->stream);
  cudaMemsetAsync(C, 0, szC * 4, c->stream);
  cudaMemsetAsync(D, 0, szD * 4, c->stream);
  if ((st = upload(c, d_rpos, rpos.data(), (size_t)m * sizeof(int), "fl: rows"))) return st;
  if ((st = upload(c, d_cpos, cpos.data(), (size_t)n * sizeof(int), "fl: cols"))) return st;
  if (m > 0) {
    int grid = std::min((m * 32 + 255) / 256, c->num_sms * 16);
    int pi = prof_begin(c, "fl_split");
    fl_split_kernel<<<grid, 256, 0, c->stream>>>(d_rowptr, d_colidx, d_vals, m, d_rpos, d_cpos, A,
                                                 npiv, B, nres, C, D, krA, krC);
    prof_end(c, pi);
    ctx_launched(c);
  }

  // ---- B <- A^-1 B
  size_t bad = 0;
  int ph = prof_begin(c, "fl_phase_trsm");
  if (npiv > 0) {
    st = zp_trsm_dev(c, true, false, npiv, nres, p, 1, A, npiv, B, nres, &bad, true, krA);
    if (st == ST_DIAG) {
      res->bad_row = bad;
      return st;  // the reference returns early (rank, det as set so far)
    }
    if (st) return st;
  }
  prof_end(c, ph);
  // ---- D <- D - C B
  ph = prof_begin(c, "fl_phase_schur");
  if (mres > 0 && nres > 0 && npiv > 0)
    if ((st = zp_gemm_dev(c, GEMM_AUTO, mres, nres, npiv, p, p - 1, C, npiv, B, nres, 1, D, nres,
                          nullptr, krC, 0)))
      return st;
  prof_end(c, ph);
  // ---- echelon form of D
  size_t rd = 0;
  uint32_t detD = 1 % p;
  std::vector<int> dpiv;
  ph = prof_begin(c, "fl_phase_echelon");
  if ((st = zp_echelon_dev(c, mres, nres, p, D, nres, &rd, &detD, &dpiv))) return st;
  prof_end(c, ph);
  ph = prof_begin(c, "fl_phase_reduce");
  det = (det * detD) % p;
  res->rank = (size_t)npiv + rd;
  res->det = (uint32_t)det;

  // ---- output assembly plans (host), then one assembly kernel
  std::vector<char> is_dpiv(nres, 0);
  for (int k : dpiv) is_dpiv[k] = 1;
  std::vector<int> rem;  // non-pivot columns of D (indices into res cols)
  for (int j = 0; j < nres; ++j)
    if (!is_dpiv[j]) rem.push_back(j);
  const int nrem = (int)rem.size();
  const int rdi = (int)rd;

  int out_rows = only_D ? rdi : m;
  std::vector<int> kind(std::max(out_rows, 1), 0), srow(std::max(out_rows, 1), 0),
      ucol(std::max(out_rows, 1), -1), vcols;
  const uint32_t *M1 = nullptr, *M2 = nullptr;
  size_t ld1 = 1, ld2 = 1;

  void *vT = nullptr;
  if (reduced) {
    // D1 | D2 split, D2 <- D1^-1 D2
    const size_t szD1 = (size_t)rdi * rdi, szD2 = (size_t)rdi * nrem;
    const size_t szB1 = only_D ? 0 : (size_t)npiv * rdi, szB2 = only_D ? 0 : (size_t)npiv * nrem;
    if ((st = ctx_buffer(c, BUF_FL_T, (szD1 + szD2 + szB1 + szB2) * 4 + 64, &vT))) return st;
    uint32_t *D1 = (uint32_t *)vT, *D2 = D1 + szD1, *B1 = D2 + szD2, *B2 = B1 + szB1;
    std::vector<int> cols_all(dpiv);
    cols_all.insert(cols_all.end(), rem.begin(), rem.end());
    int *d_cols = d_aux;
    if ((st = upload(c, d_cols, cols_all.data(), cols_all.size() * sizeof(int), "fl: columns")))
      return st;
    auto gather = [&](const uint32_t *in, size_t ldi, int rows, const int *cols, int ncols,
                      uint32_t *out, size_t ldo) {
      if (!rows || !ncols) return;
      const size_t total = (size_t)rows * ncols;
      int grid = (int)std::min<size_t>((total + 255) / 256, (size_t)c->num_sms * 16);
      gather_cols_kernel<<<grid, 256, 0, c->stream>>>(in, ldi, rows, cols, ncols, out, ldo);
      ctx_launched(c);
    };
    gather(D, nres, rdi, d_cols, rdi, D1, (size_t)std::max(rdi, 1));
    gather(D, nres, rdi, d_cols + rdi, nrem, D2, (size_t)std::max(nrem, 1));
    if (rdi > 0 && nrem > 0) {
      st = zp_trsm_dev(c, true, false, rdi, nrem, p, 1, D1, rdi, D2, nrem, &bad);
      if (st) return st;
    }
    if (!only_D) {
      gather(B, nres, npiv, d_cols, rdi, B1, (size_t)std::max(rdi, 1));
      gather(B, nres, npiv, d_cols + rdi, nrem, B2, (size_t)std::max(nrem, 1));
      if (npiv > 0 && nrem > 0 && rdi > 0)
        if ((st = zp_gemm_dev(c, GEMM_AUTO, npiv, nrem, rdi, p, p - 1, B1, rdi, D2, nrem, 1, B2,
                              nrem, nullptr)))
          return st;
    }
    // value columns: the non-pivot columns of D, in original numbering
    for (int j = 0; j < nrem; ++j) vcols.push_back(res_cols[rem[j]]);
    M1 = B2;
    ld1 = (size_t)std::max(nrem, 1);
    M2 = D2;
    ld2 = (size_t)std::max(nrem, 1);
    if (only_D) {
      for (int k = 0; k < rdi; ++k) {
        kind[k] = 2;
        srow[k] = k;
        ucol[k] = res_cols[dpiv[k]];
      }
    } else {
      int xi = 0, di = 0, o = 0;
      while (xi < npiv || di < rdi) {
        long xc = xi < npiv ? piv_cols[xi] : (long)1 << 40;
        long dc = di < rdi ? res_cols[dpiv[di]] : (long)1 << 40;
        if (xc < dc) {
          kind[o] = 1; srow[o] = xi; ucol[o] = (int)xc; ++xi;
        } else {
          kind[o] = 2; srow[o] = di; ucol[o] = (int)dc; ++di;
        }
        ++o;
      }
    }
  } else {
    // non-reduced: X pivot rows = e_piv + (A^-1 B) on the non-pivot
    // columns; D rows = echelon(D) on the non-pivot columns
    for (int j = 0; j < nres; ++j) vcols.push_back(res_cols[j]);
    M1 = B;
    ld1 = (size_t)std::max(nres, 1);
    M2 = D;
    ld2 = (size_t)std::max(nres, 1);
    if (only_D) {
      // The reference's MatrixGrid4 is handed D in its D2 slot while the
      // splicer carries only source-0/1 column blocks: no entry of D is
      // written and row k is the unit vector at the k-th non-pivot column.
      for (int k = 0; k < rdi; ++k) {
        kind[k] = 3;
        ucol[k] = res_cols[k];
      }
    } else {
      int xi = 0, di = 0, o = 0;
      while (xi < npiv || di < rdi) {
        long xc = xi < npiv ? piv_cols[xi] : (long)1 << 40;
        long dc = di < rdi ? res_cols[dpiv[di]] : (long)1 << 40;
        if (xc < dc) {
          kind[o] = 1; srow[o] = xi; ucol[o] = (int)xc; ++xi;
        } else {
          kind[o] = 2; srow[o] = di; ucol[o] = -1; ++di;
        }
        ++o;
      }
    }
  }
  prof_end(c, ph);
  res->out_rows = (size_t)out_rows;
  if (out_rows > 0) {
    // kind 3 (unit row only) is encoded as a value-less row
    const int nv = (int)vcols.size();
    std::vector<int> plan;
    plan.reserve(3 * out_rows + nv);
    for (int o = 0; o < out_rows; ++o) plan.push_back(kind[o] == 3 ? 4 : kind[o]);
    plan.insert(plan.end(), srow.begin(), srow.begin() + out_rows);
    plan.insert(plan.end(), ucol.begin(), ucol.begin() + out_rows);
    plan.insert(plan.end(), vcols.begin(), vcols.end());
    void *vP = nullptr;
    if ((st = ctx_buffer(c, BUF_MISC, plan.size() * sizeof(int) + 64, &vP))) return st;
    int *d_plan = (int *)vP;
    if ((st = upload(c, d_plan, plan.data(), plan.size() * sizeof(int), "fl: plan"))) return st;
    if (csr) {
      if ((st = fl_assemble_csr(c, out_rows, d_plan, M1, ld1, M2, ld2, nv, csr))) return st;
    } else {
      const int grid = std::min(out_rows, c->num_sms * 16);
      int pi = prof_begin(c, "fl_assemble");
      fl_assemble_kernel<<<grid, 256, 0, c->stream>>>(R, ldr, out_rows, n, d_plan, d_plan + out_rows,
                                                      d_plan + 2 * out_rows, M1, ld1, M2, ld2,
                                                      d_plan + 3 * out_rows, nv);
      prof_end(c, pi);
      ctx_launched(c);
    }
  } else if (csr) {
    void *vP = nullptr;
    if ((st = ctx_buffer(c, BUF_FL_CSR_P, 64, &vP))) return st;
    csr->rowptr = static_cast<uint64_t *>(vP);
    csr->nnz = 0;
    cudaError_t e = cudaMemsetAsync(csr->rowptr, 0, 8, c->stream);
    if (e != cudaSuccess) return ctx_cuda(c, e, "fl: csr output");
    c->fl_csr_nnz = 0;
  }
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "fl launch");
}

// ------------------------------------------------ reduced dense echelon form
//
// GaussJordan::echelonize_reduced (lela/algorithms/gauss-jordan.tcc:
// 434-466), as EchelonForm::echelonize (A, true) runs it on a DenseMatrix
// (lela/solutions/echelon-form.h:115-123).  Its recursion GaussJordanTransform
// (:27-230) picks the pivots by the rule of the non-reduced form (the first
// nonzero at or below the current row of the column reduced by the earlier
// pivot rows) and clears each pivot column in every other row by adding
// multiples of the pivot row, which keeps its pivot value x_i.  So pivot
// row i of the result is the non-reduced row U_i plus multiples of the
// later pivot rows, zero in their pivot columns: R = X U_P^-1 U, with U_P
// the pivot columns of U (upper triangular, diagonal x_i) and X =
// diag(x_i).  Here: the non-reduced form on the panels, then U_P and the
// other columns U_N gathered, U_N <- U_P^-1 U_N (the triangular solve), and
// one kernel writes row i back as x_i U_N[i] in the other columns, x_i at
// its pivot column and zero at the other pivot columns.  Rows from the rank
// on are zero already.  The standard method's reduced form,
// Elimination::echelonize_reduced (lela/algorithms/elimination.tcc:143-265),
// picks the same pivots but scales each pivot row by the inverse of its
// pivot (:222): R = U_P^-1 U (unit_pivots).

// Rows 0..r-1 of D from the solved columns: colmap[c] >= 0 is c's column in
// X, colmap[c] = -1 - j marks the pivot column of row j; the pivot values
// are the diagonal of UP.  unit: the pivots become 1 (row i not multiplied
// back by its pivot).
__global__ void reduced_assemble_kernel(uint32_t *__restrict__ D, size_t ld, int r, int n,
                                        const int *__restrict__ colmap,
                                        const uint32_t *__restrict__ X, size_t ldx,
                                        const uint32_t *__restrict__ UP, size_t ldp, Modulus mod,
                                        bool unit) {
  const size_t total = (size_t)r * n;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx / n), col = (int)(idx % n);
    const int cm = colmap[col];
    const uint32_t x = unit ? 1u : UP[(size_t)i * ldp + i];
    const uint32_t v = cm >= 0 ? X[(size_t)i * ldx + cm] : 0u;
    D[(size_t)i * ld + col] =
        cm >= 0 ? (unit ? v : mod_mul(v, x, mod)) : (-1 - cm == i ? x : 0u);
  }
}

int zp_echelon_reduced_dev(Ctx *c, int m, int n, uint32_t p, uint32_t *D, size_t ld,
                           bool unit_pivots, size_t *rank, uint32_t *det) {
  std::vector<int> piv;
  int st = zp_echelon_dev(c, m, n, p, D, ld, rank, det, &piv);
  if (st) return st;
  const int r = (int)*rank;
  if (r == 0) return ST_OK;
  if ((int)piv.size() != r) return ctx_fail(c, ST_CUDA, "reduced echelon: pivot columns missing");
  const int nrem = n - r;
  std::vector<int> colmap(n, 0), cols(piv);
  for (int j = 0; j < r; ++j) colmap[piv[j]] = -1 - j;
  for (int col = 0, k = 0; col < n; ++col)
    if (colmap[col] >= 0) {
      colmap[col] = k++;
      cols.push_back(col);
    }
  const size_t ibytes = ((size_t)2 * n * sizeof(int) + 255) & ~(size_t)255;
  const size_t pbytes = (((size_t)r * r * 4) + 255) & ~(size_t)255;
  void *vb = nullptr;
  if ((st = ctx_buffer(c, BUF_RED, ibytes + pbytes + (size_t)r * std::max(nrem, 1) * 4, &vb)))
    return st;
  int *d_map = static_cast<int *>(vb), *d_cols = d_map + n;
  uint32_t *UP = reinterpret_cast<uint32_t *>(static_cast<uint8_t *>(vb) + ibytes);
  uint32_t *X = reinterpret_cast<uint32_t *>(static_cast<uint8_t *>(vb) + ibytes + pbytes);
  cudaError_t e = cudaMemcpyAsync(d_map, colmap.data(), (size_t)n * sizeof(int),
                                  cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_cols, cols.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice,
                        c->stream);
  if (e != cudaSuccess) return ctx_cuda(c, e, "reduced echelon: columns");
  auto gather = [&](const int *sel, int ncols, uint32_t *out, size_t ldo) {
    const size_t total = (size_t)r * ncols;
    const int grid = (int)std::min<size_t>((total + 255) / 256, (size_t)c->num_sms * 16);
    gather_cols_kernel<<<grid, 256, 0, c->stream>>>(D, ld, r, sel, ncols, out, ldo);
    ctx_launched(c);
  };
  gather(d_cols, r, UP, (size_t)r);
  if (nrem > 0) {
    gather(d_cols + r, nrem, X, (size_t)nrem);
    size_t bad = 0;
    if ((st = zp_trsm_dev(c, true, false, r, nrem, p, 1, UP, (size_t)r, X, (size_t)nrem, &bad)))
      return st;
  }
  const size_t total = (size_t)r * n;
  const int grid = (int)std::min<size_t>((total + 255) / 256, (size_t)c->num_sms * 16);
  reduced_assemble_kernel<<<grid, 256, 0, c->stream>>>(D, ld, r, n, d_map, X,
                                                       (size_t)std::max(nrem, 1), UP, (size_t)r,
                                                       make_modulus(p), unit_pivots);
  ctx_launched(c);
  e = cudaGetLastError();
  return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "reduced echelon: assembly");
}

}  // namespace lela
