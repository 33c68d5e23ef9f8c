// lela_b200/csrc/zp_gemm.cu -- dense gemm over Z/p (Modular<uint32>):
//   C <- alpha * A * B + beta * C  (mod p),  p in [2, 2^32).
//
// Replaces the per-entry delayed-reduction dot products of LELA's generic
// gemm (lela/blas/level3-generic.tcc:285-322 with _dot<Modular<uint32>,
// ZpModule> of lela/blas/level1-modular.tcc:135-158).  Two kernels:
//
// 1. zp_gemm_tc_kernel<L> -- limb-split INT8 tensor-core gemm.  Every entry
//    x in [0, p) is split into L unsigned 8-bit limbs, x = sum_i x_i 2^(8i),
//    with L = 1 (p <= 2^8), 2 (p <= 2^16) or 4 (p <= 2^32).  For each pair of
//    limbs (i, j) the tensor cores form P_ij = A_i * B_j with exact signed
//    32-bit accumulation (tcgen05.mma .kind::i8, accumulators in TMEM).
//    Overflow bound: a limb product is at most 255^2 = 65025, so a K-chunk
//    of at most 33025 terms cannot exceed 2^31 - 1; the host splits K into
//    chunks of KCHUNK = 32768 (the first chunk applies beta, the others add
//    with beta = 1).  The epilogue recombines
//        A*B = sum_s 2^(8s) D_s,   D_s = sum_{i+j=s} P_ij   (D_s < 4 * 2^31)
//    reduces mod p with Barrett reduction and applies alpha and beta; the
//    result is exact, i.e. bit-identical to LELA's.
//
//    Data layout.  A is split into L planes of M x Kp bytes (K-major, i.e.
//    row-major A), B into L planes of N x Kp bytes (K-major, i.e. B^T); Kp =
//    K rounded up to 16 bytes (the TMA row-pitch rule).  One CTA owns a
//    128 x BN tile of C and stacks the limbs: the A operand of the i-th MMA
//    is A_i (128 rows), the B operand is [B_0; ..; B_{L-1}] (L*BN rows), so
//    one 128 x (L*BN) accumulator per A-limb holds P_i0 .. P_i(L-1) side by
//    side; L accumulators use all 512 TMEM columns for L = 2 and 4.
//
//    Pipeline (persistent, warp-specialised, 320 threads): warp 0 issues TMA
//    loads of 128-byte-swizzled K-blocks (128 bytes of K) into a ring of
//    shared-memory stages; warp 1 issues 4*L MMAs of K = 32 per stage and
//    releases stages with tcgen05.commit; warps 2-9 drain the accumulators
//    (one TMEM lane = one row of C per thread, two warps per lane quadrant
//    on the two halves of the tile's columns).  Every wait is bounded.
//
// 2. zp_gemm_plain_kernel -- the "plain GPU form": a CUDA-core tiled gemm
//    whose inner loop is exactly the reference's delayed-reduction dot
//    (64-bit sum of 32x32-bit products, + 2^64 mod p on wrap-around, one
//    final reduction).
// 3. zp_gemm_smallk_kernel -- CUDA-core gemm for the small-K updates of the
//    triangular solve and the echelon panels, where the tensor-core path's
//    fixed cost (limb splits, tensor maps, pipeline start) dominates.  For
//    p < 2^28 a 64-bit sum of 256 products cannot wrap, so the products are
//    summed without checks and the sums reduced every 256 terms.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdio>
#include <mutex>

#include "common.cuh"
#include "context.h"
#include "zp_gemm.h"

namespace lela {

// ------------------------------------------------------------ tile configs
//
// TcCfg<L, T>: tile variant T of the L-limb kernel.  BN = columns of C per
// tile, NMMA = L * BN (the N of one MMA: the L limbs of B stacked), STAGES
// = depth of the shared-memory ring, ACC = accumulator buffers in TMEM
// (each L * NMMA columns; at most 512 in all), EPI = epilogue warps.  With
// ACC = 2 the epilogue of one tile overlaps the MMAs of the next; with ACC =
// 1 the MMAs wait for the epilogue to drain TMEM, but each MMA is wider
// (more operations per byte of shared memory read).  The caller sees two
// shapes, wide (one limb: 256 columns; two limbs: 128 columns, one
// accumulator) and double-buffered (128 / 64 columns, two accumulators).
// Two limbs use 16 epilogue warps, one limb 16 or 8 chosen by K
// (zp_gemm_tile_pick): at short K the epilogue is most of a tile's time,
// and a tcgen05.ld wait covers all of a warp's outstanding TMEM loads, so
// only more warps hide their latency.  Four limbs have variant 0 only: with two accumulators a
// tile would be 16 columns wide, 8 per epilogue thread.
template <int L, int T>
struct TcCfg;
template <>
struct TcCfg<1, 0> {
  static constexpr int BN = 256, NMMA = 256, STAGES = 4, ACC = 2, EPI = 8;
};
template <>
struct TcCfg<1, 1> {
  static constexpr int BN = 128, NMMA = 128, STAGES = 6, ACC = 2, EPI = 16;
};
template <>
struct TcCfg<1, 2> {
  static constexpr int BN = 128, NMMA = 128, STAGES = 6, ACC = 2, EPI = 8;
};
// the GF(2) product at short K (one limb of 0/1 bytes, parity epilogue):
// wide tiles with 16 epilogue warps, 64 columns (one output word) each
template <>
struct TcCfg<1, 3> {
  static constexpr int BN = 256, NMMA = 256, STAGES = 4, ACC = 2, EPI = 16;
};
constexpr int GF2_TC_T = 3;
template <>
struct TcCfg<2, 0> {
  static constexpr int BN = 128, NMMA = 256, STAGES = 3, ACC = 1, EPI = 16;
};
template <>
struct TcCfg<2, 1> {
  static constexpr int BN = 64, NMMA = 128, STAGES = 4, ACC = 2, EPI = 16;
};
template <>
struct TcCfg<4, 0> {
  static constexpr int BN = 32, NMMA = 128, STAGES = 2, ACC = 1, EPI = 8;
};

constexpr int BM = 128;         // rows of C per tile (UMMA M)
constexpr int BK = 128;         // bytes (= limb elements) of K per stage
// Tile raster: groups of GROUP_M row-blocks, column-major inside a group,
// so the 148 tiles in flight share A's group panels and a few of B's.  B's
// limb planes are read once per group.  At 8192^3 (two limbs) a group's A
// planes are 32 MB and stay in L2 beside the streamed B panels; with 32
// row-blocks (64 MB) they did not: DRAM reads per launch went from 1.15 to
// 2.42 GB and the kernel took 4 % longer.
constexpr int GROUP_M = 16;
constexpr int TMEM_COLS = 512;
// warp 0: TMA, warp 1: MMA, warps 2 .. 2 + EPI - 1: epilogue (EPI / 4 per
// TMEM lane quadrant, each on BN / (EPI / 4) columns of a tile)
template <int L, int T>
constexpr int tc_threads() {
  return 64 + 32 * TcCfg<L, T>::EPI;
}

template <int L, int T>
struct TcLayout {
  using Cfg = TcCfg<L, T>;
  static_assert(Cfg::NMMA == L * Cfg::BN, "the B operand stacks the L limbs");
  static_assert(Cfg::ACC * L * Cfg::NMMA <= TMEM_COLS, "accumulators exceed TMEM");
  static_assert(Cfg::EPI % 4 == 0 && Cfg::BN % (Cfg::EPI / 4) == 0 &&
                    (Cfg::BN / (Cfg::EPI / 4)) % 16 == 0,
                "whole lane quadrants, 16-column chunks per epilogue warp");
  static constexpr int A_BYTES = L * BM * BK;
  static constexpr int B_BYTES = Cfg::NMMA * BK;
  static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  static constexpr int BAR_OFF = Cfg::STAGES * STAGE_BYTES;
  // full[S], empty[S], tfull[ACC], tempty[ACC], done, tmem base
  static constexpr int BAR_BYTES = 8 * (2 * Cfg::STAGES + 2 * Cfg::ACC + 1) + 8;
  static constexpr int SMEM = BAR_OFF + BAR_BYTES + 1024;
  static_assert(SMEM <= 227 * 1024, "shared memory per CTA exceeded");
};

__device__ __forceinline__ void tile_coords(int t, int tiles_m, int tiles_n, int &mb, int &nb) {
  int per_group = GROUP_M * tiles_n;
  int g = t / per_group;
  int first_m = g * GROUP_M;
  int gsize = min(GROUP_M, tiles_m - first_m);
  int w = t - g * per_group;
  mb = first_m + w % gsize;
  nb = w / gsize;
}

// Bounded wait that ignores the error word (used only to drain in-flight
// asynchronous operations before the block exits).
__device__ __forceinline__ void mbar_drain(uint64_t *bar, uint32_t parity, uint32_t *err) {
  uint64_t t0 = globaltimer_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (globaltimer_ns() - t0 > WAIT_LIMIT_NS) {
      atomicOr(err, DEVERR_TIMEOUT);
      return;
    }
  }
}

// Reduction for one and two limbs (p <= 2^16): 32-bit Barrett with mu =
// floor(2^32 / p), whose quotient estimate for v < 2^32 is the quotient or
// one less, and c32 = 2^32 mod p for the high word of a two-limb product.
struct Mod32 {
  uint32_t p, mu, c32;
  __device__ __forceinline__ static Mod32 make(uint32_t p) {
    Mod32 m;
    m.p = p;
    m.mu = (uint32_t)((1ull << 32) / p);
    m.c32 = (uint32_t)((1ull << 32) % p);
    return m;
  }
  // v mod p, up to one multiple of p too large (r < 2p)
  __device__ __forceinline__ uint32_t lazy(uint32_t v) const { return v - __umulhi(v, mu) * p; }
  __device__ __forceinline__ uint32_t full(uint32_t v) const {
    const uint32_t r = lazy(v);
    return r >= p ? r - p : r;
  }
};

// How the product v (reduced) and C combine, chosen once per launch:
// C <- v + C (alpha = 1, beta = 1: the gemm C += A*B), C <- C - v
// (alpha = p - 1, beta = 1: the trsm and elimination updates), C <- alpha v
// (beta = 0), or the general alpha v + beta C.  The first three skip the two
// modular products of the general form (the epilogue is instruction-bound
// when K is small).
enum EpiMode : int { EPI_ADD = 0, EPI_SUB = 1, EPI_SET = 2, EPI_AXPBY = 3 };

// The mode is a template parameter: the epilogue's tile loop is
// instantiated once per mode and the launch runs one of them, so the hot
// code holds no per-element branches (the epilogue shares each
// sub-partition's instruction cache with the TMA and MMA warps).
// SMALL: p <= 2^16 (one and two limbs), where every product of two
// residues fits in 32 bits and the 32-bit reduction serves.
template <int MODE, bool SMALL>
__device__ __forceinline__ uint32_t epi_combine(uint32_t v, uint32_t c, const Modulus &mod,
                                                const Mod32 &m32, uint32_t alpha,
                                                uint32_t beta) {
  const uint32_t p = SMALL ? m32.p : (uint32_t)mod.p;
  auto mul = [&](uint32_t a, uint32_t b) -> uint32_t {
    if constexpr (SMALL) return m32.full(a * b);
    else return mod_mul(a, b, mod);
  };
  if constexpr (MODE == EPI_SET) return alpha == 1u ? v : mul(alpha, v);
  if constexpr (MODE == EPI_AXPBY) {
    if constexpr (SMALL) {
      const uint32_t r = mul(alpha, v) + mul(beta, c >= p ? m32.full(c) : c);
      return r >= p ? r - p : r;
    } else {
      return mod_axpby(alpha, v, beta, c, mod);
    }
  }
  if (c >= p) c = SMALL ? m32.full(c) : mod_reduce((uint64_t)c, mod);  // a caller's non-canonical C
  if constexpr (MODE == EPI_ADD) {
    const uint32_t t = p - v;  // v + c mod p without overflow
    return c >= t ? c - t : c + v;
  }
  return c >= v ? c - v : c + (p - v);
}

// The reduced products of 16 consecutive columns of one row, from the
// TMEM accumulators of a tile (tcol: the column of the first one in the
// accumulator of A-limb 0, B-limb 0).  Warp-collective: every lane of the
// warp runs it (tcgen05.ld is .sync.aligned).  The limb products P_ij are
// below 255^2 * 32768 < 2^31 (one K chunk).
template <int L, int BN, int NMMA>
__device__ __forceinline__ void chunk_products(uint32_t tcol, uint32_t (&v)[16],
                                               const Modulus &mod, const Mod32 &m32) {
  if constexpr (L == 1) {
    // one product P_00
    uint32_t r[16];
    tmem_ld16(tcol, r);
    tmem_ld_wait();
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = m32.full(r[i]);
  } else if constexpr (L == 2) {
    // x = 2^16 P_11 + 2^8 (P_01 + P_10) + P_00 < 2^48, as hi 2^32 + lo:
    // x = lo + hi c32 (mod p), and (lo mod p, < 2p) + hi c32 < 2^32 for
    // p <= 2^16 (p = 2^16 has c32 = 0)
    uint32_t p00[16], p01[16], p10[16], p11[16];
    tmem_ld16(tcol, p00);
    tmem_ld16(tcol + BN, p01);
    tmem_ld16(tcol + NMMA, p10);
    tmem_ld16(tcol + NMMA + BN, p11);
    tmem_ld_wait();
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const uint64_t x = ((uint64_t)p11[i] << 16) + ((uint64_t)(p01[i] + p10[i]) << 8) + p00[i];
      const uint32_t t = m32.lazy((uint32_t)x) + (uint32_t)(x >> 32) * m32.c32;
      v[i] = m32.full(t);
    }
  } else {
    // L = 4: x = sum_s 2^(8s) D_s with D_s = sum_{i+j=s} P_ij, gathered as
    // x = F_a + 2^24 F_b + 2^48 D_6 (F_a = D_0 + 2^8 D_1 + 2^16 D_2 < 2^49,
    // F_b likewise from D_3..D_5, D_6 = P_33 < 2^31), then three steps of
    // Horner in 2^24 with one reduction each ((r < 2^32) 2^24 + F < 2^57).
    // Eight columns at a time; the sixteen limb products in two waits.
#pragma unroll
    for (int h = 0; h < 16; h += 8) {
      uint64_t Fa[8], Fb[8];
      uint32_t D6[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        Fa[i] = 0;
        Fb[i] = 0;
      }
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        uint32_t r[2][4][8];
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
          for (int lj = 0; lj < 4; ++lj)
            tmem_ld8(tcol + h + (2 * half + a) * NMMA + lj * BN, r[a][lj]);
        tmem_ld_wait();
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
          for (int lj = 0; lj < 4; ++lj) {
            const int sd = 2 * half + a + lj;  // the digit of this limb product
#pragma unroll
            for (int i = 0; i < 8; ++i) {
              if (sd == 6) D6[i] = r[a][lj][i];
              else if (sd < 3) Fa[i] += (uint64_t)r[a][lj][i] << (8 * sd);
              else Fb[i] += (uint64_t)r[a][lj][i] << (8 * (sd - 3));
            }
          }
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        uint32_t acc = mod_reduce((uint64_t)D6[i], mod);
        acc = mod_reduce(((uint64_t)acc << 24) + Fb[i], mod);
        v[h + i] = mod_reduce(((uint64_t)acc << 24) + Fa[i], mod);
      }
    }
  }
}

// C row segments in registers.  load_c reads n consecutive entries of row
// `crow` from column gn (entries at columns >= N read as 0; crow == nullptr:
// a row past M); 16-byte loads where the row and column allow (vec: C and
// its row stride 16-byte aligned).  store_c writes them back.
template <int NV>
__device__ __forceinline__ void load_c(uint32_t (&c)[NV], const uint32_t *crow, int gn, int N,
                                       bool vec) {
  static_assert(NV % 4 == 0, "whole vectors");
#pragma unroll
  for (int j = 0; j < NV / 4; ++j) {
    const int g = gn + 4 * j;
    if (crow != nullptr && vec && g + 3 < N) {
      const uint4 u = *reinterpret_cast<const uint4 *>(crow + g);
      c[4 * j] = u.x;
      c[4 * j + 1] = u.y;
      c[4 * j + 2] = u.z;
      c[4 * j + 3] = u.w;
    } else {
#pragma unroll
      for (int i = 0; i < 4; ++i)
        c[4 * j + i] = (crow != nullptr && g + i < N) ? crow[g + i] : 0u;
    }
  }
}
template <int NV>
__device__ __forceinline__ void store_c(const uint32_t (&c)[NV], uint32_t *crow, int gn, int N,
                                        bool vec) {
  if (crow == nullptr) return;
#pragma unroll
  for (int j = 0; j < NV / 4; ++j) {
    const int g = gn + 4 * j;
    if (vec && g + 3 < N) {
      *reinterpret_cast<uint4 *>(crow + g) = make_uint4(c[4 * j], c[4 * j + 1], c[4 * j + 2], c[4 * j + 3]);
    } else {
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (g + i < N) crow[g + i] = c[4 * j + i];
    }
  }
}

// GF(2) output (OUT = 1, one limb of 0/1 bytes): the accumulator holds the
// integer count of the row/column bit products; its parity is the GF(2)
// product.  The 256 columns of a tile are packed into four 64-bit
// LittleEndian words (bit j of word w = column 64w + j) and combined as
// C <- (beta ? C : 0) XOR (alpha ? A*B : 0); bits of the last word at
// columns >= N keep their old values.
__device__ __forceinline__ void epilogue_gf2(uint32_t tcol, int gm, int gn0, int M, int N,
                                             uint64_t *C, size_t ldc_words, uint32_t alpha,
                                             uint32_t beta, int cbeg, int cend) {
  uint64_t word = 0;
#pragma unroll 1
  for (int c0 = cbeg; c0 < cend; c0 += 16) {
    uint32_t r[16];
    tmem_ld16(tcol + c0, r);
    tmem_ld_wait();
    uint64_t bits = 0;
#pragma unroll
    for (int i = 0; i < 16; ++i) bits |= (uint64_t)(r[i] & 1u) << i;
    word |= bits << (c0 & 63);
    if ((c0 & 63) == 48) {
      const int wcol = gn0 + (c0 & ~63);
      if (gm < M && wcol < N) {
        const int valid = min(64, N - wcol);
        const uint64_t mask = valid == 64 ? ~0ull : ((1ull << valid) - 1ull);
        uint64_t *dst = C + (size_t)gm * ldc_words + (wcol >> 6);
        const bool part = valid < 64;
        const uint64_t old = (beta || part) ? *dst : 0ull;
        const uint64_t v = (beta ? old : 0ull) ^ (alpha ? word : 0ull);
        *dst = (v & mask) | (old & ~mask);
      }
      word = 0;
    }
  }
}

// K blocks [kb0, kb1) of the row tile starting at row m0: all of K, or,
// with per-row ranges kr (row r of A is zero outside columns [kr[r].x,
// kr[r].y) of the whole matrix; kbase = the whole matrix's column of this
// product's K = 0), the blocks covering the union of the tile's rows'
// ranges.  A tile whose rows are zero in all of K keeps one block: its
// product is zero either way.  Warp-collective (the warp's lanes share the
// rows), so every lane of the calling warp runs it.
__device__ __forceinline__ void tile_kblocks(const int2 *__restrict__ kr, int kbase, int m0, int M,
                                             int K, int &kb0, int &kb1) {
  const int nkb = (K + BK - 1) / BK;
  kb0 = 0;
  kb1 = nkb;
  if (kr == nullptr) return;
  int lo = 0x7fffffff, hi = -0x7fffffff;
  const int lane = threadIdx.x & 31;
  for (int r = m0 + lane; r < min(M, m0 + BM); r += 32) {
    const int2 v = kr[r];
    if (v.y > v.x) {
      lo = min(lo, v.x);
      hi = max(hi, v.y);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if (hi <= lo) {  // no row of the tile has a nonzero anywhere
    kb1 = 1;
    return;
  }
  lo = max(lo - kbase, 0);
  hi = min(hi - kbase, K);
  if (hi <= lo) {  // none inside this product's K range
    kb1 = 1;
    return;
  }
  kb0 = lo / BK;
  kb1 = (hi + BK - 1) / BK;
}

// Epilogue of the Z/p product for one thread (TMEM lane `row` of quadrant
// q, columns cbeg.. of each tile) over this CTA's tiles.  This thread's row
// segment of a tile: W = BN / (EPI / 4) columns from gn0, in blocks of EPB
// columns.
// C's block 0 is loaded before the accumulator is ready (its latency hides
// behind the tile's MMAs), block b + 1 while block b is combined; TMEM is
// released after its last read, before the last block's stores.
template <int L, int T, int MODE>
__device__ __noinline__ void epilogue_tiles(uint32_t tmem, uint64_t *tfull, uint64_t *tempty,
                                               uint32_t *err, uint32_t *C, size_t ldc, int M,
                                               int N, int tiles_m, int tiles_n, int num_tiles,
                                               const Modulus &mod, uint32_t alpha, uint32_t beta,
                                               int row, int q, int cbeg) {
  using Cfg = TcCfg<L, T>;
  constexpr int ACC = Cfg::ACC, BN = Cfg::BN, NMMA = Cfg::NMMA;
  constexpr int W = BN / (Cfg::EPI / 4);
  constexpr int EPB = W < 32 ? W : 32;
  constexpr int NB = W / EPB;
  constexpr bool READC = MODE != EPI_SET;
  const Mod32 m32 = Mod32::make(L < 4 ? (uint32_t)mod.p : 3u);
  const bool vec = ((reinterpret_cast<uintptr_t>(C) & 15u) == 0) && ((ldc & 3u) == 0);
  int it = 0;
  for (int t = blockIdx.x; t < num_tiles; t += gridDim.x, ++it) {
    int mb, nb;
    tile_coords(t, tiles_m, tiles_n, mb, nb);
    const int a = it % ACC;
    const uint32_t aph = (uint32_t)(it / ACC) & 1u;
    const int gm = mb * BM + row;
    const uint32_t tbase = tmem + (uint32_t)(a * L * NMMA) + ((uint32_t)(q * 32) << 16);
    const int gn0 = nb * BN + cbeg;
    uint32_t *crow = gm < M ? C + (size_t)gm * ldc : nullptr;
    uint32_t cb[2][EPB];
    if (READC) load_c<EPB>(cb[0], crow, gn0, N, vec);
    if (!mbar_wait(&tfull[a], aph, err)) return;
    tc_fence_after();
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      uint32_t(&cur)[EPB] = cb[b & 1];
      if (b + 1 < NB && READC) load_c<EPB>(cb[(b + 1) & 1], crow, gn0 + (b + 1) * EPB, N, vec);
#pragma unroll
      for (int h = 0; h < EPB / 16; ++h) {
        uint32_t v[16];
        chunk_products<L, BN, NMMA>(tbase + (uint32_t)(cbeg + b * EPB + 16 * h), v, mod, m32);
#pragma unroll
        for (int i = 0; i < 16; ++i)
          cur[16 * h + i] =
              epi_combine<MODE, (L < 4)>(v[i], READC ? cur[16 * h + i] : 0u, mod, m32, alpha, beta);
      }
      if (b == NB - 1) {
        tc_fence_before();
        mbar_arrive(&tempty[a]);
      }
      store_c<EPB>(cur, crow, gn0 + b * EPB, N, vec);
    }
  }
}

template <int L, int OUT, int T = 0>
__global__ void __launch_bounds__(tc_threads<L, T>(), 1)
    zp_gemm_tc_kernel(const __grid_constant__ CUtensorMap tmA,
                      const __grid_constant__ CUtensorMap tmB, void *__restrict__ Cv,
                      size_t ldc, int M, int N, int K, Modulus mod, uint32_t alpha, uint32_t beta,
                      uint32_t *err, const int2 *__restrict__ kr = nullptr, int kbase = 0) {
  static_assert(OUT == 0 || (L == 1 && (T == 0 || T == GF2_TC_T)), "GF(2) output uses one limb");
  uint32_t *C = static_cast<uint32_t *>(Cv);
  using Cfg = TcCfg<L, T>;
  using Lay = TcLayout<L, T>;
  constexpr int S = Cfg::STAGES, ACC = Cfg::ACC, BN = Cfg::BN, NMMA = Cfg::NMMA;
  constexpr uint32_t IDESC = idesc_u8_s32(BM, NMMA);

  extern __shared__ uint8_t smem_raw[];
  uint32_t base_off = smem_u32(smem_raw);
  uint8_t *smem = smem_raw + ((1024 - (base_off & 1023)) & 1023);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + Lay::BAR_OFF);
  uint64_t *empty = full + S;
  uint64_t *tfull = empty + S;
  uint64_t *tempty = tfull + ACC;
  uint64_t *done = tempty + ACC;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tiles_m = (M + BM - 1) / BM, tiles_n = (N + BN - 1) / BN;
  const int num_tiles = tiles_m * tiles_n;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < ACC; ++a) {
      mbar_init(&tfull[a], 1);
      mbar_init(&tempty[a], 32 * Cfg::EPI);
    }
    mbar_init(done, 1);
    fence_barrier_init();
    prefetch_tmap(&tmA);
    prefetch_tmap(&tmB);
  }
  if (warp == 1) tmem_alloc(tmem_slot, TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    // ------------------------------------------------------------ producer
    // The whole warp walks the tiles (their K ranges are warp-collective);
    // lane 0 issues the loads, and its status is shared each tile so that
    // the lanes leave together.
    uint32_t s = 0, ph = 0;
    uint32_t issued = 0, last_ph[S];
    for (int i = 0; i < S; ++i) last_ph[i] = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < num_tiles; t += gridDim.x) {
      int mb, nb, kb0, kb1;
      tile_coords(t, tiles_m, tiles_n, mb, nb);
      tile_kblocks(kr, kbase, mb * BM, M, K, kb0, kb1);
      if (lane == 0) {
        for (int kb = kb0; kb < kb1; ++kb) {
          if (!mbar_wait(&empty[s], ph ^ 1, err)) { ok = false; break; }
          uint8_t *sa = smem + s * Lay::STAGE_BYTES;
          uint8_t *sb = sa + Lay::A_BYTES;
          mbar_arrive_expect_tx(&full[s], Lay::STAGE_BYTES);
          tma_load_3d(sa, &tmA, &full[s], kb * BK, mb * BM, 0);
          tma_load_3d(sb, &tmB, &full[s], kb * BK, nb * BN, 0);
          issued |= 1u << s;
          last_ph[s] = ph;
          if (++s == S) { s = 0; ph ^= 1; }
        }
      }
      if (!__shfl_sync(0xffffffffu, ok ? 1 : 0, 0)) break;
    }
    if (lane == 0 && !ok) {
      // Wait for the loads already in flight before the block may exit.
      for (int i = 0; i < S; ++i)
        if (issued & (1u << i)) mbar_drain(&full[i], last_ph[i], err);
    }
  } else if (warp == 1) {
    // ----------------------------------------------------------- MMA issue
    // As the producer: the warp walks the tiles, lane 0 issues the MMAs.
    uint32_t s = 0, ph = 0;
    int it = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < num_tiles; t += gridDim.x, ++it) {
      int mb, nb, kb0, kb1;
      tile_coords(t, tiles_m, tiles_n, mb, nb);
      tile_kblocks(kr, kbase, mb * BM, M, K, kb0, kb1);
      if (lane == 0) {
        const int a = it % ACC;
        const uint32_t aph = (uint32_t)(it / ACC) & 1u;
        if (!mbar_wait(&tempty[a], aph ^ 1, err)) ok = false;
        tc_fence_after();
        const uint32_t dbase = tmem + (uint32_t)(a * L * NMMA);
        for (int kb = kb0; kb < kb1 && ok; ++kb) {
          if (!mbar_wait(&full[s], ph, err)) { ok = false; break; }
          tc_fence_after();
          uint8_t *sa = smem + s * Lay::STAGE_BYTES;
          uint8_t *sb = sa + Lay::A_BYTES;
          const uint64_t bd = smem_desc_sw128(sb);
#pragma unroll
          for (int l = 0; l < L; ++l) {
            const uint64_t ad = smem_desc_sw128(sa + l * BM * BK);
#pragma unroll
            for (int kk = 0; kk < BK / 32; ++kk) {
              // +32 bytes of K inside the 128-byte swizzled row = +2 in the
              // descriptor's (address >> 4) field.
              mma_u8(dbase + (uint32_t)(l * NMMA), ad + 2 * kk, bd + 2 * kk, IDESC,
                     (kb != kb0 || kk != 0) ? 1u : 0u);
            }
          }
          mma_commit(&empty[s]);
          if (++s == S) { s = 0; ph ^= 1; }
        }
        if (ok) mma_commit(&tfull[a]);
      }
      if (!__shfl_sync(0xffffffffu, ok ? 1 : 0, 0)) break;
    }
    if (lane == 0) {
      // All MMAs of this thread must finish before TMEM is released.
      mma_commit(done);
      mbar_drain(done, 0, err);
    }
  } else {
    // ------------------------------------------------------------ epilogue
    // EPI / 4 warps per TMEM lane quadrant, each on a BN / (EPI / 4) column
    // part of every tile
    const int q = warp & 3;  // TMEM lane quadrant this warp may access
    const int row = q * 32 + lane;
    const int part = (warp - 2) >> 2;
    const int cbeg = part * (BN / (Cfg::EPI / 4));
    if constexpr (OUT == 0) {
      const int emode = beta == 0u ? EPI_SET
                        : (beta == 1u && alpha == 1u) ? EPI_ADD
                        : (beta == 1u && alpha == (uint32_t)mod.p - 1u) ? EPI_SUB
                                                                       : EPI_AXPBY;
#define LELA_EPI(MODE)                                                                          \
  epilogue_tiles<L, T, MODE>(tmem, tfull, tempty, err, C, ldc, M, N, tiles_m, tiles_n, num_tiles, \
                             mod, alpha, beta, row, q, cbeg)
      switch (emode) {
        case EPI_ADD: LELA_EPI(EPI_ADD); break;
        case EPI_SUB: LELA_EPI(EPI_SUB); break;
        case EPI_SET: LELA_EPI(EPI_SET); break;
        default: LELA_EPI(EPI_AXPBY); break;
      }
#undef LELA_EPI
    } else {
      int it = 0;
      for (int t = blockIdx.x; t < num_tiles; t += gridDim.x, ++it) {
        int mb, nb;
        tile_coords(t, tiles_m, tiles_n, mb, nb);
        const int a = it % ACC;
        const uint32_t aph = (uint32_t)(it / ACC) & 1u;
        const int gm = mb * BM + row;
        const uint32_t tbase = tmem + (uint32_t)(a * L * NMMA) + ((uint32_t)(q * 32) << 16);
        if (!mbar_wait(&tfull[a], aph, err)) break;
        tc_fence_after();
        epilogue_gf2(tbase, gm, nb * BN, M, N, static_cast<uint64_t *>(Cv), ldc, alpha, beta,
                     cbeg, cbeg + BN / (Cfg::EPI / 4));
        tc_fence_before();
        mbar_arrive(&tempty[a]);
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, TMEM_COLS);
  }
}

// ------------------------------------------------------------ limb splits
// A (M x kc, row stride lda, u32) -> L planes of M x Kp bytes.
template <int L>
__global__ void split_rows_kernel(const uint32_t *__restrict__ A, size_t lda, int M, int kc,
                                  uint8_t *__restrict__ out, int Kp) {
  const int kq = (kc + 3) >> 2;
  const size_t total = (size_t)M * kq;
  const size_t plane = (size_t)M * Kp;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(idx / kq), k = (int)(idx % kq) * 4;
    const uint32_t *src = A + (size_t)r * lda + k;
    uint32_t v[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] = (k + i < kc) ? __ldg(src + i) : 0u;
#pragma unroll
    for (int l = 0; l < L; ++l) {
      uint32_t w = 0;
#pragma unroll
      for (int i = 0; i < 4; ++i) w |= ((v[i] >> (8 * l)) & 0xFFu) << (8 * i);
      *reinterpret_cast<uint32_t *>(out + l * plane + (size_t)r * Kp + k) = w;
    }
  }
}

// B (kc x N, row stride ldb, u32) -> L planes of N x Kp bytes (transposed),
// through a 64 (k) x 32 (n) shared-memory tile.
template <int L>
__global__ void split_cols_kernel(const uint32_t *__restrict__ B, size_t ldb, int kc, int N,
                                  uint8_t *__restrict__ out, int Kp) {
  __shared__ uint32_t tile[64][33];
  const int n0 = blockIdx.x * 32, k0 = blockIdx.y * 64;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const size_t plane = (size_t)N * Kp;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    int k = k0 + ty + 8 * i, n = n0 + tx;
    tile[ty + 8 * i][tx] = (k < kc && n < N) ? __ldg(B + (size_t)k * ldb + n) : 0u;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    int w = threadIdx.x + 256 * j;
    int n = w >> 4, kw = (w & 15) * 4;
    int gn = n0 + n, gk = k0 + kw;
    if (gn < N && gk < Kp) {
#pragma unroll
      for (int l = 0; l < L; ++l) {
        uint32_t word = 0;
#pragma unroll
        for (int i = 0; i < 4; ++i) word |= ((tile[kw + i][n] >> (8 * l)) & 0xFFu) << (8 * i);
        *reinterpret_cast<uint32_t *>(out + l * plane + (size_t)gn * Kp + gk) = word;
      }
    }
  }
}

// ------------------------------------------------------------ plain gemm
constexpr int PT = 64, PK = 32;

__global__ void __launch_bounds__(256)
    zp_gemm_plain_kernel(const uint32_t *__restrict__ A, size_t lda,
                         const uint32_t *__restrict__ B, size_t ldb, uint32_t *__restrict__ C,
                         size_t ldc, int M, int N, int K, Modulus mod, uint32_t two64,
                         uint32_t alpha, uint32_t beta) {
  __shared__ uint32_t As[PK][PT + 1];
  __shared__ uint32_t Bs[PK][PT + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int m0 = blockIdx.y * PT, n0 = blockIdx.x * PT;
  uint64_t acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0;

  for (int k0 = 0; k0 < K; k0 += PK) {
#pragma unroll
    for (int e = 0; e < (PT * PK) / 256; ++e) {
      int idx = threadIdx.x + 256 * e;
      int r = idx / PK, kk = idx % PK;  // A tile: 64 rows x 32 k
      int gm = m0 + r, gk = k0 + kk;
      As[kk][r] = (gm < M && gk < K) ? __ldg(A + (size_t)gm * lda + gk) : 0u;
      int kr = idx / PT, c = idx % PT;  // B tile: 32 k x 64 cols
      int gk2 = k0 + kr, gn = n0 + c;
      Bs[kr][c] = (gk2 < K && gn < N) ? __ldg(B + (size_t)gk2 * ldb + gn) : 0u;
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < PK; ++kk) {
      uint32_t a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          uint64_t t = (uint64_t)a[i] * b[j];
          uint64_t s = acc[i][j] + t;
          acc[i][j] = (s < t) ? s + two64 : s;
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    int gm = m0 + ty + 16 * i;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int gn = n0 + tx + 16 * j;
      if (gn >= N) continue;
      uint32_t d = mod_reduce(acc[i][j], mod);
      uint32_t c = beta ? C[(size_t)gm * ldc + gn] : 0u;
      C[(size_t)gm * ldc + gn] = mod_axpby(alpha, d, beta, c, mod);
    }
  }
}

// Same tiling as the plain kernel.  NOWRAP (p < 2^28): unchecked sums,
// reduced modulo p after every 256 terms (256 (p-1)^2 < 2^64).
template <bool NOWRAP>
__global__ void __launch_bounds__(256)
    zp_gemm_smallk_kernel(const uint32_t *__restrict__ A, size_t lda,
                          const uint32_t *__restrict__ B, size_t ldb, uint32_t *__restrict__ C,
                          size_t ldc, int M, int N, int K, Modulus mod, uint32_t two64,
                          uint32_t alpha, uint32_t beta) {
  __shared__ uint32_t As[PK][PT + 1];
  __shared__ uint32_t Bs[PK][PT + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int m0 = blockIdx.y * PT, n0 = blockIdx.x * PT;
  uint64_t acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0;

  for (int k0 = 0; k0 < K; k0 += PK) {
#pragma unroll
    for (int e = 0; e < (PT * PK) / 256; ++e) {
      int idx = threadIdx.x + 256 * e;
      int r = idx / PK, kk = idx % PK;
      int gm = m0 + r, gk = k0 + kk;
      As[kk][r] = (gm < M && gk < K) ? __ldg(A + (size_t)gm * lda + gk) : 0u;
      int kr = idx / PT, c = idx % PT;
      int gk2 = k0 + kr, gn = n0 + c;
      Bs[kr][c] = (gk2 < K && gn < N) ? __ldg(B + (size_t)gk2 * ldb + gn) : 0u;
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < PK; ++kk) {
      uint32_t a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
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
    if (NOWRAP && ((k0 / PK) & 7) == 7)
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = mod_reduce(acc[i][j], mod);
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    int gm = m0 + ty + 16 * i;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int gn = n0 + tx + 16 * j;
      if (gn >= N) continue;
      uint32_t d = mod_reduce(acc[i][j], mod);
      uint32_t c = beta ? C[(size_t)gm * ldc + gn] : 0u;
      C[(size_t)gm * ldc + gn] = mod_axpby(alpha, d, beta, c, mod);
    }
  }
}

// Scale C <- beta * C (mod p), used when K = 0 or alpha = 0.
__global__ void zp_scale_kernel(uint32_t *C, size_t ldc, int M, int N, Modulus mod,
                                uint32_t beta) {
  const size_t total = (size_t)M * N;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    size_t r = idx / N, c = idx % N;
    uint32_t *x = C + r * ldc + c;
    *x = beta ? mod_mul(*x, beta, mod) : 0u;
  }
}

// ------------------------------------------------------------------ host
static uint32_t host_two64(uint32_t p) {
  uint64_t t = 2;
  for (int i = 0; i < 6; ++i) t = (t * t) % p;
  return (uint32_t)t;
}

int zp_limbs_for(uint32_t p) { return p <= 256u ? 1 : (p <= 65536u ? 2 : 4); }

static int encode_3d(Ctx *c, CUtensorMap *tm, void *base, uint64_t d0, uint64_t d1, uint64_t d2,
                     uint64_t stride1, uint64_t stride2, uint32_t b0, uint32_t b1, uint32_t b2) {
  auto fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(c->encode_tiled);
  if (!fn) return ctx_fail(c, ST_CUDA, "cuTensorMapEncodeTiled unavailable");
  cuuint64_t dims[3] = {d0, d1, d2};
  cuuint64_t strides[2] = {stride1, stride2};
  cuuint32_t box[3] = {b0, b1, b2};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(tm, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, base, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    char msg[160];
    snprintf(msg, sizeof msg, "cuTensorMapEncodeTiled failed (%d) dims %llu %llu %llu", (int)r,
             (unsigned long long)d0, (unsigned long long)d1, (unsigned long long)d2);
    return ctx_fail(c, ST_CUDA, msg);
  }
  return ST_OK;
}

template <int L, int T = 0>
static int tc_attr(Ctx *c) {
  return ctx_smem_attr(c, (const void *)zp_gemm_tc_kernel<L, 0, T>, TcLayout<L, T>::SMEM,
                       "cudaFuncSetAttribute(zp_gemm_tc)");
}

template <int L, int T>
static int launch_tc(Ctx *c, int M, int N, int K, const Modulus &mod, uint32_t alpha,
                     const uint32_t *A, size_t lda, const uint32_t *B, size_t ldb, uint32_t beta,
                     uint32_t *C, size_t ldc, uint8_t *ws, const int2 *kr, int kbase) {
  using Cfg = TcCfg<L, T>;
  using Lay = TcLayout<L, T>;
  if (int st = tc_attr<L, T>(c)) return st;
  const int tiles = ((M + BM - 1) / BM) * ((N + Cfg::BN - 1) / Cfg::BN);
  uint32_t b = beta;
  for (int k0 = 0; k0 < K; k0 += ZP_KCHUNK) {
    const int kc = std::min(ZP_KCHUNK, K - k0);
    const int Kp = (kc + 15) & ~15;
    uint8_t *Al = ws;
    uint8_t *Bl = ws + (size_t)L * M * Kp;
    {
      const size_t total = (size_t)M * ((kc + 3) / 4);
      int grid = (int)std::min<size_t>((total + 255) / 256, (size_t)c->num_sms * 16);
      int pi = prof_begin(c, "zp_split");
      split_rows_kernel<L><<<grid, 256, 0, c->stream>>>(A + k0, lda, M, kc, Al, Kp);
      dim3 grid2((N + 31) / 32, (Kp + 63) / 64);
      split_cols_kernel<L><<<grid2, 256, 0, c->stream>>>(B + (size_t)k0 * ldb, ldb, kc, N, Bl, Kp);
      prof_end(c, pi);
      ctx_launched(c, 2);
    }
    CUtensorMap tmA, tmB;
    int st = encode_3d(c, &tmA, Al, (uint64_t)kc, (uint64_t)M, L, (uint64_t)Kp,
                       (uint64_t)M * Kp, BK, BM, L);
    if (st) return st;
    st = encode_3d(c, &tmB, Bl, (uint64_t)kc, (uint64_t)N, L, (uint64_t)Kp, (uint64_t)N * Kp, BK,
                   Cfg::BN, L);
    if (st) return st;
    const int grid = std::min(tiles, c->num_sms);
    int pi = prof_begin(c, "zp_gemm_tc");
    zp_gemm_tc_kernel<L, 0, T><<<grid, tc_threads<L, T>(), Lay::SMEM, c->stream>>>(
        tmA, tmB, C, ldc, M, N, kc, mod, alpha, b, c->dstatus, kr, kbase + k0);
    prof_end(c, pi);
    ctx_launched(c);
    b = 1;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return ctx_cuda(c, e, "zp_gemm_tc launch");
  return ST_OK;
}

size_t zp_gemm_workspace_bytes(uint32_t p, int M, int N, int K) {
  const int L = zp_limbs_for(p);
  const int kc = std::min(ZP_KCHUNK, K);
  const size_t Kp = (size_t)((kc + 15) & ~15);
  return (size_t)L * ((size_t)M + N) * Kp + 256;
}

int zp_gemm_tile_pick(const Ctx *c, int K, uint32_t p) {
  const int L = zp_limbs_for(p);
  if (L == 4) return 0;  // one variant for four limbs
  // Measured on the B200 (kernel ms, M = N = 8192, p = 65521 / 251, the
  // 32-bit reductions of the epilogue): two limbs, wide tiles with 8 / 16
  // epilogue warps: 1.346 / 1.338 at K = 8192 (with the earlier 64-bit
  // reduction 8 / 16 warps took 0.351 / 0.318 at K = 512 and 0.543 / 0.496
  // at 2048).  One limb, double-buffered tiles with 8 / 16 warps: 0.256 /
  // 0.256 at K = 2048, 0.284 / 0.322 at 3072, 0.596 / 0.642 at 8192 (0.316
  // / 0.249 at 512 with the earlier reduction).
  const bool wide = c->gemm_tile == GEMM_TILE_WIDE ||
                    (c->gemm_tile == GEMM_TILE_AUTO && L == 2 && K >= 512);
  if (L == 2) return wide ? 0 : 1;
  return wide ? 0 : (K <= 2048 ? 1 : 2);
}

int zp_gemm_pick(const Ctx *c, int M, int N, int K, uint32_t p) {
  if (c->gemm_kernel != GEMM_AUTO) return c->gemm_kernel;
  // small K: the CUDA-core kernel below its measured crossover with the
  // tensor-core path, which has a fixed cost of about 20 us (limb split and
  // launch) and then runs far faster.  Measured on the B200 (us per call,
  // small-K / tensor cores, p = 65521): 8000 x 448 x 64: 57.8 / 31.3;
  // 8000 x 64 x 64: 14.9 / 20.6; 4000 x 200 x 40: 23.9 / 20.4; p = 2^31 - 1,
  // 8000 x 448 x 64: 104.8 / 76.4 -- a crossover near 3e7 multiply-adds,
  // higher for narrow C (the tensor cores' tiles are 64 or more columns wide)
  const double work = (double)M * N * K;
  const bool smallk = K <= 256 && (work <= 2.5e7 || (N <= 96 && work <= 6.0e7));
  (void)p;
  return smallk ? GEMM_SMALLK : GEMM_TC;
}

int zp_gemm_dev(Ctx *c, int kernel, int M, int N, int K, uint32_t p, uint32_t alpha,
                const uint32_t *A, size_t lda, const uint32_t *B, size_t ldb, uint32_t beta,
                uint32_t *C, size_t ldc, uint8_t *ws_override, const int2 *kr, int kbase) {
  if (p < 2) return ctx_fail(c, ST_ARG, "modulus must be at least 2");
  if (M < 0 || N < 0 || K < 0) return ctx_fail(c, ST_ARG, "negative dimension");
  if (M == 0 || N == 0) return ST_OK;
  if (ldc < (size_t)N || (K > 0 && (lda < (size_t)K || ldb < (size_t)N)))
    return ctx_fail(c, ST_ARG, "leading dimension smaller than the row length");
  const Modulus mod = make_modulus(p);
  alpha %= p;
  beta %= p;
  if (K == 0 || alpha == 0) {
    if (beta == 1) return ST_OK;
    const size_t total = (size_t)M * N;
    int grid = (int)std::min<size_t>((total + 255) / 256, (size_t)c->num_sms * 8);
    zp_scale_kernel<<<grid, 256, 0, c->stream>>>(C, ldc, M, N, mod, beta);
    ctx_launched(c);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "zp_scale launch");
  }
  if (kernel == GEMM_AUTO) kernel = zp_gemm_pick(c, M, N, K, p);
  if (kernel == GEMM_SMALLK) {
    dim3 grid((N + PT - 1) / PT, (M + PT - 1) / PT);
    int pi = prof_begin(c, "zp_gemm_smallk");
    if (p < (1u << 28))
      zp_gemm_smallk_kernel<true><<<grid, 256, 0, c->stream>>>(A, lda, B, ldb, C, ldc, M, N, K,
                                                               mod, host_two64(p), alpha, beta);
    else
      zp_gemm_smallk_kernel<false><<<grid, 256, 0, c->stream>>>(A, lda, B, ldb, C, ldc, M, N, K,
                                                                mod, host_two64(p), alpha, beta);
    prof_end(c, pi);
    ctx_launched(c);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "zp_gemm_smallk launch");
  }
  if (kernel == GEMM_PLAIN) {
    dim3 grid((N + PT - 1) / PT, (M + PT - 1) / PT);
    int pi = prof_begin(c, "zp_gemm_plain");
    zp_gemm_plain_kernel<<<grid, 256, 0, c->stream>>>(A, lda, B, ldb, C, ldc, M, N, K, mod,
                                                      host_two64(p), alpha, beta);
    prof_end(c, pi);
    ctx_launched(c);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "zp_gemm_plain launch");
  }
  uint8_t *ws = ws_override;
  if (!ws) {
    void *w = nullptr;
    int st = ctx_workspace(c, zp_gemm_workspace_bytes(p, M, N, K), &w);
    if (st) return st;
    ws = static_cast<uint8_t *>(w);
  }
  const int tv = zp_gemm_tile_pick(c, K, p);
#define LELA_TC(L, T) launch_tc<L, T>(c, M, N, K, mod, alpha, A, lda, B, ldb, beta, C, ldc, ws, kr, kbase)
  switch (zp_limbs_for(p)) {
    case 1:
      return tv == 0 ? LELA_TC(1, 0) : tv == 1 ? LELA_TC(1, 1) : LELA_TC(1, 2);
    case 2:
      return tv == 0 ? LELA_TC(2, 0) : LELA_TC(2, 1);
#undef LELA_TC
    default:
      return launch_tc<4, 0>(c, M, N, K, mod, alpha, A, lda, B, ldb, beta, C, ldc, ws, kr, kbase);
  }
}

// ============================================ pipelined host-pointer gemm
//
// The host-pointer gemm moves (M K + K N + 2 M N) * 4 bytes over the host
// link for 2 M N K operations on the GPU: at 8192^3 the copies take about
// ten times as long as the product.  The rows of C are therefore done in
// blocks: B goes over first, then A's and C's rows block by block on the
// copy_in stream; each block's product runs on the handle stream as soon as
// its rows are in, and its rows of C go back on the copy_out stream while
// later blocks still arrive (the two directions of the link run at once).
// The result is the same product: every output element is computed by the
// same kernel from the same operands, only the launches cover fewer rows.

bool zp_gemm_pipelined(const Ctx *c, int M, int N, int K, uint32_t p, uint32_t alpha) {
  return K > 0 && K <= ZP_KCHUNK && alpha % p != 0 && M >= 2 * PIPE_MIN_ROWS &&
         zp_gemm_pick(c, M, N, K, p) == GEMM_TC;
}

template <int L>
static int host_rows(Ctx *c, int M, int N, int K, const Modulus &mod, uint32_t alpha,
                     const uint32_t *hA, size_t lda, const uint32_t *hB, size_t ldb,
                     uint32_t beta, uint32_t *hC, size_t ldc, uint32_t *dA, uint32_t *dB,
                     uint32_t *dC, uint8_t *ws) {
  using Cfg = TcCfg<L, 0>;
  using Lay = TcLayout<L, 0>;
  if (int st = tc_attr<L>(c)) return st;
  const int Kp = (K + 15) & ~15;
  // row blocks: a multiple of the tile height, at most PIPE_MAX_BLOCKS
  const int per = (M + PIPE_MAX_BLOCKS - 1) / PIPE_MAX_BLOCKS;
  const int rb = std::max(PIPE_MIN_ROWS, (per + BM - 1) / BM * BM);
  const int nblk = (M + rb - 1) / rb;
  cudaEvent_t *ready = c->pipe_ev, *done = c->pipe_ev + PIPE_MAX_BLOCKS;
  cudaEvent_t ev_start = c->pipe_ev[2 * PIPE_MAX_BLOCKS], ev_b = c->pipe_ev[2 * PIPE_MAX_BLOCKS + 1],
              ev_out = c->pipe_ev[2 * PIPE_MAX_BLOCKS + 2];
  const size_t rowA = (size_t)K * 4, rowC = (size_t)N * 4;
  // the copies start after the work already queued on the handle stream
  cudaError_t e = cudaEventRecord(ev_start, c->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(c->copy_in, ev_start, 0);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(c->copy_out, ev_start, 0);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(dB, rowC, hB, ldb * 4, rowC, (size_t)K, cudaMemcpyHostToDevice,
                          c->copy_in);
  if (e == cudaSuccess) e = cudaEventRecord(ev_b, c->copy_in);
  for (int j = 0; e == cudaSuccess && j < nblk; ++j) {
    const int r0 = j * rb, rows = std::min(rb, M - r0);
    e = cudaMemcpy2DAsync(dA + (size_t)r0 * K, rowA, hA + (size_t)r0 * lda, lda * 4, rowA,
                          (size_t)rows, cudaMemcpyHostToDevice, c->copy_in);
    if (e == cudaSuccess && beta)
      e = cudaMemcpy2DAsync(dC + (size_t)r0 * N, rowC, hC + (size_t)r0 * ldc, ldc * 4, rowC,
                            (size_t)rows, cudaMemcpyHostToDevice, c->copy_in);
    if (e == cudaSuccess) e = cudaEventRecord(ready[j], c->copy_in);
  }
  // B's limb planes once; block j's A planes in their own part of the
  // workspace, so that a block's split never overwrites planes an earlier
  // block's kernel still reads
  int st = ST_OK;
  uint8_t *Bl = ws + (size_t)L * M * Kp;
  CUtensorMap tmB;
  if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, ev_b, 0);
  if (e == cudaSuccess) {
    int pi = prof_begin(c, "zp_split");
    dim3 grid2((N + 31) / 32, (Kp + 63) / 64);
    split_cols_kernel<L><<<grid2, 256, 0, c->stream>>>(dB, (size_t)N, K, N, Bl, Kp);
    prof_end(c, pi);
    ctx_launched(c);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    st = encode_3d(c, &tmB, Bl, (uint64_t)K, (uint64_t)N, L, (uint64_t)Kp, (uint64_t)N * Kp, BK,
                   Cfg::BN, L);
  for (int j = 0; e == cudaSuccess && !st && j < nblk; ++j) {
    const int r0 = j * rb, rows = std::min(rb, M - r0);
    uint8_t *Al = ws + (size_t)L * r0 * Kp;
    e = cudaStreamWaitEvent(c->stream, ready[j], 0);
    if (e != cudaSuccess) break;
    const size_t total = (size_t)rows * ((K + 3) / 4);
    const int sgrid = (int)std::min<size_t>((total + 255) / 256, (size_t)c->num_sms * 16);
    int pi = prof_begin(c, "zp_split");
    split_rows_kernel<L><<<sgrid, 256, 0, c->stream>>>(dA + (size_t)r0 * K, (size_t)K, rows, K,
                                                       Al, Kp);
    prof_end(c, pi);
    CUtensorMap tmA;
    st = encode_3d(c, &tmA, Al, (uint64_t)K, (uint64_t)rows, L, (uint64_t)Kp,
                   (uint64_t)rows * Kp, BK, BM, L);
    if (st) break;
    const int tiles = ((rows + BM - 1) / BM) * ((N + Cfg::BN - 1) / Cfg::BN);
    pi = prof_begin(c, "zp_gemm_tc");
    zp_gemm_tc_kernel<L, 0><<<std::min(tiles, c->num_sms), tc_threads<L, 0>(), Lay::SMEM, c->stream>>>(
        tmA, tmB, dC + (size_t)r0 * N, (size_t)N, rows, N, K, mod, alpha, beta, c->dstatus);
    prof_end(c, pi);
    ctx_launched(c, 2);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventRecord(done[j], c->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->copy_out, done[j], 0);
    if (e == cudaSuccess)
      e = cudaMemcpy2DAsync(hC + (size_t)r0 * ldc, ldc * 4, dC + (size_t)r0 * N, rowC, rowC,
                            (size_t)rows, cudaMemcpyDeviceToHost, c->copy_out);
  }
  // the handle stream ends after the last copy out
  if (e == cudaSuccess && !st) e = cudaEventRecord(ev_out, c->copy_out);
  if (e == cudaSuccess && !st) e = cudaStreamWaitEvent(c->stream, ev_out, 0);
  if (e != cudaSuccess || st) {
    // copies already queued may still use the caller's buffers
    cudaStreamSynchronize(c->copy_in);
    cudaStreamSynchronize(c->copy_out);
    return st ? st : ctx_cuda(c, e, "pipelined gemm");
  }
  return ST_OK;
}

int zp_gemm_host_rows(Ctx *c, int M, int N, int K, uint32_t p, uint32_t alpha,
                      const uint32_t *hA, size_t lda, const uint32_t *hB, size_t ldb,
                      uint32_t beta, uint32_t *hC, size_t ldc, uint32_t *dA, uint32_t *dB,
                      uint32_t *dC) {
  if (!zp_gemm_pipelined(c, M, N, K, p, alpha)) return ctx_fail(c, ST_ARG, "not a pipelined gemm");
  if (int st = ctx_pipe(c)) return st;
  void *w = nullptr;
  if (int st = ctx_workspace(c, zp_gemm_workspace_bytes(p, M, N, K), &w)) return st;
  uint8_t *ws = static_cast<uint8_t *>(w);
  const Modulus mod = make_modulus(p);
  alpha %= p;
  beta %= p;
  switch (zp_limbs_for(p)) {
    case 1:
      return host_rows<1>(c, M, N, K, mod, alpha, hA, lda, hB, ldb, beta, hC, ldc, dA, dB, dC, ws);
    case 2:
      return host_rows<2>(c, M, N, K, mod, alpha, hA, lda, hB, ldb, beta, hC, ldc, dA, dB, dC, ws);
    default:
      return host_rows<4>(c, M, N, K, mod, alpha, hA, lda, hB, ldb, beta, hC, ldc, dA, dB, dC, ws);
  }
}

}  // namespace lela

// ====================================================== no-allocation gemm
//
// lela_cuda_gemm_zp_u32_noalloc: the tensor-core Z/p gemm for callers that
// cannot allocate device memory -- code running under a memory manager that
// owns every device allocation (a host framework's caching allocator or a
// fixed per-process memory budget), or latency-critical paths where
// cudaMalloc/cudaFree, which may synchronise the device, are not allowed.
// Such a caller passes device pointers for A, B and C; the limb planes the
// kernel needs as scratch live in the fixed array below instead of a
// handle's workspace, so this entry point calls no cudaMalloc, cudaFree or
// other allocating routine and needs no handle.
//
// Limits and sharing:
//  - the scratch is NOALLOC_PLANE_BYTES = 64 MiB of limb planes, enough for
//    L * (m + n) * round16(min(k, 32768)) bytes, L = 1, 2 or 4 limbs for
//    p <= 2^8, 2^16, 2^32 (e.g. m = n = k = 4096 at p = 65521); larger
//    problems are rejected with LELA_CUDA_ERR_ARG before any GPU work;
//  - the array is a file-scope __device__ variable: every GPU that loads
//    this library holds it (plus 256 bytes of status) until the process
//    exits;
//  - all calls on a device share it and it keeps the last call's contents.
//    Each call writes every scratch byte its kernel reads (the K tail of a
//    row is never read: the TMA descriptors stop at k) and clears its
//    status word first, so nothing else must start at zero.  Calls whose
//    GPU work overlaps (different streams or host threads without
//    ordering) race on the scratch and give wrong results.
//  - The first call on a device does its set-up there, with that device
//    current: it looks up the array's device address with
//    cudaGetSymbolAddress and sets the kernels' shared-memory attribute.
//    Make that first call before any stream capture.  The set-up is kept
//    for the life of the process, so the entry point must not be called
//    after cudaDeviceReset (which unloads the module the address and the
//    attributes belong to).
namespace lela {

constexpr size_t NOALLOC_STATUS_BYTES = 256;
constexpr size_t NOALLOC_PLANE_BYTES = (size_t)64 << 20;
static __device__ __align__(256) uint8_t g_noalloc_scratch[NOALLOC_STATUS_BYTES + NOALLOC_PLANE_BYTES];

namespace {

constexpr int NOALLOC_MAX_DEVICES = 64;
struct NoallocDevice {
  bool ready;
  uint8_t *base;  // device address of g_noalloc_scratch on this device
  int num_sms;
};
NoallocDevice g_noalloc_dev[NOALLOC_MAX_DEVICES];
std::mutex g_noalloc_mu;
PFN_cuTensorMapEncodeTiled_v12000 g_noalloc_encode = nullptr;

// Once per device, with that device current.
int noalloc_setup(int dev, NoallocDevice *out) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return ST_ARG;
  NoallocDevice &d = g_noalloc_dev[dev];
  if (!d.ready) {
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || ptr == nullptr) return ST_CUDA;
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return ST_CUDA;
    e = cudaFuncSetAttribute(zp_gemm_tc_kernel<1, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             TcLayout<1, 0>::SMEM);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(zp_gemm_tc_kernel<2, 0>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, TcLayout<2, 0>::SMEM);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(zp_gemm_tc_kernel<4, 0>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, TcLayout<4, 0>::SMEM);
    if (e != cudaSuccess) return ST_CUDA;
    if (!g_noalloc_encode) {
      void *fn = nullptr;
      cudaDriverEntryPointQueryResult q;
      e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
      if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) return ST_CUDA;
      g_noalloc_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    d.base = static_cast<uint8_t *>(ptr);
    d.num_sms = sms;
    d.ready = true;
  }
  *out = d;
  return ST_OK;
}

bool noalloc_map(CUtensorMap *tm, void *base, uint64_t d0, uint64_t d1, uint64_t d2,
                 uint64_t stride1, uint64_t stride2, uint32_t b0, uint32_t b1, uint32_t b2) {
  cuuint64_t dims[3] = {d0, d1, d2};
  cuuint64_t strides[2] = {stride1, stride2};
  cuuint32_t box[3] = {b0, b1, b2};
  cuuint32_t estr[3] = {1, 1, 1};
  return g_noalloc_encode(tm, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, base, dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int L>
int noalloc_launch(cudaStream_t s, const NoallocDevice &d, int M, int N, int K,
                   const Modulus &mod, uint32_t alpha, const uint32_t *A, size_t lda,
                   const uint32_t *B, size_t ldb, uint32_t beta, uint32_t *C, size_t ldc) {
  using Cfg = TcCfg<L, 0>;
  using Lay = TcLayout<L, 0>;
  uint32_t *err = reinterpret_cast<uint32_t *>(d.base);
  uint8_t *planes = d.base + NOALLOC_STATUS_BYTES;
  const int tiles = ((M + BM - 1) / BM) * ((N + Cfg::BN - 1) / Cfg::BN);
  uint32_t b = beta;
  for (int k0 = 0; k0 < K; k0 += ZP_KCHUNK) {
    const int kc = std::min(ZP_KCHUNK, K - k0);
    const int Kp = (kc + 15) & ~15;
    uint8_t *Al = planes;
    uint8_t *Bl = planes + (size_t)L * M * Kp;
    const size_t total = (size_t)M * ((kc + 3) / 4);
    int grid = (int)std::min<size_t>((total + 255) / 256, (size_t)d.num_sms * 16);
    split_rows_kernel<L><<<grid, 256, 0, s>>>(A + k0, lda, M, kc, Al, Kp);
    dim3 grid2((N + 31) / 32, (Kp + 63) / 64);
    split_cols_kernel<L><<<grid2, 256, 0, s>>>(B + (size_t)k0 * ldb, ldb, kc, N, Bl, Kp);
    CUtensorMap tmA, tmB;
    if (!noalloc_map(&tmA, Al, (uint64_t)kc, (uint64_t)M, L, (uint64_t)Kp, (uint64_t)M * Kp,
                     BK, BM, L) ||
        !noalloc_map(&tmB, Bl, (uint64_t)kc, (uint64_t)N, L, (uint64_t)Kp, (uint64_t)N * Kp,
                     BK, Cfg::BN, L))
      return ST_CUDA;
    zp_gemm_tc_kernel<L, 0><<<std::min(tiles, d.num_sms), tc_threads<L, 0>(), Lay::SMEM, s>>>(
        tmA, tmB, C, ldc, M, N, kc, mod, alpha, b, err);
    b = 1;
  }
  return cudaGetLastError() == cudaSuccess ? ST_OK : ST_CUDA;
}

}  // namespace

}  // namespace lela

extern "C" int lela_cuda_gemm_zp_u32_noalloc(size_t m, size_t n, size_t k, uint32_t p,
                                             uint32_t a, const uint32_t *A, size_t lda,
                                             const uint32_t *B, size_t ldb, uint32_t b,
                                             uint32_t *C, size_t ldc, void *stream) {
  using namespace lela;
  if (p < 2) return ST_ARG;
  if (m > (size_t)INT32_MAX || n > (size_t)INT32_MAX || k > (size_t)INT32_MAX) return ST_ARG;
  if (m == 0 || n == 0) return ST_OK;
  if (!C || (k && (!A || !B))) return ST_ARG;
  if (ldc < n || (k && (lda < k || ldb < n))) return ST_ARG;
  const int L = zp_limbs_for(p);
  const size_t kc = std::min<size_t>(k, (size_t)ZP_KCHUNK);
  const size_t need = (size_t)L * (m + n) * ((kc + 15) & ~(size_t)15);
  if (need > NOALLOC_PLANE_BYTES) return ST_ARG;  // beyond the fixed scratch

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return ST_CUDA;
  NoallocDevice d;
  int st = noalloc_setup(dev, &d);
  if (st) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const Modulus mod = make_modulus(p);
  a %= p;
  b %= p;
  if (cudaMemsetAsync(d.base, 0, sizeof(uint32_t), s) != cudaSuccess) return ST_CUDA;
  if (k == 0 || a == 0) {
    if (b != 1) {
      const size_t total = m * n;
      int grid = (int)std::min<size_t>((total + 255) / 256, (size_t)d.num_sms * 8);
      zp_scale_kernel<<<grid, 256, 0, s>>>(C, ldc, (int)m, (int)n, mod, b);
      if (cudaGetLastError() != cudaSuccess) return ST_CUDA;
    }
  } else {
    switch (L) {
      case 1: st = noalloc_launch<1>(s, d, (int)m, (int)n, (int)k, mod, a, A, lda, B, ldb, b, C, ldc); break;
      case 2: st = noalloc_launch<2>(s, d, (int)m, (int)n, (int)k, mod, a, A, lda, B, ldb, b, C, ldc); break;
      default: st = noalloc_launch<4>(s, d, (int)m, (int)n, (int)k, mod, a, A, lda, B, ldb, b, C, ldc); break;
    }
    if (st) return st;
  }
  uint32_t word = 0;
  if (cudaMemcpyAsync(&word, d.base, sizeof word, cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return ST_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return ST_CUDA;
  return (word & DEVERR_TIMEOUT) ? ST_TIMEOUT : ST_OK;
}

// ======================================================= GF(2) on tensor cores
namespace lela {

// C (packed GF(2) words) <- (beta ? C : 0) XOR (alpha ? A*B : 0) from 0/1
// byte planes Ab (M x Kp, K-major) and Bb (N x Kp, K-major) of K columns:
// the one-limb tensor-core kernel with the bit-packing epilogue.
template <int T>
static int gf2_tc_launch(Ctx *c, int M, int N, int K, const uint8_t *Ab, const uint8_t *Bb,
                         int Kp, uint32_t alpha, uint32_t beta, uint64_t *C, size_t ldc_words) {
  using Cfg = TcCfg<1, T>;
  using Lay = TcLayout<1, T>;
  if (int st = ctx_smem_attr(c, (const void *)zp_gemm_tc_kernel<1, 1, T>, Lay::SMEM,
                             "cudaFuncSetAttribute(gf2 tc)"))
    return st;
  CUtensorMap tmA, tmB;
  int st = encode_3d(c, &tmA, const_cast<uint8_t *>(Ab), (uint64_t)K, (uint64_t)M, 1,
                     (uint64_t)Kp, (uint64_t)M * Kp, BK, BM, 1);
  if (st) return st;
  st = encode_3d(c, &tmB, const_cast<uint8_t *>(Bb), (uint64_t)K, (uint64_t)N, 1, (uint64_t)Kp,
                 (uint64_t)N * Kp, BK, Cfg::BN, 1);
  if (st) return st;
  const int tiles = ((M + BM - 1) / BM) * ((N + Cfg::BN - 1) / Cfg::BN);
  int pi = prof_begin(c, "gf2_gemm_tc");
  zp_gemm_tc_kernel<1, 1, T><<<std::min(tiles, c->num_sms), tc_threads<1, T>(), Lay::SMEM,
                               c->stream>>>(tmA, tmB, C, ldc_words, M, N, K, make_modulus(2),
                                            alpha, beta, c->dstatus);
  prof_end(c, pi);
  ctx_launched(c);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "gf2 tc launch");
}

// 16 epilogue warps at short K (the echelon's block updates, K <= 512 bits:
// the 32768^2 echelon 62.0 -> 58.4 ms), 8 at long K (16384^3: 3.358 against
// 3.371 ms)
int gf2_gemm_tc_planes(Ctx *c, int M, int N, int K, const uint8_t *Ab, const uint8_t *Bb, int Kp,
                       uint32_t alpha, uint32_t beta, uint64_t *C, size_t ldc_words) {
  if (K <= 4096)
    return gf2_tc_launch<GF2_TC_T>(c, M, N, K, Ab, Bb, Kp, alpha, beta, C, ldc_words);
  return gf2_tc_launch<0>(c, M, N, K, Ab, Bb, Kp, alpha, beta, C, ldc_words);
}

}  // namespace lela
