// lela_b200/csrc/elem.cu -- matrices over Modular<uint8>, Modular<uint16>,
// Modular<float> and Modular<double> on the Modular<uint32> kernels.
//
// The reference's element types differ only in how a residue is stored
// (lela/ring/modular.h:115-330):
//  * uint8, uint16: the residue itself, 0 .. p-1 (ModularTraits<uint8>,
//    <uint16>: shift_up / shift_down keep [0, p));
//  * float, double: a symmetric representative, ModularTraits<float>::
//    reduce = fmod then shift_up (v < -p/2: v += p) then shift_down
//    (v > p/2: v -= p), so an odd p gives -(p-1)/2 .. (p-1)/2.
// Their gemm and trsm compute exact Z/p results (the float / double gemm of
// lela/blas/level3-modular.tcc:25-122 accumulates blocks of products that
// stay below 2^24 / 2^53, then reduces), so the result is a function of the
// residues alone.  Here each operand is converted to residues in a uint32
// scratch copy (one pass over HBM), the uint32 path computes, and the
// result is converted back: residue r is stored as r for the integer types
// and as r or r - p, whichever lies in [-p/2, p/2], for float and double.
// For an even p the residue p/2 has two representatives in the reference
// (+p/2 and -p/2, depending on the path that produced it); this stores +p/2.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "../../include/lela_cuda.h"
#include "common.cuh"
#include "context.h"
#include "elem.h"

namespace lela {

namespace {

template <class T>
struct Rep;
template <>
struct Rep<uint8_t> {
  static __device__ __forceinline__ uint32_t in(uint8_t x, uint32_t) { return x; }
  static __device__ __forceinline__ uint8_t out(uint32_t r, uint32_t) { return (uint8_t)r; }
};
template <>
struct Rep<uint16_t> {
  static __device__ __forceinline__ uint32_t in(uint16_t x, uint32_t) { return x; }
  static __device__ __forceinline__ uint16_t out(uint32_t r, uint32_t) { return (uint16_t)r; }
};
template <>
struct Rep<float> {
  // x is an integer of magnitude below 2^24, so the conversions are exact
  static __device__ __forceinline__ uint32_t in(float x, uint32_t p) {
    const int v = (int)x;
    return v < 0 ? (uint32_t)(v + (int)p) : (uint32_t)v;
  }
  static __device__ __forceinline__ float out(uint32_t r, uint32_t p) {
    return 2ull * r > p ? (float)((int)r - (int)p) : (float)r;
  }
};
template <>
struct Rep<double> {
  static __device__ __forceinline__ uint32_t in(double x, uint32_t p) {
    const long long v = (long long)x;
    return v < 0 ? (uint32_t)(v + (long long)p) : (uint32_t)v;
  }
  static __device__ __forceinline__ double out(uint32_t r, uint32_t p) {
    return 2ull * r > p ? (double)((long long)r - (long long)p) : (double)r;
  }
};

constexpr int CONV_THREADS = 256;
constexpr int CONV_COLS = 256;  // columns per CTA row pass

// One CTA per (row block, 256-column slice); consecutive threads take
// consecutive columns of a row, so loads and stores coalesce.
template <class T>
__global__ void __launch_bounds__(CONV_THREADS)
    to_u32_kernel(const T *__restrict__ src, size_t lds, uint32_t *__restrict__ dst, size_t ldd,
                  int rows, int cols, uint32_t p) {
  const int c = blockIdx.x * CONV_COLS + threadIdx.x;
  for (int r = blockIdx.y; r < rows; r += gridDim.y) {
    const T *s = src + (size_t)r * lds;
    uint32_t *d = dst + (size_t)r * ldd;
#pragma unroll
    for (int u = 0; u < CONV_COLS / CONV_THREADS; ++u) {
      const int cc = c + u * CONV_THREADS;
      if (cc < cols) d[cc] = Rep<T>::in(s[cc], p);
    }
  }
}

template <class T>
__global__ void __launch_bounds__(CONV_THREADS)
    from_u32_kernel(const uint32_t *__restrict__ src, size_t lds, T *__restrict__ dst, size_t ldd,
                    int rows, int cols, uint32_t p) {
  const int c = blockIdx.x * CONV_COLS + threadIdx.x;
  for (int r = blockIdx.y; r < rows; r += gridDim.y) {
    const uint32_t *s = src + (size_t)r * lds;
    T *d = dst + (size_t)r * ldd;
#pragma unroll
    for (int u = 0; u < CONV_COLS / CONV_THREADS; ++u) {
      const int cc = c + u * CONV_THREADS;
      if (cc < cols) d[cc] = Rep<T>::out(s[cc], p);
    }
  }
}

dim3 conv_grid(const Ctx *c, int rows, int cols) {
  const int gx = (cols + CONV_COLS - 1) / CONV_COLS;
  // enough CTAs for every SM several times over, capped by the rows
  const int want = std::max(1, (c->num_sms * 8 + gx - 1) / gx);
  return dim3(gx, std::min(rows, std::min(want, 65535)));
}

template <class T>
int to_u32_t(Ctx *c, const void *src, size_t lds, uint32_t *dst, size_t ldd, int rows, int cols,
             uint32_t p) {
  to_u32_kernel<T><<<conv_grid(c, rows, cols), CONV_THREADS, 0, c->stream>>>(
      static_cast<const T *>(src), lds, dst, ldd, rows, cols, p);
  ctx_launched(c);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "element conversion");
}

template <class T>
int from_u32_t(Ctx *c, const uint32_t *src, size_t lds, void *dst, size_t ldd, int rows, int cols,
               uint32_t p) {
  from_u32_kernel<T><<<conv_grid(c, rows, cols), CONV_THREADS, 0, c->stream>>>(
      src, lds, static_cast<T *>(dst), ldd, rows, cols, p);
  ctx_launched(c);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "element conversion");
}

}  // namespace

size_t elem_size(int elem) {
  switch (elem) {
    case LELA_CUDA_ELEM_U8: return 1;
    case LELA_CUDA_ELEM_U16: return 2;
    case LELA_CUDA_ELEM_U32: return 4;
    case LELA_CUDA_ELEM_F32: return 4;
    case LELA_CUDA_ELEM_F64: return 8;
    default: return 0;
  }
}

int elem_check_modulus(Ctx *c, int elem, uint32_t p) {
  if (elem_size(elem) == 0) return ctx_fail(c, ST_ARG, "unknown element type");
  if (p < 2) return ctx_fail(c, ST_ARG, "modulus must be at least 2");
  // the reference's ModularTraits<T>::valid_modulus (lela/ring/modular.h:
  // 121, 165, 211, 255, 297)
  switch (elem) {
    case LELA_CUDA_ELEM_U8:
      if (p >= (1u << 8)) return ctx_fail(c, ST_ARG, "Modular<uint8> needs p < 2^8");
      break;
    case LELA_CUDA_ELEM_U16:
      if (p >= (1u << 16)) return ctx_fail(c, ST_ARG, "Modular<uint16> needs p < 2^16");
      break;
    case LELA_CUDA_ELEM_F32:
      if (p >= 4096u) return ctx_fail(c, ST_ARG, "Modular<float> needs p < 4096");
      break;
    case LELA_CUDA_ELEM_F64:
      if (p >= (1u << 26)) return ctx_fail(c, ST_ARG, "Modular<double> needs p < 2^26");
      break;
    default: break;
  }
  return ST_OK;
}

int elem_to_u32(Ctx *c, int elem, const void *src, size_t lds, uint32_t *dst, size_t ldd,
                int rows, int cols, uint32_t p) {
  if (rows <= 0 || cols <= 0) return ST_OK;
  switch (elem) {
    case LELA_CUDA_ELEM_U8: return to_u32_t<uint8_t>(c, src, lds, dst, ldd, rows, cols, p);
    case LELA_CUDA_ELEM_U16: return to_u32_t<uint16_t>(c, src, lds, dst, ldd, rows, cols, p);
    case LELA_CUDA_ELEM_F32: return to_u32_t<float>(c, src, lds, dst, ldd, rows, cols, p);
    case LELA_CUDA_ELEM_F64: return to_u32_t<double>(c, src, lds, dst, ldd, rows, cols, p);
    default: return ctx_fail(c, ST_ARG, "unknown element type");
  }
}

int elem_from_u32(Ctx *c, int elem, const uint32_t *src, size_t lds, void *dst, size_t ldd,
                  int rows, int cols, uint32_t p) {
  if (rows <= 0 || cols <= 0) return ST_OK;
  switch (elem) {
    case LELA_CUDA_ELEM_U8: return from_u32_t<uint8_t>(c, src, lds, dst, ldd, rows, cols, p);
    case LELA_CUDA_ELEM_U16: return from_u32_t<uint16_t>(c, src, lds, dst, ldd, rows, cols, p);
    case LELA_CUDA_ELEM_F32: return from_u32_t<float>(c, src, lds, dst, ldd, rows, cols, p);
    case LELA_CUDA_ELEM_F64: return from_u32_t<double>(c, src, lds, dst, ldd, rows, cols, p);
    default: return ctx_fail(c, ST_ARG, "unknown element type");
  }
}

}  // namespace lela
