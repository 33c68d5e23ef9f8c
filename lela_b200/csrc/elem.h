// lela_b200/csrc/elem.h -- residues of the other Modular<T> element types
// (uint8, uint16, float, double) to and from uint32 device matrices.
#pragma once
#include <cstddef>
#include <cstdint>

#include "context.h"

namespace lela {

// Bytes of one element of type elem (LELA_CUDA_ELEM_*); 0 for an unknown type.
size_t elem_size(int elem);
// ST_OK when p is a valid modulus of Modular<T> for elem, else ST_ARG.
int elem_check_modulus(Ctx *c, int elem, uint32_t p);
// rows x cols device matrices, asynchronous on the handle's stream: src of
// type elem (row stride lds elements) to residues in dst (row stride ldd),
// and back.  elem must not be LELA_CUDA_ELEM_U32.
int elem_to_u32(Ctx *c, int elem, const void *src, size_t lds, uint32_t *dst, size_t ldd,
                int rows, int cols, uint32_t p);
int elem_from_u32(Ctx *c, int elem, const uint32_t *src, size_t lds, void *dst, size_t ldd,
                  int rows, int cols, uint32_t p);

}  // namespace lela
