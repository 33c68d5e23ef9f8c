// lela_b200/csrc/batch.h -- batched dense echelon blocks (device).
#pragma once
#include <cstdint>

#include "context.h"

namespace lela {

// One dense block of a batch (device pointer, row stride in elements).
struct SmallItem {
  uint32_t *A;
  uint64_t ld;
  int m, n;
  uint32_t p;
  uint32_t pad;
};

// True when an m x n block fits the one-CTA shared-memory kernel.
bool small_echelon_fits(int m, int n);

// Kernel attributes; call once before capturing a launch into a graph.
int echelon_small_batch_prepare(Ctx *c);

// One persistent launch over `count` small blocks (device item array);
// rank/det/status per block in device arrays.
int echelon_small_batch_dev(Ctx *c, int count, const SmallItem *d_items, unsigned *d_next,
                            uint64_t *d_rank, uint32_t *d_det, uint32_t *d_status);

}  // namespace lela
