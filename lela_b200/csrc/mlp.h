// lela_b200/csrc/mlp.h -- the learned cost model's kernels (device).
#pragma once
#include <cstddef>

#include "context.h"

namespace lela {

constexpr int MLP_HIDDEN = 64;
constexpr int MLP_MAX_FEATURES = 16;

size_t mlp_param_count(int F);
int mlp_forward_dev(Ctx *c, const float *params, int F, const float *X, int n, float *out);
int mlp_grad_dev(Ctx *c, const float *params, int F, const float *X, const float *target, int n,
                 float *grad, float *loss);
int mlp_adam_dev(Ctx *c, float *params, const float *grad, float *m, float *v, int count, int step,
                 float lr);

}  // namespace lela
