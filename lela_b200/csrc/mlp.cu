// lela_b200/csrc/mlp.cu -- the learned cost model: a small fully connected
// network (F inputs -> 64 -> 64 -> 1, ReLU, FP32) that predicts log time of
// a kernel choice from block features.  Inference and training run here:
// forward, backward (mean squared error) and Adam, hand-written.
//
// Parameter layout (one float array): W1[F][64], b1[64], W2[64][64], b2[64],
// W3[64], b3.  No counterpart in the reference (LELA picks its modules at
// compile time); the choice it informs never changes a result.
#include <cstdint>

#include "common.cuh"
#include "context.h"
#include "mlp.h"

namespace lela {

constexpr int H = MLP_HIDDEN;

size_t mlp_param_count(int F) { return (size_t)F * H + H + H * H + H + H + 1; }

struct MlpView {
  const float *W1, *b1, *W2, *b2, *W3, *b3;
};

__device__ __forceinline__ MlpView mlp_view(const float *p, int F) {
  MlpView v;
  v.W1 = p;
  v.b1 = v.W1 + F * H;
  v.W2 = v.b1 + H;
  v.b2 = v.W2 + H * H;
  v.W3 = v.b2 + H;
  v.b3 = v.W3 + H;
  return v;
}

// One thread per sample; the parameters live in shared memory.
__global__ void __launch_bounds__(128)
    mlp_forward_kernel(const float *__restrict__ params, int F, const float *__restrict__ X,
                       int n, float *__restrict__ out) {
  extern __shared__ float sp[];
  const int np = (int)(F * H + H + H * H + H + H + 1);
  for (int e = threadIdx.x; e < np; e += blockDim.x) sp[e] = params[e];
  __syncthreads();
  const MlpView P = mlp_view(sp, F);
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const float *x = X + (size_t)s * F;
  float h1[H];
#pragma unroll
  for (int j = 0; j < H; ++j) h1[j] = P.b1[j];
  for (int i = 0; i < F; ++i) {
    const float xi = x[i];
#pragma unroll
    for (int j = 0; j < H; ++j) h1[j] = fmaf(xi, P.W1[i * H + j], h1[j]);
  }
#pragma unroll
  for (int j = 0; j < H; ++j) h1[j] = fmaxf(h1[j], 0.f);
  float y = P.b3[0];
  for (int j = 0; j < H; ++j) {
    float a = P.b2[j];
#pragma unroll
    for (int i = 0; i < H; ++i) a = fmaf(h1[i], P.W2[i * H + j], a);
    y = fmaf(fmaxf(a, 0.f), P.W3[j], y);
  }
  out[s] = y;
}

// Gradient of the mean squared error over n samples, accumulated into grad
// (zeroed by the caller); loss[0] += sum of squared errors / n.  One thread
// per sample; per-block partial gradients are summed in shared memory and
// added to global memory once per block.
__global__ void __launch_bounds__(64)
    mlp_grad_kernel(const float *__restrict__ params, int F, const float *__restrict__ X,
                    const float *__restrict__ target, int n, float *__restrict__ grad,
                    float *__restrict__ loss) {
  extern __shared__ float sh[];
  const int np = (int)(F * H + H + H * H + H + H + 1);
  float *sp = sh;        // parameters
  float *sg = sh + np;   // block gradient
  for (int e = threadIdx.x; e < np; e += blockDim.x) {
    sp[e] = params[e];
    sg[e] = 0.f;
  }
  __syncthreads();
  const MlpView P = mlp_view(sp, F);
  float *gW1 = sg, *gb1 = gW1 + F * H, *gW2 = gb1 + H, *gb2 = gW2 + H * H, *gW3 = gb2 + H,
        *gb3 = gW3 + H;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) {
    const float *x = X + (size_t)s * F;
    float h1[H], h2[H];
#pragma unroll
    for (int j = 0; j < H; ++j) h1[j] = P.b1[j];
    for (int i = 0; i < F; ++i) {
      const float xi = x[i];
#pragma unroll
      for (int j = 0; j < H; ++j) h1[j] = fmaf(xi, P.W1[i * H + j], h1[j]);
    }
#pragma unroll
    for (int j = 0; j < H; ++j) h1[j] = fmaxf(h1[j], 0.f);
    float y = P.b3[0];
#pragma unroll 4
    for (int j = 0; j < H; ++j) {
      float a = P.b2[j];
#pragma unroll
      for (int i = 0; i < H; ++i) a = fmaf(h1[i], P.W2[i * H + j], a);
      h2[j] = fmaxf(a, 0.f);
      y = fmaf(h2[j], P.W3[j], y);
    }
    const float err = y - target[s];
    atomicAdd(loss, err * err / (float)n);
    const float dy = 2.f * err / (float)n;
    atomicAdd(gb3, dy);
    float dh1[H];
#pragma unroll
    for (int i = 0; i < H; ++i) dh1[i] = 0.f;
#pragma unroll 4
    for (int j = 0; j < H; ++j) {
      atomicAdd(&gW3[j], dy * h2[j]);
      const float dz2 = (h2[j] > 0.f) ? dy * P.W3[j] : 0.f;
      if (dz2 != 0.f) {
        atomicAdd(&gb2[j], dz2);
#pragma unroll
        for (int i = 0; i < H; ++i) {
          atomicAdd(&gW2[i * H + j], h1[i] * dz2);
          dh1[i] = fmaf(P.W2[i * H + j], dz2, dh1[i]);
        }
      }
    }
#pragma unroll
    for (int i = 0; i < H; ++i) {
      const float dz1 = (h1[i] > 0.f) ? dh1[i] : 0.f;
      if (dz1 != 0.f) {
        atomicAdd(&gb1[i], dz1);
        for (int f = 0; f < F; ++f) atomicAdd(&gW1[f * H + i], x[f] * dz1);
      }
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < np; e += blockDim.x)
    if (sg[e] != 0.f) atomicAdd(&grad[e], sg[e]);
}

// Adam (Kingma & Ba 2015) on the flat parameter vector.
__global__ void mlp_adam_kernel(float *__restrict__ params, const float *__restrict__ grad,
                                float *__restrict__ m, float *__restrict__ v, int count, float lr,
                                float b1, float b2, float eps, float c1, float c2) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < count; e += gridDim.x * blockDim.x) {
    const float g = grad[e];
    const float mm = b1 * m[e] + (1.f - b1) * g;
    const float vv = b2 * v[e] + (1.f - b2) * g * g;
    m[e] = mm;
    v[e] = vv;
    params[e] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
  }
}

int mlp_forward_dev(Ctx *c, const float *params, int F, const float *X, int n, float *out) {
  if (F < 1 || F > MLP_MAX_FEATURES || n < 0) return ctx_fail(c, ST_ARG, "mlp: bad shape");
  if (n == 0) return ST_OK;
  const size_t smem = mlp_param_count(F) * sizeof(float);
  int pi = prof_begin(c, "mlp_forward");
  mlp_forward_kernel<<<(n + 127) / 128, 128, smem, c->stream>>>(params, F, X, n, out);
  prof_end(c, pi);
  ctx_launched(c);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "mlp_forward launch");
}

int mlp_grad_dev(Ctx *c, const float *params, int F, const float *X, const float *target, int n,
                 float *grad, float *loss) {
  if (F < 1 || F > MLP_MAX_FEATURES || n < 0) return ctx_fail(c, ST_ARG, "mlp: bad shape");
  const size_t np = mlp_param_count(F);
  cudaError_t e = cudaMemsetAsync(grad, 0, np * sizeof(float), c->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(loss, 0, sizeof(float), c->stream);
  if (e != cudaSuccess) return ctx_cuda(c, e, "mlp: clear");
  if (n == 0) return ST_OK;
  // at most 2 * 5313 floats = 42.5 KB for 16 features: under the default
  // 48 KB of dynamic shared memory
  const size_t smem = 2 * np * sizeof(float);
  int pi = prof_begin(c, "mlp_grad");
  mlp_grad_kernel<<<(n + 63) / 64, 64, smem, c->stream>>>(params, F, X, target, n, grad, loss);
  prof_end(c, pi);
  ctx_launched(c);
  e = cudaGetLastError();
  return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "mlp_grad launch");
}

int mlp_adam_dev(Ctx *c, float *params, const float *grad, float *m, float *v, int count, int step,
                 float lr) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  float c1 = 1.f, c2 = 1.f;
  for (int i = 0; i < step; ++i) {
    c1 *= b1;
    c2 *= b2;
  }
  c1 = 1.f - c1;
  c2 = 1.f - c2;
  mlp_adam_kernel<<<(count + 255) / 256, 256, 0, c->stream>>>(params, grad, m, v, count, lr, b1, b2,
                                                              eps, c1, c2);
  ctx_launched(c);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "mlp_adam launch");
}

}  // namespace lela
