// lela_b200/csrc/api.cu -- the C ABI (include/lela_cuda.h): handle
// management and the host-pointer / device-pointer entry points.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <mutex>
#include <cstdio>
#include <cstring>
#include <new>
#include <thread>
#include <vector>

#include "../../include/lela_cuda.h"
#include "batch.h"
#include "common.cuh"
#include "context.h"
#include "echelon.h"
#include "elem.h"
#include "fl.h"
#include "gf2.h"
#include "mlp.h"
#include "tri.h"
#include "zp_gemm.h"

struct lela_cuda_ctx {
  lela::Ctx c;
  // Worker handles of the batched Faugere-Lachartre entry point (each with
  // its own stream and buffers), created on first use.
  std::vector<lela_cuda_ctx *> workers;
};

namespace lela {

int ctx_fail(Ctx *c, int code, const char *msg) {
  c->last_error = msg ? msg : "";
  return code;
}

int ctx_cuda(Ctx *c, cudaError_t e, const char *what) {
  char buf[256];
  snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
  c->last_error = buf;
  if (e == cudaErrorMemoryAllocation) return ST_NOMEM;
  return ST_CUDA;
}

static int grow(Ctx *c, void **buf, size_t *have, size_t bytes, const char *what) {
  if (bytes <= *have && *buf) return ST_OK;
  if (*buf) {
    // The old buffer may still be in use by queued work.
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return ctx_cuda(c, e, "cudaStreamSynchronize");
    cudaFree(*buf);
    *buf = nullptr;
    *have = 0;
  }
  size_t want = std::max(bytes, (size_t)1 << 20);
  cudaError_t e = cudaMalloc(buf, want);
  if (e != cudaSuccess) {
    *buf = nullptr;
    return ctx_cuda(c, e, what);
  }
  *have = want;
  return ST_OK;
}

int ctx_workspace(Ctx *c, size_t bytes, void **out) {
  int st = grow(c, &c->ws, &c->ws_bytes, bytes, "cudaMalloc(workspace)");
  *out = c->ws;
  return st;
}

int ctx_workspace2(Ctx *c, size_t bytes, void **out) {
  int st = grow(c, &c->ws2, &c->ws2_bytes, bytes, "cudaMalloc(workspace2)");
  *out = c->ws2;
  return st;
}

int ctx_buffer(Ctx *c, int slot, size_t bytes, void **out) {
  int st = grow(c, &c->buf[slot], &c->buf_bytes[slot], bytes, "cudaMalloc(buffer)");
  *out = c->buf[slot];
  return st;
}

int ctx_stage(Ctx *c, int slot, size_t bytes, void **out) {
  int st = grow(c, &c->stage[slot], &c->stage_bytes[slot], bytes, "cudaMalloc(staging)");
  *out = c->stage[slot];
  return st;
}

int ctx_pipe(Ctx *c) {
  if (c->pipe_ev[2 * PIPE_MAX_BLOCKS + 2]) return ST_OK;  // the last one made
  cudaError_t e = cudaSuccess;
  if (!c->copy_in) e = cudaStreamCreateWithFlags(&c->copy_in, cudaStreamNonBlocking);
  if (e == cudaSuccess && !c->copy_out)
    e = cudaStreamCreateWithFlags(&c->copy_out, cudaStreamNonBlocking);
  for (int i = 0; e == cudaSuccess && i < 2 * PIPE_MAX_BLOCKS + 3; ++i)
    if (!c->pipe_ev[i]) e = cudaEventCreateWithFlags(&c->pipe_ev[i], cudaEventDisableTiming);
  return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "copy streams");
}

int ctx_clear_status(Ctx *c) {
  cudaError_t e = cudaMemsetAsync(c->dstatus, 0, 16 * sizeof(uint32_t), c->stream);
  return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "cudaMemsetAsync(status)");
}

int ctx_check_status(Ctx *c, const char *what) {
  cudaError_t e = cudaMemcpyAsync(c->hstatus, c->dstatus, 16 * sizeof(uint32_t),
                                  cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return ctx_cuda(c, e, what);
  if (c->hstatus[0] & DEVERR_TIMEOUT) {
    char buf[160];
    snprintf(buf, sizeof buf, "%s: a device-side wait exceeded its limit", what);
    return ctx_fail(c, ST_TIMEOUT, buf);
  }
  return ST_OK;
}

int ctx_panel_map(Ctx *c, void **host, void **dev) {
  if (!c->panel_map) {
    cudaError_t e = cudaHostAlloc(&c->panel_map, PANEL_MAP_BYTES, cudaHostAllocMapped);
    if (e == cudaSuccess) e = cudaHostGetDevicePointer(&c->panel_map_dev, c->panel_map, 0);
    if (e != cudaSuccess) {
      if (c->panel_map) cudaFreeHost(c->panel_map);
      c->panel_map = c->panel_map_dev = nullptr;
      return ctx_cuda(c, e, "mapped panel result");
    }
    *reinterpret_cast<volatile uint32_t *>(static_cast<char *>(c->panel_map) + PANEL_FLAG_OFF) = 0u;
    c->panel_seq = 0;
  }
  *host = c->panel_map;
  *dev = c->panel_map_dev;
  return ST_OK;
}

int ctx_wait_flag(Ctx *c, volatile uint32_t *flag, uint32_t seq, const char *what) {
  const auto t0 = std::chrono::steady_clock::now();
  for (uint64_t spins = 1; *flag != seq; ++spins) {
    if ((spins & 1023) == 0) {
      const cudaError_t e = cudaStreamQuery(c->stream);
      if (e != cudaSuccess && e != cudaErrorNotReady) return ctx_cuda(c, e, what);
      if (e == cudaSuccess && *flag != seq) return ctx_fail(c, ST_CUDA, "panel result missing");
      const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      if (s > 60.0) return ctx_fail(c, ST_TIMEOUT, "panel search did not finish");
      std::this_thread::yield();
    }
  }
  std::atomic_thread_fence(std::memory_order_acquire);
  return ST_OK;
}

int ctx_smem_attr(Ctx *c, const void *kernel, int bytes, const char *what) {
  static std::mutex mu;
  static std::vector<std::pair<int, const void *>> done;
  std::lock_guard<std::mutex> lock(mu);
  for (const auto &d : done)
    if (d.first == c->device && d.second == kernel) return ST_OK;
  DeviceScope scope(c);
  const cudaError_t e =
      cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return ctx_cuda(c, e, what);
  done.emplace_back(c->device, kernel);
  return ST_OK;
}

static cudaEvent_t pool_event(Ctx *c) {
  if (!c->event_pool.empty()) {
    cudaEvent_t e = c->event_pool.back();
    c->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

int prof_begin(Ctx *c, const char *name) {
  if (!c->profile) return -1;
  Ctx::ProfRec r;
  r.name = name;
  r.a = pool_event(c);
  r.b = pool_event(c);
  cudaEventRecord(r.a, c->stream);
  c->prof.push_back(r);
  return (int)c->prof.size() - 1;
}

void prof_end(Ctx *c, int idx) {
  if (idx < 0 || idx >= (int)c->prof.size()) return;
  cudaEventRecord(c->prof[idx].b, c->stream);
}

}  // namespace lela

using namespace lela;

extern "C" {

int lela_cuda_create(lela_cuda_ctx **out, int device) {
  if (!out) return ST_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return ST_CUDA;
  lela_cuda_ctx *h = new (std::nothrow) lela_cuda_ctx;
  if (!h) return ST_NOMEM;
  Ctx *c = &h->c;
  c->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
  int major = 0;
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
  if (e == cudaSuccess && major != 10) {
    delete h;
    return ST_UNSUPPORTED;
  }
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) c->own_stream = true;
  if (e == cudaSuccess) e = cudaMalloc(&c->dstatus, 16 * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMemset(c->dstatus, 0, 16 * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMallocHost(&c->hstatus, 16 * sizeof(uint32_t));
  if (e == cudaSuccess) {
    cudaDriverEntryPointQueryResult q;
    e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &c->encode_tiled, cudaEnableDefault, &q);
    if (e == cudaSuccess && q != cudaDriverEntryPointSuccess) c->encode_tiled = nullptr;
  }
  if (e != cudaSuccess) {
    lela_cuda_destroy(h);
    return e == cudaErrorMemoryAllocation ? ST_NOMEM : ST_CUDA;
  }
  *out = h;
  return ST_OK;
}

int lela_cuda_destroy(lela_cuda_ctx *h) {
  if (!h) return ST_OK;
  for (lela_cuda_ctx *w : h->workers) lela_cuda_destroy(w);
  h->workers.clear();
  Ctx *c = &h->c;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->ws) cudaFree(c->ws);
  if (c->ws2) cudaFree(c->ws2);
  for (int i = 0; i < 4; ++i)
    if (c->stage[i]) cudaFree(c->stage[i]);
  for (int i = 0; i < 32; ++i)
    if (c->buf[i]) cudaFree(c->buf[i]);
  if (c->batch_exec) cudaGraphExecDestroy(c->batch_exec);
  if (c->panel_map) cudaFreeHost(c->panel_map);
  for (auto e : c->pipe_ev)
    if (e) cudaEventDestroy(e);
  if (c->copy_in) cudaStreamDestroy(c->copy_in);
  if (c->copy_out) cudaStreamDestroy(c->copy_out);
  if (c->dstatus) cudaFree(c->dstatus);
  if (c->hstatus) cudaFreeHost(c->hstatus);
  for (auto &r : c->prof) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  for (auto e : c->event_pool) cudaEventDestroy(e);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  delete h;
  return ST_OK;
}

int lela_cuda_set_stream(lela_cuda_ctx *h, void *stream) {
  if (!h) return ST_ARG;
  Ctx *c = &h->c;
  cudaStreamSynchronize(c->stream);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  c->own_stream = false;
  c->stream = static_cast<cudaStream_t>(stream);
  if (!stream) {
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
      return ST_CUDA;
    c->own_stream = true;
  }
  return ST_OK;
}

void *lela_cuda_get_stream(lela_cuda_ctx *h) { return h ? (void *)h->c.stream : nullptr; }

int lela_cuda_synchronize(lela_cuda_ctx *h) {
  if (!h) return ST_ARG;
  Ctx *c = &h->c;
  int st = ctx_check_status(c, "synchronize");
  if (st == ST_OK) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return ctx_cuda(c, e, "synchronize");
  }
  if (st != ST_OK) ctx_clear_status(c);
  return st;
}

int lela_cuda_set_gemm_kernel(lela_cuda_ctx *h, int kernel) {
  if (!h || kernel < GEMM_AUTO || kernel > GEMM_SMALLK) return ST_ARG;
  h->c.gemm_kernel = kernel;
  return ST_OK;
}

int lela_cuda_set_gemm_tile(lela_cuda_ctx *h, int tile) {
  if (!h || tile < GEMM_TILE_AUTO || tile > GEMM_TILE_DOUBLE) return ST_ARG;
  h->c.gemm_tile = tile;
  return ST_OK;
}

const char *lela_cuda_status_string(int s) {
  switch (s) {
    case ST_OK: return "ok";
    case ST_ARG: return "invalid argument";
    case ST_CUDA: return "CUDA error";
    case ST_NOMEM: return "out of device memory";
    case ST_DIAG: return "diagonal entry not invertible";
    case ST_WRONG_FORM: return "wrong matrix form";
    case ST_PIVOT: return "pivot not invertible in the ring";
    case ST_TIMEOUT: return "device-side wait timed out";
    case ST_UNSUPPORTED: return "unsupported";
    case ST_CAPACITY: return "output capacity too small";
    default: return "unknown status";
  }
}

const char *lela_cuda_last_error(lela_cuda_ctx *h) { return h ? h->c.last_error.c_str() : ""; }

int lela_cuda_num_sms(lela_cuda_ctx *h) { return h ? h->c.num_sms : 0; }

uint64_t lela_cuda_launch_count(lela_cuda_ctx *h) { return h ? h->c.launches : 0; }

int lela_cuda_profile_enable(lela_cuda_ctx *h, int on) {
  if (!h) return ST_ARG;
  h->c.profile = on != 0;
  return ST_OK;
}

int lela_cuda_profile_read(lela_cuda_ctx *h, const char *kernel, double *total_ms,
                           uint64_t *launches) {
  if (!h || !kernel || !total_ms || !launches) return ST_ARG;
  Ctx *c = &h->c;
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return ctx_cuda(c, e, "profile_read");
  double ms = 0;
  uint64_t n = 0;
  std::vector<Ctx::ProfRec> keep;
  for (auto &r : c->prof) {
    if (strcmp(r.name, kernel) == 0) {
      float t = 0;
      if (cudaEventElapsedTime(&t, r.a, r.b) == cudaSuccess) {
        ms += t;
        ++n;
      }
      c->event_pool.push_back(r.a);
      c->event_pool.push_back(r.b);
    } else {
      keep.push_back(r);
    }
  }
  c->prof.swap(keep);
  *total_ms = ms;
  *launches = n;
  return ST_OK;
}

int lela_cuda_profile_reset(lela_cuda_ctx *h) {
  if (!h) return ST_ARG;
  Ctx *c = &h->c;
  cudaStreamSynchronize(c->stream);
  for (auto &r : c->prof) {
    c->event_pool.push_back(r.a);
    c->event_pool.push_back(r.b);
  }
  c->prof.clear();
  return ST_OK;
}

int lela_cuda_gemm_zp_u32_dev(lela_cuda_ctx *h, size_t m, size_t n, size_t k, uint32_t p,
                              uint32_t a, const uint32_t *A, size_t lda, const uint32_t *B,
                              size_t ldb, uint32_t b, uint32_t *C, size_t ldc) {
  if (!h) return ST_ARG;
  Ctx *c = &h->c;
  DeviceScope ds(c);
  if (m > (size_t)INT32_MAX || n > (size_t)INT32_MAX || k > (size_t)INT32_MAX)
    return ctx_fail(c, ST_ARG, "dimension too large");
  if ((m && n && !C) || (m && k && n && (!A || !B))) return ctx_fail(c, ST_ARG, "null pointer");
  return zp_gemm_dev(c, GEMM_AUTO, (int)m, (int)n, (int)k, p, a, A, lda, B, ldb, b, C, ldc,
                     nullptr);
}

// Copy a host matrix with row stride ld into a dense device buffer
// (row stride = cols) and back.
static int h2d_matrix(Ctx *c, void *dst, const void *src, size_t rows, size_t cols, size_t ld,
                      size_t esz) {
  if (!rows || !cols) return ST_OK;
  cudaError_t e = cudaMemcpy2DAsync(dst, cols * esz, src, ld * esz, cols * esz, rows,
                                    cudaMemcpyHostToDevice, c->stream);
  return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "host->device copy");
}

static int d2h_matrix(Ctx *c, void *dst, const void *src, size_t rows, size_t cols, size_t ld,
                      size_t esz) {
  if (!rows || !cols) return ST_OK;
  cudaError_t e = cudaMemcpy2DAsync(dst, ld * esz, src, cols * esz, cols * esz, rows,
                                    cudaMemcpyDeviceToHost, c->stream);
  return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "device->host copy");
}

int lela_cuda_gemm_zp_u32(lela_cuda_ctx *h, size_t m, size_t n, size_t k, uint32_t p, uint32_t a,
                          const uint32_t *A, size_t lda, const uint32_t *B, size_t ldb, uint32_t b,
                          uint32_t *C, size_t ldc) {
  if (!h) return ST_ARG;
  Ctx *c = &h->c;
  if (m > (size_t)INT32_MAX || n > (size_t)INT32_MAX || k > (size_t)INT32_MAX)
    return ctx_fail(c, ST_ARG, "dimension too large");
  if (p < 2) return ctx_fail(c, ST_ARG, "modulus must be at least 2");
  if (m == 0 || n == 0) return ST_OK;
  if (!C || (k && (!A || !B))) return ctx_fail(c, ST_ARG, "null pointer");
  if (ldc < n || (k && (lda < k || ldb < n)))
    return ctx_fail(c, ST_ARG, "leading dimension smaller than the row length");
  DeviceScope ds(c);
  void *dA = nullptr, *dB = nullptr, *dC = nullptr;
  int st = ST_OK;
  if (!st && k) st = ctx_stage(c, 0, m * k * 4, &dA);
  if (!st && k) st = ctx_stage(c, 1, k * n * 4, &dB);
  if (!st) st = ctx_stage(c, 2, m * n * 4, &dC);
  if (!st) st = ctx_clear_status(c);
  if (!st && zp_gemm_pipelined(c, (int)m, (int)n, (int)k, p, a)) {
    // large tensor-core products: copies overlapped with the product
    st = zp_gemm_host_rows(c, (int)m, (int)n, (int)k, p, a, A, lda, B, ldb, b, C, ldc,
                           (uint32_t *)dA, (uint32_t *)dB, (uint32_t *)dC);
    if (!st) st = ctx_check_status(c, "gemm_zp_u32");
    return st;
  }
  if (!st && k) st = h2d_matrix(c, dA, A, m, k, lda, 4);
  if (!st && k) st = h2d_matrix(c, dB, B, k, n, ldb, 4);
  // With b = 0 mod p the kernels never read C.
  if (!st && (b % p) != 0) st = h2d_matrix(c, dC, C, m, n, ldc, 4);
  if (!st)
    st = zp_gemm_dev(c, GEMM_AUTO, (int)m, (int)n, (int)k, p, a, (const uint32_t *)dA, k,
                     (const uint32_t *)dB, n, b, (uint32_t *)dC, n, nullptr);
  if (!st) st = d2h_matrix(c, C, dC, m, n, ldc, 4);
  if (!st) st = ctx_check_status(c, "gemm_zp_u32");
  return st;
}

int lela_cuda_set_gf2_kernel(lela_cuda_ctx *h, int kernel) {
  if (!h || kernel < GF2_AUTO || kernel > GF2_M4RM) return ST_ARG;
  h->c.gf2_kernel = kernel;
  return ST_OK;
}

int lela_cuda_set_trsm_kernel(lela_cuda_ctx *h, int kernel) {
  if (!h || kernel < TRSM_AUTO || kernel > TRSM_INVERSE) return ST_ARG;
  h->c.trsm_kernel = kernel;
  return ST_OK;
}

int lela_cuda_gemm_gf2_dev(lela_cuda_ctx *h, size_t m, size_t n, size_t k, int a,
                           const uint64_t *A, size_t lda, const uint64_t *B, size_t ldb, int b,
                           uint64_t *C, size_t ldc) {
  if (!h) return ST_ARG;
  Ctx *c = &h->c;
  DeviceScope ds(c);
  if (m > (size_t)INT32_MAX || n > (size_t)INT32_MAX || k > (size_t)INT32_MAX)
    return ctx_fail(c, ST_ARG, "dimension too large");
  if ((m && n && !C) || (m && n && k && (!A || !B))) return ctx_fail(c, ST_ARG, "null pointer");
  return gf2_gemm_dev(c, GF2_AUTO, (int)m, (int)n, (int)k, a, A, lda, B, ldb, b, C, ldc);
}

int lela_cuda_gemm_gf2(lela_cuda_ctx *h, size_t m, size_t n, size_t k, int a, const uint64_t *A,
                       size_t lda, const uint64_t *B, size_t ldb, int b, uint64_t *C, size_t ldc) {
  if (!h) return ST_ARG;
  Ctx *c = &h->c;
  if (m > (size_t)INT32_MAX || n > (size_t)INT32_MAX || k > (size_t)INT32_MAX)
    return ctx_fail(c, ST_ARG, "dimension too large");
  if (m == 0 || n == 0) return ST_OK;
  const size_t nw = (n + 63) / 64, kw = (k + 63) / 64;
  if (!C || (k && (!A || !B))) return ctx_fail(c, ST_ARG, "null pointer");
  if (ldc < nw || (k && (lda < kw || ldb < nw)))
    return ctx_fail(c, ST_ARG, "leading dimension smaller than the row length");
  DeviceScope ds(c);
  void *dA = nullptr, *dB = nullptr, *dC = nullptr;
  int st = ST_OK;
  if (k) st = ctx_stage(c, 0, m * kw * 8, &dA);
  if (!st && k) st = ctx_stage(c, 1, k * nw * 8, &dB);
  if (!st) st = ctx_stage(c, 2, m * nw * 8, &dC);
  if (!st) st = ctx_clear_status(c);
  if (!st && gf2_gemm_pipelined(c, (int)m, (int)n, (int)k, a)) {
    // large tensor-core products: copies overlapped with the product
    st = gf2_gemm_host_rows(c, (int)m, (int)n, (int)k, A, lda, B, ldb, b, C, ldc,
                            (uint64_t *)dA, (uint64_t *)dB, (uint64_t *)dC);
    if (!st) st = ctx_check_status(c, "gemm_gf2");
    return st;
  }
  if (!st && k) st = h2d_matrix(c, dA, A, m, kw, lda, 8);
  if (!st && k) st = h2d_matrix(c, dB, B, k, nw, ldb, 8);
  // C is read when b = 1, and for the bits past column n of each row's last
  // word, which the kernels leave as they were
  if (!st && ((b & 1) || (n & 63))) st = h2d_matrix(c, dC, C, m, nw, ldc, 8);
  if (!st)
    st = gf2_gemm_dev(c, GF2_AUTO, (int)m, (int)n, (int)k, a, (const uint64_t *)dA, kw,
                      (const uint64_t *)dB, nw, b, (uint64_t *)dC, nw);
  if (!st) st = d2h_matrix(c, C, dC, m, nw, ldc, 8);
  if (!st) st = ctx_check_status(c, "gemm_gf2");
  return st;
}

int lela_cuda_echelon_gf2_dev(lela_cuda_ctx *h, size_t m, size_t n, uint64_t *A, size_t lda,
                              size_t *rank) {
  if (!h || !rank) return ST_ARG;
  Ctx *c = &h->c;
  DeviceScope ds(c);
  if (m > (size_t)INT32_MAX || n > (size_t)INT32_MAX) return ctx_fail(c, ST_ARG, "dimension too large");
  if (m && n && !A) return ctx_fail(c, ST_ARG, "null pointer");
  int st = gf2_echelon_dev(c, (int)m, (int)n, A, lda, rank);
  if (!st) st = ctx_check_status(c, "echelon_gf2");
  return st;
}

int lela_cuda_echelon_gf2(lela_cuda_ctx *h, size_t m, size_t n, uint64_t *A, size_t lda,
                          size_t *rank) {
  if (!h || !rank) return ST_ARG;
  Ctx *c = &h->c;
  if (m > (size_t)INT32_MAX || n > (size_t)INT32_MAX) return ctx_fail(c, ST_ARG, "dimension too large");
  if (m == 0 || n == 0) {
    *rank = 0;
    return ST_OK;
  }
  const size_t nw = (n + 63) / 64;
  if (!A) return ctx_fail(c, ST_ARG, "null pointer");
  if (lda < nw) return ctx_fail(c, ST_ARG, "leading dimension smaller than the row length");
  DeviceScope ds(c);
  void *dA = nullptr;
  int st = ctx_stage(c, 0, m * nw * 8, &dA);
  if (!st) st = ctx_clear_status(c);
  if (!st) st = h2d_matrix(c, dA, A, m, nw, lda, 8);
  if (!st) st = gf2_echelon_dev(c, (int)m, (int)n, (uint64_t *)dA, nw, rank);
  if (!st) st = d2h_matrix(c, A, dA, m, nw, lda, 8);
  if (!st) st = ctx_check_status(c, "echelon_gf2");
  return st;
}

int lela_cuda_echelon_zp_u32_batch(lela_cuda_ctx *h, size_t count, uint32_t *const *A,
                                   const size_t *lda, const size_t *m, const size_t *n,
                                   const uint32_t *p, const int *kernel, size_t *rank,
                                   uint32_t *det, int *status) {
  if (!h) return ST_ARG;
  Ctx *c = &h->c;
  if (count == 0) return ST_OK;
  if (!A || !lda || !m || !n || !p || !rank || !det || !status)
    return ctx_fail(c, ST_ARG, "null pointer");
  DeviceScope ds(c);
  std::vector<SmallItem> small;
  std::vector<size_t> small_idx, big_idx;
  for (size_t i = 0; i < count; ++i) {
    if (m[i] > (size_t)INT32_MAX || n[i] > (size_t)INT32_MAX || p[i] < 2 || (m[i] && n[i] && (!A[i] || lda[i] < n[i])))
      return ctx_fail(c, ST_ARG, "bad batch item");
    const int k = kernel ? kernel[i] : 0;
    const bool fits = small_echelon_fits((int)m[i], (int)n[i]);
    if (k == 1 && !fits) return ctx_fail(c, ST_ARG, "batch item too large for the small kernel");
    if ((k == 0 || k == 1) && fits && m[i] && n[i]) {
      SmallItem it{A[i], (uint64_t)lda[i], (int)m[i], (int)n[i], p[i], 0};
      small.push_back(it);
      small_idx.push_back(i);
    } else {
      big_idx.push_back(i);
    }
  }
  int st = ctx_clear_status(c);
  if (st) return st;
  // big items run on worker handles (own streams) while the small ones run
  // on this handle's stream; the caller's queued work must be done first
  const int nworkers = (int)std::min<size_t>(big_idx.size(), 8);
  if (nworkers > 1) {
    while ((int)h->workers.size() < nworkers) {
      lela_cuda_ctx *w = nullptr;
      if ((st = lela_cuda_create(&w, c->device))) return ctx_fail(c, st, "batch: worker handle");
      h->workers.push_back(w);
    }
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return ctx_cuda(c, e, "batch: synchronize");
  }
  std::vector<uint64_t> hr(small.size());
  std::vector<uint32_t> hd(small.size()), hs(small.size());
  if (!small.empty()) {
    const size_t ns = small.size();
    void *buf = nullptr;
    const size_t bytes = ns * (sizeof(SmallItem) + 8 + 4 + 4) + 256;
    if ((st = ctx_buffer(c, BUF_BATCH, bytes, &buf))) return st;
    SmallItem *d_items = (SmallItem *)buf;
    uint64_t *d_rank = (uint64_t *)(d_items + ns);
    uint32_t *d_det = (uint32_t *)(d_rank + ns);
    uint32_t *d_status = d_det + ns;
    unsigned *d_next = (unsigned *)(d_status + ns);
    cudaError_t e = cudaMemcpyAsync(d_items, small.data(), ns * sizeof(SmallItem),
                                    cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return ctx_cuda(c, e, "batch: items");
    // one persistent launch, captured in a CUDA graph; the instantiated graph
    // is kept in the handle and replayed by later calls with the same item
    // count and buffer (the item array is refreshed above, outside the graph)
    if (!(c->batch_exec && c->batch_ns == ns && c->batch_buf == buf)) {
      if (c->batch_exec) cudaGraphExecDestroy(c->batch_exec);
      c->batch_exec = nullptr;
      cudaGraph_t graph = nullptr;
      if ((st = echelon_small_batch_prepare(c))) return st;
      const bool was_profiling = c->profile;
      c->profile = false;  // no event records inside the capture
      e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) {
        c->profile = was_profiling;
        return ctx_cuda(c, e, "batch: begin capture");
      }
      st = echelon_small_batch_dev(c, (int)ns, d_items, d_next, d_rank, d_det, d_status);
      e = cudaStreamEndCapture(c->stream, &graph);
      c->profile = was_profiling;
      if (st) {
        if (graph) cudaGraphDestroy(graph);
        return st;
      }
      cudaGraphExec_t exec = nullptr;
      if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
      if (graph) cudaGraphDestroy(graph);
      if (e != cudaSuccess) return ctx_cuda(c, e, "batch: graph");
      c->batch_exec = exec;
      c->batch_ns = ns;
      c->batch_buf = buf;
    }
    int pi = prof_begin(c, "echelon_small_batch_graph");
    e = cudaGraphLaunch(c->batch_exec, c->stream);
    prof_end(c, pi);
    if (e != cudaSuccess) return ctx_cuda(c, e, "batch: graph launch");
    c->batch_rank = d_rank;
    c->batch_det = d_det;
    c->batch_status = d_status;
  }
  // big items: the panel pipeline, with the trailing-update gemm chosen per
  // item (kernel 3: CUDA cores; 4: tensor cores, two-accumulator tiles;
  // else tensor cores, wide tiles); largest first over the workers when
  // there are several
  std::vector<size_t> order(big_idx);
  std::sort(order.begin(), order.end(),
            [&](size_t a, size_t b) { return m[a] * n[a] > m[b] * n[b]; });
  std::atomic<size_t> next(0);
  std::atomic<int> fatal(0);
  auto run = [&](Ctx *wc) {
    const int saved = wc->gemm_kernel, saved_tile = wc->gemm_tile;
    for (size_t j = next++; j < order.size() && !fatal.load(); j = next++) {
      const size_t i = order[j];
      const int k = kernel ? kernel[i] : 0;
      wc->gemm_kernel = (k == 3) ? GEMM_PLAIN : GEMM_TC;
      wc->gemm_tile = (k == 4) ? GEMM_TILE_DOUBLE : (k == 2 ? GEMM_TILE_WIDE : GEMM_TILE_AUTO);
      size_t r = 0;
      uint32_t d = 1;
      int s = zp_echelon_dev(wc, (int)m[i], (int)n[i], p[i], A[i], lda[i], &r, &d, nullptr);
      if (s == ST_OK && wc != c) s = ctx_check_status(wc, "echelon_zp_u32_batch");
      if (s != ST_OK && s != ST_PIVOT) {
        int none = 0;  // the first failure reports
        if (fatal.compare_exchange_strong(none, s) && wc != c) c->last_error = wc->last_error;
        break;
      }
      rank[i] = r;
      det[i] = d;
      status[i] = s;
    }
    wc->gemm_kernel = saved;
    wc->gemm_tile = saved_tile;
  };
  if (nworkers > 1) {
    std::vector<std::thread> th;
    for (int t = 0; t < nworkers; ++t)
      th.emplace_back([&, t] {
        cudaSetDevice(c->device);
        run(&h->workers[t]->c);
      });
    for (auto &x : th) x.join();
  } else {
    run(c);
  }
  if (!small.empty()) {
    const size_t ns = small.size();
    cudaError_t e = cudaMemcpyAsync(hr.data(), c->batch_rank, ns * 8, cudaMemcpyDeviceToHost,
                                    c->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(hd.data(), c->batch_det, ns * 4, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(hs.data(), c->batch_status, ns * 4, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return ctx_cuda(c, e, "batch: small blocks");
    for (size_t j = 0; j < ns; ++j) {
      const size_t i = small_idx[j];
      rank[i] = (size_t)hr[j];
      det[i] = hd[j];
      status[i] = (int)hs[j];
    }
  }
  if (fatal.load()) {
    const std::string msg = c->last_error;
    return ctx_fail(c, fatal.load(), msg.c_str());
  }
  return ctx_check_status(c, "echelon_zp_u32_batch");
}

size_t lela_cuda_mlp_param_count(int nfeat) { return mlp_param_count(nfeat); }

int lela_cuda_mlp_forward(lela_cuda_ctx *h, const float *params, int nfeat, const float *X,
                          size_t n, float *out) {
  if (!h) return ST_ARG;
  if (n > (size_t)INT32_MAX) return ctx_fail(&h->c, ST_ARG, "mlp: too many samples");
  DeviceScope ds(&h->c);
  return mlp_forward_dev(&h->c, params, nfeat, X, (int)n, out);
}

int lela_cuda_mlp_grad(lela_cuda_ctx *h, const float *params, int nfeat, const float *X,
                       const float *target, size_t n, float *grad, float *loss) {
  if (!h) return ST_ARG;
  if (n > (size_t)INT32_MAX) return ctx_fail(&h->c, ST_ARG, "mlp: too many samples");
  DeviceScope ds(&h->c);
  return mlp_grad_dev(&h->c, params, nfeat, X, target, (int)n, grad, loss);
}

int lela_cuda_mlp_adam(lela_cuda_ctx *h, float *params, const float *grad, float *m, float *v,
                       size_t count, int step, float lr) {
  if (!h || step < 1) return ST_ARG;
  DeviceScope ds(&h->c);
  return mlp_adam_dev(&h->c, params, grad, m, v, (int)count, step, lr);
}

static int fl_finish(Ctx *c, int st, const FlResult &r, size_t *rank, uint32_t *det,
                     size_t *out_rows, size_t *bad_row) {
  if (rank) *rank = r.rank;
  if (det) *det = r.det;
  if (out_rows) *out_rows = (st == ST_OK) ? r.out_rows : 0;
  if (bad_row) *bad_row = r.bad_row;
  if (st == ST_OK) st = ctx_check_status(c, "fl_echelonize_zp_u32");
  return st;
}

// Host CSR input of the Faugere-Lachartre entry points: checked, copied to
// the device (BUF_FL_X), row heads taken on the host.
struct FlHostInput {
  uint64_t *d_rowptr = nullptr;
  uint32_t *d_col = nullptr, *d_val = nullptr;
  std::vector<uint32_t> heads, hv;
};

static int fl_host_input(Ctx *c, size_t m, size_t n, const uint64_t *rowptr,
                         const uint32_t *colidx, const uint32_t *vals, FlHostInput *in) {
  const uint64_t nnz = rowptr[m];
  if (nnz && (!colidx || !vals)) return ctx_fail(c, ST_ARG, "null pointer");
  for (size_t r = 0; r < m; ++r)
    if (rowptr[r + 1] < rowptr[r]) return ctx_fail(c, ST_ARG, "row pointers decrease");
  for (uint64_t e = 0; e < nnz; ++e)
    if (colidx[e] >= n) return ctx_fail(c, ST_ARG, "column index out of range");
  in->heads.assign(m, 0);
  in->hv.assign(m, 0);
  for (size_t r = 0; r < m; ++r) {
    const bool empty = rowptr[r + 1] == rowptr[r];
    in->heads[r] = empty ? 0 : colidx[rowptr[r]];
    in->hv[r] = empty ? 0 : vals[rowptr[r]];
  }
  void *dX = nullptr;
  const size_t xbytes = (m + 1) * 8 + nnz * 8 + 64;
  int st = ctx_buffer(c, BUF_FL_X, xbytes, &dX);
  if (st) return st;
  in->d_rowptr = (uint64_t *)dX;
  in->d_col = (uint32_t *)(in->d_rowptr + m + 1);
  in->d_val = in->d_col + nnz;
  cudaError_t e = cudaMemcpyAsync(in->d_rowptr, rowptr, (m + 1) * 8, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess && nnz)
    e = cudaMemcpyAsync(in->d_col, colidx, nnz * 4, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess && nnz)
    e = cudaMemcpyAsync(in->d_val, vals, nnz * 4, cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) return ctx_cuda(c, e, "fl: input copy");
  return ST_OK;
}

// Copies a CSR result out (kind: cudaMemcpyDeviceToHost or ToDevice):
// the row pointers always, the entries when cap allows (else
// ST_CAPACITY: the result stays in the handle for lela_cuda_fl_csr_fetch).
static int fl_csr_out(Ctx *c, const FlCsr &csr, size_t rows, cudaMemcpyKind kind,
                      uint64_t *R_rowptr, uint32_t *R_colidx, uint32_t *R_vals, size_t R_cap,
                      size_t *R_nnz) {
  if (R_nnz) *R_nnz = csr.nnz;
  cudaError_t e = cudaMemcpyAsync(R_rowptr, csr.rowptr, (rows + 1) * 8, kind, c->stream);
  if (e == cudaSuccess && csr.nnz && csr.nnz <= R_cap) {
    e = cudaMemcpyAsync(R_colidx, csr.colidx, csr.nnz * 4, kind, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(R_vals, csr.vals, csr.nnz * 4, kind, c->stream);
  }
  if (e != cudaSuccess) return ctx_cuda(c, e, "fl: csr output copy");
  if (csr.nnz > R_cap) {
    e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return ctx_cuda(c, e, "fl: csr output copy");
    return ctx_fail(c, ST_CAPACITY, "fl: the CSR result has more entries than the output arrays hold");
  }
  return ST_OK;
}

int lela_cuda_fl_echelonize_zp_u32_csr(lela_cuda_ctx *h, size_t m, size_t n, uint32_t p,
                                       const uint64_t *rowptr, const uint32_t *colidx,
                                       const uint32_t *vals, int reduced, int only_D,
                                       uint64_t *R_rowptr, uint32_t *R_colidx, uint32_t *R_vals,
                                       size_t R_cap, size_t *R_nnz, size_t *rank, uint32_t *det,
                                       size_t *out_rows, size_t *bad_row) {
  if (!h) return ST_ARG;
  Ctx *c = &h->c;
  if (m > (size_t)INT32_MAX || n > (size_t)INT32_MAX) return ctx_fail(c, ST_ARG, "dimension too large");
  if (p < 2) return ctx_fail(c, ST_ARG, "modulus must be at least 2");
  if (!rowptr || !R_rowptr || (R_cap && (!R_colidx || !R_vals)))
    return ctx_fail(c, ST_ARG, "bad output or row pointers");
  DeviceScope ds(c);
  FlHostInput in;
  int st = fl_host_input(c, m, n, rowptr, colidx, vals, &in);
  if (!st) st = ctx_clear_status(c);
  if (st) return st;
  FlResult res{};
  FlCsr csr;
  st = zp_fl_echelonize_dev(c, (int)m, (int)n, p, in.d_rowptr, in.d_col, in.d_val, rowptr,
                            in.heads.data(), in.hv.data(), reduced != 0, only_D != 0, nullptr, 0,
                            &res, &csr);
  if (st == ST_OK)
    st = fl_csr_out(c, csr, res.out_rows, cudaMemcpyDeviceToHost, R_rowptr, R_colidx, R_vals,
                    R_cap, R_nnz);
  if (st == ST_CAPACITY) {
    fl_finish(c, ST_OK, res, rank, det, out_rows, bad_row);
    return ST_CAPACITY;
  }
  return fl_finish(c, st, res, rank, det, out_rows, bad_row);
}

int lela_cuda_fl_csr_fetch(lela_cuda_ctx *h, uint32_t *colidx, uint32_t *vals, size_t cap,
                           int device) {
  if (!h) return ST_ARG;
  Ctx *c = &h->c;
  if (c->fl_csr_nnz == (size_t)-1) return ctx_fail(c, ST_ARG, "fl: no CSR result kept");
  const size_t nnz = c->fl_csr_nnz;
  if (nnz > cap) return ctx_fail(c, ST_CAPACITY, "fl: the CSR result has more entries than cap");
  if (nnz && (!colidx || !vals)) return ctx_fail(c, ST_ARG, "null pointer");
  if (!nnz) return ST_OK;
  DeviceScope ds(c);
  const size_t col_bytes = (nnz * 4 + 255) & ~(size_t)255;
  const uint8_t *b = static_cast<const uint8_t *>(c->buf[BUF_FL_CSR_V]);
  const cudaMemcpyKind kind = device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  cudaError_t e = cudaMemcpyAsync(colidx, b, nnz * 4, kind, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(vals, b + col_bytes, nnz * 4, kind, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  return e == cudaSuccess ? ST_OK : ctx_cuda(c, e, "fl: csr fetch");
}

int lela_cuda_fl_echelonize_zp_u32(lela_cuda_ctx *h, size_t m, size_t n, uint32_t p,
                                   const uint64_t *rowptr, const uint32_t *colidx,
                                   const uint32_t *vals, int reduced, int only_D, uint32_t *R,
                                   size_t ldr, size_t *rank, uint32_t *det, size_t *out_rows,
                                   size_t *bad_row) {
  if (!h) return ST_ARG;
  Ctx *c = &h->c;
  if (m > (size_t)INT32_MAX || n > (size_t)INT32_MAX) return ctx_fail(c, ST_ARG, "dimension too large");
  if (p < 2) return ctx_fail(c, ST_ARG, "modulus must be at least 2");
  if (!rowptr || (m && (!R || ldr < n))) return ctx_fail(c, ST_ARG, "bad output or row pointers");
  const uint64_t nnz = rowptr[m];
  if (nnz && (!colidx || !vals)) return ctx_fail(c, ST_ARG, "null pointer");
  for (size_t r = 0; r < m; ++r)
    if (rowptr[r + 1] < rowptr[r]) return ctx_fail(c, ST_ARG, "row pointers decrease");
  for (uint64_t e = 0; e < nnz; ++e)
    if (colidx[e] >= n) return ctx_fail(c, ST_ARG, "column index out of range");
  DeviceScope ds(c);
  std::vector<uint32_t> heads(m), hv(m);
  for (size_t r = 0; r < m; ++r) {
    const bool empty = rowptr[r + 1] == rowptr[r];
    heads[r] = empty ? 0 : colidx[rowptr[r]];
    hv[r] = empty ? 0 : vals[rowptr[r]];
  }
  void *dX = nullptr, *dR = nullptr;
  const size_t xbytes = (m + 1) * 8 + nnz * 8 + 64;
  int st = ctx_buffer(c, BUF_FL_X, xbytes, &dX);
  if (!st) st = ctx_buffer(c, BUF_FL_R, std::max<size_t>(m * n * 4, 16), &dR);
  if (st) return st;
  uint64_t *d_rowptr = (uint64_t *)dX;
  uint32_t *d_col = (uint32_t *)(d_rowptr + m + 1);
  uint32_t *d_val = d_col + nnz;
  cudaError_t e = cudaMemcpyAsync(d_rowptr, rowptr, (m + 1) * 8, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess && nnz)
    e = cudaMemcpyAsync(d_col, colidx, nnz * 4, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess && nnz)
    e = cudaMemcpyAsync(d_val, vals, nnz * 4, cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) return ctx_cuda(c, e, "fl: input copy");
  if ((st = ctx_clear_status(c))) return st;
  FlResult res{};
  st = zp_fl_echelonize_dev(c, (int)m, (int)n, p, d_rowptr, d_col, d_val, rowptr, heads.data(),
                            hv.data(), reduced != 0, only_D != 0, (uint32_t *)dR, n, &res);
  if (st == ST_OK && res.out_rows)
    st = d2h_matrix(c, R, dR, res.out_rows, n, ldr, 4);
  return fl_finish(c, st, res, rank, det, out_rows, bad_row);
}

int lela_cuda_fl_echelonize_zp_u32_dev(lela_cuda_ctx *h, size_t m, size_t n, uint32_t p,
                                       const uint64_t *rowptr, const uint32_t *colidx,
                                       const uint32_t *vals, int reduced, int only_D, uint32_t *R,
                                       size_t ldr, size_t *rank, uint32_t *det, size_t *out_rows,
                                       size_t *bad_row) {
  if (!h) return ST_ARG;
  Ctx *c = &h->c;
  DeviceScope ds(c);
  if (m > (size_t)INT32_MAX || n > (size_t)INT32_MAX) return ctx_fail(c, ST_ARG, "dimension too large");
  if (p < 2) return ctx_fail(c, ST_ARG, "modulus must be at least 2");
  if (!rowptr || (m && (!R || ldr < n))) return ctx_fail(c, ST_ARG, "bad output or row pointers");
  std::vector<uint64_t> hrow(m + 1);
  std::vector<uint32_t> heads(m), hv(m);
  void *dH = nullptr;
  int st = ctx_buffer(c, BUF_FL_HEADS, 2 * (m + 1) * 4 + 64, &dH);
  if (st) return st;
  uint32_t *d_heads = (uint32_t *)dH, *d_hv = d_heads + m + 1;
  if ((st = fl_row_heads_dev(c, (int)m, rowptr, colidx, vals, d_heads, d_hv))) return st;
  cudaError_t e = cudaMemcpyAsync(hrow.data(), rowptr, (m + 1) * 8, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess && m)
    e = cudaMemcpyAsync(heads.data(), d_heads, m * 4, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess && m) e = cudaMemcpyAsync(hv.data(), d_hv, m * 4, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return ctx_cuda(c, e, "fl: row heads");
  FlResult res{};
  st = zp_fl_echelonize_dev(c, (int)m, (int)n, p, rowptr, colidx, vals, hrow.data(), heads.data(),
                            hv.data(), reduced != 0, only_D != 0, R, ldr, &res);
  return fl_finish(c, st, res, rank, det, out_rows, bad_row);
}

int lela_cuda_fl_echelonize_zp_u32_csr_dev(lela_cuda_ctx *h, size_t m, size_t n, uint32_t p,
                                           const uint64_t *rowptr, const uint32_t *colidx,
                                           const uint32_t *vals, int reduced, int only_D,
                                           uint64_t *R_rowptr, uint32_t *R_colidx,
                                           uint32_t *R_vals, size_t R_cap, size_t *R_nnz,
                                           size_t *rank, uint32_t *det, size_t *out_rows,
                                           size_t *bad_row) {
  if (!h) return ST_ARG;
  Ctx *c = &h->c;
  DeviceScope ds(c);
  if (m > (size_t)INT32_MAX || n > (size_t)INT32_MAX) return ctx_fail(c, ST_ARG, "dimension too large");
  if (p < 2) return ctx_fail(c, ST_ARG, "modulus must be at least 2");
  if (!rowptr || !R_rowptr || (R_cap && (!R_colidx || !R_vals)))
    return ctx_fail(c, ST_ARG, "bad output or row pointers");
  std::vector<uint64_t> hrow(m + 1);
  std::vector<uint32_t> heads(m), hv(m);
  void *dH = nullptr;
  int st = ctx_buffer(c, BUF_FL_HEADS, 2 * (m + 1) * 4 + 64, &dH);
  if (st) return st;
  uint32_t *d_heads = (uint32_t *)dH, *d_hv = d_heads + m + 1;
  if ((st = fl_row_heads_dev(c, (int)m, rowptr, colidx, vals, d_heads, d_hv))) return st;
  cudaError_t e = cudaMemcpyAsync(hrow.data(), rowptr, (m + 1) * 8, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess && m)
    e = cudaMemcpyAsync(heads.data(), d_heads, m * 4, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess && m) e = cudaMemcpyAsync(hv.data(), d_hv, m * 4, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return ctx_cuda(c, e, "fl: row heads");
  FlResult res{};
  FlCsr csr;
  st = zp_fl_echelonize_dev(c, (int)m, (int)n, p, rowptr, colidx, vals, hrow.data(), heads.data(),
                            hv.data(), reduced != 0, only_D != 0, nullptr, 0, &res, &csr);
  if (st == ST_OK)
    st = fl_csr_out(c, csr, res.out_rows, cudaMemcpyDeviceToDevice, R_rowptr, R_colidx, R_vals,
                    R_cap, R_nnz);
  if (st == ST_CAPACITY) {
    fl_finish(c, ST_OK, res, rank, det, out_rows, bad_row);
    return ST_CAPACITY;
  }
  return fl_finish(c, st, res, rank, det, out_rows, bad_row);
}

namespace {

// Device bytes a handle holds in its grow-only buffers.
size_t ctx_held_bytes(const Ctx *c) {
  size_t s = c->ws_bytes + c->ws2_bytes;
  for (int i = 0; i < 32; ++i) s += c->buf_bytes[i];
  for (int i = 0; i < 4; ++i) s += c->stage_bytes[i];
  return s;
}

// Free a handle's grow-only buffers (after its queued work).
void ctx_trim(Ctx *c) {
  cudaStreamSynchronize(c->stream);
  if (c->ws) cudaFree(c->ws);
  if (c->ws2) cudaFree(c->ws2);
  c->ws = c->ws2 = nullptr;
  c->ws_bytes = c->ws2_bytes = 0;
  for (int i = 0; i < 32; ++i) {
    if (c->buf[i]) cudaFree(c->buf[i]);
    c->buf[i] = nullptr;
    c->buf_bytes[i] = 0;
  }
  for (int i = 0; i < 4; ++i) {
    if (c->stage[i]) cudaFree(c->stage[i]);
    c->stage[i] = nullptr;
    c->stage_bytes[i] = 0;
  }
}

// Upper estimate of the device bytes one FL matrix needs on a handle: the
// dense blocks A, B, C, D (4 m n), the gemm limb planes (at most 4 (m + n) m
// for the Schur complement), the triangular-solve inverses and echelon
// bookkeeping (about 5 KB per row: the echelon's block multipliers are 4 KB),
// and fixed scratch.
size_t fl_bytes_estimate(size_t m, size_t n) {
  return 4 * m * n + 4 * (m + n) * m + 5120 * m + ((size_t)256 << 20);
}

// The memory-budgeted queue of a batch: an item starts only when its
// estimate fits beside the items running (one that does not fit even alone
// runs alone).
struct MemQueue {
  std::mutex mu;
  std::condition_variable cv;
  size_t budget = 0, used = 0;
  int running = 0;
  void acquire(size_t need) {
    std::unique_lock<std::mutex> lk(mu);
    cv.wait(lk, [&] { return running == 0 || used + need <= budget; });
    used += need;
    ++running;
  }
  void release(size_t need) {
    {
      std::lock_guard<std::mutex> lk(mu);
      used -= need;
      --running;
    }
    cv.notify_all();
  }
};

}  // namespace

int lela_cuda_set_batch_memory_budget(lela_cuda_ctx *h, size_t bytes) {
  if (!h) return ST_ARG;
  h->c.batch_budget = bytes;
  return ST_OK;
}

int lela_cuda_fl_echelonize_zp_u32_batch(lela_cuda_ctx *h, size_t count, const size_t *m,
                                         const size_t *n, const uint32_t *p,
                                         const uint64_t *const *rowptr,
                                         const uint32_t *const *colidx,
                                         const uint32_t *const *vals, uint32_t *const *R,
                                         const size_t *ldr, int reduced, int nworkers,
                                         size_t *rank, uint32_t *det, int *status) {
  if (!h) return ST_ARG;
  Ctx *c = &h->c;
  DeviceScope ds(c);
  if (count == 0) return ST_OK;
  if (!m || !n || !p || !rowptr || !colidx || !vals || !R || !ldr || !rank || !det || !status)
    return ctx_fail(c, ST_ARG, "null pointer");
  if (nworkers < 1) nworkers = 1;
  if (nworkers > 16) nworkers = 16;
  if ((size_t)nworkers > count) nworkers = (int)count;
  while ((int)h->workers.size() < nworkers) {
    lela_cuda_ctx *w = nullptr;
    int st = lela_cuda_create(&w, c->device);
    if (st) return ctx_fail(c, st, "batch: worker handle");
    w->c.gemm_kernel = c->gemm_kernel;
    w->c.trsm_kernel = c->trsm_kernel;
    h->workers.push_back(w);
  }
  // Stream order: the workers' streams wait for the work queued on the
  // caller's stream so far, and the caller's stream waits for the workers'
  // at the end, so events on the caller's stream bracket the whole batch.
  cudaEvent_t start = nullptr;
  cudaError_t e = cudaEventCreateWithFlags(&start, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventRecord(start, c->stream);
  for (int t = 0; e == cudaSuccess && t < nworkers; ++t)
    e = cudaStreamWaitEvent(h->workers[t]->c.stream, start, 0);
  if (start) cudaEventDestroy(start);
  if (e != cudaSuccess) return ctx_cuda(c, e, "batch: stream order");
  // largest matrices first
  std::vector<size_t> order(count);
  for (size_t i = 0; i < count; ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return m[a] * n[a] > m[b] * n[b]; });
  // Memory budget: when the nworkers largest matrices may not fit together,
  // items wait for room and each worker frees its buffers after an item.
  MemQueue mq;
  if (c->batch_budget) {
    mq.budget = c->batch_budget;
  } else {
    size_t fr = 0, tot = 0;
    e = cudaMemGetInfo(&fr, &tot);
    if (e != cudaSuccess) return ctx_cuda(c, e, "batch: cudaMemGetInfo");
    size_t held = 0;
    for (int t = 0; t < nworkers; ++t) held += ctx_held_bytes(&h->workers[t]->c);
    mq.budget = fr / 10 * 9 + held;
  }
  size_t peak = 0;
  for (int j = 0; j < nworkers; ++j) peak += fl_bytes_estimate(m[order[j]], n[order[j]]);
  const bool tight = peak > mq.budget;
  std::atomic<size_t> next(0);
  std::atomic<int> fatal(0);
  auto work = [&](lela_cuda_ctx *w) {
    cudaSetDevice(w->c.device);
    w->c.gemm_kernel = c->gemm_kernel;
    w->c.trsm_kernel = c->trsm_kernel;
    if (tight) ctx_trim(&w->c);
    for (size_t j = next++; j < count && !fatal.load(); j = next++) {
      const size_t i = order[j];
      const size_t need = fl_bytes_estimate(m[i], n[i]);
      if (tight) mq.acquire(need);
      if (fatal.load()) {  // another worker failed while this one waited
        if (tight) mq.release(need);
        break;
      }
      size_t rows = 0, bad = 0;
      int st = lela_cuda_fl_echelonize_zp_u32_dev(w, m[i], n[i], p[i], rowptr[i], colidx[i],
                                                  vals[i], reduced, 0, R[i], ldr[i], &rank[i],
                                                  &det[i], &rows, &bad);
      status[i] = st;
      if (st != ST_OK && st != ST_WRONG_FORM && st != ST_DIAG && st != ST_PIVOT) fatal = st;
      if (tight) {
        ctx_trim(&w->c);
        mq.release(need);
      }
    }
  };
  std::vector<std::thread> th;
  for (int t = 0; t < nworkers; ++t) th.emplace_back(work, h->workers[t]);
  for (auto &x : th) x.join();
  for (int t = 0; e == cudaSuccess && t < nworkers; ++t) {
    cudaEvent_t end = nullptr;
    e = cudaEventCreateWithFlags(&end, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(end, h->workers[t]->c.stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, end, 0);
    if (end) cudaEventDestroy(end);
  }
  if (fatal.load()) return ctx_fail(c, fatal.load(), "batch: a worker failed");
  if (e != cudaSuccess) return ctx_cuda(c, e, "batch: stream order");
  return ST_OK;
}

// The dense echelon entry points: device (dev) or host pointers, the
// non-reduced form or the reduced one.
static int echelon_entry(lela_cuda_ctx *h, size_t m, size_t n, uint32_t p, uint32_t *A,
                         size_t lda, size_t *rank, uint32_t *det, bool dev, bool reduced,
                         bool unit = false) {
  if (!h || !rank || !det) return ST_ARG;
  Ctx *c = &h->c;
  DeviceScope ds(c);
  const char *what = reduced ? "echelon_reduced_zp_u32" : "echelon_zp_u32";
  if (m > (size_t)INT32_MAX || n > (size_t)INT32_MAX) return ctx_fail(c, ST_ARG, "dimension too large");
  auto run = [&](uint32_t *D, size_t ld) {
    return reduced ? zp_echelon_reduced_dev(c, (int)m, (int)n, p, D, ld, unit, rank, det)
                   : zp_echelon_dev(c, (int)m, (int)n, p, D, ld, rank, det, nullptr);
  };
  if (dev) {
    if (m && n && !A) return ctx_fail(c, ST_ARG, "null pointer");
    int st = run(A, lda);
    if (!st) st = ctx_check_status(c, what);
    return st;
  }
  if (p < 2) return ctx_fail(c, ST_ARG, "modulus must be at least 2");
  if (m == 0 || n == 0) {
    *rank = 0;
    *det = 1 % p;
    return ST_OK;
  }
  if (!A) return ctx_fail(c, ST_ARG, "null pointer");
  if (lda < n) return ctx_fail(c, ST_ARG, "leading dimension smaller than the row length");
  void *dA = nullptr;
  int st = ctx_stage(c, 0, m * n * 4, &dA);
  if (!st) st = ctx_clear_status(c);
  if (!st) st = h2d_matrix(c, dA, A, m, n, lda, 4);
  if (!st) st = run((uint32_t *)dA, n);
  if (!st) st = d2h_matrix(c, A, dA, m, n, lda, 4);
  if (!st) st = ctx_check_status(c, what);
  return st;
}

static int pluq_entry(lela_cuda_ctx *h, size_t m, size_t n, uint32_t p, uint32_t *A, size_t lda,
                      size_t *P, size_t *np, size_t *Q, size_t *nq, size_t *rank, uint32_t *det,
                      bool dev) {
  if (!h || !rank || !det || !np || !nq) return ST_ARG;
  Ctx *c = &h->c;
  DeviceScope ds(c);
  if (m > (size_t)INT32_MAX || n > (size_t)INT32_MAX) return ctx_fail(c, ST_ARG, "dimension too large");
  if (p < 2) return ctx_fail(c, ST_ARG, "modulus must be at least 2");
  if (m && n && (!A || lda < n || !P || !Q))
    return ctx_fail(c, ST_ARG, "bad matrix or permutation arrays");
  std::vector<std::pair<int, int>> vp, vq;
  int st = ctx_clear_status(c);
  if (st) return st;
  uint32_t *dA = A;
  size_t ld = lda;
  if (!dev && m && n) {
    void *s = nullptr;
    if ((st = ctx_stage(c, 0, m * n * 4, &s))) return st;
    dA = static_cast<uint32_t *>(s);
    ld = n;
    if ((st = h2d_matrix(c, dA, A, m, n, lda, 4))) return st;
  }
  st = zp_pluq_dev(c, (int)m, (int)n, p, dA, ld, &vp, &vq, rank, det);
  if (st == ST_PIVOT) return ctx_fail(c, ST_PIVOT, "Could not invert pivot-element in the ring");
  if (st) return st;
  if (!dev && m && n && (st = d2h_matrix(c, A, dA, m, n, lda, 4))) return st;
  for (size_t t = 0; t < vp.size(); ++t) {
    P[2 * t] = (size_t)vp[t].first;
    P[2 * t + 1] = (size_t)vp[t].second;
  }
  for (size_t t = 0; t < vq.size(); ++t) {
    Q[2 * t] = (size_t)vq[t].first;
    Q[2 * t + 1] = (size_t)vq[t].second;
  }
  *np = vp.size();
  *nq = vq.size();
  return ctx_check_status(c, "pluq_zp_u32");
}

int lela_cuda_pluq_zp_u32(lela_cuda_ctx *h, size_t m, size_t n, uint32_t p, uint32_t *A, size_t lda,
                          size_t *P, size_t *np, size_t *Q, size_t *nq, size_t *rank, uint32_t *det) {
  return pluq_entry(h, m, n, p, A, lda, P, np, Q, nq, rank, det, false);
}

int lela_cuda_pluq_zp_u32_dev(lela_cuda_ctx *h, size_t m, size_t n, uint32_t p, uint32_t *A,
                              size_t lda, size_t *P, size_t *np, size_t *Q, size_t *nq,
                              size_t *rank, uint32_t *det) {
  return pluq_entry(h, m, n, p, A, lda, P, np, Q, nq, rank, det, true);
}

static int transform_entry(lela_cuda_ctx *h, size_t m, size_t n, uint32_t p, uint32_t *A,
                           size_t lda, uint32_t *L, size_t ldl, size_t *P, size_t *np,
                           size_t *rank, uint32_t *det, bool dev) {
  if (!h || !rank || !det || !np) return ST_ARG;
  Ctx *c = &h->c;
  DeviceScope ds(c);
  if (m > (size_t)INT32_MAX || n > (size_t)INT32_MAX) return ctx_fail(c, ST_ARG, "dimension too large");
  if (p < 2) return ctx_fail(c, ST_ARG, "modulus must be at least 2");
  if (m && (!L || ldl < m)) return ctx_fail(c, ST_ARG, "bad transform array");
  if (m && n && (!A || lda < n || !P)) return ctx_fail(c, ST_ARG, "bad matrix or permutation array");
  std::vector<std::pair<int, int>> vp;
  int st = ctx_clear_status(c);
  if (st) return st;
  uint32_t *dA = A, *dL = L;
  size_t ld = lda, ldL = ldl;
  if (!dev && m) {
    void *s = nullptr;
    if (n) {
      if ((st = ctx_stage(c, 0, m * n * 4, &s))) return st;
      dA = static_cast<uint32_t *>(s);
      ld = n;
      if ((st = h2d_matrix(c, dA, A, m, n, lda, 4))) return st;
    }
    if ((st = ctx_stage(c, 1, m * m * 4, &s))) return st;
    dL = static_cast<uint32_t *>(s);
    ldL = m;
  }
  st = zp_echelon_transform_dev(c, (int)m, (int)n, p, dA, ld, dL, ldL, &vp, rank, det);
  if (st == ST_PIVOT) return ctx_fail(c, ST_PIVOT, "Could not invert pivot-element in the ring");
  if (st) return st;
  if (!dev && m) {
    if (n && (st = d2h_matrix(c, A, dA, m, n, lda, 4))) return st;
    if ((st = d2h_matrix(c, L, dL, m, m, ldl, 4))) return st;
  }
  for (size_t t = 0; t < vp.size(); ++t) {
    P[2 * t] = (size_t)vp[t].first;
    P[2 * t + 1] = (size_t)vp[t].second;
  }
  *np = vp.size();
  return ctx_check_status(c, "echelon_reduced_transform_zp_u32");
}

int lela_cuda_echelon_reduced_transform_zp_u32(lela_cuda_ctx *h, size_t m, size_t n, uint32_t p,
                                               uint32_t *A, size_t lda, uint32_t *L, size_t ldl,
                                               size_t *P, size_t *np, size_t *rank,
                                               uint32_t *det) {
  return transform_entry(h, m, n, p, A, lda, L, ldl, P, np, rank, det, false);
}

int lela_cuda_echelon_reduced_transform_zp_u32_dev(lela_cuda_ctx *h, size_t m, size_t n,
                                                   uint32_t p, uint32_t *A, size_t lda,
                                                   uint32_t *L, size_t ldl, size_t *P, size_t *np,
                                                   size_t *rank, uint32_t *det) {
  return transform_entry(h, m, n, p, A, lda, L, ldl, P, np, rank, det, true);
}

int lela_cuda_echelon_zp_u32_dev(lela_cuda_ctx *h, size_t m, size_t n, uint32_t p, uint32_t *A,
                                 size_t lda, size_t *rank, uint32_t *det) {
  return echelon_entry(h, m, n, p, A, lda, rank, det, true, false);
}

int lela_cuda_echelon_zp_u32(lela_cuda_ctx *h, size_t m, size_t n, uint32_t p, uint32_t *A,
                             size_t lda, size_t *rank, uint32_t *det) {
  return echelon_entry(h, m, n, p, A, lda, rank, det, false, false);
}

int lela_cuda_echelon_reduced_zp_u32_dev(lela_cuda_ctx *h, size_t m, size_t n, uint32_t p,
                                         uint32_t *A, size_t lda, int unit_pivots, size_t *rank,
                                         uint32_t *det) {
  return echelon_entry(h, m, n, p, A, lda, rank, det, true, true, unit_pivots != 0);
}

int lela_cuda_echelon_reduced_zp_u32(lela_cuda_ctx *h, size_t m, size_t n, uint32_t p,
                                     uint32_t *A, size_t lda, int unit_pivots, size_t *rank,
                                     uint32_t *det) {
  return echelon_entry(h, m, n, p, A, lda, rank, det, false, true, unit_pivots != 0);
}

int lela_cuda_trsm_csr_upper_zp_u32(lela_cuda_ctx *h, size_t n, size_t ncols, uint32_t p,
                                    uint32_t a, int diag_is_one, const uint64_t *rowptr,
                                    const uint32_t *colidx, const uint32_t *vals, uint32_t *B,
                                    size_t ldb, size_t *bad_idx) {
  if (!h) return ST_ARG;
  Ctx *c = &h->c;
  if (n > (size_t)INT32_MAX || ncols > (size_t)INT32_MAX)
    return ctx_fail(c, ST_ARG, "dimension too large");
  if (p < 2) return ctx_fail(c, ST_ARG, "modulus must be at least 2");
  if (n == 0) return ST_OK;
  if (!rowptr || (ncols && !B)) return ctx_fail(c, ST_ARG, "null pointer");
  if (ncols && ldb < ncols) return ctx_fail(c, ST_ARG, "leading dimension smaller than the row length");
  const uint64_t nnz = rowptr[n];
  if (nnz && (!colidx || !vals)) return ctx_fail(c, ST_ARG, "null pointer");
  if (rowptr[0] != 0) return ctx_fail(c, ST_ARG, "row pointers must start at 0");
  for (size_t r = 0; r < n; ++r)
    if (rowptr[r + 1] < rowptr[r]) return ctx_fail(c, ST_ARG, "row pointers decrease");
  for (uint64_t e = 0; e < nnz; ++e)
    if (colidx[e] >= n) return ctx_fail(c, ST_ARG, "column index out of range");
  DeviceScope ds(c);
  void *dX = nullptr, *dB = nullptr;
  int st = ctx_stage(c, 2, (n + 1) * 8 + nnz * 8 + 64, &dX);
  if (!st && ncols) st = ctx_stage(c, 1, n * ncols * 4, &dB);
  if (st) return st;
  uint64_t *d_rowptr = (uint64_t *)dX;
  uint32_t *d_col = (uint32_t *)(d_rowptr + n + 1);
  uint32_t *d_val = d_col + nnz;
  cudaError_t e = cudaMemcpyAsync(d_rowptr, rowptr, (n + 1) * 8, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess && nnz)
    e = cudaMemcpyAsync(d_col, colidx, nnz * 4, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess && nnz)
    e = cudaMemcpyAsync(d_val, vals, nnz * 4, cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) return ctx_cuda(c, e, "trsm csr: input copy");
  if ((st = ctx_clear_status(c))) return st;
  if (ncols && (st = h2d_matrix(c, dB, B, n, ncols, ldb, 4))) return st;
  st = zp_trsm_csr_upper_dev(c, diag_is_one != 0, (int)n, (int)ncols, p, a, d_rowptr, d_col,
                             d_val, (uint32_t *)dB, ncols, bad_idx);
  if (!st && ncols) st = d2h_matrix(c, B, dB, n, ncols, ldb, 4);
  if (!st) st = ctx_check_status(c, "trsm_csr_upper_zp_u32");
  return st;
}

int lela_cuda_trsm_csr_upper_zp_u32_dev(lela_cuda_ctx *h, size_t n, size_t ncols, uint32_t p,
                                        uint32_t a, int diag_is_one, const uint64_t *rowptr,
                                        const uint32_t *colidx, const uint32_t *vals, uint32_t *B,
                                        size_t ldb, size_t *bad_idx) {
  if (!h) return ST_ARG;
  Ctx *c = &h->c;
  DeviceScope ds(c);
  if (n > (size_t)INT32_MAX || ncols > (size_t)INT32_MAX)
    return ctx_fail(c, ST_ARG, "dimension too large");
  if (n && (!rowptr || (ncols && !B))) return ctx_fail(c, ST_ARG, "null pointer");
  return zp_trsm_csr_upper_dev(c, diag_is_one != 0, (int)n, (int)ncols, p, a, rowptr, colidx,
                               vals, B, ldb, bad_idx);
}

int lela_cuda_trsm_zp_u32_dev(lela_cuda_ctx *h, int upper, int diag_is_one, size_t m, size_t n,
                              uint32_t p, uint32_t a, const uint32_t *A, size_t lda, uint32_t *B,
                              size_t ldb, size_t *bad_idx) {
  if (!h) return ST_ARG;
  Ctx *c = &h->c;
  DeviceScope ds(c);
  if (m > (size_t)INT32_MAX || n > (size_t)INT32_MAX) return ctx_fail(c, ST_ARG, "dimension too large");
  if (m && (!A || (n && !B))) return ctx_fail(c, ST_ARG, "null pointer");
  return zp_trsm_dev(c, upper != 0, diag_is_one != 0, (int)m, (int)n, p, a, A, lda, B, ldb,
                     bad_idx);
}

int lela_cuda_trsm_zp_u32(lela_cuda_ctx *h, int upper, int diag_is_one, size_t m, size_t n,
                          uint32_t p, uint32_t a, const uint32_t *A, size_t lda, uint32_t *B,
                          size_t ldb, size_t *bad_idx) {
  if (!h) return ST_ARG;
  Ctx *c = &h->c;
  if (m > (size_t)INT32_MAX || n > (size_t)INT32_MAX) return ctx_fail(c, ST_ARG, "dimension too large");
  if (p < 2) return ctx_fail(c, ST_ARG, "modulus must be at least 2");
  if (m == 0) return ST_OK;
  if (!A || (n && !B)) return ctx_fail(c, ST_ARG, "null pointer");
  if (lda < m || (n && ldb < n)) return ctx_fail(c, ST_ARG, "leading dimension smaller than the row length");
  DeviceScope ds(c);
  void *dA = nullptr, *dB = nullptr;
  int st = ctx_stage(c, 0, m * m * 4, &dA);
  if (!st && n) st = ctx_stage(c, 1, m * n * 4, &dB);
  if (!st) st = ctx_clear_status(c);
  if (!st) st = h2d_matrix(c, dA, A, m, m, lda, 4);
  if (!st && n) st = h2d_matrix(c, dB, B, m, n, ldb, 4);
  if (!st)
    st = zp_trsm_dev(c, upper != 0, diag_is_one != 0, (int)m, (int)n, p, a, (const uint32_t *)dA,
                     m, (uint32_t *)dB, n, bad_idx);
  if (!st && n) st = d2h_matrix(c, B, dB, m, n, ldb, 4);
  if (!st) st = ctx_check_status(c, "trsm_zp_u32");
  return st;
}

// ------------------------------------------ other Modular<T> element types
// The operands go to uint32 residues in BUF_ELEM (each part aligned to 256
// bytes), the uint32 path computes, the result goes back to type T.

static size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

static int gemm_elem_dev(Ctx *c, int elem, size_t m, size_t n, size_t k, uint32_t p, uint32_t a,
                         const void *A, size_t lda, const void *B, size_t ldb, uint32_t b, void *C,
                         size_t ldc) {
  const size_t ba = al256(m * k * 4), bb = al256(k * n * 4), bc = al256(m * n * 4);
  void *buf = nullptr;
  int st = ctx_buffer(c, BUF_ELEM, ba + bb + bc, &buf);
  if (st) return st;
  uint32_t *uA = static_cast<uint32_t *>(buf);
  uint32_t *uB = reinterpret_cast<uint32_t *>(static_cast<char *>(buf) + ba);
  uint32_t *uC = reinterpret_cast<uint32_t *>(static_cast<char *>(buf) + ba + bb);
  if (k) {
    if ((st = elem_to_u32(c, elem, A, lda, uA, k, (int)m, (int)k, p))) return st;
    if ((st = elem_to_u32(c, elem, B, ldb, uB, n, (int)k, (int)n, p))) return st;
  }
  // with b = 0 mod p the kernels never read C
  if (b % p != 0 && (st = elem_to_u32(c, elem, C, ldc, uC, n, (int)m, (int)n, p))) return st;
  if ((st = zp_gemm_dev(c, GEMM_AUTO, (int)m, (int)n, (int)k, p, a, uA, k, uB, n, b, uC, n,
                        nullptr)))
    return st;
  return elem_from_u32(c, elem, uC, n, C, ldc, (int)m, (int)n, p);
}

static int gemm_elem_args(Ctx *c, int elem, size_t m, size_t n, size_t k, uint32_t p,
                          const void *A, size_t lda, const void *B, size_t ldb, const void *C,
                          size_t ldc) {
  if (int st = elem_check_modulus(c, elem, p)) return st;
  if (m > (size_t)INT32_MAX || n > (size_t)INT32_MAX || k > (size_t)INT32_MAX)
    return ctx_fail(c, ST_ARG, "dimension too large");
  if (m == 0 || n == 0) return ST_OK;
  if (!C || (k && (!A || !B))) return ctx_fail(c, ST_ARG, "null pointer");
  if (ldc < n || (k && (lda < k || ldb < n)))
    return ctx_fail(c, ST_ARG, "leading dimension smaller than the row length");
  return ST_OK;
}

int lela_cuda_gemm_zp_dev(lela_cuda_ctx *h, int elem, size_t m, size_t n, size_t k, uint32_t p,
                          uint32_t a, const void *A, size_t lda, const void *B, size_t ldb,
                          uint32_t b, void *C, size_t ldc) {
  if (!h) return ST_ARG;
  if (elem == LELA_CUDA_ELEM_U32)
    return lela_cuda_gemm_zp_u32_dev(h, m, n, k, p, a, static_cast<const uint32_t *>(A), lda,
                                     static_cast<const uint32_t *>(B), ldb, b,
                                     static_cast<uint32_t *>(C), ldc);
  Ctx *c = &h->c;
  DeviceScope ds(c);
  if (int st = gemm_elem_args(c, elem, m, n, k, p, A, lda, B, ldb, C, ldc)) return st;
  if (m == 0 || n == 0) return ST_OK;
  return gemm_elem_dev(c, elem, m, n, k, p, a, A, lda, B, ldb, b, C, ldc);
}

int lela_cuda_gemm_zp(lela_cuda_ctx *h, int elem, size_t m, size_t n, size_t k, uint32_t p,
                      uint32_t a, const void *A, size_t lda, const void *B, size_t ldb, uint32_t b,
                      void *C, size_t ldc) {
  if (!h) return ST_ARG;
  if (elem == LELA_CUDA_ELEM_U32)
    return lela_cuda_gemm_zp_u32(h, m, n, k, p, a, static_cast<const uint32_t *>(A), lda,
                                 static_cast<const uint32_t *>(B), ldb, b,
                                 static_cast<uint32_t *>(C), ldc);
  Ctx *c = &h->c;
  if (int st = gemm_elem_args(c, elem, m, n, k, p, A, lda, B, ldb, C, ldc)) return st;
  if (m == 0 || n == 0) return ST_OK;
  DeviceScope ds(c);
  const size_t es = elem_size(elem);
  void *dA = nullptr, *dB = nullptr, *dC = nullptr;
  int st = ST_OK;
  if (!st && k) st = ctx_stage(c, 0, m * k * es, &dA);
  if (!st && k) st = ctx_stage(c, 1, k * n * es, &dB);
  if (!st) st = ctx_stage(c, 2, m * n * es, &dC);
  if (!st) st = ctx_clear_status(c);
  if (!st && k) st = h2d_matrix(c, dA, A, m, k, lda, es);
  if (!st && k) st = h2d_matrix(c, dB, B, k, n, ldb, es);
  if (!st && (b % p) != 0) st = h2d_matrix(c, dC, C, m, n, ldc, es);
  if (!st) st = gemm_elem_dev(c, elem, m, n, k, p, a, dA, k, dB, n, b, dC, n);
  if (!st) st = d2h_matrix(c, C, dC, m, n, ldc, es);
  if (!st) st = ctx_check_status(c, "gemm_zp");
  return st;
}

static int trsm_elem_dev(Ctx *c, int elem, bool upper, bool unit, size_t m, size_t n, uint32_t p,
                         uint32_t a, const void *A, size_t lda, void *B, size_t ldb,
                         size_t *bad_idx) {
  const size_t ba = al256(m * m * 4), bb = al256(m * n * 4);
  void *buf = nullptr;
  int st = ctx_buffer(c, BUF_ELEM, ba + bb, &buf);
  if (st) return st;
  uint32_t *uA = static_cast<uint32_t *>(buf);
  uint32_t *uB = reinterpret_cast<uint32_t *>(static_cast<char *>(buf) + ba);
  if ((st = elem_to_u32(c, elem, A, lda, uA, m, (int)m, (int)m, p))) return st;
  if ((st = elem_to_u32(c, elem, B, ldb, uB, n, (int)m, (int)n, p))) return st;
  if ((st = zp_trsm_dev(c, upper, unit, (int)m, (int)n, p, a, uA, m, uB, n, bad_idx))) return st;
  return elem_from_u32(c, elem, uB, n, B, ldb, (int)m, (int)n, p);
}

static int trsm_elem_args(Ctx *c, int elem, size_t m, size_t n, uint32_t p, const void *A,
                          size_t lda, const void *B, size_t ldb) {
  if (int st = elem_check_modulus(c, elem, p)) return st;
  if (m > (size_t)INT32_MAX || n > (size_t)INT32_MAX) return ctx_fail(c, ST_ARG, "dimension too large");
  if (m == 0) return ST_OK;
  if (!A || (n && !B)) return ctx_fail(c, ST_ARG, "null pointer");
  if (lda < m || (n && ldb < n)) return ctx_fail(c, ST_ARG, "leading dimension smaller than the row length");
  return ST_OK;
}

int lela_cuda_trsm_zp_dev(lela_cuda_ctx *h, int elem, int upper, int diag_is_one, size_t m,
                          size_t n, uint32_t p, uint32_t a, const void *A, size_t lda, void *B,
                          size_t ldb, size_t *bad_idx) {
  if (!h) return ST_ARG;
  if (elem == LELA_CUDA_ELEM_U32)
    return lela_cuda_trsm_zp_u32_dev(h, upper, diag_is_one, m, n, p, a,
                                     static_cast<const uint32_t *>(A), lda,
                                     static_cast<uint32_t *>(B), ldb, bad_idx);
  Ctx *c = &h->c;
  DeviceScope ds(c);
  if (int st = trsm_elem_args(c, elem, m, n, p, A, lda, B, ldb)) return st;
  if (m == 0) return ST_OK;
  return trsm_elem_dev(c, elem, upper != 0, diag_is_one != 0, m, n, p, a, A, lda, B, ldb, bad_idx);
}

int lela_cuda_trsm_zp(lela_cuda_ctx *h, int elem, int upper, int diag_is_one, size_t m, size_t n,
                      uint32_t p, uint32_t a, const void *A, size_t lda, void *B, size_t ldb,
                      size_t *bad_idx) {
  if (!h) return ST_ARG;
  if (elem == LELA_CUDA_ELEM_U32)
    return lela_cuda_trsm_zp_u32(h, upper, diag_is_one, m, n, p, a,
                                 static_cast<const uint32_t *>(A), lda, static_cast<uint32_t *>(B),
                                 ldb, bad_idx);
  Ctx *c = &h->c;
  if (int st = trsm_elem_args(c, elem, m, n, p, A, lda, B, ldb)) return st;
  if (m == 0) return ST_OK;
  DeviceScope ds(c);
  const size_t es = elem_size(elem);
  void *dA = nullptr, *dB = nullptr;
  int st = ctx_stage(c, 0, m * m * es, &dA);
  if (!st && n) st = ctx_stage(c, 1, m * n * es, &dB);
  if (!st) st = ctx_clear_status(c);
  if (!st) st = h2d_matrix(c, dA, A, m, m, lda, es);
  if (!st && n) st = h2d_matrix(c, dB, B, m, n, ldb, es);
  if (!st)
    st = trsm_elem_dev(c, elem, upper != 0, diag_is_one != 0, m, n, p, a, dA, m, dB, n, bad_idx);
  if (!st && n) st = d2h_matrix(c, B, dB, m, n, ldb, es);
  if (!st) st = ctx_check_status(c, "trsm_zp");
  return st;
}

}  // extern "C"
