// lela_b200/csrc/context.h -- per-handle host state of the CUDA module.
//
// A handle owns one CUDA stream (or borrows the caller's), a growable device
// workspace, a small device status block that kernels report errors into,
// and the pinned host staging used by the host-pointer entry points.  Like
// a LELA Context (lela/blas/context.h:61-63) a handle is not re-entrant:
// use one handle per host thread.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace lela {

// Kernel families a caller (or the selector) can force.
enum GemmKernel : int {
  GEMM_AUTO = 0,    // small-K CUDA-core kernel below its crossover, else tensor cores
  GEMM_PLAIN = 1,   // CUDA-core 64-bit delayed-reduction gemm (the plain GPU form)
  GEMM_TC = 2,      // limb-split INT8 tcgen05 gemm
  GEMM_SMALLK = 3,  // CUDA-core gemm for small K (no per-term wrap check when p < 2^28)
};

// Tile variant of the tensor-core gemm (TcCfg in zp_gemm.cu): variant 0
// (wide tiles, one accumulator buffer for two and four limbs) or variant 1
// (narrower tiles, two accumulator buffers, so that a tile's epilogue
// overlaps the next tile's products); four limbs have variant 0 only.
enum GemmTile : int {
  GEMM_TILE_AUTO = 0,    // variant 0 for two limbs at K >= 512 and four limbs, else variant 1
  GEMM_TILE_WIDE = 1,    // variant 0
  GEMM_TILE_DOUBLE = 2,  // variant 1
};

// GF(2) gemm kernels.
enum Gf2Kernel : int {
  GF2_AUTO = 0,  // tensor cores
  GF2_TC = 1,    // int8-expanded tcgen05 gemm
  GF2_M4RM = 2,  // bit-packed four-Russians on CUDA cores
};

// Diagonal-block solvers of the Z/p trsm.
enum TrsmKernel : int {
  TRSM_AUTO = 0,     // inverse leaves for wide right-hand sides, else block substitution
  TRSM_BLOCKS = 1,   // 256-row diagonal blocks by substitution on CUDA cores
  TRSM_INVERSE = 2,  // 512-row diagonal blocks inverted, applied by the tensor-core gemm
};

// Most row blocks of the pipelined host-pointer gemm.
constexpr int PIPE_MAX_BLOCKS = 16;

struct Ctx {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  bool own_stream = false;

  // Device workspace (grown on demand, never shrunk until destroy).
  void *ws = nullptr;
  size_t ws_bytes = 0;
  // Second workspace for callers that need two live scratch regions.
  void *ws2 = nullptr;
  size_t ws2_bytes = 0;

  // Device status words: [0] = error bits, [1..] = auxiliary outputs.
  uint32_t *dstatus = nullptr;
  // Pinned host mirror of the status block.
  uint32_t *hstatus = nullptr;

  // Device staging buffers for the host-pointer entry points.
  void *stage[4] = {nullptr, nullptr, nullptr, nullptr};
  size_t stage_bytes[4] = {0, 0, 0, 0};
  // Copy streams and events of the pipelined host-pointer gemm (created on
  // first use): host->device on copy_in, device->host on copy_out; events
  // [0, PIPE_MAX_BLOCKS) mark a row block's operands in, the next
  // PIPE_MAX_BLOCKS its product done, then start, B in, copies out.
  cudaStream_t copy_in = nullptr, copy_out = nullptr;
  cudaEvent_t pipe_ev[2 * PIPE_MAX_BLOCKS + 3] = {};

  // Named grow-only device buffers of the algorithms (see BufSlot).
  void *buf[32] = {};
  size_t buf_bytes[32] = {};

  int gemm_kernel = GEMM_AUTO;
  int gemm_tile = GEMM_TILE_AUTO;
  int gf2_kernel = GF2_AUTO;
  int trsm_kernel = TRSM_AUTO;
  // Device-memory budget of the batched FL entry point (bytes; 0 = 90 % of
  // the free memory plus what the worker handles already hold).
  size_t batch_budget = 0;
  // Mapped (pinned, device-visible) host memory where the echelon panel
  // search publishes its result and a sequence number; created on first use.
  void *panel_map = nullptr, *panel_map_dev = nullptr;
  uint32_t panel_seq = 0;
  // Entries of the last Faugere-Lachartre CSR result kept in BUF_FL_CSR_V
  // (SIZE_MAX: none), for lela_cuda_fl_csr_fetch.
  size_t fl_csr_nnz = (size_t)-1;
  std::string last_error;

  // Instantiated CUDA graph of the small-block batch launch, replayed while
  // the item count and the batch buffer stay the same.
  cudaGraphExec_t batch_exec = nullptr;
  size_t batch_ns = 0;
  void *batch_buf = nullptr;
  // Device result arrays of the last small-block batch launch.
  uint64_t *batch_rank = nullptr;
  uint32_t *batch_det = nullptr, *batch_status = nullptr;

  // Kernel launches issued through this handle (all kernels of the library).
  uint64_t launches = 0;
  // Optional per-kernel device timing: an event pair around each launch of
  // the named kernels, summed by lela_cuda_profile_read.
  bool profile = false;
  struct ProfRec {
    const char *name;
    cudaEvent_t a, b;
  };
  std::vector<ProfRec> prof;
  std::vector<cudaEvent_t> event_pool;

  // cuTensorMapEncodeTiled, resolved through the runtime at handle creation.
  void *encode_tiled = nullptr;
};

// Buffer slots owned by the algorithms.
enum BufSlot : int {
  BUF_DINV = 0,     // inverted diagonals (trsm)
  BUF_ECH_0 = 1,    // echelon form: pivot bookkeeping
  BUF_ECH_1 = 2,
  BUF_FL_A = 3,     // Faugere-Lachartre blocks A, B, C, D
  BUF_FL_B = 4,
  BUF_FL_C = 5,
  BUF_FL_D = 6,
  BUF_FL_X = 7,     // device copy of the CSR input
  BUF_FL_IDX = 8,   // row / column classification
  BUF_FL_R = 9,     // output
  BUF_FL_T = 10,    // temporaries
  BUF_GF2_0 = 11,
  BUF_GF2_1 = 12,
  BUF_MISC = 13,
  BUF_FL_HEADS = 14,  // device row heads of a device CSR input
  BUF_TINV = 15,      // inverted 64 x 64 diagonal blocks (trsm)
  BUF_BATCH = 16,     // batch item descriptors and results
  BUF_MLP = 17,       // cost-model scratch
  BUF_TRI_W = 18,     // inverted 512-row diagonal blocks (trsm)
  BUF_TRI_T = 19,     // their assembly temporaries
  BUF_TRI_A = 20,     // dense copy of a sparse triangular operand
  BUF_RED = 21,       // reduced echelon form: column maps, pivot block, solved columns
  BUF_TRI_OCC = 22,   // occupancy of a sparse triangular operand's 64 x 64 tiles
  BUF_FL_KR = 23,     // Faugere-Lachartre: per-row column ranges of A and C
  BUF_FL_CSR_P = 24,  // Faugere-Lachartre CSR output: row counts, row pointers, scan scratch
  BUF_FL_CSR_V = 25,  // Faugere-Lachartre CSR output: column indices and values
  BUF_PLUQ = 26,      // PLUQ: kept multipliers, assembled output, column order
  BUF_ELEM = 27,      // uint32 copies of Modular<uint8/uint16/float/double> operands
  BUF_TRANSFORM = 28, // reduced form's transform: kept multipliers, triangles, pivot columns
  BUF_COUNT = 29,
};

// Grow-only allocation helpers; return ST_OK or ST_NOMEM.
int ctx_buffer(Ctx *c, int slot, size_t bytes, void **out);
int ctx_workspace(Ctx *c, size_t bytes, void **out);
int ctx_workspace2(Ctx *c, size_t bytes, void **out);
int ctx_stage(Ctx *c, int slot, size_t bytes, void **out);
// Creates the copy streams and events of the pipelined host-pointer gemm
// on first use.
int ctx_pipe(Ctx *c);
// Record a CUDA error (returns ST_CUDA) or a message (returns code).
int ctx_fail(Ctx *c, int code, const char *msg);
int ctx_cuda(Ctx *c, cudaError_t e, const char *what);
// Reset the device error word (async on the handle's stream).
int ctx_clear_status(Ctx *c);
// Read back the device error word (synchronises the stream) and map it to
// a status code.
int ctx_check_status(Ctx *c, const char *what);

// Mapped (pinned, device-visible) host memory of PANEL_MAP_BYTES where a
// panel search publishes its result (from offset 0) and then a sequence
// number (a uint32 at PANEL_FLAG_OFF); allocated on first use.
constexpr size_t PANEL_MAP_BYTES = 4096, PANEL_FLAG_OFF = 4032;
// a panel's row-transposition lists (source rows, then destination rows) are
// staged here by the host and copied to the device on the stream: a copy
// from pinned memory, so the host does not wait for it.  The host writes the
// next panel's lists only after that panel's search has signalled, which the
// stream orders after the previous copy.
constexpr size_t PANEL_PERM_OFF = 1024, PANEL_PERM_INTS = 256;
static_assert(PANEL_PERM_OFF + PANEL_PERM_INTS * 4 <= PANEL_FLAG_OFF, "staging below the flag");
int ctx_panel_map(Ctx *c, void **host, void **dev);
// Spin until *flag == seq (the work queued before the publishing kernel
// included), checking the handle's stream for errors now and then and
// giving up after a minute.
int ctx_wait_flag(Ctx *c, volatile uint32_t *flag, uint32_t seq, const char *what);

// Raise a kernel's dynamic shared-memory limit to `bytes` on the handle's
// device.  The attribute belongs to the device that is current when it is
// set, so it is set once per (device, kernel) pair, under a lock; handles on
// different devices of one process each get their own.
int ctx_smem_attr(Ctx *c, const void *kernel, int bytes, const char *what);

// Makes the handle's device current for the life of the object and then
// restores the caller's device (the device-pointer entry points run on the
// handle's stream, which belongs to that device).
struct DeviceScope {
  int prev = -1;
  bool changed = false;
  explicit DeviceScope(const Ctx *c) {
    if (cudaGetDevice(&prev) == cudaSuccess && prev != c->device)
      changed = cudaSetDevice(c->device) == cudaSuccess;
  }
  ~DeviceScope() {
    if (changed) cudaSetDevice(prev);
  }
  DeviceScope(const DeviceScope &) = delete;
  DeviceScope &operator=(const DeviceScope &) = delete;
};

// Profiling: prof_begin records the start event of a named kernel launch
// (returns an index, or -1 when profiling is off); prof_end its end event.
int prof_begin(Ctx *c, const char *name);
void prof_end(Ctx *c, int idx);
inline void ctx_launched(Ctx *c, int n = 1) { c->launches += (uint64_t)n; }

}  // namespace lela
