// qs_internal.h — host-side runtime internals shared by the libqsim translation
// units: the context (stream, scratch, error text), launch helpers and the
// device program format produced by the planner (qs_plan.cpp) and consumed by
// the tile-pass kernel (qs_pass.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <memory>
#include <string>
#include <vector>
#include <complex>
#include <stdexcept>
#include <cstdlib>
#include "../../include/qsim.h"

// ---------------------------------------------------------------- errors --
struct qs_error : std::runtime_error {
  int code;
  qs_error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define QS_CHECK_ARG(cond, msg)                                              \
  do { if (!(cond)) throw qs_error(QS_ERR_INVALID, (msg)); } while (0)

#define QS_CUDA(expr)                                                        \
  do {                                                                       \
    cudaError_t _e = (expr);                                                 \
    if (_e != cudaSuccess) {                                                 \
      int _c = (_e == cudaErrorMemoryAllocation) ? QS_ERR_NOMEM : QS_ERR_CUDA; \
      throw qs_error(_c, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
    }                                                                        \
  } while (0)

// ------------------------------------------------------------- context ----
struct qs_plan_s;

struct qs_context {
  int device = 0;
  int sm_count = 148;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  // Host-to-device copies of batch programs, so that building a batch does
  // not wait for the work queued on `stream` (created on first use).
  cudaStream_t upload_stream = nullptr;
  std::string err;
  int tile_bits = 0;    // 0: 13, or the autotuned value for the width
  int block_bits = 0;   // 0: 5 for specialised plans, 4 for the generic kernel
  // Pass specialisation (qs_jit.cpp): 0 off, 1 plans on >= jit_min_qubits,
  // 2 every plan.
  int jit_mode = 1;
  int jit_min_qubits = 24;
  // Batch plans: 0 = one launch per (pass level, tile shape), 1 = one
  // persistent launch (k_pass_queue).  Default from QSIM_BATCH_QUEUE, else 0.
  int batch_queue = 0;
  // Dense-4x4-only passes with 5-bit register blocks and 12- or 13-bit tiles
  // run on the tensor-core pass (qs_pass_tc.cu): 1 on (default), 0 off
  // (QSIM_TC=0 or qs_set_tensor_cores).
  int tensor_cores = 1;
  int64_t launches = 0;
  // Device status word of the pipelined tile passes: a kernel whose bounded
  // wait gave up ORs a cause into it (1 producer, 2 consumers); read and
  // cleared by qs_device_status.  Allocated at the first pipelined launch.
  uint32_t* dev_status = nullptr;
  // Test hook (qs_set_wait_test): the next pipelined pass withholds its first
  // tile so that the consumers' bounded wait runs out.
  int wait_test = 0;
  const void* dev_ptr_ok[4] = {nullptr, nullptr, nullptr, nullptr};  // pointers found to be device memory (qs_apply_*_dev)
  int dev_ptr_ok_device[4] = {-1, -1, -1, -1};  // the device each was checked against
  int dev_ptr_next = 0;                          // slot the next new pointer replaces

  // grow-only device scratch (reductions, sampling partials, ...)
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  // pinned host staging for scalar results
  double* pinned = nullptr;
  size_t pinned_bytes = 0;
  // qs_run_circuit's recently run plans (qs_plan.cpp), least recent first
  struct RunEntry {
    uint64_t hash;
    int n, tile_bits, block_bits, specialised;
    std::vector<qs_op> ops;
    qs_plan_s* plan;
  };
  std::vector<RunEntry> run_cache;

  void* scratch_get(size_t bytes);
  double* pinned_get(size_t bytes);
};

// The handle's upload stream (non-blocking; created on first use).
cudaStream_t qs_upload_stream(qs_context* h);

// Records a launch and checks the launch status.
void qs_after_launch(qs_context* h, const char* what);

// Launch on the handle's stream with the programmatic stream-serialisation
// attribute (the kernel must begin with qs::pdl_begin()), so that its launch
// overlaps the end of the kernel before it; QSIM_PDL=0 launches without it.
inline bool qs_pdl_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("QSIM_PDL");
    return !(e && std::atoi(e) == 0);
  }();
  return on;
}
template <typename... KArgs, typename... Args>
void qs_launch_pdl(qs_context* h, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, Args... args);
// Adjusts the launch counters (kernels replayed from, or captured into, a graph).
void qs_count_launches(qs_context* h, int64_t delta);
// Raises the release threshold of the device's default memory pool to at
// least `keep` bytes (freed stream-ordered memory stays mapped up to it).
void qs_pool_keep_at_least(int device, uint64_t keep);

// ------------------------------------------------------- device program ---
// A plan is a list of passes.  A pass streams every tile of the state once:
// the tile is the set of 2^T amplitudes whose non-tile bits are fixed; it is
// staged in shared memory, a sequence of register blocks is applied, and it
// is written back in place.  A register block gives each thread 2^R
// amplitudes (R <= 5 tile positions) on which its ops run in registers.
enum DevKind : uint8_t {
  DK_U1 = 1,     // controlled dense 2x2 on register bit t0
  DK_U2 = 2,     // dense 4x4 on register bits t0 (bit0) < t1 (bit1), no controls
  DK_X = 3,      // controlled exact swap across register bit t0
  DK_SWAP = 4,   // controlled exact swap of |..01..> and |..10..> (t0 < t1)
  DK_Y = 5,      // controlled exact Pauli-Y on t0
  DK_NEG = 6,    // negate where all control bits are set (CZ family)
  DK_PHASE = 7,  // multiply by c[0] where all control bits are set
  DK_DIAG1 = 8,  // multiply by c[b(d0)]
  DK_DIAG2 = 9,  // multiply by c[b(d1)<<1 | b(d0)]
  DK_RY = 10,    // real rotation [[c, -s], [s, c]] on t0; c[0] = (c, s)
  DK_DTAB = 11,  // merged diagonal: table over the register bits x group
                 // factor x sign mask (layout in qs_pass.cu, encode_dtab)
  DK_KRY = 12,   // one scaled real rotation per register bit set in t0, applied
                 // as a Kronecker product; c[k] = (t, form):
                 //   form 0: (a0, a1) <- (a0 - t a1, a1 + t a0)   [rotation / c]
                 //   form 1: (a0, a1) <- (t a0 - a1, a0 + t a1)   [rotation / s]
                 // (one FMA per component); the dropped positive factor (c or
                 // s) is folded into a later table op or DK_SCALE of the pass
  DK_KU1 = 13,   // one dense 2x2 per register bit (c[4k..4k+3]), likewise
  DK_SCALE = 14, // multiply every amplitude by the real c[0].x
  DK_XRY = 15,   // parity rotation on register bits t0 < t1: the pairs
                 // (x, y) = (|t0=0 t1=0>, |11>) use c[0] = (t, form), the
                 // pairs (|t0=0 t1=1>, |t0=1 t1=0>) use c[1]; each pair as in
                 // DK_KRY (the dropped factors are already in the next diagonal)
  DK_CU2 = 16,   // DK_U2 with controls (rc on register bits, gc on the index)
  DK_NOISE = 17, // stochastic channel on tile position t0, alone in a noise
                 // block (DevBlock.pos[6] == 1; tile == whole state): d0 =
                 // QS_OP_DEPOLARIZE, QS_OP_AMP_DAMP or QS_OP_DEPHASE, gc = bits
                 // of the FP64 parameter, coef = the channel's index k (its
                 // uniform is number k of the item's seed stream)
};

// Locator of a qubit inside a block: values < 8 are register positions; values
// >= 0x80 encode (0x80 | q), a qubit read from the amplitude's global index.
#define DLOC_GLOBAL 0x80

struct __align__(16) DevOp {
  uint8_t kind;
  uint8_t t0, t1;
  uint8_t rc;        // controls among the register positions (bit mask)
  uint8_t d0, d1;    // diagonal locators
  uint8_t ncoef;
  uint8_t pad0;
  uint32_t coef;     // index of the first float2 coefficient in the pass pool
  uint32_t pad1;
  uint64_t gc;       // controls read from the global index (mask of qubits)
};
static_assert(sizeof(DevOp) == 24 || sizeof(DevOp) == 32, "DevOp layout");

struct __align__(16) DevBlock {
  int8_t pos[8];     // R tile-local positions, ascending
  int32_t op_begin;  // index into the pass's op array
  int32_t op_end;
};

struct __align__(16) DevPass {
  int32_t T;         // tile bits
  int32_t R;         // register bits per block
  int32_t nblocks;
  int32_t n_qubits;
  int32_t S[16];     // tile positions (global qubit ids), ascending
  uint32_t block_off; // byte offsets from the start of this DevPass
  uint32_t op_off;
  uint32_t coef_off;
  uint32_t bytes;     // total bytes of this pass record
  uint32_t ncoef;     // float2 entries in the coefficient pool
  uint32_t has2;      // 1 if the pass holds a two-target op (U2 / SWAP), 2 if every op is an uncontrolled U2
  uint32_t pad[2];
};

// Host-side plan.
// A tile pass compiled into a kernel of its own (qs_jit.cpp).
struct JitJob;
struct JitPass {
  void* fn = nullptr;  // CUfunction
  int threads = 0, smem = 0, per_sm = 0;
  // Pipelined passes (qs_jit.cpp): tiles move by TMA through a ring of
  // shared-memory stages; the kernel takes a tensor map of the state whose
  // dimensions start at the bits st[0..rank-1] (st[0] = 0, 8-byte elements)
  // and whose box spans 2^boxb[d] elements in dimension d.
  int pipe = 0;
  int rank = 0;
  int st[5] = {0, 0, 0, 0, 0};
  int boxb[5] = {0, 0, 0, 0, 0};
};

struct qs_plan_s {
  int n_qubits = 0;
  int tile_bits = 0;
  std::vector<uint32_t> pass_offsets;   // byte offset of each DevPass in blob
  std::vector<int> pass_T, pass_R, pass_has2, pass_ncoef;
  std::vector<char> blob;               // host copy of the device program
  void* d_blob = nullptr;               // device copy
  int device = 0;
  qs_plan_info info{};
  cudaStream_t stream = nullptr;        // stream of the last upload/execution
  bool jit_tried = false;               // specialisation attempted
  std::vector<JitPass> jit;             // one per pass when specialised
  // Tensor-core passes (qs_pass_tc.cu): index of each pass's first block
  // matrix in d_mats, or -1; the matrices follow the program in d_blob's
  // allocation (built at upload when the handle uses tensor cores).
  std::vector<int64_t> pass_mats;
  float* d_mats = nullptr;
  std::shared_ptr<JitJob> jit_job;      // sources awaiting / in background compile
  bool jit_queued = false;              // jit_job handed to the background compiler
  std::string jit_err;                  // why specialisation was not used
};

// Pass specialisation (qs_jit.cpp).
int qs_jit_env_mode();                                     // QSIM_JIT (default 1)
bool qs_jit_available(std::string* why);
std::string qs_jit_source(const qs_plan_s* p, size_t pass);
bool qs_jit_compile_plan(qs_context* h, qs_plan_s* p, std::string& err);  // synchronous
void qs_jit_tiered(qs_context* h, qs_plan_s* p);                         // tiered (background)
bool qs_jit_compile_only(const qs_plan_s* p, std::string& err);         // no GPU needed
void qs_jit_launch(qs_context* h, const qs_plan_s* p, size_t pass, void* state, uint64_t ntiles, uint32_t flags);

// Tile and register-block widths for a plan on n qubits: explicit handle
// settings win; otherwise the autotuned entry for (device, n) when the plan
// runs on the generic kernel (qs_tune.cpp); otherwise 13 and 5 / 4.
void qs_plan_shape(const qs_context* h, int n, bool specialised, int& tile_bits, int& block_bits);
// Shape of a circuit's plan: qs_plan_shape, except that a circuit of dense
// two-qubit gates only on >= 12 qubits, planned for the generic kernel with
// no explicit or autotuned shape, gets 13-bit tiles and 5-bit blocks when the
// handle uses tensor cores (the tensor-core pass takes exactly those passes)
// and does not run batches as one persistent launch (which stays on the CUDA
// cores).
void qs_circuit_shape(const qs_context* h, int n, const qs_op* ops, int nops, bool specialised, int& tile_bits,
                      int& block_bits);

// Planner entry (qs_plan.cpp): builds passes for one circuit.
// `specialised`: the plan will run as specialised passes (enables the Cartan
// split of dense two-qubit gates, which only pays off there).
void qs_build_plan(int n_qubits, const qs_op* ops, int n_ops, int tile_bits, qs_plan_s* plan, int block_bits = 0,
                   bool specialised = false);
void qs_plan_upload(qs_context* h, qs_plan_s* p);
// Stream-ordered free after the work queued on `stream` (the stream the
// program last ran on; no device-wide synchronisation).
void qs_plan_free_device(void* d, cudaStream_t stream);
// Frees the plans qs_run_circuit keeps (stream-ordered after their last run).
void qs_run_cache_clear(qs_context* h);
// Runs every pass on n_states equal-width states stored back to back.
void qs_plan_run(qs_context* h, qs_plan_s* p, void* state, bool from_zero, uint64_t n_states);

// Tile-pass launcher (qs_pass.cu).  One item per (state, pass); the state is
// base + state_off (in amplitudes).  PI_FROM_ZERO makes the pass start from
// |0..0> instead of loading the tile (the state is then only written).
#define PI_FROM_ZERO 1u
struct __align__(16) PassItem {
  uint64_t state_off;
  const DevPass* pass;   // device pointer
  uint64_t ntiles;
  uint64_t tile_begin;   // prefix of ntiles over the item table
  uint32_t flags;
  uint32_t pred;           // persistent batch launch: index of the same state's previous-pass item (~0u: none)
  uint64_t noise_seed;     // seed of the uniforms of the pass's noise blocks
  uint8_t* noise_branch;   // branch taken by each noise block (by DevOp.coef), or null
  const float* mats;       // tensor-core pass: block b's matrix operands at mats + 8192 * b (or null)
};
static_assert(sizeof(PassItem) == 64, "PassItem layout");

// One 32x32 block matrix to build (k_block_mats): block `block` of `pass`,
// written as the tensor-core operand pair (TF32 high part, FP32 remainder;
// 4096 floats each) at `out`.
struct TcMatJob {
  const DevPass* pass;
  uint64_t block;
  float* out;
};
void qs_launch_block_mats(qs_context* h, cudaStream_t stream, const TcMatJob* d_jobs, int n_jobs);
// Tensor-core tile pass (qs_pass_tc.cu): every item's pass is dense-4x4-only
// with R = 5 register blocks and T bits (12 or 13), and PassItem.mats holds
// its block matrices.
bool qs_tc_enabled(const qs_context* h);
void qs_launch_pass_tc(qs_context* h, void* base, const PassItem* d_items, int n_items, uint64_t total_tiles, int T);
// One state (or n equal-width states back to back), one pass, item by value.
void qs_launch_pass_tc_single(qs_context* h, void* state, const DevPass* d_pass, int T, uint64_t ntiles,
                              uint32_t flags, const float* mats);
// Whether a pass (tile bits, block bits, has2) runs on the tensor cores.
inline bool qs_tc_pass(const qs_context* h, int T, int R, int has2) {
  return qs_tc_enabled(h) && R == 5 && has2 == 2 && (T == 12 || T == 13);
}
// has2: the pass (or any item of the launch) holds a two-target op; ncoef:
// the largest coefficient pool (float2) of the launch's passes.
void qs_launch_pass_single(qs_context* h, void* state, const DevPass* d_pass, int T, int R, uint64_t ntiles,
                           uint32_t flags, int has2, int ncoef);
// threads: CTA size (a multiple of 32, at most the default); 0 = default.
void qs_launch_pass_items(qs_context* h, void* base, const PassItem* d_items, int n_items, uint64_t total_tiles,
                          int maxT, int R, int has2, int ncoef, int threads = 0);

// The whole batch in one persistent launch (qs_pass.cu, k_pass_queue).
void qs_launch_pass_queue(qs_context* h, void* base, const PassItem* d_items, int n_items, uint64_t total_tiles,
                          int maxT, int has2, int ncoef, uint32_t* counters, uint32_t withhold, uint64_t limit_ns);

// Batch engine internals (qs_batch.cpp), shared with the noise-trajectory
// runner: a batch is a set of host plans (each uploaded into one device
// buffer) and units, each unit one state running one of the plans.
struct BatchUnit {
  int plan;                 // index into the plan list
  uint64_t state_off;       // amplitude offset of the unit's state
  uint64_t noise_seed;      // seed of the unit's noise-block uniforms
  uint8_t* noise_branch;    // device branch record, or null
};
struct qs_batch_plan_s;
// threads: CTA size of the batch's launches (0 = the tile-pass default).
// queue: run the whole batch as one persistent launch (unitary programs only).
qs_batch_plan_s* qs_batch_build_units(qs_context* h, const std::vector<qs_plan_s>& plans,
                                      const std::vector<BatchUnit>& units, bool from_zero, int threads = 0,
                                      bool queue = false);
void qs_batch_launch(qs_context* h, qs_batch_plan_s* B, void* states);
void qs_batch_release(qs_batch_plan_s* B);

// Deterministic uniforms in [0, 1) from a seed: splitmix64 (Steele, Lea and
// Flood, 2014), top 53 bits.  The k-th value (from 0) mixes seed + (k+1)
// times the golden-ratio increment, so any element can be computed on its
// own, on the host or the device.  Shared by the serving runtime's sampling
// and the noise trajectories so that both draw the same stream for a seed.
__host__ __device__ inline double qs_seed_uniform_at(uint64_t seed, uint64_t k) {
  uint64_t z = seed + (k + 1) * 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  z ^= z >> 31;
  return (double)(z >> 11) * 0x1.0p-53;
}
inline void qs_seed_uniforms(uint64_t seed, int64_t count, double* out) {
  for (int64_t i = 0; i < count; ++i) out[i] = qs_seed_uniform_at(seed, (uint64_t)i);
}
// Depolarizing branch for uniform u (the reference's ranges,
// bwk/csrc/noise_sm120.cu:262-289): [0, 1-p) identity (0), then X (1), Y (2),
// Z (3) on consecutive thirds of p.  Plain IEEE operations with no product
// feeding a sum, so host and device agree bit for bit.
__host__ __device__ inline int qs_depol_branch(double p, double u) {
  if (u < 1.0 - p) return 0;
  const double r = u - (1.0 - p), third = p / 3.0;
  if (r < third) return 1;
  if (r < 2.0 * third) return 2;
  return 3;
}

// Convenience used by several units.
inline int qs_blocks_for(qs_context* h, uint64_t items, int threads, int per_sm = 8) {
  uint64_t b = (items + threads - 1) / threads;
  uint64_t cap = (uint64_t)h->sm_count * per_sm;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

template <typename... KArgs, typename... Args>
void qs_launch_pdl(qs_context* h, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = h->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = qs_pdl_enabled() ? 1 : 0;
  QS_CUDA(cudaLaunchKernelEx(&cfg, kern, args...));
}
