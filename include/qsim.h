/*
 * qsim.h — C ABI of libqsim.so, the B200 (sm_100a) statevector engine.
 *
 * Conventions
 *   - A state is a device pointer to 2^n complex64 amplitudes (float re, float im
 *     interleaved), 16-byte aligned.  Basis index i has qubit q at bit q
 *     (little-endian, the Qiskit convention).
 *   - Gate matrices are HOST pointers to complex values, row-major, re/im
 *     interleaved.  The "*_f32" forms take complex64 (the reference's tensor
 *     dtype); program ops (qs_op) carry complex128 so that host-side fusion runs
 *     in FP64.
 *   - Two-qubit matrices: index bit 0 = first listed qubit, bit 1 = second.
 *   - Every call returns QS_OK (0) or an error code; qs_last_error() gives the
 *     message.  No C++ exception crosses this boundary.  Calls are asynchronous
 *     on the handle's stream except those that return host scalars.
 *   - One handle per host thread (a handle is not internally locked).
 *
 * Each entry point names the reference interface it replaces
 * (DarrellThomas/qiskit-blackwell, file:line).
 */
#ifndef QSIM_H
#define QSIM_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QS_OK            0
#define QS_ERR_INVALID   1   /* bad argument (reference: TORCH_CHECK RuntimeError) */
#define QS_ERR_CUDA      2   /* CUDA runtime error                                  */
#define QS_ERR_NOMEM     3   /* device allocation failed                            */
#define QS_ERR_TIMEOUT   4   /* a bounded device-side wait gave up                  */
#define QS_ERR_BUDGET    5   /* request exceeds the handle's memory budget          */
#define QS_ERR_CANCELLED 6   /* a server request was cancelled before it ran        */

#define QS_MAX_QUBITS    34
#define QS_MAX_CONTROLS  7

typedef struct qs_context* qs_handle_t;
typedef struct qs_plan_s*  qs_plan_t;

/* ---------------------------------------------------------------- ops ---- */
/* Circuit operation kinds (program IR).  Qubit roles per kind:             */
enum {
  QS_OP_U1      = 1,  /* dense 2x2 on q[0]; m = 2x2                          */
  QS_OP_U2      = 2,  /* dense 4x4; bit0 = q[0], bit1 = q[1]; m = 4x4         */
  QS_OP_DIAG1   = 3,  /* diagonal; m[0..3] = d0, d1 on q[0]                   */
  QS_OP_DIAG2   = 4,  /* diagonal; m = d[4], index = b(q[1])<<1 | b(q[0])     */
  QS_OP_MCU1    = 5,  /* controls q[0..nq-2], target q[nq-1]; m = 2x2         */
  QS_OP_MCU2    = 6,  /* controls q[0..nq-3], targets q[nq-2] (bit0), q[nq-1] */
  QS_OP_MCX     = 7,  /* exact X; controls q[0..nq-2], target q[nq-1]         */
  QS_OP_MCSWAP  = 8,  /* exact swap; controls q[0..nq-3], targets last two    */
  QS_OP_MCPHASE = 9,  /* multiply by m[0]+i m[1] where all q[0..nq-1] are 1   */
  QS_OP_Y       = 10, /* exact Pauli-Y on q[0]                                */
  QS_OP_RX      = 11, /* exp(-i m[0] X/2) on q[0]; param = parameter index    */
  QS_OP_RY      = 12, /* exp(-i m[0] Y/2) on q[0]                             */
  QS_OP_RZ      = 13, /* exp(-i m[0] Z/2) on q[0]                             */
  /* Stochastic noise channels on q[0], parameter m[0]; only
   * qs_noise_trajectories accepts them (a unitary program rejects them).   */
  QS_OP_DEPOLARIZE = 20, /* I w.p. 1-p, else X, Y, Z w.p. p/3 each          */
  QS_OP_AMP_DAMP   = 21, /* Kraus E0 = [[1,0],[0,sqrt(1-g)]], E1 = [[0,sqrt(g)],[0,0]] */
  QS_OP_DEPHASE    = 22  /* Kraus E0 = [[1,0],[0,sqrt(1-l)]], E1 = [[0,0],[0,sqrt(l)]] */
};

typedef struct qs_op {
  int32_t kind;
  int32_t nq;        /* number of entries of q[] in use                      */
  int32_t q[8];
  int32_t param;     /* parameter index for QS_OP_R*; -1 otherwise           */
  int32_t flags;     /* reserved, 0                                          */
  double  m[32];     /* up to 16 complex128 coefficients, re/im interleaved  */
} qs_op;

typedef struct qs_plan_info {
  int32_t n_qubits;
  int32_t tile_bits;
  int32_t n_passes;
  int32_t n_blocks;
  int64_t n_ops_in;      /* ops given to the planner                        */
  int64_t n_ops_fused;   /* device ops after FP64 1Q fusion                  */
  double  bytes_moved;   /* HBM bytes: passes * 16 * 2^n                     */
  double  flops;         /* FP32 flop estimate of the program                */
  int64_t n_device_ops;  /* ops in the device program (after merging)       */
  int32_t n_jit_passes;  /* passes running as specialised kernels           */
  int32_t reserved;
} qs_plan_info;

/* ------------------------------------------------------------ context ---- */
/* Reference: blackwell_backend/simulator.py:95-116 (BlackwellSimulator
 * __init__ loads the kernels); bwk/setup.py:20-44 (the one extension).      */
int  qs_create(int device, qs_handle_t* out);
int  qs_destroy(qs_handle_t h);
/* Run subsequent work on a caller-owned cudaStream_t (e.g. torch's current
 * stream), used verbatim: NULL is the legacy default stream.  A new handle
 * starts on its own non-blocking stream (see qs_get_stream).                */
int  qs_set_stream(qs_handle_t h, void* cuda_stream);
void* qs_get_stream(qs_handle_t h);
int  qs_sync(qs_handle_t h);
const char* qs_last_error(qs_handle_t h);
const char* qs_version(void);
/* Tile bits used by the fused-pass planner (10..14); 0 = automatic (the
 * autotuned value for the width, else 13).                                  */
int  qs_set_tile_bits(qs_handle_t h, int tile_bits);
/* Register-block width used by the planner (2..5 qubits per thread group);
 * 0 = automatic (5 for plans compiled into specialised passes, 4 for the
 * generic pass kernel, batches included).                                   */
int  qs_set_block_bits(qs_handle_t h, int block_bits);
/* Pass specialisation: a plan's tile passes may be compiled (NVRTC) into
 * kernels with their gate positions and coefficients built in; results are
 * bit-identical to the generic pass kernel.  Compiled kernels are cached per
 * device by source, so new plans of a known circuit use them at once.
 *   mode 0 = never;
 *   mode 1 = tiered: a plan on >= min_qubits qubits (default 24; 0 keeps the
 *            current value) uses cached kernels from its first execution;
 *            at its second execution (the plan is being reused) the missing
 *            passes go to one background compiler thread, and the plan runs
 *            on the generic kernel until they are ready;
 *   mode 2 = every plan is compiled before its first execution.
 * The default mode comes from the QSIM_JIT environment variable (0/1/2),
 * else 1.  No reference counterpart (the reference compiles its kernels
 * ahead of time).                                                           */
int  qs_set_jit(qs_handle_t h, int mode, int min_qubits);
/* Number of kernels this handle has launched since creation; h = NULL gives
 * the count over every handle of the process.                               */
int64_t qs_launch_count(qs_handle_t h);
/* Status word of the handle's device-side waits.  The specialised tile
 * passes of 10..13-qubit tiles run as pipelined kernels (TMA copies through
 * a ring of shared-memory stages, producer and consumer warps synchronised
 * by mbarriers), and a batch plan runs as one persistent launch whose CTAs
 * wait for a state's previous pass before its next; every one of these waits
 * is bounded, and a wait that runs out ORs a cause into this word (1: a
 * pass's copy warp, 2: a pass's compute warps, 4: a batch dependency, 8: a
 * tensor-core pass's block-matrix copy or MMA batch; 16: a target of
 * qs_apply_gates_fused_dev outside the state) and its CTA returns
 * (the tensor-core pass finishes its tiles with whatever the wait left),
 * leaving that part of the state unfinished or wrong.  Waits on the
 * handle's stream, stores the word in *code (0 = no wait ran out) and
 * clears it.  No reference counterpart (the reference has no device-side
 * waits).                                                                   */
int qs_device_status(qs_handle_t h, int* code);
/* How batch plans built on this handle run: on = 0 (the default, unless
 * QSIM_BATCH_QUEUE=1) one launch per (pass level, tile shape), each launch
 * covering every circuit at that level; on = 1 the whole batch in one
 * persistent launch whose CTAs take tiles from a device counter level by
 * level and wait (bounded) for each state's previous pass.  Same results
 * either way.  No reference counterpart (its batches are fixed-width, one
 * launch per gate or one CTA per circuit).                                 */
int qs_set_batch_queue(qs_handle_t h, int on);
/* Tensor cores for dense passes: on = 1 (the default, unless QSIM_TC=0)
 * runs every batch pass whose ops are all dense two-qubit gates, with 5-qubit
 * register blocks and 12- or 13-qubit tiles, on tcgen05.mma: each register
 * block is applied as one 32x32 complex matrix (the block's gates multiplied
 * on the device in FP32) in TF32 with a three-product high/low split and an
 * FP32 accumulator in tensor memory.  Results agree with the CUDA-core
 * kernel to about 1e-6 relative per block, not bit for bit.  on = 0 keeps
 * every pass on the CUDA cores.  Takes effect for batch plans built after
 * the call.  Replaces the dense per-gate update of the reference's batched
 * QV kernel (bwk/csrc/qv8_sim_sm120.cu:58-117).                            */
int qs_set_tensor_cores(qs_handle_t h, int on);
/* Test hook for the above: mode 1 = the next pipelined tile pass this handle
 * launches withholds its first tile's copy; mode 2 = the next persistent
 * batch launch leaves one pass of one state uncounted, so the state's next
 * pass never sees it finished.  Either way the waits get 50 ms, run out,
 * and qs_device_status reports them; the hook then switches itself off.
 * No reference counterpart.                                                */
int qs_set_wait_test(qs_handle_t h, int mode);

/* ------------------------------------------------------------ states ----- */
/* Reference: bwk/csrc/apply_diagonal_sm120.cu:109-113,210-224 (state_init) */
int qs_state_init(qs_handle_t h, void* state, int n_qubits);
/* |index> basis state (generalises state_init).                            */
int qs_state_init_basis(qs_handle_t h, void* state, int n_qubits, uint64_t index);
/* Reference: bwk/csrc/batch_sm120.cu:165-181 (state_init_batched)          */
int qs_state_init_batched(qs_handle_t h, void* states, int n_states, int n_qubits);
/* State buffers for callers without their own allocator (the reference's
 * states are torch tensors, `torch::zeros` in apply_diagonal_sm120.cu:
 * 210-224): 2^n complex64 from the stream-ordered pool of the handle's
 * stream (256-byte aligned; QS_ERR_NOMEM when HBM is short), freed in stream
 * order.  The copies are synchronous (they return when the data is there).
 * Any other 16-byte aligned device buffer of 2^n complex64 is a valid state. */
int qs_state_alloc(qs_handle_t h, int n_qubits, void** state_out);
int qs_state_free(qs_handle_t h, void* state);
int qs_state_copy_to_host(qs_handle_t h, const void* state, int n_qubits, void* host_c64);
int qs_state_copy_from_host(qs_handle_t h, void* state, int n_qubits, const void* host_c64);

/* ------------------------------------------------------- single gates ---- */
/* Reference: bwk/csrc/apply_gate_sm120.cu:65-114,269-307 (apply_gate).     */
int qs_apply_1q(qs_handle_t h, void* state, int n_qubits, const float* gate_c64, int target);
/* Reference: bwk/csrc/apply_gate2q_sm120.cu:84-228,232-280 (apply_gate_2q).
 * Unlike the reference (which always maps bit 0 to min(q0,q1)), bit 0 of the
 * matrix index is q0 here; blackwell_kernels.apply_gate_2q sorts the qubits to
 * keep the reference's call semantics.                                      */
int qs_apply_2q(qs_handle_t h, void* state, int n_qubits, const float* gate_c64, int q0, int q1);
/* Reference: bwk/csrc/apply_diagonal_sm120.cu:43-59,118-146 (apply_diagonal) */
int qs_apply_diag1(qs_handle_t h, void* state, int n_qubits, const float* diag_c64, int target);
/* The same four gates with the matrix in DEVICE memory (complex64,
 * row-major; the diagonal as 2 complex64): the kernel reads it, so no host
 * copy and no stream synchronisation per call.  This is how the reference's
 * bindings take their gate tensors (bwk/csrc/apply_gate_sm120.cu:274-277,
 * apply_gate2q_sm120.cu:239-242, apply_diagonal_sm120.cu:124-127,
 * apply_mcgate_sm120.cu:109: the gate must be a CUDA tensor).  The pointer is
 * checked to be device or managed memory.                                   */
int qs_apply_1q_dev(qs_handle_t h, void* state, int n_qubits, const void* gate_dev, int target);
int qs_apply_2q_dev(qs_handle_t h, void* state, int n_qubits, const void* gate_dev, int q0, int q1);
int qs_apply_diag1_dev(qs_handle_t h, void* state, int n_qubits, const void* diag_dev, int target);
int qs_apply_mc1q_dev(qs_handle_t h, void* state, int n_qubits, const void* gate_dev, const int* controls,
                      int n_controls, int target);
/* Reference: bwk/csrc/apply_diagonal_sm120.cu:177-208 (apply_diagonal_2q with
 * a CUDA tensor): as qs_apply_diag2 with the 4 diagonal entries in device
 * memory (complex64), read by the kernel.                                  */
int qs_apply_diag2_dev(qs_handle_t h, void* state, int n_qubits, const void* diag_dev, int q0, int q1);
/* Reference: bwk/csrc/apply_mc2qgate_sm120.cu:127-196 (apply_mc2qgate with a
 * CUDA tensor): as qs_apply_mc2q with the 4x4 in device memory.           */
int qs_apply_mc2q_dev(qs_handle_t h, void* state, int n_qubits, const void* gate_dev, const int* controls,
                      int n_controls, int t0, int t1);
/* Reference: bwk/csrc/apply_diagonal_sm120.cu:64-83,150-175 (apply_diagonal_phase) */
int qs_apply_phase(qs_handle_t h, void* state, int n_qubits, float phase_re, float phase_im, int target);
/* Reference: bwk/csrc/apply_diagonal_sm120.cu:88-105,177-208 (apply_diagonal_2q);
 * diag index = b(q1)<<1 | b(q0) with q0 < q1 as in the reference.          */
int qs_apply_diag2(qs_handle_t h, void* state, int n_qubits, const float* diag_c64, int q0, int q1);
/* Reference: bwk/csrc/apply_mcgate_sm120.cu:74-165 (apply_mcgate).         */
int qs_apply_mc1q(qs_handle_t h, void* state, int n_qubits, const float* gate_c64,
                  const int* controls, int n_controls, int target);
/* Reference: bwk/csrc/apply_mc2qgate_sm120.cu:88-196 (apply_mc2qgate);
 * bit 0 of the 4x4 index = min(t0,t1) as in the reference.                  */
int qs_apply_mc2q(qs_handle_t h, void* state, int n_qubits, const float* gate_c64,
                  const int* controls, int n_controls, int t0, int t1);
/* Exact permutation / sign kernels (X, CNOT, Toffoli, SWAP, CSWAP, Z, CZ):
 * values are moved or negated, never multiplied.  Reference: the same gates
 * go through apply_mcgate / apply_gate_2q with 0/1 matrices
 * (blackwell_backend/simulator.py:456-461, bwk/python/blackwell_kernels/cuquantum.py:150-171). */
int qs_apply_mcx(qs_handle_t h, void* state, int n_qubits, const int* controls, int n_controls, int target);
int qs_apply_mcswap(qs_handle_t h, void* state, int n_qubits, const int* controls, int n_controls, int t0, int t1);
int qs_apply_mcz(qs_handle_t h, void* state, int n_qubits, const int* qubits, int n);
/* Reference: bwk/csrc/apply_gate_sm120.cu:121-161,179-234,238-350
 * (apply_gates_fused, apply_gates_reg_tiled): K 1Q gates in one launch.     */
int qs_apply_gates_fused(qs_handle_t h, void* state, int n_qubits, const float* gates_c64,
                         const int* targets, int n_gates);
/* The same with the matrices (n_gates x 2x2 complex64, row-major) and the
 * targets (n_gates int32) in device memory of the handle's GPU: one launch per
 * 12 gates, no host copy, no stream synchronisation (the reference's
 * apply_gates_fused also reads device tensors: bwk/python/blackwell_kernels/
 * cuquantum.py:69-80).  Each launch stages tiles of min(n, 12) qubits that
 * hold the gates' targets and applies the gates in order in shared memory
 * (FP32 FMA chains: within ~1e-7 relative per gate of one qs_apply_1q_dev
 * call per gate, whose compensated products cost 4x the arithmetic).  A target
 * outside [0, n) is found on the device: that launch leaves the state
 * unchanged and ORs 16 into the device status word (qs_device_status).      */
int qs_apply_gates_fused_dev(qs_handle_t h, void* state, int n_qubits, const void* gates_dev,
                             const void* targets_dev, int n_gates);
/* Reference: bwk/csrc/batch_sm120.cu:53-102,185-228 (apply_gate_batched):
 * one 2x2 gate on n_states equal-width states stored back to back.          */
int qs_apply_1q_batched(qs_handle_t h, void* states, int n_states, int n_qubits,
                        const float* gate_c64, int target);
/* Reference: bwk/csrc/batch_sm120.cu:110-161,230-257 (apply_gates_batched_fused). */
int qs_apply_gates_batched_fused(qs_handle_t h, void* states, int n_states, int n_qubits,
                                 const float* gates_c64, const int* targets, int n_gates);

/* ---------------------------------------------------------- programs ----- */
/* Reference: blackwell_backend/simulator.py:247-468 (_compile_circuit 6-phase
 * fusion + _execute_compiled).  The planner fuses in FP64 on the host and cuts
 * the circuit into tile passes; each pass streams the state once.           */
int qs_plan_create(qs_handle_t h, int n_qubits, const qs_op* ops, int n_ops, qs_plan_t* out);
int qs_plan_info_get(qs_plan_t plan, qs_plan_info* info);
int qs_plan_execute(qs_handle_t h, qs_plan_t plan, void* state);
/* state := U|0..0>; the first pass synthesises |0..0> in shared memory, so
 * the state is written but never read. */
int qs_plan_execute_from_zero(qs_handle_t h, qs_plan_t plan, void* state);
/* The device program is freed in order after the work queued on the stream
 * the plan last ran on (destroy the plan before destroying that stream).   */
int qs_plan_destroy(qs_plan_t plan);
/* Host-only dry run of the planner (no device needed): fills `info` for the
 * plan qs_plan_create would build with the given tile bits (0 = default). */
int qs_plan_analyze(int n_qubits, const qs_op* ops, int n_ops, int tile_bits, qs_plan_info* info);
/* Host-only check of pass specialisation (no device needed): builds the plan
 * and compiles every pass with NVRTC without loading it.  Returns QS_OK and
 * the pass count, or QS_ERR_INVALID with the compiler's message.            */
int qs_plan_jit_check(int n_qubits, const qs_op* ops, int n_ops, int tile_bits, int block_bits, int* n_passes);
/* Host-only: the device program (passes back to back, each starting with its
 * pass header) the planner emits for these ops, copied to `out` when `cap`
 * is large enough; `*needed` = its size in bytes.  `specialised` != 0 plans
 * for specialised passes (dense two-qubit gates split into their Cartan
 * form).  For inspection and tests of the planner; no reference counterpart. */
int qs_plan_program(int n_qubits, const qs_op* ops, int n_ops, int tile_bits, int block_bits, int specialised,
                    void* out, size_t cap, size_t* needed);
/* plan + execute in one call.  The handle keeps the plans of its 16 most
 * recent circuits (of at most 4096 ops): running the same op records again
 * on the same stream reuses the plan without planning or upload.  Also what
 * qs_apply_gates_fused runs through.                                        */
int qs_run_circuit(qs_handle_t h, void* state, int n_qubits, const qs_op* ops, int n_ops);

/* ------------------------------------------------------- reductions ------ */
/* All reductions accumulate in FP64 in a fixed order: results are
 * bit-reproducible run to run and independent of batching.                 */
/* Reference: bwk/csrc/renorm_sm120.cu:23-50 (norm_reduce)                   */
int qs_norm2(qs_handle_t h, const void* state, int n_qubits, double* out_host);
/* Reference: bwk/csrc/renorm_sm120.cu:54-108 (renormalize)                  */
int qs_renorm(qs_handle_t h, void* state, int n_qubits);
/* Reference: bwk/csrc/measure_sm120.cu:115-130,186-207 (measure_probs)     */
int qs_probs(qs_handle_t h, const void* state, int n_qubits, float* probs_dev);
/* |a_i|^2 of n_amps (even) consecutive amplitudes, e.g. equal-width states
 * packed back to back (reference: qv8_sim_sm120.cu returns [C, 256] probs). */
int qs_probs_n(qs_handle_t h, const void* states, int64_t n_amps, float* probs_dev);
/* Reference: bwk/csrc/measure_sm120.cu:32-107,150-184 (measure_qubit).
 * Outcome 0 iff u < P(bit=0); the state collapses in place.                */
int qs_measure(qs_handle_t h, void* state, int n_qubits, int target, double u, int* outcome_host);
/* Reference: bwk/csrc/sample_sm120.cu:29-132 (sample).  shot k = smallest i
 * with cdf[i] >= u[k] (cdf accumulated in FP64), clamped to 2^n-1.
 * u_dev: device float64 [n_shots]; out_dev: device int64 [n_shots].         */
int qs_sample(qs_handle_t h, const void* state, int n_qubits, const double* u_dev,
              int64_t n_shots, int64_t* out_dev);
/* Shots from many states of any widths in three launches (no reference
 * counterpart; the reference samples one state per call).  State t starts at
 * amplitude state_offsets[t] of `states` and has widths[t] qubits; its
 * shots[t] shots go to out_dev in state order.  Shot k of state t uses value
 * k of seeds[t]'s splitmix64 uniform stream (the serving runtime's), drawn on
 * the device; each state's CDF and search are exactly qs_sample's, so the
 * shots equal qs_sample's with those uniforms.  widths, state_offsets, shots
 * and seeds are host arrays.                                                */
int qs_sample_batched(qs_handle_t h, const void* states, int n_states, const int32_t* widths,
                      const int64_t* state_offsets, const int64_t* shots, const uint64_t* seeds, int64_t* out_dev);
/* Reference: blackwell_backend/simulator.py:579-586 (the counts loop over the
 * shots).  Histogram of n_shots outcomes held on the device (e.g. qs_sample's
 * output): a hash table in the handle's scratch counts them on the GPU and
 * only the distinct outcomes come back, as n_distinct (outcome, count) int64
 * pairs in pairs_host (room for `capacity` pairs; QS_ERR_INVALID if there
 * are more, with *n_distinct set so the caller can retry).  The pairs come
 * in no particular order.  Waits for the handle's stream.                  */
int qs_counts(qs_handle_t h, const int64_t* shots_dev, int64_t n_shots, int64_t* pairs_host, int64_t capacity,
              int64_t* n_distinct);
/* Reference: bwk/csrc/expectation_sm120.cu:45-80,179-202 (expectation_z)    */
int qs_expect_z(qs_handle_t h, const void* state, int n_qubits, uint64_t z_mask, double* out_host);
/* Reference: bwk/csrc/expectation_sm120.cu:100-163,204-239 (expectation_pauli),
 * generalised to any X/Y/Z string: term t = coef[t] * X^x Z^z with Y counted
 * in both masks (P = i^{|x&z|} X^x Z^z).  out = sum_t coef_t <psi|P_t|psi>. */
int qs_expect_pauli_sum(qs_handle_t h, const void* state, int n_qubits,
                        const uint64_t* x_masks, const uint64_t* z_masks, const double* coefs,
                        int n_terms, double* out_host);

/* No counterpart in the reference.  Same result as qs_expect_pauli_sum, but
 * the call allocates nothing: no cudaMalloc/cudaFree, no pinned host memory.
 * For callers that cannot let a library allocate behind their back (a runtime
 * that owns all device memory through its own arena and budget, or a
 * latency-critical loop that must not pay cudaMalloc/cudaFree's implicit
 * synchronisation).  Its scratch is a fixed static device array (~40 KiB per
 * GPU, held until exit): at most QS_NOALLOC_MAX_TERMS terms, larger requests
 * fail with QS_ERR_INVALID.  All calls share that array: calls that overlap on
 * the GPU race and must be serialised by the caller.  The first call on a
 * device looks up the array's address (cudaGetSymbolAddress); make it before
 * any stream capture begins.  With lazy module loading (the CUDA default)
 * that first call is also when the driver places the array in device
 * memory, so a caller that accounts for every byte makes a warm-up call at
 * start-up.  The address is kept until exit: do not use the library on a
 * device after cudaDeviceReset. */
#define QS_NOALLOC_MAX_TERMS 1024
int qs_expect_pauli_sum_noalloc(qs_handle_t h, const void* state, int n_qubits,
                                const uint64_t* x_masks, const uint64_t* z_masks, const double* coefs,
                                int n_terms, double* out_host);

/* --------------------------------------------------------- Chebyshev ----- */
/* Reference: bwk/csrc/spmv_sm120.cu:61-142 (spmv_csr): y = a*A*x + b*y with a
 * Kahan-compensated row sum.  row_ptr/col_idx int32, values complex64.      */
int qs_spmv_csr(qs_handle_t h, const int32_t* row_ptr, const int32_t* col_idx, const void* values,
                int64_t n_rows, const void* x, void* y,
                double alpha_re, double alpha_im, double beta_re, double beta_im);
/* Reference: bwk/csrc/chebyshev_sm120.cu:24-91,97-159                       */
int qs_cheb_step(qs_handle_t h, const void* spmv_result, const void* t_prev, void* t_next, int64_t n);
int qs_cheb_accum(qs_handle_t h, void* accum, const void* t_k, double c_re, double c_im, int64_t n);
int qs_cheb_step_accum(qs_handle_t h, const void* spmv_result, const void* t_prev, void* t_next,
                       void* accum, double c_re, double c_im, int64_t n);
/* Reference: blackwell_backend/chebyshev.py:81-172 (chebyshev_evolve).  The
 * whole recurrence: one fused launch per degree (SpMV + step + accumulate),
 * no host round trip.  coeffs: host complex128 [K+1].  work: device buffer of
 * 3 * 2^n complex64.  out receives sum_k c_k T_k(scale*H) psi.             */
int qs_cheb_evolve(qs_handle_t h, const int32_t* row_ptr, const int32_t* col_idx, const void* values,
                   int n_qubits, const void* psi, void* out, const double* coeffs, int K,
                   double scale, void* work);

/* Matrix-free form of qs_cheb_evolve: H = sum_t coefs[t] P_t given by Pauli
 * masks (as qs_expect_pauli_sum), applied on the fly, so no CSR bytes are
 * read (the reference always builds a CSR, blackwell_backend/hamiltonian.py:45-69).
 * work: 2 * 2^n complex64.  Up to 32 qubits the terms without X or Y factors
 * are tabulated once as a real diagonal (4 B per amplitude, a stream-ordered
 * allocation freed by the call) and the others are paired by X mask. */
int qs_cheb_evolve_pauli(qs_handle_t h, int n_qubits, const void* psi, void* out, const uint64_t* x_masks,
                         const uint64_t* z_masks, const double* coefs, int n_terms, const double* coeffs, int K,
                         double scale, void* work);

/* ------------------------------------------------------------ batch ------ */
/* Many independent circuits of uneven width, states packed back to back.
 * ops for circuit c are ops[op_offsets[c] .. op_offsets[c+1]); its state
 * starts at amplitude state_offsets[c] of `states`.  States are initialised
 * to |0..0> by the call.  Large batches are planned in up to 8 slices, each
 * launched as soon as it is planned (host planning overlaps the GPU); if a
 * later slice fails to plan, earlier ones have run and the error is returned
 * after they finish.  Reference precedent: bwk/csrc/qv8_sim_sm120.cu:58-151,
 * bwk/csrc/batch_sm120.cu:53-279 (fixed widths only).                       */
int qs_batch_run(qs_handle_t h, int n_circuits, const int32_t* widths, const int64_t* op_offsets,
                 const qs_op* ops, void* states, const int64_t* state_offsets);
/* Reusable form: plan once (host FP64 fusion, per-circuit passes grouped into
 * launches by pass level and tile size), execute many times (e.g. under a
 * CUDA graph; execution issues no host-device copies). */
typedef struct qs_batch_plan_s* qs_batch_plan_t;
typedef struct qs_batch_info {
  int32_t n_circuits;
  int32_t n_launches;
  int64_t n_items;        /* (circuit, pass) pairs                           */
  int32_t max_passes;
  int32_t n_tc_launches;  /* of n_launches, those on the tensor cores        */
  double  bytes_moved;    /* HBM bytes of all passes (first passes write only) */
  double  flops;          /* FP32 flop estimate                              */
} qs_batch_info;
int qs_batch_plan_create(qs_handle_t h, int n_circuits, const int32_t* widths, const int64_t* op_offsets,
                         const qs_op* ops, const int64_t* state_offsets, qs_batch_plan_t* out);
int qs_batch_plan_execute(qs_handle_t h, qs_batch_plan_t plan, void* states);
int qs_batch_plan_info_get(qs_batch_plan_t plan, qs_batch_info* info);
int qs_batch_plan_destroy(qs_batch_plan_t plan);
/* Autotuner for the generic pass kernel (no reference counterpart): for each
 * distinct width 10..24 of the batch, times every tile width (12..14; the
 * whole state up to 14 qubits) and register-block width (2..5) on the first
 * circuit of that width and records the fastest per (device, width).  Every
 * later generic plan on that device and width (batches, single circuits,
 * the adjoint forward pass) uses the entry while the handle's tile and block
 * bits are 0 (automatic), so a circuit gives the same bits alone and in a
 * batch.  Synchronises the handle's stream.                                 */
int qs_autotune_batch(qs_handle_t h, int n_circuits, const int32_t* widths, const int64_t* op_offsets,
                      const qs_op* ops);
/* The tuned (tile bits, block bits) for a width; QS_ERR_INVALID if none.    */
int qs_autotune_get(int device, int width, int* tile_bits, int* block_bits);
/* Records a (tile bits, block bits) entry for a width as the autotuner would
 * (a table saved from an earlier process, or a fixed shape for profiling);
 * QS_ERR_INVALID outside tile bits 10..14, block bits 2..5.                 */
int qs_autotune_set(int device, int width, int tile_bits, int block_bits);
/* Forget the tuned entries of a device (device < 0: all devices).           */
int qs_autotune_clear(int device);

/* ---------------------------------------------------------- adjoint ------ */
/* Adjoint-method gradient of E(theta) = <psi(theta)|H|psi(theta)> for a
 * parametrised circuit (no reference counterpart; ROADMAP.md:173-175).
 * ops carry QS_OP_RX/RY/RZ with param >= 0; params: host [n_batch][n_params]
 * values overriding m[0]; energies_host [n_batch]; grads_host
 * [n_batch][n_params] accumulated in FP64.  work: device buffer of
 * 3 * 2^n complex64 per batch entry (n_batch * 3 * 2^n).                    */
int qs_adjoint_gradient(qs_handle_t h, int n_qubits, const qs_op* ops, int n_ops, int n_params,
                        const double* params, int n_batch,
                        const uint64_t* x_masks, const uint64_t* z_masks, const double* coefs, int n_terms,
                        void* work, double* energies_host, double* grads_host);
/* ------------------------------------------------------------ serving ---- */
/* Native continuous-batching server (no reference counterpart).  Requests
 * are submitted from any thread and get an id; a scheduler admits them in
 * arrival order against `budget_bytes` of HBM (each request counts the device
 * bytes it will hold), batches admitted circuits into one batch plan, and
 * `n_workers` worker threads, each with its own handle and stream, run the
 * items concurrently.  Results are the same alone and in a mix.  Errors:
 * too large for the budget -> QS_ERR_BUDGET at submit; deadline (seconds,
 * 0 = none) passed while queued -> QS_ERR_TIMEOUT; cancelled while queued or
 * at shutdown -> QS_ERR_CANCELLED; a failed item fails only its requests.  */
typedef struct qs_server_s* qs_server_t;
typedef struct qs_server_stats {
  int64_t submitted, completed, failed, queued;
  double  p50_ms, p99_ms;        /* latency (arrival -> result) of completed requests */
  double  throughput_rps;        /* completed / (last completion - first arrival)    */
  int64_t budget_bytes, free_bytes;
} qs_server_stats;
int qs_server_create(int device, int64_t budget_bytes, int n_workers, qs_server_t* out);
/* Cancels queued requests, lets admitted ones finish, joins the threads.    */
int qs_server_destroy(qs_server_t server);
/* Circuit -> `shots` samples (basis indices) drawn with uniforms from `seed`. */
int qs_server_submit_circuit(qs_server_t server, int n_qubits, const qs_op* ops, int n_ops, int64_t shots,
                             uint64_t seed, double deadline_s, int64_t* id_out);
/* Energy and adjoint gradient (as qs_adjoint_gradient) for n_batch vectors. */
int qs_server_submit_gradient(qs_server_t server, int n_qubits, const qs_op* ops, int n_ops, int n_params,
                              const double* params, int n_batch, const uint64_t* x_masks, const uint64_t* z_masks,
                              const double* coefs, int n_terms, double deadline_s, int64_t* id_out);
/* Chebyshev evolution (as qs_cheb_evolve_pauli) of a host complex64 psi0;
 * cheb_coeffs: K+1 complex FP64 coefficients.                               */
int qs_server_submit_evolution(qs_server_t server, int n_qubits, const void* psi0_host, const uint64_t* x_masks,
                               const uint64_t* z_masks, const double* coefs, int n_terms, const double* cheb_coeffs,
                               int K, double scale, double deadline_s, int64_t* id_out);
/* Waits for a request (timeout_s < 0: forever; QS_ERR_TIMEOUT if not done);
 * *status_out = the request's own status.                                   */
int qs_server_wait(qs_server_t server, int64_t id, double timeout_s, int* status_out);
int qs_server_cancel(qs_server_t server, int64_t id);
const char* qs_server_request_error(qs_server_t server, int64_t id);
int qs_server_result_samples(qs_server_t server, int64_t id, int64_t* out, int64_t n_shots);
int qs_server_result_gradient(qs_server_t server, int64_t id, double* energies, double* grads);
int qs_server_result_state(qs_server_t server, int64_t id, void* out_host_c64);
/* Forgets a finished request and its results.                               */
int qs_server_release(qs_server_t server, int64_t id);
int qs_server_stats_get(qs_server_t server, qs_server_stats* out);

/* lambda = H psi for a Pauli sum (matrix-free).                             */
int qs_apply_pauli_sum(qs_handle_t h, const void* psi, void* out, int n_qubits,
                       const uint64_t* x_masks, const uint64_t* z_masks, const double* coefs, int n_terms);

/* ------------------------------------------------------------ noise ------ */
/* Stochastic channels on one state (reference: bwk/csrc/noise_sm120.cu:238-373,
 * bound as apply_depolarizing / apply_amplitude_damping / apply_dephasing in
 * bwk/python/blackwell_kernels/cuquantum.py:352-411).  u is the caller's
 * uniform in [0, 1).  Depolarizing: [0, 1-p) identity, then X, Y, Z in
 * thirds of p (branch 0..3), chosen on the host.  Damping and dephasing pick
 * the jump branch (1) when u < p1 = g * P(q=1) (FP64 fixed-order reduction,
 * decided on the device) and renormalise the kept branch exactly.  When
 * branch_host is non-null the call waits for the branch and stores it;
 * with NULL nothing waits (the reference always synchronises).
 * Differs from the reference: its damping jump kernel keeps the |0>
 * amplitudes (noise_sm120.cu:200-204), which is not E1 and leaves the state
 * unnormalised; here the jump branch is E1 exactly.                         */
int qs_apply_depolarizing(qs_handle_t h, void* state, int n_qubits, int target, double p, double u,
                          int32_t* branch_host);
int qs_apply_amplitude_damping(qs_handle_t h, void* state, int n_qubits, int target, double gamma, double u,
                               int32_t* branch_host);
int qs_apply_dephasing(qs_handle_t h, void* state, int n_qubits, int target, double lambda, double u,
                       int32_t* branch_host);
/* Batched noise trajectories (no reference counterpart; the reference
 * applies one channel per call with a host round trip each): n_traj
 * independent runs of one circuit whose ops may include QS_OP_DEPOLARIZE,
 * QS_OP_AMP_DAMP and QS_OP_DEPHASE.  Trajectory t's uniform for noise op
 * k (in program order) is value k of the splitmix64 stream of seeds[t] (top
 * 53 bits, the serving runtime's sampling stream), so a trajectory gives the
 * same result alone or in any batch.  Up to 14 qubits every channel is
 * applied inside the tile-pass program and each trajectory runs start to
 * finish in one CTA's shared memory (one program for all trajectories, one
 * launch per program level); wider states run the unitary segments as batch
 * launches (depolarizing outcomes drawn on the host become Paulis fused by
 * the planner) and each damping / dephasing channel as two launches over all
 * trajectories.  states: device [n_traj][2^n] complex64, written from
 * |0..0>.  branches_host (optional): [n_traj][n_noise] uint8, the branch of
 * every noise op (depolarizing 0..3, damping/dephasing 0/1).               */
int qs_noise_trajectories(qs_handle_t h, int n_qubits, const qs_op* ops, int n_ops, int n_traj,
                          const uint64_t* seeds, void* states, uint8_t* branches_host);
/* Host-only inspection (no GPU needed; no reference counterpart): the
 * whole-state device program qs_noise_trajectories runs for a noisy circuit
 * of 1..14 qubits (passes back to back, as qs_plan_program; channel groups
 * are blocks with pos[6] = 1).  block_bits 0 = automatic.  Writes it to out
 * when cap suffices; *needed = its size in bytes.                           */
int qs_noise_program(int n_qubits, const qs_op* ops, int n_ops, int block_bits, void* out, size_t cap,
                     size_t* needed);

#ifdef __cplusplus
}
#endif
#endif /* QSIM_H */
