/*
 * warpsym.h -- C ABI of the B200-native evaluation and constant-fitting core.
 *
 * This library replaces the native extension `rpn_cuda_native` of WarpSymbolic
 * (src/warpsymbolic/gpu/cuda/, pybind11 exports in bindings.cpp:434-581).  Every entry point
 * below names the reference interface it stands in for.  The contract is plain C: raw device
 * pointers, element counts and a CUDA stream (passed as `void*`, a `cudaStream_t`), no torch
 * types.  The Python drop-in module `rpn_cuda_native.py` binds these symbols with ctypes.
 *
 * Conventions shared by every entry point
 *   - All array arguments are DEVICE pointers to contiguous row-major storage, unless a
 *     parameter says "host".  Layouts are the reference's: population uint8 [B, L]
 *     (PAD-terminated, left-packed), x [num_vars, D] (variables-major), constants [B, K],
 *     y [D].
 *   - Outputs are caller-allocated and written in place (bindings.cpp contract).
 *   - Work is enqueued on `stream` (NULL = legacy default stream); nothing synchronises the
 *     host.  Entry points never allocate device memory: scratch comes from a caller-provided
 *     workspace whose size is given by the matching *_workspace_bytes() query.
 *   - Return value: WS_OK or an error code; ws_last_error() returns the message (the text the
 *     reference's TORCH_CHECK would raise where the same check exists).
 *   - dtype: WS_F32 or WS_F64 for x / constants / y / floating outputs (the reference
 *     dispatches both via AT_DISPATCH_FLOATING_TYPES).
 */
#ifndef WARPSYM_H
#define WARPSYM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t ws_status;

enum {
  WS_OK = 0,
  WS_ERR_INVALID_ARGUMENT = 1, /* shape / dtype / envelope check failed            */
  WS_ERR_CUDA = 2,             /* a CUDA runtime call or launch failed              */
  WS_ERR_WORKSPACE = 3,        /* workspace pointer missing or too small            */
  WS_ERR_UNSUPPORTED = 4       /* request outside what this build implements       */
};

enum { WS_F32 = 0, WS_F64 = 1 };

/* Fitness semantics: which reference code path's validity / overflow rules to reproduce. */
enum {
  WS_POLICY_FUSED = 0,   /* rpn_eval_fused_kernel epilogue, rpn_kernels.cu:2405-2501          */
  WS_POLICY_CLASSIC = 1  /* GPUEvaluator.evaluate_batch classic path, evaluation.py:153-189   */
};

/* Per-program loss written by ws_eval_fitness. */
enum {
  WS_LOSS_RMSE = 0,  /* sqrt(mean squared error) -- the reference's fitness                 */
  WS_LOSS_MSE = 1,   /* mean squared error                                                   */
  WS_LOSS_R2 = 2,    /* 1 - MSE / Var(y), Var over the same rows in FP64                     */
  WS_LOSS_SSE = 3    /* raw sum of squared errors, always written as double                  */
};

/*
 * Token-ID map.  The reference passes these ~40 scalars to every evaluator entry point
 * (bindings.cpp:7-27, cuda_vm.py:34-82): absent tokens carry -100 / -1 / -999 and never match a
 * uint8 token.  Field order follows the reference's argument order.
 */
typedef struct ws_token_map {
  int32_t pad_id, id_x_start;
  int32_t id_C, id_pi, id_e;
  int32_t id_0, id_1, id_2, id_3, id_4, id_5, id_6, id_10;
  int32_t op_add, op_sub, op_mul, op_div, op_pow, op_mod;
  int32_t op_sin, op_cos, op_tan, op_log, op_exp;
  int32_t op_sqrt, op_abs, op_neg;
  int32_t op_fact, op_floor, op_ceil, op_sign;
  int32_t op_gamma, op_lgamma;
  int32_t op_asin, op_acos, op_atan;
  double pi_val, e_val;
} ws_token_map;

/* Phases of ws_eval_fitness: both (the normal call), or one of them.  An evaluate-only call
 * reuses the tape that a compile-only call with the same population, constants, L, dtype and
 * strict_mode left in the same workspace (used to time the evaluation kernel alone). */
enum { WS_PHASE_ALL = 0, WS_PHASE_COMPILE = 1, WS_PHASE_EVALUATE = 2 };

/* Options of the general fitness evaluator. */
typedef struct ws_fitness_opts {
  int32_t strict_mode;   /* 0 = protected operators (search), 1 = strict domain errors      */
  int32_t policy;        /* WS_POLICY_FUSED or WS_POLICY_CLASSIC                              */
  int32_t loss;          /* WS_LOSS_*                                                         */
  int32_t schedule;      /* 0 = autotuned; otherwise an index into ws_schedule_count()        */
  double invalid_value;  /* loss written for invalid programs (reference: 1e15 f32, 1e100 f64) */
  int32_t phase;         /* WS_PHASE_*                                                        */
  int32_t reserved;
} ws_fitness_opts;

/* Library identification (host). */
const char* ws_version(void);

/* Message of the most recent failed call on this host thread ("" when none). */
const char* ws_last_error(void);

/*
 * Bounds-checked build (no counterpart in the reference, whose kernels rely on TORCH_CHECK shape
 * guards, rpn_kernels.cu:2536-2557).  libwarpsym_bc.so is this library compiled with
 * -DWS_BOUNDS_CHECK: its kernels test their shared- and global-memory indices against the
 * extents of the buffers they address; an index out of range is recorded (the first per device
 * module: check site << 32 | index) and its access skipped, never faulting.  Load it in place of
 * libwarpsym.so (the Python package reads WARPSYM_LIB) to run small shapes under the checks.
 *   ws_bounds_status          -- enabled_out = 1 in the checked build (0 here, word_out then 0);
 *                                word_out = the first recorded violation, host-side checks first,
 *                                then the device modules' (read when a device is present);
 *                                reset != 0 clears the records.
 *   ws_debug_bounds_selftest  -- checked build only, host only: reads a 4-element host array at
 *                                indices 0..5 under the check; word_out = the record
 *                                ((99 << 32) | 4), and the two out-of-range reads are skipped.
 */
ws_status ws_bounds_status(int32_t* enabled_out, uint64_t* word_out, int32_t reset);
ws_status ws_debug_bounds_selftest(uint64_t* word_out);

/*
 * Classic per-(program,row) interpreter.  Replaces `eval_rpn` (bindings.cpp:434 ->
 * launch_rpn_kernel, rpn_kernels.cu:361-429; kernel rpn_kernels.cu:202-358).
 * Writes out_preds[B*D] (dtype), out_sp[B*D] (int32), out_error[B*D] (uint8) exactly as the
 * reference does (stack top or 1e30, final stack depth, error byte).  K == 0 allowed
 * (constants may be NULL; `C` then pushes 1.0).  Indices are 64-bit (no B*D < 2^31 limit).
 */
ws_status ws_eval_rpn(int32_t dtype, const uint8_t* population, int64_t B, int64_t L,
                      const void* x, int64_t num_vars, int64_t D, const void* constants,
                      int64_t K, void* out_preds, int32_t* out_sp, uint8_t* out_error,
                      const ws_token_map* ids, int32_t strict_mode, void* stream);

/*
 * Fused evaluation + RMSE.  Replaces `eval_rpn_fused` (bindings.cpp:436 ->
 * launch_rpn_eval_fused, rpn_kernels.cu:2505-2594) with the same argument checks and envelope
 * (1..4 variables, L <= 256, 1 <= D <= 1024, B > 0) and the same error texts; launch_mode
 * (0 = block, 1 = warp in the reference) is validated and otherwise ignored because the
 * schedule here is chosen by the autotuner.  out_rmse[B] uses the reference's sentinels
 * (1e15 / sqrt(1e15) in f32, 1e100 / 1e50 in f64).  Needs ws_fitness_workspace_bytes(B, L).
 */
ws_status ws_eval_rpn_fused(int32_t dtype, const uint8_t* population, int64_t B, int64_t L,
                            const void* x, int64_t num_vars, int64_t D, const void* constants,
                            int64_t K, const void* y, void* out_rmse, const ws_token_map* ids,
                            int32_t strict_mode, int32_t launch_mode, void* workspace,
                            size_t workspace_bytes, void* stream);

/*
 * General batched fitness (no envelope): any number of variables (<= 64), any D >= 1,
 * L <= 256.  This is the hot path behind GPUEvaluator.evaluate_batch (evaluation.py:45-198):
 * both the fused-kernel semantics and the classic chunked-path semantics are available
 * through opts->policy, so one launch replaces the reference's [B, D] materialisation.
 * out_loss[B] has `dtype` (double for WS_LOSS_SSE); out_ninvalid[B] (optional, may be NULL)
 * receives the number of rows whose evaluation is invalid (the reference's per-row
 * `err != 0 | sp != 1 | non-finite` count, evaluation.py:379-382).
 */
ws_status ws_eval_fitness(int32_t dtype, const uint8_t* population, int64_t B, int64_t L,
                          const void* x, int64_t num_vars, int64_t D, const void* constants,
                          int64_t K, const void* y, void* out_loss, int32_t* out_ninvalid,
                          const ws_token_map* ids, const ws_fitness_opts* opts,
                          void* workspace, size_t workspace_bytes, void* stream);

/* Bytes of device workspace ws_eval_fitness / ws_eval_rpn_fused need for B programs of
 * length L (256-byte aligned base required). */
size_t ws_fitness_workspace_bytes(int64_t B, int64_t L, int32_t dtype);

/* Number of compiled (rows-per-thread x warps x rows-per-chunk) schedules. */
int32_t ws_schedule_count(void);

/*
 * ws_eval_fitness without a workspace argument.  No counterpart in the reference.  For callers
 * that cannot allocate device memory at the point of the call -- e.g. a host runtime reaching
 * this library through a plain C FFI with only device pointers handed over by another framework,
 * or a loop that must not call cudaMalloc because it synchronises the device.  The scratch is a
 * static 64 MiB device array inside the library (held by every GPU that loads it until exit);
 * requests whose ws_fitness_workspace_bytes(B, L, dtype) exceed ws_static_scratch_bytes() are
 * rejected with an error.  All calls share the array: calls that overlap on the GPU race and must
 * be serialised.  Each call looks the array's address up on the current device (a context
 * re-created after a device reset is followed); make the first call on each device before any
 * stream capture begins.  Arguments and results are those of ws_eval_fitness.
 */
ws_status ws_eval_fitness_static(int32_t dtype, const uint8_t* population, int64_t B, int64_t L,
                                 const void* x, int64_t num_vars, int64_t D,
                                 const void* constants, int64_t K, const void* y, void* out_loss,
                                 int32_t* out_ninvalid, const ws_token_map* ids,
                                 const ws_fitness_opts* opts, void* stream);

/* Size in bytes of the static scratch used by ws_eval_fitness_static. */
size_t ws_static_scratch_bytes(void);

/*
 * Batched fitness: many independent problems -- each with its own population, constants, data
 * set (rows and variable count), vocabulary and outputs -- scored by ONE launch sequence (one
 * compile kernel, one length sort, one persistent evaluator launch) instead of one
 * `evaluate_batch` call per problem (evaluation.py:45-198, called per dataset by
 * TensorGeneticEngine, engine.py:956,1136).  A problem's results are those of ws_eval_fitness on
 * that problem alone with the same schedule, bit for bit, whatever else is in the batch (chunk
 * sizes and row splits depend on the problem's own shape only).
 *
 *   ws_batch_workspace_bytes  size of the device workspace the batch needs
 *   ws_batch_create           plans the batch (chunk sizes per problem, programs per block, row
 *                             splits, heaviest work first) and writes the problem descriptors
 *                             into the workspace with kernels on `stream` (stream-ordered; no
 *                             host synchronisation), once per set of problems
 *   ws_batch_eval             compile + sort + evaluate on `stream`: kernels and memsets only,
 *                             no host synchronisation or allocation, so a CUDA graph can capture
 *                             it and replay it after the populations / constants are rewritten
 *                             in place (their pointers and shapes are fixed by the plan)
 *   ws_batch_info             plan facts: 0 work items, 1 rows per lane, 2 programs per block,
 *                             3 dynamic shared memory per CTA, 4 resident CTAs, 5 programs
 *   ws_batch_set_cancel       attaches a device int32 flag (NULL detaches).  The evaluator's
 *                             CTAs read it before taking each work item; once it reads nonzero
 *                             the launch takes no further items and ends after those in flight
 *                             (no wait, no trap), leaving its outputs incomplete: the caller who
 *                             set the flag discards them.  With a flag attached every launch
 *                             also resets the per-program split counters, so the next launch
 *                             after a cancelled one is exact.  Works inside captured graphs (the
 *                             flag is read at run time).  No counterpart in the reference.
 *
 * All problems share dtype, program width L (<= 256), strict_mode, policy, loss, schedule and
 * invalid_value (from opts); opts->phase is ignored here (ws_batch_eval takes the phase).
 */
typedef struct ws_problem {
  const uint8_t* population;  /* [B, L] uint8                                              */
  int64_t B;
  const void* x;              /* [num_vars, D] of dtype                                    */
  int64_t num_vars, D;
  const void* constants;      /* [B, K] of dtype, or NULL with K = 0                        */
  int64_t K;
  const void* y;              /* [D] of dtype                                              */
  void* out_loss;             /* [B] of dtype (double for WS_LOSS_SSE)                     */
  int32_t* out_ninvalid;      /* [B] invalid-row counts, or NULL                           */
  const ws_token_map* ids;    /* this problem's token IDs                                  */
} ws_problem;

typedef struct ws_batch ws_batch;

ws_status ws_batch_workspace_bytes(int32_t dtype, const ws_problem* problems, int32_t n_problems,
                                   int64_t L, const ws_fitness_opts* opts, size_t* out_bytes);
ws_status ws_batch_create(int32_t dtype, const ws_problem* problems, int32_t n_problems, int64_t L,
                          const ws_fitness_opts* opts, void* workspace, size_t workspace_bytes,
                          void* stream, ws_batch** out_batch);
ws_status ws_batch_eval(ws_batch* batch, int32_t phase, void* stream);
int64_t ws_batch_info(const ws_batch* batch, int32_t what);
ws_status ws_batch_set_cancel(ws_batch* batch, const int32_t* device_flag);
void ws_batch_destroy(ws_batch* batch);

/*
 * The reference extension's genetic-operator and tracker exports, same inputs -> same outputs.
 *
 * ws_mutate_population replaces `mutate_population` (bindings.cpp:457 -> launch_mutation_kernel,
 *   rpn_kernels.cu:772-845): each non-PAD token with rand_floats[i] < mutation_rate becomes
 *   arity_k_ids[rand_ints[i] % n_k] of its own arity k (token_arities[tok], 0 outside the table).
 * ws_crossover_splicing replaces `crossover_splicing` (bindings.cpp:458 ->
 *   rpn_kernels.cu:927-1016,1266-1300): child1 = p1[0:s1] + p2[s2:e2+1] + p1[e1+1:], child2 the
 *   mirror image, PAD where a source index leaves the row; pairs whose cx_mask byte is 0 copy
 *   their parents (cx_mask may be NULL).
 * ws_constant_perturbation replaces `constant_perturbation` (bindings.cpp:463 ->
 *   rpn_kernels.cu:1455-1535): hash-seeded rows get Box-Muller multiplicative noise, clamped.
 * ws_generate_random_rpn replaces `generate_random_rpn` (bindings.cpp:507 ->
 *   genrand_kernels.cu:70-210): one valid program per row from a per-row xorshift64 stream.
 * ws_update_best / ws_check_improvement / ws_batch_update_best replace `update_best`,
 *   `check_improvement`, `batch_update_best` (bindings.cpp:565-590 ->
 *   best_tracker_kernels.cu:47-340).  The reference's update_best and check_improvement let
 *   several blocks update one result without ordering (best_tracker_kernels.cu:104-135,
 *   :168-172); here one block reduces all programs -- the reference's result whenever it is
 *   deterministic (B <= 256), otherwise the global minimum with its tie rules.
 */
ws_status ws_mutate_population(uint8_t* population, int64_t B, int64_t L, const float* rand_floats,
                               const int64_t* rand_ints, const int32_t* token_arities,
                               int64_t vocab_size, const uint8_t* arity0_ids, int64_t n0,
                               const uint8_t* arity1_ids, int64_t n1, const uint8_t* arity2_ids,
                               int64_t n2, float mutation_rate, int32_t pad_id, void* stream);
ws_status ws_crossover_splicing(const uint8_t* parent1, const uint8_t* parent2, int64_t N,
                                int64_t L, const int64_t* starts1, const int64_t* ends1,
                                const int64_t* starts2, const int64_t* ends2, uint8_t* child1,
                                uint8_t* child2, int32_t pad_id, const uint8_t* cx_mask,
                                void* stream);
ws_status ws_constant_perturbation(int32_t dtype, void* constants, int64_t B, int64_t K,
                                   float rate, float sigma, float c_min, float c_max,
                                   uint32_t seed, void* stream);
ws_status ws_generate_random_rpn(uint8_t* population, int64_t B, int64_t L,
                                 const uint8_t* terminal_ids, int64_t n_terminals,
                                 const uint8_t* unary_ids, int64_t n_unary,
                                 const uint8_t* binary_ids, int64_t n_binary, uint64_t seed,
                                 float term_weight, float unary_weight, float bin_weight,
                                 void* stream);
ws_status ws_update_best(const int64_t* population, int64_t B, int64_t L, const float* constants,
                         int64_t K, const float* fitness, int64_t* tracker_rpn,
                         float* tracker_consts, float* tracker_rmse, int32_t* tracker_idx,
                         int32_t* tracker_gen, int32_t* tracker_len, int32_t* tracker_updated,
                         int32_t current_generation, float tolerance, void* stream);
ws_status ws_check_improvement(const float* fitness, int64_t B, const float* tracked_rmse,
                               int32_t* improved, float tolerance, void* stream);
ws_status ws_batch_update_best(const uint8_t* population, int64_t B, int64_t L,
                               const float* constants, int64_t K, const float* fitness,
                               uint8_t* best_rpn, float* best_consts, float* best_rmse,
                               int32_t* best_idx, float tolerance, void* stream);

/*
 * Structural hashing and deduplication (the reference's diversity exports, bindings.cpp:513-540
 * -> diversity_kernels.cu).
 * ws_population_hashes   replaces `compute_population_hashes` (:29-108): base-31 polynomial hash
 *                        (mod 2^64) up to the first PAD, and the used-variable bitmask
 *                        (var_presence may be NULL; hashes may be NULL for the mask alone, which
 *                        replaces `compute_var_presence`, :465-515).
 * ws_structural_dedup    replaces `structural_dedup` (:121-238): hash_table holds
 *                        ws_dedup_table_slots() int64 entries set to -1 by the caller.  The
 *                        reference lets thread timing pick which member of a group is the
 *                        original; here it is the group's lowest index.
 * ws_count_unique        replaces `count_unique` (:362-405): programs with duplicate flag 0,
 *                        written to out_count[0] on the device.
 * ws_replacement_positions replaces `get_replacement_positions` (:410-460): the duplicates'
 *                        indices in ascending order (the reference's order is timing-dependent)
 *                        and their number in n_replacements[0].
 * ws_fitness_sharing_penalty replaces `fitness_sharing_penalty` (:224-355): keys
 *                        [n_islands * ws_sharing_table_slots()] int64 set to -1 and counts of the
 *                        same size set to 0 by the caller; out_penalty[B] = log2(count) of the
 *                        program's island/prefix-hash group when the count exceeds threshold.
 */
ws_status ws_population_hashes(const uint8_t* population, int64_t B, int64_t L, int64_t* hashes,
                               int32_t* var_presence, int32_t pad_id, int32_t id_x_start,
                               int32_t num_vars, void* stream);
ws_status ws_structural_dedup(const int64_t* hashes, int64_t B, int64_t* hash_table,
                              int32_t* duplicate_mask, int64_t* original_index, void* stream);
ws_status ws_count_unique(const int32_t* duplicate_mask, int64_t B, int64_t* out_count,
                          void* stream);
ws_status ws_replacement_positions(const int32_t* duplicate_mask, int64_t B, int64_t* positions,
                                   int64_t* n_replacements, void* stream);
ws_status ws_fitness_sharing_penalty(const uint8_t* population, int64_t B, int64_t L,
                                     int32_t n_islands, int32_t island_size, int32_t threshold,
                                     int32_t hash_len, int64_t* keys, int32_t* counts,
                                     float* out_penalty, void* stream);
int64_t ws_dedup_table_slots(void);
int64_t ws_sharing_table_slots(void);

/*
 * One genetic-programming generation, in place, for many problems at once.  Replaces the
 * breeding half of `evolve_generation` (rpn_kernels.cu:1810-2237: tournament K16, elitism
 * :1905-1907, subtree crossover K5/K6/K10, same-arity point mutation K7/K11, constant
 * recombination / perturbation K12/K15) with three launches per generation (elite, children,
 * copy-back) and a counter-based generator keyed by (problem seed, generation, child): a
 * problem's offspring are the same alone or batched with others, and graph replays advance each
 * problem's device-side generation counter (ws_gp_set_generation sets them all).  Semantics per child are stated in csrc/ws_gp.cu.
 *   fitness: [B] of dtype, lower is better (e.g. the MSE written by ws_batch_eval)
 *   population / constants: rewritten in place with the next generation
 */
typedef struct ws_gp_problem {
  uint8_t* population;       /* [B, L]                                                   */
  int64_t B;
  void* constants;           /* [B, K] of dtype, or NULL with K = 0 (K <= 64)            */
  int64_t K;
  const void* fitness;       /* [B] of dtype                                             */
  int64_t num_vars;
  const ws_token_map* ids;   /* this problem's token IDs                                 */
  uint64_t seed;             /* this problem's random stream                             */
  uint64_t generation;       /* this problem's next generation number (0 for a new run);
                                the device counter advances by one per ws_gp_step        */
} ws_gp_problem;

typedef struct ws_gp_opts {
  int32_t tournament_size;    /* uniform draws per tournament, >= 1                       */
  int32_t elitism;            /* 1: child 0 is the generation's best program              */
  float crossover_rate;       /* probability that a child splices a second parent's subtree */
  float mutation_rate;        /* per-token probability of a same-arity replacement        */
  float const_mutation_rate;  /* per-constant probability of multiplicative noise         */
  float const_sigma;          /* relative standard deviation of that noise                */
  float parsimony_eps;        /* fitness ties within eps go to the shorter program        */
  int32_t reserved;
} ws_gp_opts;

typedef struct ws_gp ws_gp;

ws_status ws_gp_workspace_bytes(int32_t dtype, const ws_gp_problem* problems, int32_t n_problems,
                                int64_t L, size_t* out_bytes);
ws_status ws_gp_create(int32_t dtype, const ws_gp_problem* problems, int32_t n_problems, int64_t L,
                       const ws_gp_opts* opts, void* workspace, size_t workspace_bytes,
                       void* stream, ws_gp** out);
ws_status ws_gp_step(ws_gp* gp, void* stream);
ws_status ws_gp_set_generation(ws_gp* gp, uint64_t generation, void* stream);
void ws_gp_destroy(ws_gp* gp);

/*
 * Adjoint gradient of program outputs with respect to their constants.  Replaces
 * `eval_rpn_backward` (bindings.cpp:511 -> run_rpn_backward_cuda, bindings.cpp:108-140 ->
 * launch_rpn_backward, backward_kernels.cu:286-335; kernel :13-281).
 *   grad_constants[b, k] += sum over rows d of grad_output[b, d] * d pred[b, d] / d C_k
 * with the reference's forward and adjoint rules (see ws_backward.cu); the caller zeroes
 * grad_constants first, as RPNBackwardFunction does (optimization.py:57).  grad_output [B, D] and
 * grad_constants [B, K] have `dtype`.  L <= 256 (the reference's tapes hold 64 tokens; longer
 * programs follow the same rules).  Programs whose final stack depth is not 1 contribute nothing.
 */
ws_status ws_eval_rpn_backward(int32_t dtype, const uint8_t* population, int64_t B, int64_t L,
                               const void* x, int64_t num_vars, int64_t D, const void* constants,
                               int64_t K, const void* grad_output, void* grad_constants,
                               const ws_token_map* ids, void* stream);
/* The same with caller-provided scratch of ws_eval_rpn_backward_workspace_bytes(B) bytes: the
 * programs are grouped on the device by the tape they need and each group is launched with a
 * tape sized for it (more resident warps than one launch sized for the longest program).  Same
 * results; the Python drop-in's eval_rpn_backward takes this form. */
ws_status ws_eval_rpn_backward_workspace_bytes(int64_t B, size_t* bytes);
ws_status ws_eval_rpn_backward_ws(int32_t dtype, const uint8_t* population, int64_t B, int64_t L,
                                  const void* x, int64_t num_vars, int64_t D,
                                  const void* constants, int64_t K, const void* grad_output,
                                  void* grad_constants, const ws_token_map* ids, void* workspace,
                                  size_t workspace_bytes, void* stream);

/*
 * Loss and constant gradient in one launch, without per-row tensors.  Replaces the closure of the
 * reference's torch L-BFGS (optimization.py:301-311: RPNBackwardFunction forward -> preds [B, D],
 * mse = mean_d (preds - y)^2, loss.backward() -> eval_rpn_backward with
 * grad_output = 2 (preds - y) / D).  Per program b:
 *   out_loss[b]    = mean over rows of (pred[b, d] - y[d])^2                      (double)
 *   out_grad[b, k] = d out_loss[b] / d C_k                                        (`dtype`)
 * with the forward and adjoint rules of ws_eval_rpn_backward, evaluated in `dtype` (without the
 * reference's double promotions, which only bit-exactness against it needs).  A
 * program whose final stack depth is not 1 gets an infinite loss and a zero gradient.  `active`
 * (optional, int32 [B]) skips programs with 0; their outputs are left as they are.  Results are
 * deterministic (partial sums per row range, reduced in a fixed order).  The workspace holds
 * the partial sums; its size depends on (B, L, num_vars, D, K) and the device.
 */
ws_status ws_loss_grad_workspace_bytes(int32_t dtype, int64_t B, int64_t L, int64_t num_vars,
                                       int64_t D, int64_t K, size_t* bytes);
ws_status ws_loss_grad(int32_t dtype, const uint8_t* population, int64_t B, int64_t L,
                       const void* x, int64_t num_vars, int64_t D, const void* constants,
                       int64_t K, const void* y, const int32_t* active, double* out_loss,
                       void* out_grad, const ws_token_map* ids, void* workspace,
                       size_t workspace_bytes, void* stream);

/*
 * Per-program L-BFGS over ws_loss_grad, for populations of any size.  Replaces the reference's
 * large-population constant fitting (`GPUOptimizer._lbfgs_pytorch_fallback`,
 * optimization.py:281-343: torch.optim.LBFGS with a strong-Wolfe line search over the sum of all
 * programs' losses) by one L-BFGS per program with the same algorithm (torch.optim.LBFGS.step,
 * _strong_wolfe, _cubic_interpolate) and the same options, so that for a single program the two
 * visit the same points.  `constants` [B, K] (`dtype`, K <= 32) are updated in place to the last
 * accepted iterate; out_loss [B] (optional) receives its loss, out_evals [B] (optional) the
 * loss evaluations used.  Each round is one loss-and-gradient launch over the programs still
 * running plus one state launch; with sync_every > 0 the active count is read from the device
 * every sync_every rounds (a stream synchronisation), and the call returns once no program runs.
 */
typedef struct ws_lbfgs_opts {
  int32_t max_iter;         /* iterations per program (torch: max_iter) */
  int32_t max_eval;         /* evaluations per program (torch: max_eval; the reference: 2 * max_iter) */
  int32_t history;          /* curvature pairs kept, 1..32 (torch: history_size) */
  int32_t max_ls;           /* evaluations per line search after the first (torch: 25) */
  double lr;                /* initial step scale (torch: lr = 1) */
  double tolerance_grad;    /* stop when max |g| <= this (the reference: 1e-7) */
  double tolerance_change;  /* stop on smaller steps or loss changes (the reference: 1e-9) */
  double grad_clip;         /* gradients clamped to [-clip, clip]; 0 = none (the reference: 1e4) */
  int32_t sync_every;       /* rounds between reads of the active count; 0 = never (capturable) */
  int32_t reserved;
} ws_lbfgs_opts;
ws_status ws_lbfgs_adjoint_workspace_bytes(int32_t dtype, int64_t B, int64_t L,
                                           int64_t num_vars, int64_t D, int64_t K,
                                           int32_t history, size_t* bytes);
ws_status ws_lbfgs_adjoint(int32_t dtype, const uint8_t* population, int64_t B, int64_t L,
                           const void* x, int64_t num_vars, int64_t D, void* constants, int64_t K,
                           const void* y, const ws_lbfgs_opts* opts, double* out_loss,
                           int32_t* out_evals, const ws_token_map* ids, void* workspace,
                           size_t workspace_bytes, void* stream);

/* ----------------------------------------------------------------------------------------------
 * Device steps of one `evolve_generation` call (bindings.cpp:474 -> rpn_kernels.cu:1810-2237).
 * The host sequence -- the torch random draws in the reference's order and the torch glue between
 * the steps -- is rpn_cuda_native.evolve_generation; every step below gives the reference
 * kernel's bytes / floats for the same inputs.  Row-index arrays (int64, device) may be NULL for
 * the identity; uint8 masks are torch bool tensors.
 *
 * ws_subtree_pick replaces select_subtree_range_indirect_kernel (rpn_kernels.cu:597-640): for row
 *   rows[n], len = tokens before PAD (>= 1), end = (int)(u[n] * len) clamped to [0, len),
 *   start = where the arity balance from `end` back closes (end itself for a terminal).
 * ws_splice_valid replaces validate_crossover_lengths_kernel (:642-679) followed by the
 *   reference's logical_and_ with the candidate mask (NULL = all candidates).
 * ws_splice_rows replaces crossover_splicing_mutation_kernel (:1020-1105) when `mutation` is
 *   given and crossover_splicing_kernel (:927-1016) when it is NULL: child rows c1_rows[n] /
 *   c2_rows[n] get p1[0:s1] + p2[s2:e2+1] + p1[e1+1:] and its mirror image (PAD past a source
 *   row), or their parents where cx_mask is 0; then, with a mutation, a child row r != 0 whose
 *   individual_rand[r] < cut has each token point-mutated (Philox4x32-10, see ws_evolve.cu).
 * ws_mutate_rows replaces mutation_philox_indirect_kernel (:747-770).
 * ws_sbx_constants replaces sbx_constants_kernel (:1225-1261); float32 constants.
 * ws_splice_constants replaces crossover_constants_kernel (:1107-1223); float32 constants.
 * ws_hoist_rows replaces hoist_mutation_indirect_kernel (:1363-1411).
 */
typedef struct ws_point_mutation {
  const int32_t* arities;  /* [vocab] token arities (device) */
  int32_t vocab;
  int32_t n0, n1, n2;      /* sizes of the same-arity replacement lists */
  const uint8_t* ids0;     /* [n0] / [n1] / [n2] replacement tokens (device) */
  const uint8_t* ids1;
  const uint8_t* ids2;
  float rate;              /* per-token mutation probability */
  int32_t reserved;
  uint64_t seed, generation;
} ws_point_mutation;
ws_status ws_subtree_pick(const uint8_t* population, const int64_t* rows, int64_t N, int64_t L,
                          const int32_t* arities, int32_t vocab, const float* u, int64_t* out_len,
                          int64_t* out_start, int64_t* out_end, int32_t pad_id, void* stream);
ws_status ws_splice_valid(const int64_t* len1, const int64_t* len2, const int64_t* s1,
                          const int64_t* e1, const int64_t* s2, const int64_t* e2,
                          const uint8_t* candidate, uint8_t* valid, int64_t N, int64_t L,
                          void* stream);
ws_status ws_splice_rows(const uint8_t* parent1, const uint8_t* parent2, const int64_t* p1_rows,
                         const int64_t* p2_rows, const int64_t* c1_rows, const int64_t* c2_rows,
                         const int64_t* s1, const int64_t* e1, const int64_t* s2,
                         const int64_t* e2, const uint8_t* cx_mask, uint8_t* child1,
                         uint8_t* child2, int64_t N, int64_t L, int32_t pad_id,
                         const float* individual_rand, float cut,
                         const ws_point_mutation* mutation, void* stream);
ws_status ws_mutate_rows(uint8_t* population, const int64_t* rows, int64_t N, int64_t L,
                         const float* individual_rand, float cut,
                         const ws_point_mutation* mutation, int32_t pad_id, void* stream);
ws_status ws_sbx_constants(const float* constants, const int64_t* p1_rows, const int64_t* p2_rows,
                           const float* u_sbx, const float* mask_rand, float* out1, float* out2,
                           int64_t n_pairs, int64_t K, float eta, void* stream);
ws_status ws_splice_constants(const uint8_t* population, const int64_t* p1_rows,
                              const int64_t* p2_rows, const float* consts1, const float* consts2,
                              const int64_t* s1, const int64_t* e1, const int64_t* s2,
                              const int64_t* e2, const uint8_t* cx_mask, float* child_consts,
                              const int64_t* c1_rows, const int64_t* c2_rows, int64_t N,
                              int64_t L, int64_t K, int32_t id_C, void* stream);
ws_status ws_hoist_rows(uint8_t* population, const int64_t* rows, int64_t N, int64_t L,
                        const int32_t* arities, int32_t vocab, const int64_t* rand_ints,
                        int32_t pad_id, void* stream);

/* ----------------------------------------------------------------------------------------------
 * Particle-swarm constant fitting.
 */

/*
 * Velocity / position step of every particle.  Replaces `pso_update(pos, vel, pbest, gbest, r1,
 * r2, w, c1, c2)` (bindings.cpp:470 -> launch_pso_update, pso_kernels.cu:155-187; kernel
 * :29-70):  vel = w vel + c1 r1 (pbest - pos) + c2 r2 (gbest[b] - pos);  pos += vel,
 * bit-identical.  pos, vel, pbest, r1, r2: [B, P, K]; gbest: [B, K]; all `dtype`.
 */
ws_status ws_pso_update(int32_t dtype, void* pos, void* vel, const void* pbest,
                        const void* gbest, const void* r1, const void* r2, float w, float c1,
                        float c2, int64_t B, int64_t P, int64_t K, void* stream);

/*
 * Personal and swarm bests.  Replaces `pso_update_bests(current_err, pbest_err, pbest_pos,
 * current_pos, gbest_err, gbest_pos)` (bindings.cpp:471 -> launch_pso_update_bests,
 * pso_kernels.cu:189-233; kernels :74-153) with its tie rules: a particle improves on a strictly
 * smaller error; the swarm best is replaced by the strict minimum of the personal bests, found
 * as the reference finds it (first minimum of each lane's 32-strided particles, then a
 * shuffle-down tree that takes a partner's value only when strictly smaller, which settles
 * ties); errors at or above 1e30 and NaN never win.  current_err, pbest_err: [B, P]; positions [B, P, K];
 * gbest_err [B]; gbest_pos [B, K].
 */
ws_status ws_pso_update_bests(int32_t dtype, const void* current_err, void* pbest_err,
                              void* pbest_pos, const void* current_pos, void* gbest_err,
                              void* gbest_pos, int64_t B, int64_t P, int64_t K, void* stream);

/*
 * The whole PSO loop in one launch.  Replaces `fused_pso(population, init_consts, x, y_target,
 * out_gbest_pos, out_gbest_err, num_particles, num_steps, w, c1, c2, const_min, const_max, <ids>,
 * pi_val, e_val, rng_seed)` (bindings.cpp:510 -> launch_fused_pso, fused_pso_kernels.cu:431-515;
 * kernel :208-427) with the same limits and messages (L <= 256, K <= 16, D <= 1024, particles
 * <= 64, float32 only) and the same results for the same seed: particle p of program b draws
 * curand XORWOW stream seed + b * num_particles + p; particle 0 starts at init_consts, the others
 * jittered by N(0, (0.15 range)^2) and clamped; velocities N(0, (0.02 range)^2); inertia decays
 * linearly from w to 0.4; the fitness is the RMSE under the reference PSO evaluator's rules
 * (fused_pso_kernels.cu:57-197).  Writes out_gbest_pos [B, K] and out_gbest_err [B].
 * K == 0 with a C token evaluates C as 1.0 (the reference reads outside its arrays there).
 */
ws_status ws_fused_pso(int32_t dtype, const uint8_t* population, int64_t B, int64_t L,
                       const void* init_consts, int64_t K, const void* x, int64_t num_vars,
                       int64_t D, const void* y_target, void* out_gbest_pos, void* out_gbest_err,
                       int32_t num_particles, int32_t num_steps, float w, float c1, float c2,
                       float const_min, float const_max, const ws_token_map* ids,
                       uint64_t rng_seed, void* stream);

/*
 * Constant fitting with the reference's L-BFGS kernel.  Replaces `lbfgs_optimize(population,
 * constants, x, y_target, out_rmse, max_iter=20, history_size=10, gtol=1e-7, const_min=-25,
 * const_max=25, <ids>, pi_val, e_val)` (bindings.cpp:542-563 -> launch_lbfgs_optimize,
 * lbfgs_kernels.cu:624-694; kernel :214-621) with its limits and messages (L <= 256, K <= 32,
 * D <= 1024).  constants [B, K] are updated in place; out_rmse [B] receives the final fitness.
 * The fitness, the finite-difference gradient and the iteration are the reference kernel's (see
 * ws_lbfgs.cu): its curvature history never admits a pair, and the history slots it reads
 * without writing are taken as zero.  history_size is accepted and, as in the reference,
 * unused.  K == 0 with a C token evaluates C as 1.0 (the reference reads outside its arrays).
 */
ws_status ws_lbfgs_optimize(int32_t dtype, const uint8_t* population, int64_t B, int64_t L,
                            void* constants, int64_t K, const void* x, int64_t num_vars,
                            int64_t D, const void* y_target, void* out_rmse, int32_t max_iter,
                            int32_t history_size, float gtol, float const_min, float const_max,
                            const ws_token_map* ids, void* stream);

/*
 * RPN -> infix text (host only: HOST pointers, no GPU work).  Replaces `decode_rpn(population,
 * constants, vocab, arities, PAD_ID, precision=4)` (bindings.cpp:450 -> decoder.cpp:32-152)
 * with the same text, character for character.  population uint8 [B, L] and constants [B, K]
 * (const_dtype WS_F32 / WS_F64) are host arrays; vocab[n_vocab] are the token strings by ID,
 * arities[n_arities] the arity by ID.  Writes B NUL-terminated strings into out, string b at
 * offsets[b] (offsets has B + 1 entries, offsets[B] = bytes used).  When out is NULL or
 * out_bytes is too small, returns WS_ERR_WORKSPACE with *needed_bytes set (call again).
 */
ws_status ws_decode_rpn(const uint8_t* population, int64_t B, int64_t L, const void* constants,
                        int32_t const_dtype, int64_t K, const char* const* vocab, int64_t n_vocab,
                        const int32_t* arities, int64_t n_arities, int32_t pad_id,
                        int32_t precision, char* out, size_t out_bytes, int64_t* offsets,
                        size_t* needed_bytes);

/* Operator / literal IDs of the simplifier, in the reference's argument order
 * (simplify_kernels.cu:665-678); absent ones are -1. */
typedef struct ws_simplify_ids {
  int32_t op_plus, op_minus, op_mult, op_div, op_neg, op_mod, op_pow;
  int32_t op_sin, op_cos, op_tan, op_asin, op_acos, op_atan;
  int32_t op_log, op_exp, op_sqrt, op_abs, op_gamma, op_lgamma, op_floor, op_ceil, op_sign;
  int32_t id_0, id_1, id_2, id_3, id_4, id_5, id_6;
} ws_simplify_ids;

/*
 * Rule-based simplification of programs in place.  Replaces `simplify_batch(population,
 * arities, val_table, literal_ids, literal_vals, max_passes, <ids>)` (bindings.cpp:505 ->
 * launch_simplify_batch, simplify_kernels.cu:665-713; kernel :100-601) with identical output
 * programs: the same rules in the same order, the same in-place editing and compaction, the
 * same nearest-literal folding (see ws_simplify.cu).  population int64 [B, L] (PAD = 0; only
 * the first 256 positions are rewritten, as in the reference); arities int32 [max_id];
 * val_table float32 [max_id] (the literal's value, NaN for other tokens); literal_ids int64 /
 * literal_vals float32 [n_literals] (the first 64 are used).
 */
ws_status ws_simplify_batch(int64_t* population, int64_t B, int64_t L, const int32_t* arities,
                            int64_t max_id, const float* val_table, const int64_t* literal_ids,
                            const float* literal_vals, int64_t n_literals, int32_t max_passes,
                            const ws_simplify_ids* ids, void* stream);

/* ----------------------------------------------------------------------------------------------
 * Population structure (integer, bit-exact).  Token arrays are [B, L] row-major; the arity table
 * is int32 [n_arities] indexed by token value (the reference's `token_arities`).
 */

/* Which of the reference's three stack-validity rules ws_validate_rpn_batch applies. */
enum {
  WS_VALIDATE_KERNEL = 0,  /* validate_rpn_batch_kernel, rpn_kernels.cu:850-900: tokens outside
                              the table have arity 0; PAD-contiguity; depth >= 1 after every
                              token; final depth == 1                                          */
  WS_VALIDATE_CLAMPED = 1, /* GPUOperators._validate_rpn_batch torch path, operators.py:551-570
                              (and _validate_rpn_batch_custom, :660-676): as KERNEL but the arity
                              lookup clamps the token into [0, n_arities-1]                     */
  WS_VALIDATE_STACK = 2    /* GPUSymbolicSimplifier._validate_batch_stack,
                              gpu_simplifier.py:513-579: no contiguity rule (a PAD is a no-op
                              anywhere), depth >= 1 at EVERY position, final depth == 1, at least
                              one non-PAD token; clamped lookup                                 */
};

/*
 * Per-program stack validity.  Replaces `validate_rpn_batch(population, token_arities,
 * out_valid, PAD_ID)` (bindings.cpp:462 -> launch_validate_rpn_batch, rpn_kernels.cu:902-925)
 * for mode WS_VALIDATE_KERNEL, and the two torch fallbacks above for the other modes.
 * population: token_bytes 1 (uint8, the kernel's layout) or 8 (int64, the simplifier's layout).
 * out_valid[B]: 1 = valid, 0 = invalid (a torch.bool buffer).
 */
ws_status ws_validate_rpn_batch(const void* population, int32_t token_bytes, int64_t B, int64_t L,
                                const int32_t* token_arities, int64_t n_arities, int32_t pad_id,
                                int32_t mode, uint8_t* out_valid, void* stream);

/*
 * Start of the subtree ending at every position.  Replaces `find_subtree_ranges(population,
 * token_arities, out_starts, PAD_ID, out_lengths=None)` (bindings.cpp:454 ->
 * launch_find_subtree_ranges, rpn_kernels.cu:506-537; kernel :433-504).  out_starts int64 [B, L]
 * (-1 for PAD positions and for operators whose operands are missing), identical to the
 * reference.  out_lengths int64 [B] (optional): position of the first PAD, else L.  On rows that
 * contain a PAD gap the reference's threads race on this value (every PAD that follows a
 * non-PAD, and position L-1 when it is not PAD, store their own candidate); the value written
 * here is always one of those candidates.
 */
ws_status ws_find_subtree_ranges(const uint8_t* population, int64_t B, int64_t L,
                                 const int32_t* token_arities, int64_t n_arities, int32_t pad_id,
                                 int64_t* out_starts, int64_t* out_lengths, void* stream);

/*
 * Subtree starts by the simplifier's forward recurrence.  Replaces
 * `precompute_subtree_starts(population, arities, out_starts)` (bindings.cpp:506 ->
 * launch_precompute_subtree_starts, simplify_kernels.cu:715-737; kernel :612-661).
 * population int64 [B, L]; PAD is token 0; positions >= 256 are -1 (the reference's
 * MAX_FORMULA_LEN).
 */
ws_status ws_precompute_subtree_starts(const int64_t* population, int64_t B, int64_t L,
                                       const int32_t* arities, int64_t n_arities,
                                       int64_t* out_starts, void* stream);

/*
 * Tournament selection.  Replaces `tournament_selection(fitness, errors, rand_idx, rand_cases,
 * selected_idx, lengths, mad_eps=empty)` (bindings.cpp:468 -> launch_tournament_selection,
 * rpn_kernels.cu:1670-1715; kernel :1535-1601).  fitness f32 [B]; errors f32 [B, n_data] or
 * NULL; rand_idx int64 [B, tour_size] (global candidate indices); rand_cases int32 [B] or NULL
 * (lexicase case per slot, < 0 = none); lengths f32 [B] or NULL (parsimony tie-break);
 * mad_eps f32 [n_data] or NULL.  selected_idx int64 [B].  The winner is the first candidate with
 * a strictly smaller value; with lengths, a candidate within epsilon (mad_eps[case], else 1e-3
 * with a case, else 1e-9) that is shorter also wins.  Candidate indices are not range-checked
 * (as in the reference).
 */
ws_status ws_tournament_select(const float* fitness, int64_t B, const float* errors,
                               int64_t n_data, const int64_t* rand_idx, int64_t tour_size,
                               const int32_t* rand_cases, const float* lengths,
                               const float* mad_eps, int64_t* selected_idx, void* stream);

/*
 * Island tournament on int32 offsets: candidate = base + (offset % span), clamped into [0, B-1],
 * where base/span are the island of the slot when n_islands > 1 (span = island_size, the last
 * island truncated), else the whole population.  Replaces launch_tournament_selection_offsets
 * (rpn_kernels.cu:1717-1760; kernel :1603-1668), the selection step of evolve_generation.
 */
ws_status ws_tournament_select_offsets(const float* fitness, int64_t B, const float* errors,
                                       int64_t n_data, const int32_t* rand_offsets,
                                       int64_t tour_size, const int32_t* rand_cases,
                                       const float* lengths, const float* mad_eps,
                                       int32_t island_size, int32_t n_islands,
                                       int64_t* selected_idx, void* stream);

/*
 * Host-only introspection (no GPU needed; not an evaluation path).  They expose the pieces
 * the evaluator is built from so that they can be verified exactly on a CPU:
 *   ws_debug_token_lut  -- token byte -> internal class / argument table built from the IDs
 *                          with the reference's precedence (rpn_kernels.cu:249-346);
 *   ws_debug_compile    -- compiles ONE host program into the evaluator's tape (ctrl words and
 *                          immediates, capacity max(L,1)); hdr_out = {n_instr, status
 *                          (0 ok / 1 statically invalid), spill slots, tokens};
 *   ws_debug_run_tape   -- scalar host interpretation of such a tape over D rows of a host x;
 *   ws_debug_compile_agree -- compiles B host programs with both of the compiler's emitters
 *                          (depth-first and linear) and counts the programs whose tapes differ
 *                          (the device compiles with the linear one).
 */
ws_status ws_debug_token_lut(const ws_token_map* ids, int64_t num_vars, int32_t fused_order,
                             uint8_t* cls_out, uint8_t* arg_out);
ws_status ws_debug_compile(int32_t dtype, const uint8_t* prog, int64_t L, const void* consts,
                           int64_t K, const ws_token_map* ids, int64_t num_vars,
                           int32_t strict_mode, int32_t fused_order, uint32_t* ctrl_out,
                           double* imm_out, int32_t* hdr_out);
ws_status ws_debug_run_tape(int32_t dtype, const uint32_t* ctrl, const double* imm, int32_t n,
                            const void* x, int64_t D, int32_t strict_mode, void* out_pred,
                            uint8_t* out_err);
ws_status ws_debug_compile_agree(int32_t dtype, const uint8_t* progs, int64_t B, int64_t L,
                                 const void* consts, int64_t K, const ws_token_map* ids,
                                 int64_t num_vars, int32_t strict_mode, int32_t fused_order,
                                 int32_t xmul, int64_t* mismatches_out);

#ifdef __cplusplus
}
#endif
#endif /* WARPSYM_H */
