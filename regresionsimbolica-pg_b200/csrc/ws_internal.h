// ws_internal.h -- host-side helpers shared by the translation units of libwarpsym.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>
#include <string>

#include <nvtx3/nvToolsExt.h>

#include "../../include/warpsym.h"
#include "ws_bounds.cuh"
#include "ws_ops.cuh"

namespace ws {

// Scoped NVTX range around a pipeline stage: visible to Nsight tools (`ncu --nvtx
// --nvtx-include "ws_eval_fitness/"` captures only that stage's kernels); a call without an
// attached tool is a no-op (header-only NVTX v3, nothing to link).
class NvtxRange {
 public:
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// Thread-local message of the last failed API call (read back by ws_last_error()).
void set_error(const std::string& msg);
void clear_error();

// Returns WS_ERR_INVALID_ARGUMENT with `msg` recorded.
ws_status fail(const std::string& msg);
ws_status fail_cuda(cudaError_t e, const char* where);

// Builds the token lookup table from the reference's scalar IDs.  `fused_order` selects the
// unary comparison order of rpn_eval_fused_kernel (rpn_kernels.cu:2381-2398) instead of
// rpn_eval_kernel's (rpn_kernels.cu:329-346); they differ only when two operators share an ID.
TokenLut build_lut(const ws_token_map& m, int64_t num_vars, bool fused_order);

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Device properties cached per device.
struct DeviceInfo {
  int sm_count;
  size_t smem_optin;
};
const DeviceInfo& device_info();

// Workspace layout of the fitness evaluator for B programs of L tokens.
struct FitnessWorkspace {
  size_t hdr_off, tape_off, part_off, cnt_off, misc_off, perm_off, bins_off, gspill_off;
  size_t probof_off, desc_off, lut_off, yvar_off;
  size_t gspill_bytes, total;
  int64_t max_partials;  // partial records available (B * n_splits must not exceed it)
};
// One problem (single-problem calls) with the default partial-record area.
FitnessWorkspace fitness_workspace_layout(int64_t B, int64_t L, int dtype);
// Programs of n_prob problems (total_B in all) with n_part partial records.
FitnessWorkspace fitness_workspace_layout(int64_t total_B, int64_t L, int dtype, int64_t n_prob,
                                          int64_t n_part);

// One problem of a (possibly batched) fitness launch.
struct ProblemRequest {
  const uint8_t* pop;
  int64_t B;
  const void* x;
  int64_t V, D;
  const void* consts;
  int64_t K;
  const void* y;
  void* out_loss;
  int32_t* out_ninv;
  TokenLut lut;
};
// Batches of problems evaluated by one launch sequence (ws_fitness.cu): the handle holds the
// plan; descriptors live in the caller's workspace.
ws_status batch_workspace_bytes(int dtype, const ProblemRequest* probs, int n, int64_t L,
                                int strict, int schedule, size_t* out);
ws_status batch_create(int dtype, const ProblemRequest* probs, int n, int64_t L, int strict,
                       int policy, int loss, int schedule, double invalid_value, void* workspace,
                       size_t workspace_bytes, cudaStream_t stream, void** out);
ws_status batch_eval(void* handle, int phase, cudaStream_t stream);
void batch_set_cancel(void* handle, const int32_t* flag);
void batch_destroy(void* handle);
int64_t batch_info(void* handle, int what);

// Launch of the compile + evaluate pipeline (ws_fitness.cu).
struct FitnessRequest {
  int dtype;
  const uint8_t* pop;
  int64_t B, L;
  const void* x;
  int64_t V, D;
  const void* consts;
  int64_t K;
  const void* y;
  void* out_loss;
  int32_t* out_ninv;
  int strict, policy, loss, schedule, phase;
  double invalid_value;
  TokenLut lut;
  void* workspace;
  size_t workspace_bytes;
  cudaStream_t stream;
};
ws_status launch_fitness(const FitnessRequest& rq);

// Number of evaluator schedules (index 0 = automatic choice).
int schedule_count();

// Loss (mean squared error against y) and its adjoint gradient with respect to the constants,
// under the adjoint kernel's forward rules (ws_backward.cu).  part_loss [B * n_splits] and
// part_grad [B * n_splits, K] receive per-row-range partial sums; with `loss` non-null a second
// launch reduces them into loss [B] (double) and grad [B, K] (T).  Programs with active[b] == 0
// are skipped.  With part_loss null only *n_splits_out is computed.
template <typename T>
ws_status launch_loss_grad(const uint8_t* pop, int64_t B, int64_t L, const void* x, int64_t D,
                           const void* consts, int64_t K, const void* y, const int32_t* active,
                           const ws_token_map& ids, int64_t num_vars, double* part_loss,
                           double* part_grad, double* loss, void* grad, int32_t* buckets,
                           int64_t* n_splits_out, cudaStream_t stream);
// Bytes of the `buckets` scratch of launch_loss_grad (programs grouped by operator count, each
// group launched with a tape sized for it); null buckets: one launch sized for L.
size_t loss_grad_bucket_bytes(int64_t B);

}  // namespace ws
