// ws_capi.cu -- extern "C" entry points of libwarpsym (declared in include/warpsym.h).
#include <cuda_runtime.h>
#include <cstdint>
#include <atomic>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "ws_internal.h"

namespace ws {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
void clear_error() { g_last_error.clear(); }

ws_status fail(const std::string& msg) {
  set_error(msg);
  return WS_ERR_INVALID_ARGUMENT;
}

ws_status fail_cuda(cudaError_t e, const char* where) {
  set_error(std::string("CUDA error in ") + where + ": " + cudaGetErrorString(e));
  return WS_ERR_CUDA;
}

// ---- bounds-checked build: the host word and the device modules' readers -----------------
namespace {
std::atomic<unsigned long long> g_bc_host{0ull};
std::mutex& bc_mutex() {
  static std::mutex mu;
  return mu;
}
std::vector<BcReader>& bc_readers() {
  static std::vector<BcReader> readers;
  return readers;
}
}  // namespace

void bc_host_fail(uint32_t site, uint32_t idx) {
  unsigned long long none = 0ull;
  g_bc_host.compare_exchange_strong(none, ((unsigned long long)site << 32) | idx);
}

int bc_register(BcReader reader) {
  std::lock_guard<std::mutex> g(bc_mutex());
  bc_readers().push_back(reader);
  return (int)bc_readers().size();
}

const DeviceInfo& device_info() {
  static std::mutex mu;
  static DeviceInfo cache[64];
  static bool have[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  std::lock_guard<std::mutex> g(mu);
  if (!have[dev]) {
    int sms = 0, optin = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cache[dev].sm_count = sms > 0 ? sms : 1;
    cache[dev].smem_optin = optin > 0 ? (size_t)optin : 48 * 1024;
    have[dev] = true;
  }
  return cache[dev];
}

// Token classification with the reference's precedence (rpn_kernels.cu:249-346): PAD first,
// then the variable range [id_x_start, id_x_start + num_vars), C, the literals, the binary
// operators (add, sub, mul, div, pow, else mod), then the unary operators in the order the
// chosen kernel compares them; anything else is an unknown token (an error when executed).
TokenLut build_lut(const ws_token_map& m, int64_t num_vars, bool fused_order) {
  TokenLut lut;
  std::memset(&lut, 0, sizeof(lut));
  const double lits[N_LITERALS] = {0.0, 1.0, 2.0, 3.0, 4.0, 5.0, 6.0, 10.0, m.pi_val, m.e_val};
  for (int i = 0; i < N_LITERALS; ++i) lut.lit[i] = lits[i];
  const int lit_ids[N_LITERALS] = {m.id_0, m.id_1, m.id_2, m.id_3, m.id_4,
                                   m.id_5, m.id_6, m.id_10, m.id_pi, m.id_e};
  const int bin_ids[6] = {m.op_add, m.op_sub, m.op_mul, m.op_div, m.op_pow, m.op_mod};
  const uint8_t bin_cls[6] = {T_ADD, T_SUB, T_MUL, T_DIV, T_POW, T_MOD};
  // rpn_eval_kernel order (rpn_kernels.cu:329-345)
  const int un_ids_classic[17] = {m.op_lgamma, m.op_fact, m.op_sqrt, m.op_exp,  m.op_log,  m.op_sin,
                                  m.op_cos,    m.op_tan,  m.op_abs,  m.op_neg,  m.op_floor, m.op_ceil,
                                  m.op_sign,   m.op_asin, m.op_acos, m.op_atan, m.op_gamma};
  const uint8_t un_cls_classic[17] = {T_LGAMMA, T_FACT, T_SQRT, T_EXP,  T_LOG,  T_SIN,
                                      T_COS,    T_TAN,  T_ABS,  T_NEG,  T_FLOOR, T_CEIL,
                                      T_SIGN,   T_ASIN, T_ACOS, T_ATAN, T_GAMMA};
  // rpn_eval_fused_kernel order (rpn_kernels.cu:2381-2397)
  const int un_ids_fused[17] = {m.op_lgamma, m.op_fact, m.op_sqrt, m.op_exp,  m.op_log,   m.op_sin,
                                m.op_cos,    m.op_tan,  m.op_abs,  m.op_neg,  m.op_gamma, m.op_asin,
                                m.op_acos,   m.op_atan, m.op_floor, m.op_ceil, m.op_sign};
  const uint8_t un_cls_fused[17] = {T_LGAMMA, T_FACT, T_SQRT, T_EXP,  T_LOG,   T_SIN,
                                    T_COS,    T_TAN,  T_ABS,  T_NEG,  T_GAMMA, T_ASIN,
                                    T_ACOS,   T_ATAN, T_FLOOR, T_CEIL, T_SIGN};
  const int* un_ids = fused_order ? un_ids_fused : un_ids_classic;
  const uint8_t* un_cls = fused_order ? un_cls_fused : un_cls_classic;

  for (int t = 0; t < 256; ++t) {
    uint8_t cls = T_UNKNOWN, arg = 0;
    if (t == m.pad_id) {
      cls = T_PAD;
    } else if ((int64_t)t >= (int64_t)m.id_x_start && (int64_t)t < (int64_t)m.id_x_start + num_vars) {
      cls = T_VAR;
      arg = (uint8_t)(t - m.id_x_start);
    } else if (t == m.id_C) {
      cls = T_CONST;
    } else {
      bool done = false;
      for (int i = 0; i < N_LITERALS && !done; ++i)
        if (t == lit_ids[i]) { cls = T_LIT; arg = (uint8_t)i; done = true; }
      for (int i = 0; i < 6 && !done; ++i)
        if (t == bin_ids[i]) { cls = bin_cls[i]; done = true; }
      for (int i = 0; i < 17 && !done; ++i)
        if (t == un_ids[i]) { cls = un_cls[i]; done = true; }
    }
    lut.cls[t] = cls;
    lut.arg[t] = arg;
  }
  return lut;
}

ws_status launch_eval_rows(int dtype, const uint8_t* pop, int64_t B, int64_t L, const void* x,
                           int64_t D, const void* consts, int64_t K, const TokenLut& lut,
                           void* out_preds, int32_t* out_sp, uint8_t* out_err, int strict,
                           cudaStream_t stream);

}  // namespace ws

using namespace ws;

extern "C" {

const char* ws_version(void) { return "warpsym 0.1.0 (sm_100a)"; }

const char* ws_last_error(void) { return g_last_error.c_str(); }

ws_status ws_bounds_status(int32_t* enabled_out, uint64_t* word_out, int32_t reset) {
  clear_error();
  if (!enabled_out || !word_out) return fail("null output pointer");
#ifdef WS_BOUNDS_CHECK
  *enabled_out = 1;
  unsigned long long w = g_bc_host.load();
  if (reset) g_bc_host.store(0ull);
  int n_dev = 0;
  if (cudaGetDeviceCount(&n_dev) == cudaSuccess && n_dev > 0) {
    std::lock_guard<std::mutex> g(bc_mutex());
    for (BcReader r : bc_readers()) {
      const unsigned long long v = r(reset != 0);
      if (w == 0ull) w = v;
    }
  } else {
    (void)cudaGetLastError();
  }
  *word_out = w;
#else
  (void)reset;
  *enabled_out = 0;
  *word_out = 0;
#endif
  return WS_OK;
}

ws_status ws_debug_bounds_selftest(uint64_t* word_out) {
  clear_error();
  if (!word_out) return fail("null output pointer");
#ifdef WS_BOUNDS_CHECK
  // a host array read with indices 0..5 of which 4 and 5 are out of range: both are skipped,
  // the first is recorded
  const int arr[4] = {1, 2, 3, 4};
  int sum = 0;
  g_bc_host.store(0ull);
  for (int i = 0; i < 6; ++i)
    if (WS_BC(i < 4, BC_SELFTEST, i)) sum += arr[i];
  *word_out = g_bc_host.exchange(0ull);
  if (sum != 10) return fail("bounds self-test: an out-of-range access was not skipped");
  return WS_OK;
#else
  *word_out = 0;
  return fail("not a bounds-checked build (libwarpsym_bc.so is)");
#endif
}

size_t ws_fitness_workspace_bytes(int64_t B, int64_t L, int32_t dtype) {
  if (B < 0) B = 0;
  if (L < 0) L = 0;
  return fitness_workspace_layout(B, L, dtype).total;
}

int32_t ws_schedule_count(void) { return schedule_count(); }

ws_status ws_eval_rpn(int32_t dtype, const uint8_t* population, int64_t B, int64_t L,
                      const void* x, int64_t num_vars, int64_t D, const void* constants,
                      int64_t K, void* out_preds, int32_t* out_sp, uint8_t* out_error,
                      const ws_token_map* ids, int32_t strict_mode, void* stream) {
  clear_error();
  NvtxRange nvtx("ws_eval_rpn");
  if (dtype != WS_F32 && dtype != WS_F64) return fail("x must be float32 or float64");
  if (!ids) return fail("token map is required");
  if (B < 0 || L < 0 || D < 0 || K < 0 || num_vars < 0) return fail("negative dimension");
  if (num_vars > 255) return fail("at most 255 variables are addressable by uint8 tokens");
  if (B * D == 0) return WS_OK;
  if (!population && L > 0) return fail("population pointer is null");
  if (!x && num_vars > 0) return fail("x pointer is null");
  if (K > 0 && !constants) return fail("constants pointer is null");
  if (!out_preds || !out_sp || !out_error) return fail("output pointer is null");
  const TokenLut lut = build_lut(*ids, num_vars, false);
  return launch_eval_rows(dtype, population, B, L, x, D, K > 0 ? constants : nullptr, K, lut,
                          out_preds, out_sp, out_error, strict_mode ? 1 : 0,
                          (cudaStream_t)stream);
}

static ws_status check_workspace(int64_t B, int64_t L, int32_t dtype, void* workspace,
                                 size_t bytes) {
  const size_t need = fitness_workspace_layout(B, L, dtype).total;
  if (!workspace || bytes < need) {
    set_error("workspace of " + std::to_string(need) + " bytes required (got " +
              std::to_string(bytes) + ")");
    return WS_ERR_WORKSPACE;
  }
  if (((uintptr_t)workspace & 255u) != 0) {
    set_error("workspace must be 256-byte aligned");
    return WS_ERR_WORKSPACE;
  }
  return WS_OK;
}

ws_status ws_eval_rpn_fused(int32_t dtype, const uint8_t* population, int64_t B, int64_t L,
                            const void* x, int64_t num_vars, int64_t D, const void* constants,
                            int64_t K, const void* y, void* out_rmse, const ws_token_map* ids,
                            int32_t strict_mode, int32_t launch_mode, void* workspace,
                            size_t workspace_bytes, void* stream) {
  (void)launch_mode;
  clear_error();
  NvtxRange nvtx("ws_eval_rpn_fused");
  if (dtype != WS_F32 && dtype != WS_F64) return fail("x must be float32 or float64");
  if (!ids) return fail("token map is required");
  // argument checks of launch_rpn_eval_fused, in its order (rpn_kernels.cu:2539-2545)
  if (!(B > 0 && L > 0)) return fail("population must be non-empty");
  if (!(num_vars > 0 && num_vars <= 4)) return fail("fused evaluator supports 1..4 variables");
  if (L > 256) return fail("fused evaluator program length exceeds 256");
  if (!(D > 0 && D <= 1024)) return fail("fused evaluator supports 1..1024 samples");
  if (K < 0) return fail("constants must have shape [B, K]");
  if (!population || !x || !y || !out_rmse || (K > 0 && !constants))
    return fail("null tensor pointer");
  ws_status st = check_workspace(B, L, dtype, workspace, workspace_bytes);
  if (st != WS_OK) return st;
  FitnessRequest rq;
  rq.dtype = dtype;
  rq.pop = population;
  rq.B = B;
  rq.L = L;
  rq.x = x;
  rq.V = num_vars;
  rq.D = D;
  rq.consts = K > 0 ? constants : nullptr;
  rq.K = K;
  rq.y = y;
  rq.out_loss = out_rmse;
  rq.out_ninv = nullptr;
  rq.strict = strict_mode ? 1 : 0;
  rq.policy = WS_POLICY_FUSED;
  rq.loss = WS_LOSS_RMSE;
  rq.schedule = 0;
  rq.phase = WS_PHASE_ALL;
  rq.invalid_value = dtype == WS_F32 ? (double)Limits<float>::invalid : Limits<double>::invalid;
  rq.lut = build_lut(*ids, num_vars, true);
  rq.workspace = workspace;
  rq.workspace_bytes = workspace_bytes;
  rq.stream = (cudaStream_t)stream;
  return launch_fitness(rq);
}

ws_status ws_eval_fitness(int32_t dtype, const uint8_t* population, int64_t B, int64_t L,
                          const void* x, int64_t num_vars, int64_t D, const void* constants,
                          int64_t K, const void* y, void* out_loss, int32_t* out_ninvalid,
                          const ws_token_map* ids, const ws_fitness_opts* opts,
                          void* workspace, size_t workspace_bytes, void* stream) {
  clear_error();
  if (dtype != WS_F32 && dtype != WS_F64) return fail("x must be float32 or float64");
  if (!ids || !opts) return fail("token map and options are required");
  if (B < 0 || L < 0 || K < 0) return fail("negative dimension");
  if (L > 256) return fail("program length exceeds 256");
  if (num_vars < 0 || num_vars > 64) return fail("supports 0..64 variables");
  if (D < 1 || D > (int64_t)INT32_MAX) return fail("supports 1..2^31-1 samples");
  if (opts->policy != WS_POLICY_FUSED && opts->policy != WS_POLICY_CLASSIC)
    return fail("unknown policy");
  if (opts->loss < WS_LOSS_RMSE || opts->loss > WS_LOSS_SSE) return fail("unknown loss");
  if (opts->schedule < 0 || opts->schedule >= ws_schedule_count())
    return fail("schedule index out of range");
  if (opts->phase < WS_PHASE_ALL || opts->phase > WS_PHASE_EVALUATE) return fail("unknown phase");
  if (B == 0) return WS_OK;
  if ((!population && L > 0) || (!x && num_vars > 0) || !y || !out_loss || (K > 0 && !constants))
    return fail("null tensor pointer");
  ws_status st = check_workspace(B, L, dtype, workspace, workspace_bytes);
  if (st != WS_OK) return st;
  FitnessRequest rq;
  rq.dtype = dtype;
  rq.pop = population;
  rq.B = B;
  rq.L = L;
  rq.x = x;
  rq.V = num_vars;
  rq.D = D;
  rq.consts = K > 0 ? constants : nullptr;
  rq.K = K;
  rq.y = y;
  rq.out_loss = out_loss;
  rq.out_ninv = out_ninvalid;
  rq.strict = opts->strict_mode ? 1 : 0;
  rq.policy = opts->policy;
  rq.loss = opts->loss;
  rq.schedule = opts->schedule;
  rq.phase = opts->phase;
  rq.invalid_value = opts->invalid_value;
  rq.lut = build_lut(*ids, num_vars, opts->policy == WS_POLICY_FUSED);
  rq.workspace = workspace;
  rq.workspace_bytes = workspace_bytes;
  rq.stream = (cudaStream_t)stream;
  return launch_fitness(rq);
}

static ws_status batch_requests(int32_t dtype, const ws_problem* problems, int32_t n,
                                int64_t L, const ws_fitness_opts* opts,
                                std::vector<ProblemRequest>& out) {
  if (dtype != WS_F32 && dtype != WS_F64) return fail("x must be float32 or float64");
  if (!opts) return fail("options are required");
  if (n < 0 || (n > 0 && !problems)) return fail("problem list is null");
  if (L < 1 || L > 256) return fail("program length must be in 1..256");
  if (opts->policy != WS_POLICY_FUSED && opts->policy != WS_POLICY_CLASSIC)
    return fail("unknown policy");
  if (opts->loss < WS_LOSS_RMSE || opts->loss > WS_LOSS_SSE) return fail("unknown loss");
  if (opts->schedule < 0 || opts->schedule >= ws_schedule_count())
    return fail("schedule index out of range");
  out.clear();
  for (int32_t i = 0; i < n; ++i) {
    const ws_problem& q = problems[i];
    const std::string at = "problem " + std::to_string(i) + ": ";
    if (!q.ids) return fail(at + "token map is required");
    if (q.B < 0 || q.K < 0) return fail(at + "negative dimension");
    if (q.num_vars < 0 || q.num_vars > 64) return fail(at + "supports 0..64 variables");
    if (q.D < 1 || q.D > (int64_t)INT32_MAX) return fail(at + "supports 1..2^31-1 samples");
    if (q.B > 0 && (!q.population || (!q.x && q.num_vars > 0) || !q.y || !q.out_loss ||
                    (q.K > 0 && !q.constants)))
      return fail(at + "null tensor pointer");
    ProblemRequest r;
    r.pop = q.population;
    r.B = q.B;
    r.x = q.x;
    r.V = q.num_vars;
    r.D = q.D;
    r.consts = q.K > 0 ? q.constants : nullptr;
    r.K = q.K;
    r.y = q.y;
    r.out_loss = q.out_loss;
    r.out_ninv = q.out_ninvalid;
    r.lut = build_lut(*q.ids, q.num_vars, opts->policy == WS_POLICY_FUSED);
    out.push_back(r);
  }
  return WS_OK;
}

ws_status ws_batch_workspace_bytes(int32_t dtype, const ws_problem* problems, int32_t n_problems,
                                   int64_t L, const ws_fitness_opts* opts, size_t* out_bytes) {
  clear_error();
  if (!out_bytes) return fail("out_bytes is null");
  std::vector<ProblemRequest> rq;
  ws_status st = batch_requests(dtype, problems, n_problems, L, opts, rq);
  if (st != WS_OK) return st;
  return batch_workspace_bytes(dtype, rq.data(), (int)rq.size(), L, opts->strict_mode ? 1 : 0,
                               opts->schedule, out_bytes);
}

ws_status ws_batch_create(int32_t dtype, const ws_problem* problems, int32_t n_problems, int64_t L,
                          const ws_fitness_opts* opts, void* workspace, size_t workspace_bytes,
                          void* stream, ws_batch** out_batch) {
  clear_error();
  if (!out_batch) return fail("out_batch is null");
  *out_batch = nullptr;
  std::vector<ProblemRequest> rq;
  ws_status st = batch_requests(dtype, problems, n_problems, L, opts, rq);
  if (st != WS_OK) return st;
  void* h = nullptr;
  st = batch_create(dtype, rq.data(), (int)rq.size(), L, opts->strict_mode ? 1 : 0, opts->policy,
                    opts->loss, opts->schedule, opts->invalid_value, workspace, workspace_bytes,
                    (cudaStream_t)stream, &h);
  if (st == WS_OK) *out_batch = static_cast<ws_batch*>(h);
  return st;
}

ws_status ws_batch_eval(ws_batch* batch, int32_t phase, void* stream) {
  clear_error();
  if (!batch) return fail("batch is null");
  if (phase < WS_PHASE_ALL || phase > WS_PHASE_EVALUATE) return fail("unknown phase");
  return batch_eval(batch, phase, (cudaStream_t)stream);
}

int64_t ws_batch_info(const ws_batch* batch, int32_t what) {
  if (!batch) return -1;
  return batch_info(const_cast<ws_batch*>(batch), what);
}

ws_status ws_batch_set_cancel(ws_batch* batch, const int32_t* device_flag) {
  clear_error();
  if (!batch) return fail("batch is null");
  batch_set_cancel(batch, device_flag);
  return WS_OK;
}

void ws_batch_destroy(ws_batch* batch) {
  if (batch) batch_destroy(batch);
}

}  // extern "C"
