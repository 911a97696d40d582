// ws_static.cu -- fitness evaluation without any device allocation by the caller.
//
// ws_eval_fitness needs a device workspace (program tapes, headers, sort permutation, partial
// sums).  Some callers cannot provide one at the point of the call: a host runtime that reaches
// this library through a plain C FFI and only holds device pointers handed over by another
// framework (it has no device allocator of its own), or a latency-sensitive loop that must not
// call cudaMalloc because cudaMalloc synchronises the device.  ws_eval_fitness_static serves them:
// its scratch is the fixed-size array below, part of the library's own device image, so every GPU
// that loads libwarpsym holds these 64 MiB until the process exits.
//
// Rules of use:
//   * the request's workspace must fit: ws_fitness_workspace_bytes(B, L, dtype) <= 64 MiB; the
//     largest B for a given L and dtype follows from that function (it includes a deep-spill
//     area proportional to the GPU's SM count, ~19 MB for 64-token FP32 programs on 148 SMs,
//     plus ~560 bytes per 64-token FP32 program); larger requests are rejected with a clear error
//     and nothing is launched;
//   * all calls share the one array and it keeps the last call's contents; the pipeline clears
//     what must start at zero (queue head, sort bins, split counters) itself, but two calls whose
//     work overlaps on the GPU (different streams, or different host threads) race on it --
//     serialise them;
//   * each call looks up the array's device address on the current device (cudaGetSymbolAddress,
//     with that device current), so that a context re-created after a device reset (the array
//     then lives in a new context) is followed; the lookup can load the module, so make the first
//     call on each device before any stream capture begins.  While the stream is being captured
//     the lookup is skipped and the address remembered from the last lookup is used.
#include <cuda_runtime.h>
#include <cstdint>
#include <mutex>
#include <string>

#include "ws_internal.h"

namespace ws {

constexpr size_t kStaticScratchBytes = 64ull << 20;

// The scratch itself.  In host code `g_static_scratch` is only a host-side stand-in for the
// symbol, not a device address: a kernel must be given the address obtained below.
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// Device address of g_static_scratch on the current device: looked up afresh when `stream` is not
// being captured (so a context re-created after a device reset is followed), the address
// remembered from the last such lookup when it is.
static ws_status static_scratch_address(cudaStream_t stream, void** out) {
  static std::mutex mu;
  static void* addr[64] = {nullptr};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail_cuda(e, "cudaGetDevice");
  if (dev < 0 || dev >= 64) return fail("device index out of range for the static scratch");
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &cs) != cudaSuccess) {
    (void)cudaGetLastError();  // e.g. the legacy stream while another stream captures globally
    cs = cudaStreamCaptureStatusActive;
  }
  std::lock_guard<std::mutex> g(mu);
  if (cs == cudaStreamCaptureStatusNone) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess) return fail_cuda(e, "cudaGetSymbolAddress(static scratch)");
    addr[dev] = p;
  } else if (addr[dev] == nullptr) {
    return fail("ws_eval_fitness_static: the first call on a device must come before stream "
                "capture (it looks up the static scratch's address)");
  }
  *out = addr[dev];
  return WS_OK;
}

}  // namespace ws

using namespace ws;

extern "C" {

size_t ws_static_scratch_bytes(void) { return kStaticScratchBytes; }

ws_status ws_eval_fitness_static(int32_t dtype, const uint8_t* population, int64_t B, int64_t L,
                                 const void* x, int64_t num_vars, int64_t D,
                                 const void* constants, int64_t K, const void* y, void* out_loss,
                                 int32_t* out_ninvalid, const ws_token_map* ids,
                                 const ws_fitness_opts* opts, void* stream) {
  clear_error();
  NvtxRange nvtx("ws_eval_fitness_static");
  const int64_t Bn = B < 0 ? 0 : B, Ln = L < 0 ? 0 : L;
  const size_t need = ws_fitness_workspace_bytes(Bn, Ln, dtype);
  if (need > kStaticScratchBytes) {
    return fail("request needs " + std::to_string(need) + " bytes of scratch; the static scratch of "
                "ws_eval_fitness_static holds " + std::to_string(kStaticScratchBytes) +
                " bytes (evaluate fewer programs per call, or use ws_eval_fitness with a workspace)");
  }
  void* scratch = nullptr;
  ws_status st = static_scratch_address(static_cast<cudaStream_t>(stream), &scratch);
  if (st != WS_OK) return st;
  return ws_eval_fitness(dtype, population, B, L, x, num_vars, D, constants, K, y, out_loss,
                         out_ninvalid, ids, opts, scratch, kStaticScratchBytes, stream);
}

}  // extern "C"
