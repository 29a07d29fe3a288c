// evalbox_static.cu — tsi_tape_eval_boxes_static: interval evaluation of a
// tape on device-resident boxes without allocating anything.
//
// tsi_tape_eval_boxes allocates device scratch (one interval register file
// and one operand log per box) with cudaMalloc on first use and whenever a
// call needs more.  Some callers cannot allocate at call time: a render loop
// recorded into a CUDA graph, a host with a fixed memory budget that
// reserves everything at start-up, or an embedding runtime that forbids
// allocation on its request path.  This entry point takes device pointers
// for the boxes and the output and keeps its scratch in the file-scope
// array below, which exists once per device that loads the library and stays
// allocated until the process exits.  Nothing in it needs to start at zero:
// the kernel writes every register and log entry before reading it.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "api_internal.h"
#include "interval.cuh"
#include "tsi.h"

namespace tsi {
cudaError_t launch_evalbox(bool directed, const uint2 *code, uint32_t len, uint32_t nregs, uint32_t out_reg,
                           uint32_t n, const float *boxes, int reverse, float *out, float2 *regs, float4 *log,
                           cudaStream_t st);
cudaError_t evalbox_preload();
}


// Scratch of every call: per box, nregs intervals (8 bytes each) then
// len operand-log entries (16 bytes each), boxes back to back.
static __device__ __align__(256) unsigned char g_static_scratch[TSI_STATIC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_scratch_addr[kMaxDevices];  // device address of g_static_scratch, per device

// Set-up, once per device, with that device current: the array's device
// address, and both instances of the box kernel loaded (module loading is
// lazy), so that later calls load nothing.
tsi_status scratch_address(int device, void **out) {
  if (device < 0 || device >= kMaxDevices) return TSI_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_addr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e == cudaSuccess && p) e = tsi::evalbox_preload();
    if (e != cudaSuccess || !p) {
      tsi_internal_set_error(cudaGetErrorString(e));
      cudaGetLastError();
      return TSI_ERR_CUDA;
    }
    g_scratch_addr[device] = p;
  }
  *out = g_scratch_addr[device];
  return TSI_OK;
}

}  // namespace

extern "C" TSI_API uint64_t tsi_static_scratch_bytes(void) { return TSI_STATIC_SCRATCH_BYTES; }

extern "C" TSI_API tsi_status tsi_tape_eval_boxes_static(const tsi_tape *tape, uint32_t n, const float *boxes_dev,
                                                          int32_t rounding_mode, int32_t reverse, float *out_dev,
                                                          void *cuda_stream) {
  TsiTapeView v;
  tsi_status st = tsi_internal_tape_view(tape, &v);
  if (st != TSI_OK) return st;
  if (n == 0) return TSI_OK;
  if (!boxes_dev || !out_dev) {
    tsi_internal_set_error("tsi_tape_eval_boxes_static: null device pointer");
    return TSI_ERR_INVALID_ARGUMENT;
  }
  const uint64_t regs_bytes = ((uint64_t)n * v.nregs * 8u + 255u) & ~255ull;
  const uint64_t log_bytes = (uint64_t)n * (v.len ? v.len : 1u) * 16u;
  if (regs_bytes + log_bytes > TSI_STATIC_SCRATCH_BYTES) {
    tsi_internal_set_error("tsi_tape_eval_boxes_static: n boxes x (registers + tape length) exceeds the "
                           "static scratch of TSI_STATIC_SCRATCH_BYTES; split the call");
    return TSI_ERR_BUFFER_TOO_SMALL;
  }
  // the tape's device is made current for the call; the caller's current
  // device is put back before returning
  int caller_dev = -1;
  if (cudaGetDevice(&caller_dev) != cudaSuccess) caller_dev = -1;
  if (cudaSetDevice(v.device) != cudaSuccess) {
    tsi_internal_set_error("cudaSetDevice failed");
    cudaGetLastError();
    return TSI_ERR_CUDA;
  }
  void *base = nullptr;
  st = scratch_address(v.device, &base);
  if (st == TSI_OK) {
    float2 *regs = (float2 *)base;
    float4 *log = (float4 *)((unsigned char *)base + regs_bytes);
    cudaStream_t s = cuda_stream ? (cudaStream_t)cuda_stream : v.stream;
    const cudaError_t e = tsi::launch_evalbox(rounding_mode == TSI_ROUND_DIRECTED, v.code, v.len, v.nregs, v.out_reg,
                                              n, boxes_dev, reverse, out_dev, regs, log, s);
    if (e != cudaSuccess) {
      tsi_internal_set_error(cudaGetErrorString(e));
      st = TSI_ERR_CUDA;
    }
  }
  if (caller_dev >= 0 && caller_dev != v.device) cudaSetDevice(caller_dev);
  return st;
}
