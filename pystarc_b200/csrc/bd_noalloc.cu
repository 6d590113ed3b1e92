// bd_sim_run_noalloc: the stepper for callers that cannot allocate device memory.
//
// Some host applications cannot call cudaMalloc when they want to run trajectories:
// an application whose own allocator has already reserved the GPU's memory (a
// framework's caching pool), or a process under a device-memory quota.  For them this
// entry point runs a whole batch of trajectories without allocating: the live-slot
// pool (two slot buffers), the live counts and the counters live in the file-scope
// device array below, and the per-trajectory outputs and final counters go to arrays
// the caller owns.  The call copies a few words between host and device and waits on
// its stream, so it returns only when the batch is done.
//
// The array is a fixed 9.2 MB (room for BD_NOALLOC_MAX_SLOTS = 65536 live slots);
// every GPU that loads the library keeps it until the process exits.  All calls
// share it and it keeps the last call's contents, so each call clears the counters
// it uses; two calls whose work overlaps on the GPU race on it.
#include <cstddef>
#include <cstdint>
#include <mutex>

#include <cuda_runtime.h>

#include "bd_device.cuh"
#include "pystarc_b200.h"

namespace {

constexpr int kMaxSlots = BD_NOALLOC_MAX_SLOTS;
// two slot buffers of 70 B per slot (each array rounded up to 256 B), two live
// counts and the counters, with slack for the per-array alignment
constexpr size_t kScratchBytes = 2 * (size_t)kMaxSlots * 70 + 64 * 1024;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_addr[kMaxDevices] = {};

}  // namespace

int bd_internal_device(const BdHandle* h);
int bd_internal_fail(BdHandle* h, int code, const char* msg);
int bd_internal_run_noalloc(BdHandle* h, const BdSimParams* p, unsigned char* scratch, size_t scratch_bytes,
                            int max_slots, int8_t* out_status, int32_t* out_steps, int32_t* out_returns,
                            uint64_t* counters, int K, int max_launches, cudaStream_t s);

extern "C" int bd_sim_run_noalloc(BdHandle* h, const BdSimParams* p, int8_t* out_status, int32_t* out_steps,
                                  int32_t* out_returns, uint64_t* counters, int steps_per_launch, int max_launches,
                                  void* stream) {
  if (!h) return BD_ERR_ARG;
  const int dev = bd_internal_device(h);
  if (dev < 0 || dev >= kMaxDevices) return bd_internal_fail(h, BD_ERR_ARG, "device index out of range");
  unsigned char* ptr = nullptr;
  {
    // In host code g_scratch is only a host-side stand-in for the array; its
    // device address comes from cudaGetSymbolAddress, taken once per device
    // with that device current (this is the first call's set-up).
    std::lock_guard<std::mutex> lock(g_mu);
    ptr = g_addr[dev];
    if (!ptr) {
      if (cudaSetDevice(dev) != cudaSuccess) return bd_internal_fail(h, BD_ERR_CUDA, "cudaSetDevice failed");
      const cudaError_t e = cudaGetSymbolAddress((void**)&ptr, g_scratch);
      if (e != cudaSuccess || !ptr)
        return bd_internal_fail(h, BD_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed");
      g_addr[dev] = ptr;
    }
  }
  return bd_internal_run_noalloc(h, p, ptr, kScratchBytes, kMaxSlots, out_status, out_steps, out_returns, counters,
                                 steps_per_launch, max_launches, (cudaStream_t)stream);
}
