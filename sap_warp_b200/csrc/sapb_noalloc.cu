// sapb_noalloc.cu -- the contact solve for callers that cannot allocate
// device memory.
//
// sapb_contact_solve needs a small device workspace (the persistent kernel's
// work counter) that the caller allocates.  Some callers cannot: a host that
// hands the solver only its own arrays and a stream (a plugin inside another
// runtime that owns every device allocation, or a foreign-language binding
// with no device allocator of its own) has no way to provide one.  This entry
// point uses a fixed array compiled into the library instead.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "sapb_internal.h"

namespace {

// Stated maximum: 4 KiB of scratch, held by every GPU that loads the library
// until the process exits.
constexpr size_t kNoAllocScratchBytes = 4096;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch_device_ptr[kMaxDevices] = {};
// Identity of the context each cached address belongs to: a device reset
// (cudaDeviceReset) ends that context, and the next call on the device then
// looks the address up again in the new one.
unsigned long long g_scratch_ctx_id[kMaxDevices] = {};

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Unique id of the calling thread's current context (0 if none or the
// driver cannot say), through the runtime's driver entry points: no link
// against the driver library.
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool looked_up = false;
  if (!looked_up) {
    looked_up = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
  }
  if (!get_current || !get_id) return 0;
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return 0;
  unsigned long long id = 0;
  if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

}  // namespace

extern "C" int32_t sapb_contact_solve_noalloc(const sapb_contact_problem* p, const sapb_solve_options* o,
                                              const sapb_solve_outputs* out, void* stream) {
  if (!p) {
    sapb::set_last_error("sapb_contact_solve_noalloc: null problem");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  const size_t need = sapb_contact_solve_workspace_size(p->num_envs, p->dof_per_env, p->max_contacts);
  if (need > kNoAllocScratchBytes) {
    sapb::set_last_error("sapb_contact_solve_noalloc: problem needs %zu bytes of scratch, above the %zu-byte maximum",
                         need, kNoAllocScratchBytes);
    return SAPB_ERR_WORKSPACE_TOO_SMALL;
  }
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) {
    sapb::set_last_error("sapb_contact_solve_noalloc: cudaGetDevice: %s", cudaGetErrorString(err));
    return SAPB_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    sapb::set_last_error("sapb_contact_solve_noalloc: device %d beyond the supported %d devices", dev, kMaxDevices);
    return SAPB_ERR_UNSUPPORTED;
  }
  void* scratch = nullptr;
  {
    // Set-up once per device, with that device current: the array's name is
    // a host-side stand-in, so its device address must come from the runtime.
    // The address is cached with the id of its context and looked up again
    // when the device's context has changed since (after a device reset).
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    const unsigned long long ctx = current_context_id();
    if (!g_scratch_device_ptr[dev] || ctx == 0 || ctx != g_scratch_ctx_id[dev]) {
      void* ptr = nullptr;
      err = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (err != cudaSuccess || ptr == nullptr) {
        sapb::set_last_error("sapb_contact_solve_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(err));
        return SAPB_ERR_CUDA;
      }
      g_scratch_device_ptr[dev] = ptr;
      g_scratch_ctx_id[dev] = current_context_id();  // the lookup made the context current if it was not
    }
    scratch = g_scratch_device_ptr[dev];
  }
  // The solve clears the work counter in the scratch (an async memset on
  // `stream`) before its launch.
  return sapb_contact_solve(p, o, out, scratch, kNoAllocScratchBytes, stream);
}
