// Fixed device scratch of imex_gmres_noalloc.
//
// imex_gmres stages host vectors in temporaries from cudaMallocAsync; callers that
// must not enter the device allocator during a solve (a host whose allocator owns
// the device's free memory, or a per-step path with a hard latency budget where an
// allocation may block on the pool) use imex_gmres_noalloc instead.  Its Krylov
// basis, AV ring, per-CTA partial sums, barrier state and staged host vectors all
// live in the one array below.  The array sits in its own translation unit, so its
// module (and the device memory it holds) is loaded only by callers of that entry
// point.  There is one array per device: calls that overlap on one device (two
// contexts, or two streams of one context) race on it.
#include <mutex>

#include "imex_internal.h"

namespace imex {
namespace {

static __device__ __align__(256) unsigned char g_solve_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

}  // namespace

// Device address of the scratch array on the context's device.  The context's device
// must be the current one (its memory and the kernel launch live there); a mismatch is
// refused with IMEX_ERR_INVALID rather than handing the solve another device's array.
// The first call on a device resolves the address with cudaGetSymbolAddress (with that
// device current) and later calls reuse it.  A cudaDeviceReset unloads the module and
// with it the array, and every context of that device dies with it; so imex_create
// drops the cached address of its device (forget_static_scratch), and the first call
// through a context created after a reset resolves the address again.  Without a
// reset the address resolved again is the same one.
imex_status static_scratch(imex_ctx* ctx, unsigned char** base) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_check(ctx, e, "cudaGetDevice");
  if (dev != ctx->device) {
    char msg[160];
    snprintf(msg, sizeof(msg),
             "imex_gmres_noalloc: device %d is current but the context lives on device %d; "
             "make the context's device current first",
             dev, ctx->device);
    return set_error(ctx, IMEX_ERR_INVALID, msg);
  }
  if (dev < 0 || dev >= kMaxDevices) return set_error(ctx, IMEX_ERR_UNSUPPORTED, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_solve_scratch);
    if (e != cudaSuccess) return cuda_check(ctx, e, "cudaGetSymbolAddress(static solve scratch)");
    g_scratch_ptr[dev] = static_cast<unsigned char*>(p);
  }
  *base = g_scratch_ptr[dev];
  return IMEX_OK;
}

void forget_static_scratch(int dev) {
  if (dev < 0 || dev >= kMaxDevices) return;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  g_scratch_ptr[dev] = nullptr;
}

}  // namespace imex
