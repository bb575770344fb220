// K(s) u with the fused dot product, for callers that cannot allocate device
// memory.
//
// Some callers of this library run where cudaMalloc is not available to them:
// code that executes inside a host framework which owns every device
// allocation (plugins handed pre-sized buffers), or real-time loops where
// allocating is forbidden after start-up.  pyto_matvec needs a caller-provided
// workspace for the cross-block partial sums of the dot product; this variant
// keeps that scratch in a fixed array compiled into the library instead.
//
// The scratch is a file-scope __device__ array: every GPU that loads this
// library holds it (kNoAllocSlots doubles + a counter, ~64 KB) until the
// process exits.  Its host-side name is only a stand-in for the device
// symbol, so its device address is looked up with cudaGetSymbolAddress, once
// per device, the first time the entry point runs with that device current;
// that first call should therefore come before any stream capture.  The cached
// address is not refreshed: a cudaDeviceReset (or a reset of the primary
// context) can move the array, so after one this entry point must not be
// called again in the same process.  All calls
// share the one array: the completion counter is cleared at every call, and
// two calls whose kernels overlap on the GPU (different streams, or different
// host threads) race on it, so callers must order them.
#include <mutex>

#include "krylov.cuh"

namespace pyto {

constexpr int kNoAllocSlots = 8192;  // max CTAs of the matvec launch this variant accepts
constexpr int kNoAllocMaxDevices = 64;

// [0, 256): completion counter of the cross-block reduction (bytes);
// [256, 256 + 8*kNoAllocSlots): per-CTA partial sums
static __device__ __align__(256) unsigned char g_noalloc_scratch[256 + 8 * kNoAllocSlots];

static void* g_scratch_addr[kNoAllocMaxDevices];
static std::mutex g_scratch_mu;

static int scratch_address(void** out) {
  int dev = 0;
  PYTO_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return PYTO_ERR_TOO_LARGE;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    PYTO_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return PYTO_OK;
}

}  // namespace pyto

using namespace pyto;

extern "C" int pyto_matvec_dot_noalloc(const pyto_operator_t* op, const double* s, const uint8_t* mask,
                                       const double* u, double* y, int mode, double* dot, void* stream) {
  if (!op || !s || !u || !y || !dot || u == y) return PYTO_ERR_ARG;
  if (matvec_blocks(op) > kNoAllocSlots) return PYTO_ERR_TOO_LARGE;
  void* base = nullptr;
  int rc = scratch_address(&base);
  if (rc) return rc;
  unsigned* counter = reinterpret_cast<unsigned*>(base);
  double* part = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(base) + 256);
  cudaStream_t st = (cudaStream_t)stream;
  PYTO_CUDA(cudaMemsetAsync(counter, 0, 256, st));
  return launch_matvec64(op, s, mask, u, y, mode, part, counter, dot, st);
}
