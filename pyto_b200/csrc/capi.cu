// Workspace sizing of the C ABI.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>

#include "krylov.cuh"

namespace pyto {
size_t pcg_workspace_bytes(const pyto_operator_t* op);
size_t dpcg_workspace_bytes(const pyto_operator_t* op, bool mixed);
int oc_grid_blocks();
int set_matvec_variant(int v);
int set_matvec32_variant(int v);
}  // namespace pyto

namespace pyto {
static std::atomic<long long> g_launches{0};
void count_launches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launch_count_now() { return g_launches.load(std::memory_order_relaxed); }
int g_use_graphs = 1;  // Krylov iteration chunks replayed as CUDA graphs

static thread_local char g_last_error[512] = "";
void record_error(cudaError_t e, const char* what, const char* file, int line) {
  const char* base = strrchr(file, '/');
  snprintf(g_last_error, sizeof(g_last_error), "%s:%d: %s -> %s (%s)", base ? base + 1 : file, line, what,
           cudaGetErrorName(e), cudaGetErrorString(e));
}
}  // namespace pyto

using namespace pyto;

extern "C" int pyto_tune(int kernel, int variant) {
  switch (kernel) {
    case PYTO_KERNEL_MATVEC: return set_matvec_variant(variant);
    case PYTO_KERNEL_MATVEC32: return set_matvec32_variant(variant);
    case PYTO_KERNEL_GRAPHS:
      if (variant < 0 || variant > 1) return PYTO_ERR_ARG;
      g_use_graphs = variant;
      return PYTO_OK;
    default: return PYTO_ERR_ARG;
  }
}

extern "C" const char* pyto_last_error(void) { return g_last_error; }

extern "C" long long pyto_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

extern "C" size_t pyto_workspace_bytes(const pyto_operator_t* op, int kind) {
  if (!op) return 0;
  switch (kind) {
    case PYTO_WS_REDUCE:
      return 1024 + 8 * 2 * reduce_slots(op);
    case PYTO_WS_PCG:
      return pcg_workspace_bytes(op);
    case PYTO_WS_DPCG:
      return dpcg_workspace_bytes(op, false);
    case PYTO_WS_DPCG_MIXED:
      return dpcg_workspace_bytes(op, true);
    case PYTO_WS_OC:
      return 1024 + 8 * 3 * (size_t)std::max(oc_grid_blocks(), 4 * kNumSMs);
    default:
      return 0;
  }
}
