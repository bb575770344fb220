// Shared device/host helpers of libpyto_b200 (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/pyto_b200.h"

namespace pyto {
// records the failing CUDA call of this thread (read by pyto_last_error)
void record_error(cudaError_t e, const char* what, const char* file, int line);
}  // namespace pyto

#define PYTO_CUDA(call)                                                 \
  do {                                                                  \
    cudaError_t _e = (call);                                            \
    if (_e != cudaSuccess) {                                            \
      ::pyto::record_error(_e, #call, __FILE__, __LINE__);              \
      return PYTO_ERR_CUDA;                                             \
    }                                                                   \
  } while (0)

#define PYTO_LAUNCH_CHECK() PYTO_CUDA(cudaGetLastError())

namespace pyto {
// process-wide count of kernel launches issued by the library (reported by
// pyto_launch_count; used to state how many of the library's kernels ran)
void count_launches(long long n);
}  // namespace pyto
#define PYTO_COUNT(n) ::pyto::count_launches(n)

namespace pyto {
// Function attributes (the dynamic shared-memory opt-in) belong to a device: a call
// site sets them once per device it launches on.  needed() is true until done() was
// called while that device was current.
struct PerDevice {
  unsigned long long mask = 0;  // devices 0..63
  static unsigned long long bit() {
    int d = 0;
    cudaGetDevice(&d);
    return 1ull << (d & 63);
  }
  bool needed() const { return (__atomic_load_n(&mask, __ATOMIC_ACQUIRE) & bit()) == 0; }
  void done() { __atomic_fetch_or(&mask, bit(), __ATOMIC_RELEASE); }
};

constexpr int kNumSMs = 148;        // B200
constexpr int kReduceBlocks = 1184; // max partial slots of a node-wise reduction (8 per SM)

// Grid geometry passed by value to kernels.
struct GridDims {
  int nx, ny, nz;  // elements
  int sx, sy, sz;  // nodes = elements + 1
  long long nnodes, nelem;
};

inline GridDims make_dims(const pyto_operator_t* op) {
  GridDims g;
  g.nx = op->nelx; g.ny = op->nely; g.nz = op->nelz;
  g.sx = g.nx + 1; g.sy = g.ny + 1; g.sz = g.nz + 1;
  g.nnodes = (long long)g.sx * g.sy * g.sz;
  g.nelem = (long long)g.nx * g.ny * g.nz;
  return g;
}

// Element operator in the Hadamard corner basis, passed as a kernel argument
// (lands in the constant bank: uniform, broadcast reads).
struct KHat {
  double b[8][9];   // class q block, row-major 3x3
  double kd[3];     // corner diagonal per component
};

inline KHat make_khat(const pyto_operator_t* op) {
  KHat k;
  for (int q = 0; q < 8; ++q)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) k.b[q][3 * i + j] = op->khat[q][i][j];
  for (int c = 0; c < 3; ++c) k.kd[c] = op->kdiag[c];
  return k;
}

// ---- deterministic block reductions ------------------------------------
// Sum over a block in a fixed order: warp shuffle tree, then warp 0 over the
// per-warp partials.  Result valid in thread 0.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* smem /*>= NT/32*/) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) smem[wid] = v;
  __syncthreads();
  double r = 0.0;
  if (wid == 0) {
    r = (lane < NT / 32) ? smem[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
  }
  __syncthreads();
  return r;
}

template <int NT>
__device__ __forceinline__ double block_max(double v, double* smem) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) smem[wid] = v;
  __syncthreads();
  double r = -1.0e308;
  if (wid == 0) {
    r = (lane < NT / 32) ? smem[lane] : -1.0e308;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_down_sync(0xffffffffu, r, o));
  }
  __syncthreads();
  return r;
}

// Sum of `n` partials in a fixed order by one warp; every lane gets the same
// bitwise result (xor butterfly), so all blocks that call it agree.
__device__ __forceinline__ double warp_sum_partials(const double* p, int n) {
  const int lane = threadIdx.x & 31;
  double v = 0.0;
  for (int i = lane; i < n; i += 32) v += __ldcg(p + i);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Cross-block reduction: every block deposits its value(s) (thread 0 holds
// them), the last block to arrive sums all partials and calls `fin(totals)` in
// its thread 0.  The last block sums with all its threads (thread t takes
// partials t, t+blockDim, ... in order; warps combine by xor butterfly; warp
// sums are added in warp order), so the result is deterministic: the order
// does not depend on scheduling.  The counter is reset by the last block, so it
// can be reused by the next launch on the same stream.
template <int K, typename Fin>
__device__ __forceinline__ void grid_reduce(const double (&v)[K], double* part /*[K][nblocks]*/,
                                            unsigned* counter, int nblocks, Fin fin) {
  __shared__ bool s_last;
  __shared__ double s_w[K][32];
  const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) part[(size_t)k * nblocks + bid] = v[k];
    __threadfence();
    const unsigned t = atomicAdd(counter, 1u);
    s_last = (t == (unsigned)nblocks - 1u);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double acc[K];
#pragma unroll
  for (int k = 0; k < K; ++k) acc[k] = 0.0;
  for (int i = threadIdx.x; i < nblocks; i += blockDim.x) {
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] += __ldcg(part + (size_t)k * nblocks + i);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
    if (lane == 0) s_w[k][wid] = acc[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      tot[k] = 0.0;
      for (int w = 0; w < nw; ++w) tot[k] += s_w[k][w];
    }
    fin(tot);
    *counter = 0u;
    __threadfence();
  }
}

// Cross-block step of a fused dot product whose block sum bsum is valid in thread 0.
// With a counter: grid_reduce, the last block writes the total to *dot_out.  Without
// one (deferred): every block leaves its sum for the kernel that consumes the dot
// product (deferred_sum), part[1 + b] for block b and part[0] = the number of blocks:
// no fence, atomic or last-block pass at the end of the producing kernel.
__device__ __forceinline__ void dot_finish(double bsum, double* part, unsigned* counter, double* dot_out) {
  const int nb = (int)(gridDim.x * gridDim.y * gridDim.z);
  if (counter) {
    const double v[1] = {bsum};
    grid_reduce<1>(v, part, counter, nb, [&](const double* t) { *dot_out = t[0]; });
  } else if (threadIdx.x == 0) {
    const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    part[1 + bid] = bsum;
    if (bid == 0) part[0] = (double)nb;
  }
}

// Total of the block sums left by dot_finish without a counter, in block order (thread
// t adds blocks t, t + NT, ...; then block_sum): the same bits in every thread of every
// CTA that calls it.  sred: >= NT/32 + 1 doubles.
template <int NT>
__device__ __forceinline__ double deferred_sum(const double* part, double* sred) {
  const int n = (int)part[0];
  double a = 0.0;
  for (int i = threadIdx.x; i < n; i += NT) a += part[1 + i];
  const double t = block_sum<NT>(a, sred);
  if (threadIdx.x == 0) sred[NT / 32] = t;
  __syncthreads();
  const double r = sred[NT / 32];
  __syncthreads();
  return r;
}

// Workspace carving helper (256-byte aligned sub-buffers).
struct Carver {
  char* base;
  size_t off, cap;
  template <typename T>
  T* take(size_t count) {
    off = (off + 255) & ~(size_t)255;
    T* p = (T*)(base ? base + off : nullptr);
    off += count * sizeof(T);
    return p;
  }
  bool ok() const { return base != nullptr && off <= cap; }
};

// Two FP32 lanes in one 64-bit register pair for the packed FP32x2 arithmetic of
// sm_100 (__fadd2_rn / __fmul2_rn / __ffma2_rn): two independent elements go through
// the same arithmetic in one instruction stream.  Each lane rounds exactly as the
// scalar operation.  In a namespace of its own so that fma() on floats keeps
// resolving to the global one (this fma is found by argument-dependent lookup).
namespace packed {
struct f32x2 {
  float2 v;
  f32x2() = default;
  __host__ __device__ constexpr explicit f32x2(float a) : v{a, a} {}
  __host__ __device__ constexpr f32x2(float a, float b) : v{a, b} {}
  __host__ __device__ constexpr explicit f32x2(float2 w) : v(w) {}
};
__device__ __forceinline__ f32x2 operator+(f32x2 a, f32x2 b) { return f32x2(__fadd2_rn(a.v, b.v)); }
__device__ __forceinline__ f32x2 operator-(f32x2 a) { return f32x2(-a.v.x, -a.v.y); }
__device__ __forceinline__ f32x2 operator-(f32x2 a, f32x2 b) {
  // one packed subtraction (sub.rn.f32x2), each lane rounded as the scalar a - b
  f32x2 r;
  asm("{\n\t.reg .b64 pa, pb, pd;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
      "sub.rn.f32x2 pd, pa, pb;\n\tmov.b64 {%0, %1}, pd;\n\t}"
      : "=f"(r.v.x), "=f"(r.v.y)
      : "f"(a.v.x), "f"(a.v.y), "f"(b.v.x), "f"(b.v.y));
  return r;
}
__device__ __forceinline__ f32x2 operator*(f32x2 a, f32x2 b) { return f32x2(__fmul2_rn(a.v, b.v)); }
__device__ __forceinline__ f32x2 fma(f32x2 a, f32x2 b, f32x2 c) { return f32x2(__ffma2_rn(a.v, b.v, c.v)); }
__device__ __forceinline__ f32x2& operator+=(f32x2& a, f32x2 b) { return a = a + b; }
__device__ __forceinline__ f32x2& operator-=(f32x2& a, f32x2 b) { return a = a - b; }
}  // namespace packed

}  // namespace pyto
