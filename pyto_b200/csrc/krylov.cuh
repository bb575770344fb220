// Device-resident Krylov state and helpers shared by the Jacobi PCG and the
// deflated PCG drivers.
#pragma once
#include "matvec.cuh"

namespace pyto {

constexpr int kNodeBlocks = 16 * kNumSMs;  // grid of node-wise kernels (grid-stride; 3 partials each fit the
                                           // 4 * reduce_slots partial array)
constexpr int kNodeThreads = 256;
// grid of the deflated-PCG update1 (a streaming kernel): resident at once (4 CTAs of
// 256 threads per SM at <= 64 registers); threads loop over the data
constexpr int kUpdate1Blocks = 4 * kNumSMs;

struct KrylovState {
  double rz, rz0, pq, rr, bb, alpha, beta, rtol;
  double true_rr;
  double rscale2;  // squared scale of the recurrence vectors (residual r_true = sqrt(rscale2) r); 0 means 1
  double rscale2_prev;  // rscale2 before the last residual replacement
  int iters, done, breakdown, converged;
  int max_iters, stop_rule, pad0, pad1;
};

struct Prec {
  double ikd[3];  // 1 / Ke corner diagonal per component
};

inline Prec make_prec(const pyto_operator_t* op) {
  Prec p;
  for (int c = 0; c < 3; ++c) p.ikd[c] = 1.0 / op->kdiag[c];
  return p;
}

// Jacobi: z = r / diag; fixed DOFs -> 0; |diag| < 1e-12 -> 1 (src/linear_solvers.py:85)
__device__ __forceinline__ double jacobi_apply(double r, int fl, int c, double w, const Prec& pc) {
  if ((fl >> c) & 1) return 0.0;
  if ((fl >> (3 + c)) & 1) return r;
  return r * w * pc.ikd[c];
}

// stopping test after an update: rule 0 = scipy cg (||r|| < rtol ||b||, strict),
// rule 1 = PyTO DPCG (sqrt(r.z / r0.z0) <= rtol, src/deflation.py:567)
__device__ __forceinline__ bool krylov_converged(const KrylovState& S, double rr, double rz_new) {
  if (S.rscale2 > 0.0) rr *= S.rscale2;
  if (S.stop_rule == 0) return sqrt(rr) < S.rtol * sqrt(S.bb);
  return sqrt(rz_new / S.rz0) <= S.rtol;
}

// 12 consecutive values (the 3 DOFs of 4 nodes) with 16-byte accesses; the
// address must be 16-byte aligned (node quads of 16-byte aligned vectors).
__device__ __forceinline__ void ld12(const float* p, float (&v)[12]) {
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float4 t = __ldg(reinterpret_cast<const float4*>(p) + k);
    v[4 * k] = t.x;
    v[4 * k + 1] = t.y;
    v[4 * k + 2] = t.z;
    v[4 * k + 3] = t.w;
  }
}
__device__ __forceinline__ void ld12(const double* p, double (&v)[12]) {
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const double2 t = __ldg(reinterpret_cast<const double2*>(p) + k);
    v[2 * k] = t.x;
    v[2 * k + 1] = t.y;
  }
}
__device__ __forceinline__ void st12(float* p, const float (&v)[12]) {
#pragma unroll
  for (int k = 0; k < 3; ++k)
    reinterpret_cast<float4*>(p)[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
}
__device__ __forceinline__ void st12(double* p, const double (&v)[12]) {
#pragma unroll
  for (int k = 0; k < 6; ++k) reinterpret_cast<double2*>(p)[k] = make_double2(v[2 * k], v[2 * k + 1]);
}
// One 16-byte chunk (4 floats or 2 doubles) of vector v at chunk index k
template <typename T>
struct Chunk;
template <>
struct Chunk<float> {
  static constexpr int N = 4;
  __device__ __forceinline__ static void ld(const float* p, long long k, float (&v)[4]) {
    const float4 t = __ldg(reinterpret_cast<const float4*>(p) + k);
    v[0] = t.x;
    v[1] = t.y;
    v[2] = t.z;
    v[3] = t.w;
  }
  __device__ __forceinline__ static void st(float* p, long long k, const float (&v)[4]) {
    reinterpret_cast<float4*>(p)[k] = make_float4(v[0], v[1], v[2], v[3]);
  }
};
template <>
struct Chunk<double> {
  static constexpr int N = 2;
  __device__ __forceinline__ static void ld(const double* p, long long k, double (&v)[2]) {
    const double2 t = __ldg(reinterpret_cast<const double2*>(p) + k);
    v[0] = t.x;
    v[1] = t.y;
  }
  __device__ __forceinline__ static void st(double* p, long long k, const double (&v)[2]) {
    reinterpret_cast<double2*>(p)[k] = make_double2(v[0], v[1]);
  }
};

// Jacobi weights and flags of the 4 nodes of quad t (w, fl: 16- and 4-byte aligned bases)
__device__ __forceinline__ void ld_quad_node(const double* w, const uint8_t* fl, long long t, double (&wn)[4],
                                             unsigned& f4) {
  const double2 a = __ldg(reinterpret_cast<const double2*>(w + 4 * t));
  const double2 b = __ldg(reinterpret_cast<const double2*>(w + 4 * t) + 1);
  wn[0] = a.x;
  wn[1] = a.y;
  wn[2] = b.x;
  wn[3] = b.y;
  f4 = __ldg(reinterpret_cast<const unsigned*>(fl + 4 * t));
}

// stop (optional): the solver's done flag; the launch does nothing once it is set
// (the operator launch of an iteration past convergence)
int launch_matvec64(const pyto_operator_t* op, const double* s, const uint8_t* mask, const double* u, double* y,
                    int mode, double* part, unsigned* counter, double* dot, cudaStream_t st,
                    const int* stop = nullptr);
long long matvec_blocks(const pyto_operator_t* op);
size_t reduce_slots(const pyto_operator_t* op);

}  // namespace pyto
