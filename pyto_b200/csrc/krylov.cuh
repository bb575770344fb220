// Device-resident Krylov state and helpers shared by the Jacobi PCG and the
// deflated PCG drivers.
#pragma once
#include "matvec.cuh"

namespace pyto {

constexpr int kNodeBlocks = 4 * kNumSMs;  // grid of node-wise kernels (grid-stride)
constexpr int kNodeThreads = 256;

struct KrylovState {
  double rz, rz0, pq, rr, bb, alpha, beta, rtol;
  double true_rr;
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
  if (S.stop_rule == 0) return sqrt(rr) < S.rtol * sqrt(S.bb);
  return sqrt(rz_new / S.rz0) <= S.rtol;
}

int launch_matvec64(const pyto_operator_t* op, const double* s, const uint8_t* mask, const double* u, double* y,
                    int mode, double* part, unsigned* counter, double* dot, cudaStream_t st);
long long matvec_blocks(const pyto_operator_t* op);
size_t reduce_slots(const pyto_operator_t* op);

}  // namespace pyto
