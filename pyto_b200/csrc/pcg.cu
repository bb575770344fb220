// Jacobi-preconditioned CG on the reduced system K_ff u_f = b_f
// (src/linear_solvers.py:164-168, scipy cg semantics: stop when
// ||r||_2 < rtol ||b||_2 checked once per iteration, iteration = one matvec).
//
// One iteration = 3 kernels, all scalars stay on the device:
//   1. q = K p                    (fused: p.q, last block -> state.pq)
//   2. x += a p, r -= a q         (fused: r.r and r.M^-1 r; last block tests
//                                  convergence and forms beta)
//   3. p = M^-1 r + beta p
// The host polls the state every cfg->check_every iterations.
#include <algorithm>

#include "krylov.cuh"

namespace pyto {

__global__ void k_state_init(KrylovState* S, double rtol, int max_iters, int stop_rule) {
  KrylovState z{};
  z.rtol = rtol;
  z.max_iters = max_iters;
  z.stop_rule = stop_rule;
  *S = z;
}

// r = b - t (t = K x0 or nothing), masked; p = z = M^-1 r; x = 0 when no x0.
__global__ void __launch_bounds__(kNodeThreads) k_pcg_init(GridDims g, Prec pc, const double* __restrict__ b,
                                                           const double* __restrict__ t, const double* __restrict__ w,
                                                           const uint8_t* __restrict__ fl, double* __restrict__ x,
                                                           double* __restrict__ r, double* __restrict__ p,
                                                           KrylovState* S, double* part, unsigned* counter) {
  __shared__ double sred[kNodeThreads / 32];
  double rz = 0.0, rr = 0.0, bb = 0.0;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < g.nnodes;
       n += (long long)gridDim.x * blockDim.x) {
    const int f = fl[n];
    const double wn = w[n];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const long long i = 3 * n + c;
      const bool fixed = (f >> c) & 1;
      const double bi = fixed ? 0.0 : b[i];
      const double ri = fixed ? 0.0 : bi - (t ? t[i] : 0.0);
      const double zi = jacobi_apply(ri, f, c, wn, pc);
      r[i] = ri;
      p[i] = zi;
      if (!t) x[i] = 0.0;
      rz = fma(ri, zi, rz);
      rr = fma(ri, ri, rr);
      bb = fma(bi, bi, bb);
    }
  }
  double v[3];
  v[0] = block_sum<kNodeThreads>(rz, sred);
  v[1] = block_sum<kNodeThreads>(rr, sred);
  v[2] = block_sum<kNodeThreads>(bb, sred);
  grid_reduce<3>(v, part, counter, gridDim.x, [&](const double* tot) {
    S->rz = tot[0];
    S->rz0 = tot[0];
    S->rr = tot[1];
    S->bb = tot[2];
    if (tot[2] == 0.0 || (S->stop_rule == 0 && sqrt(tot[1]) < S->rtol * sqrt(tot[2]))) {
      S->done = 1;
      S->converged = 1;
    }
  });
}

__global__ void __launch_bounds__(kNodeThreads) k_pcg_update1(GridDims g, Prec pc, const double* __restrict__ w,
                                                              const uint8_t* __restrict__ fl, double* __restrict__ x,
                                                              double* __restrict__ r, const double* __restrict__ p,
                                                              const double* __restrict__ q, KrylovState* S,
                                                              double* part, unsigned* counter) {
  __shared__ double sred[kNodeThreads / 32];
  if (S->done) return;
  const double pq = S->pq, rz = S->rz;
  const double alpha = rz / pq;
  if (!(pq > 0.0) || !isfinite(alpha)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      S->breakdown = 1;
      S->done = 1;
    }
    return;
  }
  double rr = 0.0, rzn = 0.0;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < g.nnodes;
       n += (long long)gridDim.x * blockDim.x) {
    const int f = fl[n];
    const double wn = w[n];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const long long i = 3 * n + c;
      x[i] = fma(alpha, p[i], x[i]);
      const double ri = fma(-alpha, q[i], r[i]);
      r[i] = ri;
      const double zi = jacobi_apply(ri, f, c, wn, pc);
      rr = fma(ri, ri, rr);
      rzn = fma(ri, zi, rzn);
    }
  }
  double v[2];
  v[0] = block_sum<kNodeThreads>(rr, sred);
  v[1] = block_sum<kNodeThreads>(rzn, sred);
  grid_reduce<2>(v, part, counter, gridDim.x, [&](const double* tot) {
    S->alpha = alpha;
    S->iters += 1;
    S->rr = tot[0];
    const double rz_new = tot[1];
    if (!isfinite(tot[0]) || !isfinite(rz_new)) {
      S->breakdown = 1;
      S->done = 1;
    } else if (krylov_converged(*S, tot[0], rz_new)) {
      S->converged = 1;
      S->done = 1;
    } else if (S->iters >= S->max_iters) {
      S->done = 1;
    }
    S->beta = rz_new / S->rz;
    S->rz = rz_new;
  });
}

__global__ void __launch_bounds__(kNodeThreads) k_pcg_update2(GridDims g, Prec pc, const double* __restrict__ w,
                                                              const uint8_t* __restrict__ fl,
                                                              const double* __restrict__ r, double* __restrict__ p,
                                                              const KrylovState* S) {
  if (S->done) return;
  const double beta = S->beta;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < g.nnodes;
       n += (long long)gridDim.x * blockDim.x) {
    const int f = fl[n];
    const double wn = w[n];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const long long i = 3 * n + c;
      p[i] = fma(beta, p[i], jacobi_apply(r[i], f, c, wn, pc));
    }
  }
}

// ||b_f - t_f||^2 -> S->true_rr (t = K u, masked)
__global__ void __launch_bounds__(kNodeThreads) k_true_residual(GridDims g, const double* __restrict__ b,
                                                                const double* __restrict__ t,
                                                                const uint8_t* __restrict__ fl, KrylovState* S,
                                                                double* part, unsigned* counter) {
  __shared__ double sred[kNodeThreads / 32];
  double rr = 0.0, bb = 0.0;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < g.nnodes;
       n += (long long)gridDim.x * blockDim.x) {
    const int f = fl[n];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if ((f >> c) & 1) continue;
      const double bi = b[3 * n + c];
      const double d = bi - t[3 * n + c];
      rr = fma(d, d, rr);
      bb = fma(bi, bi, bb);
    }
  }
  double v[2] = {block_sum<kNodeThreads>(rr, sred), block_sum<kNodeThreads>(bb, sred)};
  grid_reduce<2>(v, part, counter, gridDim.x, [&](const double* tot) {
    S->true_rr = tot[0];
    S->bb = tot[1];
  });
}

struct PcgWs {
  KrylovState* S;
  unsigned* counter;
  double* part;
  double *r, *p, *q, *w;
  uint8_t* fl;
};

size_t reduce_slots(const pyto_operator_t* op) {
  return (size_t)std::max<long long>(matvec_blocks(op), 2 * kReduceBlocks);
}

static PcgWs carve_pcg(const pyto_operator_t* op, void* ws, size_t bytes, size_t* need) {
  const GridDims g = make_dims(op);
  Carver cv{(char*)ws, 0, bytes};
  PcgWs W;
  W.S = cv.take<KrylovState>(1);
  W.counter = cv.take<unsigned>(64);
  W.part = cv.take<double>(4 * reduce_slots(op));
  W.r = cv.take<double>(3 * g.nnodes);
  W.p = cv.take<double>(3 * g.nnodes);
  W.q = cv.take<double>(3 * g.nnodes);
  W.w = cv.take<double>(g.nnodes);
  W.fl = cv.take<uint8_t>(g.nnodes);
  *need = cv.off + 256;
  return W;
}

size_t pcg_workspace_bytes(const pyto_operator_t* op) {
  size_t need = 0;
  carve_pcg(op, nullptr, 0, &need);
  return need;
}

}  // namespace pyto

using namespace pyto;

extern "C" int pyto_pcg_solve(const pyto_operator_t* op, const double* s, const uint8_t* mask, const double* b,
                              double* u, const pyto_solve_cfg_t* cfg, pyto_solve_status_t* status, void* ws,
                              size_t ws_bytes, void* stream) {
  if (!op || !s || !b || !u || !cfg || !status) return PYTO_ERR_ARG;
  if (!(cfg->rtol >= 0.0) || cfg->max_iters < 0 || cfg->stop_rule < 0 || cfg->stop_rule > 1) return PYTO_ERR_ARG;
  size_t need = 0;
  PcgWs W = carve_pcg(op, ws, ws_bytes, &need);
  if (!ws || ws_bytes < need) return PYTO_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  const GridDims g = make_dims(op);
  const Prec pc = make_prec(op);
  PYTO_CUDA(cudaMemsetAsync(W.counter, 0, 64 * sizeof(unsigned), st));
  k_state_init<<<1, 1, 0, st>>>(W.S, cfg->rtol, cfg->max_iters, cfg->stop_rule);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  int rc = pyto_jacobi(op, s, mask, W.w, W.fl, nullptr, stream);
  if (rc) return rc;
  const int mm = PYTO_MASK_IN | PYTO_MASK_OUT;
  if (cfg->x0_given) {
    rc = launch_matvec64(op, s, mask, u, W.q, mm, nullptr, nullptr, nullptr, st);
    if (rc) return rc;
  }
  k_pcg_init<<<kNodeBlocks, kNodeThreads, 0, st>>>(g, pc, b, cfg->x0_given ? W.q : nullptr, W.w, W.fl, u, W.r, W.p,
                                                   W.S, W.part, W.counter);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  const int every = std::max(1, cfg->check_every);
  KrylovState hs{};
  PYTO_CUDA(cudaMemcpyAsync(&hs, W.S, sizeof(hs), cudaMemcpyDeviceToHost, st));
  PYTO_CUDA(cudaStreamSynchronize(st));
  while (!hs.done && hs.iters < cfg->max_iters) {
    for (int k = 0; k < every; ++k) {
      // p is zero on fixed DOFs (p = M^-1 r + beta p, M^-1 masked): no input mask needed
      rc = launch_matvec64(op, s, mask, W.p, W.q, PYTO_MASK_OUT, W.part, W.counter, &W.S->pq, st, &W.S->done);
      if (rc) return rc;
      k_pcg_update1<<<kNodeBlocks, kNodeThreads, 0, st>>>(g, pc, W.w, W.fl, u, W.r, W.p, W.q, W.S, W.part,
                                                          W.counter);
      PYTO_COUNT(1);
      k_pcg_update2<<<kNodeBlocks, kNodeThreads, 0, st>>>(g, pc, W.w, W.fl, W.r, W.p, W.S);
      PYTO_COUNT(1);
    }
    PYTO_LAUNCH_CHECK();
    PYTO_CUDA(cudaMemcpyAsync(&hs, W.S, sizeof(hs), cudaMemcpyDeviceToHost, st));
    PYTO_CUDA(cudaStreamSynchronize(st));
  }
  // true residual in FP64
  const KrylovState before = hs;
  rc = launch_matvec64(op, s, mask, u, W.q, mm, nullptr, nullptr, nullptr, st);
  if (rc) return rc;
  k_true_residual<<<kNodeBlocks, kNodeThreads, 0, st>>>(g, b, W.q, W.fl, W.S, W.part, W.counter);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  PYTO_CUDA(cudaMemcpyAsync(&hs, W.S, sizeof(hs), cudaMemcpyDeviceToHost, st));
  PYTO_CUDA(cudaStreamSynchronize(st));
  status->converged = hs.converged;
  status->iters = hs.iters;
  status->breakdown = hs.breakdown;
  status->rel_res = hs.stop_rule == 0 ? (before.bb > 0 ? sqrt(before.rr / before.bb) : 0.0)
                                      : (before.rz0 > 0 ? sqrt(before.rz / before.rz0) : 0.0);
  status->true_rel_res = hs.bb > 0 ? sqrt(hs.true_rr / hs.bb) : 0.0;
  if (hs.breakdown) return PYTO_ERR_BREAKDOWN;
  return hs.converged ? PYTO_OK : PYTO_NOT_CONVERGED;
}
