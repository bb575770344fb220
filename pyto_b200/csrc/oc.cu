// Optimality-criteria update with bisection on the volume multiplier
// (src/topopt_ocm.py:244-283).
//
// The whole bisection runs in one cooperative kernel: every bisection step
// evaluates sum(x_new(lmid)) over the design (the design vector stays in L2),
// blocks deposit partials, a grid barrier, then every block sums the partials
// in the same fixed order and takes the same l1/l2 decision, so the lmid
// sequence is the reference's sequence.  Partials are double-buffered by step
// parity so a fast block never overwrites values a slow block still reads.
// The loop ends after a bounded number of halvings (the interval test of the
// reference needs about 70), so the kernel always terminates.
#include <cooperative_groups.h>

#include <algorithm>

#include "common.cuh"

namespace cg = cooperative_groups;

namespace pyto {

constexpr int kOcThreads = 256;
constexpr int kOcMaxSteps = 200;

__device__ __forceinline__ double oc_xnew(double x, double dc, double dv_l, double move, double xmin, double xmax) {
  double D = -dc / dv_l;
  D = fmin(fmax(D, 0.1), 10.0);
  return fmax(xmin, fmax(x - move, fmin(xmax, fmin(x + move, x * sqrt(D)))));
}

__global__ void __launch_bounds__(kOcThreads) k_oc_update(long long n, double* __restrict__ x,
                                                          const double* __restrict__ dc,
                                                          const uint8_t* __restrict__ active, long long n_act,
                                                          double volfrac, double move, double xmin, double xmax,
                                                          double* part, double* change_out) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double sred[kOcThreads / 32];
  __shared__ double s_tot;
  const double dv = 1.0 / volfrac / (double)n_act;  // compute_volume_constraint_and_gradient
  const int nb = gridDim.x;
  double l1 = 0.0, l2 = 1e12, lmid = 0.5 * (l2 + l1);
  int step = 0;
  while ((l2 - l1) / ((l1 + l2) / 2 + 1e-10) > 1e-7 && step < kOcMaxSteps) {
    lmid = 0.5 * (l2 + l1);
    const double dvl = dv * lmid;
    double acc = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
      if (!active || active[i]) acc += oc_xnew(x[i], dc[i], dvl, move, xmin, xmax);
    const double b = block_sum<kOcThreads>(acc, sred);
    double* pp = part + (size_t)(step & 1) * nb;
    if (threadIdx.x == 0) pp[blockIdx.x] = b;
    grid.sync();
    if (threadIdx.x < 32) {
      const double t = warp_sum_partials(pp, nb);
      if (threadIdx.x == 0) s_tot = t;
    }
    __syncthreads();
    const double vol = (s_tot / (double)n_act) / volfrac - 1.0;
    if (vol > 0) l1 = lmid;
    else l2 = lmid;
    ++step;
  }
  // x = xnew(lmid of the last step); change = max |x_new - x_old|
  const double dvl = dv * lmid;
  double ch = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    if (active && !active[i]) continue;
    const double xo = x[i];
    const double xn = oc_xnew(xo, dc[i], dvl, move, xmin, xmax);
    ch = fmax(ch, fabs(xn - xo));
    x[i] = xn;
  }
  const double bm = block_max<kOcThreads>(ch, sred);
  double* pp = part + (size_t)2 * nb;
  if (threadIdx.x == 0) pp[blockIdx.x] = bm;
  grid.sync();
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double m = 0.0;
    for (int i = 0; i < nb; ++i) m = fmax(m, __ldcg(pp + i));
    *change_out = m;
  }
}

int oc_grid_blocks() {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_oc_update, kOcThreads, 0) != cudaSuccess) return 0;
  int dev = 0, sms = kNumSMs;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  return std::max(1, std::min(per_sm, 2)) * sms;
}

}  // namespace pyto

using namespace pyto;

extern "C" int pyto_oc_update(const pyto_operator_t* op, double* x, const double* dc, const uint8_t* active,
                              long long n_active, double volfrac, double move, double xmin, double xmax,
                              double* change_out, void* ws, size_t ws_bytes, void* stream) {
  if (!op || !x || !dc || !change_out || !(volfrac > 0)) return PYTO_ERR_ARG;
  const GridDims g = make_dims(op);
  long long n = g.nelem;
  long long n_act = active ? n_active : n;
  if (n_act <= 0) return PYTO_ERR_ARG;
  int nb = oc_grid_blocks();
  if (nb <= 0) return PYTO_ERR_CUDA;
  nb = (int)std::min<long long>(nb, (n + kOcThreads - 1) / kOcThreads);
  Carver cv{(char*)ws, 0, ws_bytes};
  double* part = cv.take<double>(3 * (size_t)nb);
  if (!cv.ok()) return PYTO_ERR_WORKSPACE;
  void* args[] = {&n, &x, (void*)&dc, (void*)&active, &n_act, &volfrac, &move, &xmin, &xmax, &part, &change_out};
  PYTO_CUDA(cudaLaunchCooperativeKernel((const void*)k_oc_update, dim3(nb), dim3(kOcThreads), args, 0,
                                        (cudaStream_t)stream));
  PYTO_COUNT(1);
  return PYTO_OK;
}
