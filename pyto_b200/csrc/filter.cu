// Linear hat filter as a grid stencil (src/topopt_filters.py:8-38).
//
// H_ij = (r - d_ij)/r for element centres within r = rel * hx; on a box grid
// the weight depends only on the offset (dx,dy,dz), so H is a fixed stencil of
// at most (2R+1)^3 taps and Hs_i (row sum) is the sum of the in-bounds taps.
// The tap list is built on the host and passed as a kernel argument.
#include <math.h>

#include <algorithm>

#include "common.cuh"

namespace pyto {

constexpr int kMaxTaps = 343;  // radius up to 3 cells per axis

struct Taps {
  int n;
  int8_t dx[kMaxTaps], dy[kMaxTaps], dz[kMaxTaps];
  double w[kMaxTaps];
};

static int make_taps(const pyto_operator_t* op, double rel, Taps* t) {
  const double r = rel * op->hx;
  const double h[3] = {op->hx, op->hy, op->hz};
  int R[3];
  for (int d = 0; d < 3; ++d) {
    R[d] = (int)ceil(r / h[d]);
    if (R[d] > 3) return PYTO_ERR_TOO_LARGE;
  }
  t->n = 0;
  for (int dz = -R[2]; dz <= R[2]; ++dz)
    for (int dy = -R[1]; dy <= R[1]; ++dy)
      for (int dx = -R[0]; dx <= R[0]; ++dx) {
        const double px = dx * h[0], py = dy * h[1], pz = dz * h[2];
        const double d = sqrt(px * px + py * py + pz * pz);
        if (d > r) continue;
        t->dx[t->n] = (int8_t)dx;
        t->dy[t->n] = (int8_t)dy;
        t->dz[t->n] = (int8_t)dz;
        t->w[t->n] = (r - d) / r;
        t->n++;
      }
  return PYTO_OK;
}

template <int MODE>
__global__ void __launch_bounds__(256) k_filter(GridDims g, Taps t, const double* __restrict__ x,
                                                const double* __restrict__ wv, const double* __restrict__ hs,
                                                const uint8_t* __restrict__ active, double* __restrict__ y) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < g.nelem;
       e += (long long)gridDim.x * blockDim.x) {
    const int ex = (int)(e % g.nx);
    const long long rr = e / g.nx;
    const int ey = (int)(rr % g.ny);
    const int ez = (int)(rr / g.ny);
    if (active && !active[e]) {
      y[e] = 0.0;
      continue;
    }
    double acc = 0.0, ws = 0.0;
    for (int k = 0; k < t.n; ++k) {
      const int jx = ex + t.dx[k], jy = ey + t.dy[k], jz = ez + t.dz[k];
      if (jx < 0 || jx >= g.nx || jy < 0 || jy >= g.ny || jz < 0 || jz >= g.nz) continue;
      const long long j = jx + (long long)g.nx * (jy + (long long)g.ny * jz);
      if (active && !active[j]) continue;
      const double w = t.w[k];
      ws += w;
      if (MODE == PYTO_FILTER_RAW || MODE == PYTO_FILTER_DENSITY) acc = fma(w, __ldg(x + j), acc);
      if (MODE == PYTO_FILTER_CHAIN) acc = fma(w, __ldg(x + j) / __ldg(hs + j), acc);
      if (MODE == PYTO_FILTER_SENS) acc = fma(w, __ldg(wv + j) * __ldg(x + j), acc);
    }
    double out;
    if (MODE == PYTO_FILTER_RAW || MODE == PYTO_FILTER_CHAIN) out = acc;
    else if (MODE == PYTO_FILTER_DENSITY) out = acc / ws;
    else if (MODE == PYTO_FILTER_SENS) out = acc / ws / wv[e];
    else out = ws;
    y[e] = out;
  }
}

}  // namespace pyto

using namespace pyto;

extern "C" int pyto_filter(const pyto_operator_t* op, double rel_radius, int mode, const double* x,
                           const double* w, const double* hs, const uint8_t* active, double* y, void* stream) {
  if (!op || !y || !(rel_radius > 0)) return PYTO_ERR_ARG;
  if (mode != PYTO_FILTER_HS && !x) return PYTO_ERR_ARG;
  if (mode == PYTO_FILTER_CHAIN && !hs) return PYTO_ERR_ARG;
  if (mode == PYTO_FILTER_SENS && !w) return PYTO_ERR_ARG;
  if ((x && x == y) || (w && w == y)) return PYTO_ERR_ARG;
  Taps t;
  int rc = make_taps(op, rel_radius, &t);
  if (rc) return rc;
  const GridDims g = make_dims(op);
  cudaStream_t st = (cudaStream_t)stream;
  const int nb = (int)std::min<long long>((g.nelem + 255) / 256, 8 * kNumSMs);
  switch (mode) {
    case PYTO_FILTER_RAW: k_filter<PYTO_FILTER_RAW><<<nb, 256, 0, st>>>(g, t, x, w, hs, active, y); break;
    case PYTO_FILTER_DENSITY: k_filter<PYTO_FILTER_DENSITY><<<nb, 256, 0, st>>>(g, t, x, w, hs, active, y); break;
    case PYTO_FILTER_CHAIN: k_filter<PYTO_FILTER_CHAIN><<<nb, 256, 0, st>>>(g, t, x, w, hs, active, y); break;
    case PYTO_FILTER_SENS: k_filter<PYTO_FILTER_SENS><<<nb, 256, 0, st>>>(g, t, x, w, hs, active, y); break;
    case PYTO_FILTER_HS: k_filter<PYTO_FILTER_HS><<<nb, 256, 0, st>>>(g, t, x, w, hs, active, y); break;
    default: return PYTO_ERR_ARG;
  }
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}
