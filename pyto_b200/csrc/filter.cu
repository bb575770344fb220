// Linear hat filter as a grid stencil (src/topopt_filters.py:8-38).
//
// H_ij = (r - d_ij)/r for element centres within r = rel * hx; on a box grid
// the weight depends only on the offset (dx,dy,dz), so H is a fixed stencil of
// at most (2R+1)^3 taps and Hs_i (row sum) is the sum of the in-bounds taps.
// The tap list is built on the host and passed as a kernel argument.
#include <math.h>
#include <stdlib.h>

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

// Tiled stencil: a CTA produces a kFx x kFy x kFz block of outputs (256 threads,
// one (x, y) column each, marching over kFz planes) from a shared-memory copy of
// the block plus an R-element halo: v = the filtered quantity (0 outside the grid
// or on inactive elements) and m = 1 where a tap counts (in the grid and active).
// Tap offsets into the tile are precomputed on the host.  Blocks whose halo lies
// inside the grid, without an active mask, take the row sum from the host (the
// sum of all weights) and skip m.
constexpr int kFx = 32, kFy = 8, kFz = 8;

struct TileTaps {
  int n, R;
  double wsum;
  int off[kMaxTaps];
  double w[kMaxTaps];
};

static void tile_taps(const Taps& t, int R, TileTaps* tt) {
  const int PX = kFx + 2 * R, PY = kFy + 2 * R;
  tt->n = t.n;
  tt->R = R;
  tt->wsum = 0.0;
  for (int k = 0; k < t.n; ++k) {
    tt->off[k] = (t.dz[k] * PY + t.dy[k]) * PX + t.dx[k];
    tt->w[k] = t.w[k];
    tt->wsum += t.w[k];
  }
}

template <int MODE>
__global__ void __launch_bounds__(256) k_filter(GridDims g, TileTaps t, const double* __restrict__ x,
                                                const double* __restrict__ wv, const double* __restrict__ hs,
                                                const uint8_t* __restrict__ active, double* __restrict__ y) {
  extern __shared__ double fsm[];
  const int R = t.R;
  const int PX = kFx + 2 * R, PY = kFy + 2 * R, PZ = kFz + 2 * R;
  const int tile = PX * PY * PZ;
  double* sv = fsm;                                  // [PZ][PY][PX] values
  float* sm = reinterpret_cast<float*>(fsm + tile);  // [PZ][PY][PX] tap masks
  const int X0 = blockIdx.x * kFx, Y0 = blockIdx.y * kFy, Z0 = blockIdx.z * kFz;
  const bool interior = !active && X0 - R >= 0 && Y0 - R >= 0 && Z0 - R >= 0 && X0 + kFx + R <= g.nx &&
                        Y0 + kFy + R <= g.ny && Z0 + kFz + R <= g.nz;
  for (int q = threadIdx.x; q < tile; q += blockDim.x) {
    const int lx = q % PX, r2 = q / PX, ly = r2 % PY, lz = r2 / PY;
    const int gx = X0 - R + lx, gy = Y0 - R + ly, gz = Z0 - R + lz;
    double v = 0.0;
    float m = 0.f;
    if (gx >= 0 && gx < g.nx && gy >= 0 && gy < g.ny && gz >= 0 && gz < g.nz) {
      const long long j = gx + (long long)g.nx * (gy + (long long)g.ny * gz);
      if (!active || active[j]) {
        m = 1.f;
        if (MODE == PYTO_FILTER_RAW || MODE == PYTO_FILTER_DENSITY) v = __ldg(x + j);
        if (MODE == PYTO_FILTER_CHAIN) v = __ldg(x + j) / __ldg(hs + j);
        if (MODE == PYTO_FILTER_SENS) v = __ldg(wv + j) * __ldg(x + j);
      }
    }
    sv[q] = v;
    sm[q] = m;
  }
  __syncthreads();
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int ex = X0 + tx, ey = Y0 + ty;
  if (ex >= g.nx || ey >= g.ny) return;
  for (int z = 0; z < kFz && Z0 + z < g.nz; ++z) {
    const long long e = ex + (long long)g.nx * (ey + (long long)g.ny * (Z0 + z));
    if (active && !active[e]) {
      y[e] = 0.0;
      continue;
    }
    const int c = ((z + R) * PY + (ty + R)) * PX + (tx + R);
    double acc = 0.0, ws = 0.0;
    if (interior) {
      for (int k = 0; k < t.n; ++k) acc = fma(t.w[k], sv[c + t.off[k]], acc);
      ws = t.wsum;
    } else {
      for (int k = 0; k < t.n; ++k) {
        const double w = t.w[k];
        acc = fma(w, sv[c + t.off[k]], acc);
        ws = fma(w, (double)sm[c + t.off[k]], ws);
      }
    }
    double out;
    if (MODE == PYTO_FILTER_RAW || MODE == PYTO_FILTER_CHAIN) out = acc;
    else if (MODE == PYTO_FILTER_DENSITY) out = acc / ws;
    else if (MODE == PYTO_FILTER_SENS) out = acc / ws / __ldg(wv + e);
    else out = ws;
    y[e] = out;
  }
}

static size_t filter_smem(int R) {
  const size_t tile = (size_t)(kFx + 2 * R) * (kFy + 2 * R) * (kFz + 2 * R);
  return tile * (sizeof(double) + sizeof(float));
}

template <int MODE>
static int launch_filter(const GridDims& g, const TileTaps& tt, const double* x, const double* w, const double* hs,
                         const uint8_t* active, double* y, cudaStream_t st) {
  static PerDevice attr;
  if (attr.needed()) {
    PYTO_CUDA(cudaFuncSetAttribute(k_filter<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)filter_smem(3)));
    attr.done();
  }
  const dim3 grid((g.nx + kFx - 1) / kFx, (g.ny + kFy - 1) / kFy, (g.nz + kFz - 1) / kFz);
  k_filter<MODE><<<grid, 256, filter_smem(tt.R), st>>>(g, tt, x, w, hs, active, y);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
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
  int R = 0;
  for (int k = 0; k < t.n; ++k) R = std::max(R, std::max(abs(t.dx[k]), std::max(abs(t.dy[k]), abs(t.dz[k]))));
  TileTaps tt;
  tile_taps(t, R, &tt);
  const GridDims g = make_dims(op);
  cudaStream_t st = (cudaStream_t)stream;
  switch (mode) {
    case PYTO_FILTER_RAW: return launch_filter<PYTO_FILTER_RAW>(g, tt, x, w, hs, active, y, st);
    case PYTO_FILTER_DENSITY: return launch_filter<PYTO_FILTER_DENSITY>(g, tt, x, w, hs, active, y, st);
    case PYTO_FILTER_CHAIN: return launch_filter<PYTO_FILTER_CHAIN>(g, tt, x, w, hs, active, y, st);
    case PYTO_FILTER_SENS: return launch_filter<PYTO_FILTER_SENS>(g, tt, x, w, hs, active, y, st);
    case PYTO_FILTER_HS: return launch_filter<PYTO_FILTER_HS>(g, tt, x, w, hs, active, y, st);
    default: return PYTO_ERR_ARG;
  }
}

// ---------------------------------------------------------------------------
// Symmetry and extrusion maps of the element field on a full box grid
// (src/topopt_filters.py:292-393 mirror symmetry, :595-716 extrusion), composed
// with the smoothing filter as H = H_s F_1 F_2 ... (src/topopt_common.py:127-159).
// ---------------------------------------------------------------------------
namespace pyto {

__device__ __forceinline__ void elem_ijk(const GridDims& g, long long e, int& i, int& j, int& k) {
  i = (int)(e % g.nx);
  const long long r = e / g.nx;
  j = (int)(r % g.ny);
  k = (int)(r / g.ny);
}

// y_e = (F (x o pre))_e / post_e (pre, post may be null).  Mirror about the mid-plane
// normal to `axis`: F x = (x + x[mirror]) / 2 (the self-mirrored middle layer keeps x).
__global__ void k_mirror(GridDims g, int axis, const double* __restrict__ x, const double* __restrict__ pre,
                         const double* __restrict__ post, double* __restrict__ y) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < g.nelem;
       e += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    elem_ijk(g, e, i, j, k);
    if (axis == 0) i = g.nx - 1 - i;
    else if (axis == 1) j = g.ny - 1 - j;
    else k = g.nz - 1 - k;
    const long long m = i + (long long)g.nx * (j + (long long)g.ny * k);
    const double a = x[e] * (pre ? pre[e] : 1.0), b = x[m] * (pre ? pre[m] : 1.0);
    double v = 0.5 * (a + b);
    if (post) v /= post[e];
    y[e] = v;
  }
}

// Extrusion along `axis`, with the reference's weights: the element lines along axis
// are visited from the one with the lowest element id, whose first element joins its
// own line twice, so with n elements per line and w = 1/(n+1):
//   (F x)_e = w (sum_line x + x_first) * (2 if e is the line's first element else 1).
// One thread per line.
__global__ void k_extrude(GridDims g, int axis, const double* __restrict__ x, const double* __restrict__ pre,
                          const double* __restrict__ post, double* __restrict__ y) {
  const int n = axis == 0 ? g.nx : axis == 1 ? g.ny : g.nz;
  const long long stride = axis == 0 ? 1 : axis == 1 ? g.nx : (long long)g.nx * g.ny;
  const long long nlines = g.nelem / n;
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < nlines;
       l += (long long)gridDim.x * blockDim.x) {
    long long e0;  // first element of line l
    if (axis == 0) e0 = l * g.nx;
    else if (axis == 1) e0 = (l % g.nx) + (l / g.nx) * (long long)g.nx * g.ny;
    else e0 = l;
    double sum = 0.0;
    for (int t = 0; t < n; ++t) {
      const long long e = e0 + t * stride;
      sum += x[e] * (pre ? pre[e] : 1.0);
    }
    sum += x[e0] * (pre ? pre[e0] : 1.0);
    const double w = 1.0 / (n + 1);
    for (int t = 0; t < n; ++t) {
      const long long e = e0 + t * stride;
      double v = (t == 0 ? 2.0 : 1.0) * w * sum;
      if (post) v /= post[e];
      y[e] = v;
    }
  }
}

// y = x o mul / (div1 o div2) (each factor optional)
__global__ void k_vec_scale(long long n, const double* __restrict__ x, const double* __restrict__ mul,
                            const double* __restrict__ div1, const double* __restrict__ div2,
                            double* __restrict__ y) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double v = x[i];
    if (mul) v *= mul[i];
    if (div1) v /= div1[i];
    if (div2) v /= div2[i];
    y[i] = v;
  }
}

}  // namespace pyto

extern "C" int pyto_symmetry_filter(const pyto_operator_t* op, int kind, int axis, const double* x,
                                    const double* pre, const double* post, double* y, void* stream) {
  if (!op || !x || !y || x == y || axis < 0 || axis > 2) return PYTO_ERR_ARG;
  const GridDims g = make_dims(op);
  cudaStream_t st = (cudaStream_t)stream;
  if (kind == PYTO_SYM_MIRROR) {
    const int nb = (int)std::min<long long>((g.nelem + 255) / 256, 8 * kNumSMs);
    k_mirror<<<nb, 256, 0, st>>>(g, axis, x, pre, post, y);
  } else if (kind == PYTO_SYM_EXTRUDE) {
    const int n = axis == 0 ? g.nx : axis == 1 ? g.ny : g.nz;
    const long long nlines = g.nelem / n;
    const int nb = (int)std::min<long long>((nlines + 127) / 128, 8 * kNumSMs);
    k_extrude<<<nb, 128, 0, st>>>(g, axis, x, pre, post, y);
  } else {
    return PYTO_ERR_ARG;
  }
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}

extern "C" int pyto_vec_scale(int64_t n, const double* x, const double* mul, const double* div1,
                              const double* div2, double* y, void* stream) {
  if (!x || !y || n < 0) return PYTO_ERR_ARG;
  if (n == 0) return PYTO_OK;
  const int nb = (int)std::min<long long>((n + 255) / 256, 8 * kNumSMs);
  k_vec_scale<<<nb, 256, 0, (cudaStream_t)stream>>>(n, x, mul, div1, div2, y);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}
