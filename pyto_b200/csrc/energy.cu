// Element-level kernels: energies u_e^T Ke v_e, centroid stress / von Mises
// (src/hex_structural_fea.py:152-234) and the p-norm adjoint pieces
// (src/topopt_obj_cons_sensitivities.py:181-287).
//
// All per-element algebra runs in the Hadamard corner basis: with
// u^ = Phi u_e,  u_e^T Ke v_e = u^ . (K^ v^) over the eight 3x3 parity
// blocks, and the centroid gradient of a component along axis d is
// u^(mode e_d) / (4 h_d) (the reference's gradN = (2/h) * (+-1/8)).
#include <algorithm>

#include "krylov.cuh"

namespace pyto {

constexpr int kElemThreads = 256;

__device__ __forceinline__ void elem_coords(const GridDims& g, long long e, int& ex, int& ey, int& ez) {
  ex = (int)(e % g.nx);
  const long long r = e / g.nx;
  ey = (int)(r % g.ny);
  ez = (int)(r / g.ny);
}

// Hadamard transform of an element's 8 corner values of one component:
// corners in bit order k = bx + 2 by + 4 bz; H[m] = sum phi_m(corner) a(corner).
__device__ __forceinline__ void elem_fwd(const double (&a)[8], double (&H)[8]) {
  double Fb[4], Ft[4];
  face_fwd(a[0], a[1], a[2], a[3], Fb);
  face_fwd(a[4], a[5], a[6], a[7], Ft);
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    H[f] = Ft[f] + Fb[f];
    H[f + 4] = Ft[f] - Fb[f];
  }
}

// gather the 8 corners (bit order) x 3 components of element (ex,ey,ez)
__device__ __forceinline__ void gather_elem(const GridDims& g, const double* __restrict__ u, int ex, int ey, int ez,
                                            double (&a)[3][8]) {
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int bx = k & 1, by = (k >> 1) & 1, bz = k >> 2;
    const long long n = (ex + bx) + (long long)g.sx * ((ey + by) + (long long)g.sy * (ez + bz));
#pragma unroll
    for (int c = 0; c < 3; ++c) a[c][k] = __ldg(u + 3 * n + c);
  }
}

__device__ __forceinline__ double hat_energy(const KHat& kh, const double (&U)[3][8], const double (&V)[3][8]) {
  double e = 0.0;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int m = member_mode(q, c);
      if (m == 0) continue;
      double kv = 0.0;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const int n = member_mode(q, d);
        if (n == 0) continue;
        kv = fma(kh.b[q][3 * c + d], V[d][n], kv);
      }
      e = fma(U[c][m], kv, e);
    }
  }
  return e;
}

// Element energies by element columns: thread (ex, ey) of a 32 x 8 CTA marches up
// a slab of kEnSlab element layers, keeping the face transform of the top face of
// layer z as the bottom face of layer z+1, so each layer reads one node face (its
// corners are shared with the neighbouring columns through L1) and u, v reach
// DRAM once.  SAME: v == u.
constexpr int kEnSlab = 16;

__device__ __forceinline__ void load_face(const GridDims& g, const double* __restrict__ u, int ex, int ey, int z,
                                          double (&F)[3][4]) {
  const long long n00 = ex + (long long)g.sx * (ey + (long long)g.sy * z);
  const long long n01 = n00 + g.sx;
#pragma unroll
  for (int c = 0; c < 3; ++c)
    face_fwd(__ldg(u + 3 * n00 + c), __ldg(u + 3 * (n00 + 1) + c), __ldg(u + 3 * n01 + c),
             __ldg(u + 3 * (n01 + 1) + c), F[c]);
}

template <bool SAME>
__global__ void __launch_bounds__(kElemThreads) k_elem_energy(GridDims g, KHat kh, const double* __restrict__ u,
                                                              const double* __restrict__ v,
                                                              const double* __restrict__ s, double* __restrict__ ce,
                                                              double* part, unsigned* counter, double* total) {
  __shared__ double sred[kElemThreads / 32];
  const int ex = blockIdx.x * 32 + (threadIdx.x & 31), ey = blockIdx.y * 8 + (threadIdx.x >> 5);
  const int z0 = blockIdx.z * kEnSlab, z1 = min(z0 + kEnSlab, g.nz);
  double acc = 0.0;
  if (ex < g.nx && ey < g.ny) {
    double Ub[3][4], Vb[3][4];
    load_face(g, u, ex, ey, z0, Ub);
    if (!SAME) load_face(g, v, ex, ey, z0, Vb);
    for (int ez = z0; ez < z1; ++ez) {
      double Ut[3][4], Vt[3][4];
      load_face(g, u, ex, ey, ez + 1, Ut);
      if (!SAME) load_face(g, v, ex, ey, ez + 1, Vt);
      // u^ . (K^ v^) over the parity classes; mode m = f (+) or f|4 (-): Ft +- Fb
      double en = 0.0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const int m = member_mode(q, c);
          if (m == 0) continue;
          double kv = 0.0;
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            const int nm = member_mode(q, d);
            if (nm == 0) continue;
            const int f = nm & 3;
            const double vh = SAME ? ((nm & 4) ? Ut[d][f] - Ub[d][f] : Ut[d][f] + Ub[d][f])
                                   : ((nm & 4) ? Vt[d][f] - Vb[d][f] : Vt[d][f] + Vb[d][f]);
            kv = fma(kh.b[q][3 * c + d], vh, kv);
          }
          const int f = m & 3;
          const double uh = (m & 4) ? Ut[c][f] - Ub[c][f] : Ut[c][f] + Ub[c][f];
          en = fma(uh, kv, en);
        }
      }
      const long long e = ex + (long long)g.nx * (ey + (long long)g.ny * ez);
      if (ce) ce[e] = en;
      if (total) acc = fma(__ldg(s + e), en, acc);
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          Ub[c][f] = Ut[c][f];
          if (!SAME) Vb[c][f] = Vt[c][f];
        }
    }
  }
  if (total) {
    double val[1] = {block_sum<kElemThreads>(acc, sred)};
    grid_reduce<1>(val, part, counter, (int)(gridDim.x * gridDim.y * gridDim.z),
                   [&](const double* t) { *total = t[0]; });
  }
}

static dim3 energy_grid(const GridDims& g) {
  return dim3((g.nx + 31) / 32, (g.ny + 7) / 8, (g.nz + kEnSlab - 1) / kEnSlab);
}

struct StressP {
  double D[6][6];
  double ih4[3];  // 1 / (4 h_d)
};

// centroid strain (xx,yy,zz,xy,xz,yz) from the linear Hadamard modes
__device__ __forceinline__ void centroid_strain(const StressP& P, const double (&U)[3][8], double (&eps)[6]) {
  double gr[3][3];  // gr[c][d] = d u_c / d x_d
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int d = 0; d < 3; ++d) gr[c][d] = U[c][1 << d] * P.ih4[d];
  eps[0] = gr[0][0];
  eps[1] = gr[1][1];
  eps[2] = gr[2][2];
  eps[3] = gr[0][1] + gr[1][0];
  eps[4] = gr[0][2] + gr[2][0];
  eps[5] = gr[1][2] + gr[2][1];
}

__device__ __forceinline__ double von_mises(const double (&s)[6]) {
  return sqrt(0.5 * ((s[0] - s[1]) * (s[0] - s[1]) + (s[1] - s[2]) * (s[1] - s[2]) + (s[2] - s[0]) * (s[2] - s[0])) +
              3.0 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]));
}

__global__ void __launch_bounds__(kElemThreads) k_stress(GridDims g, StressP P, const double* __restrict__ u,
                                                         const double* __restrict__ x, double q,
                                                         double* __restrict__ strain, double* __restrict__ stress,
                                                         double* __restrict__ vm, double* __restrict__ sed) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < g.nelem;
       e += (long long)gridDim.x * blockDim.x) {
    int ex, ey, ez;
    elem_coords(g, e, ex, ey, ez);
    double a[3][8], U[3][8];
    gather_elem(g, u, ex, ey, ez, a);
#pragma unroll
    for (int c = 0; c < 3; ++c) elem_fwd(a[c], U[c]);
    double eps[6], sig[6];
    centroid_strain(P, U, eps);
    const double rq = pow(x[e], q);
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      double t = 0.0;
#pragma unroll
      for (int j = 0; j < 6; ++j) t = fma(P.D[i][j], eps[j], t);
      sig[i] = t * rq;
    }
    if (strain)
#pragma unroll
      for (int i = 0; i < 6; ++i) strain[6 * e + i] = eps[i];
    if (stress)
#pragma unroll
      for (int i = 0; i < 6; ++i) stress[6 * e + i] = sig[i];
    if (vm) vm[e] = von_mises(sig);
    if (sed) {
      double w = 0.0;
#pragma unroll
      for (int i = 0; i < 6; ++i) w = fma(eps[i], sig[i], w);
      sed[e] = 0.5 * w;
    }
  }
}

__global__ void __launch_bounds__(kElemThreads) k_pow_sum(long long n, const double* __restrict__ v, double P,
                                                          double* part, unsigned* counter, double* out) {
  __shared__ double sred[kElemThreads / 32];
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    acc += pow(v[i], P);
  double val[1] = {block_sum<kElemThreads>(acc, sred)};
  grid_reduce<1>(val, part, counter, gridDim.x, [&](const double* t) { *out = t[0]; });
}

// Element part of the p-norm adjoint: T1 and t_e = x^q dpn vm^(P-1) D^T DvmDs
__global__ void __launch_bounds__(kElemThreads) k_pnorm_elem(GridDims g, StressP Pp, const double* __restrict__ u,
                                                             const double* __restrict__ x, double q, double P,
                                                             const double* __restrict__ dpn_dev,
                                                             double* __restrict__ T1, double* __restrict__ tvec) {
  const double dpn = *dpn_dev;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < g.nelem;
       e += (long long)gridDim.x * blockDim.x) {
    int ex, ey, ez;
    elem_coords(g, e, ex, ey, ez);
    double a[3][8], U[3][8];
    gather_elem(g, u, ex, ey, ez, a);
#pragma unroll
    for (int c = 0; c < 3; ++c) elem_fwd(a[c], U[c]);
    double eps[6], s0[6], sig[6];
    centroid_strain(Pp, U, eps);
    const double xe = x[e];
    const double rq = pow(xe, q);  // postprocess relaxes the stress with the raw x
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      double t = 0.0;
#pragma unroll
      for (int j = 0; j < 6; ++j) t = fma(Pp.D[i][j], eps[j], t);
      s0[i] = t;  // D B u_e
      sig[i] = t * rq;
    }
    const double vmv = von_mises(sig);
    // d vm / d sigma; at vm = 0 (an unstressed or void element) vm^(P-1) d vm/d sigma
    // = vm^(P-2) V sigma has the limit 0, so the element contributes nothing
    const double iv = vmv > 0.0 ? 1.0 / vmv : 0.0;
    double dv[6];
    dv[0] = 0.5 * iv * (2.0 * sig[0] - sig[1] - sig[2]);
    dv[1] = 0.5 * iv * (2.0 * sig[1] - sig[0] - sig[2]);
    dv[2] = 0.5 * iv * (2.0 * sig[2] - sig[0] - sig[1]);
    dv[3] = 3.0 * iv * sig[3];
    dv[4] = 3.0 * iv * sig[4];
    dv[5] = 3.0 * iv * sig[5];
    const double xc = fmax(xe, 1e-12);
    const double vp = pow(vmv, P - 1.0);
    double dot = 0.0;
#pragma unroll
    for (int i = 0; i < 6; ++i) dot = fma(dv[i], s0[i], dot);
    T1[e] = dpn * (q * pow(xc, q - 1.0) * vp * dot);
    const double sc = pow(xc, q) * dpn * vp;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      double t = 0.0;
#pragma unroll
      for (int j = 0; j < 6; ++j) t = fma(Pp.D[j][i], dv[j], t);
      tvec[6 * e + i] = sc * t;
    }
  }
}

// Node-owned gather of g = sum_e B^T t_e (no atomics)
__global__ void __launch_bounds__(kElemThreads) k_pnorm_gather(GridDims g, StressP Pp,
                                                               const double* __restrict__ tvec,
                                                               double* __restrict__ gout) {
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < g.nnodes;
       n += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(n % g.sx);
    const long long r = n / g.sx;
    const int iy = (int)(r % g.sy);
    const int iz = (int)(r / g.sy);
    double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int bz = 0; bz < 2; ++bz)
#pragma unroll
      for (int by = 0; by < 2; ++by)
#pragma unroll
        for (int bx = 0; bx < 2; ++bx) {
          // node is corner (bx,by,bz) of element (ix-bx, iy-by, iz-bz)
          const int ex = ix - bx, ey = iy - by, ez = iz - bz;
          if (ex < 0 || ex >= g.nx || ey < 0 || ey >= g.ny || ez < 0 || ez >= g.nz) continue;
          const double* t = tvec + 6 * (ex + (long long)g.nx * (ey + (long long)g.ny * ez));
          const double g0 = (bx ? 1.0 : -1.0) * Pp.ih4[0];
          const double g1 = (by ? 1.0 : -1.0) * Pp.ih4[1];
          const double g2 = (bz ? 1.0 : -1.0) * Pp.ih4[2];
          acc[0] += g0 * t[0] + g1 * t[3] + g2 * t[4];
          acc[1] += g1 * t[1] + g0 * t[3] + g2 * t[5];
          acc[2] += g2 * t[2] + g0 * t[4] + g1 * t[5];
        }
#pragma unroll
    for (int c = 0; c < 3; ++c) gout[3 * n + c] = acc[c];
  }
}

static StressP make_stress(const pyto_operator_t* op) {
  StressP P;
  const double E = op->E, nu = op->nu;
  const double c = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) P.D[i][j] = 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) P.D[i][j] = c * (i == j ? 1.0 - nu : nu);
  for (int i = 3; i < 6; ++i) P.D[i][i] = c * (1.0 - 2.0 * nu) / 2.0;
  P.ih4[0] = 1.0 / (4.0 * op->hx);
  P.ih4[1] = 1.0 / (4.0 * op->hy);
  P.ih4[2] = 1.0 / (4.0 * op->hz);
  return P;
}

int elem_blocks(long long n) { return (int)std::min<long long>((n + kElemThreads - 1) / kElemThreads, 8 * kNumSMs); }

}  // namespace pyto

using namespace pyto;

extern "C" int pyto_elem_energy(const pyto_operator_t* op, const double* u, const double* v, const double* s,
                                double* ce, double* total, void* ws, size_t ws_bytes, void* stream) {
  if (!op || !u || !v || (total && !s) || (!ce && !total)) return PYTO_ERR_ARG;
  const GridDims g = make_dims(op);
  cudaStream_t st = (cudaStream_t)stream;
  double* part = nullptr;
  unsigned* counter = nullptr;
  const dim3 eg = energy_grid(g);
  const long long nb = (long long)eg.x * eg.y * eg.z;
  if (total) {
    Carver cv{(char*)ws, 0, ws_bytes};
    counter = cv.take<unsigned>(64);
    part = cv.take<double>((size_t)nb);
    if (!cv.ok()) return PYTO_ERR_WORKSPACE;
    PYTO_CUDA(cudaMemsetAsync(counter, 0, 64 * sizeof(unsigned), st));
  }
  if (u == v)
    k_elem_energy<true><<<eg, kElemThreads, 0, st>>>(g, make_khat(op), u, v, s, ce, part, counter, total);
  else
    k_elem_energy<false><<<eg, kElemThreads, 0, st>>>(g, make_khat(op), u, v, s, ce, part, counter, total);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}

extern "C" int pyto_stress(const pyto_operator_t* op, const double* u, const double* x, double q, double* strain,
                           double* stress, double* vm, double* sed, void* stream) {
  if (!op || !u || !x) return PYTO_ERR_ARG;
  const GridDims g = make_dims(op);
  k_stress<<<elem_blocks(g.nelem), kElemThreads, 0, (cudaStream_t)stream>>>(g, make_stress(op), u, x, q, strain,
                                                                             stress, vm, sed);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}

extern "C" int pyto_pnorm_sum(const pyto_operator_t* op, const double* vm, double P, double* sum_out, void* ws,
                              size_t ws_bytes, void* stream) {
  if (!op || !vm || !sum_out) return PYTO_ERR_ARG;
  const GridDims g = make_dims(op);
  cudaStream_t st = (cudaStream_t)stream;
  const int nb = elem_blocks(g.nelem);
  Carver cv{(char*)ws, 0, ws_bytes};
  unsigned* counter = cv.take<unsigned>(64);
  double* part = cv.take<double>(nb);
  if (!cv.ok()) return PYTO_ERR_WORKSPACE;
  PYTO_CUDA(cudaMemsetAsync(counter, 0, 64 * sizeof(unsigned), st));
  k_pow_sum<<<nb, kElemThreads, 0, st>>>(g.nelem, vm, P, part, counter, sum_out);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}

extern "C" int pyto_pnorm_adjoint(const pyto_operator_t* op, const double* u, const double* x, double q, double P,
                                  const double* dpn_dev, double* T1, double* gvec, double* tvec, void* stream) {
  if (!op || !u || !x || !dpn_dev || !T1 || !gvec || !tvec) return PYTO_ERR_ARG;
  const GridDims g = make_dims(op);
  cudaStream_t st = (cudaStream_t)stream;
  const StressP Pp = make_stress(op);
  k_pnorm_elem<<<elem_blocks(g.nelem), kElemThreads, 0, st>>>(g, Pp, u, x, q, P, dpn_dev, T1, tvec);
  PYTO_COUNT(1);
  k_pnorm_gather<<<elem_blocks(g.nnodes), kElemThreads, 0, st>>>(g, Pp, tvec, gvec);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}
