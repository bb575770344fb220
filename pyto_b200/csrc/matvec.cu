// FP64 operator kernels: BC mask, SIMP scaling, Jacobi data, and the
// matrix-free K(s) u (algorithm notes in matvec.cuh).
#include <algorithm>

#include "matvec.cuh"

namespace pyto {

// ---------------------------------------------------------------------------
// matrix-free y = K(s) u
// ---------------------------------------------------------------------------
template <int TX, int TY, bool DOT>
__global__ void __launch_bounds__(TX* TY, 2)
    k_matvec64(GridDims g, KHat kh, const double* __restrict__ s, const uint8_t* __restrict__ mask,
               const double* __restrict__ u, double* __restrict__ y, int zc, int mode, double* part,
               unsigned* counter, double* dot_out) {
  using T = MvTile<TX, TY>;
  __shared__ double su[2][3][T::PLANE];
  __shared__ double sc[3][TY][TX];
  __shared__ double sred[T::NT / 32];

  const int tid = threadIdx.x;
  const int tx = tid & (TX - 1), ty = tid / TX;
  const int X0 = blockIdx.x * (TX - 1), Y0 = blockIdx.y * (TY - 1);
  const int Z0 = blockIdx.z * zc;
  const int Z1 = min(Z0 + zc, g.sz);
  const int ex = X0 - 1 + tx, ey = Y0 - 1 + ty;
  const bool col_in = ex >= 0 && ex < g.nx && ey >= 0 && ey < g.ny;
  const bool mask_in = (mode & PYTO_MASK_IN) && mask != nullptr;
  const bool mask_out = (mode & PYTO_MASK_OUT) && mask != nullptr;
  const long long plane_nodes = (long long)g.sx * g.sy;

  // flat, coalesced plane loader: tile rows of PX nodes x 3 components
  double pre[T::LOADS];
  auto load_plane = [&](int k) {
#pragma unroll
    for (int i = 0; i < T::LOADS; ++i) {
      const int idx = tid + i * T::NT;
      double v = 0.0;
      if (idx < T::PLANE_D && k >= 0 && k < g.sz) {
        const int row = idx / (3 * T::PX);
        const int rem = idx - row * 3 * T::PX;
        const int nxl = rem / 3;
        const int c = rem - 3 * nxl;
        const int gx = X0 - 1 + nxl, gy = Y0 - 1 + row;
        if (gx >= 0 && gx < g.sx && gy >= 0 && gy < g.sy) {
          const long long node = gx + (long long)g.sx * gy + plane_nodes * k;
          v = __ldg(u + 3 * node + c);
          if (mask_in && ((__ldg(mask + node) >> c) & 1)) v = 0.0;
        }
      }
      pre[i] = v;
    }
  };
  auto store_plane = [&](int b) {
#pragma unroll
    for (int i = 0; i < T::LOADS; ++i) {
      const int idx = tid + i * T::NT;
      if (idx < T::PLANE_D) {
        const int row = idx / (3 * T::PX);
        const int rem = idx - row * 3 * T::PX;
        const int nxl = rem / 3;
        const int c = rem - 3 * nxl;
        su[b][c][row * T::PX + nxl] = pre[i];
      }
    }
  };
  auto load_s = [&](int ez) -> double {
    if (!col_in || ez < 0 || ez >= g.nz) return 0.0;
    return __ldg(s + ex + (long long)g.nx * (ey + (long long)g.ny * ez));
  };
  auto face = [&](int b, double (&F)[3][4]) {
    const int i00 = ty * T::PX + tx;
#pragma unroll
    for (int c = 0; c < 3; ++c)
      face_fwd(su[b][c][i00], su[b][c][i00 + 1], su[b][c][i00 + T::PX], su[b][c][i00 + T::PX + 1], F[c]);
  };

  // prologue: bottom plane of the first element layer
  load_plane(Z0 - 1);
  store_plane(0);
  load_plane(Z0);
  double s_next = load_s(Z0 - 1);
  __syncthreads();
  double Fb[3][4], Gp[3][4];
  face(0, Fb);
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int f = 0; f < 4; ++f) Gp[c][f] = 0.0;

  double dot = 0.0;
  const bool owner = tx < TX - 1 && ty < TY - 1 && (X0 + tx) < g.sx && (Y0 + ty) < g.sy;

  for (int ez = Z0 - 1; ez < Z1; ++ez) {
    const int bt = (ez - Z0 + 2) & 1;  // buffer of plane ez+1
    store_plane(bt);
    if (ez + 2 <= Z1) load_plane(ez + 2);
    const double se = s_next;
    if (ez + 1 < Z1) s_next = load_s(ez + 1);
    __syncthreads();

    double Ft[3][4], Gn[3][4];
    face(bt, Ft);
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int f = 0; f < 4; ++f) Gn[c][f] = 0.0;
    hex8_core<double>(kh, se, Fb, Ft, Gp, Gn);  // Gp: plane ez complete, Gn: pending for ez+1

    if (ez >= Z0) {
      double cT[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        double c00, c10, c01, c11;
        face_inv(Gp[c], c00, c10, c01, c11);
        cT[c] = c11 + __shfl_down_sync(0xffffffffu, c01, 1);
        sc[c][ty][tx] = c10 + __shfl_down_sync(0xffffffffu, c00, 1);
      }
      // u of the owned node (for the fused dot) before the exchange barrier
      double un[3] = {0.0, 0.0, 0.0};
      if (DOT && owner) {
        const int bb = (ez - Z0 + 1) & 1;  // buffer of plane ez
        const int li = (ty + 1) * T::PX + tx + 1;
#pragma unroll
        for (int c = 0; c < 3; ++c) un[c] = su[bb][c][li];
      }
      __syncthreads();
      if (owner) {
        const long long node = (X0 + tx) + (long long)g.sx * (Y0 + ty) + plane_nodes * ez;
        const int mk = mask_out ? (int)__ldg(mask + node) : 0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          double v = cT[c] + sc[c][ty + 1][tx];
          if ((mk >> c) & 1) v = 0.0;
          y[3 * node + c] = v;
          if (DOT) dot = fma(un[c], v, dot);
        }
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        Fb[c][f] = Ft[c][f];
        Gp[c][f] = Gn[c][f];
      }
  }
  if (DOT) {
    const double bsum = block_sum<T::NT>(dot, sred);
    double v[1] = {bsum};
    grid_reduce<1>(v, part, counter, (int)(gridDim.x * gridDim.y * gridDim.z),
                   [&](const double* t) { *dot_out = t[0]; });
  }
}

// launcher used by the entry point and by the solvers
int launch_matvec64(const pyto_operator_t* op, const double* s, const uint8_t* mask, const double* u, double* y,
                    int mode, double* part, unsigned* counter, double* dot, cudaStream_t st) {
  constexpr int TX = 32, TY = 8;
  const GridDims g = make_dims(op);
  const KHat kh = make_khat(op);
  const MvLaunch L = matvec_launch<TX, TY>(g);
  if (dot)
    k_matvec64<TX, TY, true><<<L.grid, TX * TY, 0, st>>>(g, kh, s, mask, u, y, L.zc, mode, part, counter, dot);
  else
    k_matvec64<TX, TY, false><<<L.grid, TX * TY, 0, st>>>(g, kh, s, mask, u, y, L.zc, mode, nullptr, nullptr,
                                                          nullptr);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}

long long matvec_blocks(const pyto_operator_t* op) { return matvec_launch<32, 8>(make_dims(op)).nblocks; }

// ---------------------------------------------------------------------------
// BC mask, SIMP, Jacobi
// ---------------------------------------------------------------------------
__global__ void k_bc_mask(const int64_t* __restrict__ fixed, int64_t n, long long ndof, unsigned* mask_words) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t d = fixed[i];
    if (d < 0 || d >= ndof) continue;
    const int64_t node = d / 3;
    const int c = (int)(d - 3 * node);
    atomicOr(mask_words + (node >> 2), 1u << (8 * (node & 3) + c));
  }
}

__global__ void k_simp(const double* __restrict__ x, const uint8_t* __restrict__ active, int64_t n, double p,
                       double emin, double* __restrict__ s, double* __restrict__ ds) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double xi = x[i];
    const bool on = active == nullptr || active[i] != 0;
    s[i] = on ? emin + pow(xi, p) * (1.0 - emin) : 0.0;
    if (ds) ds[i] = on ? p * pow(xi, p - 1.0) * (1.0 - emin) : 0.0;
  }
}

// node-owned: sum of s over the (up to) 8 incident elements
__global__ void k_jacobi(GridDims g, KHat kh, const double* __restrict__ s, const uint8_t* __restrict__ mask,
                         double* __restrict__ winv, uint8_t* __restrict__ flags, double* __restrict__ diag) {
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < g.nnodes;
       n += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(n % g.sx);
    const long long r = n / g.sx;
    const int iy = (int)(r % g.sy);
    const int iz = (int)(r / g.sy);
    double acc = 0.0;
#pragma unroll
    for (int dz = -1; dz <= 0; ++dz)
#pragma unroll
      for (int dy = -1; dy <= 0; ++dy)
#pragma unroll
        for (int dx = -1; dx <= 0; ++dx) {
          const int ex = ix + dx, ey = iy + dy, ez = iz + dz;
          if (ex >= 0 && ex < g.nx && ey >= 0 && ey < g.ny && ez >= 0 && ez < g.nz)
            acc += s[ex + (long long)g.nx * (ey + (long long)g.ny * ez)];
        }
    int fl = mask ? (mask[n] & 7) : 0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double d = kh.kd[c] * acc;
      if (fabs(d) < 1e-12) fl |= 8 << c;
      if (diag) diag[3 * n + c] = d;
    }
    winv[n] = acc != 0.0 ? 1.0 / acc : 0.0;
    flags[n] = (uint8_t)fl;
  }
}

}  // namespace pyto

using namespace pyto;

extern "C" int pyto_bc_mask(const pyto_operator_t* op, const int64_t* fixed_dofs, int64_t n_fixed, uint8_t* mask,
                            void* stream) {
  if (!op || !mask || (n_fixed > 0 && !fixed_dofs) || ((uintptr_t)mask & 3)) return PYTO_ERR_ARG;
  const GridDims g = make_dims(op);
  cudaStream_t st = (cudaStream_t)stream;
  // the buffer holds round_up(nnodes, 4) bytes (see the header contract)
  PYTO_CUDA(cudaMemsetAsync(mask, 0, (size_t)((g.nnodes + 3) / 4) * 4, st));
  if (n_fixed > 0) {
    const int nb = (int)std::min<int64_t>((n_fixed + 255) / 256, 4 * kNumSMs);
    k_bc_mask<<<nb, 256, 0, st>>>(fixed_dofs, n_fixed, 3 * g.nnodes, (unsigned*)mask);
    PYTO_COUNT(1);
    PYTO_LAUNCH_CHECK();
  }
  return PYTO_OK;
}

extern "C" int pyto_simp(const double* x, const uint8_t* active, int64_t n, double penal, double emin, double* s,
                         double* ds, void* stream) {
  if (!x || !s || n < 0) return PYTO_ERR_ARG;
  if (n == 0) return PYTO_OK;
  const int nb = (int)std::min<int64_t>((n + 255) / 256, 8 * kNumSMs);
  k_simp<<<nb, 256, 0, (cudaStream_t)stream>>>(x, active, n, penal, emin, s, ds);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}

extern "C" int pyto_jacobi(const pyto_operator_t* op, const double* s, const uint8_t* mask, double* winv,
                           uint8_t* flags, double* diag_out, void* stream) {
  if (!op || !s || !winv || !flags) return PYTO_ERR_ARG;
  const GridDims g = make_dims(op);
  const int nb = (int)std::min<long long>((g.nnodes + 255) / 256, 8 * kNumSMs);
  k_jacobi<<<nb, 256, 0, (cudaStream_t)stream>>>(g, make_khat(op), s, mask, winv, flags, diag_out);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}

extern "C" int pyto_matvec(const pyto_operator_t* op, const double* s, const uint8_t* mask, const double* u,
                           double* y, int mode, double* dot, void* ws, size_t ws_bytes, void* stream) {
  if (!op || !s || !u || !y || u == y) return PYTO_ERR_ARG;
  double* part = nullptr;
  unsigned* counter = nullptr;
  if (dot) {
    Carver cv{(char*)ws, 0, ws_bytes};
    counter = cv.take<unsigned>(64);
    part = cv.take<double>((size_t)matvec_blocks(op));
    if (!cv.ok()) return PYTO_ERR_WORKSPACE;
    PYTO_CUDA(cudaMemsetAsync(counter, 0, 64 * sizeof(unsigned), (cudaStream_t)stream));
  }
  return launch_matvec64(op, s, mask, u, y, mode, part, counter, dot, (cudaStream_t)stream);
}
