// Thermal hex8 path (src/hex_thermal_fea.py:19-117): K(s) = sum_e s_e Ke with the
// 8x8 conduction matrix of a box element (src/hex_element_stiffness.py:340-385),
// one temperature DOF per node (edofMatThermal = the element's corner nodes,
// src/hex_mesher.py:1120-1133), applied matrix-free; Jacobi PCG with scipy cg's
// stopping test; element energies T_e^T Ke T_e for the thermal compliance.
//
// For a box element every coordinate reflection is a symmetry of Ke, so
// Ke[a][b] depends only on which coordinates of corners a and b differ:
// Ke[a][b] = k[bits(a) ^ bits(b)] with the corner's (x, y, z) offsets as bits
// 0, 1, 2 -- eight numbers instead of 64.  Each node sums the contributions of
// its (up to) 8 elements from its 27 neighbours (node-owned: no atomics,
// bitwise reproducible).
#include <algorithm>

#include "krylov.cuh"

namespace pyto {

// reference corner order (src/hex_mesher.py:120-124) -> offset bits x | y<<1 | z<<2
__host__ __device__ constexpr int corner_bits(int k) {
  return (k == 0) ? 0 : (k == 1) ? 1 : (k == 2) ? 3 : (k == 3) ? 2 : (k == 4) ? 4 : (k == 5) ? 5 : (k == 6) ? 7 : 6;
}

struct TK {
  double k[8];  // Ke as a function of the differing offset bits
};

inline GridDims thermal_dims(const pyto_thermal_t* t) {
  GridDims g;
  g.nx = t->nelx; g.ny = t->nely; g.nz = t->nelz;
  g.sx = g.nx + 1; g.sy = g.ny + 1; g.sz = g.nz + 1;
  g.nnodes = (long long)g.sx * g.sy * g.sz;
  g.nelem = (long long)g.nx * g.ny * g.nz;
  return g;
}

inline TK make_tk(const pyto_thermal_t* t) {
  TK k;
  for (int d = 0; d < 8; ++d) k.k[d] = t->kxor[d];
  return k;
}

// y_n = sum_{e ni n} s_e sum_d k[d] u(n + sigma_e o d); mode bit 0: u read as 0 on fixed
// nodes, bit 1: y written as 0 on fixed nodes.  Optional dot = sum u_masked . y
// (deterministic cross-block reduction).
__global__ void __launch_bounds__(256) k_thermal_matvec(GridDims g, TK tk, const double* __restrict__ s,
                                                        const uint8_t* __restrict__ mask,
                                                        const double* __restrict__ u, double* __restrict__ y,
                                                        int mode, double* part, unsigned* counter, double* dot) {
  __shared__ double sred[8];
  double acc_dot = 0.0;
  const long long P = (long long)g.sx * g.sy;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < g.nnodes;
       n += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(n % g.sx);
    const long long r = n / g.sx;
    const int iy = (int)(r % g.sy);
    const int iz = (int)(r / g.sy);
    // 3x3x3 neighbourhood (0 outside the grid or, with MASK_IN, on fixed nodes)
    double U[3][3][3];
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
      for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
          const int jx = ix + dx, jy = iy + dy, jz = iz + dz;
          double v = 0.0;
          if (jx >= 0 && jx < g.sx && jy >= 0 && jy < g.sy && jz >= 0 && jz < g.sz) {
            const long long m = jx + (long long)g.sx * jy + P * jz;
            v = __ldg(u + m);
            if ((mode & PYTO_MASK_IN) && mask && (mask[m] & 1)) v = 0.0;
          }
          U[dz + 1][dy + 1][dx + 1] = v;
        }
    double acc = 0.0;
#pragma unroll
    for (int oz = 0; oz < 2; ++oz)
#pragma unroll
      for (int oy = 0; oy < 2; ++oy)
#pragma unroll
        for (int ox = 0; ox < 2; ++ox) {
          const int ex = ix - ox, ey = iy - oy, ez = iz - oz;  // n is corner (ox, oy, oz) of e
          if (ex < 0 || ex >= g.nx || ey < 0 || ey >= g.ny || ez < 0 || ez >= g.nz) continue;
          const double se = __ldg(s + ex + (long long)g.nx * (ey + (long long)g.ny * ez));
          double t = 0.0;
#pragma unroll
          for (int d = 0; d < 8; ++d) {
            const int mx = (d & 1) ? 1 - 2 * ox : 0, my = (d & 2) ? 1 - 2 * oy : 0, mz = (d & 4) ? 1 - 2 * oz : 0;
            t = fma(tk.k[d], U[mz + 1][my + 1][mx + 1], t);
          }
          acc = fma(se, t, acc);
        }
    if ((mode & PYTO_MASK_OUT) && mask && (mask[n] & 1)) acc = 0.0;
    y[n] = acc;
    if (dot) acc_dot = fma(U[1][1][1], acc, acc_dot);
  }
  if (dot) {
    double v[1] = {block_sum<256>(acc_dot, sred)};
    grid_reduce<1>(v, part, counter, gridDim.x, [&](const double* tot) { *dot = tot[0]; });
  }
}

// The same operator as a z-march over node planes (the decomposition of the structural
// tile kernel, one temperature per node).  Ke[a][b] = k[a ^ b] is diagonal in the corner
// Walsh basis phi_m(a) = prod_{d in m} (2 a_d - 1): Ke phi_m = lam_m phi_m with
// lam_m = sum_d k[d] (-1)^popcount(m & d) (lam_0 = 0 for conduction).  Per element:
// the 2-D transform of its top face (the bottom face is the previous layer's top), the
// even / odd z-combinations, lam_m / 8 per mode, s applied per output pair (bottom face +=
// s (even - odd), top face = s (even + odd)), the inverse transform of the completed
// bottom face: 48 FP64 operations instead of 64 FMAs from 27 gathered neighbours.  A CTA
// of 32 x TY threads owns 31 x (TY - 1) node columns and a slab of node planes staged
// through a shared-memory ring (8-byte cp.async, zero-filled outside the grid); node sums
// combine one shuffle (x) and one shared-memory exchange (y), each formed by one thread:
// no atomics, bitwise reproducible.
struct TLam {
  double lam[8];  // lam_m / 8 of the Walsh modes (m = x | y << 1 | z << 2)
};

inline TLam make_tlam(const pyto_thermal_t* t) {
  TLam L;
  for (int m = 0; m < 8; ++m) {
    double v = 0.0;
    for (int d = 0; d < 8; ++d) v += ((__builtin_popcount(m & d) & 1) ? -1.0 : 1.0) * t->kxor[d];
    L.lam[m] = v / 8.0;
  }
  return L;
}

__device__ __forceinline__ void cp_async8(void* sdst, const void* gsrc, int valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gsrc), "r"(valid) : "memory");
}
__device__ __forceinline__ void th_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void th_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <int TY>
struct ThTile {
  static constexpr int TX = 32, NT = TX * TY, PX = TX + 1, PY = TY + 1, SLOT = PX * PY;
  static constexpr int LOOK = 3, RING = 8;  // planes ez+2 .. ez+1+LOOK in flight at layer ez
  static constexpr int LOADS = (SLOT + NT - 1) / NT;
  static_assert(LOOK + 3 <= RING, "ring holds planes ez-1 .. ez+1+LOOK");
};

template <int TY, bool DOT, bool MASKIN>
__global__ void __launch_bounds__(32 * TY) k_thermal_march(GridDims g, TLam L, const double* __restrict__ s,
                                                           const uint8_t* __restrict__ mask,
                                                           const double* __restrict__ u, double* __restrict__ y,
                                                           int zc, int mode, double* part, unsigned* counter,
                                                           double* dot_out) {
  using C = ThTile<TY>;
  constexpr int TX = C::TX, NT = C::NT, PX = C::PX, PY = C::PY, SLOT = C::SLOT, RING = C::RING, LOOK = C::LOOK;
  __shared__ double su[RING * SLOT];
  __shared__ uint8_t sm[RING * SLOT];
  __shared__ double sc[2][TY][TX];
  __shared__ double sred[NT / 32];
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  const int X0 = blockIdx.x * (TX - 1), Y0 = blockIdx.y * (TY - 1);
  const int Z0 = blockIdx.z * zc, Z1 = min(Z0 + zc, g.sz);
  const int ex = X0 - 1 + tx, ey = Y0 - 1 + ty;
  const bool in_col = ex >= 0 && ex < g.nx && ey >= 0 && ey < g.ny;
  const bool stage_mask = MASKIN && mask != nullptr;  // input masking reads the staged flags
  const bool mask_out = mask != nullptr && (mode & PYTO_MASK_OUT);
  const long long pn = (long long)g.sx * g.sy;
  const int pe = g.nx * g.ny;
  // this thread's staged nodes of a plane: tile position, global node of plane 0
  int ld_t[C::LOADS];
  long long ld_n[C::LOADS];
  bool ld_on[C::LOADS];
#pragma unroll
  for (int i = 0; i < C::LOADS; ++i) {
    const int t = tid + i * NT;
    const int ly = t / PX, lx = t - ly * PX;
    const int gx = X0 - 1 + lx, gy = Y0 - 1 + ly;
    ld_t[i] = t;
    ld_on[i] = t < SLOT && gx >= 0 && gx < g.sx && gy >= 0 && gy < g.sy;
    ld_n[i] = gx + (long long)g.sx * gy;
  }
  auto issue = [&](int k) {  // k >= -1
    const int slot = k & (RING - 1);
    const bool kin = k >= 0 && k < g.sz;
#pragma unroll
    for (int i = 0; i < C::LOADS; ++i) {
      if (C::LOADS * NT == SLOT || ld_t[i] < SLOT) {
        const bool on = kin && ld_on[i];
        const long long n = ld_n[i] + pn * (on ? k : 0);
        cp_async8(su + slot * SLOT + ld_t[i], u + (on ? n : 0), on ? 8 : 0);
        if (stage_mask) sm[slot * SLOT + ld_t[i]] = on ? mask[n] : 0;
      }
    }
    th_commit();
  };
  // Walsh transform of this thread's element face in plane k (x fastest)
  auto face = [&](int k, double (&F)[4]) {
    const double* b = su + (k & (RING - 1)) * SLOT + ty * PX + tx;
    double a00 = b[0], a10 = b[1], a01 = b[PX], a11 = b[PX + 1];
    if (stage_mask) {
      const uint8_t* q = sm + (k & (RING - 1)) * SLOT + ty * PX + tx;
      if (q[0] & 1) a00 = 0.0;
      if (q[1] & 1) a10 = 0.0;
      if (q[PX] & 1) a01 = 0.0;
      if (q[PX + 1] & 1) a11 = 0.0;
    }
    face_fwd(a00, a10, a01, a11, F);
  };
  const bool own = tx < TX - 1 && ty < TY - 1 && X0 + tx < g.sx && Y0 + ty < g.sy;
  const long long nown = (X0 + tx) + (long long)g.sx * (Y0 + ty);
  double cT = 0.0, dot = 0.0;
  auto output = [&](int k) {  // plane k's sums are complete (its layer-k exchange is in sc[k & 1])
    if (!own) return;
    const long long n = nown + pn * k;
    double v = cT + sc[k & 1][ty + 1][tx];
    const int slot = k & (RING - 1), t = (ty + 1) * PX + tx + 1;
    const int mk = mask_out ? mask[n] : (stage_mask ? sm[slot * SLOT + t] : 0);
    if (mask_out && (mk & 1)) v = 0.0;
    y[n] = v;
    if (DOT) {
      double uv = su[slot * SLOT + t];
      if (stage_mask && (sm[slot * SLOT + t] & 1)) uv = 0.0;
      dot = fma(uv, v, dot);
    }
  };
  long long eidx = ex + (long long)g.nx * ey + (long long)pe * (Z0 - 1);
  double s_next = (in_col && Z0 - 1 >= 0) ? __ldg(s + eidx) : 0.0;
#pragma unroll
  for (int k = 0; k < LOOK; ++k) {
    if (Z0 - 1 + k <= Z1) issue(Z0 - 1 + k);
    else th_commit();
  }
  double Fb[4], Ft[4], Gs[4] = {0.0, 0.0, 0.0, 0.0}, Gn[4];
  th_wait<LOOK - 1>();
  __syncthreads();
  face(Z0 - 1, Fb);
  for (int ez = Z0 - 1; ez < Z1; ++ez) {
    th_wait<LOOK - 2>();  // plane ez+1 has landed
    __syncthreads();
    if (ez - 1 >= Z0) output(ez - 1);
    if (ez + LOOK <= Z1) issue(ez + LOOK);
    else th_commit();
    face(ez + 1, Ft);
    const double sv = s_next;  // 0 for an element outside the grid or the slab
    eidx += pe;
    s_next = (in_col && ez + 1 < Z1 && ez + 1 < g.nz) ? __ldg(s + eidx) : 0.0;
    // modes: f = face mode, z-parity p; lam index f | p << 2 (lam_0, the constant mode,
    // vanishes for a conduction Ke but is kept for any Ke with the box symmetry)
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      const double oo = L.lam[f | 4] * (Ft[f] - Fb[f]);
      const double eo = L.lam[f] * (Ft[f] + Fb[f]);
      Gs[f] = fma(sv, eo - oo, Gs[f]);
      Gn[f] = sv * (eo + oo);
    }
    if (ez >= Z0) {
      double c00, c10, c01, c11;
      face_inv(Gs, c00, c10, c01, c11);
      cT = c11 + __shfl_down_sync(0xffffffffu, c01, 1);
      sc[ez & 1][ty][tx] = c10 + __shfl_down_sync(0xffffffffu, c00, 1);
    }
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      Fb[f] = Ft[f];
      Gs[f] = Gn[f];
    }
  }
  th_wait<0>();
  __syncthreads();
  if (Z1 - 1 >= Z0) output(Z1 - 1);
  if (DOT) {
    double v[1] = {block_sum<NT>(dot, sred)};
    grid_reduce<1>(v, part, counter, (int)(gridDim.x * gridDim.y * gridDim.z),
                   [&](const double* t) { *dot_out = t[0]; });
  }
}

// winv[n] = 1 / diag_n (diag_n = k[0] sum_{e ni n} s_e), flags: bit 0 fixed, bit 3 clamp
// (|diag| < 1e-12 -> preconditioner 1, src/linear_solvers.py:71-87)
__global__ void k_thermal_jacobi(GridDims g, double k0, const double* __restrict__ s,
                                 const uint8_t* __restrict__ mask, double* __restrict__ winv,
                                 uint8_t* __restrict__ flags) {
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < g.nnodes;
       n += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(n % g.sx);
    const long long r = n / g.sx;
    const int iy = (int)(r % g.sy);
    const int iz = (int)(r / g.sy);
    double acc = 0.0;
    for (int oz = 0; oz < 2; ++oz)
      for (int oy = 0; oy < 2; ++oy)
        for (int ox = 0; ox < 2; ++ox) {
          const int ex = ix - ox, ey = iy - oy, ez = iz - oz;
          if (ex >= 0 && ex < g.nx && ey >= 0 && ey < g.ny && ez >= 0 && ez < g.nz)
            acc += s[ex + (long long)g.nx * (ey + (long long)g.ny * ez)];
        }
    const double d = k0 * acc;
    int fl = mask ? (mask[n] & 1) : 0;
    if (fabs(d) < 1e-12) fl |= 8;
    winv[n] = fl & 8 ? 1.0 : 1.0 / d;
    flags[n] = (uint8_t)fl;
  }
}

__device__ __forceinline__ double tjacobi(double r, int fl, double w) { return (fl & 1) ? 0.0 : r * w; }

__global__ void __launch_bounds__(kNodeThreads) k_tpcg_init(long long n, const double* __restrict__ b,
                                                            const double* __restrict__ t,
                                                            const double* __restrict__ w,
                                                            const uint8_t* __restrict__ fl, double* __restrict__ x,
                                                            double* __restrict__ r, double* __restrict__ p,
                                                            KrylovState* S, double* part, unsigned* counter) {
  __shared__ double sred[kNodeThreads / 32];
  double rz = 0.0, rr = 0.0, bb = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int f = fl[i];
    const bool fixed = f & 1;
    const double bi = fixed ? 0.0 : b[i];
    const double ri = fixed ? 0.0 : bi - (t ? t[i] : 0.0);
    const double zi = tjacobi(ri, f, w[i]);
    r[i] = ri;
    p[i] = zi;
    if (!t) x[i] = 0.0;
    rz = fma(ri, zi, rz);
    rr = fma(ri, ri, rr);
    bb = fma(bi, bi, bb);
  }
  double v[3] = {block_sum<kNodeThreads>(rz, sred), block_sum<kNodeThreads>(rr, sred),
                 block_sum<kNodeThreads>(bb, sred)};
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

__global__ void __launch_bounds__(kNodeThreads) k_tpcg_update1(long long n, const double* __restrict__ w,
                                                               const uint8_t* __restrict__ fl,
                                                               double* __restrict__ x, double* __restrict__ r,
                                                               const double* __restrict__ p,
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
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    x[i] = fma(alpha, p[i], x[i]);
    const double ri = fma(-alpha, q[i], r[i]);
    r[i] = ri;
    const double zi = tjacobi(ri, fl[i], w[i]);
    rr = fma(ri, ri, rr);
    rzn = fma(ri, zi, rzn);
  }
  double v[2] = {block_sum<kNodeThreads>(rr, sred), block_sum<kNodeThreads>(rzn, sred)};
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

__global__ void __launch_bounds__(kNodeThreads) k_tpcg_update2(long long n, const double* __restrict__ w,
                                                               const uint8_t* __restrict__ fl,
                                                               const double* __restrict__ r, double* __restrict__ p,
                                                               const KrylovState* S) {
  if (S->done) return;
  const double beta = S->beta;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = fma(beta, p[i], tjacobi(r[i], fl[i], w[i]));
}

__global__ void __launch_bounds__(kNodeThreads) k_tpcg_true_res(long long n, const double* __restrict__ b,
                                                                const double* __restrict__ t,
                                                                const uint8_t* __restrict__ fl, KrylovState* S,
                                                                double* part, unsigned* counter) {
  __shared__ double sred[kNodeThreads / 32];
  double rr = 0.0, bb = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    if (fl[i] & 1) continue;
    const double d = b[i] - t[i];
    rr = fma(d, d, rr);
    bb = fma(b[i], b[i], bb);
  }
  double v[2] = {block_sum<kNodeThreads>(rr, sred), block_sum<kNodeThreads>(bb, sred)};
  grid_reduce<2>(v, part, counter, gridDim.x, [&](const double* tot) {
    S->true_rr = tot[0];
    S->bb = tot[1];
  });
}

// ce[e] = u_e^T Ke v_e; with s: total = sum s_e ce_e
__global__ void __launch_bounds__(256) k_thermal_energy(GridDims g, TK tk, const double* __restrict__ u,
                                                        const double* __restrict__ v, const double* __restrict__ s,
                                                        double* __restrict__ ce, double* part, unsigned* counter,
                                                        double* total) {
  __shared__ double sred[8];
  double acc = 0.0;
  const long long P = (long long)g.sx * g.sy;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < g.nelem;
       e += (long long)gridDim.x * blockDim.x) {
    const int ex = (int)(e % g.nx);
    const long long r = e / g.nx;
    const int ey = (int)(r % g.ny);
    const int ez = (int)(r / g.ny);
    const long long n0 = ex + (long long)g.sx * ey + P * ez;
    double ue[8], ve[8];
#pragma unroll
    for (int b = 0; b < 8; ++b) {  // bit order
      const long long m = n0 + (b & 1) + (long long)g.sx * ((b >> 1) & 1) + P * (b >> 2);
      ue[b] = u[m];
      ve[b] = v[m];
    }
    double c = 0.0;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      double t = 0.0;
#pragma unroll
      for (int b = 0; b < 8; ++b) t = fma(tk.k[a ^ b], ve[b], t);
      c = fma(ue[a], t, c);
    }
    ce[e] = c;
    if (s) acc = fma(s[e], c, acc);
  }
  if (total) {
    double vv[1] = {block_sum<256>(acc, sred)};
    grid_reduce<1>(vv, part, counter, gridDim.x, [&](const double* tot) { *total = tot[0]; });
  }
}

// mask[n] = 1 for the listed nodes (out-of-range ids ignored)
__global__ void k_thermal_mask(const int64_t* __restrict__ nodes, int64_t n, long long nnodes,
                               uint8_t* __restrict__ mask) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = nodes[i];
    if (v >= 0 && v < nnodes) mask[v] = 1;
  }
}

constexpr int kThermalBlocks = 8 * kNumSMs;

struct TPcgWs {
  KrylovState* S;
  unsigned* counter;
  double* part;
  double *r, *p, *q, *w;
  uint8_t* fl;
};

static TPcgWs carve_tpcg(const pyto_thermal_t* t, void* ws, size_t bytes, size_t* need) {
  const GridDims g = thermal_dims(t);
  Carver cv{(char*)ws, 0, bytes};
  TPcgWs W;
  W.S = cv.take<KrylovState>(1);
  W.counter = cv.take<unsigned>(64);
  W.part = cv.take<double>(3 * (size_t)std::max(kThermalBlocks, kNodeBlocks));
  W.r = cv.take<double>(g.nnodes);
  W.p = cv.take<double>(g.nnodes);
  W.q = cv.take<double>(g.nnodes);
  W.w = cv.take<double>(g.nnodes);
  W.fl = cv.take<uint8_t>(g.nnodes);
  *need = cv.off + 256;
  return W;
}

template <int TY, bool DOT, bool MI>
static int thermal_march_t(const GridDims& g, const TLam& L, const double* s, const uint8_t* mask, const double* u,
                           double* y, int mode, double* part, unsigned* counter, double* dot, cudaStream_t st) {
  const int bx = (g.sx + 30) / 31, by = (g.sy + TY - 2) / (TY - 1);
  // slab split: about two waves of CTAs, at most kThermalBlocks (the partial sums) and
  // at least 4 planes per slab
  const long long nxy = (long long)bx * by;
  long long nbz = std::max<long long>(1, std::min<long long>((2LL * 3 * kNumSMs + nxy - 1) / nxy,
                                                             kThermalBlocks / nxy));
  nbz = std::min<long long>(nbz, std::max(1, g.sz / 4));
  const int zc = (int)((g.sz + nbz - 1) / nbz);
  const dim3 grid(bx, by, (g.sz + zc - 1) / zc);
  if ((long long)grid.x * grid.y * grid.z > kThermalBlocks && DOT) return PYTO_ERR_TOO_LARGE;
  k_thermal_march<TY, DOT, MI><<<grid, 32 * TY, 0, st>>>(g, L, s, mask, u, y, zc, mode, part, counter, dot);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}

static int thermal_mv(const pyto_thermal_t* t, const double* s, const uint8_t* mask, const double* u, double* y,
                      int mode, double* part, unsigned* counter, double* dot, cudaStream_t st) {
  const GridDims g = thermal_dims(t);
  const TLam L = make_tlam(t);
  const bool mi = (mode & PYTO_MASK_IN) && mask != nullptr;
  // grids whose tiles alone exceed the partial-sum slots keep the node-owned kernel
  if ((long long)((g.sx + 30) / 31) * ((g.sy + 6) / 7) > kThermalBlocks) {
    const int nb = (int)std::min<long long>((g.nnodes + 255) / 256, kThermalBlocks);
    k_thermal_matvec<<<nb, 256, 0, st>>>(g, make_tk(t), s, mask, u, y, mode, part, counter, dot);
    PYTO_COUNT(1);
    PYTO_LAUNCH_CHECK();
    return PYTO_OK;
  }
  if (dot)
    return mi ? thermal_march_t<8, true, true>(g, L, s, mask, u, y, mode, part, counter, dot, st)
              : thermal_march_t<8, true, false>(g, L, s, mask, u, y, mode, part, counter, dot, st);
  return mi ? thermal_march_t<8, false, true>(g, L, s, mask, u, y, mode, part, counter, dot, st)
            : thermal_march_t<8, false, false>(g, L, s, mask, u, y, mode, part, counter, dot, st);
}

}  // namespace pyto

using namespace pyto;

extern "C" int pyto_ke_hex8_thermal(double k, double hx, double hy, double hz, double* ke_out) {
  if (!ke_out || !(hx > 0 && hy > 0 && hz > 0)) return PYTO_ERR_ARG;
  // 2x2x2 Gauss (exact for this integrand): Ke = sum_g k grad N^T grad N det J w
  const double gp[2] = {-0.5773502691896257, 0.5773502691896257};
  const int cx[8] = {-1, 1, 1, -1, -1, 1, 1, -1}, cy[8] = {-1, -1, 1, 1, -1, -1, 1, 1},
            cz[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
  const double det = hx * hy * hz / 8.0;
  for (int i = 0; i < 64; ++i) ke_out[i] = 0.0;
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int c = 0; c < 2; ++c) {
        const double xi = gp[a], eta = gp[b], zeta = gp[c];
        double gx[8], gy[8], gz[8];
        for (int n = 0; n < 8; ++n) {
          gx[n] = 0.125 * cx[n] * (1 + eta * cy[n]) * (1 + zeta * cz[n]) * 2.0 / hx;
          gy[n] = 0.125 * (1 + xi * cx[n]) * cy[n] * (1 + zeta * cz[n]) * 2.0 / hy;
          gz[n] = 0.125 * (1 + xi * cx[n]) * (1 + eta * cy[n]) * cz[n] * 2.0 / hz;
        }
        for (int i = 0; i < 8; ++i)
          for (int j = 0; j < 8; ++j) ke_out[8 * i + j] += k * (gx[i] * gx[j] + gy[i] * gy[j] + gz[i] * gz[j]) * det;
      }
  return PYTO_OK;
}

extern "C" int pyto_thermal_init(pyto_thermal_t* t, int32_t nelx, int32_t nely, int32_t nelz, double hx, double hy,
                                 double hz, double k, const double* ke) {
  if (!t || nelx < 1 || nely < 1 || nelz < 1) return PYTO_ERR_ARG;
  if ((long long)(nelx + 1) * (nely + 1) * (nelz + 1) >= (1ll << 31)) return PYTO_ERR_TOO_LARGE;
  t->nelx = nelx; t->nely = nely; t->nelz = nelz; t->pad = 0;
  t->hx = hx; t->hy = hy; t->hz = hz; t->k = k;
  if (ke) {
    for (int i = 0; i < 64; ++i) t->ke[i] = ke[i];
  } else {
    const int rc = pyto_ke_hex8_thermal(k, hx, hy, hz, t->ke);
    if (rc) return rc;
  }
  // Ke[a][b] = k[bits(a) ^ bits(b)]: check the box symmetry of the given matrix
  double scale = 0.0;
  for (int i = 0; i < 64; ++i) scale = std::max(scale, fabs(t->ke[i]));
  for (int d = 0; d < 8; ++d) t->kxor[d] = 0.0;
  for (int a = 0; a < 8; ++a) t->kxor[corner_bits(0) ^ corner_bits(a)] = t->ke[a];
  for (int a = 0; a < 8; ++a)
    for (int b = 0; b < 8; ++b)
      if (fabs(t->ke[8 * a + b] - t->kxor[corner_bits(a) ^ corner_bits(b)]) > 1e-12 * scale) return PYTO_ERR_ARG;
  return PYTO_OK;
}

extern "C" int pyto_thermal_mask(const pyto_thermal_t* t, const int64_t* fixed_nodes, int64_t n_fixed,
                                 uint8_t* mask, void* stream) {
  if (!t || !mask || n_fixed < 0 || (n_fixed > 0 && !fixed_nodes)) return PYTO_ERR_ARG;
  const GridDims g = thermal_dims(t);
  cudaStream_t st = (cudaStream_t)stream;
  PYTO_CUDA(cudaMemsetAsync(mask, 0, (size_t)g.nnodes, st));
  if (n_fixed > 0) {
    const int nb = (int)std::min<int64_t>((n_fixed + 255) / 256, 4 * kNumSMs);
    k_thermal_mask<<<nb, 256, 0, st>>>(fixed_nodes, n_fixed, g.nnodes, mask);
    PYTO_COUNT(1);
    PYTO_LAUNCH_CHECK();
  }
  return PYTO_OK;
}

extern "C" size_t pyto_thermal_workspace_bytes(const pyto_thermal_t* t) {
  if (!t) return 0;
  size_t need = 0;
  carve_tpcg(t, nullptr, 0, &need);
  return need;
}

extern "C" int pyto_thermal_matvec(const pyto_thermal_t* t, const double* s, const uint8_t* mask, const double* u,
                                   double* y, int mode, double* dot, void* ws, size_t ws_bytes, void* stream) {
  if (!t || !s || !u || !y || u == y) return PYTO_ERR_ARG;
  double* part = nullptr;
  unsigned* counter = nullptr;
  if (dot) {
    Carver cv{(char*)ws, 0, ws_bytes};
    counter = cv.take<unsigned>(64);
    part = cv.take<double>(kThermalBlocks);
    if (!cv.ok()) return PYTO_ERR_WORKSPACE;
    PYTO_CUDA(cudaMemsetAsync(counter, 0, 64 * sizeof(unsigned), (cudaStream_t)stream));
  }
  return thermal_mv(t, s, mask, u, y, mode, part, counter, dot, (cudaStream_t)stream);
}

extern "C" int pyto_thermal_energy(const pyto_thermal_t* t, const double* u, const double* v, const double* s,
                                   double* ce, double* total, void* ws, size_t ws_bytes, void* stream) {
  if (!t || !u || !ce || (total && !s)) return PYTO_ERR_ARG;
  const GridDims g = thermal_dims(t);
  double* part = nullptr;
  unsigned* counter = nullptr;
  cudaStream_t st = (cudaStream_t)stream;
  if (total) {
    Carver cv{(char*)ws, 0, ws_bytes};
    counter = cv.take<unsigned>(64);
    part = cv.take<double>(kThermalBlocks);
    if (!cv.ok()) return PYTO_ERR_WORKSPACE;
    PYTO_CUDA(cudaMemsetAsync(counter, 0, 64 * sizeof(unsigned), st));
  }
  const int nb = (int)std::min<long long>((g.nelem + 255) / 256, kThermalBlocks);
  k_thermal_energy<<<nb, 256, 0, st>>>(g, make_tk(t), u, v ? v : u, total ? s : nullptr, ce, part, counter, total);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}

extern "C" int pyto_thermal_pcg_solve(const pyto_thermal_t* t, const double* s, const uint8_t* mask,
                                      const double* b, double* u, const pyto_solve_cfg_t* cfg,
                                      pyto_solve_status_t* status, void* ws, size_t ws_bytes, void* stream) {
  if (!t || !s || !b || !u || !cfg || !status) return PYTO_ERR_ARG;
  if (!(cfg->rtol >= 0.0) || cfg->max_iters < 0 || cfg->stop_rule < 0 || cfg->stop_rule > 1) return PYTO_ERR_ARG;
  size_t need = 0;
  TPcgWs W = carve_tpcg(t, ws, ws_bytes, &need);
  if (!ws || ws_bytes < need) return PYTO_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  const GridDims g = thermal_dims(t);
  const long long n = g.nnodes;
  PYTO_CUDA(cudaMemsetAsync(W.counter, 0, 64 * sizeof(unsigned), st));
  {
    KrylovState z{};
    z.rtol = cfg->rtol;
    z.max_iters = cfg->max_iters;
    z.stop_rule = cfg->stop_rule;
    PYTO_CUDA(cudaMemcpyAsync(W.S, &z, sizeof(z), cudaMemcpyHostToDevice, st));
  }
  const int nbj = (int)std::min<long long>((n + 255) / 256, kThermalBlocks);
  k_thermal_jacobi<<<nbj, 256, 0, st>>>(g, t->kxor[0], s, mask, W.w, W.fl);
  PYTO_COUNT(1);
  int rc;
  const int mm = PYTO_MASK_IN | PYTO_MASK_OUT;
  if (cfg->x0_given) {
    rc = thermal_mv(t, s, mask, u, W.q, mm, nullptr, nullptr, nullptr, st);
    if (rc) return rc;
  }
  k_tpcg_init<<<kNodeBlocks, kNodeThreads, 0, st>>>(n, b, cfg->x0_given ? W.q : nullptr, W.w, W.fl, u, W.r, W.p, W.S,
                                                    W.part, W.counter);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  const int every = std::max(1, cfg->check_every);
  KrylovState hs{};
  PYTO_CUDA(cudaMemcpyAsync(&hs, W.S, sizeof(hs), cudaMemcpyDeviceToHost, st));
  PYTO_CUDA(cudaStreamSynchronize(st));
  while (!hs.done && hs.iters < cfg->max_iters) {
    for (int k = 0; k < every; ++k) {
      // p is zero on fixed nodes: the output mask suffices
      rc = thermal_mv(t, s, mask, W.p, W.q, PYTO_MASK_OUT, W.part, W.counter, &W.S->pq, st);
      if (rc) return rc;
      k_tpcg_update1<<<kNodeBlocks, kNodeThreads, 0, st>>>(n, W.w, W.fl, u, W.r, W.p, W.q, W.S, W.part, W.counter);
      PYTO_COUNT(1);
      k_tpcg_update2<<<kNodeBlocks, kNodeThreads, 0, st>>>(n, W.w, W.fl, W.r, W.p, W.S);
      PYTO_COUNT(1);
    }
    PYTO_LAUNCH_CHECK();
    PYTO_CUDA(cudaMemcpyAsync(&hs, W.S, sizeof(hs), cudaMemcpyDeviceToHost, st));
    PYTO_CUDA(cudaStreamSynchronize(st));
  }
  const KrylovState before = hs;
  rc = thermal_mv(t, s, mask, u, W.q, mm, nullptr, nullptr, nullptr, st);
  if (rc) return rc;
  k_tpcg_true_res<<<kNodeBlocks, kNodeThreads, 0, st>>>(n, b, W.q, W.fl, W.S, W.part, W.counter);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  PYTO_CUDA(cudaMemcpyAsync(&hs, W.S, sizeof(hs), cudaMemcpyDeviceToHost, st));
  PYTO_CUDA(cudaStreamSynchronize(st));
  status->converged = hs.converged;
  status->iters = hs.iters;
  status->breakdown = hs.breakdown;
  status->reserved = 0;
  status->rel_res = hs.stop_rule == 0 ? (before.bb > 0 ? sqrt(before.rr / before.bb) : 0.0)
                                      : (before.rz0 > 0 ? sqrt(before.rz / before.rz0) : 0.0);
  status->true_rel_res = hs.bb > 0 ? sqrt(hs.true_rr / hs.bb) : 0.0;
  if (hs.breakdown) return PYTO_ERR_BREAKDOWN;
  return hs.converged ? PYTO_OK : PYTO_NOT_CONVERGED;
}
