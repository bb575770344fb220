// Aggregation-deflated PCG (src/deflation.py:386-584) on the GPU.
//
// Deflation space W: per node group g, rigid-body modes about the group
// centre c_g (rel = x - c_g):
//   mode 0,1,2: translations;  mode 3: (0,-rel_z,rel_y);  mode 4: (rel_z,0,-rel_x);
//   mode 5: (-rel_y,rel_x,0)                         (src/deflation.py:415-450)
// W is never stored: restriction W^T v reduces per group over its nodes, and
// prolongation W mu is evaluated per node from its group's mu and centre.
//
// Coarse matrix E = W_f^T K_ff W_f (W rows of fixed DOFs dropped, as
// W[free_dofs] in src/linear_solvers.py:184).  Rigid modes lie in the null
// space of every element matrix, so only elements whose corners span two or
// more groups (or touch a fixed DOF) contribute; each such element adds
// s_e (Phi M_g)^T K^ (Phi M_h) to block (g, h).  Row blocks are accumulated
// per group in shared memory and written once (no global atomics).
//
// E^-1 is formed explicitly (dense, FP64) by a blocked in-place sweep
// (Gauss-Jordan on the SPD matrix, 64x64 pivot blocks); each DPCG iteration
// then applies it with one dense GEMV, which is a single fully parallel pass
// instead of two latency-bound triangular solves.
#include <algorithm>
#include <vector>

#include "coarse_nd.cuh"
#include "krylov.cuh"
#include "sweep.cuh"

namespace pyto {

// boundary-list chunks: kRkChunk list entries per CTA of the K-restriction and
// of the coarse assembly
constexpr int kRkThreads = 128;
constexpr int kRkChunk = 2 * kRkThreads;
constexpr int kRkMaxChunks = 65536;

// node ids fit in int32 (checked by pyto_operator_init), so 32-bit division suffices
__device__ __forceinline__ void node_xyz(const GridDims& g, long long n, double hx, double hy, double hz, double& x,
                                         double& y, double& z) {
  const int ni = (int)n;
  const int r = ni / g.sx;
  const int ix = ni - r * g.sx;
  const int iz = r / g.sy;
  const int iy = r - iz * g.sy;
  x = hx * ix;
  y = hy * iy;
  z = hz * iz;
}

// mode vector (3 components) of mode a at relative position rel
__device__ __forceinline__ void rigid_mode(int a, double rx, double ry, double rz, double (&w)[3]) {
  w[0] = w[1] = w[2] = 0.0;
  switch (a) {
    case 0: w[0] = 1.0; break;
    case 1: w[1] = 1.0; break;
    case 2: w[2] = 1.0; break;
    case 3: w[1] = -rz; w[2] = ry; break;
    case 4: w[0] = rz; w[2] = -rx; break;
    default: w[0] = -ry; w[1] = rx; break;
  }
}

struct DeflP {
  double hx, hy, hz;
  int modes, ngroups;
  long long nc;
};

// Hadamard transform of the restriction of mode a of group G to the element's
// corners (zero at corners of other groups and at fixed DOFs); xyz: corner
// coordinates in bit order
__device__ __forceinline__ void mode_hat(const double (&xyz)[8][3], const int (&gr)[8], const int (&mk)[8], int G,
                                         const double* __restrict__ gc, int a, double (&H)[3][8]) {
  const double c0 = gc[3 * (long long)G], c1 = gc[3 * (long long)G + 1], c2 = gc[3 * (long long)G + 2];
  double A[3][8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    double w[3] = {0.0, 0.0, 0.0};
    if (gr[k] == G) rigid_mode(a, xyz[k][0] - c0, xyz[k][1] - c1, xyz[k][2] - c2, w);
#pragma unroll
    for (int c = 0; c < 3; ++c) A[c][k] = ((mk[k] >> c) & 1) ? 0.0 : w[c];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    double Fb[4], Ft[4];
    face_fwd(A[c][0], A[c][1], A[c][2], A[c][3], Fb);
    face_fwd(A[c][4], A[c][5], A[c][6], A[c][7], Ft);
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      H[c][f] = Ft[f] + Fb[f];
      H[c][f + 4] = Ft[f] - Fb[f];
    }
  }
}

// ---------------------------------------------------------------------------
// coarse matrix assembly
// ---------------------------------------------------------------------------
// Row block E[g, :] of one group per CTA (no global atomics): the CTA visits
// the elements touching group g; for each element with corners outside g (or
// on fixed DOFs) it adds s_e (Phi M_g)^T K^ (Phi M_h) for every corner group h
// into a shared-memory accumulator (one 6x6 slot per neighbour group), then
// writes its row blocks.  Every block of E is written by exactly one CTA.
constexpr int kAsmThreads = 256;
__global__ void __launch_bounds__(kAsmThreads) k_coarse_rows(GridDims g, KHat kh, DeflP dp,
                                                            const double* __restrict__ s,
                                                            const uint8_t* __restrict__ mask,
                                                            const int32_t* __restrict__ ngrp,
                                                            const double* __restrict__ gc,
                                                            const int32_t* __restrict__ gbox,
                                                            const int32_t* __restrict__ nptr,
                                                            const int32_t* __restrict__ nlist,
                                                            double* __restrict__ E) {
  extern __shared__ double acc[];  // [nnbr][36]
  __shared__ int snb[128];
  const int G = blockIdx.x;
  const int nb0 = nptr[G], nnb = nptr[G + 1] - nb0;
  for (int t = threadIdx.x; t < nnb; t += blockDim.x) snb[t] = nlist[nb0 + t];
  for (int t = threadIdx.x; t < nnb * 36; t += blockDim.x) acc[t] = 0.0;
  __syncthreads();
  const int* bx = gbox + 6 * G;
  const int ex0 = bx[0], ey0 = bx[2], ez0 = bx[4];
  const int lx = bx[1] - ex0 + 1, ly = bx[3] - ey0 + 1, lz = bx[5] - ez0 + 1;
  const long long nvis = (long long)lx * ly * lz;
  for (long long t = threadIdx.x; t < nvis; t += blockDim.x) {
    const int ex = ex0 + (int)(t % lx);
    const int ey = ey0 + (int)((t / lx) % ly);
    const int ez = ez0 + (int)(t / ((long long)lx * ly));
    const long long e = ex + (long long)g.nx * (ey + (long long)g.ny * ez);
    const double se = s[e];
    if (se == 0.0) continue;
    int gr[8], mk[8];
    double xyz[8][3];
    bool mine = false, other = false;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int bxk = k & 1, byk = (k >> 1) & 1, bzk = k >> 2;
      const long long nd = (ex + bxk) + (long long)g.sx * ((ey + byk) + (long long)g.sy * (ez + bzk));
      gr[k] = ngrp[nd];
      mk[k] = mask ? (mask[nd] & 7) : 0;
      xyz[k][0] = dp.hx * (ex + bxk);
      xyz[k][1] = dp.hy * (ey + byk);
      xyz[k][2] = dp.hz * (ez + bzk);
      mine |= (gr[k] == G);
      other |= (gr[k] != G) || (mk[k] != 0);
    }
    if (!mine || !other) continue;
    double Hg[6][3][8];
    for (int a = 0; a < dp.modes; ++a) mode_hat(xyz, gr, mk, G, gc, a, Hg[a]);
    int H[8], nh = 0;
    for (int k = 0; k < 8; ++k) {
      bool seen = false;
      for (int t2 = 0; t2 < nh; ++t2) seen |= (H[t2] == gr[k]);
      if (!seen) H[nh++] = gr[k];
    }
    for (int hi = 0; hi < nh; ++hi) {
      const int h = H[hi];
      int slot = 0;
      while (slot < nnb && snb[slot] != h) ++slot;
      if (slot == nnb) continue;  // not possible for a consistent neighbour list
      for (int b = 0; b < dp.modes; ++b) {
        double Hh[3][8], Z[3][8];
        mode_hat(xyz, gr, mk, h, gc, b, Hh);
        for (int q = 0; q < 8; ++q)
          for (int c = 0; c < 3; ++c) {
            const int m = member_mode(q, c);
            if (m == 0) continue;
            double o = 0.0;
            for (int d = 0; d < 3; ++d) {
              const int n = member_mode(q, d);
              if (n == 0) continue;
              o = fma(kh.b[q][3 * c + d], Hh[d][n], o);
            }
            Z[c][m] = se * o;
          }
        for (int a = 0; a < dp.modes; ++a) {
          double v = 0.0;
          for (int c = 0; c < 3; ++c)
            for (int m = 1; m < 8; ++m) v = fma(Hg[a][c][m], Z[c][m], v);
          if (v != 0.0) atomicAdd(&acc[slot * 36 + a * 6 + b], v);
        }
      }
    }
  }
  __syncthreads();
  const int M = dp.modes;
  for (int t = threadIdx.x; t < nnb * M * M; t += blockDim.x) {
    const int slot = t / (M * M), a = (t / M) % M, b = t % M;
    E[((long long)G * M + a) * dp.nc + (long long)snb[slot] * M + b] = acc[slot * 36 + a * 6 + b];
  }
}

// Hadamard transform (8 corner modes, the ordering of hex8_core) of component c
// of rigid mode a of group Gs restricted to the element's corners in Gs with
// free DOF c; rel0: corner 0 relative to the group centre, h: element size.
__device__ __forceinline__ void mode_comp_hat(const int (&gr)[8], const int (&mk)[8], int Gs, int c, int a,
                                              const double (&rel0)[3], const double (&h)[3], double (&H)[8]) {
  double v[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    double w = 0.0;
    if (gr[k] == Gs && !((mk[k] >> c) & 1)) {
      const double rx = rel0[0] + ((k & 1) ? h[0] : 0.0), ry = rel0[1] + (((k >> 1) & 1) ? h[1] : 0.0),
                   rz = rel0[2] + ((k >> 2) ? h[2] : 0.0);
      // component c of mode a: [tx,ty,tz, rx:(0,-z,y), ry:(z,0,-x), rz:(-y,x,0)]
      if (a < 3) w = (a == c) ? 1.0 : 0.0;
      else if (a == 3) w = (c == 1) ? -rz : (c == 2) ? ry : 0.0;
      else if (a == 4) w = (c == 0) ? rz : (c == 2) ? -rx : 0.0;
      else w = (c == 0) ? -ry : (c == 1) ? rx : 0.0;
    }
    v[k] = w;
  }
  double Fb[4], Ft[4];
  face_fwd(v[0], v[1], v[2], v[3], Fb);
  face_fwd(v[4], v[5], v[6], v[7], Ft);
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    H[f] = Ft[f] + Fb[f];
    H[f + 4] = Ft[f] - Fb[f];
  }
}

// 8-point Hadamard transform of corner values (the basis of mode_comp_hat)
__device__ __forceinline__ void had8(const double (&v)[8], double (&H)[8]) {
  double Fb[4], Ft[4];
  face_fwd(v[0], v[1], v[2], v[3], Fb);
  face_fwd(v[4], v[5], v[6], v[7], Ft);
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    H[f] = Ft[f] + Fb[f];
    H[f + 4] = Ft[f] - Fb[f];
  }
}

// For an element without fixed DOFs the masked rigid modes of group Gs are linear
// combinations of four corner vectors: the indicator of the corners in Gs (ind) and
// ind times the local corner coordinates lx, ly, lz (corner offsets times h).  Their
// Hadamard transforms go to B[(i*8 + m) * stride] (shared memory, i = ind, lx, ly, lz).
__device__ __forceinline__ void group_base_hat(const int (&gr)[8], int Gs, const double (&h)[3], double* B,
                                               int stride) {
  double v[8], H[8];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const double ind = (gr[k] == Gs) ? 1.0 : 0.0;
      const double l = (i == 0) ? 1.0 : (i == 1) ? ((k & 1) ? h[0] : 0.0) : (i == 2) ? (((k >> 1) & 1) ? h[1] : 0.0)
                                                                           : ((k >> 2) ? h[2] : 0.0);
      v[k] = ind * l;
    }
    had8(v, H);
#pragma unroll
    for (int m = 0; m < 8; ++m) B[(i * 8 + m) * stride] = H[m];
  }
}

// Component c, Hadamard mode m of masked rigid mode b (position d + local) from the
// base vectors B (no fixed DOFs): [tx,ty,tz, rx:(0,-z,y), ry:(z,0,-x), rz:(-y,x,0)]
__device__ __forceinline__ double mode_hat_from_base(const double* B, int stride, int b, int c, int m,
                                                     const double (&d)[3]) {
  const double b0 = B[m * stride];
  auto pos = [&](int ax) { return d[ax] * b0 + B[((ax + 1) * 8 + m) * stride]; };  // (d + l)_ax ind
  if (b < 3) return (b == c) ? b0 : 0.0;
  if (b == 3) return (c == 1) ? -pos(2) : (c == 2) ? pos(1) : 0.0;
  if (b == 4) return (c == 0) ? pos(2) : (c == 2) ? -pos(0) : 0.0;
  return (c == 0) ? -pos(1) : (c == 1) ? pos(0) : 0.0;
}

// Row blocks E[G, :] from the boundary element lists: one CTA per list chunk
// (chunk tables as for k_restrict_K), one entry per thread per pass.  For entry
// (G, e) and every group H at a corner of e, s_e (Phi W_G|e)^T K^ (Phi W_H|e) is
// added into a shared-memory accumulator of G's neighbour slots, which is then
// added into E with global atomics.  The sums are formed in 64-bit fixed point with
// a power-of-two scale per row group (2^gexp[G], chosen by k_group_scale so that the
// sum of the magnitudes of all of G's contributions stays below 2^61): integer
// addition is associative, so E does not depend on the order of the atomics and
// the coarse operator, its inverse and the solve are bitwise reproducible.  Each
// contribution is rounded once, to 2^-gexp[G], at most 2^-61 of that magnitude
// bound.  E is accumulated as int64 bits in place; k_coarse_from_fixed converts it.
// Only the blocks E[G, H] with H <= G are formed (E is symmetric; k_sym_pass
// copies them into E[H, G]), and the mode loops are unrolled (M = dp.modes).
constexpr int kCrThreads = 128;
// BSR: E is block-sparse in the neighbour-slot order (block (G, nbr_list[nbr_ptr[G] + j])
// at slot nbr_ptr[G] + j, M x M row-major): the nested-dissection coarse solver.
template <int M, bool BSR = false>
__global__ void __launch_bounds__(kCrThreads, 3) k_coarse_rows2(GridDims g, KHat kh, DeflP dp,
                                                             const double* __restrict__ s,
                                                             const uint8_t* __restrict__ mask,
                                                             const int32_t* __restrict__ ngrp,
                                                             const double* __restrict__ gc,
                                                             const int32_t* __restrict__ bptr,
                                                             const int32_t* __restrict__ blist,
                                                             const int32_t* __restrict__ cptr,
                                                             const int32_t* __restrict__ cgrp,
                                                             const int32_t* __restrict__ nptr,
                                                             const int32_t* __restrict__ nlist,
                                                             const int* __restrict__ gexp,
                                                             unsigned long long* __restrict__ E) {
  extern __shared__ double cr_smem[];
  double* sbase = cr_smem;                  // [2][32][kCrThreads] group base vectors
  unsigned long long* acc = reinterpret_cast<unsigned long long*>(cr_smem + 64 * kCrThreads);  // [nnb][36]
  __shared__ int snb[128];
  const int ch = blockIdx.x;
  if (ch >= cptr[dp.ngroups]) return;
  const int G = cgrp[ch];
  const double scale = ldexp(1.0, gexp[G]);
  const int nb0 = nptr[G], nnb = nptr[G + 1] - nb0;
  for (int t = threadIdx.x; t < nnb; t += blockDim.x) snb[t] = nlist[nb0 + t];
  for (int t = threadIdx.x; t < nnb * 36; t += blockDim.x) acc[t] = 0ull;
  __syncthreads();
  const double h[3] = {dp.hx, dp.hy, dp.hz};
  const int end = bptr[G + 1];
  const int pn = g.sx * g.sy;
  for (int r = 0; r < kRkChunk / kCrThreads; ++r) {
    const int t = bptr[G] + (ch - cptr[G]) * kRkChunk + r * kCrThreads + threadIdx.x;
    if (t >= end) continue;
    const int e = blist[t];
    const double se = s[e];
    if (se == 0.0) continue;
    const int rr = e / g.nx;
    const int ex = e - rr * g.nx;
    const int ez = rr / g.ny;
    const int ey = rr - ez * g.ny;
    const int n0 = ex + g.sx * (ey + g.sy * ez);
    int gr[8], mk[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int nd = n0 + (k & 1) + g.sx * ((k >> 1) & 1) + pn * (k >> 2);
      gr[k] = ngrp[nd];
      mk[k] = mask ? (mask[nd] & 7) : 0;
    }
    // distinct corner groups and their slots in G's neighbour list
    int Hs[8], Sl[8], nh = 0;
    for (int k = 0; k < 8; ++k) {
      bool seen = false;
      for (int q = 0; q < nh; ++q) seen |= (Hs[q] == gr[k]);
      if (seen) continue;
      if (gr[k] > G) continue;  // E[G, H] for H > G comes from the mirror
      int slot = 0;
      while (slot < nnb && snb[slot] != gr[k]) ++slot;
      if (slot == nnb) continue;  // not possible for a consistent neighbour list
      Hs[nh] = gr[k];
      Sl[nh] = slot;
      ++nh;
    }
    const double relG[3] = {dp.hx * ex - gc[3 * G], dp.hy * ey - gc[3 * G + 1], dp.hz * ez - gc[3 * G + 2]};
    bool anyfix = false;
#pragma unroll
    for (int k = 0; k < 8; ++k) anyfix |= mk[k] != 0;
    if (!anyfix) {
      // B_GH[a][b] = s (Phi W_G,a)^T K^ (Phi W_H,b): for each (H, b) apply K^ once to
      // mode b of H, then form all modes a of G from 12 dot products with G's base
      double* BG = sbase + threadIdx.x;
      double* BH = sbase + 32 * kCrThreads + threadIdx.x;
      group_base_hat(gr, G, h, BG, kCrThreads);
      for (int hi = 0; hi < nh; ++hi) {
        const int H = Hs[hi];
        const double relH[3] = {dp.hx * ex - gc[3 * H], dp.hy * ey - gc[3 * H + 1], dp.hz * ez - gc[3 * H + 2]};
        group_base_hat(gr, H, h, BH, kCrThreads);
#pragma unroll
        for (int b = 0; b < M; ++b) {
          double Hh[3][8];
#pragma unroll
          for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int m = 0; m < 8; ++m) Hh[c][m] = mode_hat_from_base(BH, kCrThreads, b, c, m, relH);
          double Y[3][8];  // K^ Hh (rows m = 0 vanish)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            Y[c][0] = 0.0;
#pragma unroll
            for (int m = 1; m < 8; ++m) {
              const int q = m ^ (1 << c);
              double o = 0.0;
#pragma unroll
              for (int dd = 0; dd < 3; ++dd) {
                const int md = member_mode(q, dd);
                if (md == 0) continue;
                o = fma(kh.b[q][3 * c + dd], Hh[dd][md], o);
              }
              Y[c][m] = o;
            }
          }
          double D[4][3];  // base vector i of G . Y[c]
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              double t = 0.0;
#pragma unroll
              for (int m = 1; m < 8; ++m) t = fma(BG[(i * 8 + m) * kCrThreads], Y[c][m], t);
              D[i][c] = t;
            }
          double vab[6];
          vab[0] = D[0][0];
          vab[1] = D[0][1];
          vab[2] = D[0][2];
          if (M == 6) {
            vab[3] = -(relG[2] * D[0][1] + D[3][1]) + (relG[1] * D[0][2] + D[2][2]);
            vab[4] = (relG[2] * D[0][0] + D[3][0]) - (relG[0] * D[0][2] + D[1][2]);
            vab[5] = -(relG[1] * D[0][0] + D[2][0]) + (relG[0] * D[0][1] + D[1][1]);
          }
#pragma unroll
          for (int a = 0; a < M; ++a) {
            const long long qv = __double2ll_rn(se * vab[a] * scale);
            if (qv != 0) atomicAdd(&acc[Sl[hi] * 36 + a * 6 + b], (unsigned long long)qv);
          }
        }
      }
      continue;
    }
#pragma unroll
    for (int a = 0; a < M; ++a) {
      double Hg[3][8];
#pragma unroll
      for (int c = 0; c < 3; ++c) mode_comp_hat(gr, mk, G, c, a, relG, h, Hg[c]);
      // Z = s_e K^ Hg (rows m = 0 vanish)
      double Z[3][8];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        Z[c][0] = 0.0;
#pragma unroll
        for (int m = 1; m < 8; ++m) {
          const int q = m ^ (1 << c);
          double o = 0.0;
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            const int md = member_mode(q, d);
            if (md == 0) continue;
            o = fma(kh.b[q][3 * c + d], Hg[d][md], o);
          }
          Z[c][m] = se * o;
        }
      }
      for (int hi = 0; hi < nh; ++hi) {
        const int H = Hs[hi];
        const double relH[3] = {dp.hx * ex - gc[3 * H], dp.hy * ey - gc[3 * H + 1], dp.hz * ez - gc[3 * H + 2]};
#pragma unroll
        for (int b = 0; b < M; ++b) {
          double v = 0.0;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            double Hh[8];
            mode_comp_hat(gr, mk, H, c, b, relH, h, Hh);
#pragma unroll
            for (int m = 1; m < 8; ++m) v = fma(Z[c][m], Hh[m], v);
          }
          const long long qv = __double2ll_rn(v * scale);
          if (qv != 0) atomicAdd(&acc[Sl[hi] * 36 + a * 6 + b], (unsigned long long)qv);
        }
      }
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nnb * M * M; t += blockDim.x) {
    const int slot = t / (M * M), a = (t / M) % M, b = t % M;
    const unsigned long long v = acc[slot * 36 + a * 6 + b];
    if (v != 0ull) {
      if (BSR) atomicAdd(&E[((long long)(nb0 + slot) * M + a) * M + b], v);
      else atomicAdd(&E[((long long)G * M + a) * dp.nc + (long long)snb[slot] * M + b], v);
    }
  }
}

// Fixed-point scale of each row group G: gexp[G] = 61 - e with 2^e above
//   B_G = |Ke|_rows * 8 * max(1, R_G) * max(1, R'_G) * sum_{e in G's list} |s_e|,
// a bound of the sum of the magnitudes of G's contributions: a contribution of
// element e is |s_e w_G^T Ke w_H| <= |s_e| |Ke|_2 |w_G| |w_H| over the element's 8
// corners, |w| <= sqrt(8) max(1, |rel|) for any rigid mode, R_G the largest distance
// from G's centre to a corner of G's element box, R'_G the same from the centres of
// G's neighbour groups.  One block per group, deterministic reduction.
__global__ void __launch_bounds__(256) k_group_scale(DeflP dp, double ke_rows, const double* __restrict__ s,
                                                      const double* __restrict__ gc,
                                                      const int32_t* __restrict__ gbox,
                                                      const int32_t* __restrict__ bptr,
                                                      const int32_t* __restrict__ blist,
                                                      const int32_t* __restrict__ nptr,
                                                      const int32_t* __restrict__ nlist, int* __restrict__ gexp) {
  __shared__ double sred[8];
  const int G = blockIdx.x;
  double acc = 0.0;
  for (int t = bptr[G] + threadIdx.x; t < bptr[G + 1]; t += blockDim.x) acc += fabs(s[blist[t]]);
  const double ssum = block_sum<256>(acc, sred);
  if (threadIdx.x != 0) return;
  const int* bx = gbox + 6 * G;
  const double lo[3] = {dp.hx * bx[0], dp.hy * bx[2], dp.hz * bx[4]};
  const double hi[3] = {dp.hx * (bx[1] + 1), dp.hy * (bx[3] + 1), dp.hz * (bx[5] + 1)};
  auto reach = [&](const double* c) {  // largest distance from c to a corner of the box
    double r2 = 0.0;
    for (int d = 0; d < 3; ++d) {
      const double a = fmax(fabs(lo[d] - c[d]), fabs(hi[d] - c[d]));
      r2 += a * a;
    }
    return sqrt(r2);
  };
  const double RG = reach(gc + 3 * (long long)G);
  double RH = RG;
  for (int k = nptr[G]; k < nptr[G + 1]; ++k) RH = fmax(RH, reach(gc + 3 * (long long)nlist[k]));
  const double B = ke_rows * 8.0 * fmax(1.0, RG) * fmax(1.0, RH) * ssum;
  int e = 0;
  if (B > 0.0 && isfinite(B)) frexp(B, &e);  // B < 2^e
  gexp[G] = (B > 0.0 && isfinite(B)) ? 61 - e : 0;
}

// E (int64 fixed-point bits of the blocks with H <= G) -> FP64 values
__global__ void k_coarse_from_fixed(long long n, int modes, const int* __restrict__ gexp, double* E) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n * n;
       t += (long long)gridDim.x * blockDim.x) {
    const long long i = t / n;
    const long long q = reinterpret_cast<const long long*>(E)[t];
    E[t] = ldexp((double)q, -gexp[i / modes]);
  }
}


// mean |diag(E)| (one block) -> *out
__global__ void k_diag_mean(long long nc, const double* __restrict__ E, double* out) {
  __shared__ double sred[8];
  double acc = 0.0;
  for (long long i = threadIdx.x; i < nc; i += blockDim.x) acc += fabs(E[i * nc + i]);
  const double t = block_sum<256>(acc, sred);
  if (threadIdx.x == 0) *out = t / (double)nc;
}


// The symmetric passes over the dense coarse matrix, by 32 x 32 tile pairs (I >= J; one
// CTA of 32 x 8 threads stages tile (I, J) and tile (J, I) with loads along rows and
// writes both back the same way), entry (i, j) with a = E[i][j], b = E[j][i]:
//   kSymMirror: the row-group-lower blocks into the upper ones (E is assembled for
//               group(row) >= group(col) only): both = the value of the lower group side;
//               entries of one group block are left as they are;
//   kSymFinish: (E + E^T) / 2, a zero diagonal entry -> 1, plus the diagonal shift;
//   kSymNegate: -A from the lower 64 x 64 tiles (the sweep's result) into both halves.
constexpr int kSymMirror = 0, kSymFinish = 1, kSymNegate = 2;
__global__ void __launch_bounds__(256) k_sym_pass(long long n, int modes, double* E, int op, double shift,
                                                  const double* mean_diag) {
  __shared__ double ta[32][33], tb[32][33];
  const long long t = blockIdx.x;
  long long I = (long long)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while (I * (I + 1) / 2 > t) --I;
  while ((I + 1) * (I + 2) / 2 <= t) ++I;
  const long long J = t - I * (I + 1) / 2;
  const long long i0 = 32 * I, j0 = 32 * J;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
#pragma unroll
  for (int r = ty; r < 32; r += 8) {
    const long long ia = i0 + r, ja = j0 + tx, ib = j0 + r, jb = i0 + tx;
    ta[r][tx] = (ia < n && ja < n) ? E[ia * n + ja] : 0.0;  // rows of tile (I, J)
    tb[r][tx] = (ib < n && jb < n) ? E[ib * n + jb] : 0.0;  // rows of tile (J, I)
  }
  __syncthreads();
  const double sh = (op == kSymFinish) ? (mean_diag ? shift * (*mean_diag) : shift) : 0.0;
  // thread (ty, tx) writes row r of tile (I, J): entry (i0 + r, j0 + tx), and row r of
  // tile (J, I): entry (j0 + r, i0 + tx)
#pragma unroll
  for (int r = ty; r < 32; r += 8) {
    const long long i = i0 + r, j = j0 + tx;
    if (i < n && j < n) {
      const double a = ta[r][tx], b = tb[tx][r];  // E[i][j], E[j][i]
      double v;
      if (op == kSymMirror) {
        const long long gi = i / modes, gj = j / modes;
        v = gi > gj ? a : gi < gj ? b : a;
      } else if (op == kSymFinish) {
        v = (i == j) ? ((a == 0.0 ? 1.0 : a) + sh) : 0.5 * (a + b);
      } else {
        v = ((i >> 6) >= (j >> 6)) ? -a : -b;
      }
      E[i * n + j] = v;
    }
    const long long i2 = j0 + r, j2 = i0 + tx;  // the transposed entry (i2, j2)
    if (I != J && i2 < n && j2 < n) {
      const double a = tb[r][tx], b = ta[tx][r];  // E[i2][j2], E[j2][i2]
      double v;
      if (op == kSymMirror) {
        const long long gi = i2 / modes, gj = j2 / modes;
        v = gi > gj ? a : gi < gj ? b : a;
      } else if (op == kSymFinish) {
        v = 0.5 * (b + a);
      } else {
        v = ((i2 >> 6) >= (j2 >> 6)) ? -a : -b;
      }
      E[i2 * n + j2] = v;
    }
  }
}

static int sym_pass(long long n, int modes, double* E, int op, double shift, const double* mean_diag,
                    cudaStream_t st) {
  const long long nt = (n + 31) / 32;
  k_sym_pass<<<(int)(nt * (nt + 1) / 2), 256, 0, st>>>(n, modes, E, op, shift, mean_diag);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}

// ---------------------------------------------------------------------------
// blocked sweep inversion: after all pivot blocks A = -E^-1
//   P = A_KK^-1, U = P A_K:, A_ij -= A_iK U_Kj, A_Kj = U_Kj, A_iK = U_Ki^T, A_KK = -P
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_sweep_pivot(long long n, int k0, int bk, const double* __restrict__ A,
                                                     double* __restrict__ P) {
  sweep_pivot_block(n, k0, bk, A, P);
}

// Rp = A_K: (copy), U = P Rp   (16 columns per block).  Only the lower tiles
// (and the full diagonal tiles) of A are current, so row K right of the pivot
// block is read from column K below it.
__global__ void __launch_bounds__(256) k_sweep_panel(long long n, int k0, int bk, const double* __restrict__ A,
                                                     const double* __restrict__ P, double* __restrict__ Rp,
                                                     double* __restrict__ U) {
  sweep_panel_cols(n, k0, bk, A, P, Rp, U, (long long)blockIdx.x * 16);
}

// tile update of the lower 64x64 tiles (ti >= tj, one CTA each, 1-D grid),
// 256 threads x (4x4) outputs, k in chunks of 32.  k1 >= 0: the CTA of the next
// pivot tile (k1, k1) -- block 0, so it starts first -- goes on to sweep it in
// registers and writes Pn = A_k1k1^-1 for the next step, behind the other tiles.
__global__ void __launch_bounds__(256, 2) k_sweep_update(long long n, int k0, int bk, double* __restrict__ A,
                                                      const double* __restrict__ P, const double* __restrict__ Rp,
                                                      const double* __restrict__ U, int k1, double* __restrict__ Pn) {
  const long long ntiles = gridDim.x;
  long long b = blockIdx.x;
  if (k1 >= 0) {  // rotate the numbering so that block 0 is tile (k1/64, k1/64)
    const long long t1 = k1 / 64;
    b = (b + t1 * (t1 + 1) / 2 + t1) % ntiles;
  }
  long long ti = (long long)((sqrt(8.0 * (double)b + 1.0) - 1.0) * 0.5);
  while (ti * (ti + 1) / 2 > b) --ti;
  while ((ti + 1) * (ti + 2) / 2 <= b) ++ti;
  const long long tj = b - ti * (ti + 1) / 2;
  sweep_update_tile(n, k0, bk, A, P, Rp, U, ti, tj, k1, Pn, k1 >= 0 ? (int)std::min<long long>(kSweepB, n - k1) : 0);
}


// ---------------------------------------------------------------------------
// DPCG pieces
// ---------------------------------------------------------------------------
// v = W_f^T y.  Block (group, chunk) reduces up to kRestrictChunk nodes of one
// group (CSR order) to 6 partials; the last block to finish sums each group's
// chunk partials in chunk order, so the result does not depend on scheduling.
constexpr int kRestrictChunk = 2048;
constexpr int kRestrictMaxBlocks = 65536;
template <typename T>
__global__ void __launch_bounds__(256) k_restrict(GridDims g, DeflP dp, const int32_t* __restrict__ gptr,
                                                  const int32_t* __restrict__ gnodes, const double* __restrict__ gc,
                                                  const uint8_t* __restrict__ fl, const T* __restrict__ y,
                                                  int nch, double* __restrict__ part) {
  __shared__ double sred[8 * 6];
  const int grp = blockIdx.x / nch, ch = blockIdx.x % nch;
  const int beg = gptr[grp] + ch * kRestrictChunk;
  const int end = min(gptr[grp + 1], beg + kRestrictChunk);
  const double cx = gc[3 * grp], cy = gc[3 * grp + 1], cz = gc[3 * grp + 2];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int t = beg + threadIdx.x; t < end; t += blockDim.x) {
    const int n = gnodes[t];
    double x, yy, z;
    node_xyz(g, n, dp.hx, dp.hy, dp.hz, x, yy, z);
    const double rx = x - cx, ry = yy - cy, rz = z - cz;
    const int f = fl[n];
    const double vx = (f & 1) ? 0.0 : (double)y[3 * n], vy = (f & 2) ? 0.0 : (double)y[3 * n + 1],
                 vz = (f & 4) ? 0.0 : (double)y[3 * n + 2];
    acc[0] += vx;
    acc[1] += vy;
    acc[2] += vz;
    acc[3] += -rz * vy + ry * vz;
    acc[4] += rz * vx - rx * vz;
    acc[5] += -ry * vx + rx * vy;
  }
  // block reduction of the 6 sums in a fixed order (one barrier pair)
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int a = 0; a < 6; ++a) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[a] += __shfl_down_sync(0xffffffffu, acc[a], o);
  }
  if (lane == 0)
#pragma unroll
    for (int a = 0; a < 6; ++a) sred[wid * 6 + a] = acc[a];
  __syncthreads();
  if (threadIdx.x < 6) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += sred[w * 6 + threadIdx.x];
    part[(size_t)blockIdx.x * 6 + threadIdx.x] = t;
  }
}

// v = W_f^T K(s) z from the boundary elements of each group.  For element e of
// group G's list, y_e = s_e Ke z_e in the Hadamard basis (as in the matvec, in
// the vector precision T), then the rigid modes of G are contracted with y_e at
// the corners of e that lie in G, free DOFs only, accumulating in FP64.
// Elements whose corners all lie in G and are free contribute
// w_e^T Ke z_e = (Ke w_e)^T z_e = 0 and are not listed.
//
// Each group's list is cut into chunks of kRkChunk entries, one CTA per chunk
// (kRkThreads threads, two entries each); cptr is the CSR of chunks per group
// and cgrp the group of each chunk.  A CTA writes its partial sums; the last
// CTA of a group to finish (per-group counter) adds the group's partials in
// chunk order, so the result does not depend on scheduling, and resets the
// counter.  Output: v[G*modes + a].

// cptr[G] = sum_{G' < G} ceil(len(G') / kRkChunk), cgrp[c] = group of chunk c
// (one block of 1024 threads)
__global__ void __launch_bounds__(1024) k_chunk_ptr(int ngroups, const int32_t* __restrict__ bptr,
                                                    int32_t* __restrict__ cptr, int32_t* __restrict__ cgrp) {
  __shared__ int sc[1024];
  const int per = (ngroups + 1023) / 1024;
  const int g0 = threadIdx.x * per, g1 = min(ngroups, g0 + per);
  int loc = 0;
  for (int gg = g0; gg < g1; ++gg) loc += (bptr[gg + 1] - bptr[gg] + kRkChunk - 1) / kRkChunk;
  sc[threadIdx.x] = loc;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {  // inclusive scan
    const int v = threadIdx.x >= o ? sc[threadIdx.x - o] : 0;
    __syncthreads();
    sc[threadIdx.x] += v;
    __syncthreads();
  }
  int run = sc[threadIdx.x] - loc;
  for (int gg = g0; gg < g1; ++gg) {
    cptr[gg] = run;
    const int nch = (bptr[gg + 1] - bptr[gg] + kRkChunk - 1) / kRkChunk;
    for (int c = 0; c < nch; ++c) cgrp[run + c] = gg;
    run += nch;
  }
  if (threadIdx.x == 1023) cptr[ngroups] = sc[1023];
}

// adds the contribution of boundary element e to the 6 mode sums of group G
template <typename T>
__device__ __forceinline__ void rk_element(const GridDims& g, const KHatT<T>& kh, const DeflP& dp, int e, int G, T se,
                                           const uint8_t* __restrict__ fl, const int32_t* __restrict__ ngrp,
                                           double c0, double c1, double c2, const T* __restrict__ z,
                                           double (&acc)[6]) {
  const int r = e / g.nx;
  const int ex = e - r * g.nx;
  const int ez = r / g.ny;
  const int ey = r - ez * g.ny;
  const int n0 = ex + g.sx * (ey + g.sy * ez);
  const int pn = g.sx * g.sy;
  int gr[8], mk[8];
  T u[3][8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int nd = n0 + (k & 1) + g.sx * ((k >> 1) & 1) + pn * (k >> 2);
    gr[k] = ngrp[nd];
    mk[k] = fl[nd] & 7;
#pragma unroll
    for (int c = 0; c < 3; ++c) u[c][k] = ((mk[k] >> c) & 1) ? T(0) : z[3 * (long long)nd + c];
  }
  T Fb[3][4], Ft[3][4], Gb[3][4], Gt[3][4];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    face_fwd(u[c][0], u[c][1], u[c][2], u[c][3], Fb[c]);
    face_fwd(u[c][4], u[c][5], u[c][6], u[c][7], Ft[c]);
#pragma unroll
    for (int f = 0; f < 4; ++f) Gb[c][f] = Gt[c][f] = T(0);
  }
  hex8_core<T, KHatT<T>>(kh, se, Fb, Ft, Gb, Gt);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    face_inv(Gb[c], u[c][0], u[c][1], u[c][2], u[c][3]);
    face_inv(Gt[c], u[c][4], u[c][5], u[c][6], u[c][7]);
  }
  // contraction with the rigid modes of G in the vector precision, per element;
  // the element sums are accumulated in FP64
  const T bx = (T)(dp.hx * ex - c0), by = (T)(dp.hy * ey - c1), bz = (T)(dp.hz * ez - c2);
  const T hx = (T)dp.hx, hy = (T)dp.hy, hz = (T)dp.hz;
  T em[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    if (gr[k] != G) continue;
    const T yx = (mk[k] & 1) ? T(0) : u[0][k], yy = (mk[k] & 2) ? T(0) : u[1][k], yz = (mk[k] & 4) ? T(0) : u[2][k];
    const T rx = (k & 1) ? bx + hx : bx, ry = ((k >> 1) & 1) ? by + hy : by, rz = (k >> 2) ? bz + hz : bz;
    em[0] += yx;
    em[1] += yy;
    em[2] += yz;
    em[3] += -rz * yy + ry * yz;
    em[4] += rz * yx - rx * yz;
    em[5] += -ry * yx + rx * yy;
  }
#pragma unroll
  for (int a = 0; a < 6; ++a) acc[a] += (double)em[a];
}

// a / d for 0 <= a < 2^31 from a double reciprocal (exact after the correction)
__device__ __forceinline__ int div_by(int a, int d, double inv) {
  int q = (int)((double)a * inv);
  q -= (q * d > a);
  q += ((q + 1) * d <= a);
  return q;
}

// rk_element for an element without fixed DOFs whose corners in G are the bits of
// cmask (from the list's per-entry metadata): no group or mask loads, no selects
template <typename T>
__device__ __forceinline__ void rk_element_free(const GridDims& g, const KHatT<T>& kh, const DeflP& dp, int e,
                                                unsigned cmask, T se, double inx, double iny, double c0, double c1,
                                                double c2, const T* __restrict__ z, double (&acc)[6]) {
  const int r = div_by(e, g.nx, inx);
  const int ex = e - r * g.nx;
  const int ez = div_by(r, g.ny, iny);
  const int ey = r - ez * g.ny;
  const int n0 = ex + g.sx * (ey + g.sy * ez);
  const int pn = g.sx * g.sy;
  T u[3][8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const T* zn = z + 3 * (n0 + (k & 1) + g.sx * ((k >> 1) & 1) + pn * (k >> 2));
#pragma unroll
    for (int c = 0; c < 3; ++c) u[c][k] = zn[c];
  }
  T Fb[3][4], Ft[3][4], Gb[3][4], Gt[3][4];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    face_fwd(u[c][0], u[c][1], u[c][2], u[c][3], Fb[c]);
    face_fwd(u[c][4], u[c][5], u[c][6], u[c][7], Ft[c]);
#pragma unroll
    for (int f = 0; f < 4; ++f) Gb[c][f] = Gt[c][f] = T(0);
  }
  hex8_core<T, KHatT<T>>(kh, se, Fb, Ft, Gb, Gt);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    face_inv(Gb[c], u[c][0], u[c][1], u[c][2], u[c][3]);
    face_inv(Gt[c], u[c][4], u[c][5], u[c][6], u[c][7]);
  }
  const T bx = (T)(dp.hx * ex - c0), by = (T)(dp.hy * ey - c1), bz = (T)(dp.hz * ez - c2);
  const T hx = (T)dp.hx, hy = (T)dp.hy, hz = (T)dp.hz;
  T em[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const T in = ((cmask >> k) & 1) ? T(1) : T(0);
    const T yx = in * u[0][k], yy = in * u[1][k], yz = in * u[2][k];
    const T rx = (k & 1) ? bx + hx : bx, ry = ((k >> 1) & 1) ? by + hy : by, rz = (k >> 2) ? bz + hz : bz;
    em[0] += yx;
    em[1] += yy;
    em[2] += yz;
    em[3] += -rz * yy + ry * yz;
    em[4] += rz * yx - rx * yz;
    em[5] += -ry * yx + rx * yy;
  }
#pragma unroll
  for (int a = 0; a < 6; ++a) acc[a] += (double)em[a];
}

template <typename T>
__global__ void __launch_bounds__(kRkThreads, sizeof(T) == 4 ? 6 : 4) k_restrict_K(GridDims g, KHatT<T> kh, DeflP dp, const T* __restrict__ s,
                                                           const uint8_t* __restrict__ fl,
                                                           const int32_t* __restrict__ ngrp,
                                                           const double* __restrict__ gc,
                                                           const int32_t* __restrict__ bptr,
                                                           const int32_t* __restrict__ blist,
                                                           const int32_t* __restrict__ cptr,
                                                           const int32_t* __restrict__ cgrp, const T* __restrict__ z,
                                                           double* __restrict__ part, unsigned* __restrict__ gcount,
                                                           double* __restrict__ v, const KrylovState* S,
                                                           const uint16_t* __restrict__ meta) {
  __shared__ double sred[kRkThreads / 32 * 6];
  __shared__ int s_last;
  if (S && S->done) return;
  const int ch = blockIdx.x;
  if (ch >= cptr[dp.ngroups]) return;
  const int G = cgrp[ch];
  const int c0g = cptr[G], nch = cptr[G + 1] - c0g;
  const int end = bptr[G + 1];
  const int t0 = bptr[G] + (ch - c0g) * kRkChunk + threadIdx.x;
  const double c0 = gc[3 * G], c1 = gc[3 * G + 1], c2 = gc[3 * G + 2];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  const int e0 = t0 < end ? blist[t0] : -1;
  const int e1 = t0 + kRkThreads < end ? blist[t0 + kRkThreads] : -1;
  const T s0 = e0 >= 0 ? s[e0] : T(0);
  const T s1 = e1 >= 0 ? s[e1] : T(0);
  // bits 0-7 of an entry's metadata: its element's corners in G; bit 8: the element
  // has a fixed DOF (general path)
  const unsigned m0 = (meta && e0 >= 0) ? meta[t0] : 0x100u, m1 = (meta && e1 >= 0) ? meta[t0 + kRkThreads] : 0x100u;
  const double inx = 1.0 / g.nx, iny = 1.0 / g.ny;
  if (s0 != T(0)) {
    if (m0 & 0x100u) rk_element<T>(g, kh, dp, e0, G, s0, fl, ngrp, c0, c1, c2, z, acc);
    else rk_element_free<T>(g, kh, dp, e0, m0, s0, inx, iny, c0, c1, c2, z, acc);
  }
  if (s1 != T(0)) {
    if (m1 & 0x100u) rk_element<T>(g, kh, dp, e1, G, s1, fl, ngrp, c0, c1, c2, z, acc);
    else rk_element_free<T>(g, kh, dp, e1, m1, s1, inx, iny, c0, c1, c2, z, acc);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int a = 0; a < 6; ++a) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[a] += __shfl_down_sync(0xffffffffu, acc[a], o);
  }
  if (lane == 0)
#pragma unroll
    for (int a = 0; a < 6; ++a) sred[wid * 6 + a] = acc[a];
  __syncthreads();
  if (threadIdx.x < 6) {
    double tt = 0.0;
#pragma unroll
    for (int w = 0; w < kRkThreads / 32; ++w) tt += sred[w * 6 + threadIdx.x];
    if (nch == 1) {  // single chunk: it is the group's sum
      if (threadIdx.x < dp.modes) v[(size_t)G * dp.modes + threadIdx.x] = tt;
    } else {
      part[(size_t)ch * 6 + threadIdx.x] = tt;
    }
  }
  if (nch == 1) return;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(&gcount[G], 1u) == (unsigned)(nch - 1));
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (threadIdx.x < dp.modes) {
    double tt = 0.0;
    for (int c = c0g; c < c0g + nch; ++c) tt += __ldcg(part + (size_t)c * 6 + threadIdx.x);
    v[(size_t)G * dp.modes + threadIdx.x] = tt;
  }
  if (threadIdx.x == 0) gcount[G] = 0;
}

// mu = Einv v for a compact coarse vector v (nc entries, nc even): one warp per row,
// 16-byte loads in batches of 8 per lane, double-buffered so that the next batch is
// in flight while the current one is consumed (v through the read-only cache);
// 4 warps per CTA, all rows resident in one wave at the coarse sizes used.
constexpr int kGemvBatch = 8;
__global__ void __launch_bounds__(128) k_gemv_rows(long long nc, const double* __restrict__ Einv,
                                                   const double* __restrict__ v, double* __restrict__ mu,
                                                   const KrylovState* S) {
  if (S && S->done) return;
  const int lane = threadIdx.x & 31;
  const long long row = 4 * (long long)blockIdx.x + (threadIdx.x >> 5);
  if (row >= nc) return;
  const int h = (int)(nc >> 1);
  const double2* a2p = reinterpret_cast<const double2*>(Einv + row * nc);
  const double2* v2 = reinterpret_cast<const double2*>(v);
  double2 e[2][kGemvBatch];
  auto load = [&](int jb, double2 (&d)[kGemvBatch]) {
#pragma unroll
    for (int k = 0; k < kGemvBatch; ++k)
      if (jb + 32 * k < h) d[k] = __ldg(a2p + jb + 32 * k);
  };
  double a0 = 0.0, a1 = 0.0;
  auto use = [&](int jb, const double2 (&d)[kGemvBatch]) {
#pragma unroll
    for (int k = 0; k < kGemvBatch; ++k)
      if (jb + 32 * k < h) {
        const double2 x = __ldg(v2 + jb + 32 * k);
        a0 = fma(d[k].x, x.x, a0);
        a1 = fma(d[k].y, x.y, a1);
      }
  };
  constexpr int step = 32 * kGemvBatch;
  int jb = lane;
  load(jb, e[0]);
  for (; jb < h; jb += 2 * step) {
    if (jb + step < h) load(jb + step, e[1]);
    use(jb, e[0]);
    if (jb + step >= h) break;
    if (jb + 2 * step < h) load(jb + 2 * step, e[0]);
    use(jb + step, e[1]);
  }
  double acc = a0 + a1;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) mu[row] = acc;
}

// mu = Einv v for a compact coarse vector v (nc entries), one warp per row with
// 16-byte loads (nc even) and four independent partial sums per lane.
__global__ void __launch_bounds__(256) k_gemv(long long nc, const double* __restrict__ Einv,
                                              const double* __restrict__ v, double* __restrict__ mu,
                                              const KrylovState* S) {
  extern __shared__ double sv[];
  if (S && S->done) return;
  for (long long i = threadIdx.x; i < nc; i += blockDim.x) sv[i] = v[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  for (long long row = (long long)blockIdx.x * 8 + (threadIdx.x >> 5); row < nc; row += (long long)gridDim.x * 8) {
    const double* a = Einv + row * nc;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    if ((nc & 1) == 0) {
      // eight 16-byte loads per lane in flight (the kernel is bound by memory-level
      // parallelism: one row per warp, a few warps per SM)
      const double2* a2p = reinterpret_cast<const double2*>(a);
      const double2* v2 = reinterpret_cast<const double2*>(sv);
      const int h = (int)(nc >> 1);
      int j = lane;
      for (; j + 7 * 32 < h; j += 8 * 32) {
        double2 e[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) e[k] = __ldg(a2p + j + 32 * k);
#pragma unroll
        for (int k = 0; k < 8; k += 2) {
          const double2 x0 = v2[j + 32 * k], x1 = v2[j + 32 * (k + 1)];
          a0 = fma(e[k].x, x0.x, a0);
          a1 = fma(e[k].y, x0.y, a1);
          a2 = fma(e[k + 1].x, x1.x, a2);
          a3 = fma(e[k + 1].y, x1.y, a3);
        }
      }
      for (; j < h; j += 32) {
        const double2 e0 = __ldg(a2p + j), x0 = v2[j];
        a0 = fma(e0.x, x0.x, a0);
        a1 = fma(e0.y, x0.y, a1);
      }
    } else {
      for (long long j = lane; j < nc; j += 32) a0 = fma(__ldg(a + j), sv[j], a0);
    }
    double acc = (a0 + a1) + (a2 + a3);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) mu[row] = acc;
  }
}

// mu = Einv v (one warp per row); v = W^T y is formed while staging it in
// shared memory, summing each group's chunk partials in chunk order
__global__ void __launch_bounds__(256) k_coarse_gemv(long long nc, int modes, int nch, const double* __restrict__ Einv,
                                                     const double* __restrict__ part, double* __restrict__ mu,
                                                     const KrylovState* S) {
  extern __shared__ double sv[];
  if (S && S->done) return;
  for (long long i = threadIdx.x; i < nc; i += blockDim.x) {
    const long long gg = i / modes, a = i - gg * modes;
    double t = 0.0;
    for (int c = 0; c < nch; ++c) t += __ldg(part + (gg * nch + c) * 6 + a);
    sv[i] = t;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  for (long long row = (long long)blockIdx.x * 8 + (threadIdx.x >> 5); row < nc; row += (long long)gridDim.x * 8) {
    const double* a = Einv + row * nc;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    long long j = lane;
    for (; j + 96 < nc; j += 128) {
      a0 = fma(__ldg(a + j), sv[j], a0);
      a1 = fma(__ldg(a + j + 32), sv[j + 32], a1);
      a2 = fma(__ldg(a + j + 64), sv[j + 64], a2);
      a3 = fma(__ldg(a + j + 96), sv[j + 96], a3);
    }
    for (; j < nc; j += 32) a0 = fma(__ldg(a + j), sv[j], a0);
    double acc = (a0 + a1) + (a2 + a3);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) mu[row] = acc;
  }
}

// prolongation term of node n: (W mu) at its 3 DOFs
__device__ __forceinline__ void prolong_node(const GridDims& g, const DeflP& dp, long long n,
                                             const int32_t* __restrict__ ngrp, const double* __restrict__ gc,
                                             const double* __restrict__ mu, double (&w)[3]) {
  const int grp = ngrp[n];
  double x, y, z;
  node_xyz(g, n, dp.hx, dp.hy, dp.hz, x, y, z);
  const double* c = gc + 3 * (long long)grp;
  const double rx = x - c[0], ry = y - c[1], rz = z - c[2];
  const double* m = mu + (long long)grp * dp.modes;
  w[0] = m[0];
  w[1] = m[1];
  w[2] = m[2];
  if (dp.modes == 6) {
    w[0] += rz * m[4] - ry * m[5];
    w[1] += -rz * m[3] + rx * m[5];
    w[2] += ry * m[3] - rx * m[4];
  }
}

// x = W mu (masked); ADD: x += W mu on the free DOFs (fixed DOFs set to 0)
template <typename T, bool ADD = false>
__global__ void __launch_bounds__(256) k_prolong(GridDims g, DeflP dp, const int32_t* __restrict__ ngrp,
                                                 const double* __restrict__ gc, const double* __restrict__ mu,
                                                 const uint8_t* __restrict__ fl, T* __restrict__ x) {
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < g.nnodes;
       n += (long long)gridDim.x * blockDim.x) {
    double w[3];
    prolong_node(g, dp, n, ngrp, gc, mu, w);
    const int f = fl[n];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const bool fixed = (f >> c) & 1;  // fixed DOFs are 0 in both forms
      if (ADD)
        x[3 * n + c] = fixed ? T(0) : x[3 * n + c] + (T)w[c];
      else
        x[3 * n + c] = fixed ? T(0) : (T)w[c];
    }
  }
}

// r = b - t (FP64, fixed DOFs masked)
__global__ void k_residual64(long long n, const double* __restrict__ b, const double* __restrict__ t,
                             const uint8_t* __restrict__ fl, double* __restrict__ r) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    r[i] = ((fl[i / 3] >> (i % 3)) & 1) ? 0.0 : b[i] - t[i];
}

// r = b - t (masked), z = M^-1 r; reductions r.z, r.r, b.b (FP64)
template <typename T>
__global__ void __launch_bounds__(kNodeThreads) k_dpcg_init(GridDims g, Prec pc, const T* __restrict__ b,
                                                            const T* __restrict__ t, const double* __restrict__ w,
                                                            const uint8_t* __restrict__ fl, T* __restrict__ r,
                                                            T* __restrict__ z, KrylovState* S, double* part,
                                                            unsigned* counter) {
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
      const T bi = fixed ? T(0) : b[i];
      const T ri = fixed ? T(0) : bi - t[i];
      const T zi = (T)jacobi_apply((double)ri, f, c, wn, pc);
      r[i] = ri;
      z[i] = zi;
      rz = fma((double)ri, (double)zi, rz);
      rr = fma((double)ri, (double)ri, rr);
      bb = fma((double)bi, (double)bi, bb);
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

// x += a p, r -= a q, z = M^-1 r (stored), FP64 reductions -> beta, convergence
template <typename T>
__device__ __forceinline__ void update1_dof(const Prec& pc, int f, int c, double wn, T al, T& x, T& r, T& z, T p,
                                            T q, double& rr, double& rzn) {
  x = fma(al, p, x);
  r = fma(-al, q, r);
  z = (T)jacobi_apply((double)r, f, c, wn, pc);
  rr = fma((double)r, (double)r, rr);
  rzn = fma((double)r, (double)z, rzn);
}

// alpha = r.z / p.q; x += alpha p; r -= alpha q; z = M^-1 r; r.r, r.z (FP64).
// Threads take 16-byte chunks of the vectors (grid-stride); the DOFs after the
// last full chunk are done one at a time.
template <typename T>
__global__ void __launch_bounds__(kNodeThreads, 4) k_dpcg_update1(GridDims g, Prec pc, const double* __restrict__ w,
                                                               const uint8_t* __restrict__ fl, T* __restrict__ x,
                                                               T* __restrict__ r, T* __restrict__ z,
                                                               const T* __restrict__ p, const T* __restrict__ q,
                                                               KrylovState* S, double* part, unsigned* counter,
                                                               const double* qpart) {
  __shared__ double sred[kNodeThreads / 32 + 1];
  if (S->done) return;
  // p.Kp: from the operator's block sums (qpart, deferred) or its finished total
  const double pq = qpart ? deferred_sum<kNodeThreads>(qpart, sred) : S->pq, rz = S->rz;
  if (qpart && blockIdx.x == 0 && threadIdx.x == 0) S->pq = pq;
  const double alpha = rz / pq;
  if (!(pq > 0.0) || !isfinite(alpha)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      S->breakdown = 1;
      S->done = 1;
    }
    return;
  }
  const T al = (T)alpha;
  double rr = 0.0, rzn = 0.0;
  // stream 16-byte chunks (N DOFs) of x, r, p, q; the Jacobi weight and flags of a
  // DOF's node come through the read-only cache
  using CK = Chunk<T>;
  constexpr int N = CK::N;
  const long long ndof = 3 * g.nnodes, nck = ndof / N;
  const long long gt = blockIdx.x * (long long)blockDim.x + threadIdx.x, gs = (long long)gridDim.x * blockDim.x;
  auto chunk = [&](long long ck, T (&xv)[N], T (&rv)[N], const T (&pv)[N], const T (&qv)[N], T (&zv)[N]) {
#pragma unroll
    for (int j = 0; j < N; ++j) {
      const unsigned d = (unsigned)(N * ck) + j;  // DOF ids fit in int32 (pyto_operator_init)
      const unsigned n = d / 3;
      update1_dof<T>(pc, __ldg(fl + n), (int)(d - 3 * n), __ldg(w + n), al, xv[j], rv[j], zv[j], pv[j], qv[j], rr,
                     rzn);
    }
  };
  for (long long k = gt; k < nck; k += gs) {
    T xv[N], rv[N], pv[N], qv[N], zv[N];
    CK::ld(x, k, xv);
    CK::ld(r, k, rv);
    CK::ld(p, k, pv);
    CK::ld(q, k, qv);
    chunk(k, xv, rv, pv, qv, zv);
    CK::st(x, k, xv);
    CK::st(r, k, rv);
    CK::st(z, k, zv);
  }
  if (gt < ndof - N * nck) {  // DOFs after the last full chunk
    const unsigned i = (unsigned)(N * nck + gt), n = i / 3;
    T xi = x[i], ri = r[i], zi;
    update1_dof<T>(pc, fl[n], (int)(i - 3 * n), w[n], al, xi, ri, zi, p[i], q[i], rr, rzn);
    x[i] = xi;
    r[i] = ri;
    z[i] = zi;
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

// p = z + beta p - W mu  (beta = 0 for the start vector)
template <typename T>
__device__ __forceinline__ void update2_node(const GridDims& g, const DeflP& dp, long long n, int grp, int f,
                                             const double* __restrict__ gc, const double* __restrict__ mu, T beta,
                                             const T* zv, T* pv, bool first) {
  double x, y, zz;
  node_xyz(g, n, dp.hx, dp.hy, dp.hz, x, y, zz);
  const double* c = gc + 3 * (long long)grp;
  const double rx = x - c[0], ry = y - c[1], rz = zz - c[2];
  const double* m = mu + (long long)grp * dp.modes;
  double w0 = m[0], w1 = m[1], w2 = m[2];
  if (dp.modes == 6) {
    w0 += rz * m[4] - ry * m[5];
    w1 += -rz * m[3] + rx * m[5];
    w2 += ry * m[3] - rx * m[4];
  }
  const double wv[3] = {w0, w1, w2};
#pragma unroll
  for (int c2 = 0; c2 < 3; ++c2) {
    const T pi = first ? T(0) : pv[c2];
    pv[c2] = ((f >> c2) & 1) ? T(0) : (T)(fma(beta, pi, zv[c2]) - (T)wv[c2]);
  }
}

// p = z + beta p - W mu (first: p = z - W mu); quads of 4 nodes as in update1
template <typename T>
__global__ void __launch_bounds__(kNodeThreads) k_dpcg_update2(GridDims g, DeflP dp, const int32_t* __restrict__ ngrp,
                                                               const double* __restrict__ gc,
                                                               const double* __restrict__ mu,
                                                               const uint8_t* __restrict__ fl,
                                                               const T* __restrict__ z, T* __restrict__ p,
                                                               const KrylovState* S, int first) {
  if (!first && S->done) return;
  const T beta = first ? T(0) : (T)S->beta;
  const long long nq = g.nnodes / 4;
  const long long gt = blockIdx.x * (long long)blockDim.x + threadIdx.x, gs = (long long)gridDim.x * blockDim.x;
  for (long long t = gt; t < nq; t += gs) {
    T zv[12], pv[12];
    ld12(z + 12 * t, zv);
    if (!first) ld12(p + 12 * t, pv);
    const int4 gq = __ldg(reinterpret_cast<const int4*>(ngrp + 4 * t));
    const unsigned f4 = __ldg(reinterpret_cast<const unsigned*>(fl + 4 * t));
    const int gr[4] = {gq.x, gq.y, gq.z, gq.w};
#pragma unroll
    for (int j = 0; j < 4; ++j)
      update2_node<T>(g, dp, 4 * t + j, gr[j], (f4 >> (8 * j)) & 0xff, gc, mu, beta, zv + 3 * j, pv + 3 * j,
                      first != 0);
    st12(p + 12 * t, pv);
  }
  if (gt < g.nnodes - 4 * nq) {
    const long long n = 4 * nq + gt;
    T zv[3] = {z[3 * n], z[3 * n + 1], z[3 * n + 2]};
    T pv[3] = {p[3 * n], p[3 * n + 1], p[3 * n + 2]};
    update2_node<T>(g, dp, n, ngrp[n], fl[n], gc, mu, beta, zv, pv, first != 0);
    p[3 * n] = pv[0];
    p[3 * n + 1] = pv[1];
    p[3 * n + 2] = pv[2];
  }
}

__global__ void k_state_init2(KrylovState* S, double rtol, int max_iters, int stop_rule) {
  KrylovState z{};
  z.rtol = rtol;
  z.max_iters = max_iters;
  z.stop_rule = stop_rule;
  *S = z;
}

__global__ void __launch_bounds__(kNodeThreads) k_true_residual2(GridDims g, const double* __restrict__ b,
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

struct DpcgWs {
  KrylovState* S;
  unsigned* counter;
  double* part;
  double *r, *p, *q, *z, *w;
  uint8_t* fl;
  double *cv, *mu;     // coarse vectors
  double* rpart;       // restriction partials
  double* qpart;       // the operator's p.Kp block sums, summed by update1
  int32_t* cptr;       // boundary-list chunk table [ngroups+1]
  int32_t* cgrp;       // group of each chunk [kRkMaxChunks]
  unsigned* gcount;    // per-group chunk counters [ngroups]
  int* gexp;           // fixed-point exponent of each row group of the coarse assembly
  double *P, *Rp, *U;  // sweep scratch
  // mixed-precision inner solve (FP32 vectors), carved only for the mixed solver
  float *r32, *p32, *q32, *z32, *x32, *b32, *s32;
};

constexpr long long kMaxCoarse = 24576;  // dense coarse path: coarse vector staged in shared memory (192 KB)
constexpr long long kMaxGroups = 65536;  // groups of a deflation space (the per-group workspace tables)
constexpr long long kMaxNdCoarse = 6 * kMaxGroups;  // coarse unknowns of the nested-dissection path
constexpr double kReliableDelta = 1e-2;  // FP64 residual replacement each time ||r|| drops 100-fold
constexpr int kReliableSegment = 100;    // and at least every this many iterations
constexpr int kReliablePoll = 20;        // replacement triggers tested at least this often
constexpr int kMaxRestarts = 64;         // direction restarts before giving up

static DpcgWs carve_dpcg(const pyto_operator_t* op, long long nc, void* ws, size_t bytes, size_t* need,
                         bool mixed = false) {
  const GridDims g = make_dims(op);
  Carver cv{(char*)ws, 0, bytes};
  DpcgWs W{};
  W.S = cv.take<KrylovState>(1);
  W.counter = cv.take<unsigned>(64);
  W.part = cv.take<double>(4 * reduce_slots(op));
  W.qpart = cv.take<double>(reduce_slots(op) + 1);
  W.r = cv.take<double>(3 * g.nnodes);
  W.p = cv.take<double>(3 * g.nnodes);
  W.q = cv.take<double>(3 * g.nnodes);
  W.z = cv.take<double>(3 * g.nnodes);
  W.w = cv.take<double>(g.nnodes);
  W.fl = cv.take<uint8_t>(g.nnodes);
  W.rpart = cv.take<double>((size_t)6 * kRestrictMaxBlocks);
  W.cptr = cv.take<int32_t>((size_t)kMaxGroups + 1);
  W.cgrp = cv.take<int32_t>((size_t)kRkMaxChunks);
  W.gcount = cv.take<unsigned>((size_t)kMaxGroups);
  W.gexp = cv.take<int>((size_t)kMaxGroups);
  W.cv = cv.take<double>(2 * (nc > 0 ? nc : 1));  // k_restrict_K writes 6 slots per group
  W.mu = cv.take<double>(nc > 0 ? nc : 1);
  const long long ncd = std::min(nc > 0 ? nc : 1, kMaxCoarse);  // dense sweep scratch
  W.P = cv.take<double>(2 * kSweepB * kSweepB);
  W.Rp = cv.take<double>(kSweepB * ncd);
  W.U = cv.take<double>(kSweepB * ncd);
  if (mixed) {
    W.r32 = cv.take<float>(3 * g.nnodes);
    W.p32 = cv.take<float>(3 * g.nnodes);
    W.q32 = cv.take<float>(3 * g.nnodes);
    W.z32 = cv.take<float>(3 * g.nnodes);
    W.x32 = cv.take<float>(3 * g.nnodes);
    W.b32 = cv.take<float>(3 * g.nnodes);
    W.s32 = cv.take<float>(g.nelem);
  }
  *need = cv.off + 256;
  return W;
}

size_t dpcg_workspace_bytes(const pyto_operator_t* op, bool mixed) {
  size_t need = 0;
  carve_dpcg(op, kMaxNdCoarse, nullptr, 0, &need, mixed);
  return need;
}

static DeflP make_deflp(const pyto_operator_t* op, const pyto_deflation_t* d) {
  DeflP dp;
  dp.hx = op->hx;
  dp.hy = op->hy;
  dp.hz = op->hz;
  dp.modes = d->modes;
  dp.ngroups = d->ngroups;
  dp.nc = (long long)d->ngroups * d->modes;
  return dp;
}

static bool defl_ok(const pyto_deflation_t* d) {
  if (!(d && d->ngroups > 0 && (d->modes == 3 || d->modes == 6) && d->node_group && d->group_ptr &&
        d->group_nodes && d->group_center && (d->coarse_inv || d->coarse_nd) && d->group_box && d->nbr_ptr &&
        d->nbr_list &&
        d->max_group_nodes > 0 && d->max_nbr > 0 && d->max_nbr <= 128))
    return false;
  const long long nch = (d->max_group_nodes + kRestrictChunk - 1) / kRestrictChunk;
  return (long long)d->ngroups * nch <= kRestrictMaxBlocks && d->ngroups <= kMaxGroups;
}

// v[g*modes + a] = sum over chunks c of part[(g*nch + c)*6 + a], chunks in order
__global__ void k_restrict_sum(long long nc, int modes, int nch, const double* __restrict__ part,
                               double* __restrict__ v) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nc;
       i += (long long)gridDim.x * blockDim.x) {
    const long long gg = i / modes, a = i - gg * modes;
    double t = 0.0;
    for (int c = 0; c < nch; ++c) t += part[(gg * nch + c) * 6 + a];
    v[i] = t;
  }
}

// mu = Einv W_f^T y
template <typename T>
static int coarse_solve(const GridDims& g, const DeflP& dp, const pyto_deflation_t* d, const T* y, const DpcgWs& W,
                        const KrylovState* S, cudaStream_t st) {
  const int nch = (d->max_group_nodes + kRestrictChunk - 1) / kRestrictChunk;
  k_restrict<T><<<dp.ngroups * nch, 256, 0, st>>>(g, dp, d->group_ptr, d->group_nodes, d->group_center, W.fl, y,
                                                  nch, W.rpart);
  PYTO_COUNT(1);
  if (d->coarse_nd) {
    k_restrict_sum<<<(int)std::min<long long>((dp.nc + 255) / 256, 4 * kNumSMs), 256, 0, st>>>(dp.nc, dp.modes,
                                                                                               nch, W.rpart, W.cv);
    PYTO_COUNT(1);
    return nd_solve(d->coarse_nd, W.cv, W.mu, S, st);
  }
  const size_t shm = (size_t)dp.nc * sizeof(double);
  const int nb = (int)std::min<long long>((dp.nc + 7) / 8, 4 * kNumSMs);
  k_coarse_gemv<<<nb, 256, shm, st>>>(dp.nc, dp.modes, nch, d->coarse_inv, W.rpart, W.mu, S);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}

// p = z + beta p - W Einv W_f^T K(s) z from the boundary element lists (chunk
// tables built by chunk_setup for the current solve); first: p = z - W Einv W_f^T K z
template <typename T>
static int coarse_update_K(const pyto_operator_t* op, const GridDims& g, const DeflP& dp, const pyto_deflation_t* d,
                           const T* s, const T* z, T* p, const DpcgWs& W, int nchunks, const KrylovState* S,
                           int first, cudaStream_t st) {
  k_restrict_K<T><<<nchunks, kRkThreads, 0, st>>>(g, make_khat_t<T>(make_khat(op)), dp, s, W.fl, d->node_group,
                                                  d->group_center, d->bel_ptr, d->bel_list, W.cptr, W.cgrp, z,
                                                  W.rpart, W.gcount, W.cv, S, d->bel_meta);
  PYTO_COUNT(1);
  if (d->coarse_nd) {
    const int rc = nd_solve(d->coarse_nd, W.cv, W.mu, first ? nullptr : S, st);
    if (rc) return rc;
  } else if ((dp.nc & 1) == 0) {
    k_gemv_rows<<<(int)((dp.nc + 3) / 4), 128, 0, st>>>(dp.nc, d->coarse_inv, W.cv, W.mu, first ? nullptr : S);
  } else {
    const size_t shm = (size_t)dp.nc * sizeof(double);
    const int nb = (int)std::min<long long>((dp.nc + 7) / 8, 8 * kNumSMs);
    k_gemv<<<nb, 256, shm, st>>>(dp.nc, d->coarse_inv, W.cv, W.mu, first ? nullptr : S);
  }
  PYTO_COUNT(1);
  k_dpcg_update2<T><<<kNodeBlocks, kNodeThreads, 0, st>>>(g, dp, d->node_group, d->group_center, W.mu, W.fl, z, p,
                                                          S, first);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}

// Upper bound of the chunk count of the boundary lists (0: no lists) or a
// negative status.  Uses defl->bel_count when set; otherwise reads the list
// size from the device (a synchronising copy).
static int chunk_bound(const pyto_deflation_t* d, cudaStream_t st) {
  if (!d->bel_ptr || !d->bel_list) return 0;
  int total = d->bel_count;
  if (total <= 0) {
    PYTO_CUDA(cudaMemcpyAsync(&total, d->bel_ptr + d->ngroups, sizeof(int), cudaMemcpyDeviceToHost, st));
    PYTO_CUDA(cudaStreamSynchronize(st));
  }
  const long long bound = (long long)total / kRkChunk + d->ngroups;  // >= number of chunks
  if (total < 0 || bound > kRkMaxChunks) return PYTO_ERR_TOO_LARGE;
  return (int)std::max<long long>(bound, 1);
}

// Chunk tables of the boundary lists (no host synchronisation: safe under
// stream capture).  The group counters are zeroed here and left at zero by
// every k_restrict_K launch.
static int chunk_tables(const pyto_deflation_t* d, const DpcgWs& W, cudaStream_t st) {
  k_chunk_ptr<<<1, 1024, 0, st>>>(d->ngroups, d->bel_ptr, W.cptr, W.cgrp);
  PYTO_COUNT(1);
  PYTO_CUDA(cudaMemsetAsync(W.gcount, 0, (size_t)d->ngroups * sizeof(unsigned), st));
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}

// chunk_bound + chunk_tables; returns the chunk count (0: no lists) or a negative status
static int chunk_setup(const pyto_deflation_t* d, const DpcgWs& W, cudaStream_t st) {
  const int nch = chunk_bound(d, st);
  if (nch <= 0) return nch;
  const int rc = chunk_tables(d, W, st);
  return rc ? rc : nch;
}

// W_f^T K z from the boundary lists when they are short; with more list entries than half
// the elements (fine aggregates: most elements straddle groups, each in several lists) a
// full matvec K z and a node-wise restriction move fewer bytes.  The lists are still used
// by the coarse assembly.
static bool restrict_from_lists(const pyto_deflation_t* d, const GridDims& g, int nchunks) {
  if (nchunks <= 0) return false;
  return d->bel_count <= 0 || 2LL * d->bel_count <= g.nelem;
}

static int gemv_smem_ok(long long nc) {
  static PerDevice attr;
  if (attr.needed()) {
    if (cudaFuncSetAttribute(k_coarse_gemv, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(kMaxCoarse * sizeof(double))) != cudaSuccess ||
        cudaFuncSetAttribute(k_gemv, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(kMaxCoarse * sizeof(double))) != cudaSuccess)
      return PYTO_ERR_CUDA;
    attr.done();
  }
  return nc <= kMaxCoarse ? PYTO_OK : PYTO_ERR_TOO_LARGE;
}

}  // namespace pyto

using namespace pyto;

// Coarse operator assembly E = W_f^T K(s) W_f into defl->coarse_inv (no host
// synchronisation: safe under stream capture).  With nchunks > 0 the boundary-list
// chunk tables must be built.
static int coarse_assemble_launch(const pyto_operator_t* op, const double* s, const uint8_t* mask,
                                  const pyto_deflation_t* defl, const DpcgWs& W, int nchunks, cudaStream_t st) {
  const DeflP dp = make_deflp(op, defl);
  const GridDims g = make_dims(op);
  const bool nd = defl->coarse_nd != nullptr;
  if (nd && nchunks <= 0) return PYTO_ERR_ARG;  // the block-sparse assembly needs the boundary lists
  double* E = nd ? nd_matrix(defl->coarse_nd) : defl->coarse_inv;
  if (!E) return PYTO_ERR_ARG;
  const long long n = dp.nc;
  PYTO_CUDA(cudaMemsetAsync(E, 0, nd ? (size_t)nd_matrix_bytes(defl->coarse_nd) : (size_t)n * n * sizeof(double),
                            st));
  const size_t shm = (size_t)defl->max_nbr * 36 * sizeof(double);
  if (nchunks > 0) {
    const size_t shm2 = shm + 64 * kCrThreads * sizeof(double);
    static PerDevice attr;
    if (attr.needed()) {
      const int need = (int)(64 * kCrThreads * sizeof(double) + 128 * 36 * sizeof(double));
      PYTO_CUDA(cudaFuncSetAttribute(k_coarse_rows2<6>, cudaFuncAttributeMaxDynamicSharedMemorySize, need));
      PYTO_CUDA(cudaFuncSetAttribute(k_coarse_rows2<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, need));
      PYTO_CUDA(cudaFuncSetAttribute(k_coarse_rows2<6, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, need));
      PYTO_CUDA(cudaFuncSetAttribute(k_coarse_rows2<3, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, need));
      // three CTAs of ~74 KB per SM (the register bound allows three)
      PYTO_CUDA(cudaFuncSetAttribute(k_coarse_rows2<6>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
      PYTO_CUDA(cudaFuncSetAttribute(k_coarse_rows2<3>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
      PYTO_CUDA(cudaFuncSetAttribute(k_coarse_rows2<6, true>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
      PYTO_CUDA(cudaFuncSetAttribute(k_coarse_rows2<3, true>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
      attr.done();
    }
    double ke_rows = 0.0;  // max absolute row sum of Ke (>= its spectral norm)
    for (int i = 0; i < 24; ++i) {
      double r = 0.0;
      for (int j = 0; j < 24; ++j) r += fabs(op->ke[24 * i + j]);
      ke_rows = std::max(ke_rows, r);
    }
    k_group_scale<<<dp.ngroups, 256, 0, st>>>(dp, ke_rows, s, defl->group_center, defl->group_box, defl->bel_ptr,
                                             defl->bel_list, defl->nbr_ptr, defl->nbr_list, W.gexp);
    PYTO_COUNT(1);
    unsigned long long* Eq = reinterpret_cast<unsigned long long*>(E);
    if (nd) {  // converted, symmetrised and shifted by nd_factor
      if (dp.modes == 6)
        k_coarse_rows2<6, true><<<nchunks, kCrThreads, shm2, st>>>(
            g, make_khat(op), dp, s, mask, defl->node_group, defl->group_center, defl->bel_ptr, defl->bel_list,
            W.cptr, W.cgrp, defl->nbr_ptr, defl->nbr_list, W.gexp, Eq);
      else
        k_coarse_rows2<3, true><<<nchunks, kCrThreads, shm2, st>>>(
            g, make_khat(op), dp, s, mask, defl->node_group, defl->group_center, defl->bel_ptr, defl->bel_list,
            W.cptr, W.cgrp, defl->nbr_ptr, defl->nbr_list, W.gexp, Eq);
      PYTO_COUNT(1);
      PYTO_LAUNCH_CHECK();
      return PYTO_OK;
    }
    if (dp.modes == 6)
      k_coarse_rows2<6><<<nchunks, kCrThreads, shm2, st>>>(g, make_khat(op), dp, s, mask, defl->node_group,
                                                          defl->group_center, defl->bel_ptr, defl->bel_list, W.cptr,
                                                          W.cgrp, defl->nbr_ptr, defl->nbr_list, W.gexp, Eq);
    else
      k_coarse_rows2<3><<<nchunks, kCrThreads, shm2, st>>>(g, make_khat(op), dp, s, mask, defl->node_group,
                                                          defl->group_center, defl->bel_ptr, defl->bel_list, W.cptr,
                                                          W.cgrp, defl->nbr_ptr, defl->nbr_list, W.gexp, Eq);
    PYTO_COUNT(1);
    k_coarse_from_fixed<<<(int)std::min<long long>((n * n + 255) / 256, 8 * kNumSMs), 256, 0, st>>>(n, dp.modes,
                                                                                                   W.gexp, E);
    PYTO_COUNT(1);
    const int rc = sym_pass(n, dp.modes, E, kSymMirror, 0.0, nullptr, st);
    if (rc) return rc;
  } else {
    k_coarse_rows<<<dp.ngroups, kAsmThreads, shm, st>>>(g, make_khat(op), dp, s, mask, defl->node_group,
                                                         defl->group_center, defl->group_box, defl->nbr_ptr,
                                                         defl->nbr_list, E);
    PYTO_COUNT(1);
  }
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}

// E (in defl->coarse_inv) -> (sym(E) + shift I)^-1 in place: symmetrise, identity for
// vanishing rows, diagonal shift, blocked sweep inversion.
static int coarse_invert_launch(const pyto_deflation_t* defl, const DpcgWs& W, cudaStream_t st) {
  double* E = defl->coarse_inv;
  const long long n = (long long)defl->ngroups * defl->modes;
  if (defl->shift_relative) {
    k_diag_mean<<<1, 256, 0, st>>>(n, E, W.part);
    PYTO_COUNT(1);
  }
  {
    const int rc = sym_pass(n, defl->modes, E, kSymFinish, defl->shift, defl->shift_relative ? W.part : nullptr, st);
    if (rc) return rc;
  }
  PYTO_LAUNCH_CHECK();
  const int tiles = (int)((n + 63) / 64);
  static PerDevice attr;
  if (attr.needed()) {
    PYTO_CUDA(cudaFuncSetAttribute(k_sweep_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSweepTileSmem));
    attr.done();
  }
  // pivot block inverses alternate between two buffers: the update of step K sweeps
  // the pivot block of step K+1 into the other one
  k_sweep_pivot<<<1, 256, 0, st>>>(n, 0, (int)std::min<long long>(kSweepB, n), E, W.P);
  PYTO_COUNT(1);
  int step = 0;
  for (long long k0 = 0; k0 < n; k0 += kSweepB, ++step) {
    const int bk = (int)std::min<long long>(kSweepB, n - k0);
    double* Pc = W.P + (step & 1) * kSweepB * kSweepB;
    double* Pn = W.P + ((step + 1) & 1) * kSweepB * kSweepB;
    const long long k1 = k0 + kSweepB < n ? k0 + kSweepB : -1;
    k_sweep_panel<<<(int)((n + 15) / 16), 256, 0, st>>>(n, (int)k0, bk, E, Pc, W.Rp, W.U);
    PYTO_COUNT(1);
    k_sweep_update<<<(int)((long long)tiles * (tiles + 1) / 2), 256, kSweepTileSmem, st>>>(n, (int)k0, bk, E, Pc,
                                                                                          W.Rp, W.U,
                                                                             (int)k1, Pn);
    PYTO_COUNT(1);
  }
  {
    const int rc = sym_pass(n, defl->modes, E, kSymNegate, 0.0, nullptr, st);
    if (rc) return rc;
  }
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}

static int dpcg_setup_launch(const pyto_operator_t* op, const double* s, const uint8_t* mask,
                             const pyto_deflation_t* defl, const DpcgWs& W, int nchunks, cudaStream_t st) {
  const int rc = coarse_assemble_launch(op, s, mask, defl, W, nchunks, st);
  if (rc) return rc;
  if (defl->coarse_nd)
    return nd_factor(defl->coarse_nd, defl->nbr_ptr, defl->nbr_list, W.gexp, defl->shift, defl->shift_relative,
                     st);
  return coarse_invert_launch(defl, W, st);
}

extern "C" int pyto_dpcg_setup(const pyto_operator_t* op, const double* s, const uint8_t* mask,
                               pyto_deflation_t* defl, void* ws, size_t ws_bytes, void* stream) {
  if (!op || !s || !defl_ok(defl)) return PYTO_ERR_ARG;
  const DeflP dp = make_deflp(op, defl);
  int rc0 = gemv_smem_ok(defl->coarse_nd ? 0 : dp.nc);
  if (rc0) return rc0;
  size_t need = 0;
  DpcgWs W = carve_dpcg(op, dp.nc, ws, ws_bytes, &need);
  if (!ws || ws_bytes < need) return PYTO_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  const int nchunks = chunk_setup(defl, W, st);
  if (nchunks < 0) return nchunks;
  return dpcg_setup_launch(op, s, mask, defl, W, nchunks, st);
}

namespace pyto {

// ---------------------------------------------------------------------------
// A chunk of Krylov iterations (the kernels between two host polls) captured
// once per solve on a private stream and replayed as one CUDA graph: removes
// the gaps between the ~5 launches of every iteration.  The kernels of a
// converged state return at once, so a replay past convergence is harmless.
// Launches are counted per replay.
// ---------------------------------------------------------------------------
long long launch_count_now();
extern int g_use_graphs;

struct ChunkGraph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  long long per_replay = 0;
  ChunkGraph() = default;
  ChunkGraph(const ChunkGraph&) = delete;
  ChunkGraph& operator=(const ChunkGraph&) = delete;
  ~ChunkGraph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
  // body(stream) issues the chunk's launches and returns a status
  template <typename F>
  int build(F&& body) {
    cudaStream_t cs = nullptr;
    PYTO_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    const long long n0 = launch_count_now();
    int rc = PYTO_OK;
    const cudaError_t eb = cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed);
    if (eb != cudaSuccess) {
      record_error(eb, "cudaStreamBeginCapture(chunk)", __FILE__, __LINE__);
      rc = PYTO_ERR_CUDA;
    } else {
      rc = body(cs);
      const cudaError_t ee = cudaStreamEndCapture(cs, &graph);
      if (!rc && ee != cudaSuccess) {
        record_error(ee, "cudaStreamEndCapture(chunk)", __FILE__, __LINE__);
        rc = PYTO_ERR_CUDA;
      }
      if (!rc) {
        const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
        if (ei != cudaSuccess) {
          record_error(ei, "cudaGraphInstantiate(chunk)", __FILE__, __LINE__);
          rc = PYTO_ERR_CUDA;
        }
      }
    }
    per_replay = launch_count_now() - n0;
    count_launches(-per_replay);  // counted when replayed
    cudaGetLastError();
    cudaStreamDestroy(cs);
    return rc;
  }
  int launch(cudaStream_t st) {
    PYTO_CUDA(cudaGraphLaunch(exec, st));
    count_launches(per_replay);
    return PYTO_OK;
  }
};

template <typename T>
struct DVec {
  T *r, *p, *q, *z;
};

int launch_matvec32(const pyto_operator_t* op, const float* s, const uint8_t* mask, const float* u, float* y,
                    int mode, double* part, unsigned* counter, double* dot, cudaStream_t st,
                    const int* stop = nullptr);

// K(s) u for the iteration vectors p and z only: both are zero on fixed DOFs (z =
// M^-1 r is, by jacobi_apply; p = z + beta p - W mu is, by update2_node), so the
// input mask would select the same values and is skipped.
static int matvec_t(const pyto_operator_t* op, const double* s, const uint8_t* mask, const double* u, double* y,
                    double* part, unsigned* counter, double* dot, cudaStream_t st, const int* stop = nullptr) {
  return launch_matvec64(op, s, mask, u, y, PYTO_MASK_OUT, part, counter, dot, st, stop);
}
static int matvec_t(const pyto_operator_t* op, const float* s, const uint8_t* mask, const float* u, float* y,
                    double* part, unsigned* counter, double* dot, cudaStream_t st, const int* stop = nullptr) {
  return launch_matvec32(op, s, mask, u, y, PYTO_MASK_OUT, part, counter, dot, st, stop);
}

// One deflated PCG run (src/deflation.py:504-584) in vector precision T;
// scalars, reductions and the coarse space are FP64.  Jacobi data (W.w, W.fl)
// must be set.  On return *hs holds the final device state.
template <typename T>
static int dpcg_run(const pyto_operator_t* op, const T* s, const uint8_t* mask, const pyto_deflation_t* defl,
                    const T* b, T* u, DVec<T> V, const DpcgWs& W, double rtol, int max_iters, int stop_rule,
                    int every, KrylovState* hs, cudaStream_t st) {
  const DeflP dp = make_deflp(op, defl);
  const GridDims g = make_dims(op);
  const Prec pc = make_prec(op);
  int rc;
  k_state_init2<<<1, 1, 0, st>>>(W.S, rtol, max_iters, stop_rule);
  PYTO_COUNT(1);
  // coarse start: x = W Einv W_f^T b   (src/deflation.py:532-537)
  if ((rc = coarse_solve(g, dp, defl, b, W, nullptr, st))) return rc;
  k_prolong<T><<<kNodeBlocks, kNodeThreads, 0, st>>>(g, dp, defl->node_group, defl->group_center, W.mu, W.fl, u);
  PYTO_COUNT(1);
  // r = b - K x, z = M r
  if ((rc = matvec_t(op, s, mask, u, V.q, nullptr, nullptr, nullptr, st))) return rc;
  k_dpcg_init<T><<<kNodeBlocks, kNodeThreads, 0, st>>>(g, pc, b, V.q, W.w, W.fl, V.r, V.z, W.S, W.part, W.counter);
  PYTO_COUNT(1);
  // p0 = z - W Einv W^T K z
  const int nchunks = chunk_setup(defl, W, st);
  if (nchunks < 0) return nchunks;
  const bool lists = restrict_from_lists(defl, g, nchunks);
  if (lists) {
    if ((rc = coarse_update_K(op, g, dp, defl, s, V.z, V.p, W, nchunks, W.S, 1, st))) return rc;
  } else {
    if ((rc = matvec_t(op, s, mask, V.z, V.q, nullptr, nullptr, nullptr, st))) return rc;
    if ((rc = coarse_solve(g, dp, defl, V.q, W, nullptr, st))) return rc;
    k_dpcg_update2<T><<<kNodeBlocks, kNodeThreads, 0, st>>>(g, dp, defl->node_group, defl->group_center, W.mu,
                                                            W.fl, V.z, V.p, W.S, 1);
    PYTO_COUNT(1);
  }
  PYTO_LAUNCH_CHECK();
  auto chunk = [&](cudaStream_t cs) -> int {
    int e;
    for (int k = 0; k < every; ++k) {
      if ((e = matvec_t(op, s, mask, V.p, V.q, W.qpart, nullptr, &W.S->pq, cs, &W.S->done))) return e;
      k_dpcg_update1<T><<<kUpdate1Blocks, kNodeThreads, 0, cs>>>(g, pc, W.w, W.fl, u, V.r, V.z, V.p, V.q, W.S, W.part,
                                                              W.counter, W.qpart);
      PYTO_COUNT(1);
      // mu = Einv W^T K z (from the boundary lists, or K z -> q then W^T q), p = z + beta p - W mu
      if (lists) {
        if ((e = coarse_update_K(op, g, dp, defl, s, V.z, V.p, W, nchunks, W.S, 0, cs))) return e;
      } else {
        if ((e = matvec_t(op, s, mask, V.z, V.q, nullptr, nullptr, nullptr, cs))) return e;
        if ((e = coarse_solve(g, dp, defl, V.q, W, W.S, cs))) return e;
        k_dpcg_update2<T><<<kNodeBlocks, kNodeThreads, 0, cs>>>(g, dp, defl->node_group, defl->group_center, W.mu,
                                                                W.fl, V.z, V.p, W.S, 0);
        PYTO_COUNT(1);
      }
    }
    PYTO_LAUNCH_CHECK();
    return PYTO_OK;
  };
  // the chunk graph is captured while the set-up queued before it still runs on the GPU
  ChunkGraph cg;
  if (g_use_graphs && (rc = cg.build(chunk))) return rc;
  PYTO_CUDA(cudaMemcpyAsync(hs, W.S, sizeof(*hs), cudaMemcpyDeviceToHost, st));
  PYTO_CUDA(cudaStreamSynchronize(st));
  while (!hs->done && hs->iters < max_iters) {
    if ((rc = g_use_graphs ? cg.launch(st) : chunk(st))) return rc;
    PYTO_LAUNCH_CHECK();
    PYTO_CUDA(cudaMemcpyAsync(hs, W.S, sizeof(*hs), cudaMemcpyDeviceToHost, st));
    PYTO_CUDA(cudaStreamSynchronize(st));
  }
  return PYTO_OK;
}

template <typename A, typename B>
__global__ void k_cast(long long n, const A* __restrict__ a, B* __restrict__ b) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = (B)a[i];
}

// Reliable update: r = b - t in FP64 (t = K u, fixed DOFs masked).  With
// scaled = 1 the recurrence vectors are normalised: r_T = r / ||r||, z_T =
// M^-1 r_T, and the state records rscale2 = ||r||^2 (the FP32 recurrence then
// works on O(1) values whatever the magnitude of b); otherwise r_T = r.  Two
// passes: the first forms ||r||^2 and ||b||^2, the second writes r_T, z_T and
// r_T.z_T.  The last block of the second pass sets rr (recurrence units),
// true_rr = ||r||^2, bb, rz, clears the breakdown flag and sets converged/done
// from the FP64 residual.
__global__ void __launch_bounds__(kNodeThreads) k_residual_norms(GridDims g, const double* __restrict__ b,
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
      const double bi = b[3 * n + c], ri = bi - t[3 * n + c];
      rr = fma(ri, ri, rr);
      bb = fma(bi, bi, bb);
    }
  }
  double v[2] = {block_sum<kNodeThreads>(rr, sred), block_sum<kNodeThreads>(bb, sred)};
  grid_reduce<2>(v, part, counter, gridDim.x, [&](const double* tot) {
    S->true_rr = tot[0];
    S->bb = tot[1];
    S->rscale2_prev = S->rscale2;
    S->rscale2 = tot[0] > 0.0 ? tot[0] : 1.0;
  });
}

template <typename T>
__global__ void __launch_bounds__(kNodeThreads) k_reliable(GridDims g, Prec pc, const double* __restrict__ b,
                                                           const double* __restrict__ t, const double* __restrict__ w,
                                                           const uint8_t* __restrict__ fl, T* __restrict__ r32,
                                                           T* __restrict__ z32, T* __restrict__ p, KrylovState* S,
                                                           double* part, unsigned* counter, int scaled) {
  __shared__ double sred[kNodeThreads / 32];
  const double isc = scaled ? 1.0 / sqrt(S->rscale2) : 1.0;
  // the kept search direction moves to the units of the new residual
  const T psc = (scaled && p && S->rscale2_prev > 0.0) ? (T)sqrt(S->rscale2_prev / S->rscale2) : T(1);
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
      const double ri = (fixed ? 0.0 : bi - t[i]) * isc;
      const T rf = (T)ri;
      const T zf = (T)jacobi_apply((double)rf, f, c, wn, pc);
      r32[i] = rf;
      z32[i] = zf;
      if (psc != T(1)) p[i] *= psc;
      rz = fma((double)rf, (double)zf, rz);
      rr = fma(ri, ri, rr);
      bb = fma(bi, bi, bb);
    }
  }
  double v[3];
  v[0] = block_sum<kNodeThreads>(rz, sred);
  v[1] = block_sum<kNodeThreads>(rr, sred);
  v[2] = block_sum<kNodeThreads>(bb, sred);
  grid_reduce<3>(v, part, counter, gridDim.x, [&](const double* tot) {
    // tot[1] = ||r_T||^2, tot[2] = ||b||^2 (b is not scaled)
    S->rz = tot[0];
    S->rr = tot[1];
    if (!scaled) {
      S->true_rr = tot[1];
      S->rscale2 = 0.0;
    }
    S->bb = tot[2];
    S->breakdown = 0;
    const int conv = (tot[2] == 0.0 || sqrt(S->true_rr) <= S->rtol * sqrt(tot[2])) ? 1 : 0;
    S->converged = conv;
    S->done = conv;
  });
}

// u += sqrt(S->rscale2) (double) x   (the FP32 iterate is in the units of the
// normalised residual)
__global__ void k_add_f32(long long n, const float* __restrict__ x, const KrylovState* S, double* __restrict__ u) {
  const double sc = S->rscale2 > 0.0 ? sqrt(S->rscale2) : 1.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    u[i] = fma(sc, (double)x[i], u[i]);
}

}  // namespace pyto

using namespace pyto;


// Deflated PCG with reliable updates, vectors in precision T (float: the
// mixed solver; double: the FP64 solver with residual replacement).  The
// recurrence runs on T vectors with the T operator (FP64 reductions, scalars and
// coarse inverse); u is FP64.  Whenever the recursive residual has dropped by
// delta since the last update, or meets rtol, the iterate is folded into u,
// the coarse part of the true residual is removed (u += W Einv W_f^T (b - K u):
// the DEF2 recurrence never changes W_f^T r), and the residual is replaced by
// b - K u computed in FP64; the search direction is kept.
template <typename T>
struct RelVec;
template <>
struct RelVec<float> {
  static float* r(const DpcgWs& W) { return W.r32; }
  static float* p(const DpcgWs& W) { return W.p32; }
  static float* q(const DpcgWs& W) { return W.q32; }
  static float* z(const DpcgWs& W) { return W.z32; }
};
template <>
struct RelVec<double> {
  static double* r(const DpcgWs& W) { return W.r; }
  static double* p(const DpcgWs& W) { return W.p; }
  static double* q(const DpcgWs& W) { return W.q; }
  static double* z(const DpcgWs& W) { return W.z; }
};

template <typename T>
static int dpcg_reliable(const pyto_operator_t* op, const double* s, const uint8_t* mask,
                         const pyto_deflation_t* defl, const double* b, double* u, const pyto_solve_cfg_t* cfg,
                         double delta, pyto_solve_status_t* status, const DpcgWs& W, cudaStream_t st) {
  constexpr bool F32 = sizeof(T) == 4;
  const DeflP dp = make_deflp(op, defl);
  const GridDims g = make_dims(op);
  const Prec pc = make_prec(op);
  const long long nd = 3 * g.nnodes;
  const int nb = (int)std::min<long long>((nd + 255) / 256, 8 * kNumSMs);
  int every = std::max(1, cfg->check_every);
  T* r = RelVec<T>::r(W);
  T* p = RelVec<T>::p(W);
  T* q = RelVec<T>::q(W);
  T* z = RelVec<T>::z(W);
  T* x = nullptr;  // iterate of the recurrence: FP32 accumulator, or u itself
  const T* sT = nullptr;
  if constexpr (F32) {
    x = W.x32;
    sT = W.s32;
  } else {
    x = u;
    sT = s;
  }
  int rc;
  PYTO_CUDA(cudaMemsetAsync(W.counter, 0, 64 * sizeof(unsigned), st));
  if ((rc = pyto_jacobi(op, s, mask, W.w, W.fl, nullptr, st))) return rc;
  if constexpr (F32) {
    k_cast<double, float><<<nb, 256, 0, st>>>(g.nelem, s, W.s32);
    PYTO_COUNT(1);
  }
  const int nchunks = chunk_setup(defl, W, st);
  if (nchunks < 0) return nchunks;
  const bool lists = restrict_from_lists(defl, g, nchunks);
  k_state_init2<<<1, 1, 0, st>>>(W.S, cfg->rtol, cfg->max_iters, 0);
  PYTO_COUNT(1);
  // start: the coarse solution u = W Einv W_f^T b (src/deflation.py:532-537), or the
  // caller's u (cfg->x0_given), whose residual's coarse part the first replacement removes
  const bool warm = cfg->x0_given != 0;
  if (!warm) {
    if ((rc = coarse_solve(g, dp, defl, b, W, nullptr, st))) return rc;
    k_prolong<double><<<kNodeBlocks, kNodeThreads, 0, st>>>(g, dp, defl->node_group, defl->group_center, W.mu, W.fl,
                                                           u);
    PYTO_COUNT(1);
  }

  auto reliable = [&](bool coarse) -> int {
    int e;
    if (coarse) {
      if ((e = launch_matvec64(op, s, mask, u, W.q, PYTO_MASK_IN | PYTO_MASK_OUT, nullptr, nullptr, nullptr, st)))
        return e;
      // the FP64 residual goes to W.r: free at this point (for T = double it is the
      // recurrence residual, replaced below); W.q (K u) is likewise dead here
      k_residual64<<<nb, 256, 0, st>>>(nd, b, W.q, W.fl, W.r);
      PYTO_COUNT(1);
      if ((e = coarse_solve(g, dp, defl, (const double*)W.r, W, nullptr, st))) return e;
      k_prolong<double, true><<<kNodeBlocks, kNodeThreads, 0, st>>>(g, dp, defl->node_group, defl->group_center,
                                                                    W.mu, W.fl, u);
      PYTO_COUNT(1);
    }
    if ((e = launch_matvec64(op, s, mask, u, W.q, PYTO_MASK_IN | PYTO_MASK_OUT, nullptr, nullptr, nullptr, st)))
      return e;
    if constexpr (F32) {
      k_residual_norms<<<kNodeBlocks, kNodeThreads, 0, st>>>(g, b, W.q, W.fl, W.S, W.part, W.counter);
      PYTO_COUNT(1);
    }
    k_reliable<T><<<kNodeBlocks, kNodeThreads, 0, st>>>(g, pc, b, W.q, W.w, W.fl, r, z, coarse ? p : nullptr, W.S,
                                                        W.part, W.counter, F32 ? 1 : 0);
    PYTO_COUNT(1);
    if constexpr (F32) PYTO_CUDA(cudaMemsetAsync(W.x32, 0, nd * sizeof(float), st));
    return PYTO_OK;
  };
  auto restart_p = [&]() -> int {  // p = z - W Einv W^T K z
    int e;
    if (lists) {
      if ((e = coarse_update_K(op, g, dp, defl, sT, (const T*)z, p, W, nchunks, W.S, 1, st))) return e;
    } else {
      if ((e = matvec_t(op, sT, mask, z, q, nullptr, nullptr, nullptr, st))) return e;
      if ((e = coarse_solve(g, dp, defl, (const T*)q, W, nullptr, st))) return e;
      k_dpcg_update2<T><<<kNodeBlocks, kNodeThreads, 0, st>>>(g, dp, defl->node_group, defl->group_center, W.mu,
                                                              W.fl, z, p, W.S, 1);
      PYTO_COUNT(1);
    }
    return PYTO_OK;
  };
  if ((rc = reliable(warm))) return rc;
  if ((rc = restart_p())) return rc;
  PYTO_LAUNCH_CHECK();
  // the replacement triggers are tested between chunks: at most kReliablePoll
  // iterations apart whatever the caller's polling interval (a longer unreplaced
  // run of the low-precision recurrence loses the accuracy the replacement restores)
  every = std::min(every, kReliablePoll);
  auto chunk = [&](cudaStream_t cs) -> int {
    int e;
    for (int k = 0; k < every; ++k) {
      if ((e = matvec_t(op, sT, mask, p, q, W.qpart, nullptr, &W.S->pq, cs, &W.S->done))) return e;
      k_dpcg_update1<T><<<kUpdate1Blocks, kNodeThreads, 0, cs>>>(g, pc, W.w, W.fl, x, r, z, p, q, W.S, W.part,
                                                              W.counter, W.qpart);
      PYTO_COUNT(1);
      if (lists) {
        if ((e = coarse_update_K(op, g, dp, defl, sT, (const T*)z, p, W, nchunks, W.S, 0, cs))) return e;
      } else {
        if ((e = matvec_t(op, sT, mask, z, q, nullptr, nullptr, nullptr, cs))) return e;
        if ((e = coarse_solve(g, dp, defl, (const T*)q, W, W.S, cs))) return e;
        k_dpcg_update2<T><<<kNodeBlocks, kNodeThreads, 0, cs>>>(g, dp, defl->node_group, defl->group_center, W.mu,
                                                                W.fl, z, p, W.S, 0);
        PYTO_COUNT(1);
      }
    }
    PYTO_LAUNCH_CHECK();
    return PYTO_OK;
  };
  // the chunk graph is captured while the set-up queued before it still runs on the GPU
  ChunkGraph cg;
  if (g_use_graphs && (rc = cg.build(chunk))) return rc;
  KrylovState hs{};
  PYTO_CUDA(cudaMemcpyAsync(&hs, W.S, sizeof(hs), cudaMemcpyDeviceToHost, st));
  PYTO_CUDA(cudaStreamSynchronize(st));
  double rr_ref = hs.rr;
  double true_prev = hs.true_rr;  // true ||r||^2 at the previous update
  int updates = 1, restarts = 0, seg0 = 0;
  const double d2 = delta * delta;
  while (!hs.converged && hs.iters < cfg->max_iters) {
    if ((rc = g_use_graphs ? cg.launch(st) : chunk(st))) return rc;
    PYTO_LAUNCH_CHECK();
    PYTO_CUDA(cudaMemcpyAsync(&hs, W.S, sizeof(hs), cudaMemcpyDeviceToHost, st));
    PYTO_CUDA(cudaStreamSynchronize(st));
    if (!(hs.done || hs.rr <= d2 * rr_ref || hs.iters - seg0 >= kReliableSegment)) continue;
    // fold the FP32 iterate into u; replace the recursive residual by the true one
    if constexpr (F32) {
      k_add_f32<<<nb, 256, 0, st>>>(nd, W.x32, W.S, u);
      PYTO_COUNT(1);
    }
    const bool brk = hs.breakdown != 0;
    if ((rc = reliable(true))) return rc;
    ++updates;
    PYTO_LAUNCH_CHECK();
    PYTO_CUDA(cudaMemcpyAsync(&hs, W.S, sizeof(hs), cudaMemcpyDeviceToHost, st));
    PYTO_CUDA(cudaStreamSynchronize(st));
    // p.Kp <= 0, or a segment that did not halve the true residual: restart the
    // search direction from the new residual (the recurrence has lost the
    // conjugacy that the low-precision operator could support)
    if (!hs.converged && (brk || hs.true_rr > 0.25 * true_prev)) {
      if (++restarts > kMaxRestarts) break;
      if ((rc = restart_p())) return rc;
    }
    rr_ref = hs.rr;
    true_prev = hs.true_rr;
    seg0 = hs.iters;
  }
  status->converged = hs.converged;
  status->iters = hs.iters;
  status->breakdown = restarts > kMaxRestarts ? 1 : 0;
  status->reserved = updates;
  status->rel_res = hs.bb > 0 ? sqrt(hs.rr * (hs.rscale2 > 0.0 ? hs.rscale2 : 1.0) / hs.bb) : 0.0;
  status->true_rel_res = hs.bb > 0 ? sqrt(hs.true_rr / hs.bb) : 0.0;
  if (status->breakdown && !hs.converged) return PYTO_ERR_BREAKDOWN;
  return hs.converged ? PYTO_OK : PYTO_NOT_CONVERGED;
}

extern "C" int pyto_dpcg_mixed_solve(const pyto_operator_t* op, const double* s, const uint8_t* mask,
                                     const pyto_deflation_t* defl, const double* b, double* u,
                                     const pyto_solve_cfg_t* cfg, double delta, pyto_solve_status_t* status,
                                     void* ws, size_t ws_bytes, void* stream) {
  if (!op || !s || !b || !u || !cfg || !status || !defl_ok(defl)) return PYTO_ERR_ARG;
  if (!(cfg->rtol > 0.0) || !(delta > 0.0) || !(delta < 1.0) || cfg->max_iters < 0) return PYTO_ERR_ARG;
  if (((uintptr_t)b | (uintptr_t)u | (uintptr_t)defl->node_group) & 15) return PYTO_ERR_ARG;
  const DeflP dp = make_deflp(op, defl);
  int rc = gemv_smem_ok(defl->coarse_nd ? 0 : dp.nc);
  if (rc) return rc;
  size_t need = 0;
  DpcgWs W = carve_dpcg(op, dp.nc, ws, ws_bytes, &need, true);
  if (!ws || ws_bytes < need) return PYTO_ERR_WORKSPACE;
  return dpcg_reliable<float>(op, s, mask, defl, b, u, cfg, delta, status, W, (cudaStream_t)stream);
}

extern "C" int pyto_dpcg_solve(const pyto_operator_t* op, const double* s, const uint8_t* mask,
                               const pyto_deflation_t* defl, const double* b, double* u, const pyto_solve_cfg_t* cfg,
                               pyto_solve_status_t* status, void* ws, size_t ws_bytes, void* stream) {
  if (!op || !s || !b || !u || !cfg || !status || !defl_ok(defl)) return PYTO_ERR_ARG;
  if (!(cfg->rtol >= 0.0) || cfg->max_iters < 0 || cfg->stop_rule < 0 || cfg->stop_rule > 2) return PYTO_ERR_ARG;
  if (((uintptr_t)b | (uintptr_t)u | (uintptr_t)defl->node_group) & 15) return PYTO_ERR_ARG;
  const DeflP dp = make_deflp(op, defl);
  int rc = gemv_smem_ok(defl->coarse_nd ? 0 : dp.nc);
  if (rc) return rc;
  size_t need = 0;
  DpcgWs W = carve_dpcg(op, dp.nc, ws, ws_bytes, &need);
  if (!ws || ws_bytes < need) return PYTO_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  if (cfg->x0_given && cfg->stop_rule != 2) return PYTO_ERR_ARG;  // rules 0/1 start from the coarse solution
  if (cfg->stop_rule == 2) {
    if (!(cfg->rtol > 0.0)) return PYTO_ERR_ARG;
    return dpcg_reliable<double>(op, s, mask, defl, b, u, cfg, kReliableDelta, status, W, st);
  }
  const GridDims g = make_dims(op);
  PYTO_CUDA(cudaMemsetAsync(W.counter, 0, 64 * sizeof(unsigned), st));
  if ((rc = pyto_jacobi(op, s, mask, W.w, W.fl, nullptr, stream))) return rc;
  KrylovState hs{};
  rc = dpcg_run<double>(op, s, mask, defl, b, u, DVec<double>{W.r, W.p, W.q, W.z}, W, cfg->rtol, cfg->max_iters,
                        cfg->stop_rule, std::max(1, cfg->check_every), &hs, st);
  if (rc) return rc;
  const KrylovState before = hs;
  if ((rc = launch_matvec64(op, s, mask, u, W.q, PYTO_MASK_IN | PYTO_MASK_OUT, nullptr, nullptr, nullptr, st)))
    return rc;
  k_true_residual2<<<kNodeBlocks, kNodeThreads, 0, st>>>(g, b, W.q, W.fl, W.S, W.part, W.counter);
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

// ---------------------------------------------------------------------------
// Batched solves in one CUDA graph
// ---------------------------------------------------------------------------
// Every item becomes one branch of the graph (branches are independent and run
// concurrently): the coarse set-up of pyto_dpcg_setup, the start of the
// deflated PCG, and a conditional WHILE node whose body is one iteration
// (matvec + dot, update, W^T K z from the boundary lists, coarse correction
// and direction update) followed by a one-thread kernel that sets the loop
// condition from the device-side stopping flag.  The flag is raised on
// convergence, breakdown or max_iters, so every loop ends; kernels of a
// converged item return at once.  A launch of the graph solves every item;
// the item buffers are read at each launch, so new densities and loads only
// need the buffers rewritten.

__global__ void k_while_cond(cudaGraphConditionalHandle h, const KrylovState* S) {
  cudaGraphSetConditional(h, S->done ? 0u : 1u);
}

struct pyto_batch {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<const KrylovState*> S;
};

// setup: nullptr = this branch builds the coarse inverse and records *setup_done;
// otherwise the branch waits for that event (items sharing one deflation space)
static int batch_branch(const pyto_batch_item_t& it, const pyto_solve_cfg_t* cfg, cudaStream_t si,
                        cudaStream_t sb, const KrylovState** S_out, cudaEvent_t setup_done, bool do_setup) {
  const pyto_operator_t* op = it.op;
  const pyto_deflation_t* defl = it.defl;
  if (!op || !it.s || !it.b || !it.u || !defl_ok(defl) || !defl->bel_ptr || !defl->bel_list || defl->bel_count <= 0)
    return PYTO_ERR_ARG;
  if (((uintptr_t)it.b | (uintptr_t)it.u | (uintptr_t)defl->node_group) & 15) return PYTO_ERR_ARG;
  const DeflP dp = make_deflp(op, defl);
  int rc = gemv_smem_ok(dp.nc);
  if (rc) return rc;
  size_t need = 0;
  const DpcgWs W = carve_dpcg(op, dp.nc, it.ws, it.ws_bytes, &need);
  if (!it.ws || it.ws_bytes < need) return PYTO_ERR_WORKSPACE;
  const int nchunks = chunk_bound(defl, si);
  if (nchunks <= 0) return nchunks < 0 ? nchunks : PYTO_ERR_ARG;
  if ((rc = chunk_tables(defl, W, si))) return rc;
  if (do_setup) {
    if ((rc = dpcg_setup_launch(op, it.s, it.mask, defl, W, nchunks, si))) return rc;
    PYTO_CUDA(cudaEventRecord(setup_done, si));
  } else {
    PYTO_CUDA(cudaStreamWaitEvent(si, setup_done, 0));
  }
  // start of the deflated PCG (as dpcg_run)
  const GridDims g = make_dims(op);
  const Prec pc = make_prec(op);
  PYTO_CUDA(cudaMemsetAsync(W.counter, 0, 64 * sizeof(unsigned), si));
  if ((rc = pyto_jacobi(op, it.s, it.mask, W.w, W.fl, nullptr, si))) return rc;
  k_state_init2<<<1, 1, 0, si>>>(W.S, cfg->rtol, cfg->max_iters, cfg->stop_rule);
  PYTO_COUNT(1);
  if ((rc = coarse_solve(g, dp, defl, it.b, W, nullptr, si))) return rc;
  k_prolong<double><<<kNodeBlocks, kNodeThreads, 0, si>>>(g, dp, defl->node_group, defl->group_center, W.mu, W.fl,
                                                         it.u);
  PYTO_COUNT(1);
  if ((rc = launch_matvec64(op, it.s, it.mask, it.u, W.q, PYTO_MASK_IN | PYTO_MASK_OUT, nullptr, nullptr, nullptr,
                            si)))
    return rc;
  k_dpcg_init<double><<<kNodeBlocks, kNodeThreads, 0, si>>>(g, pc, it.b, W.q, W.w, W.fl, W.r, W.z, W.S, W.part,
                                                           W.counter);
  PYTO_COUNT(1);
  if ((rc = coarse_update_K(op, g, dp, defl, it.s, (const double*)W.z, W.p, W, nchunks, W.S, 1, si))) return rc;
  // the iteration loop: a conditional WHILE node made the capture's next dependency
  cudaStreamCaptureStatus cs;
  cudaGraph_t cg = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  PYTO_CUDA(cudaStreamGetCaptureInfo(si, &cs, nullptr, &cg, &deps, &ndeps));
  if (cs != cudaStreamCaptureStatusActive) return PYTO_ERR_CUDA;
  cudaGraphConditionalHandle h;
  PYTO_CUDA(cudaGraphConditionalHandleCreate(&h, cg, 1u, cudaGraphCondAssignDefault));
  cudaGraphNodeParams np = {};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t cnode;
  PYTO_CUDA(cudaGraphAddNode(&cnode, cg, deps, ndeps, &np));
  cudaGraph_t body = np.conditional.phGraph_out[0];
  PYTO_CUDA(cudaStreamUpdateCaptureDependencies(si, &cnode, 1, cudaStreamSetCaptureDependencies));
  PYTO_CUDA(cudaStreamBeginCaptureToGraph(sb, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  int brc = launch_matvec64(op, it.s, it.mask, W.p, W.q, PYTO_MASK_OUT, W.part, W.counter, &W.S->pq,  // p: masked
                            sb);
  if (!brc) {
    k_dpcg_update1<double><<<kUpdate1Blocks, kNodeThreads, 0, sb>>>(g, pc, W.w, W.fl, it.u, W.r, W.z, W.p, W.q, W.S,
                                                                W.part, W.counter, nullptr);
    PYTO_COUNT(1);
    brc = coarse_update_K(op, g, dp, defl, it.s, (const double*)W.z, W.p, W, nchunks, W.S, 0, sb);
  }
  if (!brc) {
    k_while_cond<<<1, 1, 0, sb>>>(h, W.S);
    PYTO_COUNT(1);
    const cudaError_t el = cudaGetLastError();
    if (el != cudaSuccess) {
      record_error(el, "k_while_cond launch", __FILE__, __LINE__);
      brc = PYTO_ERR_CUDA;
    }
  }
  cudaGraph_t captured = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(sb, &captured);
  if (brc) return brc;
  if (ec != cudaSuccess) {
    record_error(ec, "cudaStreamEndCapture(body)", __FILE__, __LINE__);
    return PYTO_ERR_CUDA;
  }
  // FP64 true residual of the result
  if ((rc = launch_matvec64(op, it.s, it.mask, it.u, W.q, PYTO_MASK_IN | PYTO_MASK_OUT, nullptr, nullptr, nullptr,
                            si)))
    return rc;
  k_true_residual2<<<kNodeBlocks, kNodeThreads, 0, si>>>(g, it.b, W.q, W.fl, W.S, W.part, W.counter);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  *S_out = W.S;
  return PYTO_OK;
}

extern "C" int pyto_batch_create(const pyto_batch_item_t* items, int n, const pyto_solve_cfg_t* cfg,
                                 pyto_batch_t* out, void* stream) {
  if (!items || n <= 0 || !cfg || !out) return PYTO_ERR_ARG;
  if (!(cfg->rtol >= 0.0) || cfg->max_iters <= 0 || cfg->stop_rule < 0 || cfg->stop_rule > 1) return PYTO_ERR_ARG;
  for (int i = 0; i < n; ++i)  // the batched graph uses the dense coarse inverse
    if (!items[i].defl || items[i].defl->coarse_nd) return PYTO_ERR_ARG;
  *out = nullptr;
  (void)stream;  // nothing runs at creation: the capture uses a private non-blocking stream
  cudaStream_t st = nullptr;
  std::vector<cudaStream_t> ss(n, nullptr);
  std::vector<cudaEvent_t> ev(2 * n + 1, nullptr);  // [0, n): joins, n: fork, (n, 2n]: set-up done
  cudaStream_t sb = nullptr;
  auto* B = new pyto_batch();
  B->S.assign(n, nullptr);
  int rc = PYTO_OK;
  bool capturing = false;
  auto fail = [&](int code) {
    rc = code;
    return code;
  };
  // true when the call succeeded; a failure is recorded for pyto_last_error
  auto ok_ = [](cudaError_t e, const char* what, int line) {
    if (e != cudaSuccess) record_error(e, what, __FILE__, line);
    return e == cudaSuccess;
  };
#define PYTO_OK_(call) ok_((call), #call, __LINE__)
  do {
    if (!PYTO_OK_(cudaStreamCreateWithFlags(&sb, cudaStreamNonBlocking)) ||
        !PYTO_OK_(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking))) {
      fail(PYTO_ERR_CUDA);
      break;
    }
    bool ok = true;
    for (int i = 0; i < n && ok; ++i) ok = PYTO_OK_(cudaStreamCreateWithFlags(&ss[i], cudaStreamNonBlocking));
    for (int i = 0; i <= 2 * n && ok; ++i)
      ok = PYTO_OK_(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming));
    if (!ok) { fail(PYTO_ERR_CUDA); break; }
    if (!PYTO_OK_(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed))) { fail(PYTO_ERR_CUDA); break; }
    capturing = true;
    if (!PYTO_OK_(cudaEventRecord(ev[n], st))) { fail(PYTO_ERR_CUDA); break; }
    for (int i = 0; i < n && !rc; ++i) {
      if (!PYTO_OK_(cudaStreamWaitEvent(ss[i], ev[n], 0))) { fail(PYTO_ERR_CUDA); break; }
      int owner = i;  // first item with the same deflation space builds its coarse inverse
      for (int j = 0; j < i; ++j)
        if (items[j].defl == items[i].defl) {
          owner = j;
          break;
        }
      if (owner != i && (items[owner].op != items[i].op || items[owner].s != items[i].s ||
                         items[owner].mask != items[i].mask)) {
        fail(PYTO_ERR_ARG);  // a shared deflation space needs the same operator, s and mask
        break;
      }
      const int r = batch_branch(items[i], cfg, ss[i], sb, &B->S[i], ev[n + 1 + owner], owner == i);
      if (r) { fail(r); break; }
      if (!PYTO_OK_(cudaEventRecord(ev[i], ss[i])) || !PYTO_OK_(cudaStreamWaitEvent(st, ev[i], 0))) {
        fail(PYTO_ERR_CUDA);
        break;
      }
    }
  } while (false);
  if (capturing) {
    cudaGraph_t gph = nullptr;
    const bool ended = PYTO_OK_(cudaStreamEndCapture(st, &gph));
    if (!rc && !ended) rc = PYTO_ERR_CUDA;
    if (!rc) {
      B->graph = gph;
      if (!PYTO_OK_(cudaGraphInstantiate(&B->exec, B->graph, 0))) rc = PYTO_ERR_CUDA;
    } else if (gph) {
      cudaGraphDestroy(gph);
    }
  }
  cudaGetLastError();  // errors are reported through rc
  for (auto e : ev)
    if (e) cudaEventDestroy(e);
  for (auto s2 : ss)
    if (s2) cudaStreamDestroy(s2);
  if (sb) cudaStreamDestroy(sb);
  if (st) cudaStreamDestroy(st);
  if (rc) {
    if (B->exec) cudaGraphExecDestroy(B->exec);
    if (B->graph) cudaGraphDestroy(B->graph);
    delete B;
    return rc;
  }
  *out = B;
  return PYTO_OK;
#undef PYTO_OK_
}

extern "C" int pyto_batch_launch(pyto_batch_t b, void* stream) {
  if (!b || !b->exec) return PYTO_ERR_ARG;
  PYTO_CUDA(cudaGraphLaunch(b->exec, (cudaStream_t)stream));
  return PYTO_OK;
}

extern "C" int pyto_batch_status(pyto_batch_t b, pyto_solve_status_t* status, void* stream) {
  if (!b || !status) return PYTO_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<KrylovState> hs(b->S.size());
  for (size_t i = 0; i < b->S.size(); ++i)
    PYTO_CUDA(cudaMemcpyAsync(&hs[i], b->S[i], sizeof(KrylovState), cudaMemcpyDeviceToHost, st));
  PYTO_CUDA(cudaStreamSynchronize(st));
  int worst = PYTO_OK;
  for (size_t i = 0; i < b->S.size(); ++i) {
    const KrylovState& k = hs[i];
    pyto_solve_status_t& o = status[i];
    o.converged = k.converged;
    o.iters = k.iters;
    o.breakdown = k.breakdown;
    o.reserved = 0;
    o.rel_res = k.bb > 0 ? sqrt((k.stop_rule == 0 ? k.rr : k.rz) / (k.stop_rule == 0 ? k.bb : k.rz0)) : 0.0;
    o.true_rel_res = k.bb > 0 ? sqrt(k.true_rr / k.bb) : 0.0;
    if (k.breakdown) worst = PYTO_ERR_BREAKDOWN;
    else if (!k.converged && worst == PYTO_OK) worst = PYTO_NOT_CONVERGED;
  }
  return worst;
}

extern "C" int pyto_batch_destroy(pyto_batch_t b) {
  if (!b) return PYTO_OK;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  delete b;
  return PYTO_OK;
}

// ---------------------------------------------------------------------------
// Building blocks of a deflated PCG whose vectors are split across ranks (slabs
// of node planes).  The host composes them between its collectives: halo
// exchange before each operator application, a sum over ranks of the dot
// products, of the restricted coarse vectors and of the coarse matrix.  A rank
// marks its halo nodes as fixed in the mask it passes here, so outputs, dot
// products and restrictions cover its own nodes only.
// ---------------------------------------------------------------------------
namespace pyto {

// p = a z + b p - W mu on free DOFs, 0 on fixed ones (z may be null: a z = 0)
__global__ void __launch_bounds__(256) k_prolong_axpby(GridDims g, DeflP dp, const int32_t* __restrict__ ngrp,
                                                       const double* __restrict__ gc, const double* __restrict__ mu,
                                                       const uint8_t* __restrict__ fl, double a,
                                                       const double* __restrict__ z, double b,
                                                       double* __restrict__ p) {
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < g.nnodes;
       n += (long long)gridDim.x * blockDim.x) {
    double w[3];
    prolong_node(g, dp, n, ngrp, gc, mu, w);
    const int f = fl[n];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const long long i = 3 * n + c;
      double v = -w[c];
      if (z) v = fma(a, z[i], v);
      if (b != 0.0) v = fma(b, p[i], v);
      p[i] = ((f >> c) & 1) ? 0.0 : v;
    }
  }
}

// x += alpha p (if p, x given); r -= alpha q (if q given); z = M r (Jacobi,
// src/linear_solvers.py:71-87); the sums r.r and r.z over the free DOFs
// (deterministic cross-block reduction) -> dots
__global__ void __launch_bounds__(kNodeThreads) k_cg_update(GridDims g, Prec pc, const double* __restrict__ w,
                                                            const uint8_t* __restrict__ fl, double alpha,
                                                            const double* __restrict__ p,
                                                            const double* __restrict__ q, double* __restrict__ x,
                                                            double* __restrict__ r, double* __restrict__ z,
                                                            double* __restrict__ part, unsigned* __restrict__ counter,
                                                            double* __restrict__ dots) {
  __shared__ double sred[kNodeThreads / 32];
  double rr = 0.0, rz = 0.0;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < g.nnodes;
       n += (long long)gridDim.x * blockDim.x) {
    const int f = fl[n];
    const double wn = w[n];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const long long i = 3 * n + c;
      double ri = r[i];
      if (q) {
        ri = fma(-alpha, q[i], ri);
        r[i] = ri;
      }
      if (p && x) x[i] = fma(alpha, p[i], x[i]);
      const double zi = jacobi_apply(ri, f, c, wn, pc);
      z[i] = zi;
      if (!((f >> c) & 1)) {
        rr = fma(ri, ri, rr);
        rz = fma(ri, zi, rz);
      }
    }
  }
  double v[2] = {block_sum<kNodeThreads>(rr, sred), block_sum<kNodeThreads>(rz, sred)};
  grid_reduce<2>(v, part, counter, gridDim.x, [&](const double* tot) {
    dots[0] = tot[0];
    dots[1] = tot[1];
  });
}

}  // namespace pyto

extern "C" int pyto_coarse_assemble(const pyto_operator_t* op, const double* s, const uint8_t* mask,
                                    pyto_deflation_t* defl, void* ws, size_t ws_bytes, void* stream) {
  if (!op || !s || !defl_ok(defl) || defl->coarse_nd) return PYTO_ERR_ARG;  // the dense coarse matrix only
  const DeflP dp = make_deflp(op, defl);
  if (dp.nc > kMaxCoarse) return PYTO_ERR_TOO_LARGE;
  size_t need = 0;
  DpcgWs W = carve_dpcg(op, dp.nc, ws, ws_bytes, &need);
  if (!ws || ws_bytes < need) return PYTO_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  const int nchunks = chunk_setup(defl, W, st);
  if (nchunks < 0) return nchunks;
  return coarse_assemble_launch(op, s, mask, defl, W, nchunks, st);
}

extern "C" int pyto_coarse_invert(const pyto_operator_t* op, pyto_deflation_t* defl, void* ws, size_t ws_bytes,
                                  void* stream) {
  if (!op || !defl_ok(defl) || defl->coarse_nd) return PYTO_ERR_ARG;
  const DeflP dp = make_deflp(op, defl);
  int rc0 = gemv_smem_ok(dp.nc);
  if (rc0) return rc0;
  size_t need = 0;
  DpcgWs W = carve_dpcg(op, dp.nc, ws, ws_bytes, &need);
  if (!ws || ws_bytes < need) return PYTO_ERR_WORKSPACE;
  return coarse_invert_launch(defl, W, (cudaStream_t)stream);
}

extern "C" int pyto_coarse_restrict(const pyto_operator_t* op, const pyto_deflation_t* defl, const uint8_t* mask,
                                    const double* y, double* v, void* ws, size_t ws_bytes, void* stream) {
  if (!op || !mask || !y || !v || !defl_ok(defl)) return PYTO_ERR_ARG;
  const DeflP dp = make_deflp(op, defl);
  if (dp.nc > kMaxCoarse) return PYTO_ERR_TOO_LARGE;
  size_t need = 0;
  DpcgWs W = carve_dpcg(op, dp.nc, ws, ws_bytes, &need);
  if (!ws || ws_bytes < need) return PYTO_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  const GridDims g = make_dims(op);
  const int nch = (defl->max_group_nodes + kRestrictChunk - 1) / kRestrictChunk;
  k_restrict<double><<<dp.ngroups * nch, 256, 0, st>>>(g, dp, defl->group_ptr, defl->group_nodes,
                                                       defl->group_center, mask, y, nch, W.rpart);
  PYTO_COUNT(1);
  k_restrict_sum<<<(int)std::min<long long>((dp.nc + 255) / 256, 4 * kNumSMs), 256, 0, st>>>(dp.nc, dp.modes, nch,
                                                                                             W.rpart, v);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}

extern "C" int pyto_coarse_apply(const pyto_deflation_t* defl, const double* v, double* mu, void* stream) {
  if (!defl_ok(defl) || defl->coarse_nd || !v || !mu || v == mu) return PYTO_ERR_ARG;
  const long long nc = (long long)defl->ngroups * defl->modes;
  if (nc > kMaxCoarse) return PYTO_ERR_TOO_LARGE;
  int rc0 = gemv_smem_ok(nc);
  if (rc0) return rc0;
  cudaStream_t st = (cudaStream_t)stream;
  if ((nc & 1) == 0 && ((uintptr_t)v & 15) == 0) {
    k_gemv_rows<<<(int)((nc + 3) / 4), 128, 0, st>>>(nc, defl->coarse_inv, v, mu, nullptr);
  } else {
    const size_t shm = (size_t)nc * sizeof(double);
    const int nb = (int)std::min<long long>((nc + 7) / 8, 8 * kNumSMs);
    k_gemv<<<nb, 256, shm, st>>>(nc, defl->coarse_inv, v, mu, nullptr);
  }
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}

extern "C" int pyto_coarse_prolong(const pyto_operator_t* op, const pyto_deflation_t* defl, const uint8_t* mask,
                                   const double* mu, double a, const double* z, double b, double* p, void* stream) {
  if (!op || !mask || !mu || !p || !defl_ok(defl)) return PYTO_ERR_ARG;
  const GridDims g = make_dims(op);
  const int nb = (int)std::min<long long>((g.nnodes + 255) / 256, 8 * kNumSMs);
  k_prolong_axpby<<<nb, 256, 0, (cudaStream_t)stream>>>(g, make_deflp(op, defl), defl->node_group,
                                                        defl->group_center, mu, mask, a, z, b, p);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}

extern "C" int pyto_cg_update(const pyto_operator_t* op, const double* winv, const uint8_t* flags, double alpha,
                              const double* p, const double* q, double* x, double* r, double* z, double* dots,
                              void* ws, size_t ws_bytes, void* stream) {
  if (!op || !winv || !flags || !r || !z || !dots || (!p != !x)) return PYTO_ERR_ARG;
  Carver cv{(char*)ws, 0, ws_bytes};
  unsigned* counter = cv.take<unsigned>(64);
  double* part = cv.take<double>(2 * (size_t)kNodeBlocks);
  if (!cv.ok()) return PYTO_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  PYTO_CUDA(cudaMemsetAsync(counter, 0, 64 * sizeof(unsigned), st));
  k_cg_update<<<kNodeBlocks, kNodeThreads, 0, st>>>(make_dims(op), make_prec(op), winv, flags, alpha, p, q, x, r, z,
                                                    part, counter, dots);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}
