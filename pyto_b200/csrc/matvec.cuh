// Matrix-free hex8 operator helpers (FP64 and FP32): the element core in the
// Hadamard basis, face transforms and the tile decomposition shared by the
// operator kernels and the deflation kernels.
//
// Work decomposition.  A CTA owns a box of (TX-1) x (TY-1) node columns and a
// slab of node planes [Z0, Z1).  Its TX x TY threads each own one *element
// column* (ex, ey) = (X0-1+tx, Y0-1+ty) and march up the element layers
// ez = Z0-1 .. Z1-1.  Elements of the one-element halo are recomputed by the
// neighbouring CTAs, so every node's sum is formed by exactly one thread and
// no atomics are needed (results are bitwise reproducible).
//
// Per element, in the Hadamard corner basis (see element.cu): face transforms
// of the bottom and top faces (8 add/comp each), their z-combination, 57 FMAs
// of the block operator scaled by s_e, inverse z-split into bottom/top face
// contributions; a face is inverse-transformed once after both elements that
// share it were accumulated.  Node contributions of the 4 columns around a
// vertical node line are combined with one shuffle (x) and one shared-memory
// exchange (y).  The node-plane staging of the two kernels that use these
// helpers is described in matvec.cu and matvec_chunked.cuh.
#pragma once
#include "common.cuh"

namespace pyto {

template <int TX, int TY>
struct MvTile {
  static_assert(TX == 32, "x-combine uses warp shuffles: one warp per row");
  static constexpr int NT = TX * TY;
  static constexpr int PX = TX + 1, PY = TY + 1;
  static constexpr int PLANE = PX * PY;
  static constexpr int PLANE_D = 3 * PLANE;
  static constexpr int LOADS = (PLANE_D + NT - 1) / NT;
};

// The block operator's coefficients in the kernel's precision (no per-use conversion
// from the FP64 KHat in FP32 kernels).
template <typename T>
struct KHatT {
  T b[8][9];
};

template <typename T>
inline KHatT<T> make_khat_t(const KHat& kh) {
  KHatT<T> k;
  for (int q = 0; q < 8; ++q)
    for (int i = 0; i < 9; ++i) k.b[q][i] = (T)kh.b[q][i];
  return k;
}

// Mode of component c in parity class q (the pair (c, q ^ (1<<c))).
__host__ __device__ constexpr int member_mode(int q, int c) { return q ^ (1 << c); }

// Element core in the Hadamard basis.  Fb/Ft: face transforms of bottom/top
// faces, [comp][face mode].  Adds the bottom-face part of s*K^u to Gb and the
// top-face part to Gt.  KH: KHat or KHatT<T> (coefficients b[8][9]).
template <typename T, typename KH = KHat>
__device__ __forceinline__ void hex8_core(const KH& kh, T s, const T (&Fb)[3][4], const T (&Ft)[3][4],
                                          T (&Gb)[3][4], T (&Gt)[3][4]) {
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    T v[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int m = member_mode(q, d);
      const int f = m & 3;
      if (m == 0) {
        v[d] = T(0);
      } else if (m & 4) {
        v[d] = s * (Ft[d][f] - Fb[d][f]);
      } else {
        v[d] = s * (Ft[d][f] + Fb[d][f]);
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int m = member_mode(q, c);
      if (m == 0) continue;
      const int f = m & 3;
      T o = T(0);
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        if (member_mode(q, d) == 0) continue;
        o = fma((T)kh.b[q][3 * c + d], v[d], o);
      }
      if (m & 4) {
        Gb[c][f] -= o;
        Gt[c][f] += o;
      } else {
        Gb[c][f] += o;
        Gt[c][f] += o;
      }
    }
  }
}

// 2-D Hadamard transform of a face's 4 corner values (a_xy).
template <typename T>
__device__ __forceinline__ void face_fwd(T a00, T a10, T a01, T a11, T (&F)[4]) {
  const T s0 = a00 + a10, d0 = a10 - a00, s1 = a01 + a11, d1 = a11 - a01;
  F[0] = s0 + s1;
  F[1] = d0 + d1;
  F[2] = s1 - s0;
  F[3] = d1 - d0;
}

// Inverse (= transpose) face transform: corner values from face-mode values.
template <typename T>
__device__ __forceinline__ void face_inv(const T (&G)[4], T& c00, T& c10, T& c01, T& c11) {
  const T A = G[0] - G[2], B = G[1] - G[3], C = G[0] + G[2], D = G[1] + G[3];
  c00 = A - B;
  c10 = A + B;
  c01 = C - D;
  c11 = C + D;
}

constexpr long long kMatvecMaxBlocks = 4096;  // CTA cap of the slab split

// Node planes per CTA for bx x by tiles per plane with `slots` CTAs resident on the
// device: of the splits into slabs of zc = ceil(sz / nb) planes (zc >= 4 unless
// sz < 4, at most max(kMatvecMaxBlocks, bx by) CTAs), the one with the least
// (waves of `slots` CTAs) x (zc + 2), the 2 standing for the recomputed halo layer and
// the pipeline start of a slab.  A partly filled last wave leaves SMs idle for a
// whole slab, so the split is chosen against the wave count, not a CTA target.
inline int matvec_zc(int bx, int by, int sz, int slots) {
  const long long nxy = (long long)bx * by;
  const int zmin = sz < 4 ? sz : 4;
  long long nbmax = kMatvecMaxBlocks / nxy;
  const long long nbz_max = (sz + zmin - 1) / zmin;
  if (nbmax > nbz_max) nbmax = nbz_max;
  if (nbmax < 1) nbmax = 1;
  if (slots < 1) slots = 1;
  int best_zc = sz;
  long long best = -1;
  for (long long nb = 1; nb <= nbmax; ++nb) {
    const int zc = (int)((sz + nb - 1) / nb);
    if (zc < zmin) break;
    const long long nbz = (sz + zc - 1) / zc;
    const long long cost = ((nxy * nbz + slots - 1) / slots) * (zc + 2);
    if (best < 0 || cost < best) {
      best = cost;
      best_zc = zc;
    }
  }
  return best_zc;
}

struct MvLaunch {
  dim3 grid;
  int zc;
  long long nblocks;
};

template <int TX, int TY>
inline MvLaunch matvec_launch(const GridDims& g, int slots) {
  MvLaunch L;
  const int bx = (g.sx + TX - 2) / (TX - 1), by = (g.sy + TY - 2) / (TY - 1);
  L.zc = matvec_zc(bx, by, g.sz, slots);
  const int bz = (g.sz + L.zc - 1) / L.zc;
  L.grid = dim3(bx, by, bz);
  L.nblocks = (long long)bx * by * bz;
  return L;
}

// Upper bound of the CTA count of every operator launch: a split never exceeds
// max(kMatvecMaxBlocks, tiles per plane), and the 31 x 3-node tile has the most tiles.
inline long long matvec_block_bound(const GridDims& g) {
  const long long nxy = (long long)((g.sx + 30) / 31) * ((g.sy + 2) / 3);
  return nxy > kMatvecMaxBlocks ? nxy : kMatvecMaxBlocks;
}

}  // namespace pyto
