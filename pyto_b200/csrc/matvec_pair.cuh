// Matrix-free K(s) u, FP32: two element rows per thread as the lanes of packed FP32x2
// values, with the element core specialised to the block structure of K^ (included
// by matvec.cu after matvec_chunked2.cuh).
//
// Decomposition, staging and node combination are those of k_matvec_chunked2 (a CTA
// of 32 x TY threads, two y-adjacent element columns per thread, 31 x (2 TY - 1)
// owned node columns, a z-march over a slab of node planes).  What differs:
//
// * The element core runs per pair of parity classes (q, q + 4), which share the
//   face modes of their inputs: the even and odd z-combinations Ft +- Fb of those
//   face modes feed both classes, and the two classes' outputs of each component are
//   the even and odd parts of one face mode of the bottom and top faces.  s is
//   applied once per output pair: bottom += s (even - odd), top = s (even + odd).
// * For an isotropic box element the hourglass mode 7 (x y z) of classes 3, 5 and 6
//   decouples from the other two components (KS_BOX: 45 multiply-adds per element
//   instead of 57); for a cube, class 0 and 7 blocks are (d - e) I + e 1 1^T, the
//   2 x 2 part of classes 3, 5, 6 is a 1 1^T (KS_CUBE: 33).  The launcher checks the
//   structure of the operator's K^ and picks the form; a Ke without it runs
//   k_matvec_chunked2.
// * The plane ring has 8 slots (slot = plane & 7) with four planes in flight; a
//   thread's chunk rows and shared-memory destinations are set up once per launch.
// * The fused u.y sums each node's three products in FP32 (the accuracy of the FP32
//   y itself) and accumulates the node sums in FP64.
//
// Each thread's arithmetic is fixed, and every node sum is formed by one thread in
// a fixed order: results are bitwise reproducible (they differ from the other
// operator kernels in rounding only).
#pragma once
#include <type_traits>

#include "matvec_chunked2.cuh"

namespace pyto {

enum { KS_DENSE = 0, KS_BOX = 1, KS_CUBE = 2 };

template <int TY>
struct PairTile {
  static constexpr int TX = 32, NT = TX * TY, PX = TX + 1, PY = 2 * TY + 1;
  static constexpr int CH = 4;                                // floats per 16-byte chunk
  static constexpr int NCH = (CH - 1 + 3 * PX + CH - 1) / CH;  // chunks per row
  static constexpr int PITCH = NCH * CH;
  static constexpr int SLOT = PY * PITCH;
  static constexpr int LOADS = (PY * NCH + NT - 1) / NT;
  static constexpr int MPITCH = 48, MCH = 3, MSLOT = PY * MPITCH;
  static constexpr int RING = 8, LOOK = 4;  // planes ez+2 .. ez+1+LOOK in flight at layer ez
  static constexpr size_t su = (size_t)RING * SLOT;
  static constexpr size_t sc = 2 * 3 * TY * TX;
  static constexpr size_t bytes = sizeof(float) * (su + sc) + (size_t)RING * MSLOT;
  static_assert(PY * MCH <= NT, "one mask chunk per thread");
  static_assert(LOOK + 3 <= RING, "ring holds planes ez-1 .. ez+1+LOOK");
  static_assert((sizeof(float) * PITCH) % 16 == 0 && (sizeof(float) * SLOT) % 16 == 0, "16-byte destinations");
};

// Coefficients of the element core as packed pairs {k, k}.  A packed multiply-add has
// no scalar-broadcast operand, so a coefficient taken from the parameter bank costs
// two moves at every use; the cube form has eight distinct coefficients, built once
// per thread and kept in registers.  KS_BOX reads K^'s entries at the use.
struct BoxCoef {
  const KHatT<float>& kh;
  __device__ __forceinline__ packed::f32x2 at(int q, int i) const { return packed::f32x2(kh.b[q][i]); }
};
struct CubeCoef {
  // classes 0 / 7: d - e and e of (d - e) I + e 1 1^T; classes 1, 2, 4: diagonal a1 and
  // off-diagonal b1 of the 2 x 2 block; classes 3, 5, 6: a3 of the a 1 1^T block and the
  // mode-7 diagonal c3
  packed::f32x2 d0, e0, d7, e7, a1, b1, a3, c3;
  __device__ __forceinline__ explicit CubeCoef(const KHatT<float>& kh)
      : d0(kh.b[0][0]), e0(kh.b[0][1]), d7(kh.b[7][0]), e7(kh.b[7][1]), a1(kh.b[1][4]), b1(kh.b[1][5]),
        a3(kh.b[3][0]), c3(kh.b[3][8]) {}
};

// Block of parity class Q applied to v (component order), in the structure KS.  For the
// rigid member of classes 1, 2, 4 (mode 0) the output is not formed (left untouched).
template <int KS, int Q, typename CF>
__device__ __forceinline__ void pair_block(const CF& k, const packed::f32x2 (&v)[3], packed::f32x2 (&o)[3]) {
  using P = packed::f32x2;
  constexpr int R = (Q == 1) ? 0 : (Q == 2) ? 1 : (Q == 4) ? 2 : -1;  // rigid member
  constexpr int H = (Q == 6) ? 0 : (Q == 5) ? 1 : (Q == 3) ? 2 : -1;  // member in mode 7
  if constexpr (KS == KS_CUBE) {
    if constexpr (Q == 0 || Q == 7) {
      const P d = (Q == 0) ? k.d0 : k.d7, e = (Q == 0) ? k.e0 : k.e7;
      const P et = e * ((v[0] + v[1]) + v[2]);
#pragma unroll
      for (int c = 0; c < 3; ++c) o[c] = fma(d, v[c], et);
    } else if constexpr (H >= 0) {
      constexpr int I = (H == 0) ? 1 : 0, J = (H == 2) ? 1 : 2;
      const P t = k.a3 * (v[I] + v[J]);
      o[I] = t;
      o[J] = t;
      o[H] = k.c3 * v[H];
    } else {
      constexpr int I = (R == 0) ? 1 : 0, J = (R == 2) ? 1 : 2;
      o[I] = fma(k.b1, v[J], k.a1 * v[I]);
      o[J] = fma(k.b1, v[I], k.a1 * v[J]);
    }
  } else if constexpr (H >= 0) {
    constexpr int I = (H == 0) ? 1 : 0, J = (H == 2) ? 1 : 2;
    o[I] = fma(k.at(Q, 3 * I + J), v[J], k.at(Q, 3 * I + I) * v[I]);
    o[J] = fma(k.at(Q, 3 * J + I), v[I], k.at(Q, 3 * J + J) * v[J]);
    o[H] = k.at(Q, 3 * H + H) * v[H];
  } else {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (c == R) continue;
      bool first = true;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        if (d == R) continue;
        o[c] = first ? k.at(Q, 3 * c + d) * v[d] : fma(k.at(Q, 3 * c + d), v[d], o[c]);
        first = false;
      }
    }
  }
}

// Element core for the class pair (QP, QP + 4): bottom face modes Gs += s (even - odd),
// top face modes Gn = s (even + odd) of the three components' face mode (QP ^ 2^c) & 3.
template <int KS, int QP, typename CF>
__device__ __forceinline__ void pair_classes(const CF& k, packed::f32x2 sv, packed::f32x2 nsv,
                                             const packed::f32x2 (&Fb)[3][4], const packed::f32x2 (&Ft)[3][4],
                                             packed::f32x2 (&Gs)[3][4], packed::f32x2 (&Gn)[3][4]) {
  using P = packed::f32x2;
  // class QP takes the even combination of components 0, 1 and the odd one of 2; class
  // QP + 4 the others.  The even input of a rigid member (mode 0) is not needed.
  P v0[3], v1[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int f = (QP ^ (1 << d)) & 3;
    const bool even_used = (d < 2) ? (QP != (1 << d)) : (QP != 0);
    const P od = Ft[d][f] - Fb[d][f];
    if (d < 2) {
      v1[d] = od;
      if (even_used) v0[d] = Ft[d][f] + Fb[d][f];
    } else {
      v0[d] = od;
      if (even_used) v1[d] = Ft[d][f] + Fb[d][f];
    }
  }
  P o0[3], o1[3];
  pair_block<KS, QP>(k, v0, o0);
  pair_block<KS, QP + 4>(k, v1, o1);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int f = (QP ^ (1 << c)) & 3;
    const bool even_rigid = (c < 2) ? (QP == (1 << c)) : (QP == 0);
    const P oo = (c < 2) ? o1[c] : o0[c];
    if (even_rigid) {
      Gs[c][f] = fma(nsv, oo, Gs[c][f]);
      Gn[c][f] = sv * oo;
    } else {
      const P eo = (c < 2) ? o0[c] : o1[c];
      Gs[c][f] = fma(sv, eo - oo, Gs[c][f]);
      Gn[c][f] = sv * (eo + oo);
    }
  }
}

template <int KS, typename CF>
__device__ __forceinline__ void pair_core(const CF& k, packed::f32x2 sv, const packed::f32x2 (&Fb)[3][4],
                                          const packed::f32x2 (&Ft)[3][4], packed::f32x2 (&Gs)[3][4],
                                          packed::f32x2 (&Gn)[3][4]) {
  const packed::f32x2 nsv = -sv;
  pair_classes<KS, 0>(k, sv, nsv, Fb, Ft, Gs, Gn);
  pair_classes<KS, 1>(k, sv, nsv, Fb, Ft, Gs, Gn);
  pair_classes<KS, 2>(k, sv, nsv, Fb, Ft, Gs, Gn);
  pair_classes<KS, 3>(k, sv, nsv, Fb, Ft, Gs, Gn);
}

template <int TY, bool DOT, bool MASKIN, int MINB, int KS>
__global__ void __launch_bounds__(32 * TY, MINB)
    k_matvec_pair(GridDims g, KHatT<float> kh, const float* __restrict__ s, const uint8_t* __restrict__ mask,
                  const float* __restrict__ u, float* __restrict__ y, int zc, int mode, double* part,
                  unsigned* counter, double* dot_out, const int* stop) {
  if (stop && *stop) return;  // the solver's state is done: an iteration past convergence
  using C = PairTile<TY>;
  using P = packed::f32x2;
  constexpr int TX = C::TX, NT = C::NT, PY = C::PY, CH = C::CH, NCH = C::NCH, PITCH = C::PITCH;
  constexpr int SLOT = C::SLOT, MPITCH = C::MPITCH, MSLOT = C::MSLOT, RING = C::RING, LOOK = C::LOOK;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float* su = reinterpret_cast<float*>(smem_raw);                 // [RING][PY][PITCH]
  float* sc = su + C::su;                                         // [2][3][TY][TX]
  uint8_t* smk = reinterpret_cast<uint8_t*>(sc + C::sc);          // [RING][PY][MPITCH]
  __shared__ double sred[NT / 32];

  const int tid = threadIdx.x;
  const int tx = tid & 31, ty = tid >> 5;
  const int X0 = blockIdx.x * (TX - 1), Y0 = blockIdx.y * (2 * TY - 1);
  const int Z0 = blockIdx.z * zc;
  const int Z1 = min(Z0 + zc, g.sz);
  const int ex = X0 - 1 + tx, eya = Y0 - 1 + 2 * ty, eyb = eya + 1;
  const bool colx = ex >= 0 && ex < g.nx;
  const bool in_a = colx && eya >= 0 && eya < g.ny, in_b = colx && eyb >= 0 && eyb < g.ny;
  using CF = typename std::conditional<KS == KS_CUBE, CubeCoef, BoxCoef>::type;
  const CF coef{kh};
  const bool use_mask = mask != nullptr && (MASKIN || (mode & PYTO_MASK_OUT));
  const bool mask_out = (mode & PYTO_MASK_OUT) && mask != nullptr;
  const int pn = g.sx * g.sy;  // node and DOF ids fit in int32
  const int pe = g.nx * g.ny;
  const int ulen = (int)(3 * g.nnodes);
  const int mlen = (int)((g.nnodes + 3) / 4 * 4);

  // this thread's chunk copies of a plane: float offset of its row's first value in
  // plane 0 (the 16-byte chunk containing the value of plane k starts at
  // ((n3 + 3 pn k) & ~3) + 4 j), shared destination; a chunk outside the grid's rows
  // (or past the tile's rows) is off
  int ld_n3[C::LOADS], ld_j4[C::LOADS], ld_dst[C::LOADS];
  bool ld_on[C::LOADS];
#pragma unroll
  for (int i = 0; i < C::LOADS; ++i) {
    const int q = tid + i * NT;
    const int ly = q / NCH, j = q - ly * NCH;
    const int gy = Y0 - 1 + ly;
    ld_on[i] = q < PY * NCH && gy >= 0 && gy < g.sy;
    ld_n3[i] = 3 * (X0 - 1 + g.sx * gy);
    ld_j4[i] = j * CH;
    ld_dst[i] = (q < PY * NCH) ? ly * PITCH + j * CH : 0;
  }
  const int mly = tid / C::MCH, mj = tid - mly * C::MCH;
  const bool m_thread = use_mask && tid < PY * C::MCH;
  const bool m_on = m_thread && Y0 - 1 + mly >= 0 && Y0 - 1 + mly < g.sy;
  const int m_n0 = X0 - 1 + g.sx * (Y0 - 1 + mly);
  const int m_dst = mly * MPITCH + 16 * mj;

  auto issue_plane = [&](int k) {  // k >= -1
    const int slot = k & (RING - 1);
    const bool kin = k >= 0 && k < g.sz;
    float* d = su + slot * SLOT;
#pragma unroll
    for (int i = 0; i < C::LOADS; ++i) {
      if (C::LOADS * NT == PY * NCH || tid + i * NT < PY * NCH) {
        const int o = ((ld_n3[i] + 3 * pn * k) & ~(CH - 1)) + ld_j4[i];
        int valid = 0;
        if (kin && ld_on[i] && o >= 0) valid = min(16, 4 * (ulen - o));
        cp_async16(d + ld_dst[i], u + (valid > 0 ? o : 0), valid > 0 ? valid : 0);
      }
    }
    if (m_thread) {
      const int o = ((m_n0 + pn * k) & ~15) + 16 * mj;
      int valid = 0;
      if (kin && m_on && o >= 0) valid = min(16, max(0, mlen - o));
      cp_async16(smk + slot * MSLOT + m_dst, mask + (valid > 0 ? o : 0), valid);
    }
    cp_async_commit();
  };

  const int n0l = X0 - 1 + g.sx * (Y0 - 1 + 2 * ty), n0m = n0l + g.sx, n0h = n0m + g.sx;
  // offsets of this thread's first tile node in its three shared-memory rows (the row
  // alignment of plane k shifts by 3 pn k, i.e. by (3 pn k) & 3)
  const int rl = (3 * n0l) & 3, rm = (3 * n0m) & 3, rh = (3 * n0h) & 3;
  const int pshift = (3 * pn) & 3;

  auto face2p = [&](int k, P (&F)[3][4]) {
    const int slot = k & (RING - 1);
    const int sh = pshift * k;
    const float* base = su + slot * SLOT + 3 * tx;
    const float* pl = base + (2 * ty) * PITCH + ((rl + sh) & 3);
    const float* pm = base + (2 * ty + 1) * PITCH + ((rm + sh) & 3);
    const float* ph = base + (2 * ty + 2) * PITCH + ((rh + sh) & 3);
    int ml0 = 0, ml1 = 0, mm0 = 0, mm1 = 0, mh0 = 0, mh1 = 0;
    if (MASKIN) {
      const int pk = pn * k;
      const uint8_t* mb = smk + slot * MSLOT + tx;
      const uint8_t* ql = mb + (2 * ty) * MPITCH + ((n0l + pk) & 15);
      const uint8_t* qm = mb + (2 * ty + 1) * MPITCH + ((n0m + pk) & 15);
      const uint8_t* qh = mb + (2 * ty + 2) * MPITCH + ((n0h + pk) & 15);
      ml0 = ql[0];
      ml1 = ql[1];
      mm0 = qm[0];
      mm1 = qm[1];
      mh0 = qh[0];
      mh1 = qh[1];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float l0 = pl[c], l1 = pl[3 + c], m0 = pm[c], m1 = pm[3 + c], h0 = ph[c], h1 = ph[3 + c];
      if (MASKIN) {
        if ((ml0 >> c) & 1) l0 = 0.0f;
        if ((ml1 >> c) & 1) l1 = 0.0f;
        if ((mm0 >> c) & 1) m0 = 0.0f;
        if ((mm1 >> c) & 1) m1 = 0.0f;
        if ((mh0 >> c) & 1) h0 = 0.0f;
        if ((mh1 >> c) & 1) h1 = 0.0f;
      }
      face_fwd(P(l0, m0), P(l1, m1), P(m0, h0), P(m1, h1), F[c]);
    }
  };

  const bool xown = tx < TX - 1 && (X0 + tx) < g.sx;
  const bool own_m = xown && (Y0 + 2 * ty) < g.sy;
  const bool own_h = xown && ty < TY - 1 && (Y0 + 2 * ty + 1) < g.sy;
  double dot = 0.0;
  float cM[3] = {0.0f, 0.0f, 0.0f}, cH[3] = {0.0f, 0.0f, 0.0f};
  auto out_node = [&](int slot, int row, int nrow, int r0, const float (&v0)[3], const float* add) {
    int mk = 0;
    if (mask_out || MASKIN) mk = smk[slot * MSLOT + row * MPITCH + (nrow & 15) + tx + 1];
    const int dof = 3 * (nrow + 1 + tx);
    const float* ub = su + slot * SLOT + row * PITCH + r0 + 3 * (tx + 1);
    float nd = 0.0f;  // the node's three products u_c y_c, summed in FP32
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float v = add ? v0[c] + add[c * TY * TX] : v0[c];
      if (mask_out && ((mk >> c) & 1)) v = 0.0f;
      y[dof + c] = v;
      if (DOT) {
        float uv = ub[c];
        if (MASKIN && ((mk >> c) & 1)) uv = 0.0f;
        nd = fmaf(uv, v, nd);
      }
    }
    if (DOT) dot += (double)nd;  // node sums accumulated in FP64
  };
  auto output = [&](int k) {
    const int slot = k & (RING - 1);
    const int pk = pn * k;
    const int sh = pshift * k;
    if (own_m) out_node(slot, 2 * ty + 1, n0m + pk, (rm + sh) & 3, cM, nullptr);
    if (own_h)
      out_node(slot, 2 * ty + 2, n0h + pk, (rh + sh) & 3, cH, sc + (k & 1) * (3 * TY * TX) + (ty + 1) * TX + tx);
  };

  int eidx = ex + g.nx * eya + pe * (Z0 - 1);
  float sa_next = (in_a && Z0 - 1 >= 0) ? __ldg(s + eidx) : 0.0f;
  float sb_next = (in_b && Z0 - 1 >= 0) ? __ldg(s + eidx + g.nx) : 0.0f;

#pragma unroll
  for (int k = 0; k < LOOK; ++k) {
    if (Z0 - 1 + k <= Z1) issue_plane(Z0 - 1 + k);
    else cp_async_commit();
  }
  auto layer = [&](int ez, const P (&Fb)[3][4], P (&Ft)[3][4], P (&Gs)[3][4], P (&Gn)[3][4]) {
    cp_async_wait_n<LOOK - 2>();  // plane ez+1 has landed
    __syncthreads();
    if (ez - 1 >= Z0) output(ez - 1);
    if (ez + 1 + LOOK - 1 <= Z1) issue_plane(ez + LOOK);
    else cp_async_commit();
    face2p(ez + 1, Ft);
    const P sv(sa_next, sb_next);  // 0 for an element outside the grid or the slab
    eidx += pe;
    const bool nxt = ez + 1 < Z1 && ez + 1 < g.nz;
    sa_next = (in_a && nxt) ? __ldg(s + eidx) : 0.0f;
    sb_next = (in_b && nxt) ? __ldg(s + eidx + g.nx) : 0.0f;
    pair_core<KS>(coef, sv, Fb, Ft, Gs, Gn);
    if (ez >= Z0) {
      float* scb = sc + (ez & 1) * (3 * TY * TX) + ty * TX + tx;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        P c00, c10, c01, c11;
        face_inv(Gs[c], c00, c10, c01, c11);  // lane x: element a, lane y: element b
        cM[c] = (c11.v.x + c10.v.y) + __shfl_down_sync(0xffffffffu, c01.v.x + c00.v.y, 1);
        cH[c] = c11.v.y + __shfl_down_sync(0xffffffffu, c01.v.y, 1);
        scb[c * TY * TX] = c10.v.x + __shfl_down_sync(0xffffffffu, c00.v.x, 1);
      }
    }
  };
  P FA[3][4], FB[3][4], GA[3][4], GB[3][4];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int f = 0; f < 4; ++f) GA[c][f] = P(0.0f);
  cp_async_wait_n<LOOK - 1>();  // plane Z0-1
  __syncthreads();
  face2p(Z0 - 1, FA);
  for (int ez = Z0 - 1; ez < Z1; ez += 2) {
    layer(ez, FA, FB, GA, GB);
    if (ez + 1 < Z1) layer(ez + 1, FB, FA, GB, GA);
  }
  cp_async_wait_n<0>();
  __syncthreads();
  if (Z1 - 1 >= Z0) output(Z1 - 1);
  if (DOT) {
    dot_finish(block_sum<NT>(dot, sred), part, counter, dot_out);
  }
}

// Structure of K^ for the specialised cores: KS_CUBE, KS_BOX or KS_DENSE (any other Ke).
inline int khat_structure(const KHat& kh) {
  double kmax = 0.0;
  for (int q = 0; q < 8; ++q)
    for (int i = 0; i < 9; ++i) kmax = fmax(kmax, fabs(kh.b[q][i]));
  const double tol = 1e-12 * kmax;
  auto eq = [&](double a, double b) { return fabs(a - b) <= tol; };
  const int hq[3] = {6, 5, 3};  // class whose member c is mode 7
  for (int h = 0; h < 3; ++h) {
    const double* b = kh.b[hq[h]];
    for (int d = 0; d < 3; ++d)
      if (d != h && (fabs(b[3 * h + d]) > tol || fabs(b[3 * d + h]) > tol)) return KS_DENSE;
  }
  bool cube = true;
  for (int q : {0, 7}) {
    const double* b = kh.b[q];
    cube = cube && eq(b[0], b[4]) && eq(b[0], b[8]) && eq(b[1], b[2]) && eq(b[1], b[5]) && eq(b[1], b[3]) &&
           eq(b[1], b[6]) && eq(b[1], b[7]);
  }
  for (int h = 0; h < 3; ++h) {
    const double* b = kh.b[hq[h]];
    const int I = (h == 0) ? 1 : 0, J = (h == 2) ? 1 : 2;
    cube = cube && eq(b[3 * I + I], b[3 * J + J]) && eq(b[3 * I + I], b[3 * I + J]) && eq(b[3 * I + J], b[3 * J + I]);
  }
  // the cube form keeps one (a1, b1) for classes 1, 2, 4 and one (a3, c3) for 3, 5, 6
  const int rq[3] = {1, 2, 4};
  for (int r = 0; r < 3; ++r) {
    const double* b = kh.b[rq[r]];
    const int I = (r == 0) ? 1 : 0, J = (r == 2) ? 1 : 2;
    const double* b1 = kh.b[1];
    cube = cube && eq(b[3 * I + I], b1[4]) && eq(b[3 * J + J], b1[4]) && eq(b[3 * I + J], b1[5]) &&
           eq(b[3 * J + I], b1[5]);
  }
  for (int h = 0; h < 3; ++h) {
    const double* b = kh.b[hq[h]];
    const int I = (h == 0) ? 1 : 0;
    cube = cube && eq(b[3 * I + I], kh.b[3][0]) && eq(b[3 * h + h], kh.b[3][8]);
  }
  return cube ? KS_CUBE : KS_BOX;
}

// FP32 coefficients in the layout pair_block reads (KS_CUBE: classes 0 and 7 hold
// d - e and e in b[0], b[1]).
inline KHatT<float> make_khat_pair(const KHat& kh, int ks) {
  KHatT<float> k = make_khat_t<float>(kh);
  if (ks == KS_CUBE)
    for (int q : {0, 7}) {
      k.b[q][0] = (float)(kh.b[q][0] - kh.b[q][1]);
      k.b[q][1] = (float)kh.b[q][1];
    }
  return k;
}

}  // namespace pyto
