// Matrix-free K(s) u, chunk-staged with two element rows per thread (included by
// matvec.cu after matvec_chunked.cuh).
//
// As k_matvec_chunked (16-byte chunk staging of node-plane rows, register-resident
// faces and pending sums, two register sets alternating between layers), but each
// thread marches the two y-adjacent element columns (ex, ey) and (ex, ey+1): a CTA of
// 32 x TY threads covers 2 TY element rows and owns 31 x (2 TY - 1) node columns.
// The node row between a thread's two elements is read once and its sums are formed
// in the thread (one x shuffle); only the row between two threads goes through
// shared memory, once per two elements.  The per-layer overhead (chunk copies,
// addressing, the barrier, the s loads) is shared by two elements.  Same arithmetic
// per element as the other kernels, so results agree to rounding.
#pragma once
#include "matvec_chunked.cuh"

namespace pyto {

template <typename T, int TY>
struct ChunkTile2 {
  static constexpr int TX = 32, NT = TX * TY, PX = TX + 1, PY = 2 * TY + 1;
  static constexpr int CH = 16 / (int)sizeof(T);
  static constexpr int NCH = (CH - 1 + 3 * PX + CH - 1) / CH;
  static constexpr int PITCH = NCH * CH;
  static constexpr int SLOT = PY * PITCH;
  static constexpr int LOADS = (PY * NCH + NT - 1) / NT;
  static constexpr int MPITCH = 48, MCH = 3, MSLOT = PY * MPITCH;
  static constexpr int LOOK = 3, RING = LOOK + 3;
  static constexpr size_t su = (size_t)RING * SLOT;  // T
  static constexpr size_t sc = 2 * 3 * TY * TX;      // T: lower rows' partials, per layer parity
  static constexpr size_t bytes = sizeof(T) * (su + sc) + (size_t)RING * MSLOT;
  static_assert(PY * MCH <= NT, "one mask chunk per thread");
  static_assert((sizeof(T) * PITCH) % 16 == 0 && (sizeof(T) * SLOT) % 16 == 0, "16-byte chunk destinations");
};

// Element core in the Hadamard basis (the arithmetic of k_matvec_chunked): adds the
// bottom-face part of s K^ (Fb, Ft) to Gs and writes the top-face part to Gn.
// For packed FP32x2 values T, the FP32 coefficients are broadcast to both lanes.
template <typename T, typename KC>
__device__ __forceinline__ void chunk_elem_core(const KHatT<KC>& kh, T sv, const T (&Fb)[3][4], const T (&Ft)[3][4],
                                                T (&Gs)[3][4], T (&Gn)[3][4]) {
#pragma unroll
  for (int qp = 0; qp < 4; ++qp) {
    T gt[3];
    bool gt_set[3] = {false, false, false};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int q = qp + 4 * h;
      T v[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const int m = member_mode(q, d);
        const int f = m & 3;
        v[d] = (m == 0) ? T(0) : ((m & 4) ? sv * (Ft[d][f] - Fb[d][f]) : sv * (Ft[d][f] + Fb[d][f]));
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int m = member_mode(q, c);
        if (m == 0) continue;
        const int f = m & 3;
        T o = T(0);
        bool first = true;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          if (member_mode(q, d) == 0) continue;
          const T kc = T(kh.b[q][3 * c + d]);
          o = first ? kc * v[d] : fma(kc, v[d], o);
          first = false;
        }
        Gs[c][f] += (m & 4) ? -o : o;
        gt[c] = gt_set[c] ? gt[c] + o : o;
        gt_set[c] = true;
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) Gn[c][(qp ^ (1 << c)) & 3] = gt_set[c] ? gt[c] : T(0);
  }
}

// PACK (FP32 only): the two elements of a thread go through the element core as the
// two lanes of packed FP32x2 values (face transforms, z-combination, block operator,
// accumulation and inverse transforms: one instruction for both).  Elements outside
// the grid have s = 0 and staged values that are finite (zero-filled outside u), so
// the core runs for both lanes and adds exact zeros for a missing element.
template <typename T, int TY, bool DOT, bool MASKIN, int MINB, bool PACK = false>
__global__ void __launch_bounds__(32 * TY, MINB)
    k_matvec_chunked2(GridDims g, KHatT<T> kh, const T* __restrict__ s, const uint8_t* __restrict__ mask,
                      const T* __restrict__ u, T* __restrict__ y, int zc, int mode, double* part, unsigned* counter,
                      double* dot_out, const int* stop) {
  if (stop && *stop) return;  // the solver's state is done: an iteration past convergence
  using C = ChunkTile2<T, TY>;
  constexpr int TX = C::TX, NT = C::NT, PY = C::PY, CH = C::CH, NCH = C::NCH, PITCH = C::PITCH;
  constexpr int SLOT = C::SLOT, MPITCH = C::MPITCH, MSLOT = C::MSLOT, RING = C::RING, LOOK = C::LOOK;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* su = reinterpret_cast<T*>(smem_raw);                 // [RING][PY][PITCH]
  T* sc = su + C::su;                                     // [2][3][TY][TX]
  uint8_t* smk = reinterpret_cast<uint8_t*>(sc + C::sc);  // [RING][PY][MPITCH]
  __shared__ double sred[NT / 32];

  const int tid = threadIdx.x;
  const int tx = tid & 31, ty = tid >> 5;
  const int X0 = blockIdx.x * (TX - 1), Y0 = blockIdx.y * (2 * TY - 1);
  const int Z0 = blockIdx.z * zc;
  const int Z1 = min(Z0 + zc, g.sz);
  const int ex = X0 - 1 + tx, eya = Y0 - 1 + 2 * ty, eyb = eya + 1;
  const bool colx = ex >= 0 && ex < g.nx;
  const bool in_a = colx && eya >= 0 && eya < g.ny, in_b = colx && eyb >= 0 && eyb < g.ny;
  const bool use_mask = mask != nullptr && (MASKIN || (mode & PYTO_MASK_OUT));
  const bool mask_out = (mode & PYTO_MASK_OUT) && mask != nullptr;
  const int pn = g.sx * g.sy;              // node and DOF ids fit in int32
  const int pe = g.nx * g.ny;
  const int ulen = (int)(3 * g.nnodes);
  const int mlen = (int)((g.nnodes + 3) / 4 * 4);

  // loader: chunk (tile row ly, chunk j) of each plane, as in k_matvec_chunked
  int ld_n0[C::LOADS], ld_dst[C::LOADS], ld_jo[C::LOADS];
  bool ld_on[C::LOADS];
#pragma unroll
  for (int i = 0; i < C::LOADS; ++i) {
    const int q = tid + i * NT;
    const int ly = q / NCH, j = q - ly * NCH;
    const int gy = Y0 - 1 + ly;
    ld_on[i] = q < PY * NCH && gy >= 0 && gy < g.sy;
    ld_n0[i] = X0 - 1 + g.sx * gy;
    ld_dst[i] = (q < PY * NCH) ? ly * PITCH + j * CH : 0;
    ld_jo[i] = j * CH;
  }
  const int mly = tid / C::MCH, mj = tid - mly * C::MCH;
  const bool m_thread = use_mask && tid < PY * C::MCH;
  const bool m_on = m_thread && Y0 - 1 + mly >= 0 && Y0 - 1 + mly < g.sy;
  const int m_n0 = X0 - 1 + g.sx * (Y0 - 1 + mly);

  auto slot_of = [](int k) { return (int)((unsigned)(k + RING) % (unsigned)RING); };  // k >= -1
  auto issue_plane = [&](int k) {
    const int slot = slot_of(k);
    const bool kin = k >= 0 && k < g.sz;
    const int pk = pn * (kin ? k : 0);
    T* d = su + slot * SLOT;
#pragma unroll
    for (int i = 0; i < C::LOADS; ++i) {
      if (tid + i * NT < PY * NCH) {
        const int f0 = (3 * (ld_n0[i] + pk)) & ~(CH - 1);
        const int o = f0 + ld_jo[i];
        int valid = 0;
        if (kin && ld_on[i] && o >= 0) valid = (int)sizeof(T) * min(CH, max(0, ulen - o));
        cp_async16(d + ld_dst[i], u + (valid > 0 ? o : 0), valid);
      }
    }
    if (m_thread) {
      const int o = ((m_n0 + pk) & ~15) + 16 * mj;
      int valid = 0;
      if (kin && m_on && o >= 0) valid = min(16, max(0, mlen - o));
      cp_async16(smk + slot * MSLOT + mly * MPITCH + 16 * mj, mask + (valid > 0 ? o : 0), valid);
    }
    cp_async_commit();
  };

  // node index (plane 0) of the first tile node of this thread's tile rows 2ty (low),
  // 2ty+1 (mid) and 2ty+2 (high)
  const int n0l = X0 - 1 + g.sx * (Y0 - 1 + 2 * ty), n0m = n0l + g.sx, n0h = n0m + g.sx;

  // face transforms of the two elements from plane k (element a: rows low/mid,
  // element b: rows mid/high; the mid row is read once)
  auto face2 = [&](int k, T (&Fa)[3][4], T (&Fb)[3][4]) {
    const int slot = slot_of(k);
    const int pk = pn * k;
    const int nl = n0l + pk, nm = n0m + pk, nh = n0h + pk;
    const T* base = su + slot * SLOT + 3 * tx;
    const T* pl = base + (2 * ty) * PITCH + ((3 * nl) & (CH - 1));
    const T* pm = base + (2 * ty + 1) * PITCH + ((3 * nm) & (CH - 1));
    const T* ph = base + (2 * ty + 2) * PITCH + ((3 * nh) & (CH - 1));
    int ml0 = 0, ml1 = 0, mm0 = 0, mm1 = 0, mh0 = 0, mh1 = 0;
    if (MASKIN) {
      const uint8_t* mb = smk + slot * MSLOT + tx;
      const uint8_t* ql = mb + (2 * ty) * MPITCH + (nl & 15);
      const uint8_t* qm = mb + (2 * ty + 1) * MPITCH + (nm & 15);
      const uint8_t* qh = mb + (2 * ty + 2) * MPITCH + (nh & 15);
      ml0 = ql[0];
      ml1 = ql[1];
      mm0 = qm[0];
      mm1 = qm[1];
      mh0 = qh[0];
      mh1 = qh[1];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      T l0 = pl[c], l1 = pl[3 + c], m0 = pm[c], m1 = pm[3 + c], h0 = ph[c], h1 = ph[3 + c];
      if (MASKIN) {
        if ((ml0 >> c) & 1) l0 = T(0);
        if ((ml1 >> c) & 1) l1 = T(0);
        if ((mm0 >> c) & 1) m0 = T(0);
        if ((mm1 >> c) & 1) m1 = T(0);
        if ((mh0 >> c) & 1) h0 = T(0);
        if ((mh1 >> c) & 1) h1 = T(0);
      }
      face_fwd(l0, l1, m0, m1, Fa[c]);
      face_fwd(m0, m1, h0, h1, Fb[c]);
    }
  };

  // owned nodes: tile row 2ty+1 (mid, summed in the thread) and, but for the last
  // thread row, tile row 2ty+2 (high, completed by the next thread row's low partial)
  const bool xown = tx < TX - 1 && (X0 + tx) < g.sx;
  const bool own_m = xown && (Y0 + 2 * ty) < g.sy;
  const bool own_h = xown && ty < TY - 1 && (Y0 + 2 * ty + 1) < g.sy;
  double dot = 0.0;
  T cM[3] = {T(0), T(0), T(0)}, cH[3] = {T(0), T(0), T(0)};
  auto out_node = [&](int slot, int row, int nrow, const T (&v0)[3], const T* add) {
    int mk = 0;
    if (mask_out || MASKIN) mk = smk[slot * MSLOT + row * MPITCH + (nrow & 15) + tx + 1];
    const int dof = 3 * (nrow + 1 + tx);
    const T* ub = su + slot * SLOT + row * PITCH + ((3 * nrow) & (CH - 1)) + 3 * (tx + 1);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      T v = add ? v0[c] + add[c * TY * TX] : v0[c];
      if (mask_out && ((mk >> c) & 1)) v = T(0);
      y[dof + c] = v;
      if (DOT) {
        T uv = ub[c];
        if (MASKIN && ((mk >> c) & 1)) uv = T(0);
        dot = fma((double)uv, (double)v, dot);
      }
    }
  };
  auto output = [&](int k) {
    const int slot = slot_of(k);
    const int pk = pn * k;
    if (own_m) out_node(slot, 2 * ty + 1, n0m + pk, cM, nullptr);
    if (own_h) out_node(slot, 2 * ty + 2, n0h + pk, cH, sc + (k & 1) * (3 * TY * TX) + (ty + 1) * TX + tx);
  };

  // elements of this thread at layer ez (a; b = a + nx), advanced by pe per layer
  int eidx = ex + g.nx * eya + pe * (Z0 - 1);
  T sa_next = (in_a && Z0 - 1 >= 0) ? __ldg(s + eidx) : T(0);
  T sb_next = (in_b && Z0 - 1 >= 0) ? __ldg(s + eidx + g.nx) : T(0);

#pragma unroll
  for (int k = 0; k < LOOK; ++k) {
    if (Z0 - 1 + k <= Z1) issue_plane(Z0 - 1 + k);
    else cp_async_commit();
  }
  if constexpr (PACK) {
    static_assert(sizeof(T) == 4, "packed form is FP32");
    using P = packed::f32x2;
    // face transforms of both elements from plane k as lane pairs (a, b)
    auto face2p = [&](int k, P (&F)[3][4]) {
      const int slot = slot_of(k);
      const int pk = pn * k;
      const int nl = n0l + pk, nm = n0m + pk, nh = n0h + pk;
      const T* base = su + slot * SLOT + 3 * tx;
      const T* pl = base + (2 * ty) * PITCH + ((3 * nl) & (CH - 1));
      const T* pm = base + (2 * ty + 1) * PITCH + ((3 * nm) & (CH - 1));
      const T* ph = base + (2 * ty + 2) * PITCH + ((3 * nh) & (CH - 1));
      int ml0 = 0, ml1 = 0, mm0 = 0, mm1 = 0, mh0 = 0, mh1 = 0;
      if (MASKIN) {
        const uint8_t* mb = smk + slot * MSLOT + tx;
        const uint8_t* ql = mb + (2 * ty) * MPITCH + (nl & 15);
        const uint8_t* qm = mb + (2 * ty + 1) * MPITCH + (nm & 15);
        const uint8_t* qh = mb + (2 * ty + 2) * MPITCH + (nh & 15);
        ml0 = ql[0];
        ml1 = ql[1];
        mm0 = qm[0];
        mm1 = qm[1];
        mh0 = qh[0];
        mh1 = qh[1];
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        T l0 = pl[c], l1 = pl[3 + c], m0 = pm[c], m1 = pm[3 + c], h0 = ph[c], h1 = ph[3 + c];
        if (MASKIN) {
          if ((ml0 >> c) & 1) l0 = T(0);
          if ((ml1 >> c) & 1) l1 = T(0);
          if ((mm0 >> c) & 1) m0 = T(0);
          if ((mm1 >> c) & 1) m1 = T(0);
          if ((mh0 >> c) & 1) h0 = T(0);
          if ((mh1 >> c) & 1) h1 = T(0);
        }
        face_fwd(P(l0, m0), P(l1, m1), P(m0, h0), P(m1, h1), F[c]);
      }
    };
    auto layerp = [&](int ez, const P (&Fb)[3][4], P (&Ft)[3][4], P (&Gs)[3][4], P (&Gn)[3][4]) {
      cp_async_wait_n<LOOK - 1>();
      __syncthreads();
      if (ez - 1 >= Z0) output(ez - 1);
      if (ez + 1 + LOOK <= Z1) issue_plane(ez + 1 + LOOK);
      else cp_async_commit();
      face2p(ez + 1, Ft);
      const P sv(sa_next, sb_next);  // 0 for an element outside the grid or the slab
      eidx += pe;
      const bool nxt = ez + 1 < Z1 && ez + 1 < g.nz;
      sa_next = (in_a && nxt) ? __ldg(s + eidx) : T(0);
      sb_next = (in_b && nxt) ? __ldg(s + eidx + g.nx) : T(0);
      chunk_elem_core<P>(kh, sv, Fb, Ft, Gs, Gn);
      if (ez >= Z0) {
        T* scb = sc + (ez & 1) * (3 * TY * TX) + ty * TX + tx;
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
    cp_async_wait_n<LOOK - 1>();
    __syncthreads();
    if (Z0 - 1 + LOOK <= Z1) issue_plane(Z0 - 1 + LOOK);
    else cp_async_commit();
    face2p(Z0 - 1, FA);
    for (int ez = Z0 - 1; ez < Z1; ez += 2) {
      layerp(ez, FA, FB, GA, GB);
      if (ez + 1 < Z1) layerp(ez + 1, FB, FA, GB, GA);
    }
  } else {
    // One element layer for both elements (see k_matvec_chunked for the roles of the
    // register sets; here each role holds the two elements' arrays)
    auto layer = [&](int ez, const T (&Fba)[3][4], const T (&Fbb)[3][4], T (&Fta)[3][4], T (&Ftb)[3][4],
                     T (&Gsa)[3][4], T (&Gsb)[3][4], T (&Gna)[3][4], T (&Gnb)[3][4]) {
      cp_async_wait_n<LOOK - 1>();
      __syncthreads();
      if (ez - 1 >= Z0) output(ez - 1);
      if (ez + 1 + LOOK <= Z1) issue_plane(ez + 1 + LOOK);
      else cp_async_commit();
      face2(ez + 1, Fta, Ftb);
      const T sva = sa_next, svb = sb_next;
      eidx += pe;
      const bool nxt = ez + 1 < Z1 && ez + 1 < g.nz;
      sa_next = (in_a && nxt) ? __ldg(s + eidx) : T(0);
      sb_next = (in_b && nxt) ? __ldg(s + eidx + g.nx) : T(0);
      const bool lay = ez >= 0 && ez < g.nz;
      if (in_a && lay) {
        chunk_elem_core<T>(kh, sva, Fba, Fta, Gsa, Gna);
      } else {
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int f = 0; f < 4; ++f) Gna[c][f] = T(0);
      }
      if (in_b && lay) {
        chunk_elem_core<T>(kh, svb, Fbb, Ftb, Gsb, Gnb);
      } else {
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int f = 0; f < 4; ++f) Gnb[c][f] = T(0);
      }
      if (ez >= Z0) {
        T* scb = sc + (ez & 1) * (3 * TY * TX) + ty * TX + tx;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          T a00, a10, a01, a11, b00, b10, b01, b11;
          face_inv(Gsa[c], a00, a10, a01, a11);
          face_inv(Gsb[c], b00, b10, b01, b11);
          cM[c] = (a11 + b10) + __shfl_down_sync(0xffffffffu, a01 + b00, 1);  // mid row, in the thread
          cH[c] = b11 + __shfl_down_sync(0xffffffffu, b01, 1);                // high row, this thread's part
          scb[c * TY * TX] = a10 + __shfl_down_sync(0xffffffffu, a00, 1);     // low row: the row below's high
        }
      }
    };

    T FAa[3][4], FAb[3][4], FBa[3][4], FBb[3][4], GAa[3][4], GAb[3][4], GBa[3][4], GBb[3][4];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int f = 0; f < 4; ++f) GAa[c][f] = GAb[c][f] = T(0);
    cp_async_wait_n<LOOK - 1>();
    __syncthreads();
    if (Z0 - 1 + LOOK <= Z1) issue_plane(Z0 - 1 + LOOK);
    else cp_async_commit();
    face2(Z0 - 1, FAa, FAb);
    for (int ez = Z0 - 1; ez < Z1; ez += 2) {
      layer(ez, FAa, FAb, FBa, FBb, GAa, GAb, GBa, GBb);
      if (ez + 1 < Z1) layer(ez + 1, FBa, FBb, FAa, FAb, GBa, GBb, GAa, GAb);
    }
  }
  cp_async_wait_n<0>();
  __syncthreads();
  if (Z1 - 1 >= Z0) output(Z1 - 1);
  if (DOT) {
    dot_finish(block_sum<NT>(dot, sred), part, counter, dot_out);
  }
}

}  // namespace pyto
