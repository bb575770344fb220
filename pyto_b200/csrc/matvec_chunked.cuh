// Matrix-free K(s) u, chunk-staged form (included by matvec.cu).
//
// Same decomposition and arithmetic as k_matvec (matvec.cuh): a CTA of 32 x TY
// threads owns 31 x (TY-1) node columns and a slab of node planes; each thread
// marches one element column up z; node sums are formed by exactly one thread
// (x shuffle + y exchange through shared memory), so results are bitwise
// reproducible and equal to k_matvec's.  What changes is the data movement:
//
// * a node plane of the tile (TY+1 rows of 33 nodes) is copied as whole rows of
//   16-byte chunks (`cp.async.cg`, 16-byte aligned global chunks covering the row;
//   the row's first value lands at offset rem = (3 n0) mod (16 / sizeof(T)) of its
//   shared-memory row), one or two chunks per thread instead of three 4- or 8-byte
//   copies per node; the BC mask rows likewise (3 chunks per row);
// * the top face transform of layer ez is kept in registers as the bottom face of
//   layer ez+1 (one face transform per element instead of two);
// * the pending top-face accumulators live in registers;
// * the operator coefficients are passed in T (no per-use conversion).
//
// Chunks may cover nodes left or right of the tile's row (the neighbouring row's
// data) and rows or planes outside the grid are zero-filled; element columns and
// layers outside the grid skip the element core, so such values are never used.
// Requires u and the mask to be 16-byte aligned (the launcher falls back to
// k_matvec otherwise).
#pragma once
#include "matvec.cuh"

namespace pyto {

template <typename T, int TY, bool GS = false>
struct ChunkTile {
  static constexpr int TX = 32, NT = TX * TY, PX = TX + 1, PY = TY + 1;
  static constexpr int CH = 16 / (int)sizeof(T);                   // values per 16-byte chunk
  static constexpr int NCH = (CH - 1 + 3 * PX + CH - 1) / CH;      // chunks per row (rem <= CH-1)
  static constexpr int PITCH = NCH * CH;                           // T per shared-memory row
  static constexpr int SLOT = PY * PITCH;                          // T per plane
  static constexpr int LOADS = (PY * NCH + NT - 1) / NT;           // chunks per thread per plane
  static constexpr int MPITCH = 48;                                // mask bytes per row (rem <= 15)
  static constexpr int MCH = 3;                                    // mask chunks per row
  static constexpr int MSLOT = PY * MPITCH;
  static constexpr int LOOK = 3;                                   // planes loaded ahead of use
  static constexpr int RING = LOOK + 3;                            // planes ez-1 .. ez+1+LOOK
  static constexpr size_t su = (size_t)RING * SLOT;                // T
  static constexpr size_t sc = 2 * 3 * TY * TX;                    // T
  static constexpr size_t sG = GS ? 12 * NT : 0;                   // T
  static constexpr size_t bytes = sizeof(T) * (su + sc + sG) + (size_t)RING * MSLOT;
  static_assert(PY * MCH <= NT, "one mask chunk per thread");
  static_assert((sizeof(T) * PITCH) % 16 == 0 && (sizeof(T) * SLOT) % 16 == 0, "16-byte chunk destinations");
};

template <bool B, typename A>
__device__ __forceinline__ A& pick_ref(A& a, A& b) {
  if constexpr (B) return a;
  else return b;
}

// 16-byte asynchronous copy; bytes past `valid` (0..16) are zero-filled and not read
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc, int valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gsrc), "r"(valid) : "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait_n() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// GS: the pending top-face accumulators live in shared memory (12 values per thread)
// instead of registers, for the FP64 operator whose register state would otherwise
// limit residency.
// RF: the bottom face is transformed again from its shared-memory plane each layer
// instead of being kept in registers (fewer live registers, more shared loads).
template <typename T, int TY, bool DOT, bool MASKIN, int MINB, bool GS = false, bool RF = false>
__global__ void __launch_bounds__(32 * TY, MINB)
    k_matvec_chunked(GridDims g, KHatT<T> kh, const T* __restrict__ s, const uint8_t* __restrict__ mask,
                     const T* __restrict__ u, T* __restrict__ y, int zc, int mode, double* part, unsigned* counter,
                     double* dot_out, const int* stop) {
  if (stop && *stop) return;  // the solver's state is done: an iteration past convergence
  using C = ChunkTile<T, TY, GS>;
  constexpr int TX = C::TX, NT = C::NT, PY = C::PY, CH = C::CH, NCH = C::NCH, PITCH = C::PITCH;
  constexpr int SLOT = C::SLOT, MPITCH = C::MPITCH, MSLOT = C::MSLOT, RING = C::RING, LOOK = C::LOOK;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* su = reinterpret_cast<T*>(smem_raw);                              // [RING][PY][PITCH]
  T* sc = su + C::su;                                                  // [2][3][TY][TX]
  T* sG = sc + C::sc;                                                  // [12][NT] (GS)
  uint8_t* smk = reinterpret_cast<uint8_t*>(sG + C::sG);               // [RING][PY][MPITCH]
  __shared__ double sred[NT / 32];

  const int tid = threadIdx.x;
  const int tx = tid & 31, ty = tid >> 5;
  const int X0 = blockIdx.x * (TX - 1), Y0 = blockIdx.y * (TY - 1);
  const int Z0 = blockIdx.z * zc;
  const int Z1 = min(Z0 + zc, g.sz);
  const int ex = X0 - 1 + tx, ey = Y0 - 1 + ty;
  const bool col_in = ex >= 0 && ex < g.nx && ey >= 0 && ey < g.ny;
  const bool use_mask = mask != nullptr && (MASKIN || (mode & PYTO_MASK_OUT));
  const bool mask_out = (mode & PYTO_MASK_OUT) && mask != nullptr;
  const int pn = g.sx * g.sy;              // nodes per plane (node and DOF ids fit in int32)
  const int pe = g.nx * g.ny;              // elements per layer
  const int ulen = (int)(3 * g.nnodes);    // values of u
  const int mlen = (int)((g.nnodes + 3) / 4 * 4);  // mask bytes (the buffer holds round_up(nnodes, 4))

  // ---- loader: chunk (row ly, chunk j) of each plane; node index of the row's first
  //      tile node in plane 0, and whether the row is inside the grid
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
  const bool m_on = use_mask && tid < PY * C::MCH && Y0 - 1 + mly >= 0 && Y0 - 1 + mly < g.sy;
  const int m_n0 = X0 - 1 + g.sx * (Y0 - 1 + mly);
  const bool m_thread = use_mask && tid < PY * C::MCH;

  auto slot_of = [](int k) { return (int)((unsigned)(k + RING) % (unsigned)RING); };  // k >= -1
  auto issue_plane = [&](int k) {
    const int slot = slot_of(k);
    const bool kin = k >= 0 && k < g.sz;
    const int pk = pn * (kin ? k : 0);
    T* d = su + slot * SLOT;
#pragma unroll
    for (int i = 0; i < C::LOADS; ++i) {
      if (tid + i * NT < PY * NCH) {
        const int f0 = (3 * (ld_n0[i] + pk)) & ~(CH - 1);  // chunk-aligned first value of the row
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

  // node index (plane 0) of the first tile node of this thread's rows ty and ty+1
  const int n0a = X0 - 1 + g.sx * (Y0 - 1 + ty), n0b = n0a + g.sx;

  // face transform of this thread's element column from plane k (corners (tx..tx+1, ty..ty+1))
  auto face = [&](int k, T (&F)[3][4]) {
    const int slot = slot_of(k);
    const int pk = pn * k;
    const int na = n0a + pk, nb = n0b + pk;
    const T* pa = su + slot * SLOT + ty * PITCH + ((3 * na) & (CH - 1)) + 3 * tx;
    const T* pb = su + slot * SLOT + (ty + 1) * PITCH + ((3 * nb) & (CH - 1)) + 3 * tx;
    int m00 = 0, m10 = 0, m01 = 0, m11 = 0;
    if (MASKIN) {
      const uint8_t* ma = smk + slot * MSLOT + ty * MPITCH + (na & 15) + tx;
      const uint8_t* mb = smk + slot * MSLOT + (ty + 1) * MPITCH + (nb & 15) + tx;
      m00 = ma[0];
      m10 = ma[1];
      m01 = mb[0];
      m11 = mb[1];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      T a00 = pa[c], a10 = pa[3 + c], a01 = pb[c], a11 = pb[3 + c];
      if (MASKIN) {
        if ((m00 >> c) & 1) a00 = T(0);
        if ((m10 >> c) & 1) a10 = T(0);
        if ((m01 >> c) & 1) a01 = T(0);
        if ((m11 >> c) & 1) a11 = T(0);
      }
      face_fwd(a00, a10, a01, a11, F[c]);
    }
  };

  const bool owner = tx < TX - 1 && ty < TY - 1 && (X0 + tx) < g.sx && (Y0 + ty) < g.sy;
  double dot = 0.0;
  T cT[3] = {T(0), T(0), T(0)};
  // owned node (tile (tx+1, ty+1)) of plane k: its three sums, BC mask, fused u.y
  auto output = [&](int k) {
    if (!owner) return;
    const int slot = slot_of(k);
    const int nb = n0b + pn * k;
    int mk = 0;
    if (mask_out || MASKIN) mk = smk[slot * MSLOT + (ty + 1) * MPITCH + (nb & 15) + tx + 1];
    const int dof = 3 * (nb + 1 + tx);
    const T* scb = sc + (k & 1) * (3 * TY * TX) + (ty + 1) * TX + tx;
    const T* ub = su + slot * SLOT + (ty + 1) * PITCH + ((3 * nb) & (CH - 1)) + 3 * (tx + 1);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      T v = cT[c] + scb[c * TY * TX];
      if (mask_out && ((mk >> c) & 1)) v = T(0);
      y[dof + c] = v;
      if (DOT) {
        T uv = ub[c];
        if (MASKIN && ((mk >> c) & 1)) uv = T(0);
        dot = fma((double)uv, (double)v, dot);
      }
    }
  };

  // element of this column at layer ez, advanced by pe per layer
  int eidx = ex + g.nx * ey + pe * (Z0 - 1);
  T s_next = (col_in && Z0 - 1 >= 0) ? __ldg(s + eidx) : T(0);

  // prologue: planes Z0-1 .. Z0-2+LOOK in flight; the loop starts with a pre-layer
  // (ez = Z0-2) that only transforms plane Z0-1 into the first bottom face
#pragma unroll
  for (int k = 0; k < LOOK; ++k) {
    if (Z0 - 1 + k <= Z1) issue_plane(Z0 - 1 + k);
    else cp_async_commit();
  }
  // One element layer.  Fb: bottom face (plane ez), read; Ft: top face (plane ez+1),
  // written; Gs: on entry the pending top-face part of layer ez-1, on exit the complete
  // face-mode sums of plane ez; Gn: written, the top-face part of layer ez.  The loop
  // below alternates two register sets between the roles, so nothing is copied.
  auto layer = [&](int ez, const T (&Fkeep)[3][4], T (&Ft)[3][4], T (&Gs)[3][4], T (&Gn)[3][4]) {
    cp_async_wait_n<LOOK - 1>();  // plane ez+1 landed (this thread's chunks)
    __syncthreads();              // ... and everyone's; layer ez-1 finished everywhere
    if (ez - 1 >= Z0) output(ez - 1);
    if (ez + 1 + LOOK <= Z1) issue_plane(ez + 1 + LOOK);
    else cp_async_commit();
    face(ez + 1, Ft);  // columns outside the grid read (unused) neighbouring data
    T Fre[3][4];
    if constexpr (RF) face(ez, Fre);
    const T(&Fb)[3][4] = pick_ref<RF>(static_cast<const T(&)[3][4]>(Fre), Fkeep);
    const T sv = s_next;
    eidx += pe;
    s_next = (col_in && ez + 1 < Z1 && ez + 1 < g.nz) ? __ldg(s + eidx) : T(0);
    if constexpr (GS) {
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int f = 0; f < 4; ++f) Gs[c][f] = sG[(c * 4 + f) * NT + tid];
    }
    if (col_in && ez >= 0 && ez < g.nz) {
      // classes in pairs (qp, qp^4): after a pair its three top-face entries are final
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
              const T kc = kh.b[q][3 * c + d];
              o = first ? kc * v[d] : fma(kc, v[d], o);
              first = false;
            }
            Gs[c][f] += (m & 4) ? -o : o;
            gt[c] = gt_set[c] ? gt[c] + o : o;
            gt_set[c] = true;
          }
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const int f = (qp ^ (1 << c)) & 3;
          if constexpr (GS) sG[(c * 4 + f) * NT + tid] = gt_set[c] ? gt[c] : T(0);
          else Gn[c][f] = gt_set[c] ? gt[c] : T(0);
        }
      }
    } else {
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          if constexpr (GS) sG[(c * 4 + f) * NT + tid] = T(0);
          else Gn[c][f] = T(0);
        }
    }
    if (ez >= Z0) {
      T* scb = sc + (ez & 1) * (3 * TY * TX) + ty * TX + tx;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        T c00, c10, c01, c11;
        face_inv(Gs[c], c00, c10, c01, c11);
        cT[c] = c11 + __shfl_down_sync(0xffffffffu, c01, 1);
        scb[c * TY * TX] = c10 + __shfl_down_sync(0xffffffffu, c00, 1);
      }
    }
  };

  T FA[3][4], FB[3][4], GA[3][4], GB[3][4];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      GA[c][f] = T(0);
      if constexpr (GS) sG[(c * 4 + f) * NT + tid] = T(0);
    }
  // pre-layer: the bottom face of layer Z0-1 from plane Z0-1
  cp_async_wait_n<LOOK - 1>();
  __syncthreads();
  if (Z0 - 1 + LOOK <= Z1) issue_plane(Z0 - 1 + LOOK);
  else cp_async_commit();
  if constexpr (!RF) face(Z0 - 1, FA);
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

}  // namespace pyto
