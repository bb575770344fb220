// FP64 operator kernels: BC mask, SIMP scaling, Jacobi data, and the
// matrix-free K(s) u (algorithm notes in matvec.cuh).
#include <algorithm>
#include <atomic>

#include <cuda_bf16.h>

#include "matvec.cuh"

namespace pyto {

// ---------------------------------------------------------------------------
// matrix-free y = K(s) u
//
// Tile kernel (k_matvec).  Node planes stream through a 5-slot shared-memory
// ring (SoA per component) by cp.async, one 4- or 8-byte copy per node value
// (zero-fill outside the grid), with the BC mask staged beside them.  Per
// element layer ez (one barrier):
//   1. wait for plane ez+1, barrier; write the owned nodes of plane ez-1 (their
//      4 column contributions were combined in the previous layer: x by
//      shuffle, y through `sc`);
//   2. issue the copies of plane ez+3;
//   3. element core for layer ez from the face transforms of planes ez and
//      ez+1 (both read from the ring); the bottom-face part plus the pending
//      top-face part of layer ez-1 (in the thread's shared-memory slots `sG`)
//      completes plane ez, which is inverse-transformed and combined across
//      columns for output in the next layer.
// The chunk-staged kernel (matvec_chunked.cuh) keeps this order but copies
// whole rows as 16-byte chunks and holds faces and pending sums in registers.
// ---------------------------------------------------------------------------
template <typename T, int TY, bool TC = false>
struct MvSmem {
  static constexpr int TX = 32, NT = TX * TY, PX = TX + 1, PY = TY + 1, PLANE = PX * PY, RING = 5;
  static constexpr size_t su = RING * 3 * PLANE;  // T
  static constexpr size_t sG = 12 * NT;           // T
  static constexpr size_t sc = 2 * 3 * TY * TX;   // T
  static constexpr size_t base = sizeof(T) * (su + sG + sc) + RING * PLANE + 16;
  // tensor-core element core: A tile [NT rows x 80 bf16], B tile [32 x 80 bf16], both in
  // the K-major no-swizzle core-matrix layout (8 rows x 16 bytes per core matrix),
  // then the mbarrier and the TMEM address
  static constexpr size_t tc_off = (base + 127) / 128 * 128;
  static constexpr size_t tcA = (size_t)NT * 160, tcB = 32 * 160;
  static constexpr size_t bytes = TC ? tc_off + tcA + tcB + 16 : base;
};

// ---------------------------------------------------------------------------
// Tensor-core element core (FP32 operator, BF16 split hi/lo on tcgen05)
//
// Per element layer each thread's element contributes one row of
//   D[e, (c,m)] = sum_(d,n) V_e[(d,n)] K^[(c,m),(d,n)]
// (V_e: the Hadamard corner coefficients of the element's u, 24 values; K^: the
// 24x24 parity-block operator).  With x = hi(x) + lo(x) in BF16,
// A = [V_hi | V_lo | V_hi] (80 columns with zero padding) and B = [K_hi; K_hi; K_lo]
// give D = V_hi K_hi + V_lo K_hi + V_hi K_lo, accumulated in FP32 in TMEM by
// tcgen05.mma (M = 128 rows per MMA, N = 32, K = 5 x 16) issued by one thread; the
// CTA waits on an mbarrier (bounded) and each thread reads its row back with
// tcgen05.ld.  s_e scales the result in FP32.
// ---------------------------------------------------------------------------
__device__ unsigned g_mv_tc_error;  // set when a tensor-core wait gave up (a bug, never expected)

__device__ __forceinline__ uint64_t umma_sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  // start >> 4 (14 bits), leading / stride byte offsets >> 4, descriptor version 1,
  // no swizzle, base offset 0
  return (uint64_t)((addr & 0x3FFFF) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
         ((uint64_t)1 << 46);
}
// kind::f16 instruction descriptor: D FP32, A and B BF16, both K-major, N = 32, M = 128
constexpr uint32_t kUmmaIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);
constexpr uint32_t kUmmaLbo = 128, kUmmaSbo = 1280;  // bytes: next core matrix along K / along rows

// byte offset of (row, 16-byte chunk j) in a core-matrix tile of 80 bf16 columns
__device__ __forceinline__ uint32_t umma_row_off(int row, int j) {
  return (uint32_t)((row >> 3) * kUmmaSbo + j * kUmmaLbo + (row & 7) * 16);
}

__device__ __forceinline__ uint32_t bf2_pack(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}

// bounded wait for the mbarrier phase `ph`; false if the bound was hit
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t mb, uint32_t ph) {
  uint32_t done = 0;
  for (int it = 0; it < (1 << 20) && !done; ++it)
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\tselp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(mb), "r"(ph)
        : "memory");
  return done != 0;
}

// asynchronous global->shared copy of one T (4 or 8 bytes); zero-fill when !valid
template <typename T>
__device__ __forceinline__ void cp_async_t(T* sdst, const T* gsrc, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
  const int n = valid ? (int)sizeof(T) : 0;  // 0: zero-fill, the source is not read
  if (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gsrc), "r"(n) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sa), "l"(gsrc), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

}  // namespace pyto
#include "matvec_chunked.cuh"
#include "matvec_chunked2.cuh"
#include "matvec_pair.cuh"
namespace pyto {

template <typename T, int TY, bool DOT, bool MASKIN, int MINB, bool TC = false>
__global__ void __launch_bounds__(32 * TY, MINB)
    k_matvec(GridDims g, KHat kh, const T* __restrict__ s, const uint8_t* __restrict__ mask,
             const T* __restrict__ u, T* __restrict__ y, int zc, int mode, double* part, unsigned* counter,
             double* dot_out, const int* stop) {
  static_assert(!TC || sizeof(T) == 4, "the tensor-core element core is the FP32 operator's");
  if (stop && *stop) return;  // the solver's state is done: an iteration past convergence
  using M = MvSmem<T, TY, TC>;
  constexpr int TX = M::TX, NT = M::NT, PX = M::PX, PLANE = M::PLANE;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* su = reinterpret_cast<T*>(smem_raw);  // [RING][3][PLANE]
  T* sG = su + M::su;                      // [12][NT] pending top-face accumulators
  T* sc = sG + M::sG;                      // [2][3][TY][TX] y-combine partials
  uint8_t* smk = reinterpret_cast<uint8_t*>(sc + M::sc);  // [RING][PLANE] BC mask
  __shared__ double sred[NT / 32];

  const int tid = threadIdx.x;
  const int tx = tid & 31, ty = tid >> 5;
  const int X0 = blockIdx.x * (TX - 1), Y0 = blockIdx.y * (TY - 1);
  const int Z0 = blockIdx.z * zc;
  const int Z1 = min(Z0 + zc, g.sz);
  const int ex = X0 - 1 + tx, ey = Y0 - 1 + ty;
  const bool col_in = ex >= 0 && ex < g.nx && ey >= 0 && ey < g.ny;
  const bool mask_out = (mode & PYTO_MASK_OUT) && mask != nullptr;
  // node ids and DOF ids fit in int32 (checked by pyto_operator_init)
  const int pn = g.sx * g.sy;  // nodes per plane
  const int pe = g.nx * g.ny;  // elements per layer

  // tensor-core element core: B tile, mbarrier, TMEM (32 columns per 128 rows)
  constexpr int NH = TC ? NT / 128 : 1;
  constexpr uint32_t TCOLS = 32 * NH;
  uint32_t tc_a = 0, tc_b = 0, tc_mb = 0, tc_tm = 0, tc_ph = 0;
  bool tc_fail = false;
  if constexpr (TC) {
    static_assert(NT % 128 == 0, "tensor-core tiles need 128-thread multiples");
    unsigned char* tcp = smem_raw + M::tc_off;
    tc_a = (uint32_t)__cvta_generic_to_shared(tcp);
    tc_b = tc_a + (uint32_t)M::tcA;
    tc_mb = tc_b + (uint32_t)M::tcB;
    uint32_t* tm_slot = reinterpret_cast<uint32_t*>(tcp + M::tcA + M::tcB + 8);
    // B rows n (outputs (c,m) = 8c+m, 24..31 zero), columns k: [K_hi | K_hi | K_lo | 0]
    for (int i = tid; i < 32 * 10; i += NT) {
      const int n = i / 10, j = i % 10;
      float val[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int k = 8 * j + e;
        const int seg = k / 24, kk = k % 24;
        float v = 0.f;
        if (n < 24 && seg < 3) {
          const int c = n >> 3, m = n & 7, d = kk >> 3, nm = kk & 7;
          const int q = m ^ (1 << c);
          if (m != 0 && nm != 0 && (nm ^ (1 << d)) == q) {
            const float kf = (float)kh.b[q][3 * c + d];
            const float hi = __bfloat162float(__float2bfloat16_rn(kf));
            v = (seg < 2) ? hi : kf - hi;
          }
        }
        val[e] = v;
      }
      uint4 w4;
      w4.x = bf2_pack(val[0], val[1]);
      w4.y = bf2_pack(val[2], val[3]);
      w4.z = bf2_pack(val[4], val[5]);
      w4.w = bf2_pack(val[6], val[7]);
      *reinterpret_cast<uint4*>(tcp + M::tcA + umma_row_off(n, j)) = w4;
    }
    if (tid == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_mb));
      asm volatile("fence.mbarrier_init.release.cluster;");
    }
    if (tid < 32) {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                       (uint32_t)__cvta_generic_to_shared(tm_slot)),
                   "r"(TCOLS));
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    tc_tm = *tm_slot;
  }

  // staging slots: node (tx, ty) of the (TX+1) x (TY+1) tile, plus the last
  // tile row / column for the first TX+1+TY threads
  auto plane_off = [&](int lx, int ly) -> int {
    const int gx = X0 - 1 + lx, gy = Y0 - 1 + ly;
    return (gx >= 0 && gx < g.sx && gy >= 0 && gy < g.sy) ? gx + g.sx * gy : -1;
  };
  int lxe = -1, lye = 0;
  if (tid < PX) {
    lxe = tid;
    lye = TY;
  } else if (tid < PX + TY) {
    lxe = TX;
    lye = tid - PX;
  }
  const bool has_e = lxe >= 0;
  const int offm = plane_off(tx, ty);
  const int offe = has_e ? plane_off(lxe, lye) : -1;
  const int sim = ty * PX + tx, sie = lye * PX + (has_e ? lxe : 0);

  // ring slots of planes ez-1 .. ez+3 (r_i holds plane ez-1+i), rotated once per layer
  int r0 = 0, r1 = 1, r2 = 2, r3 = 3, r4 = 4;

  // plane k is issued into the slot held by `slot`; n_off: its first node of the plane
  auto issue_plane = [&](int k, int slot) {
    const bool kin = k >= 0 && k < g.sz;
    T* d = su + slot * (3 * PLANE);
    const int nb = kin ? pn * k : 0;
    {
      const bool v = kin && offm >= 0;
      const T* src = u + 3 * (v ? nb + offm : 0);
#pragma unroll
      for (int c = 0; c < 3; ++c) cp_async_t(d + c * PLANE + sim, src + c, v);
    }
    if (has_e) {
      const bool v = kin && offe >= 0;
      const T* src = u + 3 * (v ? nb + offe : 0);
#pragma unroll
      for (int c = 0; c < 3; ++c) cp_async_t(d + c * PLANE + sie, src + c, v);
    }
    cp_async_commit();
  };
  int mm = 0, me = 0;
  auto load_mask = [&](int k) {
    mm = me = 0;
    if (mask && k >= 0 && k < g.sz) {
      const int nb = pn * k;
      if (offm >= 0) mm = __ldg(mask + nb + offm);
      if (offe >= 0) me = __ldg(mask + nb + offe);
    }
  };
  auto store_mask = [&](int slot) {
    uint8_t* d = smk + slot * PLANE;
    d[sim] = (uint8_t)mm;
    if (has_e) d[sie] = (uint8_t)me;
  };
  auto face = [&](int slot, T (&F)[3][4]) {
    const T* b = su + slot * (3 * PLANE) + sim;
    int m00 = 0, m10 = 0, m01 = 0, m11 = 0;
    if (MASKIN) {
      const uint8_t* mb = smk + slot * PLANE + sim;
      m00 = mb[0];
      m10 = mb[1];
      m01 = mb[PX];
      m11 = mb[PX + 1];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const T* bc = b + c * PLANE;
      T a00 = bc[0], a10 = bc[1], a01 = bc[PX], a11 = bc[PX + 1];
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
  const int li = (ty + 1) * PX + tx + 1;  // owned node in the tile
  double dot = 0.0;
  T cT[3] = {T(0), T(0), T(0)};
  auto output = [&](int k, int slot) {  // owned node of plane k
    if (!owner) return;
    const int mk = mask_out ? (int)smk[slot * PLANE + li] : 0;
    const int dof = 3 * ((X0 + tx) + g.sx * (Y0 + ty) + pn * k);
    const T* scb = sc + (k & 1) * (3 * TY * TX) + (ty + 1) * TX + tx;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      T v = cT[c] + scb[c * TY * TX];
      if ((mk >> c) & 1) v = T(0);
      y[dof + c] = v;
      if (DOT) {
        T uv = su[slot * (3 * PLANE) + c * PLANE + li];
        if (MASKIN && ((smk[slot * PLANE + li] >> c) & 1)) uv = T(0);
        dot = fma((double)uv, (double)v, dot);
      }
    }
  };
  // element index of this column at layer ez, advanced by pe per layer
  int eidx = ex + g.nx * ey + pe * (Z0 - 1);

  // prologue (layer Z0-1 is next): planes Z0-1 -> r1, Z0 -> r2, Z0+1 -> r3 in flight;
  // masks of Z0-1, Z0 staged; mask of Z0+1 in registers (staged in the first layer)
  issue_plane(Z0 - 1, r1);
  issue_plane(Z0, r2);
  load_mask(Z0 - 1);
  store_mask(r1);
  load_mask(Z0);
  store_mask(r2);
  load_mask(Z0 + 1);
  T s_next = (col_in && Z0 - 1 >= 0) ? __ldg(s + eidx) : T(0);
#pragma unroll
  for (int i = 0; i < 12; ++i) sG[i * NT + tid] = T(0);
  if (Z0 + 1 <= Z1) issue_plane(Z0 + 1, r3);
  else cp_async_commit();

  // layer ez: planes ez (slot r1), ez+1 (r2) landed; ez+2 (r3) may be in flight
  for (int ez = Z0 - 1; ez < Z1; ++ez) {
    cp_async_wait1();
    __syncthreads();
    if (ez - 1 >= Z0) output(ez - 1, r0);
    store_mask(r3);  // mask of plane ez+2 (unused for planes beyond Z1)
    load_mask(ez + 3);
    if (ez + 3 <= Z1) issue_plane(ez + 3, r4);
    else cp_async_commit();
    const T se = s_next;
    eidx += pe;
    s_next = (col_in && ez + 1 < Z1 && ez + 1 < g.nz) ? __ldg(s + eidx) : T(0);
    const T sv = (ez >= 0 && ez < g.nz) ? se : T(0);
    T Fb[3][4], Ft[3][4], Gs[3][4];
    face(r1, Fb);
    face(r2, Ft);
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int f = 0; f < 4; ++f) Gs[c][f] = sG[(c * 4 + f) * NT + tid];
    if constexpr (TC) {
      // A row of this thread: [V_hi | V_lo | V_hi | 0], V[(d,n)] = Ft[d][f] +- Fb[d][f], V[(d,0)] = 0
      float V[24];
#pragma unroll
      for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int nm = 0; nm < 8; ++nm) {
          const int f = nm & 3;
          V[8 * d + nm] = (nm == 0) ? 0.f : ((nm & 4) ? (float)(Ft[d][f] - Fb[d][f]) : (float)(Ft[d][f] + Fb[d][f]));
        }
      unsigned char* arow = smem_raw + M::tc_off;
#pragma unroll
      for (int j = 0; j < 10; ++j) {
        float val[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int k = 8 * j + e, seg = k / 24, kk = k % 24;
          float v = 0.f;
          if (seg < 3) {
            const float hi = __bfloat162float(__float2bfloat16_rn(V[kk]));
            v = (seg == 1) ? V[kk] - hi : hi;
          }
          val[e] = v;
        }
        uint4 w4;
        w4.x = bf2_pack(val[0], val[1]);
        w4.y = bf2_pack(val[2], val[3]);
        w4.z = bf2_pack(val[4], val[5]);
        w4.w = bf2_pack(val[6], val[7]);
        *reinterpret_cast<uint4*>(arow + umma_row_off(tid, j)) = w4;
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;");
      __syncthreads();
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
        for (int h = 0; h < NH; ++h)
#pragma unroll
          for (int ks = 0; ks < 5; ++ks) {
            const uint64_t ad = umma_sdesc(tc_a + h * 16 * kUmmaSbo + ks * 2 * kUmmaLbo, kUmmaLbo, kUmmaSbo);
            const uint64_t bd = umma_sdesc(tc_b + ks * 2 * kUmmaLbo, kUmmaLbo, kUmmaSbo);
            const uint32_t acc = ks > 0 ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
                    tc_tm + 32u * h),
                "l"(ad), "l"(bd), "r"(kUmmaIdesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
          }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(tc_mb)
                     : "memory");
      }
      if (!mbar_wait_bounded(tc_mb, tc_ph)) {
        tc_fail = true;
        atomicOr(&g_mv_tc_error, 1u);
      }
      tc_ph ^= 1u;
      asm volatile("tcgen05.fence::after_thread_sync;");
      uint32_t D[32];
      const int wq = tid >> 5;
      const uint32_t la = tc_tm + ((uint32_t)(32 * (wq & 3)) << 16) + 32u * (uint32_t)(wq >> 2);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,"
          "%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(D[0]), "=r"(D[1]), "=r"(D[2]), "=r"(D[3]), "=r"(D[4]), "=r"(D[5]), "=r"(D[6]), "=r"(D[7]),
            "=r"(D[8]), "=r"(D[9]), "=r"(D[10]), "=r"(D[11]), "=r"(D[12]), "=r"(D[13]), "=r"(D[14]), "=r"(D[15]),
            "=r"(D[16]), "=r"(D[17]), "=r"(D[18]), "=r"(D[19]), "=r"(D[20]), "=r"(D[21]), "=r"(D[22]),
            "=r"(D[23]), "=r"(D[24]), "=r"(D[25]), "=r"(D[26]), "=r"(D[27]), "=r"(D[28]), "=r"(D[29]),
            "=r"(D[30]), "=r"(D[31])
          : "r"(la));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;");
      // bottom face gets o(c,f) - o(c,f|4); the top face's pending part is o(c,f) + o(c,f|4)
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          const T o0 = sv * (T)__uint_as_float(D[8 * c + f]), o1 = sv * (T)__uint_as_float(D[8 * c + f + 4]);
          Gs[c][f] += o0 - o1;
          sG[(c * 4 + f) * NT + tid] = o0 + o1;
        }
    } else
    // classes in pairs (qp, qp^4): after a pair, its three top-face entries are final
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
            const T kc = (T)kh.b[q][3 * c + d];
            o = first ? kc * v[d] : fma(kc, v[d], o);
            first = false;
          }
          Gs[c][f] += (m & 4) ? -o : o;
          gt[c] = gt_set[c] ? gt[c] + o : o;
          gt_set[c] = true;
        }
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) sG[(c * 4 + ((qp ^ (1 << c)) & 3)) * NT + tid] = gt_set[c] ? gt[c] : T(0);
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
    const int rt = r0;
    r0 = r1;
    r1 = r2;
    r2 = r3;
    r3 = r4;
    r4 = rt;
  }
  cp_async_wait0();
  __syncthreads();
  if constexpr (TC) {
    if (tc_fail && tid == 0) (void)mbar_wait_bounded(tc_mb, tc_ph ^ 1u);  // let a late MMA finish
    __syncthreads();
    if (tid < 32) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tc_tm), "r"(TCOLS));
  }
  if (Z1 - 1 >= Z0) output(Z1 - 1, r0);
  if (DOT) {
    dot_finish(block_sum<NT>(dot, sred), part, counter, dot_out);
  }
}

// CTAs of `kernel` resident per SM at `threads` threads and `smem` bytes of dynamic
// shared memory (the kernel's attributes already set), times the SM count.
template <typename K>
static int resident_slots(K kernel, int threads, size_t smem) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem) != cudaSuccess || n < 1) n = 1;
  return n * kNumSMs;
}

template <typename T, int TY, bool DOT, bool MI, int MINB, bool TC = false>
static int launch_mv_t(size_t smem, const GridDims& g, const KHat& kh, const T* s, const uint8_t* mask, const T* u,
                       T* y, int mode, double* part, unsigned* counter, double* dot, cudaStream_t st,
                       const int* stop) {
  static PerDevice attr;
  static std::atomic<int> slots{0};
  if (attr.needed()) {
    PYTO_CUDA(cudaFuncSetAttribute(k_matvec<T, TY, DOT, MI, MINB, TC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
    slots.store(resident_slots(k_matvec<T, TY, DOT, MI, MINB, TC>, 32 * TY, smem));
    attr.done();
  }
  const MvLaunch L = matvec_launch<32, TY>(g, slots.load());
  k_matvec<T, TY, DOT, MI, MINB, TC><<<L.grid, 32 * TY, smem, st>>>(g, kh, s, mask, u, y, L.zc, mode, part, counter,
                                                                    dot, stop);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}

template <typename T, int TY, int MINB, bool TC = false>
static int launch_mv(const GridDims& g, const KHat& kh, const T* s, const uint8_t* mask, const T* u, T* y, int mode,
                     double* part, unsigned* counter, double* dot, cudaStream_t st, const int* stop = nullptr) {
  const size_t smem = MvSmem<T, TY, TC>::bytes;
  const bool mi = (mode & PYTO_MASK_IN) && mask != nullptr;
  if (dot)
    return mi ? launch_mv_t<T, TY, true, true, MINB, TC>(smem, g, kh, s, mask, u, y, mode, part, counter, dot, st,
                                                         stop)
              : launch_mv_t<T, TY, true, false, MINB, TC>(smem, g, kh, s, mask, u, y, mode, part, counter, dot,
                                                           st, stop);
  return mi ? launch_mv_t<T, TY, false, true, MINB, TC>(smem, g, kh, s, mask, u, y, mode, nullptr, nullptr,
                                                        nullptr, st, stop)
            : launch_mv_t<T, TY, false, false, MINB, TC>(smem, g, kh, s, mask, u, y, mode, nullptr, nullptr,
                                                         nullptr, st, stop);
}

template <typename T, int TY, bool DOT, bool MI, int MINB, bool GS, bool RF>
static int launch_mvc_t(const GridDims& g, const KHatT<T>& kh, const T* s, const uint8_t* mask, const T* u, T* y,
                        int mode, double* part, unsigned* counter, double* dot, cudaStream_t st, const int* stop) {
  constexpr size_t smem = ChunkTile<T, TY, GS>::bytes;
  static PerDevice attr;
  static std::atomic<int> slots{0};
  if (attr.needed()) {
    PYTO_CUDA(cudaFuncSetAttribute(k_matvec_chunked<T, TY, DOT, MI, MINB, GS, RF>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    slots.store(resident_slots(k_matvec_chunked<T, TY, DOT, MI, MINB, GS, RF>, 32 * TY, smem));
    attr.done();
  }
  const MvLaunch L = matvec_launch<32, TY>(g, slots.load());
  k_matvec_chunked<T, TY, DOT, MI, MINB, GS, RF><<<L.grid, 32 * TY, smem, st>>>(g, kh, s, mask, u, y, L.zc, mode, part,
                                                                        counter, dot, stop);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}

// chunk-staged kernel; u and the mask must be 16-byte aligned, else k_matvec (same results)
template <typename T, int TY, int MINB, bool GS = false, bool RF = false>
static int launch_mvc(const GridDims& g, const KHat& kh, const T* s, const uint8_t* mask, const T* u, T* y, int mode,
                      double* part, unsigned* counter, double* dot, cudaStream_t st, const int* stop) {
  if (((uintptr_t)u & 15) || ((uintptr_t)mask & 15))
    return launch_mv<T, TY, MINB>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
  const KHatT<T> kt = make_khat_t<T>(kh);
  const bool mi = (mode & PYTO_MASK_IN) && mask != nullptr;
  if (dot)
    return mi ? launch_mvc_t<T, TY, true, true, MINB, GS, RF>(g, kt, s, mask, u, y, mode, part, counter, dot, st, stop)
              : launch_mvc_t<T, TY, true, false, MINB, GS, RF>(g, kt, s, mask, u, y, mode, part, counter, dot, st, stop);
  return mi ? launch_mvc_t<T, TY, false, true, MINB, GS, RF>(g, kt, s, mask, u, y, mode, nullptr, nullptr, nullptr,
                                                         st, stop)
            : launch_mvc_t<T, TY, false, false, MINB, GS, RF>(g, kt, s, mask, u, y, mode, nullptr, nullptr, nullptr,
                                                          st, stop);
}

template <typename T, int TY, bool DOT, bool MI, int MINB, bool PACK>
static int launch_mvc2_t(const GridDims& g, const KHatT<T>& kh, const T* s, const uint8_t* mask,
                         const T* u, T* y, int mode, double* part, unsigned* counter, double* dot, cudaStream_t st,
                         const int* stop) {
  constexpr size_t smem = ChunkTile2<T, TY>::bytes;
  static PerDevice attr;
  static std::atomic<int> slots{0};
  if (attr.needed()) {
    PYTO_CUDA(cudaFuncSetAttribute(k_matvec_chunked2<T, TY, DOT, MI, MINB, PACK>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    slots.store(resident_slots(k_matvec_chunked2<T, TY, DOT, MI, MINB, PACK>, 32 * TY, smem));
    attr.done();
  }
  const int bx = (g.sx + 30) / 31, by = (g.sy + 2 * TY - 2) / (2 * TY - 1);
  const int zc = matvec_zc(bx, by, g.sz, slots.load());
  const dim3 grid(bx, by, (g.sz + zc - 1) / zc);
  k_matvec_chunked2<T, TY, DOT, MI, MINB, PACK><<<grid, 32 * TY, smem, st>>>(g, kh, s, mask, u, y, zc, mode, part,
                                                                             counter, dot, stop);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}

// two element rows per thread (PACK: as packed FP32x2 lanes); u and the mask 16-byte
// aligned, else the tile kernel
template <typename T, int TY, int MINB, bool PACK = false>
static int launch_mvc2(const GridDims& g, const KHat& kh, const T* s, const uint8_t* mask, const T* u, T* y, int mode,
                       double* part, unsigned* counter, double* dot, cudaStream_t st, const int* stop) {
  if (((uintptr_t)u & 15) || ((uintptr_t)mask & 15))
    return launch_mv<T, TY, MINB>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
  const KHatT<T> kt = make_khat_t<T>(kh);
  const bool mi = (mode & PYTO_MASK_IN) && mask != nullptr;
  if (dot)
    return mi ? launch_mvc2_t<T, TY, true, true, MINB, PACK>(g, kt, s, mask, u, y, mode, part, counter, dot, st, stop)
              : launch_mvc2_t<T, TY, true, false, MINB, PACK>(g, kt, s, mask, u, y, mode, part, counter, dot, st,
                                                              stop);
  return mi ? launch_mvc2_t<T, TY, false, true, MINB, PACK>(g, kt, s, mask, u, y, mode, nullptr, nullptr, nullptr, st,
                                                            stop)
            : launch_mvc2_t<T, TY, false, false, MINB, PACK>(g, kt, s, mask, u, y, mode, nullptr, nullptr, nullptr,
                                                             st, stop);
}

template <int TY, bool DOT, bool MI, int MINB, int KS>
static int launch_pair_t(const GridDims& g, const KHatT<float>& kh, const float* s, const uint8_t* mask,
                         const float* u, float* y, int mode, double* part, unsigned* counter, double* dot,
                         cudaStream_t st, const int* stop) {
  constexpr size_t smem = PairTile<TY>::bytes;
  static PerDevice attr;
  static std::atomic<int> slots{0};
  if (attr.needed()) {
    PYTO_CUDA(cudaFuncSetAttribute(k_matvec_pair<TY, DOT, MI, MINB, KS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
    slots.store(resident_slots(k_matvec_pair<TY, DOT, MI, MINB, KS>, 32 * TY, smem));
    attr.done();
  }
  const int bx = (g.sx + 30) / 31, by = (g.sy + 2 * TY - 2) / (2 * TY - 1);
  const int zc = matvec_zc(bx, by, g.sz, slots.load());
  const dim3 grid(bx, by, (g.sz + zc - 1) / zc);
  k_matvec_pair<TY, DOT, MI, MINB, KS><<<grid, 32 * TY, smem, st>>>(g, kh, s, mask, u, y, zc, mode, part, counter,
                                                                    dot, stop);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  return PYTO_OK;
}

template <int TY, int MINB, int KS>
static int launch_pair_ks(const GridDims& g, const KHatT<float>& kt, const float* s, const uint8_t* mask,
                          const float* u, float* y, int mode, double* part, unsigned* counter, double* dot,
                          cudaStream_t st, const int* stop) {
  const bool mi = (mode & PYTO_MASK_IN) && mask != nullptr;
  if (dot)
    return mi ? launch_pair_t<TY, true, true, MINB, KS>(g, kt, s, mask, u, y, mode, part, counter, dot, st, stop)
              : launch_pair_t<TY, true, false, MINB, KS>(g, kt, s, mask, u, y, mode, part, counter, dot, st, stop);
  return mi ? launch_pair_t<TY, false, true, MINB, KS>(g, kt, s, mask, u, y, mode, nullptr, nullptr, nullptr, st,
                                                       stop)
            : launch_pair_t<TY, false, false, MINB, KS>(g, kt, s, mask, u, y, mode, nullptr, nullptr, nullptr, st,
                                                        stop);
}

// packed two-row kernel with the element core specialised to K^'s structure; a Ke
// without that structure, or u / the mask not 16-byte aligned: k_matvec_chunked2 /
// the tile kernel
template <int TY, int MINB>
static int launch_pair(const GridDims& g, const KHat& kh, const float* s, const uint8_t* mask, const float* u,
                       float* y, int mode, double* part, unsigned* counter, double* dot, cudaStream_t st,
                       const int* stop) {
  const int ks = khat_structure(kh);
  if (ks == KS_DENSE || ((uintptr_t)u & 15) || ((uintptr_t)mask & 15))
    return launch_mvc2<float, TY, MINB, true>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
  const KHatT<float> kt = make_khat_pair(kh, ks);
  if (ks == KS_CUBE)
    return launch_pair_ks<TY, MINB, KS_CUBE>(g, kt, s, mask, u, y, mode, part, counter, dot, st, stop);
  return launch_pair_ks<TY, MINB, KS_BOX>(g, kt, s, mask, u, y, mode, part, counter, dot, st, stop);
}

// Tile variant of the FP64 matvec (2 = default: fastest measured at 192x96x96):
//   0: 32x8 threads, 2 CTAs/SM (128 registers)   1: 32x8, 1 CTA/SM (no register cap)
//   2: 32x4, 3 CTAs/SM                            3: 32x16, 1 CTA/SM
static int g_mv_variant = 2;
// Tile variant of the FP32 matvec (same numbering; 4 and 5: the tile shapes of 0 and
// 2 with the element core on the tensor cores, BF16 split hi/lo; 8-11: chunk-staged
// kernel; 12-14: chunk-staged with two element rows per thread; 15-17: the same with
// the two rows as packed FP32x2 lanes; 18, 19: packed two-row kernel with the element
// core specialised to K^'s structure, 18 = default: fastest measured at 192x96x96)
static int g_mv32_variant = 18;

int launch_matvec64(const pyto_operator_t* op, const double* s, const uint8_t* mask, const double* u, double* y,
                    int mode, double* part, unsigned* counter, double* dot, cudaStream_t st,
                    const int* stop = nullptr) {
  const GridDims g = make_dims(op);
  const KHat kh = make_khat(op);
  const int tv = (op->tune & 0xff) - 1;  // per-grid choice of the autotuner, else the library default
  switch ((tv >= 0 && tv <= 3) || (tv >= 8 && tv <= 10) ? tv : g_mv_variant) {
    case 8: return launch_mvc<double, 4, 3, true, true>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
    case 9: return launch_mvc<double, 8, 1>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
    case 10: return launch_mvc<double, 4, 2>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
    case 1: return launch_mv<double, 8, 1>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
    case 2: return launch_mv<double, 4, 3>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
    case 3: return launch_mv<double, 16, 1>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
    default: return launch_mv<double, 8, 2>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
  }
}

int launch_matvec32(const pyto_operator_t* op, const float* s, const uint8_t* mask, const float* u, float* y,
                    int mode, double* part, unsigned* counter, double* dot, cudaStream_t st,
                    const int* stop = nullptr) {
  const GridDims g = make_dims(op);
  const KHat kh = make_khat(op);
  const int tv = ((op->tune >> 8) & 0xff) - 1;
  switch ((tv >= 0 && tv <= 5) || (tv >= 8 && tv <= 19) ? tv : g_mv32_variant) {
    case 18: return launch_pair<4, 3>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
    case 19: return launch_pair<8, 1>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
    case 15: return launch_mvc2<float, 8, 2, true>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
    case 16: return launch_mvc2<float, 4, 3, true>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
    case 17: return launch_mvc2<float, 8, 1, true>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
    case 12: return launch_mvc2<float, 8, 2>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
    case 13: return launch_mvc2<float, 4, 3>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
    case 14: return launch_mvc2<float, 8, 1>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
    case 8: return launch_mvc<float, 8, 3>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
    case 9: return launch_mvc<float, 8, 2>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
    case 10: return launch_mvc<float, 4, 6>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
    case 11: return launch_mvc<float, 16, 1>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
    case 1: return launch_mv<float, 8, 1>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
    case 2: return launch_mv<float, 4, 3>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
    case 3: return launch_mv<float, 16, 1>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
    case 4: return launch_mv<float, 8, 2, true>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
    case 5: return launch_mv<float, 4, 3, true>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
    default: return launch_mv<float, 8, 2>(g, kh, s, mask, u, y, mode, part, counter, dot, st, stop);
  }
}

// upper bound of the CTA count of any operator launch (sizes the per-CTA partial sums)
long long matvec_blocks(const pyto_operator_t* op) { return matvec_block_bound(make_dims(op)); }

int set_matvec_variant(int v) {
  if (v < 0 || (v > 3 && v < 8) || v > 10) return PYTO_ERR_ARG;
  g_mv_variant = v;
  return PYTO_OK;
}

int set_matvec32_variant(int v) {
  if (v < 0 || (v > 5 && v < 8) || v > 19) return PYTO_ERR_ARG;
  g_mv32_variant = v;
  return PYTO_OK;
}

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

extern "C" int pyto_tensor_core_status(int reset) {
  unsigned v = 0;
  PYTO_CUDA(cudaMemcpyFromSymbol(&v, g_mv_tc_error, sizeof(v)));
  if (reset) {
    const unsigned z = 0;
    PYTO_CUDA(cudaMemcpyToSymbol(g_mv_tc_error, &z, sizeof(z)));
  }
  return (int)v;
}

extern "C" int pyto_matvec_f32(const pyto_operator_t* op, const float* s, const uint8_t* mask, const float* u,
                               float* y, int mode, double* dot, void* ws, size_t ws_bytes, void* stream) {
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
  return launch_matvec32(op, s, mask, u, y, mode, part, counter, dot, (cudaStream_t)stream);
}
