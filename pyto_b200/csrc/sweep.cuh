// Blocked Gauss-Jordan sweep of a symmetric matrix held in its lower 64 x 64 tiles
// (the diagonal tiles in full), as device functions of one 256-thread CTA; used by the
// dense coarse inverse (deflation.cu) and by the frontal matrices of the
// nested-dissection coarse solver (coarse_nd.cu).  After sweeping pivot blocks K:
//   P = A_KK^-1, U = P A_K:, A_ij -= A_iK U_Kj, A_Kj = U_Kj, A_iK = U_Ki^T, A_KK = -P,
// so sweeping all pivots leaves -A^-1, and sweeping the leading pivots s of
// [[A_ss, A_sb], [A_bs, A_bb]] leaves -A_ss^-1, A_bs A_ss^-1 and the Schur complement
// A_bb - A_bs A_ss^-1 A_sb.
#pragma once
#include <algorithm>

#include "common.cuh"

namespace pyto {

constexpr int kSweepB = 64;

// Element k of a 4-vector held in registers, by selects (a dynamic index would put
// the array in local memory).
__device__ __forceinline__ double pick4(double v0, double v1, double v2, double v3, int k) {
  double r = v0;
  r = (k == 1) ? v1 : r;
  r = (k == 2) ? v2 : r;
  r = (k == 3) ? v3 : r;
  return r;
}

// In-place sweep of the symmetric 64 x 64 block held by 256 threads (thread (ty, tx)
// owns rows ty + 16a, columns tx + 16b), leaving -M^-1 (pivot by pivot:
//   M_pp -> -1/M_pp,  M_pj -> M_pj/M_pp,  M_ip -> M_ip/M_pp,  M_ij -= M_ip M_pj / M_pp).
// Padding pivots (identity rows/columns beyond bk) are decoupled, so they are swept with
// the rest.  Blocked by 16: for each 16-pivot block K, one warp sweeps the 16 x 16
// diagonal block in registers (lane 2r + h holds row r, columns 8h..8h+7; the pivot row
// and column arrive by shuffles, so the 16 pivots cost no CTA barrier), then all threads
// apply the block step (U = P M_K: with P = M_KK^-1; M_ij -= M_iK U_Kj; M_Kj = U_Kj,
// M_iK = U_Ki, M_KK = -P), four barriers per block.  M stays symmetric throughout, so
// the column panel M_:K is read as the row panel M_K:.  sm: >= kSweepPivotSmem doubles.
constexpr int kSweepPivotSmem = 2 * 16 * 64 + 16 * 16;
__device__ __forceinline__ void sweep_pivot_blocked(double (&R)[4][4], double* sm) {
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double* sRow = sm;            // [16][64]: M_K: before the block step
  double* sU = sm + 16 * 64;    // [16][64]: U = P M_K:
  double* sP = sm + 2 * 16 * 64;  // [16][16]: P = M_KK^-1
#pragma unroll 1
  for (int K = 0; K < 4; ++K) {
#pragma unroll
    for (int b = 0; b < 4; ++b) sRow[ty * 64 + tx + 16 * b] = pick4(R[0][b], R[1][b], R[2][b], R[3][b], K);
    __syncthreads();
    if (threadIdx.x < 32) {  // warp 0: Gauss-Jordan sweep of M_KK in registers
      const int l = threadIdx.x, r = l >> 1, h = l & 1;
      double X[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) X[k] = sRow[r * 64 + 16 * K + 8 * h + k];
#pragma unroll
      for (int p = 0; p < 16; ++p) {
        const double mpp = __shfl_sync(0xffffffffu, X[p & 7], 2 * p + (p >> 3));
        const double ip = 1.0 / mpp;
        double rowv[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) rowv[k] = __shfl_sync(0xffffffffu, X[k], 2 * p + h);
        const double colv = __shfl_sync(0xffffffffu, X[p & 7], 2 * r + (p >> 3));
        const double f = -colv * ip;
#pragma unroll
        for (int k = 0; k < 8; ++k) X[k] = fma(f, rowv[k], X[k]);
        if (r == p) {
#pragma unroll
          for (int k = 0; k < 8; ++k) X[k] = rowv[k] * ip;
        }
        if ((p >> 3) == h) X[p & 7] = (r == p) ? -ip : colv * ip;
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) sP[r * 16 + 8 * h + k] = -X[k];
    }
    __syncthreads();
    // U_Kj = sum_k P[ty][k] M_K:[k][j] for the thread's columns j = tx + 16b
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      double u0 = 0.0, u1 = 0.0;  // two chains of 8
#pragma unroll
      for (int k = 0; k < 16; k += 2) {
        u0 = fma(sP[ty * 16 + k], sRow[k * 64 + tx + 16 * b], u0);
        u1 = fma(sP[ty * 16 + k + 1], sRow[(k + 1) * 64 + tx + 16 * b], u1);
      }
      sU[ty * 64 + tx + 16 * b] = u0 + u1;
    }
    __syncthreads();
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int i = ty + 16 * a, j = tx + 16 * b;
        if (a == K && b == K) {
          R[a][b] = -sP[ty * 16 + tx];
        } else if (a == K) {
          R[a][b] = sU[ty * 64 + j];
        } else if (b == K) {
          R[a][b] = sU[tx * 64 + i];
        } else {
          double t0 = 0.0, t1 = 0.0;  // two chains of 8
#pragma unroll
          for (int k = 0; k < 16; k += 2) {
            t0 = fma(sRow[k * 64 + i], sU[k * 64 + j], t0);
            t1 = fma(sRow[(k + 1) * 64 + i], sU[(k + 1) * 64 + j], t1);
          }
          R[a][b] -= t0 + t1;
        }
      }
    __syncthreads();
  }
}

// P = A_KK^-1 of the pivot block at k0 (bk <= 64 pivots; identity padding), by 256 threads
__device__ __forceinline__ void sweep_pivot_block(long long n, int k0, int bk, const double* __restrict__ A,
                                                  double* __restrict__ P) {
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double R[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int i = ty + 16 * a, j = tx + 16 * b;
      R[a][b] = (i < bk && j < bk) ? A[(k0 + i) * n + (k0 + j)] : (i == j ? 1.0 : 0.0);
    }
  __shared__ double sm[kSweepPivotSmem];
  sweep_pivot_blocked(R, sm);
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) P[(ty + 16 * a) * kSweepB + tx + 16 * b] = -R[a][b];  // P = A_KK^-1
}

// Rp = A_K: (copy), U = P Rp for the 16 columns from j0.  Only the lower tiles (and the
// full diagonal tiles) of A are current, so row K right of the pivot block is read from
// column K below it.
__device__ __forceinline__ void sweep_panel_cols(long long n, int k0, int bk, const double* __restrict__ A,
                                                 const double* __restrict__ P, double* __restrict__ Rp,
                                                 double* __restrict__ U, long long j0) {
  __shared__ double sP[kSweepB][kSweepB];
  __shared__ double sR[kSweepB][17];
  // 256 threads: every load of P and of the 16 columns issued before the first store
  double vp[kSweepB * kSweepB / 256], vr[kSweepB * 16 / 256];
#pragma unroll
  for (int r = 0; r < kSweepB * kSweepB / 256; ++r) vp[r] = P[threadIdx.x + 256 * r];
#pragma unroll
  for (int r = 0; r < kSweepB * 16 / 256; ++r) {
    const int t = threadIdx.x + 256 * r, i = t / 16, jj = t % 16;
    const long long j = j0 + jj;
    vr[r] = (i < bk && j < n) ? ((j < k0 + kSweepB) ? A[(k0 + i) * n + j] : A[j * n + (k0 + i)]) : 0.0;
  }
#pragma unroll
  for (int r = 0; r < kSweepB * kSweepB / 256; ++r) {
    const int t = threadIdx.x + 256 * r;
    sP[t / kSweepB][t % kSweepB] = vp[r];
  }
#pragma unroll
  for (int r = 0; r < kSweepB * 16 / 256; ++r) {
    const int t = threadIdx.x + 256 * r, i = t / 16, jj = t % 16;
    const long long j = j0 + jj;
    sR[i][jj] = vr[r];
    if (i < bk && j < n) Rp[i * n + j] = vr[r];
  }
  __syncthreads();
  for (int t = threadIdx.x; t < kSweepB * 16; t += blockDim.x) {
    const int i = t / 16, jj = t % 16;
    const long long j = j0 + jj;
    if (i >= bk || j >= n) continue;
    double acc = 0.0;
    for (int k = 0; k < bk; ++k) acc = fma(sP[i][k], sR[k][jj], acc);
    U[i * n + j] = acc;
  }
}

// Dynamic shared memory of sweep_update_tile: the tile rows' A_iK and the tile columns'
// U_Kj for all bk <= 64 pivots (2 x 64 x 64 doubles).
constexpr int kSweepP = 68;  // operand row pitch: the tensor-core fragment loads are free of bank conflicts
constexpr size_t kSweepTileSmem = 2 * 64 * kSweepP * sizeof(double);

// acc[i][j] = sum_k L[k][i] U[k][j] over the 64 x 64 tile (k < kmax, a multiple of 4;
// L, U: k-major in shared memory, pitch kSweepP) on the FP64 tensor cores: warp w owns
// rows 8w..8w+7, eight m8n8k4 products per 4 k; lane (g = lane / 4, t = lane % 4) holds
// A[g][t] = L[k + t][8w + g], B[t][g] = U[k + t][8c + g] and C[g][2t], C[g][2t + 1].
// The 8 x 64 result rows are written to S (pitch 65) for the caller's own layout.
__device__ __forceinline__ void sweep_tile_mma(const double* L, const double* U, int kmax, double* S) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  double c[8][2];
#pragma unroll
  for (int q = 0; q < 8; ++q) c[q][0] = c[q][1] = 0.0;
#pragma unroll 2
  for (int k = 0; k < kmax; k += 4) {
    const double a = L[(k + t) * kSweepP + 8 * w + g];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const double b = U[(k + t) * kSweepP + 8 * q + g];
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                   : "+d"(c[q][0]), "+d"(c[q][1])
                   : "d"(a), "d"(b));
    }
  }
  __syncthreads();  // L and U consumed: S may overlay them
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    S[(8 * w + g) * 65 + 8 * q + 2 * t] = c[q][0];
    S[(8 * w + g) * 65 + 8 * q + 2 * t + 1] = c[q][1];
  }
  __syncthreads();
}

// Update of the lower 64 x 64 tile (ti, tj) by 256 threads x (4 x 4) outputs for the
// pivot block at k0 (tiles in row or column K take U / -P); k1 >= 0 and (ti, tj) =
// (k1, k1) / 64: then sweep that tile as the next pivot block into Pn (bk1 pivots).
// Every global load of the tile (its A entries, the bk rows of A_iK and U_Kj) is issued
// before the first is used, then staged in shared memory (kSweepTileSmem, dynamic).
__device__ __forceinline__ void sweep_update_tile(long long n, int k0, int bk, double* __restrict__ A,
                                                  const double* __restrict__ P, const double* __restrict__ Rp,
                                                  const double* __restrict__ U, long long ti, long long tj, int k1,
                                                  double* __restrict__ Pn, int bk1) {
  extern __shared__ double sw_dyn[];
  double* sL = sw_dyn;                 // [64][kSweepP]: A_iK for the tile rows (Rp[k][i0 + c])
  double* sU = sw_dyn + 64 * kSweepP;  // [64][kSweepP]: U_Kj for the tile columns
  const long long i0 = ti * 64, j0 = tj * 64;
  const bool rowK = (i0 == k0), colK = (j0 == k0);
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  // a full pivot block: row / column K tiles are U / -P throughout.  A partial one (bk <
  // 64: the last pivots of a partial sweep) leaves non-pivot rows and columns in those
  // tiles, which take the rank-bk update below like any other tile.
  if ((rowK || colK) && bk == kSweepB) {
    for (int t = threadIdx.x; t < 64 * 64; t += blockDim.x) {
      const int ii = t / 64, jj = t % 64;
      const long long i = i0 + ii, j = j0 + jj;
      if (i >= n || j >= n) continue;
      double v;
      if (rowK && colK) v = (ii < bk && jj < bk) ? -P[ii * kSweepB + jj] : A[i * n + j];
      else if (rowK) v = (ii < bk) ? U[ii * n + j] : A[i * n + j];
      else v = (jj < bk) ? U[jj * n + i] : A[i * n + j];
      A[i * n + j] = v;
    }
    return;
  }
  // the tile's own entries and the operand rows, all loads in flight together
  double a_in[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const long long i = i0 + ty + 16 * a, j = j0 + tx + 16 * b;
      a_in[a][b] = (i < n && j < n) ? A[i * n + j] : 0.0;
    }
  constexpr int PER = 64 * 64 / 256;  // operand entries per thread and operand
#pragma unroll
  for (int r = 0; r < PER; ++r) {  // 8-byte asynchronous copies (zero-filled outside)
    const int t = threadIdx.x + 256 * r, k = t / 64, c = t % 64;
    const bool okl = k < bk && i0 + c < n, oku = k < bk && j0 + c < n;
    const unsigned dl = (unsigned)__cvta_generic_to_shared(sL + k * kSweepP + c),
                   du = (unsigned)__cvta_generic_to_shared(sU + k * kSweepP + c);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dl),
                 "l"(okl ? Rp + k * n + i0 + c : Rp), "r"(okl ? 8 : 0) : "memory");
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(du),
                 "l"(oku ? U + k * n + j0 + c : U), "r"(oku ? 8 : 0) : "memory");
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncthreads();
  // the rank-bk product on the tensor cores (operand rows >= bk are zero), then each
  // thread takes its 4 x 4 outputs (rows ty + 16a, columns tx + 16b)
  sweep_tile_mma(sL, sU, (bk + 3) & ~3, sw_dyn);
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = sw_dyn[(ty + 16 * a) * 65 + tx + 16 * b];
  const bool pivot_next = k1 >= 0 && i0 == k1 && j0 == k1;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int ii = ty + 16 * a, jj = tx + 16 * b;
      const long long i = i0 + ii, j = j0 + jj;
      if (i < n && j < n) {
        const bool pi = rowK && ii < bk, pj = colK && jj < bk;  // pivot row / column
        double v;
        if (pi && pj) v = -P[ii * kSweepB + jj];
        else if (pi) v = U[ii * n + j];
        else if (pj) v = U[jj * n + i];
        else v = a_in[a][b] - acc[a][b];
        A[i * n + j] = v;
        acc[a][b] = v;
      }
    }
  if (!pivot_next) return;
  // the next pivot block, as k_sweep_pivot would load it (identity padding)
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int i = ty + 16 * a, j = tx + 16 * b;
      if (!(i < bk1 && j < bk1)) acc[a][b] = (i == j) ? 1.0 : 0.0;
    }
  __syncthreads();
  sweep_pivot_blocked(acc, sw_dyn);  // the operand rows are consumed
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) Pn[(ty + 16 * a) * kSweepB + tx + 16 * b] = -acc[a][b];
}


}  // namespace pyto
