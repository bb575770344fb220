// MMA update of the density-based optimiser on the device: one subproblem of
// the method of moving asymptotes (K. Svanberg's 2007 formulation, which the
// third-party mmasub that src/mmaWrapper.py:91-94 calls implements), m <= 4
// constraints, n design variables.
//
//   mmasub:  moving asymptotes low/upp (asyinit 0.5, asyincr 1.2, asydecr 0.7,
//            clamped to [0.01, 10] (xmax - xmin) from x), bounds alfa/beta (albefa
//            0.1, move), the convex approximation p0, q0, P, Q (raa0 1e-5) and b;
//   subsolv: the primal-dual interior-point Newton method for the subproblem,
//            epsi = 1, 0.1, ..., down to 1e-7; per Newton step the (m+1)
//            system in (dlam, dz), the step to the boundary (factor 1.01), and
//            backtracking (halving, at most 50) until the residual norm drops;
//            at most 200 Newton steps per epsi.
//
// All of it runs in one cooperative kernel: each pass over the n variables
// deposits per-block partial sums, a grid barrier, and then every block sums the
// partials in the same fixed order and takes the same decisions on its own copy
// of the m-sized dual variables, so no host round trip and a deterministic
// result.  Partials are double-buffered by pass parity (as in the OC update).
#include <cooperative_groups.h>

#include <algorithm>

#include "common.cuh"

namespace cg = cooperative_groups;

namespace pyto {

constexpr int kMmaThreads = 256;
constexpr int kMmaMaxM = 4;
constexpr int kMmaSlots = 20;  // partial values per block and pass

struct MmaP {
  long long n;
  int m, iter;
  double a0, a[kMmaMaxM], c[kMmaMaxM], d[kMmaMaxM], fval[kMmaMaxM];
  double move, xmin_s, xmax_s;
};

struct MmaArrays {
  double *x, *low, *upp;                 // in/out
  const double *xold1, *xold2, *xmin, *xmax, *df0dx, *dfdx;
  double *alfa, *beta, *p0, *q0, *P, *Q;  // [n], P and Q [m][n]
  double *xsi, *eta, *xo, *xsio, *etao;   // [n]
  double* part;                           // [2][nblocks][kMmaSlots]
  double* dual;                           // out: y[m], z, lam[m], mu[m], zet, s[m], epsi, iterations
};

// Dual (m-sized) state, replicated in every block
struct MmaDual {
  double y[kMmaMaxM], z, lam[kMmaMaxM], mu[kMmaMaxM], zet, s[kMmaMaxM];
};

// Block reduction of K values held by every thread (sums), deposited as partials
template <int K>
__device__ __forceinline__ void block_deposit(double (&v)[K], double* sred, double* out) {
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const double t = block_sum<kMmaThreads>(v[k], sred);
    if (threadIdx.x == 0) out[k] = t;
  }
}

// Fixed-order sum of the partials of slot k over all blocks (every thread of
// every block gets the same bits)
__device__ __forceinline__ double gather_sum(const double* pp, int nb, int k) {
  double t = 0.0;
  for (int b = 0; b < nb; ++b) t += __ldcg(pp + (size_t)b * kMmaSlots + k);
  return t;
}
__device__ __forceinline__ double gather_max(const double* pp, int nb, int k) {
  double t = -1e308;
  for (int b = 0; b < nb; ++b) t = fmax(t, __ldcg(pp + (size_t)b * kMmaSlots + k));
  return t;
}

// Newton direction of variable i at state (x, xsi, eta) for the dual step
// (dlam): dx, dxsi, deta.  Also returns delx, diagx and GG (for pass A).
struct Dir {
  double dx, dxsi, deta;
};

__device__ __forceinline__ void elem_terms(const MmaP& P, const MmaArrays& A, long long i, double x,
                                           const MmaDual& D, double epsi, double& plam, double& qlam,
                                           double& ux1, double& xl1, double (&GG)[kMmaMaxM], double& delx,
                                           double& diagx, double xsi, double eta) {
  const double lo = A.low[i], up = A.upp[i], al = A.alfa[i], be = A.beta[i];
  ux1 = up - x;
  xl1 = x - lo;
  const double ux2 = ux1 * ux1, xl2 = xl1 * xl1, ux3 = ux1 * ux2, xl3 = xl1 * xl2;
  plam = A.p0[i];
  qlam = A.q0[i];
  for (int j = 0; j < P.m; ++j) {
    const double pj = A.P[(size_t)j * P.n + i], qj = A.Q[(size_t)j * P.n + i];
    plam = fma(pj, D.lam[j], plam);
    qlam = fma(qj, D.lam[j], qlam);
    GG[j] = pj / ux2 - qj / xl2;
  }
  const double dpsidx = plam / ux2 - qlam / xl2;
  delx = dpsidx - epsi / (x - al) + epsi / (be - x);
  diagx = 2.0 * (plam / ux3 + qlam / xl3) + xsi / (x - al) + eta / (be - x);
}

__global__ void __launch_bounds__(kMmaThreads) k_mma(MmaP P, MmaArrays A) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double sred[kMmaThreads / 32];
  const int nb = gridDim.x;
  const long long n = P.n;
  const int m = P.m;
  const long long i0 = blockIdx.x * (long long)blockDim.x + threadIdx.x, istep = (long long)gridDim.x * blockDim.x;
  int pass = 0;
  auto slot = [&](int p) { return A.part + (size_t)(p & 1) * nb * kMmaSlots; };

  // ---- mmasub: asymptotes, bounds, approximation; subsolv start point ----
  {
    double bacc[kMmaMaxM] = {0, 0, 0, 0};
    for (long long i = i0; i < n; i += istep) {
      const double xv = A.x[i];
      const double xmn = A.xmin ? A.xmin[i] : P.xmin_s, xmx = A.xmax ? A.xmax[i] : P.xmax_s;
      const double span = xmx - xmn;
      double lo, up;
      if (P.iter <= 2) {
        lo = xv - 0.5 * span;
        up = xv + 0.5 * span;
      } else {
        const double x1 = A.xold1[i], x2 = A.xold2[i];
        const double zzz = (xv - x1) * (x1 - x2);
        const double f = zzz > 0.0 ? 1.2 : (zzz < 0.0 ? 0.7 : 1.0);
        lo = xv - f * (x1 - A.low[i]);
        up = xv + f * (A.upp[i] - x1);
        lo = fmin(fmax(lo, xv - 10.0 * span), xv - 0.01 * span);
        up = fmax(fmin(up, xv + 10.0 * span), xv + 0.01 * span);
      }
      const double al = fmax(fmax(lo + 0.1 * (xv - lo), xv - P.move * span), xmn);
      const double be = fmin(fmin(up - 0.1 * (up - xv), xv + P.move * span), xmx);
      const double xmamiinv = 1.0 / fmax(span, 1e-5);
      const double ux1 = up - xv, xl1 = xv - lo, ux2 = ux1 * ux1, xl2 = xl1 * xl1;
      const double g0 = A.df0dx[i];
      double p0 = fmax(g0, 0.0), q0 = fmax(-g0, 0.0);
      const double pq0 = 0.001 * (p0 + q0) + 1e-5 * xmamiinv;
      A.p0[i] = (p0 + pq0) * ux2;
      A.q0[i] = (q0 + pq0) * xl2;
      for (int j = 0; j < m; ++j) {
        const double gj = A.dfdx[(size_t)j * n + i];
        double pj = fmax(gj, 0.0), qj = fmax(-gj, 0.0);
        const double pq = 0.001 * (pj + qj) + 1e-5 * xmamiinv;
        pj = (pj + pq) * ux2;
        qj = (qj + pq) * xl2;
        A.P[(size_t)j * n + i] = pj;
        A.Q[(size_t)j * n + i] = qj;
        bacc[j] += pj / ux1 + qj / xl1;
      }
      A.low[i] = lo;
      A.upp[i] = up;
      A.alfa[i] = al;
      A.beta[i] = be;
      const double xs = 0.5 * (al + be);
      A.x[i] = xs;
      A.xsi[i] = fmax(1.0 / (xs - al), 1.0);
      A.eta[i] = fmax(1.0 / (be - xs), 1.0);
    }
    block_deposit<kMmaMaxM>(bacc, sred, slot(pass) + (size_t)blockIdx.x * kMmaSlots);
  }
  grid.sync();
  double b[kMmaMaxM];
  for (int j = 0; j < m; ++j) b[j] = gather_sum(slot(pass), nb, j) - P.fval[j];
  ++pass;

  MmaDual D;
  for (int j = 0; j < m; ++j) {
    D.y[j] = 1.0;
    D.lam[j] = 1.0;
    D.mu[j] = fmax(1.0, 0.5 * P.c[j]);
    D.s[j] = 1.0;
  }
  D.z = 1.0;
  D.zet = 1.0;

  // residual of the subproblem at the current state: (norm, max |.|); one pass
  auto residual = [&](double epsi, double& rnorm, double& rmax) {
    double v[2 + kMmaMaxM] = {0, 0, 0, 0, 0, 0};
    double vmax = 0.0;
    for (long long i = i0; i < n; i += istep) {
      const double x = A.x[i], xsi = A.xsi[i], eta = A.eta[i];
      const double ux1 = A.upp[i] - x, xl1 = x - A.low[i];
      double plam = A.p0[i], qlam = A.q0[i];
      for (int j = 0; j < m; ++j) {
        const double pj = A.P[(size_t)j * n + i], qj = A.Q[(size_t)j * n + i];
        plam = fma(pj, D.lam[j], plam);
        qlam = fma(qj, D.lam[j], qlam);
        v[2 + j] += pj / ux1 + qj / xl1;
      }
      const double rex = plam / (ux1 * ux1) - qlam / (xl1 * xl1) - xsi + eta;
      const double rexsi = xsi * (x - A.alfa[i]) - epsi, reeta = eta * (A.beta[i] - x) - epsi;
      v[0] += rex * rex + rexsi * rexsi + reeta * reeta;
      vmax = fmax(vmax, fmax(fabs(rex), fmax(fabs(rexsi), fabs(reeta))));
    }
    double* pp = slot(pass);
    block_deposit<2 + kMmaMaxM>(v, sred, pp + (size_t)blockIdx.x * kMmaSlots);
    const double bm = block_max<kMmaThreads>(vmax, sred);
    if (threadIdx.x == 0) pp[(size_t)blockIdx.x * kMmaSlots + 1] = bm;
    grid.sync();
    double ss = gather_sum(pp, nb, 0), mx = gather_max(pp, nb, 1);
    double alam = 0.0;
    for (int j = 0; j < m; ++j) alam += P.a[j] * D.lam[j];
    for (int j = 0; j < m; ++j) {
      const double gv = gather_sum(pp, nb, 2 + j);
      const double rey = P.c[j] + P.d[j] * D.y[j] - D.mu[j] - D.lam[j];
      const double relam = gv - P.a[j] * D.z - D.y[j] + D.s[j] - b[j];
      const double remu = D.mu[j] * D.y[j] - epsi, res = D.lam[j] * D.s[j] - epsi;
      ss += rey * rey + relam * relam + remu * remu + res * res;
      mx = fmax(mx, fmax(fmax(fabs(rey), fabs(relam)), fmax(fabs(remu), fabs(res))));
    }
    const double rez = P.a0 - D.zet - alam, rezet = D.zet * D.z - epsi;
    ss += rez * rez + rezet * rezet;
    mx = fmax(mx, fmax(fabs(rez), fabs(rezet)));
    rnorm = sqrt(ss);
    rmax = mx;
    ++pass;
  };

  int newton = 0;
  double epsi = 1.0;
  while (epsi > 1e-7) {
    double rnorm, rmax;
    residual(epsi, rnorm, rmax);
    int ittt = 0;
    while (rmax > 0.9 * epsi && ittt < 200) {
      ++ittt;
      ++newton;
      // pass A: gvec, Alam = GG diag(1/diagx) GG^T, GG (delx / diagx); keep the old state
      {
        double v[kMmaSlots];
        for (int k = 0; k < kMmaSlots; ++k) v[k] = 0.0;
        for (long long i = i0; i < n; i += istep) {
          const double x = A.x[i], xsi = A.xsi[i], eta = A.eta[i];
          A.xo[i] = x;
          A.xsio[i] = xsi;
          A.etao[i] = eta;
          double plam, qlam, ux1, xl1, GG[kMmaMaxM], delx, diagx;
          elem_terms(P, A, i, x, D, epsi, plam, qlam, ux1, xl1, GG, delx, diagx, xsi, eta);
          const double idx = 1.0 / diagx;
          int k = 2 * m;
          for (int j = 0; j < m; ++j) {
            v[j] += A.P[(size_t)j * n + i] / ux1 + A.Q[(size_t)j * n + i] / xl1;
            v[m + j] += GG[j] * delx * idx;
            for (int l = j; l < m; ++l) v[k++] += GG[j] * GG[l] * idx;
          }
        }
        double* pp = slot(pass);
        for (int k = 0; k < kMmaSlots; ++k) {
          const double t = block_sum<kMmaThreads>(v[k], sred);
          if (threadIdx.x == 0) pp[(size_t)blockIdx.x * kMmaSlots + k] = t;
        }
      }
      grid.sync();
      // the (m+1) system in every block (same partials, same order, same bits)
      double dlam[kMmaMaxM], dz;
      {
        const double* pp = slot(pass);
        double gvec[kMmaMaxM], gd[kMmaMaxM], AA[kMmaMaxM + 1][kMmaMaxM + 2];
        int k = 2 * m;
        for (int j = 0; j < m; ++j) {
          gvec[j] = gather_sum(pp, nb, j);
          gd[j] = gather_sum(pp, nb, m + j);
        }
        for (int j = 0; j < m; ++j)
          for (int l = j; l < m; ++l) {
            const double t = gather_sum(pp, nb, k++);
            AA[j][l] = t;
            AA[l][j] = t;
          }
        double alam = 0.0;
        for (int j = 0; j < m; ++j) alam += P.a[j] * D.lam[j];
        const double delz = P.a0 - alam - epsi / D.z;
        for (int j = 0; j < m; ++j) {
          const double dely = P.c[j] + P.d[j] * D.y[j] - D.lam[j] - epsi / D.y[j];
          const double dellam = gvec[j] - P.a[j] * D.z - D.y[j] - b[j] + epsi / D.lam[j];
          const double diagy = P.d[j] + D.mu[j] / D.y[j];
          AA[j][j] += D.s[j] / D.lam[j] + 1.0 / diagy;
          AA[j][m] = P.a[j];
          AA[m][j] = P.a[j];
          AA[j][m + 1] = dellam + dely / diagy - gd[j];
        }
        AA[m][m] = -D.zet / D.z;
        AA[m][m + 1] = delz;
        // Gaussian elimination with partial pivoting on the (m+1) x (m+2) augmented matrix
        const int M1 = m + 1;
        for (int c = 0; c < M1; ++c) {
          int piv = c;
          for (int r = c + 1; r < M1; ++r)
            if (fabs(AA[r][c]) > fabs(AA[piv][c])) piv = r;
          if (piv != c)
            for (int q = 0; q <= M1; ++q) {
              const double t = AA[c][q];
              AA[c][q] = AA[piv][q];
              AA[piv][q] = t;
            }
          for (int r = c + 1; r < M1; ++r) {
            const double f = AA[r][c] / AA[c][c];
            for (int q = c; q <= M1; ++q) AA[r][q] -= f * AA[c][q];
          }
        }
        double sol[kMmaMaxM + 1];
        for (int r = M1 - 1; r >= 0; --r) {
          double t = AA[r][M1];
          for (int q = r + 1; q < M1; ++q) t -= AA[r][q] * sol[q];
          sol[r] = t / AA[r][r];
        }
        for (int j = 0; j < m; ++j) dlam[j] = sol[j];
        dz = sol[m];
      }
      ++pass;
      // dual directions and the step to the boundary of the dual scalars
      double dy[kMmaMaxM], dmu[kMmaMaxM], ds[kMmaMaxM], dzet;
      double stm = 1.0;
      for (int j = 0; j < m; ++j) {
        const double dely = P.c[j] + P.d[j] * D.y[j] - D.lam[j] - epsi / D.y[j];
        const double diagy = P.d[j] + D.mu[j] / D.y[j];
        dy[j] = -dely / diagy + dlam[j] / diagy;
        dmu[j] = -D.mu[j] + epsi / D.y[j] - (D.mu[j] * dy[j]) / D.y[j];
        ds[j] = -D.s[j] + epsi / D.lam[j] - (D.s[j] * dlam[j]) / D.lam[j];
        stm = fmax(stm, fmax(fmax(-1.01 * dy[j] / D.y[j], -1.01 * dlam[j] / D.lam[j]),
                             fmax(-1.01 * dmu[j] / D.mu[j], -1.01 * ds[j] / D.s[j])));
      }
      dzet = -D.zet + epsi / D.z - D.zet * dz / D.z;
      stm = fmax(stm, fmax(-1.01 * dz / D.z, -1.01 * dzet / D.zet));
      // pass B: primal directions and their step to the boundary
      auto direction = [&](long long i, double x, double xsi, double eta, Dir& r) {
        double plam, qlam, ux1, xl1, GG[kMmaMaxM], delx, diagx;
        elem_terms(P, A, i, x, D, epsi, plam, qlam, ux1, xl1, GG, delx, diagx, xsi, eta);
        double gd = 0.0;
        for (int j = 0; j < m; ++j) gd += GG[j] * dlam[j];
        r.dx = -delx / diagx - gd / diagx;
        const double xa = x - A.alfa[i], bx = A.beta[i] - x;
        r.dxsi = -xsi + epsi / xa - (xsi * r.dx) / xa;
        r.deta = -eta + epsi / bx + (eta * r.dx) / bx;
      };
      {
        double st = 0.0;
        for (long long i = i0; i < n; i += istep) {
          const double x = A.xo[i], xsi = A.xsio[i], eta = A.etao[i];
          Dir r;
          direction(i, x, xsi, eta, r);
          st = fmax(st, fmax(fmax(-1.01 * r.dx / (x - A.alfa[i]), 1.01 * r.dx / (A.beta[i] - x)),
                             fmax(-1.01 * r.dxsi / xsi, -1.01 * r.deta / eta)));
        }
        const double bm = block_max<kMmaThreads>(st, sred);
        if (threadIdx.x == 0) slot(pass)[(size_t)blockIdx.x * kMmaSlots] = bm;
      }
      grid.sync();
      stm = fmax(stm, gather_max(slot(pass), nb, 0));
      ++pass;
      double steg = 1.0 / stm;
      const MmaDual Dold = D;
      // backtracking on the residual norm
      int itto = 0;
      double resinew = 2.0 * rnorm, rmaxnew = rmax;
      while (resinew > rnorm && itto < 50) {
        ++itto;
        for (int j = 0; j < m; ++j) {
          D.y[j] = Dold.y[j] + steg * dy[j];
          D.lam[j] = Dold.lam[j] + steg * dlam[j];
          D.mu[j] = Dold.mu[j] + steg * dmu[j];
          D.s[j] = Dold.s[j] + steg * ds[j];
        }
        D.z = Dold.z + steg * dz;
        D.zet = Dold.zet + steg * dzet;
        // the directions use the old dual state
        const MmaDual Dnew = D;
        D = Dold;
        for (long long i = i0; i < n; i += istep) {
          const double x = A.xo[i], xsi = A.xsio[i], eta = A.etao[i];
          Dir r;
          direction(i, x, xsi, eta, r);
          A.x[i] = x + steg * r.dx;
          A.xsi[i] = xsi + steg * r.dxsi;
          A.eta[i] = eta + steg * r.deta;
        }
        D = Dnew;
        // (the residual pass reads the new x, xsi, eta of this thread's own entries;
        // the barrier inside it orders the writes of all threads before the sums)
        residual(epsi, resinew, rmaxnew);
        steg *= 0.5;
      }
      rnorm = resinew;
      rmax = rmaxnew;
    }
    epsi *= 0.1;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double* o = A.dual;
    for (int j = 0; j < m; ++j) {
      o[j] = D.y[j];
      o[1 + m + j] = D.lam[j];
      o[1 + 2 * m + j] = D.mu[j];
      o[2 + 3 * m + j] = D.s[j];
    }
    o[m] = D.z;
    o[1 + 3 * m] = D.zet;
    o[2 + 4 * m] = (double)newton;
  }
}

// KKT residual of the original problem at (x, duals) with the new gradients
// (kktcheck): sum of squares and max |.| of the n-sized part -> out[0], out[1]
__global__ void __launch_bounds__(256) k_mma_kkt(long long n, int m, const double* __restrict__ x,
                                                 const double* __restrict__ xsi, const double* __restrict__ eta,
                                                 const double* __restrict__ xmin, const double* __restrict__ xmax,
                                                 double xmin_s, double xmax_s, const double* __restrict__ df0dx,
                                                 const double* __restrict__ dfdx, const double* __restrict__ dual,
                                                 double* part, unsigned* counter, double* out) {
  __shared__ double sred[8];
  double ss = 0.0, mx = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double rex = df0dx[i] - xsi[i] + eta[i];
    for (int j = 0; j < m; ++j) rex = fma(dfdx[(size_t)j * n + i], dual[1 + m + j], rex);
    const double rxsi = xsi[i] * (x[i] - (xmin ? xmin[i] : xmin_s));
    const double reta = eta[i] * ((xmax ? xmax[i] : xmax_s) - x[i]);
    ss += rex * rex + rxsi * rxsi + reta * reta;
    mx = fmax(mx, fmax(fabs(rex), fmax(fabs(rxsi), fabs(reta))));
  }
  double v[1] = {block_sum<256>(ss, sred)};
  const double bm = block_max<256>(mx, sred);
  grid_reduce<1>(v, part, counter, gridDim.x, [&](const double* tot) { out[0] = tot[0]; });
  (void)bm;
  if (threadIdx.x == 0) atomicMax(reinterpret_cast<unsigned long long*>(out + 1), __double_as_longlong(bm));
}

int mma_grid_blocks() {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mma, kMmaThreads, 0) != cudaSuccess) return 0;
  int dev = 0, sms = kNumSMs;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  return std::max(1, std::min(per_sm, 2)) * sms;
}

// the partials buffer is carved for the largest grid either kernel launches, so that
// every array after it sits at the same offset for pyto_mma_update and pyto_mma_kkt
constexpr int kMmaCarveBlocks = 4 * kNumSMs;

struct MmaWs {
  double *alfa, *beta, *p0, *q0, *P, *Q, *xsi, *eta, *xo, *xsio, *etao, *part, *dual, *kpart;
  unsigned* counter;
};

static MmaWs carve_mma(long long n, int m, void* ws, size_t bytes, size_t* need) {
  Carver cv{(char*)ws, 0, bytes};
  MmaWs W;
  W.counter = cv.take<unsigned>(64);
  W.dual = cv.take<double>(32);
  W.part = cv.take<double>(2 * (size_t)kMmaCarveBlocks * kMmaSlots);
  W.kpart = cv.take<double>(4 * (size_t)kNumSMs);
  W.alfa = cv.take<double>(n);
  W.beta = cv.take<double>(n);
  W.p0 = cv.take<double>(n);
  W.q0 = cv.take<double>(n);
  W.P = cv.take<double>((size_t)m * n);
  W.Q = cv.take<double>((size_t)m * n);
  W.xsi = cv.take<double>(n);
  W.eta = cv.take<double>(n);
  W.xo = cv.take<double>(n);
  W.xsio = cv.take<double>(n);
  W.etao = cv.take<double>(n);
  *need = cv.off + 256;
  return W;
}

}  // namespace pyto

using namespace pyto;

extern "C" size_t pyto_mma_workspace_bytes(int64_t n, int m) {
  if (n <= 0 || m < 1 || m > kMmaMaxM) return 0;
  size_t need = 0;
  carve_mma(n, m, nullptr, 0, &need);
  return need;
}

extern "C" int pyto_mma_update(int64_t n, int m, int iter, double* x, const double* xold1, const double* xold2,
                               const double* xmin, const double* xmax, double xmin_s, double xmax_s,
                               const double* df0dx, const double* fval, const double* dfdx, double* low, double* upp,
                               double a0, const double* a, const double* c, const double* d, double move,
                               double* dual_out, void* ws, size_t ws_bytes, void* stream) {
  if (n <= 0 || m < 1 || m > kMmaMaxM || iter < 1 || !x || !df0dx || !fval || !dfdx || !low || !upp || !a ||
      !c || !d || !(move > 0))
    return PYTO_ERR_ARG;
  if (iter > 2 && (!xold1 || !xold2)) return PYTO_ERR_ARG;
  int nb = mma_grid_blocks();
  if (nb <= 0) return PYTO_ERR_CUDA;
  nb = (int)std::min<long long>(std::min(nb, kMmaCarveBlocks), std::max<long long>(1, (n + kMmaThreads - 1) / kMmaThreads));
  size_t need = 0;
  MmaWs W = carve_mma(n, m, ws, ws_bytes, &need);
  if (!ws || ws_bytes < need) return PYTO_ERR_WORKSPACE;
  MmaP P{};
  P.n = n;
  P.m = m;
  P.iter = iter;
  P.a0 = a0;
  for (int j = 0; j < m; ++j) {
    P.a[j] = a[j];
    P.c[j] = c[j];
    P.d[j] = d[j];
    P.fval[j] = fval[j];
  }
  P.move = move;
  P.xmin_s = xmin_s;
  P.xmax_s = xmax_s;
  MmaArrays A{};
  A.x = x;
  A.low = low;
  A.upp = upp;
  A.xold1 = xold1;
  A.xold2 = xold2;
  A.xmin = xmin;
  A.xmax = xmax;
  A.df0dx = df0dx;
  A.dfdx = dfdx;
  A.alfa = W.alfa;
  A.beta = W.beta;
  A.p0 = W.p0;
  A.q0 = W.q0;
  A.P = W.P;
  A.Q = W.Q;
  A.xsi = W.xsi;
  A.eta = W.eta;
  A.xo = W.xo;
  A.xsio = W.xsio;
  A.etao = W.etao;
  A.part = W.part;
  A.dual = W.dual;
  void* args[] = {&P, &A};
  cudaStream_t st = (cudaStream_t)stream;
  PYTO_CUDA(cudaLaunchCooperativeKernel((const void*)k_mma, dim3(nb), dim3(kMmaThreads), args, 0, st));
  PYTO_COUNT(1);
  if (dual_out) PYTO_CUDA(cudaMemcpyAsync(dual_out, W.dual, sizeof(double) * (3 + 4 * m), cudaMemcpyDeviceToDevice, st));
  return PYTO_OK;
}

extern "C" int pyto_mma_kkt(int64_t n, int m, const double* x, const double* xmin, const double* xmax,
                            double xmin_s, double xmax_s, const double* df0dx, const double* fval,
                            const double* dfdx, double a0, const double* a, const double* c, const double* d,
                            double* kkt_out, void* ws, size_t ws_bytes, void* stream) {
  if (n <= 0 || m < 1 || m > kMmaMaxM || !x || !df0dx || !fval || !dfdx || !a || !c || !d || !kkt_out)
    return PYTO_ERR_ARG;
  size_t need = 0;
  MmaWs W = carve_mma(n, m, ws, ws_bytes, &need);
  if (!ws || ws_bytes < need) return PYTO_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  double host_dual[3 + 4 * kMmaMaxM];
  PYTO_CUDA(cudaMemcpyAsync(host_dual, W.dual, sizeof(double) * (3 + 4 * m), cudaMemcpyDeviceToHost, st));
  PYTO_CUDA(cudaMemsetAsync(W.counter, 0, 64 * sizeof(unsigned), st));
  PYTO_CUDA(cudaMemsetAsync(W.kpart, 0, 4 * kNumSMs * sizeof(double), st));
  double* dev_out = W.kpart + 2 * kNumSMs;  // [0]: sum of squares, [1]: max (as ordered bits, >= 0)
  const int nb = (int)std::min<long long>((n + 255) / 256, kNumSMs);
  k_mma_kkt<<<nb, 256, 0, st>>>(n, m, x, W.xsi, W.eta, xmin, xmax, xmin_s, xmax_s, df0dx, dfdx, W.dual, W.kpart,
                                W.counter, dev_out);
  PYTO_COUNT(1);
  PYTO_LAUNCH_CHECK();
  double dev_res[2];
  PYTO_CUDA(cudaMemcpyAsync(dev_res, dev_out, sizeof(dev_res), cudaMemcpyDeviceToHost, st));
  PYTO_CUDA(cudaStreamSynchronize(st));
  // the m-sized part of the KKT residual on the host
  double ss = dev_res[0], mx = dev_res[1];
  const double* y = host_dual;
  const double z = host_dual[m], *lam = host_dual + 1 + m, *mu = host_dual + 1 + 2 * m, zet = host_dual[1 + 3 * m];
  const double* s = host_dual + 2 + 3 * m;
  double alam = 0.0;
  for (int j = 0; j < m; ++j) alam += a[j] * lam[j];
  for (int j = 0; j < m; ++j) {
    const double r1 = c[j] + d[j] * y[j] - mu[j] - lam[j], r2 = fval[j] - a[j] * z - y[j] + s[j];
    const double r3 = mu[j] * y[j], r4 = lam[j] * s[j];
    ss += r1 * r1 + r2 * r2 + r3 * r3 + r4 * r4;
    mx = std::max(mx, std::max(std::max(fabs(r1), fabs(r2)), std::max(fabs(r3), fabs(r4))));
  }
  const double r5 = a0 - zet - alam, r6 = zet * z;
  ss += r5 * r5 + r6 * r6;
  mx = std::max(mx, std::max(fabs(r5), fabs(r6)));
  kkt_out[0] = sqrt(ss);
  kkt_out[1] = mx;
  return PYTO_OK;
}
