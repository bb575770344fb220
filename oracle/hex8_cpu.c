/*
 * hex8_cpu.c -- OpenMP C restatement of PyTO's CPU solve path for the voxel hex8
 * cantilever (TEST INFRASTRUCTURE: the oracle's compiled half and the timed CPU
 * baseline; never linked into or called by the product library).
 *
 * What it restates, per solve, in the reference's order:
 *   1. assembly of the reduced stiffness K_ff = (sum_e s_e Ke)[free][:, free] as a
 *      CSR matrix (src/hex_structural_fea.py:87-102 builds the COO triplets and
 *      converts to CSR; src/bound_cond.py:40-70 slices the free rows and columns).
 *      The CSR holds every structurally present entry (27 neighbour nodes x 3
 *      components per row, minus fixed columns), with columns in ascending DOF
 *      order, exactly the pattern scipy's COO->CSR conversion yields;
 *   2. the Jacobi preconditioner 1/diag with |d| < 1e-12 -> 1
 *      (src/linear_solvers.py:71-87);
 *   3a. Jacobi PCG, scipy cg recurrence, stop on ||r||_2 < rtol ||b||_2
 *       (src/linear_solvers.py:164-168), or
 *   3b. deflated PCG (src/deflation.py:504-584): E = W^T K W (dense, symmetrised)
 *       plus a diagonal shift, a dense Cholesky factorisation of E (the reference
 *       factorises once and solves per application), coarse start x = W E^-1 W^T b,
 *       p0 = z - W E^-1 W^T K z, and per iteration two products with K (K p and
 *       K z) and one coarse solve.  Stopping rule 0 as in 3a (true relative
 *       residual semantics) or 1, the reference's sqrt(r.z / r0.z0) <= rtol
 *       (src/deflation.py:567); rigid-body W of node groups (src/deflation.py:386-457).
 *
 * Element corner order (src/hex_mesher.py:120-124): (0,0,0),(1,0,0),(1,1,0),
 * (0,1,0),(0,0,1),(1,0,1),(1,1,1),(0,1,1); node n = ix + sx*(iy + sy*iz),
 * DOF 3n + c (src/hex_mesher.py:1085-1094).
 *
 * All entry points are plain C with host pointers; threads come from OpenMP
 * (OMP_NUM_THREADS, default: all cores).
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int nx, ny, nz, sx, sy, sz;
  int64_t nnodes, ndof, nfree;
  double ke[576];
  uint8_t* mask;       /* [nnodes] bits 0-2: fixed components */
  int64_t* free_of;    /* [ndof] free index or -1 */
  int64_t* dof_of;     /* [nfree] DOF of each free index */
  /* CSR of K_ff */
  int64_t* rowptr;     /* [nfree+1] */
  int32_t* col;        /* [nnz] */
  double* val;         /* [nnz] */
  int64_t nnz;
  double* minv;        /* [nfree] Jacobi */
  double t_assemble;
} hex8_cpu_t;

static const int kCorner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                  {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};

static int corner_id(int bx, int by, int bz) {
  for (int k = 0; k < 8; ++k)
    if (kCorner[k][0] == bx && kCorner[k][1] == by && kCorner[k][2] == bz) return k;
  return -1;
}

int hex8_cpu_threads(void) { return omp_get_max_threads(); }

void* hex8_cpu_create(int nx, int ny, int nz, const double* ke, const uint8_t* node_mask) {
  if (nx < 1 || ny < 1 || nz < 1 || !ke || !node_mask) return NULL;
  hex8_cpu_t* h = (hex8_cpu_t*)calloc(1, sizeof(hex8_cpu_t));
  if (!h) return NULL;
  h->nx = nx; h->ny = ny; h->nz = nz;
  h->sx = nx + 1; h->sy = ny + 1; h->sz = nz + 1;
  h->nnodes = (int64_t)h->sx * h->sy * h->sz;
  h->ndof = 3 * h->nnodes;
  memcpy(h->ke, ke, sizeof(h->ke));
  h->mask = (uint8_t*)malloc(h->nnodes);
  h->free_of = (int64_t*)malloc(sizeof(int64_t) * h->ndof);
  if (!h->mask || !h->free_of) return NULL;
  memcpy(h->mask, node_mask, h->nnodes);
  int64_t k = 0;
  for (int64_t d = 0; d < h->ndof; ++d) h->free_of[d] = ((h->mask[d / 3] >> (d % 3)) & 1) ? -1 : k++;
  h->nfree = k;
  h->dof_of = (int64_t*)malloc(sizeof(int64_t) * (k ? k : 1));
  for (int64_t d = 0; d < h->ndof; ++d)
    if (h->free_of[d] >= 0) h->dof_of[h->free_of[d]] = d;
  return h;
}

void hex8_cpu_destroy(void* hp) {
  hex8_cpu_t* h = (hex8_cpu_t*)hp;
  if (!h) return;
  free(h->mask); free(h->free_of); free(h->dof_of);
  free(h->rowptr); free(h->col); free(h->val); free(h->minv);
  free(h);
}

int64_t hex8_cpu_nfree(void* hp) { return ((hex8_cpu_t*)hp)->nfree; }
int64_t hex8_cpu_nnz(void* hp) { return ((hex8_cpu_t*)hp)->nnz; }
double hex8_cpu_assemble_seconds(void* hp) { return ((hex8_cpu_t*)hp)->t_assemble; }

/* Row of node n, component c: values of the 27x3 neighbour columns (index
 * ((dz+1)*3 + (dy+1))*3 + (dx+1), component d) summed over the elements shared. */
static void node_row(const hex8_cpu_t* h, const double* s, int ix, int iy, int iz, int c, double* acc) {
  memset(acc, 0, sizeof(double) * 81);
  for (int ez = iz - 1; ez <= iz; ++ez) {
    if (ez < 0 || ez >= h->nz) continue;
    for (int ey = iy - 1; ey <= iy; ++ey) {
      if (ey < 0 || ey >= h->ny) continue;
      for (int ex = ix - 1; ex <= ix; ++ex) {
        if (ex < 0 || ex >= h->nx) continue;
        double se = s[ex + (int64_t)h->nx * (ey + (int64_t)h->ny * ez)];
        int a = corner_id(ix - ex, iy - ey, iz - ez);
        const double* kr = h->ke + (3 * a + c) * 24;
        for (int b = 0; b < 8; ++b) {
          int dx = ex + kCorner[b][0] - ix, dy = ey + kCorner[b][1] - iy, dz = ez + kCorner[b][2] - iz;
          int slot = ((dz + 1) * 3 + (dy + 1)) * 3 + (dx + 1);
          for (int d = 0; d < 3; ++d) acc[3 * slot + d] += se * kr[3 * b + d];
        }
      }
    }
  }
}

/* Assemble K_ff(s) into CSR (pattern and values, as the reference rebuilds its
 * matrix every solve) and the Jacobi inverse diagonal. */
int hex8_cpu_assemble(void* hp, const double* s) {
  hex8_cpu_t* h = (hex8_cpu_t*)hp;
  if (!h || !s) return -1;
  double t0 = omp_get_wtime();
  free(h->rowptr); free(h->col); free(h->val); free(h->minv);
  int64_t nf = h->nfree;
  h->rowptr = (int64_t*)malloc(sizeof(int64_t) * (nf + 1));
  h->minv = (double*)malloc(sizeof(double) * (nf ? nf : 1));
  if (!h->rowptr || !h->minv) return -2;
  /* count: free neighbour DOFs of the row's node */
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < nf; ++i) {
    int64_t n = h->dof_of[i] / 3;
    int ix = (int)(n % h->sx), iy = (int)((n / h->sx) % h->sy), iz = (int)(n / ((int64_t)h->sx * h->sy));
    int64_t cnt = 0;
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          int jx = ix + dx, jy = iy + dy, jz = iz + dz;
          if (jx < 0 || jy < 0 || jz < 0 || jx >= h->sx || jy >= h->sy || jz >= h->sz) continue;
          int64_t m = jx + (int64_t)h->sx * (jy + (int64_t)h->sy * jz);
          for (int d = 0; d < 3; ++d) cnt += ((h->mask[m] >> d) & 1) ? 0 : 1;
        }
    h->rowptr[i + 1] = cnt;
  }
  h->rowptr[0] = 0;
  for (int64_t i = 0; i < nf; ++i) h->rowptr[i + 1] += h->rowptr[i];
  h->nnz = h->rowptr[nf];
  h->col = (int32_t*)malloc(sizeof(int32_t) * (h->nnz ? h->nnz : 1));
  h->val = (double*)malloc(sizeof(double) * (h->nnz ? h->nnz : 1));
  if (!h->col || !h->val) return -2;
#pragma omp parallel
  {
    double acc[81];
#pragma omp for schedule(static)
    for (int64_t i = 0; i < nf; ++i) {
      int64_t dof = h->dof_of[i], n = dof / 3;
      int c = (int)(dof % 3);
      int ix = (int)(n % h->sx), iy = (int)((n / h->sx) % h->sy), iz = (int)(n / ((int64_t)h->sx * h->sy));
      node_row(h, s, ix, iy, iz, c, acc);
      int64_t k = h->rowptr[i];
      double diag = 0.0;
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            int jx = ix + dx, jy = iy + dy, jz = iz + dz;
            if (jx < 0 || jy < 0 || jz < 0 || jx >= h->sx || jy >= h->sy || jz >= h->sz) continue;
            int64_t m = jx + (int64_t)h->sx * (jy + (int64_t)h->sy * jz);
            int slot = ((dz + 1) * 3 + (dy + 1)) * 3 + (dx + 1);
            for (int d = 0; d < 3; ++d) {
              int64_t j = h->free_of[3 * m + d];
              if (j < 0) continue;
              h->col[k] = (int32_t)j;
              h->val[k] = acc[3 * slot + d];
              if (j == i) diag = acc[3 * slot + d];
              ++k;
            }
          }
      h->minv[i] = fabs(diag) < 1e-12 ? 1.0 : 1.0 / diag;
    }
  }
  h->t_assemble = omp_get_wtime() - t0;
  return 0;
}

/* Copy of the CSR (for checking the assembly against the oracle's scipy matrix). */
int hex8_cpu_csr(void* hp, int64_t* rowptr, int32_t* col, double* val) {
  hex8_cpu_t* h = (hex8_cpu_t*)hp;
  if (!h || !h->rowptr) return -1;
  memcpy(rowptr, h->rowptr, sizeof(int64_t) * (h->nfree + 1));
  memcpy(col, h->col, sizeof(int32_t) * h->nnz);
  memcpy(val, h->val, sizeof(double) * h->nnz);
  return 0;
}

static void spmv(const hex8_cpu_t* h, const double* x, double* y) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < h->nfree; ++i) {
    double a = 0.0;
    for (int64_t k = h->rowptr[i]; k < h->rowptr[i + 1]; ++k) a += h->val[k] * x[h->col[k]];
    y[i] = a;
  }
}

static double dot(int64_t n, const double* a, const double* b) {
  double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

/* Full-length b -> free vector; free vector -> full-length u (fixed entries 0). */
static void gather_free(const hex8_cpu_t* h, const double* full, double* f) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < h->nfree; ++i) f[i] = full[h->dof_of[i]];
}
static void scatter_free(const hex8_cpu_t* h, const double* f, double* full) {
#pragma omp parallel for schedule(static)
  for (int64_t d = 0; d < h->ndof; ++d) full[d] = 0.0;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < h->nfree; ++i) full[h->dof_of[i]] = f[i];
}

static double true_rel_res(const hex8_cpu_t* h, const double* b, const double* x, double* tmp) {
  spmv(h, x, tmp);
  double rr = 0.0;
#pragma omp parallel for reduction(+ : rr) schedule(static)
  for (int64_t i = 0; i < h->nfree; ++i) rr += (b[i] - tmp[i]) * (b[i] - tmp[i]);
  double bb = dot(h->nfree, b, b);
  return bb > 0 ? sqrt(rr / bb) : 0.0;
}

/* Jacobi PCG with scipy cg's recurrence and stopping test (x0 = 0). */
int hex8_cpu_pcg(void* hp, const double* b_full, double* u_full, double rtol, int max_iters, int* iters_out,
                 double* true_rel_out, double* t_solve_out) {
  hex8_cpu_t* h = (hex8_cpu_t*)hp;
  if (!h || !h->rowptr) return -1;
  double t0 = omp_get_wtime();
  int64_t n = h->nfree;
  double *b = malloc(8 * n), *x = calloc(n, 8), *r = malloc(8 * n), *z = malloc(8 * n), *p = malloc(8 * n),
         *q = malloc(8 * n);
  gather_free(h, b_full, b);
  memcpy(r, b, 8 * n);
  double bn = sqrt(dot(n, b, b)), rz = 0.0;
  int it = 0, conv = bn == 0.0;
  for (it = 0; it < max_iters && !conv; ++it) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) z[i] = h->minv[i] * r[i];
    double rz_new = dot(n, r, z);
    if (it == 0) {
      memcpy(p, z, 8 * n);
    } else {
      double beta = rz_new / rz;
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    }
    rz = rz_new;
    spmv(h, p, q);
    double alpha = rz / dot(n, p, q);
    double rr = 0.0;
#pragma omp parallel for reduction(+ : rr) schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * q[i];
      rr += r[i] * r[i];
    }
    conv = sqrt(rr) < rtol * bn;
  }
  *iters_out = it;
  *true_rel_out = true_rel_res(h, b, x, q);
  scatter_free(h, x, u_full);
  *t_solve_out = omp_get_wtime() - t0;
  free(b); free(x); free(r); free(z); free(p); free(q);
  return conv ? 0 : 1;
}

/* ---- deflation ----------------------------------------------------------- */
typedef struct {
  int ng, modes, nc, wn;  /* wn: non-zeros per W row (1 for 3 modes, 3 for 6) */
  int64_t* gptr;   /* free rows grouped: [ng+1] */
  int64_t* grows;  /* free row ids by group */
  int32_t* wcol;   /* [nfree*wn] W columns of each free row */
  double* wval;    /* [nfree*wn] W values */
  double* L;       /* [nc*nc] Cholesky factor (lower, row-major) */
} defl_t;

/* W (restricted to the free rows), built once per deflation space like the
 * reference's create_deflation_matrix (src/deflation.py:386-457): columns
 * 6g+{0,1,2} translations, 6g+3 rotation about x (0,-z,y), 6g+4 about y (z,0,-x),
 * 6g+5 about z (-y,x,0) with rel = xyz - centre[g]; 3 modes: column 3g+c. */
static void build_w(const hex8_cpu_t* h, defl_t* D, const int32_t* node_group, const double* centre,
                    const double* hxyz) {
  int wn = D->wn;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < h->nfree; ++i) {
    int64_t dof = h->dof_of[i], n = dof / 3;
    int c = (int)(dof % 3), g = node_group[n];
    int32_t* cols = D->wcol + i * wn;
    double* vals = D->wval + i * wn;
    if (D->modes == 3) {
      cols[0] = 3 * g + c; vals[0] = 1.0;
      continue;
    }
    int ix = (int)(n % h->sx), iy = (int)((n / h->sx) % h->sy), iz = (int)(n / ((int64_t)h->sx * h->sy));
    double rx = ix * hxyz[0] - centre[3 * g], ry = iy * hxyz[1] - centre[3 * g + 1],
           rz = iz * hxyz[2] - centre[3 * g + 2];
    int b = 6 * g;
    cols[0] = b + c; vals[0] = 1.0;
    if (c == 0) { cols[1] = b + 4; vals[1] = rz; cols[2] = b + 5; vals[2] = -ry; }
    else if (c == 1) { cols[1] = b + 3; vals[1] = -rz; cols[2] = b + 5; vals[2] = rx; }
    else { cols[1] = b + 3; vals[1] = ry; cols[2] = b + 4; vals[2] = -rx; }
  }
}

/* v_c = W^T v (per group, thread-exclusive rows of the coarse vector). */
static void restrict_w(const defl_t* D, const double* v, double* vc) {
#pragma omp parallel for schedule(dynamic, 4)
  for (int g = 0; g < D->ng; ++g) {
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int64_t k = D->gptr[g]; k < D->gptr[g + 1]; ++k) {
      int64_t i = D->grows[k];
      for (int a = 0; a < D->wn; ++a) acc[D->wcol[i * D->wn + a] - D->modes * g] += D->wval[i * D->wn + a] * v[i];
    }
    for (int a = 0; a < D->modes; ++a) vc[D->modes * g + a] = acc[a];
  }
}

/* out = W mu. */
static void prolong_w(const hex8_cpu_t* h, const defl_t* D, const double* mu, double* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < h->nfree; ++i) {
    double a = 0.0;
    for (int k = 0; k < D->wn; ++k) a += D->wval[i * D->wn + k] * mu[D->wcol[i * D->wn + k]];
    out[i] = a;
  }
}

/* E = W^T K W over the CSR (src/deflation.py:517-521): rows of E owned by the
 * group of the CSR row, so each thread writes its own rows. */
static void coarse_matrix(const hex8_cpu_t* h, const defl_t* D, double* E) {
  const int wn = D->wn, nc = D->nc;
#pragma omp parallel for schedule(dynamic, 1)
  for (int g = 0; g < D->ng; ++g) {
    for (int64_t k = D->gptr[g]; k < D->gptr[g + 1]; ++k) {
      int64_t i = D->grows[k];
      const int32_t* ci = D->wcol + i * wn;
      const double* vi = D->wval + i * wn;
      for (int64_t q = h->rowptr[i]; q < h->rowptr[i + 1]; ++q) {
        const int32_t* cj = D->wcol + (int64_t)h->col[q] * wn;
        const double* vj = D->wval + (int64_t)h->col[q] * wn;
        double kv = h->val[q];
        for (int a = 0; a < wn; ++a) {
          double* er = E + (int64_t)ci[a] * nc;
          double w = vi[a] * kv;
          for (int bb = 0; bb < wn; ++bb) er[cj[bb]] += w * vj[bb];
        }
      }
    }
  }
}

static int defl_init(const hex8_cpu_t* h, defl_t* D, const int32_t* node_group, int ng, const double* centre,
                     int modes, const double* hxyz) {
  D->ng = ng; D->modes = modes; D->nc = ng * modes; D->wn = modes == 6 ? 3 : 1;
  int64_t n = h->nfree;
  D->gptr = (int64_t*)calloc(ng + 1, sizeof(int64_t));
  D->grows = (int64_t*)malloc(sizeof(int64_t) * (n ? n : 1));
  D->wcol = (int32_t*)malloc(sizeof(int32_t) * (n ? n : 1) * D->wn);
  D->wval = (double*)malloc(sizeof(double) * (n ? n : 1) * D->wn);
  D->L = NULL;
  if (!D->gptr || !D->grows || !D->wcol || !D->wval) return -2;
  for (int64_t i = 0; i < n; ++i) D->gptr[node_group[h->dof_of[i] / 3] + 1]++;
  for (int g = 0; g < ng; ++g) D->gptr[g + 1] += D->gptr[g];
  int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * ng);
  memcpy(fill, D->gptr, sizeof(int64_t) * ng);
  for (int64_t i = 0; i < n; ++i) D->grows[fill[node_group[h->dof_of[i] / 3]]++] = i;
  free(fill);
  build_w(h, D, node_group, centre, hxyz);
  return 0;
}

static void defl_free(defl_t* D) {
  free(D->gptr); free(D->grows); free(D->wcol); free(D->wval); free(D->L);
}

/* W^T K_ff W (unshifted, as assembled) into E[nc*nc], for checking. */
int hex8_cpu_coarse_matrix(void* hp, const int32_t* node_group, int ng, const double* centre, int modes,
                           const double* hxyz, double* E) {
  hex8_cpu_t* h = (hex8_cpu_t*)hp;
  if (!h || !h->rowptr || (modes != 3 && modes != 6) || ng < 1) return -1;
  defl_t D;
  if (defl_init(h, &D, node_group, ng, centre, modes, hxyz)) return -2;
  memset(E, 0, sizeof(double) * (size_t)D.nc * D.nc);
  coarse_matrix(h, &D, E);
  defl_free(&D);
  return 0;
}

/* Blocked right-looking Cholesky of the row-major n x n SPD matrix A (lower
 * factor in place; the upper triangle is left untouched).  Returns 0 or the
 * failing pivot + 1. */
static int cholesky(double* A, int n) {
  const int nb = 64;
  for (int k0 = 0; k0 < n; k0 += nb) {
    int k1 = k0 + nb < n ? k0 + nb : n;
    for (int k = k0; k < k1; ++k) {  /* unblocked factor of the panel columns k0..k1 */
      double d = A[(int64_t)k * n + k];
      for (int j = k0; j < k; ++j) d -= A[(int64_t)k * n + j] * A[(int64_t)k * n + j];
      if (!(d > 0.0)) return k + 1;
      d = sqrt(d);
      A[(int64_t)k * n + k] = d;
#pragma omp parallel for schedule(static)
      for (int i = k + 1; i < n; ++i) {
        double a = A[(int64_t)i * n + k];
        for (int j = k0; j < k; ++j) a -= A[(int64_t)i * n + j] * A[(int64_t)k * n + j];
        A[(int64_t)i * n + k] = a / d;
      }
    }
    /* trailing update of the lower part: A[i][j] -= sum_p L[i][p] L[j][p], p in panel */
#pragma omp parallel for schedule(dynamic, 8)
    for (int i = k1; i < n; ++i) {
      const double* li = A + (int64_t)i * n + k0;
      for (int j = k1; j <= i; ++j) {
        const double* lj = A + (int64_t)j * n + k0;
        double a = 0.0;
        for (int p = 0; p < k1 - k0; ++p) a += li[p] * lj[p];
        A[(int64_t)i * n + j] -= a;
      }
    }
  }
  return 0;
}

/* Copy the lower factor's transpose into the upper triangle (row-major U = L^T),
 * so that both triangular sweeps read contiguous rows. */
static void mirror_factor(double* L, int n) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) L[(int64_t)i * n + j] = L[(int64_t)j * n + i];
}

/* Solve L L^T x = b in place; F holds L in its lower and L^T in its upper
 * triangle (row-major).  Blocked: each 64-row diagonal block is solved in order,
 * the rows after it (forward) or before it (backward) are updated in parallel. */
static void cholesky_solve(const double* F, int n, double* x) {
  const int nb = 64;
  for (int k0 = 0; k0 < n; k0 += nb) {
    int k1 = k0 + nb < n ? k0 + nb : n;
    for (int i = k0; i < k1; ++i) {
      double a = x[i];
      const double* fi = F + (int64_t)i * n;
      for (int j = k0; j < i; ++j) a -= fi[j] * x[j];
      x[i] = a / fi[i];
    }
#pragma omp parallel for schedule(static)
    for (int i = k1; i < n; ++i) {
      const double* fi = F + (int64_t)i * n;
      double a = 0.0;
      for (int j = k0; j < k1; ++j) a += fi[j] * x[j];
      x[i] -= a;
    }
  }
  for (int k1 = n; k1 > 0; k1 -= nb) {
    int k0 = k1 - nb > 0 ? k1 - nb : 0;
    for (int i = k1 - 1; i >= k0; --i) {
      double a = x[i];
      const double* fi = F + (int64_t)i * n;
      for (int j = i + 1; j < k1; ++j) a -= fi[j] * x[j];
      x[i] = a / fi[i];
    }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < k0; ++i) {
      const double* fi = F + (int64_t)i * n;
      double a = 0.0;
      for (int j = k0; j < k1; ++j) a += fi[j] * x[j];
      x[i] -= a;
    }
  }
}

/* Deflated PCG.  node_group[nnodes] (group of each node), centre[ng*3] (group
 * centroids), modes 6 or 3; the shift added to the symmetrised E is
 * shift * mean(diag E) when shift_relative, else shift (the reference: 1e-10
 * absolute, src/deflation.py:521).  stop_rule 0: ||r|| < rtol ||b||; 1: the
 * reference's sqrt(r.z / r0.z0) <= rtol.  times[0] = coarse set-up (E and its
 * factor), times[1] = iterations. */
int hex8_cpu_dpcg(void* hp, const int32_t* node_group, int ng, const double* centre, int modes, double shift,
                  int shift_relative, const double* hxyz, const double* b_full, double* u_full, double rtol,
                  int max_iters, int stop_rule, int* iters_out, double* true_rel_out, double* times) {
  hex8_cpu_t* h = (hex8_cpu_t*)hp;
  if (!h || !h->rowptr || (modes != 3 && modes != 6) || ng < 1) return -1;
  defl_t D;
  int64_t n = h->nfree;
  /* the deflation space (groups, W) is built once per mesh in the reference:
     not part of the timed per-solve set-up */
  if (defl_init(h, &D, node_group, ng, centre, modes, hxyz)) return -2;
  int nc = D.nc;
  double t0 = omp_get_wtime();
  D.L = (double*)calloc((size_t)nc * nc, sizeof(double));
  double* E = D.L;
  coarse_matrix(h, &D, E);
  double md = 0.0;
  for (int i = 0; i < nc; ++i) md += E[(int64_t)i * nc + i];
  md /= nc;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nc; ++i)
    for (int j = 0; j < i; ++j) {
      double a = 0.5 * (E[(int64_t)i * nc + j] + E[(int64_t)j * nc + i]);
      E[(int64_t)i * nc + j] = a;
    }
  double sh = shift_relative ? shift * md : shift;
  for (int i = 0; i < nc; ++i) E[(int64_t)i * nc + i] += sh;
  int bad = cholesky(E, nc);
  if (!bad) mirror_factor(E, nc);
  double t1 = omp_get_wtime();
  times[0] = t1 - t0;
  if (bad) {
    defl_free(&D);
    return -4;
  }
  double *b = malloc(8 * n), *x = malloc(8 * n), *r = malloc(8 * n), *z = malloc(8 * n), *p = malloc(8 * n),
         *q = malloc(8 * n), *kz = malloc(8 * n), *wm = malloc(8 * n), *vc = malloc(8 * (size_t)nc);
  gather_free(h, b_full, b);
  double bn = sqrt(dot(n, b, b));
  /* coarse start x = W E^-1 W^T b; r = b - K x */
  restrict_w(&D, b, vc);
  cholesky_solve(D.L, nc, vc);
  prolong_w(h, &D, vc, x);
  spmv(h, x, q);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    r[i] = b[i] - q[i];
    z[i] = h->minv[i] * r[i];
  }
  /* p0 = z - W E^-1 W^T K z */
  spmv(h, z, kz);
  restrict_w(&D, kz, vc);
  cholesky_solve(D.L, nc, vc);
  prolong_w(h, &D, vc, wm);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) p[i] = z[i] - wm[i];
  double rz = dot(n, r, z), rz0 = rz;
  int it = 0, conv = bn == 0.0;
  for (it = 0; it < max_iters && !conv;) {
    spmv(h, p, q);
    double alpha = rz / dot(n, p, q);
    double rr = 0.0, rz_new = 0.0;
#pragma omp parallel for reduction(+ : rr, rz_new) schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * q[i];
      z[i] = h->minv[i] * r[i];
      rr += r[i] * r[i];
      rz_new += r[i] * z[i];
    }
    ++it;
    if (stop_rule == 1 ? sqrt(rz_new / rz0) <= rtol : sqrt(rr) < rtol * bn) {
      conv = 1;
      break;
    }
    double beta = rz_new / rz;
    spmv(h, z, kz);
    restrict_w(&D, kz, vc);
    cholesky_solve(D.L, nc, vc);
    prolong_w(h, &D, vc, wm);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i] - wm[i];
    rz = rz_new;
  }
  *iters_out = it;
  times[1] = omp_get_wtime() - t1;
  *true_rel_out = true_rel_res(h, b, x, q);
  scatter_free(h, x, u_full);
  free(b); free(x); free(r); free(z); free(p); free(q); free(kz); free(wm); free(vc);
  defl_free(&D);
  return conv ? 0 : 1;
}

/* Density filter rho = (H x) / Hs with H_ij = (r - d_ij)/r for d_ij <= r on the
 * element-centre grid (src/topopt_filters.py:8-38; r = rel * hx), for preparing
 * the bench densities on the host. */
int hex8_cpu_density_filter(int nx, int ny, int nz, const double* hxyz, double rel, const double* x, double* rho) {
  double r = rel * hxyz[0];
  int R[3];
  for (int d = 0; d < 3; ++d) R[d] = (int)ceil(r / hxyz[d]) + 1;
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < (int64_t)nx * ny * nz; ++e) {
    int ex = (int)(e % nx), ey = (int)((e / nx) % ny), ez = (int)(e / ((int64_t)nx * ny));
    double num = 0.0, den = 0.0;
    for (int dz = -R[2]; dz <= R[2]; ++dz)
      for (int dy = -R[1]; dy <= R[1]; ++dy)
        for (int dx = -R[0]; dx <= R[0]; ++dx) {
          int jx = ex + dx, jy = ey + dy, jz = ez + dz;
          if (jx < 0 || jy < 0 || jz < 0 || jx >= nx || jy >= ny || jz >= nz) continue;
          double d = sqrt((dx * hxyz[0]) * (dx * hxyz[0]) + (dy * hxyz[1]) * (dy * hxyz[1]) +
                          (dz * hxyz[2]) * (dz * hxyz[2]));
          if (d > r) continue;
          double w = (r - d) / r;
          num += w * x[jx + (int64_t)nx * (jy + (int64_t)ny * jz)];
          den += w;
        }
    rho[e] = num / den;
  }
  return 0;
}
