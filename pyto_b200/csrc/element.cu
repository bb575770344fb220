// Host-side element set-up: hex8 Ke and its Hadamard-basis block form.
//
// Ke follows src/hex_element_stiffness.py:232-286 (2x2x2 Gauss, isotropic D,
// B rows xx,yy,zz,xy,yz,xz).  For a box element every reflection x->-x, y->-y,
// z->-z is a symmetry, so in the corner basis of the 8 Hadamard modes
// phi_m(corner) = prod_{d in m} (2 b_d - 1), (b = corner bit coordinates),
// K^ = Phi Ke Phi^T / 64 couples (component c, mode m) only with pairs of the
// same reflection parity.  Class q (bits = which reflections flip the pair)
// holds exactly one mode per component, m = q ^ (1 << c); K^ is therefore
// eight 3x3 blocks (57 non-zeros once the three rigid translations, m = 0,
// which Ke annihilates, are dropped) instead of a dense 24x24.
#include <math.h>
#include <string.h>

#include "common.cuh"

namespace {

// reference corner order -> bit coordinates (src/hex_mesher.py:120-124)
const int kCornerBits[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                               {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};

double phi(int m, int a) {
  double v = 1.0;
  for (int d = 0; d < 3; ++d)
    if (m & (1 << d)) v *= (kCornerBits[a][d] ? 1.0 : -1.0);
  return v;
}

void constitutive(double E, double nu, double D[6][6]) {
  const double c = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) D[i][j] = 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) D[i][j] = c * (i == j ? 1.0 - nu : nu);
  for (int i = 3; i < 6; ++i) D[i][i] = c * (1.0 - 2.0 * nu) / 2.0;
}

}  // namespace

extern "C" int pyto_version(void) { return 1; }

extern "C" size_t pyto_struct_size(int which) {
  switch (which) {
    case 0: return sizeof(pyto_operator_t);
    case 1: return sizeof(pyto_solve_cfg_t);
    case 2: return sizeof(pyto_solve_status_t);
    case 3: return sizeof(pyto_deflation_t);
    case 4: return sizeof(pyto_batch_item_t);
    case 5: return sizeof(pyto_thermal_t);
    default: return 0;
  }
}

extern "C" int pyto_ke_hex8(double E, double nu, double hx, double hy, double hz, double* ke) {
  if (!ke || !(hx > 0) || !(hy > 0) || !(hz > 0) || !(nu < 0.5) || !(nu > -1.0)) return PYTO_ERR_ARG;
  double D[6][6];
  constitutive(E, nu, D);
  const double g = 0.5773502691896257;  // 1/sqrt(3), the 2-point Gauss abscissa
  const double gp[2] = {-g, g};
  const double xs[8] = {-1, 1, 1, -1, -1, 1, 1, -1}, ys[8] = {-1, -1, 1, 1, -1, -1, 1, 1},
               zs[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
  const double h[3] = {hx, hy, hz};
  for (int i = 0; i < 576; ++i) ke[i] = 0.0;
  const double detJ = (hx / 2.0) * (hy / 2.0) * (hz / 2.0);
  for (int ia = 0; ia < 2; ++ia)
    for (int ib = 0; ib < 2; ++ib)
      for (int ic = 0; ic < 2; ++ic) {
        const double xi = gp[ia], eta = gp[ib], zeta = gp[ic];
        double grad[8][3];
        for (int n = 0; n < 8; ++n) {
          grad[n][0] = 0.125 * xs[n] * (1 + eta * ys[n]) * (1 + zeta * zs[n]) * (2.0 / h[0]);
          grad[n][1] = 0.125 * (1 + xi * xs[n]) * ys[n] * (1 + zeta * zs[n]) * (2.0 / h[1]);
          grad[n][2] = 0.125 * (1 + xi * xs[n]) * (1 + eta * ys[n]) * zs[n] * (2.0 / h[2]);
        }
        double B[6][24];
        memset(B, 0, sizeof(B));
        for (int l = 0; l < 8; ++l) {
          B[0][3 * l] = grad[l][0];
          B[1][3 * l + 1] = grad[l][1];
          B[2][3 * l + 2] = grad[l][2];
          B[3][3 * l] = grad[l][1];
          B[3][3 * l + 1] = grad[l][0];
          B[4][3 * l + 1] = grad[l][2];
          B[4][3 * l + 2] = grad[l][1];
          B[5][3 * l] = grad[l][2];
          B[5][3 * l + 2] = grad[l][0];
        }
        double DB[6][24];
        for (int i = 0; i < 6; ++i)
          for (int j = 0; j < 24; ++j) {
            double acc = 0.0;
            for (int k = 0; k < 6; ++k) acc += D[i][k] * B[k][j];
            DB[i][j] = acc;
          }
        for (int i = 0; i < 24; ++i)
          for (int j = 0; j < 24; ++j) {
            double acc = 0.0;
            for (int k = 0; k < 6; ++k) acc += B[k][i] * DB[k][j];
            ke[24 * i + j] += acc * detJ;
          }
      }
  return PYTO_OK;
}

extern "C" int pyto_operator_init(pyto_operator_t* op, int32_t nelx, int32_t nely, int32_t nelz, double hx,
                                  double hy, double hz, double E, double nu, const double* ke) {
  if (!op || nelx < 1 || nely < 1 || nelz < 1) return PYTO_ERR_ARG;
  // node DOF ids must fit in int32 for the kernels' index arithmetic
  const double nn = (double)(nelx + 1) * (nely + 1) * (nelz + 1);
  if (nn * 3.0 > 2147483647.0) return PYTO_ERR_TOO_LARGE;
  memset(op, 0, sizeof(*op));
  op->nelx = nelx; op->nely = nely; op->nelz = nelz;
  op->hx = hx; op->hy = hy; op->hz = hz;
  op->E = E; op->nu = nu;
  if (ke) {
    memcpy(op->ke, ke, sizeof(op->ke));
  } else {
    int st = pyto_ke_hex8(E, nu, hx, hy, hz, op->ke);
    if (st != PYTO_OK) return st;
  }
  double kh[24][24];
  double kmax = 0.0;
  for (int i = 0; i < 576; ++i) kmax = fmax(kmax, fabs(op->ke[i]));
  if (!(kmax > 0.0) || !isfinite(kmax)) return PYTO_ERR_ARG;
  for (int c = 0; c < 3; ++c)
    for (int m = 0; m < 8; ++m)
      for (int d = 0; d < 3; ++d)
        for (int n = 0; n < 8; ++n) {
          double acc = 0.0;
          for (int a = 0; a < 8; ++a) {
            const double pa = phi(m, a);
            for (int b = 0; b < 8; ++b) acc += pa * op->ke[24 * (3 * a + c) + (3 * b + d)] * phi(n, b);
          }
          kh[8 * c + m][8 * d + n] = acc / 64.0;
        }
  // every entry outside the parity blocks (and every translation row/column)
  // must vanish for a box hex8 Ke
  const double tol = 1e-9 * kmax;
  for (int c = 0; c < 3; ++c)
    for (int m = 0; m < 8; ++m)
      for (int d = 0; d < 3; ++d)
        for (int n = 0; n < 8; ++n) {
          const int qa = m ^ (1 << c), qb = n ^ (1 << d);
          const bool in_block = (qa == qb) && m != 0 && n != 0;
          if (!in_block && fabs(kh[8 * c + m][8 * d + n]) > tol) return PYTO_ERR_ARG;
        }
  for (int q = 0; q < 8; ++q)
    for (int c = 0; c < 3; ++c)
      for (int d = 0; d < 3; ++d) {
        const int m = q ^ (1 << c), n = q ^ (1 << d);
        op->khat[q][c][d] = (m == 0 || n == 0) ? 0.0 : kh[8 * c + m][8 * d + n];
      }
  for (int c = 0; c < 3; ++c) {
    op->kdiag[c] = op->ke[24 * c + c];
    for (int a = 1; a < 8; ++a)
      if (fabs(op->ke[24 * (3 * a + c) + 3 * a + c] - op->kdiag[c]) > tol) return PYTO_ERR_ARG;
  }
  return PYTO_OK;
}
