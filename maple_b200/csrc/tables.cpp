// Host-side FP64 element tables for the periodic voxel cell.
//
// Element matrices follow maple/core/utils/_utils.py:39-196 (isotropic C with
// float32 entries, 3x3x3 Gauss quadrature, X0 from the pinned element solve);
// the child-prolongation weights follow the trilinear Galerkin coarsening of
// maple/core/utils/EBE_GMG.py:202-337.  All tables are computed for a voxel of
// edge 1 (r = 1) and rescaled by the caller: Ke ~ 1/r, Fe ~ 1/r^2, X0 ~ 1/r.
#include "tables.h"

#include <cmath>
#include <cstring>

namespace maple {

const int kCorner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                           {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};

static void solve_dense(int n, double* A, double* B, int nrhs) {
  // Gaussian elimination with partial pivoting, A (n x n) row-major, B (n x nrhs).
  for (int k = 0; k < n; ++k) {
    int p = k;
    for (int i = k + 1; i < n; ++i)
      if (std::fabs(A[i * n + k]) > std::fabs(A[p * n + k])) p = i;
    if (p != k) {
      for (int j = 0; j < n; ++j) std::swap(A[k * n + j], A[p * n + j]);
      for (int j = 0; j < nrhs; ++j) std::swap(B[k * nrhs + j], B[p * nrhs + j]);
    }
    for (int i = k + 1; i < n; ++i) {
      double f = A[i * n + k] / A[k * n + k];
      for (int j = k; j < n; ++j) A[i * n + j] -= f * A[k * n + j];
      for (int j = 0; j < nrhs; ++j) B[i * nrhs + j] -= f * B[k * nrhs + j];
    }
  }
  for (int k = n - 1; k >= 0; --k) {
    for (int j = 0; j < nrhs; ++j) {
      double s = B[k * nrhs + j];
      for (int i = k + 1; i < n; ++i) s -= A[k * n + i] * B[i * nrhs + j];
      B[k * nrhs + j] = s / A[k * n + k];
    }
  }
}

static void shape_grads(double xi, double eta, double zeta, double g[3][8]) {
  for (int a = 0; a < 8; ++a) {
    double sx = 2 * kCorner[a][0] - 1, sy = 2 * kCorner[a][1] - 1, sz = 2 * kCorner[a][2] - 1;
    g[0][a] = sx * (1 + sy * eta) * (1 + sz * zeta) / 8.0;
    g[1][a] = sy * (1 + sx * xi) * (1 + sz * zeta) / 8.0;
    g[2][a] = sz * (1 + sx * xi) * (1 + sy * eta) / 8.0;
  }
}

void element_tables(double E, double nu, double kappa, ElementTables* t) {
  std::memset(t, 0, sizeof(*t));
  // isotropic C with the float32 entries of utils/_utils.py:42
  double lam = nu / (1.0 + nu) / (1.0 - 2.0 * nu) * E;
  double mu = 1.0 / (2.0 * (1.0 + nu)) * E;
  double l2m = (double)(float)(lam + 2 * mu);
  lam = (double)(float)lam;
  mu = (double)(float)mu;
  double C[6][6] = {};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) C[i][j] = (i == j) ? l2m : lam;
  for (int i = 3; i < 6; ++i) C[i][i] = mu;

  const double gp[3] = {-std::sqrt(3.0 / 5.0), 0.0, std::sqrt(3.0 / 5.0)};
  const double gw[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
  const double h = 0.5;  // half edge of a unit voxel (r = 1)
  for (int ii = 0; ii < 3; ++ii)
    for (int jj = 0; jj < 3; ++jj)
      for (int kk = 0; kk < 3; ++kk) {
        double g[3][8];
        shape_grads(gp[ii], gp[jj], gp[kk], g);
        // Jacobian of the axis-aligned cube is diag(h); d/dx = (1/h) d/dxi
        double w = gw[ii] * gw[jj] * gw[kk] * h * h * h;
        double dN[3][8];
        for (int c = 0; c < 3; ++c)
          for (int a = 0; a < 8; ++a) dN[c][a] = g[c][a] / h;
        double B[6][24] = {};
        for (int a = 0; a < 8; ++a) {
          int c = 3 * a;
          B[0][c] = dN[0][a];
          B[1][c + 1] = dN[1][a];
          B[2][c + 2] = dN[2][a];
          B[3][c] = dN[1][a]; B[3][c + 1] = dN[0][a];
          B[4][c + 1] = dN[2][a]; B[4][c + 2] = dN[1][a];
          B[5][c] = dN[2][a]; B[5][c + 2] = dN[0][a];
        }
        double CB[6][24] = {};
        for (int p = 0; p < 6; ++p)
          for (int q = 0; q < 24; ++q)
            for (int s = 0; s < 6; ++s) CB[p][q] += C[p][s] * B[s][q];
        for (int p = 0; p < 24; ++p) {
          for (int q = 0; q < 24; ++q) {
            double s = 0;
            for (int m = 0; m < 6; ++m) s += B[m][p] * CB[m][q];
            t->Ke3[p * 24 + q] += w * s;
          }
          for (int q = 0; q < 6; ++q) t->Fe3[p * 6 + q] += w * (B[0][p] * C[0][q] + B[1][p] * C[1][q] + B[2][p] * C[2][q] +
                                                                 B[3][p] * C[3][q] + B[4][p] * C[4][q] + B[5][p] * C[5][q]);
        }
        for (int a = 0; a < 8; ++a) {
          for (int b = 0; b < 8; ++b)
            t->Ke1[a * 8 + b] += w * kappa * (dN[0][a] * dN[0][b] + dN[1][a] * dN[1][b] + dN[2][a] * dN[2][b]);
          for (int c = 0; c < 3; ++c) t->Fe1[a * 3 + c] += w * kappa * dN[c][a];
        }
      }
  // X0: pinned element solves (utils/_utils.py:105-108, 188-195)
  {
    const int fixed[6] = {0, 1, 2, 4, 5, 11};
    int freeidx[18], nf = 0;
    for (int i = 0; i < 24; ++i) {
      bool f = false;
      for (int k = 0; k < 6; ++k) f |= (fixed[k] == i);
      if (!f) freeidx[nf++] = i;
    }
    double A[18 * 18], Bm[18 * 6];
    for (int i = 0; i < nf; ++i) {
      for (int j = 0; j < nf; ++j) A[i * nf + j] = t->Ke3[freeidx[i] * 24 + freeidx[j]];
      for (int j = 0; j < 6; ++j) Bm[i * 6 + j] = t->Fe3[freeidx[i] * 6 + j];
    }
    solve_dense(nf, A, Bm, 6);
    for (int i = 0; i < nf; ++i)
      for (int j = 0; j < 6; ++j) t->X03[freeidx[i] * 6 + j] = Bm[i * 6 + j];
  }
  {
    double A[7 * 7], Bm[7 * 3];
    for (int i = 0; i < 7; ++i) {
      for (int j = 0; j < 7; ++j) A[i * 7 + j] = t->Ke1[(i + 1) * 8 + (j + 1)];
      for (int j = 0; j < 3; ++j) Bm[i * 3 + j] = t->Fe1[(i + 1) * 3 + j];
    }
    solve_dense(7, A, Bm, 3);
    for (int i = 0; i < 7; ++i)
      for (int j = 0; j < 3; ++j) t->X01[(i + 1) * 3 + j] = Bm[i * 3 + j];
  }
  // Ke0 X0 (used by the energy sums)
  for (int p = 0; p < 24; ++p)
    for (int q = 0; q < 6; ++q) {
      double s = 0;
      for (int m = 0; m < 24; ++m) s += t->Ke3[p * 24 + m] * t->X03[m * 6 + q];
      t->KX3[p * 6 + q] = s;
    }
  for (int p = 0; p < 8; ++p)
    for (int q = 0; q < 3; ++q) {
      double s = 0;
      for (int m = 0; m < 8; ++m) s += t->Ke1[p * 8 + m] * t->X01[m * 3 + q];
      t->KX1[p * 3 + q] = s;
    }
  // child prolongation weights: W[c][a][b] = weight of coarse corner b at the
  // corner a of child c (child c = 4*cx + 2*cy + cz inside the coarse element)
  for (int c = 0; c < 8; ++c) {
    int co[3] = {(c >> 2) & 1, (c >> 1) & 1, c & 1};
    for (int a = 0; a < 8; ++a)
      for (int b = 0; b < 8; ++b) {
        double w = 1;
        for (int ax = 0; ax < 3; ++ax) {
          double p = co[ax] + kCorner[a][ax];
          w *= 1.0 - std::fabs(p / 2.0 - kCorner[b][ax]);
        }
        t->W[(c * 8 + a) * 8 + b] = w;
      }
  }
  // M_c = (W_c (x) I)^T Ke0 (W_c (x) I): level-1 coarse element matrix of a
  // child of unit density, for both physics
  for (int c = 0; c < 8; ++c) {
    const double* W = &t->W[c * 64];
    for (int a = 0; a < 8; ++a)
      for (int b = 0; b < 8; ++b) {
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) {
            double s = 0;
            for (int a2 = 0; a2 < 8; ++a2)
              for (int b2 = 0; b2 < 8; ++b2) s += W[a2 * 8 + a] * W[b2 * 8 + b] * t->Ke3[(3 * a2 + i) * 24 + 3 * b2 + j];
            t->M3[(c * 24 + 3 * a + i) * 24 + 3 * b + j] = s;
          }
        double s = 0;
        for (int a2 = 0; a2 < 8; ++a2)
          for (int b2 = 0; b2 < 8; ++b2) s += W[a2 * 8 + a] * W[b2 * 8 + b] * t->Ke1[a2 * 8 + b2];
        t->M1[(c * 8 + a) * 8 + b] = s;
      }
  }
  for (int f = 0; f < 64; ++f) {
    const int fx = f >> 4, fy = (f >> 2) & 3, fz = f & 3;
    const int c1 = ((fx >> 1) << 2) | ((fy >> 1) << 1) | (fz >> 1);
    const int c0 = ((fx & 1) << 2) | ((fy & 1) << 1) | (fz & 1);
    const double* W = &t->W[c1 * 64];
    for (int a = 0; a < 8; ++a)
      for (int b = 0; b < 8; ++b) {
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) {
            double s = 0;
            for (int a2 = 0; a2 < 8; ++a2)
              for (int b2 = 0; b2 < 8; ++b2)
                s += W[a2 * 8 + a] * W[b2 * 8 + b] * t->M3[(c0 * 24 + 3 * a2 + i) * 24 + 3 * b2 + j];
            t->G3[(f * 24 + 3 * a + i) * 24 + 3 * b + j] = s;
          }
        double s = 0;
        for (int a2 = 0; a2 < 8; ++a2)
          for (int b2 = 0; b2 < 8; ++b2) s += W[a2 * 8 + a] * W[b2 * 8 + b] * t->M1[(c0 * 8 + a2) * 8 + b2];
        t->G1[(f * 8 + a) * 8 + b] = s;
      }
  }
  // Upper bound of lambda_max(D^-1 A) for any assembly of scaled copies of Ke0,
  // D = assembled (block) diagonal: max_e lambda_max(D_e^-1 K_e), obtained by
  // power iteration on the element matrix (it is the same for every element).
  for (int phys = 0; phys < 2; ++phys) {
    int D = phys == 0 ? 3 : 1, k = 8 * D;
    const double* K = phys == 0 ? t->Ke3 : t->Ke1;
    // block-diagonal inverse
    double Binv[24 * 24] = {};
    for (int a = 0; a < 8; ++a) {
      double blk[9], inv[9] = {};
      for (int i = 0; i < D; ++i)
        for (int j = 0; j < D; ++j) blk[i * D + j] = K[(D * a + i) * k + D * a + j];
      for (int i = 0; i < D; ++i) inv[i * D + i] = 1.0;
      solve_dense(D, blk, inv, D);
      for (int i = 0; i < D; ++i)
        for (int j = 0; j < D; ++j) Binv[(D * a + i) * k + D * a + j] = inv[i * D + j];
    }
    double v[24], w[24], lam_est = 0;
    for (int i = 0; i < k; ++i) v[i] = 1.0 + 0.37 * i - 0.05 * i * i;
    for (int it = 0; it < 500; ++it) {
      double Kv[24];
      for (int i = 0; i < k; ++i) {
        double s = 0;
        for (int j = 0; j < k; ++j) s += K[i * k + j] * v[j];
        Kv[i] = s;
      }
      double nrm = 0;
      for (int i = 0; i < k; ++i) {
        double s = 0;
        for (int j = 0; j < k; ++j) s += Binv[i * k + j] * Kv[j];
        w[i] = s;
        nrm += s * s;
      }
      nrm = std::sqrt(nrm);
      double vn = 0;
      for (int i = 0; i < k; ++i) vn += v[i] * v[i];
      lam_est = nrm / std::sqrt(vn);
      for (int i = 0; i < k; ++i) v[i] = w[i] / nrm;
    }
    t->lam_elem[phys] = lam_est;
  }
}

}  // namespace maple
