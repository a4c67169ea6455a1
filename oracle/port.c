/*
 * Multithreaded C restatement of the FP64 oracle (oracle/ihd_oracle.py).
 *
 * TEST AND MEASUREMENT INFRASTRUCTURE ONLY.  It is the CPU baseline that
 * bench.py times beside the GPU path (the reference's own path is Python and
 * cannot run on the measuring host), and tests/test_port_oracle.py checks it
 * against the numpy oracle.  The product (maple_b200) never links or calls it.
 *
 * It runs the reference's algorithm (xing-yuu/MAPLE, paths under
 * src/maple/core) on all host cores with OpenMP:
 *   - periodic voxel operator K(rho) with Ke_e = rho_e Ke0 (utils/model.py:108,
 *     utils/EBE_GMG.py:412-430), applied as the assembled 27-point node
 *     stencil of the same element sums;
 *   - Galerkin coarse element matrices Kc = sum_children Pc^T K_child Pc with
 *     trilinear Pc (utils/EBE_GMG.py:202-337, utils/EBE_GMG_scalar.py:135-230);
 *   - V-cycles (utils/EBE_GMG.py:886-984) with 8-colour Gauss-Seidel, omega 1,
 *     point-diagonal inverse (EBE_GMG.py:354-459), pre/post sweeps
 *     smooth_iter = [2,2,3,4,5]; the elastic recursion smooths coarse levels
 *     with one sweep (EBE_GMG.py:955-963 does not forward smooth_iter), the
 *     scalar one forwards it (EBE_GMG_scalar.py:802-811); the coarsest level
 *     gets one extra sweep;
 *   - cycles from the given start until every load case has
 *     ||f - K u|| <= rtol ||f|| (the reference runs a fixed count);
 *   - energy sums C^H / kappa^H (utils/model.py:33-95), objective terms
 *     (utils/objective.py:11-41), the analytic adjoint of the autograd call
 *     (main_IHD_v3.py:688), the periodic k^3 box filter
 *     (main_IHD_v3.py:342-359) and the 60-step OC bisection
 *     (main_IHD_v3.py:362-380).
 *
 * Layouts follow the oracle: node / element id x*n*n + y*n + z; vectors
 * [node][D][R]; element-local corners 000,100,110,010,001,101,111,011.
 */
#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

static const int HX[8] = {0, 1, 1, 0, 0, 1, 1, 0};
static const int HY[8] = {0, 0, 1, 1, 0, 0, 1, 1};
static const int HZ[8] = {0, 0, 0, 0, 1, 1, 1, 1};

static inline int wrapi(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

typedef struct {
  int n;
  double* S;     /* node stencils [N][27][D][D] */
  double* dinv;  /* [N][D] */
  double* ke;    /* element matrices [N][8D][8D] (levels >= 1; NULL on level 0) */
  double *u, *f, *r; /* [N][D][R] (u, f: levels >= 1; r: all) */
} Level;

/* ------------------------------------------------------------------------ */
/* operator hierarchy                                                       */
/* ------------------------------------------------------------------------ */

/* S[node][k] = sum over the 8 elements around the node of the element block
 * coupling it (local corner a) to the neighbour at local corner b; level 0
 * uses rho_e * Ke0. */
static void assemble_stencil(int n, int D, const double* ke, const double* rho, const double* Ke0, double* S) {
  const int N = n * n * n, K = 8 * D, DD = D * D;
#pragma omp parallel for schedule(static)
  for (int node = 0; node < N; ++node) {
    double* s = S + (size_t)node * 27 * DD;
    memset(s, 0, sizeof(double) * 27 * DD);
    const int x = node / (n * n), y = (node / n) % n, z = node % n;
    for (int a = 0; a < 8; ++a) {
      const int e = (wrapi(x - HX[a], n) * n + wrapi(y - HY[a], n)) * n + wrapi(z - HZ[a], n);
      const double* Ke = ke ? ke + (size_t)e * K * K : Ke0;
      const double sc = ke ? 1.0 : rho[e];
      for (int b = 0; b < 8; ++b) {
        const int k = (HX[b] - HX[a] + 1) * 9 + (HY[b] - HY[a] + 1) * 3 + (HZ[b] - HZ[a] + 1);
        for (int d = 0; d < D; ++d)
          for (int c = 0; c < D; ++c) s[k * DD + d * D + c] += sc * Ke[(a * D + d) * K + b * D + c];
      }
    }
  }
}

static void diag_inverse(int n, int D, const double* S, double* dinv) {
  const int N = n * n * n, DD = D * D;
#pragma omp parallel for schedule(static)
  for (int node = 0; node < N; ++node)
    for (int d = 0; d < D; ++d) {
      const double v = S[(size_t)node * 27 * DD + 13 * DD + d * D + d];
      dinv[(size_t)node * D + d] = v == 0.0 ? 1.0 : 1.0 / v; /* EBE_GMG.py:387-388 */
    }
}

/* trilinear weight of coarse corner b at fine position p in {0,1,2}^3 */
static double pchild(int c, int a, int b) {
  const int p[3] = {((c >> 2) & 1) + HX[a], ((c >> 1) & 1) + HY[a], (c & 1) + HZ[a]};
  const int o[3] = {HX[b], HY[b], HZ[b]};
  double w = 1.0;
  for (int i = 0; i < 3; ++i) w *= 1.0 - fabs(0.5 * p[i] - o[i]);
  return w;
}

/* Kc_E = sum_c (Pc x I)^T K_child (Pc x I), child c = (x%2)*4 + (y%2)*2 + z%2 */
static void coarsen(int n, int D, const double* ke, const double* rho, const double* Ke0, double* kc) {
  const int nc = n / 2, K = 8 * D, NC = nc * nc * nc;
  double P[8][8][8];
  for (int c = 0; c < 8; ++c)
    for (int a = 0; a < 8; ++a)
      for (int b = 0; b < 8; ++b) P[c][a][b] = pchild(c, a, b);
#pragma omp parallel
  {
    double* T = (double*)malloc(sizeof(double) * K * K);
#pragma omp for schedule(static)
    for (int E = 0; E < NC; ++E) {
      double* out = kc + (size_t)E * K * K;
      memset(out, 0, sizeof(double) * K * K);
      const int X = E / (nc * nc), Y = (E / nc) % nc, Z = E % nc;
      for (int c = 0; c < 8; ++c) {
        const int ex = 2 * X + ((c >> 2) & 1), ey = 2 * Y + ((c >> 1) & 1), ez = 2 * Z + (c & 1);
        const int e = (ex * n + ey) * n + ez;
        const double* Ke = ke ? ke + (size_t)e * K * K : Ke0;
        const double sc = ke ? 1.0 : rho[e];
        /* T = Ke (P x I): T[i][b*D+d] = sum_a Ke[i][a*D+d] P[a][b] */
        for (int i = 0; i < K; ++i)
          for (int b = 0; b < 8; ++b)
            for (int d = 0; d < D; ++d) {
              double t = 0.0;
              for (int a = 0; a < 8; ++a) t += Ke[i * K + a * D + d] * P[c][a][b];
              T[i * K + b * D + d] = sc * t;
            }
        /* out += (P x I)^T T */
        for (int b = 0; b < 8; ++b)
          for (int d = 0; d < D; ++d)
            for (int j = 0; j < K; ++j) {
              double t = 0.0;
              for (int a = 0; a < 8; ++a) t += P[c][a][b] * T[(a * D + d) * K + j];
              out[(b * D + d) * K + j] += t;
            }
      }
    }
    free(T);
  }
}

/* ------------------------------------------------------------------------ */
/* level operations, specialised for (D, R) = (3, 6) and (1, 3)             */
/* ------------------------------------------------------------------------ */
#define DEF_OPS(D, R)                                                                                            \
  static inline void resid_##D(int n, const double* S, const double* u, const double* f, int node, double* out) { \
    const int x = node / (n * n), y = (node / n) % n, z = node % n;                                              \
    for (int i = 0; i < D * R; ++i) out[i] = f[(size_t)node * D * R + i];                                        \
    const double* s = S + (size_t)node * 27 * D * D;                                                             \
    int k = 0;                                                                                                   \
    for (int dx = -1; dx <= 1; ++dx) {                                                                           \
      const int xx = wrapi(x + dx, n);                                                                           \
      for (int dy = -1; dy <= 1; ++dy) {                                                                         \
        const int yy = wrapi(y + dy, n);                                                                         \
        for (int dz = -1; dz <= 1; ++dz, ++k) {                                                                  \
          const double* un = u + (size_t)((xx * n + yy) * n + wrapi(z + dz, n)) * D * R;                         \
          const double* sk = s + k * D * D;                                                                      \
          for (int d = 0; d < D; ++d)                                                                            \
            for (int c = 0; c < D; ++c) {                                                                        \
              const double a = sk[d * D + c];                                                                    \
              for (int q = 0; q < R; ++q) out[d * R + q] -= a * un[c * R + q];                                   \
            }                                                                                                    \
        }                                                                                                        \
      }                                                                                                          \
    }                                                                                                            \
  }                                                                                                              \
  static void gs_##D(const Level* L, double* u, const double* f, int reverse) {                                  \
    const int n = L->n, h = n / 2 > 0 ? n / 2 : 1;                                                               \
    for (int cc = 0; cc < 8; ++cc) {                                                                             \
      const int c = reverse ? 7 - cc : cc;                                                                       \
      const int cx = (c >> 2) & 1, cy = (c >> 1) & 1, cz = c & 1;                                                \
      _Pragma("omp parallel for schedule(static)") for (int i = 0; i < h * h * h; ++i) {                        \
        const int x = 2 * (i / (h * h)) + cx, y = 2 * ((i / h) % h) + cy, z = 2 * (i % h) + cz;                 \
        if (x >= n || y >= n || z >= n) continue;                                                                \
        const int node = (x * n + y) * n + z;                                                                    \
        double r[D * R];                                                                                         \
        resid_##D(n, L->S, u, f, node, r);                                                                       \
        for (int d = 0; d < D; ++d)                                                                              \
          for (int q = 0; q < R; ++q) u[(size_t)node * D * R + d * R + q] += L->dinv[(size_t)node * D + d] * r[d * R + q]; \
      }                                                                                                          \
    }                                                                                                            \
  }                                                                                                              \
  static void matvec_##D(const Level* L, const double* u, double* out) {                                         \
    const int n = L->n, N = n * n * n;                                                                           \
    _Pragma("omp parallel for schedule(static)") for (int node = 0; node < N; ++node) {                          \
      const int x = node / (n * n), y = (node / n) % n, z = node % n;                                            \
      double acc[D * R];                                                                                         \
      for (int i = 0; i < D * R; ++i) acc[i] = 0.0;                                                              \
      const double* s = L->S + (size_t)node * 27 * D * D;                                                        \
      int k = 0;                                                                                                 \
      for (int dx = -1; dx <= 1; ++dx)                                                                           \
        for (int dy = -1; dy <= 1; ++dy)                                                                         \
          for (int dz = -1; dz <= 1; ++dz, ++k) {                                                                \
            const double* un = u + (size_t)((wrapi(x + dx, n) * n + wrapi(y + dy, n)) * n + wrapi(z + dz, n)) * D * R; \
            const double* sk = s + k * D * D;                                                                    \
            for (int d = 0; d < D; ++d)                                                                          \
              for (int c = 0; c < D; ++c) {                                                                      \
                const double a = sk[d * D + c];                                                                  \
                for (int q = 0; q < R; ++q) acc[d * R + q] += a * un[c * R + q];                                 \
              }                                                                                                  \
          }                                                                                                      \
      for (int i = 0; i < D * R; ++i) out[(size_t)node * D * R + i] = acc[i];                                    \
    }                                                                                                            \
  }                                                                                                              \
  static void residual_##D(const Level* L, const double* u, const double* f, double* out) {                      \
    const int n = L->n, N = n * n * n;                                                                           \
    _Pragma("omp parallel for schedule(static)") for (int node = 0; node < N; ++node)                            \
        resid_##D(n, L->S, u, f, node, out + (size_t)node * D * R);                                              \
  }

DEF_OPS(3, 6)
DEF_OPS(1, 3)

static void gs_sweeps(const Level* L, int D, double* u, const double* f, int sweeps, int reverse) {
  for (int s = 0; s < sweeps; ++s) {
    if (D == 3)
      gs_3(L, u, f, reverse);
    else
      gs_1(L, u, f, reverse);
  }
}

static void residual(const Level* L, int D, const double* u, const double* f, double* out) {
  if (D == 3)
    residual_3(L, u, f, out);
  else
    residual_1(L, u, f, out);
}

/* rc = P^T r: coarse node J gathers fine 2J + delta, weights prod w(delta_i),
 * w(0) = 1, w(+-1) = 1/2 (the transpose of the P of EBE_GMG.py:531-647) */
static void restrict_(int nf, int DR, const double* r, double* rc) {
  const int nc = nf / 2, NC = nc * nc * nc;
  static const double w[3] = {0.5, 1.0, 0.5};
#pragma omp parallel for schedule(static)
  for (int J = 0; J < NC; ++J) {
    const int X = J / (nc * nc), Y = (J / nc) % nc, Z = J % nc;
    double* o = rc + (size_t)J * DR;
    for (int i = 0; i < DR; ++i) o[i] = 0.0;
    for (int dx = -1; dx <= 1; ++dx)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dz = -1; dz <= 1; ++dz) {
          const int fi = (wrapi(2 * X + dx, nf) * nf + wrapi(2 * Y + dy, nf)) * nf + wrapi(2 * Z + dz, nf);
          const double ww = w[dx + 1] * w[dy + 1] * w[dz + 1];
          for (int i = 0; i < DR; ++i) o[i] += ww * r[(size_t)fi * DR + i];
        }
  }
}

/* u += P uc: even fine index takes coarse i/2, odd takes (i-1)/2 and (i+1)/2
 * with 1/2 each (weights prod(1 - |rem/2 - off|), EBE_GMG.py:531-647) */
static void prolong_add(int nf, int DR, const double* uc, double* u) {
  const int nc = nf / 2, N = nf * nf * nf;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < N; ++i) {
    const int p[3] = {i / (nf * nf), (i / nf) % nf, i % nf};
    int lo[3], cnt[3];
    double wt[3];
    for (int a = 0; a < 3; ++a) {
      lo[a] = p[a] / 2;
      cnt[a] = (p[a] & 1) ? 2 : 1;
      wt[a] = (p[a] & 1) ? 0.5 : 1.0;
    }
    for (int ax = 0; ax < cnt[0]; ++ax)
      for (int ay = 0; ay < cnt[1]; ++ay)
        for (int az = 0; az < cnt[2]; ++az) {
          const int J = (wrapi(lo[0] + ax, nc) * nc + wrapi(lo[1] + ay, nc)) * nc + wrapi(lo[2] + az, nc);
          const double ww = wt[0] * wt[1] * wt[2];
          for (int k = 0; k < DR; ++k) u[(size_t)i * DR + k] += ww * uc[(size_t)J * DR + k];
        }
  }
}

typedef struct {
  int L, D, R;
  Level lv[8];
} Hier;

static int smooth_count(int D, int l) {
  static const int si[5] = {2, 2, 3, 4, 5};
  if (D == 3) return l == 0 ? si[0] : 1;
  return si[l < 4 ? l : 4];
}

/* sym: post-smoothing (and the coarsest level's second half) in reverse
 * colour order, a symmetric cycle (the oracle's vcycle(symmetric=True)) */
static void vcycle(Hier* H, int l, double* u, const double* f, int sym) {
  Level* L = &H->lv[l];
  const int D = H->D, DR = H->D * H->R, nu = smooth_count(D, l);
  gs_sweeps(L, D, u, f, nu, 0);
  if (l == H->L - 1) {
    gs_sweeps(L, D, u, f, sym ? nu : 1, sym);
    return;
  }
  Level* C = &H->lv[l + 1];
  residual(L, D, u, f, L->r);
  restrict_(L->n, DR, L->r, C->f);
  memset(C->u, 0, sizeof(double) * (size_t)C->n * C->n * C->n * DR);
  vcycle(H, l + 1, C->u, C->f, sym);
  prolong_add(L->n, DR, C->u, u);
  gs_sweeps(L, D, u, f, nu, sym);
}

static void build(Hier* H, int n, int levels, int D, int R, const double* rho, const double* Ke0) {
  H->D = D;
  H->R = R;
  H->L = 0;
  const double* ke = NULL;
  for (int l = 0; l < levels; ++l) {
    if (l > 0 && (n % 2 || n < 2)) break;
    Level* L = &H->lv[l];
    memset(L, 0, sizeof(*L));
    if (l > 0) {
      const int nc = n / 2, K = 8 * D;
      L->ke = (double*)malloc(sizeof(double) * (size_t)nc * nc * nc * K * K);
      coarsen(n, D, ke, rho, Ke0, L->ke);
      n = nc;
      ke = L->ke;
    }
    const size_t N = (size_t)n * n * n;
    L->n = n;
    L->S = (double*)malloc(sizeof(double) * N * 27 * D * D);
    L->dinv = (double*)malloc(sizeof(double) * N * D);
    assemble_stencil(n, D, l ? L->ke : NULL, rho, Ke0, L->S);
    diag_inverse(n, D, L->S, L->dinv);
    L->r = (double*)malloc(sizeof(double) * N * D * R);
    if (l > 0) {
      L->u = (double*)malloc(sizeof(double) * N * D * R);
      L->f = (double*)malloc(sizeof(double) * N * D * R);
    }
    H->L = l + 1;
  }
}

static void destroy(Hier* H) {
  for (int l = 0; l < H->L; ++l) {
    free(H->lv[l].S);
    free(H->lv[l].dinv);
    free(H->lv[l].ke);
    free(H->lv[l].u);
    free(H->lv[l].f);
    free(H->lv[l].r);
  }
}

/* per-column ||v||^2 of [N][D][R] */
static void col_norms2(size_t N, int D, int R, const double* v, double* out) {
  for (int q = 0; q < R; ++q) out[q] = 0.0;
#pragma omp parallel
  {
    double loc[6] = {0, 0, 0, 0, 0, 0};
#pragma omp for schedule(static)
    for (size_t i = 0; i < N; ++i)
      for (int d = 0; d < D; ++d)
        for (int q = 0; q < R; ++q) {
          const double t = v[i * D * R + d * R + q];
          loc[q] += t * t;
        }
#pragma omp critical
    for (int q = 0; q < R; ++q) out[q] += loc[q];
  }
}

/* F = sum_e rho_e Fe0 at the element's corners (utils/_utils.py:453-507) */
static void assemble_rhs(int n, int D, int R, const double* rho, const double* Fe0, double* F) {
  const int N = n * n * n;
#pragma omp parallel for schedule(static)
  for (int node = 0; node < N; ++node) {
    const int x = node / (n * n), y = (node / n) % n, z = node % n;
    double* o = F + (size_t)node * D * R;
    for (int i = 0; i < D * R; ++i) o[i] = 0.0;
    for (int a = 0; a < 8; ++a) {
      const int e = (wrapi(x - HX[a], n) * n + wrapi(y - HY[a], n)) * n + wrapi(z - HZ[a], n);
      for (int d = 0; d < D; ++d)
        for (int q = 0; q < R; ++q) o[d * R + q] += rho[e] * Fe0[(a * D + d) * R + q];
    }
  }
}

/* per-column sum of a*b over [N][D][R] */
static void col_dots(size_t N, int D, int R, const double* a, const double* b, double* out) {
  for (int q = 0; q < R; ++q) out[q] = 0.0;
#pragma omp parallel
  {
    double loc[6] = {0, 0, 0, 0, 0, 0};
#pragma omp for schedule(static)
    for (size_t i = 0; i < N; ++i)
      for (int d = 0; d < D; ++d)
        for (int q = 0; q < R; ++q) loc[q] += a[i * D * R + d * R + q] * b[i * D * R + d * R + q];
#pragma omp critical
    for (int q = 0; q < R; ++q) out[q] += loc[q];
  }
}

/* The symmetric V-cycle (one cycle from zero on the residual) as the
 * preconditioner of a conjugate gradient, per load case (Polak-Ribiere
 * beta): the oracle's gmg_solve(method="pcg").  Returns the iterations. */
static int solve_pcg(Hier* H, double* u, const double* f, double rtol, int max_it) {
  Level* L0 = &H->lv[0];
  const size_t N = (size_t)L0->n * L0->n * L0->n;
  const int D = H->D, R = H->R, DR = D * R;
  const size_t len = N * DR;
  double *r = (double*)malloc(sizeof(double) * len), *z = (double*)malloc(sizeof(double) * len);
  double *p = (double*)malloc(sizeof(double) * len), *q = (double*)malloc(sizeof(double) * len);
  double* ro = (double*)malloc(sizeof(double) * len);
  double fn[6], rn[6], rz[6], pq[6], zr[6], alpha[6], beta[6];
  col_norms2(N, D, R, f, fn);
  residual(L0, D, u, f, r);
  int it = 0;
  col_norms2(N, D, R, r, rn);
  int ok = 1;
  for (int c = 0; c < R; ++c) ok &= sqrt(rn[c]) <= rtol * fmax(sqrt(fn[c]), 1e-300);
  if (!(rtol > 0 && ok)) {
    memset(z, 0, sizeof(double) * len);
    vcycle(H, 0, z, r, 1);
    memcpy(p, z, sizeof(double) * len);
    col_dots(N, D, R, r, z, rz);
    for (it = 1; it <= max_it; ++it) {
      if (D == 3)
        matvec_3(L0, p, q);
      else
        matvec_1(L0, p, q);
      col_dots(N, D, R, p, q, pq);
      for (int c = 0; c < R; ++c) alpha[c] = pq[c] > 0 ? rz[c] / pq[c] : 0.0;
      memcpy(ro, r, sizeof(double) * len);
#pragma omp parallel for schedule(static)
      for (size_t i = 0; i < N; ++i)
        for (int k = 0; k < DR; ++k) {
          const double a = alpha[k % R];
          u[i * DR + k] += a * p[i * DR + k];
          r[i * DR + k] -= a * q[i * DR + k];
        }
      col_norms2(N, D, R, r, rn);
      ok = 1;
      for (int c = 0; c < R; ++c) ok &= sqrt(rn[c]) <= rtol * fmax(sqrt(fn[c]), 1e-300);
      if (rtol > 0 && ok) break;
      memset(z, 0, sizeof(double) * len);
      vcycle(H, 0, z, r, 1);
#pragma omp parallel for schedule(static)
      for (size_t i = 0; i < len; ++i) ro[i] = r[i] - ro[i];
      col_dots(N, D, R, z, ro, zr);
      for (int c = 0; c < R; ++c) beta[c] = rz[c] != 0 ? zr[c] / rz[c] : 0.0;
      col_dots(N, D, R, r, z, rz);
#pragma omp parallel for schedule(static)
      for (size_t i = 0; i < N; ++i)
        for (int k = 0; k < DR; ++k) p[i * DR + k] = z[i * DR + k] + beta[k % R] * p[i * DR + k];
    }
    if (it > max_it) it = max_it;
  }
  free(r);
  free(z);
  free(p);
  free(q);
  free(ro);
  return it;
}

/* V-cycles until every column has ||f - K u|| <= rtol ||f||; returns cycles */
static int solve(Hier* H, double* u, const double* f, double rtol, int max_cycles) {
  Level* L0 = &H->lv[0];
  const size_t N = (size_t)L0->n * L0->n * L0->n;
  const int D = H->D, R = H->R;
  double fn[6], rn[6];
  col_norms2(N, D, R, f, fn);
  int it = 0;
  for (it = 1; it <= max_cycles; ++it) {
    vcycle(H, 0, u, f, 0);
    residual(L0, D, u, f, L0->r);
    col_norms2(N, D, R, L0->r, rn);
    int ok = 1;
    for (int q = 0; q < R; ++q) ok &= sqrt(rn[q]) <= rtol * fmax(sqrt(fn[q]), 1e-300);
    if (rtol > 0 && ok) break;
  }
  return it > max_cycles ? max_cycles : it;
}

/* C^H = sum_e (X0 - u_e)^T rho_e Ke0 (X0 - u_e) and per-element energies
 * (X0 - u_e)^T Ke0 (X0 - u_e) [N][R][R] (utils/model.py:33-95) */
static void homogenize(int n, int D, int R, const double* u, const double* rho, const double* Ke0, const double* X0,
                       double* Hout, double* energy) {
  const int N = n * n * n, K = 8 * D;
  for (int i = 0; i < R * R; ++i) Hout[i] = 0.0;
#pragma omp parallel
  {
    double Lm[24 * 6], KL[24 * 6], loc[36];
    for (int i = 0; i < R * R; ++i) loc[i] = 0.0;
#pragma omp for schedule(static)
    for (int e = 0; e < N; ++e) {
      const int x = e / (n * n), y = (e / n) % n, z = e % n;
      for (int a = 0; a < 8; ++a) {
        const int node = (wrapi(x + HX[a], n) * n + wrapi(y + HY[a], n)) * n + wrapi(z + HZ[a], n);
        for (int d = 0; d < D; ++d)
          for (int q = 0; q < R; ++q)
            Lm[(a * D + d) * R + q] = X0[(a * D + d) * R + q] - u[(size_t)node * D * R + d * R + q];
      }
      for (int i = 0; i < K; ++i)
        for (int q = 0; q < R; ++q) {
          double t = 0.0;
          for (int j = 0; j < K; ++j) t += Ke0[i * K + j] * Lm[j * R + q];
          KL[i * R + q] = t;
        }
      double* en = energy + (size_t)e * R * R;
      for (int p = 0; p < R; ++p)
        for (int q = 0; q < R; ++q) {
          double t = 0.0;
          for (int i = 0; i < K; ++i) t += Lm[i * R + p] * KL[i * R + q];
          en[p * R + q] = t;
          loc[p * R + q] += rho[e] * t;
        }
    }
#pragma omp critical
    for (int i = 0; i < R * R; ++i) Hout[i] += loc[i];
  }
}

/* inverse of a 6x6 matrix by Gauss-Jordan with partial pivoting */
static void inv6(const double* A, double* Ainv) {
  double M[6][12];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 12; ++j) M[i][j] = j < 6 ? A[i * 6 + j] : (j - 6 == i ? 1.0 : 0.0);
  for (int c = 0; c < 6; ++c) {
    int p = c;
    for (int i = c + 1; i < 6; ++i)
      if (fabs(M[i][c]) > fabs(M[p][c])) p = i;
    if (p != c)
      for (int j = 0; j < 12; ++j) {
        const double t = M[c][j];
        M[c][j] = M[p][j];
        M[p][j] = t;
      }
    const double piv = M[c][c];
    for (int j = 0; j < 12; ++j) M[c][j] /= piv;
    for (int i = 0; i < 6; ++i)
      if (i != c) {
        const double f = M[i][c];
        for (int j = 0; j < 12; ++j) M[i][j] -= f * M[c][j];
      }
  }
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) Ainv[i * 6 + j] = M[i][j + 6];
}

/* J = wE E + wG G + wK trace(kappa) and dJ/dC^H, dJ/dkappa
 * (utils/objective.py:11-41, 180-251) */
static double objective(const double* w3, const double* CH, const double* kap, double* gC, double* gK) {
  double A[36], S[36];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) A[i * 6 + j] = 0.5 * (CH[i * 6 + j] + CH[j * 6 + i]) + (i == j ? 1e-9 : 0.0);
  inv6(A, S);
  double J = 0.0;
  for (int i = 0; i < 36; ++i) gC[i] = 0.0;
  for (int i = 0; i < 9; ++i) gK[i] = 0.0;
  for (int t = 0; t < 2; ++t) {
    const double w = w3[t];
    if (w == 0.0) continue;
    double m = 0.0, G[36];
    for (int i = 0; i < 36; ++i) G[i] = 0.0;
    for (int i = 3 * t; i < 3 * t + 3; ++i) {
      m += 1.0 / S[i * 6 + i];
      for (int a = 0; a < 6; ++a)
        for (int b = 0; b < 6; ++b) G[a * 6 + b] += S[a * 6 + i] * S[i * 6 + b] / (S[i * 6 + i] * S[i * 6 + i]);
    }
    J += w * m / 3.0;
    for (int a = 0; a < 6; ++a)
      for (int b = 0; b < 6; ++b) gC[a * 6 + b] += w * 0.5 * (G[a * 6 + b] + G[b * 6 + a]) / 3.0;
  }
  if (w3[2] != 0.0) {
    J += w3[2] * (kap[0] + kap[4] + kap[8]);
    gK[0] = gK[4] = gK[8] = w3[2];
  }
  return J;
}

int port_threads(int nthreads) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
  return omp_get_max_threads();
}

/*
 * One OC iteration (main_IHD_v3.py:620-716, symmetry "none", no penalties)
 * of one r^3 cell.  tabs: Ke3[576] Fe3[144] X03[144] Ke1[64] Fe1[24] X01[24]
 * of the voxel (edge 1/r).  w3: (w_E, w_G, w_kappa).  u3 [N][3][6] / u1
 * [N][1][3]: initial iterates when warm3 / warm1, else zero; they return
 * the solutions.  method 0: V-cycles to rtol (the reference's iteration);
 * 1: the V-cycle as the preconditioner of a flexible CG.  out: J, C^H[36],
 * kappa[9], elastic and thermal cycles (or CG iterations), max|dx|,
 * mean|dx| (50 values).  Returns 0, or 1 on a bad argument.
 */
int port_oc_iteration(int r, int levels, const double* tabs, const double* x, const double* w3, double vf,
                      double penal, double rho_min, double move, double xmin, int filter_k, double rtol,
                      int max_cycles, int method, double* u3, int warm3, double* u1, int warm1, double* x_next,
                      double* out) {
  if (r < 2 || r % 2 || levels < 1 || levels > 8 || (filter_k > 1 && filter_k % 2 == 0) || method < 0 ||
      method > 1)
    return 1;
  const int N = r * r * r;
  const double *Ke3 = tabs, *Fe3 = tabs + 576, *X03 = tabs + 720, *Ke1 = tabs + 864, *Fe1 = tabs + 928,
               *X01 = tabs + 952;
  double* xc = (double*)malloc(sizeof(double) * N);
  double* rho = (double*)malloc(sizeof(double) * N);
  double* dJ = (double*)calloc(N, sizeof(double));
  double* tmp = (double*)malloc(sizeof(double) * N);
#pragma omp parallel for schedule(static)
  for (int e = 0; e < N; ++e) {
    xc[e] = fmin(fmax(x[e], xmin), 1.0);
    rho[e] = rho_min + (1.0 - rho_min) * pow(xc[e], penal);
  }
  double CH[36] = {0}, kap[9] = {0}, gC[36], gK[9];
  for (int i = 0; i < 36; ++i) CH[i] = i % 7 == 0 ? 1.0 : 0.0;
  for (int i = 0; i < 9; ++i) kap[i] = i % 4 == 0 ? 1.0 : 0.0;
  double* en3 = NULL;
  double* en1 = NULL;
  int cyc[2] = {0, 0};
  for (int ph = 0; ph < 2; ++ph) {
    const int D = ph ? 1 : 3, R = ph ? 3 : 6;
    if ((ph == 0 && w3[0] == 0.0 && w3[1] == 0.0) || (ph == 1 && w3[2] == 0.0)) continue;
    const double *Ke0 = ph ? Ke1 : Ke3, *Fe0 = ph ? Fe1 : Fe3, *X0 = ph ? X01 : X03;
    double* u = ph ? u1 : u3;
    if (!(ph ? warm1 : warm3)) memset(u, 0, sizeof(double) * (size_t)N * D * R);
    Hier H;
    build(&H, r, levels, D, R, rho, Ke0);
    double* F = (double*)malloc(sizeof(double) * (size_t)N * D * R);
    assemble_rhs(r, D, R, rho, Fe0, F);
    cyc[ph] = method == 1 ? solve_pcg(&H, u, F, rtol, max_cycles) : solve(&H, u, F, rtol, max_cycles);
    free(F);
    destroy(&H);
    double* en = (double*)malloc(sizeof(double) * (size_t)N * R * R);
    homogenize(r, D, R, u, rho, Ke0, X0, ph ? kap : CH, en);
    if (ph)
      en1 = en;
    else
      en3 = en;
  }
  const double J = objective(w3, CH, kap, gC, gK);
  /* dJ/dx_e = p (1 - rho_min) xc^(p-1) sum_ij g_ij energy_e,ij (main_IHD_v3.py:688) */
#pragma omp parallel for schedule(static)
  for (int e = 0; e < N; ++e) {
    double s = 0.0;
    if (en3)
      for (int i = 0; i < 36; ++i) s += gC[i] * en3[(size_t)e * 36 + i];
    if (en1)
      for (int i = 0; i < 9; ++i) s += gK[i] * en1[(size_t)e * 9 + i];
    dJ[e] = s * penal * (1.0 - rho_min) * pow(xc[e], penal - 1.0);
  }
  free(en3);
  free(en1);
  /* periodic k^3 box mean (main_IHD_v3.py:342-359) */
  if (filter_k > 1) {
    const int p = filter_k / 2;
#pragma omp parallel for schedule(static)
    for (int e = 0; e < N; ++e) {
      const int xx = e / (r * r), yy = (e / r) % r, zz = e % r;
      double s = 0.0;
      for (int dx = -p; dx <= p; ++dx)
        for (int dy = -p; dy <= p; ++dy)
          for (int dz = -p; dz <= p; ++dz)
            s += dJ[((((xx + dx) % r + r) % r) * r + (((yy + dy) % r + r) % r)) * r + (((zz + dz) % r + r) % r)];
      tmp[e] = s / (double)(filter_k * filter_k * filter_k);
    }
    memcpy(dJ, tmp, sizeof(double) * N);
  }
  /* OC bisection; the design of the last step is returned (main_IHD_v3.py:362-380) */
  double l1 = 1e-12, l2 = 1e6;
  for (int it = 0; it < 60; ++it) {
    const double lam = 0.5 * (l1 + l2);
    double s = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : s)
    for (int e = 0; e < N; ++e) {
      const double xv = x[e];
      double xn = xv * sqrt(fmax(dJ[e], 1e-12) / lam);
      xn = fmin(fmax(xn, xv - move), xv + move);
      xn = fmin(fmax(xn, xmin), 1.0);
      x_next[e] = xn;
      s += xn;
    }
    if (s / N > vf)
      l1 = lam;
    else
      l2 = lam;
  }
  double dmax = 0.0, dsum = 0.0;
#pragma omp parallel for schedule(static) reduction(max : dmax) reduction(+ : dsum)
  for (int e = 0; e < N; ++e) {
    x_next[e] = fmin(fmax(x_next[e], xmin), 1.0);
    const double d = fabs(x_next[e] - x[e]);
    dmax = fmax(dmax, d);
    dsum += d;
  }
  out[0] = J;
  for (int i = 0; i < 36; ++i) out[1 + i] = CH[i];
  for (int i = 0; i < 9; ++i) out[37 + i] = kap[i];
  out[46] = cyc[0];
  out[47] = cyc[1];
  out[48] = dmax;
  out[49] = dsum / N;
  free(xc);
  free(rho);
  free(dJ);
  free(tmp);
  return 0;
}
