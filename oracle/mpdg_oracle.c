/*
 * mpdg_oracle.c -- FP64 CPU restatement of MeltPoolDG's matrix-free heat and
 * advection-diffusion operators.  TEST INFRASTRUCTURE ONLY (the checker of the
 * CUDA path; see mpdg_oracle.h for the reference call sites restated here).
 *
 * Two independent evaluation routes are provided:
 *   orc_vmult        sum factorisation: nodal values -> (S,D) 1D contractions ->
 *                    quadrature-point kernel -> transposed contractions
 *                    (what deal.II's FEEvaluation::evaluate/integrate computes);
 *   orc_vmult_brute  dense element matrices assembled from full tensor
 *                    quadrature, like the reference's matrix-based path
 *                    source/level_set/advection_diffusion_operator.cpp:78-206.
 * Both follow the same operator definitions:
 *   heat     v = rho_cp/dt u + rho_cp (vel . grad u),  g = k(T) grad u
 *            (+ dk/dT grad T u with full_tangent)         heat_diffuse_operator.cpp:1029-1078
 *            Robin face term alpha u v                    heat_diffuse_operator.cpp:1088-1129
 *   advdiff  v = u/dt + theta (vel . grad u), g = theta D grad u
 *                                                         advection_diffusion_operator.cpp:471-493
 * Constrained (Dirichlet) DoFs are read as zero and never written, which is
 * what MatrixFree::loop with read_dof_values/distribute_local_to_global does.
 */
#include "mpdg_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define MAXN 10
#define MAXN3 (MAXN * MAXN * MAXN)

/* ------------------------------------------------------------------ 1D rules */

static void legendre_eval(int n, double x, double *p, double *dp)
{
  /* P_n and P_n' on [-1,1] by the three-term recurrence */
  double p0 = 1.0, p1 = x;
  if (n == 0) { *p = 1.0; *dp = 0.0; return; }
  for (int k = 2; k <= n; ++k) {
    double pk = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
    p0 = p1;
    p1 = pk;
  }
  *p = p1;
  *dp = (fabs(x) < 1.0) ? n * (x * p1 - p0) / (x * x - 1.0) : 0.5 * x * n * (n + 1.0);
  if (fabs(x) >= 1.0) *dp = (x > 0 ? 1.0 : ((n % 2) ? 1.0 : -1.0)) * 0.5 * n * (n + 1.0);
}

void orc_gauss_legendre(int n, double *x, double *w)
{
  for (int i = 0; i < n; ++i) {
    double z = cos(M_PI * (i + 0.75) / (n + 0.5)), p, dp;
    for (int it = 0; it < 100; ++it) {
      legendre_eval(n, z, &p, &dp);
      double dz = p / dp;
      z -= dz;
      if (fabs(dz) < 1e-16) break;
    }
    legendre_eval(n, z, &p, &dp);
    /* ascending order on [0,1] */
    x[n - 1 - i] = 0.5 * (1.0 + z);
    w[n - 1 - i] = 1.0 / ((1.0 - z * z) * dp * dp); /* = 2/((1-z^2)P'^2) / 2 */
  }
}

void orc_gauss_lobatto(int n, double *x)
{
  /* endpoints plus the roots of P'_{n-1}; (1-z^2) P''_m = 2 z P'_m - m(m+1) P_m */
  const int m = n - 1;
  x[0] = 0.0;
  x[n - 1] = 1.0;
  for (int i = 1; i < n - 1; ++i) {
    double z = -cos(M_PI * i / m), p, dp;
    for (int it = 0; it < 100; ++it) {
      legendre_eval(m, z, &p, &dp);
      double ddp = (2.0 * z * dp - m * (m + 1.0) * p) / (1.0 - z * z);
      double dz = dp / ddp;
      z -= dz;
      if (fabs(dz) < 1e-16) break;
    }
    x[i] = 0.5 * (1.0 + z);
  }
}

void orc_shape_tables(int n, const double *xq, int nq, double *S, double *D)
{
  double z[MAXN];
  orc_gauss_lobatto(n, z);
  for (int q = 0; q < nq; ++q)
    for (int i = 0; i < n; ++i) {
      double v = 1.0, d = 0.0;
      for (int j = 0; j < n; ++j)
        if (j != i) v *= (xq[q] - z[j]) / (z[i] - z[j]);
      for (int k = 0; k < n; ++k) {
        if (k == i) continue;
        double t = 1.0 / (z[i] - z[k]);
        for (int j = 0; j < n; ++j)
          if (j != i && j != k) t *= (xq[q] - z[j]) / (z[i] - z[j]);
        d += t;
      }
      S[q * n + i] = v;
      D[q * n + i] = d;
    }
}

/* -------------------------------------------------------------- mesh helpers */

typedef struct {
  int dim, p, n;      /* n = p + 1 points per direction */
  int nc[3];
  long NX, NY, NZ, N;
  long n_cells;
  double xq[MAXN], wq[MAXN];
  double S[MAXN * MAXN], D[MAXN * MAXN];
  /* Dc[q*n+r]: derivative of the Lagrange polynomial r on the Gauss points at
   * x_q (exact on values of degree < n); D2 = Dc D: second derivatives of the
   * Gauss-Lobatto basis at the Gauss points */
  double Dc[MAXN * MAXN], D2[MAXN * MAXN];
} geo_t;

static void geo_init(const orc_mesh *m, geo_t *g)
{
  g->dim = m->dim;
  g->p = m->degree;
  g->n = m->degree + 1;
  g->nc[0] = m->nc[0];
  g->nc[1] = m->nc[1];
  g->nc[2] = (m->dim == 3) ? m->nc[2] : 1;
  g->NX = (long)g->nc[0] * g->p + 1;
  g->NY = (long)g->nc[1] * g->p + 1;
  g->NZ = (m->dim == 3) ? (long)g->nc[2] * g->p + 1 : 1;
  g->N = g->NX * g->NY * g->NZ;
  g->n_cells = (long)g->nc[0] * g->nc[1] * g->nc[2];
  orc_gauss_legendre(g->n, g->xq, g->wq);
  orc_shape_tables(g->n, g->xq, g->n, g->S, g->D);
  const int n = g->n;
  for (int q = 0; q < n; ++q)
    for (int r = 0; r < n; ++r) {
      double d = 0.0;
      for (int k = 0; k < n; ++k) {
        if (k == r) continue;
        double t = 1.0 / (g->xq[r] - g->xq[k]);
        for (int j = 0; j < n; ++j)
          if (j != r && j != k) t *= (g->xq[q] - g->xq[j]) / (g->xq[r] - g->xq[j]);
        d += t;
      }
      g->Dc[q * n + r] = d;
    }
  for (int q = 0; q < n; ++q)
    for (int i = 0; i < n; ++i) {
      double s2 = 0.0;
      for (int r = 0; r < n; ++r) s2 += g->Dc[q * n + r] * g->D[r * n + i];
      g->D2[q * n + i] = s2;
    }
}

long orc_n_dofs(const orc_mesh *m)
{
  geo_t g;
  geo_init(m, &g);
  return g.N;
}

static long vert_index(const geo_t *g, int vx, int vy, int vz)
{
  return ((long)vz * (g->nc[1] + 1) + vy) * (g->nc[0] + 1) + vx;
}

/* vertices of cell (ix,iy,iz): vc[c][a], c = bx + 2 by + 4 bz */
static void cell_vertices(const orc_mesh *m, const geo_t *g, int ix, int iy, int iz,
                          double vc[8][3])
{
  const int nv = (g->dim == 3) ? 8 : 4;
  for (int c = 0; c < nv; ++c) {
    long v = vert_index(g, ix + (c & 1), iy + ((c >> 1) & 1), iz + ((c >> 2) & 1));
    for (int a = 0; a < 3; ++a) vc[c][a] = (a < g->dim) ? m->vert[v * g->dim + a] : 0.0;
  }
}

/* multilinear map at reference point xi: position x and Jacobian J[a][b] = dx_a/dxi_b */
static void map_point(const geo_t *g, double vc[8][3], const double xi[3], double x[3],
                      double J[3][3])
{
  const int dim = g->dim, nv = 1 << dim;
  for (int a = 0; a < 3; ++a) {
    x[a] = 0.0;
    for (int b = 0; b < 3; ++b) J[a][b] = 0.0;
  }
  for (int c = 0; c < nv; ++c) {
    double f[3], df[3];
    for (int d = 0; d < dim; ++d) {
      int bit = (c >> d) & 1;
      f[d] = bit ? xi[d] : 1.0 - xi[d];
      df[d] = bit ? 1.0 : -1.0;
    }
    double B = 1.0;
    for (int d = 0; d < dim; ++d) B *= f[d];
    for (int b = 0; b < dim; ++b) {
      double dB = df[b];
      for (int d = 0; d < dim; ++d)
        if (d != b) dB *= f[d];
      for (int a = 0; a < dim; ++a) J[a][b] += vc[c][a] * dB;
    }
    for (int a = 0; a < dim; ++a) x[a] += vc[c][a] * B;
  }
  if (dim == 2) J[2][2] = 1.0;
}

/* inverse and determinant of a 3x3 (2D embedded with J[2][2] = 1) */
static double inverse3(double J[3][3], double Ji[3][3])
{
  double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
               J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
               J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
  double id = 1.0 / det;
  Ji[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) * id;
  Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
  Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
  Ji[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) * id;
  Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
  Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
  Ji[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) * id;
  Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
  Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
  return det;
}

/* Curvature term of the physical Laplacian at reference point xi of the
 * (bi/tri)linear map of corners vc.  With K_j[a][b] = d2 x_j / dxi_a dxi_b
 * (only mixed derivatives are nonzero for this map) and Gt = J^-1 J^-T,
 *   lap u = sum_ab Gt_ab d2u/dxi_a dxi_b - sum_a lam_a du/dxi_a,
 *   lam_a = sum_j (J^-1)_aj sum_bc Gt_bc K_j[b][c],
 * which follows from d(J^-1)/dxi_c = -J^-1 (dJ/dxi_c) J^-1.  This is the
 * Laplacian FEEvaluation::get_laplacian returns on non-affine cells
 * (advection_diffusion_operator.cpp:483-486, with jacobian gradients). */
static void map_second(const geo_t *g, double vc[8][3], const double xi[3], double K[3][3][3])
{
  const int dim = g->dim, nv = 1 << dim;
  memset(K, 0, sizeof(double) * 27);
  for (int c = 0; c < nv; ++c)
    for (int a = 0; a < dim; ++a)
      for (int b = a + 1; b < dim; ++b) {
        double d2 = 1.0;
        for (int d = 0; d < dim; ++d) {
          const int bit = (c >> d) & 1;
          d2 *= (d == a || d == b) ? (bit ? 1.0 : -1.0) : (bit ? xi[d] : 1.0 - xi[d]);
        }
        for (int j = 0; j < dim; ++j) {
          K[j][a][b] += vc[c][j] * d2;
          K[j][b][a] += vc[c][j] * d2;
        }
      }
}

static void map_lambda(const geo_t *g, double vc[8][3], const double xi[3], double Ji[3][3], double lam[3])
{
  const int dim = g->dim;
  double K[3][3][3];
  map_second(g, vc, xi, K);
  double Gt[3][3];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      double t = 0.0;
      for (int i = 0; i < dim; ++i) t += Ji[a][i] * Ji[b][i];
      Gt[a][b] = t;
    }
  double kap[3] = {0.0, 0.0, 0.0};
  for (int j = 0; j < dim; ++j)
    for (int a = 0; a < dim; ++a)
      for (int b = 0; b < dim; ++b) kap[j] += Gt[a][b] * K[j][a][b];
  for (int a = 0; a < 3; ++a) {
    double t = 0.0;
    for (int j = 0; j < dim; ++j) t += Ji[a][j] * kap[j];
    lam[a] = (a < dim) ? t : 0.0;
  }
}

static void cell_dofs(const geo_t *g, int ix, int iy, int iz, long *idx)
{
  const int n = g->n, nz = (g->dim == 3) ? n : 1;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i)
        idx[(k * n + j) * n + i] =
          ((long)(iz * g->p + k) * g->NY + (iy * g->p + j)) * g->NX + (ix * g->p + i);
}

void orc_dof_coordinates(const orc_mesh *m, double *xyz)
{
  geo_t g;
  geo_init(m, &g);
  double z[MAXN];
  orc_gauss_lobatto(g.n, z);
  const int nz = (g.dim == 3) ? g.n : 1;
  for (int iz = 0; iz < g.nc[2]; ++iz)
    for (int iy = 0; iy < g.nc[1]; ++iy)
      for (int ix = 0; ix < g.nc[0]; ++ix) {
        double vc[8][3];
        long idx[MAXN3];
        cell_vertices(m, &g, ix, iy, iz, vc);
        cell_dofs(&g, ix, iy, iz, idx);
        for (int k = 0; k < nz; ++k)
          for (int j = 0; j < g.n; ++j)
            for (int i = 0; i < g.n; ++i) {
              double xi[3] = {z[i], z[j], (g.dim == 3) ? z[k] : 0.0}, x[3], J[3][3];
              map_point(&g, vc, xi, x, J);
              long gi = idx[(k * g.n + j) * g.n + i];
              for (int a = 0; a < g.dim; ++a) xyz[gi * g.dim + a] = x[a];
            }
      }
}

/* ---------------------------------------------------------- velocity at a point */

static void velocity_at(const orc_op *op, int dim, const double x[3], double u[3])
{
  u[0] = u[1] = u[2] = 0.0;
  switch (op->vel_kind) {
    case ORC_VEL_ROTATION: {
      const double s = op->vel_param[0];
      u[0] = s * x[dim - 1];
      u[dim - 1] = -s * x[0];
      break;
    }
    case ORC_VEL_VORTEX:
      u[0] = sin(M_PI * x[0]) * cos(M_PI * x[1]);
      u[1] = -cos(M_PI * x[0]) * sin(M_PI * x[1]);
      break;
    case ORC_VEL_CONST:
      for (int d = 0; d < dim; ++d) u[d] = op->vel_param[d];
      break;
    default:
      break;
  }
}

/* ----------------------------------------------------- sum factorisation kernels */

/* out = M (n x n, row = output point) applied along direction dir; transpose: M^T */
static void contract(const geo_t *g, const double *M, int transpose, int dir, const double *in,
                     double *out)
{
  const int n = g->n, nz = (g->dim == 3) ? n : 1;
  const int ext[3] = {n, n, nz};
  const int stride[3] = {1, n, n * n};
  const int total = n * n * nz;
  for (int t = 0; t < total; ++t) {
    int c[3] = {t % n, (t / n) % n, t / (n * n)};
    double s = 0.0;
    int base = t - c[dir] * stride[dir];
    for (int r = 0; r < ext[dir]; ++r) {
      double a = transpose ? M[r * n + c[dir]] : M[c[dir] * n + r];
      s += a * in[base + r * stride[dir]];
    }
    out[t] = s;
  }
}

/* values and reference gradients at the quadrature points */
static void evaluate(const geo_t *g, const double *u, double *val, double grad[3][MAXN3])
{
  double t1[MAXN3], t2[MAXN3];
  const int dim = g->dim;
  /* value: S along every direction */
  if (val) {
    contract(g, g->S, 0, 0, u, t1);
    contract(g, g->S, 0, 1, t1, (dim == 3) ? t2 : val);
    if (dim == 3) contract(g, g->S, 0, 2, t2, val);
  }
  if (grad)
    for (int b = 0; b < dim; ++b) {
      const double *M0 = (b == 0) ? g->D : g->S;
      const double *M1 = (b == 1) ? g->D : g->S;
      const double *M2 = (b == 2) ? g->D : g->S;
      contract(g, M0, 0, 0, u, t1);
      contract(g, M1, 0, 1, t1, (dim == 3) ? t2 : grad[b]);
      if (dim == 3) contract(g, M2, 0, 2, t2, grad[b]);
    }
}

/* out += S^T(val) + sum_b D_b^T(grad[b]) */
static void integrate(const geo_t *g, const double *val, double grad[3][MAXN3], double *out)
{
  double t1[MAXN3], t2[MAXN3];
  const int dim = g->dim, n = g->n, nz = (dim == 3) ? n : 1, total = n * n * nz;
  for (int b = -1; b < dim; ++b) {
    const double *src = (b < 0) ? val : grad[b];
    if (!src) continue;
    const double *M0 = (b == 0) ? g->D : g->S;
    const double *M1 = (b == 1) ? g->D : g->S;
    const double *M2 = (b == 2) ? g->D : g->S;
    if (dim == 3) {
      contract(g, M2, 1, 2, src, t1);
      contract(g, M1, 1, 1, t1, t2);
      contract(g, M0, 1, 0, t2, t1);
    } else {
      contract(g, M1, 1, 1, src, t2);
      contract(g, M0, 1, 0, t2, t1);
    }
    for (int t = 0; t < total; ++t) out[t] += t1[t];
  }
}

/* per-cell quadrature-point data shared by the tangent, the residual and the diagonal */
typedef struct {
  double JxW, Ji[3][3], x[3], vel[3];
  double lam[3]; /* curvature term of the physical Laplacian (map_lambda) */
  double T, gradT[3]; /* physical */
  double Told, H;     /* T_old and the heaviside at the point */
} qdata_t;

/* ----------------------------------------------------------- material laws
 * (rho c_p, k, d(rho c_p)/dT, dk/dT) at a point: Material::compute_parameters_internal
 * (material.templates.hpp:213-500) with the solid fraction of :748-760, the cubic
 * solid/liquid interpolation of :546-600 (level_set_tools.hpp:66-90) and the gas
 * weight of compute_two_phase_fluid_property (:513-523); rho c_p = rho * c_p and its
 * derivative by the product rule (heat_diffuse_operator.cpp:1176-1199) unless the
 * volume-specific capacity is interpolated itself */
static double ls_value(double fs, double vl, double vs)
{
  if (fs == 0.0) return vl;
  if (fs == 1.0) return vs;
  return vl + (vs - vl) * (-2.0 * fs * fs * fs + 3.0 * fs * fs);
}

static double ls_deriv(double fs, double inv_mushy, double vl, double vs)
{
  if (fs == 0.0 || fs == 1.0) return 0.0;
  return -inv_mushy * (vs - vl) * (-6.0 * fs * fs + 6.0 * fs);
}

static int mat_has_T(const orc_op *op)
{
  return op->material == ORC_MAT_LIQUID_SOLID || op->material == ORC_MAT_GAS_LIQUID_SOLID;
}

/* Apparent heat capacity of the latent heat of fusion L over the mushy zone
 * [Ts, Tl] (ApparentCapacity::evaluate / compute_temperature_derivative,
 * source/heat/apparent_capacity.cpp), as a function of the solid fraction fs
 * and its T derivative; 0 outside 0 < fs < 1.  Profiles:
 *   constant:   L / (Tl - Ts);
 *   poly4_bell: L r b(xi), r = 2 / (Tl - Ts), xi = 1 - 2 fs,
 *               b(x) = 15/16 x^4 - 15/8 x^2 + 15/16 (unit integral on [-1, 1]);
 *   qlq:        at T = Tl - fs (Tl - Ts), two ramps 0 -> C_peak -> 0 over
 *               [Ts, T_peak] and [T_peak, Tl] (T_peak the midpoint, C_peak =
 *               2 L / (Tl - Ts)), each quadratic with zero slope over delta =
 *               (Tl - Ts) / 6 at both ends and linear in between. */
static void qlq_ramp(double x, double x1, double x2, double y1, double y2, double delta, double *f, double *df)
{
  /* slope s of the linear part: the two quadratic ends y1 + s/(2 delta) (x-x1)^2
   * and y2 - s/(2 delta) (x2-x)^2 meet it with continuous value and slope */
  const double s = (y2 - y1) / (x2 - x1 - delta);
  if (x < x1 + delta) {
    *f = y1 + 0.5 * s / delta * (x - x1) * (x - x1);
    *df = s * (x - x1) / delta;
  } else if (x > x2 - delta) {
    *f = y2 - 0.5 * s / delta * (x2 - x) * (x2 - x);
    *df = s * (x2 - x) / delta;
  } else {
    *f = y1 + 0.5 * s * delta + s * (x - x1 - delta);
    *df = s;
  }
}

static void apparent_capacity_fs(const orc_op *op, double fs, double *c, double *dc)
{
  *c = *dc = 0.0;
  if (!(op->latent_heat > 0.0) || fs <= 0.0 || fs >= 1.0) return;
  const double L = op->latent_heat, Ts = op->solidus, Tl = op->liquidus, dT = Tl - Ts;
  if (op->apparent_capacity == ORC_AC_CONSTANT) {
    *c = L / dT;
  } else if (op->apparent_capacity == ORC_AC_POLY4_BELL) {
    const double r = 2.0 / dT, xi = 1.0 - 2.0 * fs, x2 = xi * xi;
    *c = L * r * (15.0 / 16.0 * x2 * x2 - 15.0 / 8.0 * x2 + 15.0 / 16.0);
    *dc = L * r * r * (15.0 / 4.0 * x2 * xi - 15.0 / 4.0 * xi);
  } else {
    const double T = Tl - fs * dT, Tp = 0.5 * (Ts + Tl), Cp = 2.0 * L / dT, delta = dT / 6.0;
    if (T <= Tp) qlq_ramp(T, Ts, Tp, 0.0, Cp, delta, c, dc);
    else qlq_ramp(T, Tp, Tl, Cp, 0.0, delta, c, dc);
  }
}

void orc_apparent_capacity(const orc_op *op, double T, double *c, double *dc)
{
  const double fs = fmin(fmax((op->liquidus - T) / (op->liquidus - op->solidus), 0.0), 1.0);
  apparent_capacity_fs(op, fs, c, dc);
}

static void mat_eval(const orc_op *op, double T, double H, double *rc, double *k, double *drc, double *dk)
{
  if (op->material == ORC_MAT_LINEAR) {
    *rc = op->rho_cp;
    *k = op->k0 * (1.0 + op->k_alpha * T);
    *drc = 0.0;
    *dk = op->k0 * op->k_alpha;
    return;
  }
  const int gas = op->material == ORC_MAT_GAS_LIQUID || op->material == ORC_MAT_GAS_LIQUID_SOLID;
  const int sol = mat_has_T(op);
  const double inv_mushy = sol ? 1.0 / (op->liquidus - op->solidus) : 0.0;
  double fs = 0.0;
  if (sol) fs = op->solid_liquid_sharp ? (T < op->solidus ? 1.0 : 0.0)
                                       : fmin(fmax((op->liquidus - T) * inv_mushy, 0.0), 1.0);
  const double w = gas ? (op->two_phase_sharp ? (H > 0.5 ? 1.0 : 0.0) : H) : 1.0;
  double v[4], dv[4]; /* rho, c_p, k, rho c_p of the liquid(-solid) phase */
  const double rcl = op->mat_rho[1] * op->mat_cp[1], rcs = op->mat_rho[2] * op->mat_cp[2];
  const double vl[4] = {op->mat_rho[1], op->mat_cp[1], op->mat_k[1], rcl};
  const double vs[4] = {op->mat_rho[2], op->mat_cp[2], op->mat_k[2], rcs};
  const double vg[4] = {op->mat_rho[0], op->mat_cp[0], op->mat_k[0], op->mat_rho[0] * op->mat_cp[0]};
  for (int e = 0; e < 4; ++e) {
    v[e] = sol ? ls_value(fs, vl[e], vs[e]) : vl[e];
    dv[e] = sol ? ls_deriv(fs, inv_mushy, vl[e], vs[e]) : 0.0;
    if (sol && e == 1) {
      /* latent heat: c_p of the solid/liquid mix gains the apparent capacity
       * (material.templates.hpp:566-578, 604-616), before the gas weighting */
      double c, dc;
      apparent_capacity_fs(op, fs, &c, &dc);
      v[1] += c;
      dv[1] += dc;
    }
    if (gas) {
      v[e] = (1.0 - w) * vg[e] + w * v[e];
      dv[e] = w * dv[e];
    }
  }
  *k = v[2];
  *dk = dv[2];
  if (op->volume_specific) {
    if (op->latent_heat > 0.0 && sol) {
      fprintf(stderr, "orc: the apparent capacity is not defined for the volume-specific heat capacity\n");
      abort();
    }
    *rc = v[3];
    *drc = dv[3];
  } else {
    *rc = v[0] * v[1];
    *drc = dv[1] * v[0] + dv[0] * v[1];
  }
}

static void cell_qdata(const orc_mesh *m, const orc_op *op, const geo_t *g, int ix, int iy,
                       int iz, const long *idx, qdata_t *qd)
{
  const int n = g->n, dim = g->dim, nz = (dim == 3) ? n : 1, nqt = n * n * nz;
  double vc[8][3];
  cell_vertices(m, g, ix, iy, iz, vc);
  /* temperature at the quadrature points (values and reference gradients) */
  double Tl[MAXN3], Tv[MAXN3], Tg[3][MAXN3];
  int haveT = op->temperature != NULL;
  if (haveT) {
    for (int t = 0; t < nqt; ++t) Tl[t] = op->temperature[idx[t]];
    evaluate(g, Tl, Tv, Tg);
  }
  double Ov[MAXN3], Hv[MAXN3];
  if (op->temperature_old) {
    double l[MAXN3];
    for (int t = 0; t < nqt; ++t) l[t] = op->temperature_old[idx[t]];
    evaluate(g, l, Ov, NULL);
  }
  if (op->heaviside) {
    double l[MAXN3];
    for (int t = 0; t < nqt; ++t) l[t] = op->heaviside[idx[t]];
    evaluate(g, l, Hv, NULL);
  }
  double Vv[3][MAXN3];
  if (op->vel_kind == ORC_VEL_NODAL)
    for (int d = 0; d < dim; ++d) {
      double Vl[MAXN3];
      for (int t = 0; t < nqt; ++t) Vl[t] = op->vel_nodal[(long)d * g->N + idx[t]];
      evaluate(g, Vl, Vv[d], NULL);
    }
  for (int qz = 0; qz < nz; ++qz)
    for (int qy = 0; qy < n; ++qy)
      for (int qx = 0; qx < n; ++qx) {
        int q = (qz * n + qy) * n + qx;
        double xi[3] = {g->xq[qx], g->xq[qy], (dim == 3) ? g->xq[qz] : 0.0};
        double w = g->wq[qx] * g->wq[qy] * ((dim == 3) ? g->wq[qz] : 1.0);
        double J[3][3];
        map_point(g, vc, xi, qd[q].x, J);
        double det = inverse3(J, qd[q].Ji);
        qd[q].JxW = det * w;
        map_lambda(g, vc, xi, qd[q].Ji, qd[q].lam);
        if (op->vel_kind == ORC_VEL_NODAL) {
          for (int d = 0; d < 3; ++d) qd[q].vel[d] = (d < dim) ? Vv[d][q] : 0.0;
        } else {
          velocity_at(op, dim, qd[q].x, qd[q].vel);
        }
        qd[q].T = haveT ? Tv[q] : 0.0;
        qd[q].Told = op->temperature_old ? Ov[q] : 0.0;
        qd[q].H = op->heaviside ? Hv[q] : 0.0;
        for (int a = 0; a < 3; ++a) {
          double s = 0.0;
          if (haveT)
            for (int b = 0; b < dim; ++b) s += qd[q].Ji[b][a] * Tg[b][q];
          qd[q].gradT[a] = (a < dim) ? s : 0.0;
        }
      }
}

/* quadrature-point kernel of the tangent: returns value coefficient v and the
 * physical flux f for the trial value u and physical gradient gu */
static void tangent_qp(const orc_op *op, int dim, const qdata_t *qd, double u, const double gu[3],
                       double *v, double f[3])
{
  double vgu = 0.0;
  for (int a = 0; a < dim; ++a) vgu += qd->vel[a] * gu[a];
  if (op->kind == ORC_HEAT) {
    /* heat_diffuse_operator.cpp:1040-1062 */
    double rc, k, drc, dk;
    mat_eval(op, qd->T, qd->H, &rc, &k, &drc, &dk);
    *v = rc / op->dt * u + rc * vgu;
    const int deriv = (op->material == ORC_MAT_LINEAR) ? op->full_tangent : mat_has_T(op);
    for (int a = 0; a < 3; ++a) f[a] = k * gu[a] + (deriv ? dk * qd->gradT[a] * u : 0.0);
    if (deriv && op->material != ORC_MAT_LINEAR) {
      double vgT = 0.0;
      for (int a = 0; a < dim; ++a) vgT += qd->vel[a] * qd->gradT[a];
      *v += drc / op->dt * (qd->T - qd->Told) * u + drc * vgT * u;
    }
  } else {
    *v = u / op->dt + op->theta * vgu;
    for (int a = 0; a < 3; ++a) f[a] = op->theta * op->diffusivity * gu[a];
  }
}

static int cell_colour(int ix, int iy, int iz) { return (ix & 1) | ((iy & 1) << 1) | ((iz & 1) << 2); }

/* SUPG parameter of a cell (compute_stabilization_parameter,
 * advection_diffusion_operator.cpp:499-533; cell size = diameter / sqrt(dim),
 * scratch_data.cpp:249-266) */
static double cell_tau(const orc_mesh *m, const orc_op *op, const geo_t *g, int ix, int iy, int iz,
                       const qdata_t *qd)
{
  if (!op->supg || op->kind != ORC_ADVDIFF) return 0.0;
  const int dim = g->dim, nqt = g->n * g->n * ((dim == 3) ? g->n : 1);
  double vc[8][3];
  cell_vertices(m, g, ix, iy, iz, vc);
  const int pairs3[4][2] = {{0, 7}, {1, 6}, {2, 5}, {3, 4}}, pairs2[2][2] = {{0, 3}, {1, 2}};
  double diam = 0.0;
  for (int k = 0; k < ((dim == 3) ? 4 : 2); ++k) {
    const int a = (dim == 3) ? pairs3[k][0] : pairs2[k][0], b = (dim == 3) ? pairs3[k][1] : pairs2[k][1];
    double d2 = 0.0;
    for (int c = 0; c < dim; ++c) d2 += (vc[a][c] - vc[b][c]) * (vc[a][c] - vc[b][c]);
    diam = fmax(diam, sqrt(d2));
  }
  const double h = diam / sqrt((double)dim);
  if (op->supg_coefficient >= 0.0) return op->supg_coefficient * h;
  double umax = 0.0;
  for (int q = 0; q < nqt; ++q) {
    double s2 = 0.0;
    for (int a = 0; a < dim; ++a) s2 += qd[q].vel[a] * qd[q].vel[a];
    umax = fmax(umax, sqrt(s2));
  }
  return (umax >= 1e-6) ? h / umax : 0.0;
}

/* SUPG parameter of a cell given by its corners vc and DoFs idx (mapped
 * meshes): as cell_tau, with the velocity at the mapped Gauss points (the
 * nodal field interpolated through idx) */
static double tau_vc(const orc_op *op, const geo_t *g, double vc[8][3], const long *idx)
{
  if (!op->supg || op->kind != ORC_ADVDIFF) return 0.0;
  const int dim = g->dim, n = g->n, nz = (dim == 3) ? n : 1, nqt = n * n * nz;
  const int pairs3[4][2] = {{0, 7}, {1, 6}, {2, 5}, {3, 4}}, pairs2[2][2] = {{0, 3}, {1, 2}};
  double diam = 0.0;
  for (int k = 0; k < ((dim == 3) ? 4 : 2); ++k) {
    const int a = (dim == 3) ? pairs3[k][0] : pairs2[k][0], b = (dim == 3) ? pairs3[k][1] : pairs2[k][1];
    double d2 = 0.0;
    for (int c = 0; c < dim; ++c) d2 += (vc[a][c] - vc[b][c]) * (vc[a][c] - vc[b][c]);
    diam = fmax(diam, sqrt(d2));
  }
  const double h = diam / sqrt((double)dim);
  if (op->supg_coefficient >= 0.0) return op->supg_coefficient * h;
  double umax = 0.0;
  for (int q = 0; q < nqt; ++q) {
    const int qq[3] = {q % n, (q / n) % n, q / (n * n)};
    const double xi[3] = {g->xq[qq[0]], g->xq[qq[1]], (dim == 3) ? g->xq[qq[2]] : 0.0};
    double x[3], J[3][3], u[3] = {0.0, 0.0, 0.0};
    map_point(g, vc, xi, x, J);
    if (op->vel_kind == ORC_VEL_NODAL) {
      for (int t = 0; t < nqt; ++t) {
        const int c[3] = {t % n, (t / n) % n, t / (n * n)};
        double phi = 1.0;
        for (int d = 0; d < dim; ++d) phi *= g->S[qq[d] * n + c[d]];
        for (int d = 0; d < dim; ++d) u[d] += op->vel_nodal[(long)d * g->N + idx[t]] * phi;
      }
    } else {
      velocity_at(op, dim, x, u);
    }
    double s2 = 0.0;
    for (int a = 0; a < dim; ++a) s2 += u[a] * u[a];
    umax = fmax(umax, sqrt(s2));
  }
  return (umax >= 1e-6) ? h / umax : 0.0;
}

/* physical Laplacian at the quadrature points from the reference gradients:
 * sum_ab Gt_ab d2u/dxi_a dxi_b - lam . grad_ref u (map_lambda), the second
 * reference derivatives by collocation differentiation of the gradients */
static void laplacian_qp(const geo_t *g, double ug[3][MAXN3], const qdata_t *qd, double *lap)
{
  const int dim = g->dim, nqt = g->n * g->n * ((dim == 3) ? g->n : 1);
  double t[MAXN3];
  for (int q = 0; q < nqt; ++q) {
    lap[q] = 0.0;
    for (int a = 0; a < dim; ++a) lap[q] -= qd[q].lam[a] * ug[a][q];
  }
  for (int a = 0; a < dim; ++a)
    for (int b = a; b < dim; ++b) {
      contract(g, g->Dc, 0, b, ug[a], t); /* d/dxi_b of du/dxi_a */
      for (int q = 0; q < nqt; ++q) {
        double gab = 0.0;
        for (int i = 0; i < dim; ++i) gab += qd[q].Ji[a][i] * qd[q].Ji[b][i];
        lap[q] += ((a == b) ? 1.0 : 2.0) * gab * t[q];
      }
    }
}

/* one cell of the sum-factorised tangent; adds into dst (caller guarantees no race) */
static void apply_cell(const orc_mesh *m, const orc_op *op, const geo_t *g, int ix, int iy,
                       int iz, double *dst, const double *src)
{
  const int n = g->n, dim = g->dim, nz = (dim == 3) ? n : 1, nqt = n * n * nz;
  long idx[MAXN3];
  cell_dofs(g, ix, iy, iz, idx);
  static __thread qdata_t qd[MAXN3];
  cell_qdata(m, op, g, ix, iy, iz, idx, qd);
  double ul[MAXN3], uv[MAXN3], ug[3][MAXN3], out[MAXN3], lap[MAXN3];
  for (int t = 0; t < nqt; ++t)
    ul[t] = (op->dirichlet && op->dirichlet[idx[t]]) ? 0.0 : src[idx[t]];
  evaluate(g, ul, uv, ug);
  const double tau = cell_tau(m, op, g, ix, iy, iz, qd);
  const int supg = op->supg && op->kind == ORC_ADVDIFF;
  if (supg && op->diffusivity != 0.0) laplacian_qp(g, ug, qd, lap);
  for (int q = 0; q < nqt; ++q) {
    double gu[3] = {0, 0, 0}, v, f[3];
    for (int a = 0; a < dim; ++a)
      for (int b = 0; b < dim; ++b) gu[a] += qd[q].Ji[b][a] * ug[b][q];
    tangent_qp(op, dim, &qd[q], uv[q], gu, &v, f);
    if (supg) {
      const double r = v - ((op->diffusivity != 0.0) ? op->theta * op->diffusivity * lap[q] : 0.0);
      for (int a = 0; a < dim; ++a) f[a] += tau * qd[q].vel[a] * r;
    }
    uv[q] = v * qd[q].JxW;
    for (int b = 0; b < dim; ++b) {
      double s = 0.0;
      for (int a = 0; a < dim; ++a) s += qd[q].Ji[b][a] * f[a];
      ug[b][q] = s * qd[q].JxW;
    }
  }
  memset(out, 0, sizeof(double) * nqt);
  integrate(g, uv, ug, out);
  for (int t = 0; t < nqt; ++t)
    if (!(op->dirichlet && op->dirichlet[idx[t]])) dst[idx[t]] += out[t];
}

/* ------------------------------------------------------------ Robin faces (heat) */

/* Boundary-face terms of the heat operator on face (d, s) of a cell: convection
 * (robin_faces, coefficient alpha) and radiation (rad_faces, emissivity eps),
 * heat_diffuse_operator.cpp:1088-1129 (tangent) and :719-778 (residual).
 * TANGENT: (alpha + 4 eps sigma T_q^3) u_q tested with N, or its diagonal;
 * RESIDUAL: -alpha (T_q - T_inf) - eps sigma (T_q^4 - T_rad^4) tested with N.
 * T_q is the face interpolant of op->temperature.  Face shape functions are
 * products of 1D S tables (nodal on GL nodes, so the trace uses the face's own
 * dofs only). */
enum { ROB_TANGENT = 0, ROB_RESIDUAL = 1 };

static void face_terms_id(const orc_op *op, int id, int *conv, int *rad)
{
  const int bit = 1 << id;
  *conv = op->kind == ORC_HEAT && (op->robin_faces & bit) && op->robin_alpha != 0.0;
  *rad = op->kind == ORC_HEAT && (op->rad_faces & bit) && op->rad_emissivity != 0.0;
}

static void face_terms(const orc_op *op, int d, int s, int *conv, int *rad)
{
  const int bit = 1 << (2 * d + s);
  *conv = op->kind == ORC_HEAT && (op->robin_faces & bit) && op->robin_alpha != 0.0;
  *rad = op->kind == ORC_HEAT && (op->rad_faces & bit) && op->rad_emissivity != 0.0;
}

static int has_face_terms(const orc_op *op)
{
  for (int f = 0; f < 6; ++f) {
    int c, r;
    face_terms(op, f / 2, f % 2, &c, &r);
    if (c || r) return 1;
  }
  return 0;
}

/* face terms of local face (d, s) of the cell with corners vc, selected by
 * boundary id `id` (bit of robin_faces / rad_faces) */
static void robin_face_apply_vc(const orc_op *op, const geo_t *g, double vc[8][3], int d, int s, int id,
                                int mode, const long *idx, const double *ul_cell, double *out_cell,
                                double *diag_cell)
{
  const int n = g->n, dim = g->dim;
  int conv, rad;
  face_terms_id(op, id, &conv, &rad);
  if (!conv && !rad) return;
  const double es = op->rad_emissivity * ORC_STEFAN_BOLTZMANN;
  int t0 = (d == 0) ? 1 : 0;           /* tangential directions */
  int t1 = (dim == 3) ? ((d == 2) ? 1 : 2) : -1;
  const int nq1 = (dim == 3) ? n : 1, nb = (dim == 3) ? n : 1;
  for (int qb = 0; qb < nq1; ++qb)
    for (int qa = 0; qa < n; ++qa) {
      double xi[3] = {0, 0, 0};
      xi[d] = s ? 1.0 : 0.0;
      xi[t0] = g->xq[qa];
      if (t1 >= 0) xi[t1] = g->xq[qb];
      double x[3], J[3][3];
      map_point(g, vc, xi, x, J);
      double w = g->wq[qa] * ((t1 >= 0) ? g->wq[qb] : 1.0), ds;
      if (dim == 2) {
        ds = sqrt(J[0][t0] * J[0][t0] + J[1][t0] * J[1][t0]);
      } else {
        double a0[3] = {J[0][t0], J[1][t0], J[2][t0]}, a1[3] = {J[0][t1], J[1][t1], J[2][t1]};
        double c[3] = {a0[1] * a1[2] - a0[2] * a1[1], a0[2] * a1[0] - a0[0] * a1[2],
                       a0[0] * a1[1] - a0[1] * a1[0]};
        ds = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
      }
      const double JxW = ds * w;
      /* face dofs: local index with coordinate d fixed to 0 or p */
      double uq = 0.0, Tq = 0.0;
      for (int b = 0; b < nb; ++b)
        for (int a = 0; a < n; ++a) {
          int c[3] = {0, 0, 0};
          c[d] = s ? n - 1 : 0;
          c[t0] = a;
          if (t1 >= 0) c[t1] = b;
          int li = (c[2] * n + c[1]) * n + c[0];
          double phi = g->S[qa * n + a] * ((t1 >= 0) ? g->S[qb * n + b] : 1.0);
          if (ul_cell) uq += phi * ul_cell[li];
          if (op->temperature) Tq += phi * op->temperature[idx[li]];
        }
      const double coef = (conv ? op->robin_alpha : 0.0) + (rad ? 4.0 * es * Tq * Tq * Tq : 0.0);
      double val = coef * uq;
      if (mode == ROB_RESIDUAL)
        val = -(conv ? op->robin_alpha * (Tq - op->robin_t_inf) : 0.0) -
              (rad ? es * (Tq * Tq * Tq * Tq - op->rad_t_inf * op->rad_t_inf * op->rad_t_inf * op->rad_t_inf)
                   : 0.0);
      for (int b = 0; b < nb; ++b)
        for (int a = 0; a < n; ++a) {
          int c[3] = {0, 0, 0};
          c[d] = s ? n - 1 : 0;
          c[t0] = a;
          if (t1 >= 0) c[t1] = b;
          int li = (c[2] * n + c[1]) * n + c[0];
          double phi = g->S[qa * n + a] * ((t1 >= 0) ? g->S[qb * n + b] : 1.0);
          if (diag_cell) diag_cell[li] += coef * phi * phi * JxW;
          if (out_cell) out_cell[li] += val * phi * JxW;
        }
    }
}

static void robin_face_apply(const orc_mesh *m, const orc_op *op, const geo_t *g, int ix, int iy, int iz,
                             int d, int s, int mode, const long *idx, const double *ul_cell, double *out_cell,
                             double *diag_cell)
{
  double vc[8][3];
  cell_vertices(m, g, ix, iy, iz, vc);
  robin_face_apply_vc(op, g, vc, d, s, 2 * d + s, mode, idx, ul_cell, out_cell, diag_cell);
}

/* adds the face matrices of a mapped cell's boundary faces to its element
 * matrix A (columns by unit local vectors through robin_face_apply_vc) */
static void add_face_matrices(const orc_mapped *m, const orc_op *op, const geo_t *g, long K, double vc[8][3],
                              const long *idx, double *A)
{
  if (!m->face_ids) return;
  const int n = g->n, nqt = n * n * n;
  double e[MAXN3], col[MAXN3];
  for (int f = 0; f < 6; ++f) {
    const int id = m->face_ids[K * 6 + f];
    if (id < 0) continue;
    for (int u = 0; u < nqt; ++u) {
      memset(e, 0, sizeof(double) * nqt);
      memset(col, 0, sizeof(double) * nqt);
      e[u] = 1.0;
      robin_face_apply_vc(op, g, vc, f / 2, f % 2, id, ROB_TANGENT, idx, e, col, NULL);
      for (int t = 0; t < nqt; ++t) A[t * nqt + u] += col[t];
    }
  }
}

static int cell_on_face(const geo_t *g, int ix, int iy, int iz, int d, int s)
{
  int c[3] = {ix, iy, iz};
  return s ? (c[d] == g->nc[d] - 1) : (c[d] == 0);
}

static void apply_robin(const orc_mesh *m, const orc_op *op, const geo_t *g, double *dst,
                        const double *src)
{
  if (!has_face_terms(op)) return;
  const int n = g->n, dim = g->dim, nz = (dim == 3) ? n : 1, nqt = n * n * nz;
  for (int iz = 0; iz < g->nc[2]; ++iz)
    for (int iy = 0; iy < g->nc[1]; ++iy)
      for (int ix = 0; ix < g->nc[0]; ++ix)
        for (int d = 0; d < dim; ++d)
          for (int s = 0; s < 2; ++s) {
            int conv, rad;
            face_terms(op, d, s, &conv, &rad);
            if (!(conv || rad) || !cell_on_face(g, ix, iy, iz, d, s)) continue;
            long idx[MAXN3];
            double ul[MAXN3], out[MAXN3];
            cell_dofs(g, ix, iy, iz, idx);
            for (int t = 0; t < nqt; ++t) {
              ul[t] = (op->dirichlet && op->dirichlet[idx[t]]) ? 0.0 : src[idx[t]];
              out[t] = 0.0;
            }
            robin_face_apply(m, op, g, ix, iy, iz, d, s, ROB_TANGENT, idx, ul, out, NULL);
            for (int t = 0; t < nqt; ++t)
              if (!(op->dirichlet && op->dirichlet[idx[t]])) dst[idx[t]] += out[t];
          }
}

/* ------------------------------------------------------------------- vmult */

void orc_vmult_cells(const orc_mesh *m, const orc_op *op, double *dst, const double *src,
                     long cell_begin, long cell_end)
{
  geo_t g;
  geo_init(m, &g);
  const long nxy = (long)g.nc[0] * g.nc[1];
  /* colour loop: cells of one parity colour share no DoF, so they may run in parallel */
  for (int colour = 0; colour < 8; ++colour) {
#pragma omp parallel for schedule(dynamic, 16)
    for (long c = cell_begin; c < cell_end; ++c) {
      int iz = (int)(c / nxy), iy = (int)((c / g.nc[0]) % g.nc[1]), ix = (int)(c % g.nc[0]);
      if (cell_colour(ix, iy, iz) != colour) continue;
      apply_cell(m, op, &g, ix, iy, iz, dst, src);
    }
  }
}

void orc_vmult(const orc_mesh *m, const orc_op *op, double *dst, const double *src)
{
  geo_t g;
  geo_init(m, &g);
  memset(dst, 0, sizeof(double) * g.N);
  orc_vmult_cells(m, op, dst, src, 0, g.n_cells);
  apply_robin(m, op, &g, dst, src);
}

/* ----------------------------------------------- brute-force element matrices */

static void element_matrix_vc(const orc_op *op, const geo_t *g, double vc[8][3], const long *idx, double tau,
                              double *A);

static void element_matrix(const orc_mesh *m, const orc_op *op, const geo_t *g, int ix, int iy,
                           int iz, const long *idx, double *A /* nqt x nqt */)
{
  double vc[8][3];
  cell_vertices(m, g, ix, iy, iz, vc);
  double tau = 0.0;
  if (op->supg && op->kind == ORC_ADVDIFF) {
    static __thread qdata_t qdc[MAXN3];
    orc_op plain = *op;
    plain.temperature = NULL;
    cell_qdata(m, &plain, g, ix, iy, iz, idx, qdc);
    tau = cell_tau(m, op, g, ix, iy, iz, qdc);
  }
  element_matrix_vc(op, g, vc, idx, tau, A);
}

/* element matrix of the cell with corners vc (x fastest) and global DoFs idx
 * (the fields are read through idx) */
static void element_matrix_vc(const orc_op *op, const geo_t *g, double vc[8][3], const long *idx, double tau,
                              double *A)
{
  const int n = g->n, dim = g->dim, nz = (dim == 3) ? n : 1, nqt = n * n * nz;
  memset(A, 0, sizeof(double) * nqt * nqt);
  static __thread double phi[MAXN3], gphi[MAXN3][3];
  for (int qz = 0; qz < nz; ++qz)
    for (int qy = 0; qy < n; ++qy)
      for (int qx = 0; qx < n; ++qx) {
        const int qq[3] = {qx, qy, qz};
        double xi[3] = {g->xq[qx], g->xq[qy], (dim == 3) ? g->xq[qz] : 0.0};
        double w = g->wq[qx] * g->wq[qy] * ((dim == 3) ? g->wq[qz] : 1.0);
        qdata_t qd;
        double J[3][3];
        map_point(g, vc, xi, qd.x, J);
        double det = inverse3(J, qd.Ji);
        qd.JxW = det * w;
        double Kq[3][3][3];
        map_second(g, vc, xi, Kq);
        /* shape values and physical gradients by direct products */
        for (int t = 0; t < nqt; ++t) {
          int c[3] = {t % n, (t / n) % n, t / (n * n)};
          double f[3], df[3];
          for (int d = 0; d < 3; ++d) {
            f[d] = (d < dim) ? g->S[qq[d] * n + c[d]] : 1.0;
            df[d] = (d < dim) ? g->D[qq[d] * n + c[d]] : 0.0;
          }
          phi[t] = f[0] * f[1] * f[2];
          double gr[3] = {df[0] * f[1] * f[2], f[0] * df[1] * f[2], f[0] * f[1] * df[2]};
          for (int a = 0; a < 3; ++a) {
            double s = 0.0;
            for (int b = 0; b < dim; ++b) s += qd.Ji[b][a] * gr[b];
            gphi[t][a] = (a < dim) ? s : 0.0;
          }
        }
        /* fields at this point by direct summation */
        qd.T = qd.Told = qd.H = 0.0;
        qd.gradT[0] = qd.gradT[1] = qd.gradT[2] = 0.0;
        for (int t = 0; t < nqt; ++t) {
          if (op->temperature_old) qd.Told += op->temperature_old[idx[t]] * phi[t];
          if (op->heaviside) qd.H += op->heaviside[idx[t]] * phi[t];
        }
        if (op->temperature)
          for (int t = 0; t < nqt; ++t) {
            double Tt = op->temperature[idx[t]];
            qd.T += Tt * phi[t];
            for (int a = 0; a < 3; ++a) qd.gradT[a] += Tt * gphi[t][a];
          }
        if (op->vel_kind == ORC_VEL_NODAL) {
          for (int d = 0; d < 3; ++d) {
            qd.vel[d] = 0.0;
            if (d < dim)
              for (int t = 0; t < nqt; ++t) qd.vel[d] += op->vel_nodal[(long)d * g->N + idx[t]] * phi[t];
          }
        } else {
          velocity_at(op, dim, qd.x, qd.vel);
        }
        for (int j = 0; j < nqt; ++j) {
          double v, fl[3];
          tangent_qp(op, dim, &qd, phi[j], gphi[j], &v, fl);
          if (op->supg && op->kind == ORC_ADVDIFF) {
            /* Laplacian of basis j: the physical Hessian
             * J^-T (Hhat - sum_i (grad phi)_i K_i) J^-1 (chain rule of the map),
             * traced; Hhat from products of the 1D value, derivative and
             * second-derivative tables */
            int c[3] = {j % n, (j / n) % n, j / (n * n)};
            double Hh[3][3];
            for (int a = 0; a < 3; ++a)
              for (int b = 0; b < 3; ++b) {
                if (a >= dim || b >= dim) {
                  Hh[a][b] = 0.0;
                  continue;
                }
                double pr = 1.0;
                for (int e = 0; e < dim; ++e) {
                  const int k = (e == a) + (e == b);
                  const double *tab1 = (k == 0) ? g->S : (k == 1) ? g->D : g->D2;
                  pr *= tab1[qq[e] * n + c[e]];
                }
                Hh[a][b] = pr;
              }
            for (int i = 0; i < dim; ++i)
              for (int a = 0; a < dim; ++a)
                for (int b = 0; b < dim; ++b) Hh[a][b] -= gphi[j][i] * Kq[i][a][b];
            double lapj = 0.0;
            for (int i = 0; i < dim; ++i)
              for (int a = 0; a < dim; ++a)
                for (int b = 0; b < dim; ++b) lapj += qd.Ji[a][i] * Hh[a][b] * qd.Ji[b][i];
            const double r = v - op->theta * op->diffusivity * lapj;
            for (int a = 0; a < dim; ++a) fl[a] += tau * qd.vel[a] * r;
          }
          for (int i = 0; i < nqt; ++i)
            A[i * nqt + j] += (v * phi[i] + fl[0] * gphi[i][0] + fl[1] * gphi[i][1] +
                               fl[2] * gphi[i][2]) * qd.JxW;
        }
      }
}

void orc_vmult_brute(const orc_mesh *m, const orc_op *op, double *dst, const double *src)
{
  geo_t g;
  geo_init(m, &g);
  const int n = g.n, nz = (g.dim == 3) ? n : 1, nqt = n * n * nz;
  memset(dst, 0, sizeof(double) * g.N);
  double *A = (double *)malloc(sizeof(double) * nqt * nqt);
  for (int iz = 0; iz < g.nc[2]; ++iz)
    for (int iy = 0; iy < g.nc[1]; ++iy)
      for (int ix = 0; ix < g.nc[0]; ++ix) {
        long idx[MAXN3];
        cell_dofs(&g, ix, iy, iz, idx);
        element_matrix(m, op, &g, ix, iy, iz, idx, A);
        for (int i = 0; i < nqt; ++i) {
          if (op->dirichlet && op->dirichlet[idx[i]]) continue;
          double s = 0.0;
          for (int j = 0; j < nqt; ++j)
            if (!(op->dirichlet && op->dirichlet[idx[j]])) s += A[i * nqt + j] * src[idx[j]];
          dst[idx[i]] += s;
        }
      }
  free(A);
  apply_robin(m, op, &g, dst, src);
}

/* ---------------------------------------------------------------- diagonal */

void orc_diagonal(const orc_mesh *m, const orc_op *op, double *diag)
{
  geo_t g;
  geo_init(m, &g);
  const int n = g.n, dim = g.dim, nz = (dim == 3) ? n : 1, nqt = n * n * nz;
  memset(diag, 0, sizeof(double) * g.N);
  const long nxy = (long)g.nc[0] * g.nc[1];
  for (int colour = 0; colour < 8; ++colour) {
#pragma omp parallel
    {
      double *A = (double *)malloc(sizeof(double) * nqt * nqt);
#pragma omp for schedule(dynamic, 16)
      for (long c = 0; c < g.n_cells; ++c) {
        int iz = (int)(c / nxy), iy = (int)((c / g.nc[0]) % g.nc[1]), ix = (int)(c % g.nc[0]);
        if (cell_colour(ix, iy, iz) != colour) continue;
        long idx[MAXN3];
        cell_dofs(&g, ix, iy, iz, idx);
        element_matrix(m, op, &g, ix, iy, iz, idx, A);
        double dc[MAXN3];
        for (int i = 0; i < nqt; ++i) dc[i] = A[i * nqt + i];
        for (int d = 0; d < dim; ++d)
          for (int s = 0; s < 2; ++s)
            if (cell_on_face(&g, ix, iy, iz, d, s))
              robin_face_apply(m, op, &g, ix, iy, iz, d, s, ROB_TANGENT, idx, NULL, NULL, dc);
        for (int i = 0; i < nqt; ++i)
          if (!(op->dirichlet && op->dirichlet[idx[i]])) diag[idx[i]] += dc[i];
      }
      free(A);
    }
  }
  if (op->dirichlet)
    for (long i = 0; i < g.N; ++i)
      if (op->dirichlet[i]) diag[i] = 1.0;
}

/* inversion rules: heat_diffuse_operator.cpp:282-283 (|d| > 1e-10),
 * advection_diffusion_operator.cpp:437-439 (|d| > 1e-14 max(1, |d|_inf)) */
void orc_invert_diagonal(const orc_mesh *m, const orc_op *op, double *diag)
{
  const long N = orc_n_dofs(m);
  double thr = 1e-10;
  if (op->kind == ORC_ADVDIFF) {
    double mx = 1.0;
    for (long i = 0; i < N; ++i) mx = fmax(mx, fabs(diag[i]));
    thr = 1e-14 * mx;
  }
  for (long i = 0; i < N; ++i) diag[i] = (fabs(diag[i]) > thr) ? 1.0 / diag[i] : 1.0;
}

/* -------------------------------------------------------------- residuals */

void orc_rhs_heat(const orc_mesh *m, const orc_op *op, double *dst, const double *t_old,
                  const double *heat_source, const unsigned char *scatter_mask)
{
  geo_t g;
  geo_init(m, &g);
  const int n = g.n, dim = g.dim, nz = (dim == 3) ? n : 1, nqt = n * n * nz;
  const long nxy = (long)g.nc[0] * g.nc[1];
  for (int colour = 0; colour < 8; ++colour) {
#pragma omp parallel for schedule(dynamic, 16)
    for (long c = 0; c < g.n_cells; ++c) {
      int iz = (int)(c / nxy), iy = (int)((c / g.nc[0]) % g.nc[1]), ix = (int)(c % g.nc[0]);
      if (cell_colour(ix, iy, iz) != colour) continue;
      long idx[MAXN3];
      cell_dofs(&g, ix, iy, iz, idx);
      static __thread qdata_t qd[MAXN3];
      cell_qdata(m, op, &g, ix, iy, iz, idx, qd);
      double ol[MAXN3], ov[MAXN3], ql[MAXN3], qv[MAXN3], val[MAXN3], grd[3][MAXN3], out[MAXN3];
      for (int t = 0; t < nqt; ++t) {
        ol[t] = t_old[idx[t]];
        ql[t] = heat_source ? heat_source[idx[t]] : 0.0;
      }
      evaluate(&g, ol, ov, NULL);
      evaluate(&g, ql, qv, NULL);
      for (int q = 0; q < nqt; ++q) {
        /* heat_diffuse_operator.cpp:482-518 */
        double rc, k, drc, dk;
        mat_eval(op, qd[q].T, qd[q].H, &rc, &k, &drc, &dk);
        double v = rc / op->dt * (qd[q].T - ov[q]) - qv[q];
        double vg = 0.0;
        for (int a = 0; a < dim; ++a) vg += qd[q].gradT[a] * qd[q].vel[a];
        v += rc * vg;
        val[q] = -v * qd[q].JxW;
        for (int b = 0; b < dim; ++b) {
          double s = 0.0;
          for (int a = 0; a < dim; ++a) s += qd[q].Ji[b][a] * k * qd[q].gradT[a];
          grd[b][q] = -s * qd[q].JxW;
        }
      }
      memset(out, 0, sizeof(double) * nqt);
      integrate(&g, val, grd, out);
      for (int t = 0; t < nqt; ++t)
        if (!(scatter_mask && scatter_mask[idx[t]])) dst[idx[t]] += out[t];
    }
  }
  /* convective and radiative faces (heat_diffuse_operator.cpp:719-778) */
  if (has_face_terms(op)) {
    for (int iz = 0; iz < g.nc[2]; ++iz)
      for (int iy = 0; iy < g.nc[1]; ++iy)
        for (int ix = 0; ix < g.nc[0]; ++ix)
          for (int d = 0; d < dim; ++d)
            for (int s = 0; s < 2; ++s) {
              if (!cell_on_face(&g, ix, iy, iz, d, s)) continue;
              long idx[MAXN3];
              double out[MAXN3];
              cell_dofs(&g, ix, iy, iz, idx);
              for (int t = 0; t < nqt; ++t) out[t] = 0.0;
              robin_face_apply(m, op, &g, ix, iy, iz, d, s, ROB_RESIDUAL, idx, NULL, out, NULL);
              for (int t = 0; t < nqt; ++t)
                if (!(scatter_mask && scatter_mask[idx[t]])) dst[idx[t]] += out[t];
            }
  }
}

void orc_rhs_advdiff(const orc_mesh *m, const orc_op *op, double *dst, const double *phi_old,
                     const unsigned char *scatter_mask)
{
  geo_t g;
  geo_init(m, &g);
  const int n = g.n, dim = g.dim, nz = (dim == 3) ? n : 1, nqt = n * n * nz;
  const long nxy = (long)g.nc[0] * g.nc[1];
  orc_op op2 = *op;
  op2.temperature = NULL;
  for (int colour = 0; colour < 8; ++colour) {
#pragma omp parallel for schedule(dynamic, 16)
    for (long c = 0; c < g.n_cells; ++c) {
      int iz = (int)(c / nxy), iy = (int)((c / g.nc[0]) % g.nc[1]), ix = (int)(c % g.nc[0]);
      if (cell_colour(ix, iy, iz) != colour) continue;
      long idx[MAXN3];
      cell_dofs(&g, ix, iy, iz, idx);
      static __thread qdata_t qd[MAXN3];
      cell_qdata(m, &op2, &g, ix, iy, iz, idx, qd);
      double ul[MAXN3], uv[MAXN3], ug[3][MAXN3], out[MAXN3], lap[MAXN3];
      for (int t = 0; t < nqt; ++t) ul[t] = phi_old[idx[t]];
      evaluate(&g, ul, uv, ug);
      const int supg = op->supg && op->kind == ORC_ADVDIFF;
      const double tau = cell_tau(m, op, &g, ix, iy, iz, qd);
      if (supg && op->diffusivity != 0.0) laplacian_qp(&g, ug, qd, lap);
      for (int q = 0; q < nqt; ++q) {
        double gp[3] = {0, 0, 0}, vg = 0.0;
        for (int a = 0; a < dim; ++a) {
          for (int b = 0; b < dim; ++b) gp[a] += qd[q].Ji[b][a] * ug[b][q];
          vg += qd[q].vel[a] * gp[a];
        }
        const double res = uv[q] / op->dt - (1.0 - op->theta) * vg;
        uv[q] = res * qd[q].JxW;
        /* SUPG: tau vel (res + (1 - theta) D lap) tested with grad N */
        const double rs = supg ? res + ((op->diffusivity != 0.0) ? (1.0 - op->theta) * op->diffusivity * lap[q] : 0.0)
                               : 0.0;
        for (int b = 0; b < dim; ++b) {
          double s = 0.0;
          for (int a = 0; a < dim; ++a)
            s += qd[q].Ji[b][a] * (-(1.0 - op->theta) * op->diffusivity * gp[a] + (supg ? tau * qd[q].vel[a] * rs : 0.0));
          ug[b][q] = s * qd[q].JxW;
        }
      }
      memset(out, 0, sizeof(double) * nqt);
      integrate(&g, uv, ug, out);
      for (int t = 0; t < nqt; ++t)
        if (!(scatter_mask && scatter_mask[idx[t]])) dst[idx[t]] += out[t];
    }
  }
}

/* integrated L2 norm with QGauss(p+1): VectorTools::compute_norm,
 * source/utilities/vector_tools.cpp:170-201 */
/* per-cell integrated L2 norms (what VectorTools::integrate_difference writes
 * into its Vector<float> of cell errors, before the float rounding) */
void orc_l2_norm_cells(const orc_mesh *m, const double *u, double *cell_norms)
{
  geo_t g;
  geo_init(m, &g);
  const int n = g.n, dim = g.dim, nz = (dim == 3) ? n : 1, nqt = n * n * nz;
#pragma omp parallel for schedule(static)
  for (long c = 0; c < g.n_cells; ++c) {
    const long nxy = (long)g.nc[0] * g.nc[1];
    int iz = (int)(c / nxy), iy = (int)((c / g.nc[0]) % g.nc[1]), ix = (int)(c % g.nc[0]);
    long idx[MAXN3];
    double ul[MAXN3], uv[MAXN3], vc[8][3];
    cell_dofs(&g, ix, iy, iz, idx);
    cell_vertices(m, &g, ix, iy, iz, vc);
    for (int t = 0; t < nqt; ++t) ul[t] = u[idx[t]];
    evaluate(&g, ul, uv, NULL);
    double s = 0.0;
    for (int qz = 0; qz < nz; ++qz)
      for (int qy = 0; qy < n; ++qy)
        for (int qx = 0; qx < n; ++qx) {
          double xi[3] = {g.xq[qx], g.xq[qy], (dim == 3) ? g.xq[qz] : 0.0}, x[3], J[3][3], Ji[3][3];
          map_point(&g, vc, xi, x, J);
          double w = g.wq[qx] * g.wq[qy] * ((dim == 3) ? g.wq[qz] : 1.0);
          double v = uv[(qz * n + qy) * n + qx];
          s += v * v * inverse3(J, Ji) * w;
        }
    cell_norms[c] = sqrt(s);
  }
}

double orc_l2_norm(const orc_mesh *m, const double *u)
{
  geo_t g;
  geo_init(m, &g);
  const int n = g.n, dim = g.dim, nz = (dim == 3) ? n : 1, nqt = n * n * nz;
  double total = 0.0;
#pragma omp parallel for reduction(+ : total) schedule(static)
  for (long c = 0; c < g.n_cells; ++c) {
    const long nxy = (long)g.nc[0] * g.nc[1];
    int iz = (int)(c / nxy), iy = (int)((c / g.nc[0]) % g.nc[1]), ix = (int)(c % g.nc[0]);
    long idx[MAXN3];
    double ul[MAXN3], uv[MAXN3], vc[8][3];
    cell_dofs(&g, ix, iy, iz, idx);
    cell_vertices(m, &g, ix, iy, iz, vc);
    for (int t = 0; t < nqt; ++t) ul[t] = u[idx[t]];
    evaluate(&g, ul, uv, NULL);
    double s = 0.0;
    for (int qz = 0; qz < nz; ++qz)
      for (int qy = 0; qy < n; ++qy)
        for (int qx = 0; qx < n; ++qx) {
          double xi[3] = {g.xq[qx], g.xq[qy], (dim == 3) ? g.xq[qz] : 0.0}, x[3], J[3][3], Ji[3][3];
          map_point(&g, vc, xi, x, J);
          double w = g.wq[qx] * g.wq[qy] * ((dim == 3) ? g.wq[qz] : 1.0);
          double v = uv[(qz * n + qy) * n + qx];
          s += v * v * inverse3(J, Ji) * w;
        }
    total += s;
  }
  return sqrt(total);
}

/* ------------------------------------------------------------- Krylov solvers */

static double dotv(long N, const double *a, const double *b)
{
  double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (long i = 0; i < N; ++i) s += a[i] * b[i];
  return s;
}

/* Chebyshev semi-iteration on D^-1 A with zero start (residual polynomial of
 * the given degree; degree-1 operator applies); degree 1 is a scaled Jacobi */
void orc_prec_apply(const orc_mesh *m, const orc_op *op, const orc_prec *P, double *z,
                    const double *r)
{
  const long N = orc_n_dofs(m);
  if (!P || P->type == ORC_PREC_IDENTITY) {
    memcpy(z, r, sizeof(double) * N);
    return;
  }
  if (P->type == ORC_PREC_JACOBI) {
    for (long i = 0; i < N; ++i) z[i] = P->inv_diag[i] * r[i];
    return;
  }
  const double a = P->lambda_min, b = P->lambda_max;
  const double theta = 0.5 * (b + a), delta = 0.5 * (b - a), sigma = theta / delta;
  double rho = 1.0 / sigma;
  double *d = (double *)malloc(sizeof(double) * N), *t = (double *)malloc(sizeof(double) * N);
  for (long i = 0; i < N; ++i) {
    d[i] = P->inv_diag[i] * r[i] / theta;
    z[i] = d[i];
  }
  for (int k = 1; k < P->degree; ++k) {
    orc_vmult(m, op, t, z);
    double rho_new = 1.0 / (2.0 * sigma - rho);
    for (long i = 0; i < N; ++i) {
      d[i] = rho_new * rho * d[i] + 2.0 * rho_new / delta * P->inv_diag[i] * (r[i] - t[i]);
      z[i] += d[i];
    }
    rho = rho_new;
  }
  free(d);
  free(t);
}

/* preconditioned CG, deal.II SolverCG + ReductionControl semantics:
 * converged when |r_k| <= max(abs_tol, rel_tol |r_0|), |.| the l2 norm of the
 * unpreconditioned residual; *n_it = iterations performed */
int orc_cg(const orc_mesh *m, const orc_op *op, const orc_prec *P, const double *b, double *x,
           double rel_tol, double abs_tol, int max_it, int *n_it, double *res_hist)
{
  const long N = orc_n_dofs(m);
  double *r = malloc(sizeof(double) * N), *z = malloc(sizeof(double) * N),
         *p = malloc(sizeof(double) * N), *Ap = malloc(sizeof(double) * N);
  orc_vmult(m, op, Ap, x);
  for (long i = 0; i < N; ++i) r[i] = b[i] - Ap[i];
  double res = sqrt(dotv(N, r, r));
  const double tol = fmax(abs_tol, rel_tol * res);
  if (res_hist) res_hist[0] = res;
  int it = 0, status = 1;
  if (res <= tol) status = 0;
  double rz = 0.0;
  if (status) {
    orc_prec_apply(m, op, P, z, r);
    memcpy(p, z, sizeof(double) * N);
    rz = dotv(N, r, z);
  }
  while (status && it < max_it) {
    orc_vmult(m, op, Ap, p);
    const double alpha = rz / dotv(N, p, Ap);
    for (long i = 0; i < N; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * Ap[i];
    }
    ++it;
    res = sqrt(dotv(N, r, r));
    if (res_hist) res_hist[it] = res;
    if (res <= tol) {
      status = 0;
      break;
    }
    orc_prec_apply(m, op, P, z, r);
    const double rz_new = dotv(N, r, z), beta = rz_new / rz;
    rz = rz_new;
    for (long i = 0; i < N; ++i) p[i] = z[i] + beta * p[i];
  }
  *n_it = it;
  free(r);
  free(z);
  free(p);
  free(Ap);
  return status;
}

/* right-preconditioned restarted GMRES (modified Gram-Schmidt, Givens rotations);
 * the monitored residual is that of the unpreconditioned system, as in
 * deal.II SolverGMRES with right_preconditioning = true (linear_solver.hpp:112-119) */
int orc_gmres(const orc_mesh *m, const orc_op *op, const orc_prec *P, const double *b, double *x,
              double rel_tol, double abs_tol, int max_it, int restart, int *n_it,
              double *res_hist)
{
  const long N = orc_n_dofs(m);
  const int mk = restart;
  double *V = malloc(sizeof(double) * N * (mk + 1));
  double *w = malloc(sizeof(double) * N), *z = malloc(sizeof(double) * N);
  double *H = calloc((size_t)(mk + 1) * mk, sizeof(double));
  double *cs = malloc(sizeof(double) * mk), *sn = malloc(sizeof(double) * mk),
         *gv = malloc(sizeof(double) * (mk + 1)), *y = malloc(sizeof(double) * mk);
  int it = 0, status = 1;
  double tol = -1.0;
  for (;;) {
    orc_vmult(m, op, w, x);
    for (long i = 0; i < N; ++i) V[i] = b[i] - w[i];
    double beta = sqrt(dotv(N, V, V));
    if (tol < 0.0) {
      tol = fmax(abs_tol, rel_tol * beta);
      if (res_hist) res_hist[0] = beta;
    }
    if (beta <= tol) {
      status = 0;
      break;
    }
    if (it >= max_it) break;
    for (long i = 0; i < N; ++i) V[i] /= beta;
    for (int k = 0; k <= mk; ++k) gv[k] = 0.0;
    gv[0] = beta;
    int j = 0;
    for (; j < mk && it < max_it; ++j) {
      orc_prec_apply(m, op, P, z, V + (long)j * N);
      orc_vmult(m, op, w, z);
      for (int k = 0; k <= j; ++k) {
        double h = dotv(N, w, V + (long)k * N);
        H[k * mk + j] = h;
        for (long i = 0; i < N; ++i) w[i] -= h * V[(long)k * N + i];
      }
      double hn = sqrt(dotv(N, w, w));
      H[(j + 1) * mk + j] = hn;
      for (long i = 0; i < N; ++i) V[(long)(j + 1) * N + i] = (hn > 0.0) ? w[i] / hn : 0.0;
      for (int k = 0; k < j; ++k) {
        double t = cs[k] * H[k * mk + j] + sn[k] * H[(k + 1) * mk + j];
        H[(k + 1) * mk + j] = -sn[k] * H[k * mk + j] + cs[k] * H[(k + 1) * mk + j];
        H[k * mk + j] = t;
      }
      double a = H[j * mk + j], c = H[(j + 1) * mk + j], r = sqrt(a * a + c * c);
      cs[j] = a / r;
      sn[j] = c / r;
      H[j * mk + j] = r;
      H[(j + 1) * mk + j] = 0.0;
      gv[j + 1] = -sn[j] * gv[j];
      gv[j] = cs[j] * gv[j];
      ++it;
      if (res_hist) res_hist[it] = fabs(gv[j + 1]);
      if (fabs(gv[j + 1]) <= tol) {
        ++j;
        status = 0;
        break;
      }
    }
    /* x += M^-1 V y */
    for (int k = j - 1; k >= 0; --k) {
      double s = gv[k];
      for (int l = k + 1; l < j; ++l) s -= H[k * mk + l] * y[l];
      y[k] = s / H[k * mk + k];
    }
    for (long i = 0; i < N; ++i) w[i] = 0.0;
    for (int k = 0; k < j; ++k)
      for (long i = 0; i < N; ++i) w[i] += y[k] * V[(long)k * N + i];
    orc_prec_apply(m, op, P, z, w);
    for (long i = 0; i < N; ++i) x[i] += z[i];
    if (status == 0 || it >= max_it) break;
  }
  *n_it = it;
  free(V);
  free(w);
  free(z);
  free(H);
  free(cs);
  free(sn);
  free(gv);
  free(y);
  return status;
}

/* largest eigenvalue of D^-1 A from n_steps of CG-Lanczos (Jacobi-preconditioned
 * CG on A x = start from x = 0); Sturm bisection on the tridiagonal matrix */
double orc_estimate_lambda_max(const orc_mesh *m, const orc_op *op, const double *inv_diag,
                               const double *start, int n_steps)
{
  const long N = orc_n_dofs(m);
  double *r = malloc(sizeof(double) * N), *z = malloc(sizeof(double) * N),
         *p = malloc(sizeof(double) * N), *Ap = malloc(sizeof(double) * N);
  double al[64], be[64];
  memcpy(r, start, sizeof(double) * N);
  for (long i = 0; i < N; ++i) z[i] = inv_diag[i] * r[i];
  memcpy(p, z, sizeof(double) * N);
  double rz = dotv(N, r, z);
  int k = 0;
  for (; k < n_steps && k < 64; ++k) {
    orc_vmult(m, op, Ap, p);
    al[k] = rz / dotv(N, p, Ap);
    for (long i = 0; i < N; ++i) r[i] -= al[k] * Ap[i];
    for (long i = 0; i < N; ++i) z[i] = inv_diag[i] * r[i];
    double rz_new = dotv(N, r, z);
    be[k] = rz_new / rz;
    rz = rz_new;
    for (long i = 0; i < N; ++i) p[i] = z[i] + be[k] * p[i];
  }
  /* tridiagonal T: T_jj = 1/al_j + be_{j-1}/al_{j-1}, T_{j,j+1} = sqrt(be_j)/al_j */
  double dg[64], of[64];
  for (int j = 0; j < k; ++j) {
    dg[j] = 1.0 / al[j] + ((j > 0) ? be[j - 1] / al[j - 1] : 0.0);
    of[j] = (j + 1 < k) ? sqrt(be[j]) / al[j] : 0.0;
  }
  double lo = 0.0, hi = 0.0;
  for (int j = 0; j < k; ++j)
    hi = fmax(hi, dg[j] + fabs(of[j]) + ((j > 0) ? fabs(of[j - 1]) : 0.0));
  for (int itb = 0; itb < 200; ++itb) {
    double mid = 0.5 * (lo + hi);
    int cnt = 0;
    double q = 1.0;
    for (int j = 0; j < k; ++j) {
      q = dg[j] - mid - ((j > 0) ? of[j - 1] * of[j - 1] / q : 0.0);
      if (q == 0.0) q = -1e-300;
      if (q < 0.0) ++cnt;
    }
    if (cnt >= k) hi = mid; /* all eigenvalues below mid */
    else lo = mid;
  }
  free(r);
  free(z);
  free(p);
  free(Ap);
  return hi;
}


/* ============================================================ hanging nodes
 * Two-level meshes (see mpdg_oracle.h).  Brute force: per cell the element
 * matrix A_K (element_matrix) and the local-to-global constraint weights C_K;
 * dst += C_K^T A_K C_K src.  deal.II applies the same constraints inside
 * FEEvaluation::read_dof_values / distribute_local_to_global for meshes with
 * hanging nodes (refinement 2:1). */

void orc2_hanging_matrix(int degree, double *P)
{
  const int n = degree + 1;
  double z[MAXN], xs[MAXN], S[MAXN * MAXN], D[MAXN * MAXN];
  orc_gauss_lobatto(n, z);
  for (int s = 0; s < 2; ++s) {
    for (int j = 0; j < n; ++j) xs[j] = 0.5 * (s + z[j]);
    orc_shape_tables(n, xs, n, S, D);
    for (int j = 0; j < n; ++j)
      for (int jp = 0; jp < n; ++jp) P[(s * n + j) * n + jp] = S[j * n + jp];
  }
}

long orc2_n_dofs(const orc_mesh2 *m) { return orc_n_dofs(&m->coarse) + orc_n_dofs(&m->fine); }

/* constraint weights of the local DoFs of a cell: up to n^2 (global, weight) each */
typedef struct {
  int cnt[MAXN3];
  long g[MAXN3][MAXN * MAXN];
  double w[MAXN3][MAXN * MAXN];
} cmap_t;

static void cell_cmap(const geo_t *gc, const geo_t *gf, int fine, int ix, int iy, int iz, const double *P,
                      cmap_t *cm)
{
  const int n = gf->n, p = gf->p;
  const long Nc = gc->N;
  const geo_t *g = fine ? gf : gc;
  long idx[MAXN3];
  cell_dofs(g, ix, iy, iz, idx);
  for (int t = 0; t < n * n * n; ++t) {
    const int i = t % n, j = (t / n) % n, k = t / (n * n);
    if (fine && ix == 0 && i == 0) {
      const int cy = iy / 2, sy = iy % 2, cz = iz / 2, sz = iz % 2;
      int c = 0;
      for (int kp = 0; kp < n; ++kp)
        for (int jp = 0; jp < n; ++jp) {
          cm->g[t][c] = ((long)(cz * p + kp) * gc->NY + (cy * p + jp)) * gc->NX + (gc->NX - 1);
          cm->w[t][c] = P[(sy * n + j) * n + jp] * P[(sz * n + k) * n + kp];
          ++c;
        }
      cm->cnt[t] = c;
    } else {
      cm->cnt[t] = 1;
      cm->g[t][0] = (fine ? Nc : 0) + idx[t];
      cm->w[t][0] = 1.0;
    }
  }
}

static int hanging_slot(const geo_t *gc, const geo_t *gf, long gidx)
{
  if (gidx < gc->N) return 0;
  return ((gidx - gc->N) % gf->NX) == 0;
}

static void orc2_check(const orc_mesh2 *m, const orc_op *op)
{
  if (m->coarse.dim != 3 || m->fine.dim != 3 || m->coarse.degree != m->fine.degree ||
      m->fine.nc[1] != 2 * m->coarse.nc[1] || m->fine.nc[2] != 2 * m->coarse.nc[2] ||
      op->temperature || op->robin_faces || op->rad_faces || op->vel_kind == ORC_VEL_NODAL || op->full_tangent ||
      op->material != ORC_MAT_LINEAR) {
    fprintf(stderr, "orc2: unsupported two-level configuration\n");
    abort();
  }
}

void orc2_vmult(const orc_mesh2 *m, const orc_op *op, double *dst, const double *src)
{
  orc2_check(m, op);
  geo_t gc, gf;
  geo_init(&m->coarse, &gc);
  geo_init(&m->fine, &gf);
  const int n = gc.n, nqt = n * n * n;
  double P[2 * MAXN * MAXN];
  orc2_hanging_matrix(gc.p, P);
  const long N = gc.N + gf.N;
  memset(dst, 0, sizeof(double) * N);
  double *A = (double *)malloc(sizeof(double) * nqt * nqt);
  cmap_t *cm = (cmap_t *)malloc(sizeof(cmap_t));
  for (int fine = 0; fine < 2; ++fine) {
    const geo_t *g = fine ? &gf : &gc;
    const orc_mesh *mm = fine ? &m->fine : &m->coarse;
    for (int iz = 0; iz < g->nc[2]; ++iz)
      for (int iy = 0; iy < g->nc[1]; ++iy)
        for (int ix = 0; ix < g->nc[0]; ++ix) {
          long idx[MAXN3];
          cell_dofs(g, ix, iy, iz, idx);
          element_matrix(mm, op, g, ix, iy, iz, idx, A);
          cell_cmap(&gc, &gf, fine, ix, iy, iz, P, cm);
          double ul[MAXN3];
          for (int t = 0; t < nqt; ++t) {
            double v = 0.0;
            for (int c = 0; c < cm->cnt[t]; ++c) {
              const long gg = cm->g[t][c];
              if (!(op->dirichlet && op->dirichlet[gg])) v += cm->w[t][c] * src[gg];
            }
            ul[t] = v;
          }
          for (int t = 0; t < nqt; ++t) {
            double o = 0.0;
            for (int u = 0; u < nqt; ++u) o += A[t * nqt + u] * ul[u];
            for (int c = 0; c < cm->cnt[t]; ++c) {
              const long gg = cm->g[t][c];
              if (!(op->dirichlet && op->dirichlet[gg]) && !hanging_slot(&gc, &gf, gg))
                dst[gg] += cm->w[t][c] * o;
            }
          }
        }
  }
  free(A);
  free(cm);
}

void orc2_diagonal(const orc_mesh2 *m, const orc_op *op, double *diag)
{
  orc2_check(m, op);
  geo_t gc, gf;
  geo_init(&m->coarse, &gc);
  geo_init(&m->fine, &gf);
  const int n = gc.n, nqt = n * n * n;
  double P[2 * MAXN * MAXN];
  orc2_hanging_matrix(gc.p, P);
  const long N = gc.N + gf.N;
  memset(diag, 0, sizeof(double) * N);
  double *A = (double *)malloc(sizeof(double) * nqt * nqt);
  cmap_t *cm = (cmap_t *)malloc(sizeof(cmap_t));
  for (int fine = 0; fine < 2; ++fine) {
    const geo_t *g = fine ? &gf : &gc;
    const orc_mesh *mm = fine ? &m->fine : &m->coarse;
    for (int iz = 0; iz < g->nc[2]; ++iz)
      for (int iy = 0; iy < g->nc[1]; ++iy)
        for (int ix = 0; ix < g->nc[0]; ++ix) {
          long idx[MAXN3];
          cell_dofs(g, ix, iy, iz, idx);
          element_matrix(mm, op, g, ix, iy, iz, idx, A);
          cell_cmap(&gc, &gf, fine, ix, iy, iz, P, cm);
          /* (C^T A C)_{gg} = sum_{t,u} w_t(g) A_tu w_u(g) */
          for (int t = 0; t < nqt; ++t)
            for (int c = 0; c < cm->cnt[t]; ++c) {
              const long gg = cm->g[t][c];
              if (hanging_slot(&gc, &gf, gg)) continue;
              double s = 0.0;
              for (int u = 0; u < nqt; ++u)
                for (int d = 0; d < cm->cnt[u]; ++d)
                  if (cm->g[u][d] == gg) s += A[t * nqt + u] * cm->w[u][d];
              diag[gg] += cm->w[t][c] * s;
            }
        }
  }
  for (long i = 0; i < N; ++i)
    if ((op->dirichlet && op->dirichlet[i]) || hanging_slot(&gc, &gf, i)) diag[i] = 1.0;
  free(A);
  free(cm);
}

void orc2_distribute(const orc_mesh2 *m, double *u)
{
  geo_t gc, gf;
  geo_init(&m->coarse, &gc);
  geo_init(&m->fine, &gf);
  const int n = gc.n, p = gc.p;
  double P[2 * MAXN * MAXN];
  orc2_hanging_matrix(p, P);
  for (long Z = 0; Z < gf.NZ; ++Z)
    for (long Y = 0; Y < gf.NY; ++Y) {
      /* the fine cell (iy, iz) containing the node, any of them (continuous trace) */
      const int iy = (int)((Y == gf.NY - 1) ? gf.nc[1] - 1 : Y / p), j = (int)(Y - (long)iy * p);
      const int iz = (int)((Z == gf.NZ - 1) ? gf.nc[2] - 1 : Z / p), k = (int)(Z - (long)iz * p);
      const int cy = iy / 2, sy = iy % 2, cz = iz / 2, sz = iz % 2;
      double v = 0.0;
      for (int kp = 0; kp < n; ++kp)
        for (int jp = 0; jp < n; ++jp)
          v += P[(sy * n + j) * n + jp] * P[(sz * n + k) * n + kp] *
               u[((long)(cz * p + kp) * gc.NY + (cy * p + jp)) * gc.NX + (gc.NX - 1)];
      u[gc.N + (Z * gf.NY + Y) * gf.NX] = v;
    }
}

void orc2_dof_coordinates(const orc_mesh2 *m, double *xyz)
{
  orc_dof_coordinates(&m->coarse, xyz);
  orc_dof_coordinates(&m->fine, xyz + 3 * orc_n_dofs(&m->coarse));
}

/* ------------------------------------------------------------- mapped meshes
 * Unstructured hexahedral meshes given by each cell's corners and its cell->DoF
 * map (the form a deal.II DoFHandler / MatrixFree layout takes after renumbering
 * each cell's DoFs lexicographically), with homogeneous affine constraints
 * (AffineConstraints lines: x_c = sum_e w_e x_{m_e}; masters unconstrained).
 * The operator is sum_K C_K^T A_K C_K as in read_dof_values /
 * distribute_local_to_global with constraints (heat_diffuse_operator.cpp:
 * 199-241): constrained DoFs are read through their constraint and never
 * written; Dirichlet DoFs are read as 0 and never written. */
static void mapped_entries(const orc_mapped *m, long gidx, long *cnt, const long **g, const double **w,
                           long *own, double *one)
{
  if (m->cons_ptr && m->cons_ptr[gidx + 1] > m->cons_ptr[gidx]) {
    *cnt = m->cons_ptr[gidx + 1] - m->cons_ptr[gidx];
    *g = m->cons_idx + m->cons_ptr[gidx];
    *w = m->cons_w + m->cons_ptr[gidx];
  } else {
    *own = gidx;
    *one = 1.0;
    *cnt = 1;
    *g = own;
    *w = one;
  }
}

static int mapped_constrained(const orc_mapped *m, long gidx)
{
  return m->cons_ptr && m->cons_ptr[gidx + 1] > m->cons_ptr[gidx];
}

static void mapped_geo(const orc_mapped *m, geo_t *g)
{
  orc_mesh dummy = {3, m->degree, {1, 1, 1}, NULL};
  geo_init(&dummy, g);
  g->N = m->n_dofs; /* component stride of a nodal velocity field */
}

static void mapped_cell(const orc_mapped *m, long K, double vc[8][3], long *idx, int nqt)
{
  for (int v = 0; v < 8; ++v)
    for (int a = 0; a < 3; ++a) vc[v][a] = m->cell_vertices[(K * 8 + v) * 3 + a];
  for (int t = 0; t < nqt; ++t) idx[t] = m->cell_dofs[K * nqt + t];
}

void orcm_vmult(const orc_mapped *m, const orc_op *op, double *dst, const double *src)
{
  geo_t g;
  mapped_geo(m, &g);
  const int n = g.n, nqt = n * n * n;
  memset(dst, 0, sizeof(double) * m->n_dofs);
  double *A = (double *)malloc(sizeof(double) * nqt * nqt);
  for (long K = 0; K < m->n_cells; ++K) {
    double vc[8][3], ul[MAXN3];
    long idx[MAXN3];
    mapped_cell(m, K, vc, idx, nqt);
    element_matrix_vc(op, &g, vc, idx, tau_vc(op, &g, vc, idx), A);
    add_face_matrices(m, op, &g, K, vc, idx, A);
    for (int t = 0; t < nqt; ++t) {
      long cnt, own;
      double one, v = 0.0;
      const long *gg;
      const double *ww;
      mapped_entries(m, idx[t], &cnt, &gg, &ww, &own, &one);
      for (long e = 0; e < cnt; ++e)
        if (!(op->dirichlet && op->dirichlet[gg[e]])) v += ww[e] * src[gg[e]];
      ul[t] = v;
    }
    for (int t = 0; t < nqt; ++t) {
      double o = 0.0;
      for (int u = 0; u < nqt; ++u) o += A[t * nqt + u] * ul[u];
      long cnt, own;
      double one;
      const long *gg;
      const double *ww;
      mapped_entries(m, idx[t], &cnt, &gg, &ww, &own, &one);
      for (long e = 0; e < cnt; ++e)
        if (!(op->dirichlet && op->dirichlet[gg[e]]) && !mapped_constrained(m, gg[e])) dst[gg[e]] += ww[e] * o;
    }
  }
  free(A);
}

/* (C^T A C)_gg = sum_K sum_{t,u} w_t(g) A_K(t,u) w_u(g); Dirichlet and
 * constrained DoFs get 1 */
void orcm_diagonal(const orc_mapped *m, const orc_op *op, double *diag)
{
  geo_t g;
  mapped_geo(m, &g);
  const int n = g.n, nqt = n * n * n;
  memset(diag, 0, sizeof(double) * m->n_dofs);
  double *A = (double *)malloc(sizeof(double) * nqt * nqt);
  for (long K = 0; K < m->n_cells; ++K) {
    double vc[8][3];
    long idx[MAXN3];
    mapped_cell(m, K, vc, idx, nqt);
    element_matrix_vc(op, &g, vc, idx, tau_vc(op, &g, vc, idx), A);
    add_face_matrices(m, op, &g, K, vc, idx, A);
    /* distinct targets of the cell and their weights per local DoF */
    long tg[4 * MAXN3];
    int nt = 0;
    for (int t = 0; t < nqt; ++t) {
      long cnt, own;
      double one;
      const long *gg;
      const double *ww;
      mapped_entries(m, idx[t], &cnt, &gg, &ww, &own, &one);
      for (long e = 0; e < cnt; ++e) {
        int found = 0;
        for (int q = 0; q < nt; ++q) found |= tg[q] == gg[e];
        if (!found && nt < 4 * MAXN3) tg[nt++] = gg[e];
      }
    }
    for (int q = 0; q < nt; ++q) {
      const long target = tg[q];
      if (mapped_constrained(m, target) || (op->dirichlet && op->dirichlet[target])) continue;
      double wt[MAXN3];
      for (int t = 0; t < nqt; ++t) {
        long cnt, own;
        double one;
        const long *gg;
        const double *ww;
        mapped_entries(m, idx[t], &cnt, &gg, &ww, &own, &one);
        wt[t] = 0.0;
        for (long e = 0; e < cnt; ++e)
          if (gg[e] == target) wt[t] += ww[e];
      }
      double s = 0.0;
      for (int t = 0; t < nqt; ++t)
        if (wt[t] != 0.0)
          for (int u = 0; u < nqt; ++u) s += wt[t] * A[t * nqt + u] * wt[u];
      diag[target] += s;
    }
  }
  for (long i = 0; i < m->n_dofs; ++i)
    if (mapped_constrained(m, i) || (op->dirichlet && op->dirichlet[i])) diag[i] = 1.0;
  free(A);
}
