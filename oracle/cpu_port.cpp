// CPU port of the matrix-free heat / advection-diffusion operator apply and of
// CG with the Jacobi preconditioner: the timed CPU baseline of bench.py (its
// reference arm and cpu_baseline legs).  It is neither the product nor the
// checker -- the oracle (mpdg_oracle.c) checks it (tests/test_cpu_port.py).
//
// What it restates, and from where:
//  * the operators of source/heat/heat_diffuse_operator.cpp:955-1086 (heat
//    tangent: rho_cp/dt u + rho_cp vel.grad u, k(T) grad u, k(T) = k0 (1 + a T))
//    and source/level_set/advection_diffusion_operator.cpp:450-495 (u/dt +
//    theta vel.grad u, theta D grad u), on FE_Q(p) with Gauss-Lobatto nodes and
//    QGauss(p+1) (source/utilities/fe_util.cpp:18-57), trilinear geometry;
//  * the cell loop of deal.II's MatrixFree as the reference uses it
//    (heat_diffuse_operator.cpp:199-241): dst zeroed, then per cell gather
//    (constrained DoFs read as 0), sum-factorised evaluate / integrate, scatter
//    (constrained DoFs never written);
//  * the diagonal by unit vectors per cell (MatrixFreeTools::compute_diagonal,
//    heat_diffuse_operator.cpp:297-391) and SolverCG with ReductionControl and
//    the Jacobi preconditioner (linear_solver.hpp:26-134,
//    preconditioner_jacobi.hpp:50-69).
//
// How it is tuned, the way deal.II's MatrixFree is on a CPU:
//  * the degree is a template parameter (every 1D loop has compile-time bounds);
//  * cells are processed in SIMD batches of kW cells of one parity colour, the
//    batch index innermost in every array, so -O3 -march=native vectorises each
//    contraction over the batch (deal.II's VectorizedArray);
//  * geometry is precomputed once: on general cells the 7 merged values per
//    quadrature point (c_mass JxW and the symmetric c_diff k(T_q) JxW J^-1 J^-T,
//    the temperature folded in once, as it is fixed during a linear solve) and
//    c_vel JxW J^-1 vel; on axis-aligned uniform cells nothing but h;
//  * OpenMP over the batches of a colour: cells of a colour share no DoF, so the
//    scatter needs no atomics; one parallel region per apply.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

constexpr int kW = 8;  // cells per SIMD batch
constexpr int kMaxN = 5;

// ------------------------------------------------------------ 1D tables
void legendre(int n, double x, double &p, double &dp)
{
  double p0 = 1.0, p1 = x;
  if (n == 0) {
    p = 1.0;
    dp = 0.0;
    return;
  }
  for (int k = 2; k <= n; ++k) {
    const double pk = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
    p0 = p1;
    p1 = pk;
  }
  p = p1;
  dp = n * (x * p1 - p0) / (x * x - 1.0);
}

// Gauss-Legendre points and weights on [0, 1] (Newton on P_n)
void gauss01(int n, double *x, double *w)
{
  for (int i = 0; i < n; ++i) {
    double z = std::cos(M_PI * (i + 0.75) / (n + 0.5)), p = 0, dp = 1;
    for (int it = 0; it < 100; ++it) {
      legendre(n, z, p, dp);
      const double dz = p / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    legendre(n, z, p, dp);
    x[n - 1 - i] = 0.5 * (z + 1.0);
    w[n - 1 - i] = 1.0 / ((1.0 - z * z) * dp * dp);
  }
}

// Gauss-Lobatto points on [0, 1]: the end points and the roots of P'_{n-1}
void lobatto01(int n, double *x)
{
  x[0] = 0.0;
  x[n - 1] = 1.0;
  const int m = n - 1;
  for (int i = 1; i < m; ++i) {
    double z = -std::cos(M_PI * i / m);
    for (int it = 0; it < 100; ++it) {
      // P'_m(z) = 0: Newton with P'' from the Legendre equation
      double p, dp;
      legendre(m, z, p, dp);
      const double d2p = (2.0 * z * dp - m * (m + 1.0) * p) / (1.0 - z * z);
      const double dz = dp / d2p;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    x[i] = 0.5 * (z + 1.0);
  }
}

// value and derivative at t of the i-th Lagrange polynomial on the nodes z
void lagrange(int n, const double *z, int i, double t, double &v, double &d)
{
  v = 1.0;
  d = 0.0;
  for (int j = 0; j < n; ++j) {
    if (j == i) continue;
    const double f = (t - z[j]) / (z[i] - z[j]);
    d = d * f + v / (z[i] - z[j]);
    v *= f;
  }
}

struct Tables {
  int n = 0;
  double S[kMaxN * kMaxN];   // S[q n + i] = l_i(x_q), l_i on the Gauss-Lobatto nodes
  double Dc[kMaxN * kMaxN];  // Dc[q n + r] = l'_r(x_q), l_r on the Gauss points (collocation)
  double w[kMaxN], xq[kMaxN];
  double D[kMaxN * kMaxN];   // D[q n + i] = l_i'(x_q) (nodal basis; the geometry set-up)
};

Tables make_tables(int p)
{
  Tables t;
  const int n = p + 1;
  t.n = n;
  double z[kMaxN];
  gauss01(n, t.xq, t.w);
  lobatto01(n, z);
  for (int q = 0; q < n; ++q)
    for (int i = 0; i < n; ++i) {
      double v, d;
      lagrange(n, z, i, t.xq[q], v, d);
      t.S[q * n + i] = v;
      t.D[q * n + i] = d;
      lagrange(n, t.xq, i, t.xq[q], v, d);
      t.Dc[q * n + i] = d;
    }
  return t;
}

// ------------------------------------------------------------ operator data
struct Port {
  int degree = 1, n = 2;
  int nc[3] = {1, 1, 1};
  long NX = 0, NY = 0, NZ = 0, N = 0;
  int kind = 0;  // 0 heat, 1 advection-diffusion
  bool uniform = false;
  double h[3] = {0, 0, 0}, origin[3] = {0, 0, 0};
  double c_mass = 0, c_vel = 0, c_diff = 0;
  int vel_kind = 0;  // 0 none, 2 vortex
  std::vector<uint8_t> mask;  // constrained DoFs (empty: none)
  Tables T;
  // batches of kW cells of one colour: first batch of each colour, lattice
  // offsets of the cells' first DoF (-1: padding lane), batch flags
  int colour_first[9] = {0};
  std::vector<long> g0;          // [batch][kW]
  std::vector<int> cell_xyz;     // [batch][kW][3]
  std::vector<uint8_t> touches;  // batch has a constrained DoF
  // general cells: [batch][7][n^3][kW] merged coefficients, [batch][3][n^3][kW] velocity terms
  std::vector<double> coef, velb;
  // uniform cells with the vortex velocity: sin / cos of pi x at the quadrature
  // x-coordinates of every cell column ([ix n + qx]) and likewise in y
  std::vector<double> sinx, cosx, siny, cosy;
  long n_batches = 0;
};

// trilinear map of a cell's 8 corners at reference point xi: position and Jacobian
void map_point(const double (&v)[8][3], const double xi[3], double x[3], double J[3][3])
{
  for (int a = 0; a < 3; ++a) {
    x[a] = 0.0;
    for (int b = 0; b < 3; ++b) J[a][b] = 0.0;
  }
  for (int c = 0; c < 8; ++c) {
    const int bx = c & 1, by = (c >> 1) & 1, bz = (c >> 2) & 1;
    const double fx = bx ? xi[0] : 1 - xi[0], fy = by ? xi[1] : 1 - xi[1], fz = bz ? xi[2] : 1 - xi[2];
    const double dx = bx ? 1 : -1, dy = by ? 1 : -1, dz = bz ? 1 : -1;
    const double N = fx * fy * fz, dN[3] = {dx * fy * fz, fx * dy * fz, fx * fy * dz};
    for (int a = 0; a < 3; ++a) {
      x[a] += N * v[c][a];
      for (int b = 0; b < 3; ++b) J[a][b] += v[c][a] * dN[b];
    }
  }
}

double inverse3(const double (&J)[3][3], double (&I)[3][3])
{
  const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1], c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2],
               c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
  const double id = 1.0 / det;
  I[0][0] = c00 * id;
  I[1][0] = c01 * id;
  I[2][0] = c02 * id;
  I[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
  I[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
  I[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
  I[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
  I[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
  I[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
  return det;
}

void vortex(const double x[3], double u[3])
{
  u[0] = std::sin(M_PI * x[0]) * std::cos(M_PI * x[1]);
  u[1] = -std::cos(M_PI * x[0]) * std::sin(M_PI * x[1]);
  u[2] = 0.0;
}

// ------------------------------------------------------------ sum factorisation
// out = M applied along direction dir (transposed when TR) to every line of the
// n^3 tensor; arrays are [n^3][kW], the batch innermost
template <int n, int dir, bool TR, bool ADD>
inline void sweep(const double *__restrict M, const double (*__restrict in)[kW], double (*__restrict out)[kW])
{
  constexpr int s = dir == 0 ? 1 : dir == 1 ? n : n * n;
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b) {
      const int base = dir == 0 ? a * n * n + b * n : dir == 1 ? a * n * n + b : a * n + b;
      for (int q = 0; q < n; ++q) {
        double acc[kW];
#pragma omp simd
        for (int w = 0; w < kW; ++w) acc[w] = ADD ? out[base + q * s][w] : 0.0;
        for (int k = 0; k < n; ++k) {
          const double m = TR ? M[k * n + q] : M[q * n + k];
#pragma omp simd
          for (int w = 0; w < kW; ++w) acc[w] += m * in[base + k * s][w];
        }
#pragma omp simd
        for (int w = 0; w < kW; ++w) out[base + q * s][w] = acc[w];
      }
    }
}

// the local operator on one batch: u (nodal, [n^3][kW]) -> out (nodal)
template <int n>
inline void local_apply(const Port &P, long batch, const double (*__restrict u)[kW], double (*__restrict out)[kW])
{
  constexpr int n2 = n * n, n3 = n2 * n;
  alignas(64) double t1[n3][kW], t2[n3][kW], uq[n3][kW], g0[n3][kW], g1[n3][kW], g2[n3][kW];
  const Tables &T = P.T;
  // values at the Gauss points, then collocation derivatives
  sweep<n, 0, false, false>(T.S, u, t1);
  sweep<n, 1, false, false>(T.S, t1, t2);
  sweep<n, 2, false, false>(T.S, t2, uq);
  sweep<n, 0, false, false>(T.Dc, uq, g0);
  sweep<n, 1, false, false>(T.Dc, uq, g1);
  sweep<n, 2, false, false>(T.Dc, uq, g2);
  if (!P.uniform) {
    const double *c = P.coef.data() + batch * 7L * n3 * kW;
    const double *vb = P.velb.empty() ? nullptr : P.velb.data() + batch * 3L * n3 * kW;
    for (int q = 0; q < n3; ++q) {
      const double *cm = c + (long)q * kW, *G00 = cm + n3 * kW, *G01 = cm + 2 * n3 * kW, *G02 = cm + 3 * n3 * kW,
                   *G11 = cm + 4 * n3 * kW, *G12 = cm + 5 * n3 * kW, *G22 = cm + 6 * n3 * kW;
#pragma omp simd
      for (int w = 0; w < kW; ++w) {
        const double a = g0[q][w], b = g1[q][w], d = g2[q][w];
        double v = cm[w] * uq[q][w];
        if (vb) v += vb[(long)q * kW + w] * a + vb[(long)(n3 + q) * kW + w] * b + vb[(long)(2 * n3 + q) * kW + w] * d;
        uq[q][w] = v;
        g0[q][w] = G00[w] * a + G01[w] * b + G02[w] * d;
        g1[q][w] = G01[w] * a + G11[w] * b + G12[w] * d;
        g2[q][w] = G02[w] * a + G12[w] * b + G22[w] * d;
      }
    }
  } else {
    const double hv = P.h[0] * P.h[1] * P.h[2];
    const int *xyz = P.cell_xyz.data() + batch * kW * 3;
    for (int qz = 0; qz < n; ++qz)
      for (int qy = 0; qy < n; ++qy)
        for (int qx = 0; qx < n; ++qx) {
          const int q = (qz * n + qy) * n + qx;
          const double JxW = hv * T.w[qx] * T.w[qy] * T.w[qz];
          const double km = P.c_mass * JxW, kd0 = P.c_diff * JxW / (P.h[0] * P.h[0]),
                       kd1 = P.c_diff * JxW / (P.h[1] * P.h[1]), kd2 = P.c_diff * JxW / (P.h[2] * P.h[2]);
          if (P.vel_kind == 2) {
            double b0[kW], b1[kW];
            const double c0 = P.c_vel * JxW / P.h[0], c1 = P.c_vel * JxW / P.h[1];
            for (int w = 0; w < kW; ++w) {
              const int ax = xyz[3 * w] * n + qx, ay = xyz[3 * w + 1] * n + qy;
              b0[w] = c0 * P.sinx[ax] * P.cosy[ay];
              b1[w] = -c1 * P.cosx[ax] * P.siny[ay];
            }
#pragma omp simd
            for (int w = 0; w < kW; ++w) {
              uq[q][w] = km * uq[q][w] + b0[w] * g0[q][w] + b1[w] * g1[q][w];
              g0[q][w] *= kd0;
              g1[q][w] *= kd1;
              g2[q][w] *= kd2;
            }
          } else {
#pragma omp simd
            for (int w = 0; w < kW; ++w) {
              uq[q][w] *= km;
              g0[q][w] *= kd0;
              g1[q][w] *= kd1;
              g2[q][w] *= kd2;
            }
          }
        }
  }
  // test functions: S^T (val + Dc_x^T f_x + Dc_y^T f_y + Dc_z^T f_z)
  sweep<n, 0, true, true>(T.Dc, g0, uq);
  sweep<n, 1, true, true>(T.Dc, g1, uq);
  sweep<n, 2, true, true>(T.Dc, g2, uq);
  sweep<n, 2, true, false>(T.S, uq, t1);
  sweep<n, 1, true, false>(T.S, t1, t2);
  sweep<n, 0, true, false>(T.S, t2, out);
}

template <int n>
void apply_batch(const Port &P, long batch, const double *__restrict src, double *__restrict dst)
{
  constexpr int n2 = n * n, n3 = n2 * n;
  constexpr int p = n - 1;
  alignas(64) double u[n3][kW], out[n3][kW];
  const long *g0 = P.g0.data() + batch * kW;
  const long NX = P.NX, zs = P.NX * P.NY;
  const bool masked = !P.mask.empty() && P.touches[batch];
  (void)p;
  for (int w = 0; w < kW; ++w) {
    const long b = g0[w];
    if (b < 0) {
      for (int l = 0; l < n3; ++l) u[l][w] = 0.0;
      continue;
    }
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          const long g = b + k * zs + j * NX + i;
          u[(k * n + j) * n + i][w] = (masked && P.mask[g]) ? 0.0 : src[g];
        }
  }
  local_apply<n>(P, batch, u, out);
  for (int w = 0; w < kW; ++w) {
    const long b = g0[w];
    if (b < 0) continue;
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          const long g = b + k * zs + j * NX + i;
          if (!(masked && P.mask[g])) dst[g] += out[(k * n + j) * n + i][w];
        }
  }
}

template <int n>
void vmult_n(const Port &P, double *dst, const double *src)
{
#pragma omp parallel
  {
#pragma omp for schedule(static)
    for (long i = 0; i < P.N; ++i) dst[i] = 0.0;
    for (int c = 0; c < 8; ++c) {
#pragma omp for schedule(static)
      for (long b = P.colour_first[c]; b < P.colour_first[c + 1]; ++b) apply_batch<n>(P, b, src, dst);
    }
  }
}

void vmult(const Port &P, double *dst, const double *src)
{
  switch (P.n) {
    case 2: vmult_n<2>(P, dst, src); break;
    case 3: vmult_n<3>(P, dst, src); break;
    case 4: vmult_n<4>(P, dst, src); break;
    case 5: vmult_n<5>(P, dst, src); break;
    default: break;
  }
}

// diagonal by unit vectors per cell batch (MatrixFreeTools::compute_diagonal)
template <int n>
void diagonal_n(const Port &P, double *diag)
{
  constexpr int n3 = n * n * n;
#pragma omp parallel
  {
#pragma omp for schedule(static)
    for (long i = 0; i < P.N; ++i) diag[i] = 0.0;
    for (int c = 0; c < 8; ++c) {
#pragma omp for schedule(static)
      for (long b = P.colour_first[c]; b < P.colour_first[c + 1]; ++b) {
        alignas(64) double u[n3][kW], out[n3][kW], loc[n3][kW];
        const long *g0 = P.g0.data() + b * kW;
        for (int l = 0; l < n3; ++l) {
          for (int m = 0; m < n3; ++m)
            for (int w = 0; w < kW; ++w) u[m][w] = (m == l) ? 1.0 : 0.0;
          local_apply<n>(P, b, u, out);
          for (int w = 0; w < kW; ++w) loc[l][w] = out[l][w];
        }
        const long NX = P.NX, zs = P.NX * P.NY;
        for (int w = 0; w < kW; ++w) {
          if (g0[w] < 0) continue;
          for (int k = 0; k < n; ++k)
            for (int j = 0; j < n; ++j)
              for (int i = 0; i < n; ++i) {
                const long g = g0[w] + k * zs + j * NX + i;
                diag[g] += loc[(k * n + j) * n + i][w];
              }
        }
      }
    }
#pragma omp for schedule(static)
    for (long i = 0; i < P.N; ++i)
      if (!P.mask.empty() && P.mask[i]) diag[i] = 1.0;
  }
}

void build(Port &P, const double *vert, const double *temperature, double k_alpha)
{
  const int p = P.degree, n = P.n, n3 = n * n * n;
  P.T = make_tables(p);
  // colour-major batches of kW cells, lexicographic (x fastest) within a colour
  std::vector<long> g0;
  std::vector<int> xyz;
  std::vector<uint8_t> touches;
  long nb = 0;
  for (int c = 0; c < 8; ++c) {
    P.colour_first[c] = (int)nb;
    std::vector<int> cells;
    for (int iz = (c >> 2) & 1; iz < P.nc[2]; iz += 2)
      for (int iy = (c >> 1) & 1; iy < P.nc[1]; iy += 2)
        for (int ix = c & 1; ix < P.nc[0]; ix += 2) {
          cells.push_back(ix);
          cells.push_back(iy);
          cells.push_back(iz);
        }
    const long cnt = (long)cells.size() / 3;
    for (long b0 = 0; b0 < cnt; b0 += kW, ++nb) {
      bool t = false;
      for (int w = 0; w < kW; ++w) {
        const long ci = b0 + w;
        if (ci < cnt) {
          const int ix = cells[3 * ci], iy = cells[3 * ci + 1], iz = cells[3 * ci + 2];
          const long base = ((long)iz * p * P.NY + (long)iy * p) * P.NX + (long)ix * p;
          g0.push_back(base);
          xyz.insert(xyz.end(), {ix, iy, iz});
          if (!P.mask.empty())
            for (int k = 0; k < n && !t; ++k)
              for (int j = 0; j < n && !t; ++j)
                for (int i = 0; i < n && !t; ++i)
                  if (P.mask[base + (k * P.NY + j) * P.NX + i]) t = true;
        } else {
          g0.push_back(-1);
          xyz.insert(xyz.end(), {0, 0, 0});
        }
      }
      touches.push_back(t ? 1 : 0);
    }
  }
  P.colour_first[8] = (int)nb;
  P.n_batches = nb;
  P.g0.swap(g0);
  P.cell_xyz.swap(xyz);
  P.touches.swap(touches);
  if (P.uniform) {
    if (P.vel_kind == 2) {
      P.sinx.resize((size_t)P.nc[0] * n);
      P.cosx.resize(P.sinx.size());
      P.siny.resize((size_t)P.nc[1] * n);
      P.cosy.resize(P.siny.size());
      for (int i = 0; i < P.nc[0]; ++i)
        for (int q = 0; q < n; ++q) {
          const double x = P.origin[0] + (i + P.T.xq[q]) * P.h[0];
          P.sinx[i * n + q] = std::sin(M_PI * x);
          P.cosx[i * n + q] = std::cos(M_PI * x);
        }
      for (int i = 0; i < P.nc[1]; ++i)
        for (int q = 0; q < n; ++q) {
          const double y = P.origin[1] + (i + P.T.xq[q]) * P.h[1];
          P.siny[i * n + q] = std::sin(M_PI * y);
          P.cosy[i * n + q] = std::cos(M_PI * y);
        }
    }
    return;
  }
  // general cells: merged coefficients per quadrature point, set up once
  P.coef.assign((size_t)nb * 7 * n3 * kW, 0.0);
  if (P.vel_kind != 0) P.velb.assign((size_t)nb * 3 * n3 * kW, 0.0);
  const long VX = P.nc[0] + 1, VY = P.nc[1] + 1;
#pragma omp parallel for schedule(static)
  for (long b = 0; b < nb; ++b)
    for (int w = 0; w < kW; ++w) {
      if (P.g0[b * kW + w] < 0) continue;
      const int ix = P.cell_xyz[(b * kW + w) * 3], iy = P.cell_xyz[(b * kW + w) * 3 + 1],
                iz = P.cell_xyz[(b * kW + w) * 3 + 2];
      double v[8][3];
      for (int c = 0; c < 8; ++c) {
        const long vi = ((long)(iz + ((c >> 2) & 1)) * VY + (iy + ((c >> 1) & 1))) * VX + ix + (c & 1);
        for (int a = 0; a < 3; ++a) v[c][a] = vert[3 * vi + a];
      }
      // temperature at the Gauss points (nodal values interpolated with S)
      std::vector<double> Tq(n3, 0.0);
      if (temperature && k_alpha != 0.0) {
        std::vector<double> Tl(n3), t1(n3), t2(n3);
        const long base = P.g0[b * kW + w];
        for (int k = 0; k < n; ++k)
          for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) Tl[(k * n + j) * n + i] = temperature[base + (k * P.NY + j) * P.NX + i];
        for (int k = 0; k < n; ++k)
          for (int j = 0; j < n; ++j)
            for (int q = 0; q < n; ++q) {
              double s = 0;
              for (int i = 0; i < n; ++i) s += P.T.S[q * n + i] * Tl[(k * n + j) * n + i];
              t1[(k * n + j) * n + q] = s;
            }
        for (int k = 0; k < n; ++k)
          for (int q = 0; q < n; ++q)
            for (int i = 0; i < n; ++i) {
              double s = 0;
              for (int j = 0; j < n; ++j) s += P.T.S[q * n + j] * t1[(k * n + j) * n + i];
              t2[(k * n + q) * n + i] = s;
            }
        for (int q = 0; q < n; ++q)
          for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
              double s = 0;
              for (int k = 0; k < n; ++k) s += P.T.S[q * n + k] * t2[(k * n + j) * n + i];
              Tq[(q * n + j) * n + i] = s;
            }
      }
      for (int qz = 0; qz < n; ++qz)
        for (int qy = 0; qy < n; ++qy)
          for (int qx = 0; qx < n; ++qx) {
            const int q = (qz * n + qy) * n + qx;
            const double xi[3] = {P.T.xq[qx], P.T.xq[qy], P.T.xq[qz]};
            double x[3], J[3][3], I[3][3];
            map_point(v, xi, x, J);
            const double det = inverse3(J, I);
            const double JxW = det * P.T.w[qx] * P.T.w[qy] * P.T.w[qz];
            const double k = P.c_diff * (1.0 + k_alpha * Tq[q]);
            double G[3][3];
            for (int a = 0; a < 3; ++a)
              for (int c = 0; c < 3; ++c) {
                double s = 0;
                for (int e = 0; e < 3; ++e) s += I[a][e] * I[c][e];
                G[a][c] = k * JxW * s;
              }
            double *cb = P.coef.data() + ((size_t)b * 7 * n3) * kW;
            const double vals[7] = {P.c_mass * JxW, G[0][0], G[0][1], G[0][2], G[1][1], G[1][2], G[2][2]};
            for (int m = 0; m < 7; ++m) cb[((size_t)m * n3 + q) * kW + w] = vals[m];
            if (P.vel_kind == 2) {
              double vel[3];
              vortex(x, vel);
              double *vb = P.velb.data() + ((size_t)b * 3 * n3) * kW;
              for (int a = 0; a < 3; ++a) {
                double s = 0;
                for (int e = 0; e < 3; ++e) s += I[a][e] * vel[e];
                vb[((size_t)a * n3 + q) * kW + w] = P.c_vel * JxW * s;
              }
            }
          }
    }
}

double dotp(long N, const double *a, const double *b)
{
  double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (long i = 0; i < N; ++i) s += a[i] * b[i];
  return s;
}

}  // namespace

extern "C" {

typedef struct {
  int degree;
  int nc[3];
  const double *vertices;        // (nc0+1)(nc1+1)(nc2+1) x 3, x fastest
  const uint8_t *dirichlet_mask; // n_dofs or NULL
  int uniform;                   // 1: axis-aligned uniform box cells (only h is used)
  int kind;                      // 0 heat, 1 advection-diffusion
  double dt, rho_cp, k0, k_alpha;
  const double *temperature;     // heat with k_alpha != 0: nodal T (n_dofs)
  double theta, diffusivity;
  int vel_kind;                  // 0 none, 2 vortex
} port_desc;

void *port_create(const port_desc *d)
{
  if (!d || d->degree < 1 || d->degree > 4) return nullptr;
  Port *P = new Port();
  P->degree = d->degree;
  P->n = d->degree + 1;
  for (int a = 0; a < 3; ++a) P->nc[a] = d->nc[a];
  P->NX = (long)d->nc[0] * d->degree + 1;
  P->NY = (long)d->nc[1] * d->degree + 1;
  P->NZ = (long)d->nc[2] * d->degree + 1;
  P->N = P->NX * P->NY * P->NZ;
  P->kind = d->kind;
  const bool heat = d->kind == 0;
  P->c_mass = heat ? d->rho_cp / d->dt : 1.0 / d->dt;
  P->c_vel = heat ? d->rho_cp : d->theta;
  P->c_diff = heat ? d->k0 : d->theta * d->diffusivity;
  P->vel_kind = d->vel_kind;
  // k(T) on uniform cells goes through the general coefficient stream
  P->uniform = d->uniform && !(heat && d->k_alpha != 0.0);
  if (d->dirichlet_mask) P->mask.assign(d->dirichlet_mask, d->dirichlet_mask + P->N);
  const double *V = d->vertices;
  for (int a = 0; a < 3; ++a) {
    P->origin[a] = V[a];
    const long last = (a == 0) ? d->nc[0] : (a == 1) ? (long)d->nc[1] * (d->nc[0] + 1)
                                                     : (long)d->nc[2] * (d->nc[0] + 1) * (d->nc[1] + 1);
    P->h[a] = (V[3 * last + a] - V[a]) / d->nc[a];
  }
  build(*P, V, heat ? d->temperature : nullptr, heat ? d->k_alpha : 0.0);
  return P;
}

void port_destroy(void *p) { delete static_cast<Port *>(p); }

long port_n_dofs(void *p) { return static_cast<Port *>(p)->N; }

int port_threads(void) { return omp_get_max_threads(); }

void port_vmult(void *p, double *dst, const double *src) { vmult(*static_cast<Port *>(p), dst, src); }

void port_diagonal(void *p, double *diag)
{
  const Port &P = *static_cast<Port *>(p);
  switch (P.n) {
    case 2: diagonal_n<2>(P, diag); break;
    case 3: diagonal_n<3>(P, diag); break;
    case 4: diagonal_n<4>(P, diag); break;
    case 5: diagonal_n<5>(P, diag); break;
    default: break;
  }
}

// CG + Jacobi from x (deal.II SolverCG, ReductionControl: converged when
// |r| <= max(abs_tol, rel_tol |r0|)); the inverse diagonal uses the heat
// operator's threshold rule (1/d where |d| > 1e-10, else 1).  Returns the
// iterations, or -1 without convergence.
int port_cg_jacobi(void *p, double *x, const double *b, double rel_tol, double abs_tol, int max_it,
                   double *final_residual)
{
  const Port &P = *static_cast<Port *>(p);
  const long N = P.N;
  std::vector<double> r(N), z(N), q(N), Ap(N), inv(N);
  port_diagonal(p, inv.data());
#pragma omp parallel for schedule(static)
  for (long i = 0; i < N; ++i) inv[i] = std::fabs(inv[i]) > 1e-10 ? 1.0 / inv[i] : 1.0;
  vmult(P, Ap.data(), x);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < N; ++i) r[i] = b[i] - Ap[i];
  const double res0 = std::sqrt(dotp(N, r.data(), r.data()));
  const double tol = std::max(abs_tol, rel_tol * res0);
  double res = res0;
  int it = 0;
  if (res0 > tol) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < N; ++i) {
      z[i] = inv[i] * r[i];
      q[i] = z[i];
    }
    double rz = dotp(N, r.data(), z.data());
    while (true) {
      vmult(P, Ap.data(), q.data());
      const double alpha = rz / dotp(N, q.data(), Ap.data());
      double rr = 0.0;
#pragma omp parallel for reduction(+ : rr) schedule(static)
      for (long i = 0; i < N; ++i) {
        x[i] += alpha * q[i];
        r[i] -= alpha * Ap[i];
        rr += r[i] * r[i];
      }
      ++it;
      res = std::sqrt(rr);
      if (res <= tol || it >= max_it) break;
#pragma omp parallel for schedule(static)
      for (long i = 0; i < N; ++i) z[i] = inv[i] * r[i];
      const double rz_new = dotp(N, r.data(), z.data());
      const double beta = rz_new / rz;
      rz = rz_new;
#pragma omp parallel for schedule(static)
      for (long i = 0; i < N; ++i) q[i] = z[i] + beta * q[i];
    }
  }
  if (final_residual) *final_residual = res;
  return res <= tol ? it : -1;
}

}  // extern "C"
