// Matrix-free cell kernels of the heat and advection-diffusion operators (sm_100a).
//
// One cell is handled by n*n threads (n = degree + 1): thread (i, j) keeps the
// DoF column (i, j, 0..n-1) in registers.  Contractions along z run in
// registers, along x and y through a per-cell shared-memory tile.  Values at
// the Gauss points come from the 1D interpolation matrix S (Gauss-Lobatto basis
// at the Gauss points); gradients from the collocation derivative matrix Dc on
// the Gauss points, which is exact for the interpolated polynomial.  The
// quadrature-point kernels restate
//   heat:    source/heat/heat_diffuse_operator.cpp:1029-1078 (tangent),
//            :479-505 (residual), with the k(T) = k0 (1 + a T) law;
//   advdiff: source/level_set/advection_diffusion_operator.cpp:471-493 (tangent),
//            :318-353 (rhs).
// Cells of one parity colour share no DoF; a launch per colour adds the cell
// results into dst with plain loads and stores (atomic-free, deterministic).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <vector>

#include "mpdg_internal.h"

namespace mpdg {

// ------------------------------------------------------------------ 1D tables

// even-odd form of an n x n matrix M with M[n-1-q][n-1-k] = +-M[q][k]
// (values at, or derivatives on, point sets symmetric about 1/2): for q, k < h
// = n/2, e = (M[q][k] + M[q][n-1-k]) / 2 and o = (M[q][k] - M[q][n-1-k]) / 2
// act on the even and odd combinations in[k] +- in[n-1-k]; cm holds the middle
// column M[q][h], rm the middle row M[h][k] and mm = M[h][h] (n odd)
constexpr int kMaxH = kMaxN / 2;
template <typename Real>
struct EO {
  Real e[kMaxH * kMaxH];
  Real o[kMaxH * kMaxH];
  Real cm[kMaxH];
  Real rm[kMaxH];
  Real mm;
};

template <typename Real>
struct Tables {
  Real S[kMaxN * kMaxN];   // S[q*n+i]  = phi_i(x_q): Gauss-Lobatto basis at Gauss points
  Real D[kMaxN * kMaxN];   // D[q*n+i]  = phi_i'(x_q)
  Real Dc[kMaxN * kMaxN];  // Dc[q*n+r] = l_r'(x_q): collocation derivative on Gauss points
  Real w[kMaxN];           // Gauss weights on [0,1]
  Real x[kMaxN];           // Gauss points on [0,1]
  // hanging-node interpolation of a 2:1 refined face: H[(s*n + j)*n + j'] =
  // Gauss-Lobatto basis j' at the fine node (s + z_j) / 2 of subface s
  Real H[2 * kMaxN * kMaxN];
  // even-odd forms of S (symmetric), Dc (antisymmetric) and their transposes
  EO<Real> eS, eSt, eDc, eDct;
};

__constant__ Tables<double> c_tab64[kMaxDegree + 1];
__constant__ Tables<float> c_tab32[kMaxDegree + 1];

template <typename Real>
__device__ __forceinline__ const Tables<Real> &tab(int p);
template <>
__device__ __forceinline__ const Tables<double> &tab<double>(int p) { return c_tab64[p]; }
template <>
__device__ __forceinline__ const Tables<float> &tab<float>(int p) { return c_tab32[p]; }

namespace {

void legendre(int n, double x, double &p, double &dp)
{
  double p0 = 1.0, p1 = x;
  if (n == 0) { p = 1.0; dp = 0.0; return; }
  for (int k = 2; k <= n; ++k) {
    const double pk = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
    p0 = p1;
    p1 = pk;
  }
  p = p1;
  dp = n * (x * p1 - p0) / (x * x - 1.0);
}

// Gauss-Legendre points/weights on [0,1], ascending
void gauss(int n, double *x, double *w)
{
  for (int i = 0; i < n; ++i) {
    double z = std::cos(M_PI * (i + 0.75) / (n + 0.5)), p, dp;
    for (int it = 0; it < 100; ++it) {
      legendre(n, z, p, dp);
      const double dz = p / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    legendre(n, z, p, dp);
    x[n - 1 - i] = 0.5 * (1.0 + z);
    w[n - 1 - i] = 1.0 / ((1.0 - z * z) * dp * dp);
  }
}

// Gauss-Lobatto nodes on [0,1]: endpoints and roots of P'_{n-1}
void lobatto(int n, double *x)
{
  const int m = n - 1;
  x[0] = 0.0;
  x[n - 1] = 1.0;
  for (int i = 1; i < n - 1; ++i) {
    double z = -std::cos(M_PI * i / m), p, dp;
    for (int it = 0; it < 100; ++it) {
      legendre(m, z, p, dp);
      const double ddp = (2.0 * z * dp - m * (m + 1.0) * p) / (1.0 - z * z);
      const double dz = dp / ddp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    x[i] = 0.5 * (1.0 + z);
  }
}

// value and derivative at t of the Lagrange polynomial through nodes z, index i
void lagrange(int n, const double *z, int i, double t, double &v, double &d)
{
  v = 1.0;
  d = 0.0;
  for (int j = 0; j < n; ++j)
    if (j != i) v *= (t - z[j]) / (z[i] - z[j]);
  for (int k = 0; k < n; ++k) {
    if (k == i) continue;
    double s = 1.0 / (z[i] - z[k]);
    for (int j = 0; j < n; ++j)
      if (j != i && j != k) s *= (t - z[j]) / (z[i] - z[j]);
    d += s;
  }
}

bool g_tables_ready = false;

// even-odd form of the n x n matrix M (row-major, or its transpose)
template <typename Real>
void even_odd(int n, const double *M, bool transpose, EO<Real> &t)
{
  auto m = [&](int q, int k) { return transpose ? M[k * n + q] : M[q * n + k]; };
  const int h = n / 2;
  for (int q = 0; q < h; ++q) {
    for (int k = 0; k < h; ++k) {
      t.e[q * kMaxH + k] = (Real)(0.5 * (m(q, k) + m(q, n - 1 - k)));
      t.o[q * kMaxH + k] = (Real)(0.5 * (m(q, k) - m(q, n - 1 - k)));
    }
    t.cm[q] = (n & 1) ? (Real)m(q, h) : Real(0);
    t.rm[q] = (n & 1) ? (Real)m(h, q) : Real(0);
  }
  t.mm = (n & 1) ? (Real)m(h, h) : Real(0);
}

void upload_tables()
{
  if (g_tables_ready) return;
  Tables<double> t64[kMaxDegree + 1];
  Tables<float> t32[kMaxDegree + 1];
  std::memset(t64, 0, sizeof(t64));
  std::memset(t32, 0, sizeof(t32));
  for (int p = 1; p <= kMaxDegree; ++p) {
    const int n = p + 1;
    double xq[kMaxN], wq[kMaxN], zl[kMaxN];
    gauss(n, xq, wq);
    lobatto(n, zl);
    for (int q = 0; q < n; ++q) {
      t64[p].w[q] = wq[q];
      t64[p].x[q] = xq[q];
      for (int i = 0; i < n; ++i) {
        double v, d;
        lagrange(n, zl, i, xq[q], v, d);
        t64[p].S[q * n + i] = v;
        t64[p].D[q * n + i] = d;
        lagrange(n, xq, i, xq[q], v, d);
        t64[p].Dc[q * n + i] = d;
      }
    }
    for (int sub = 0; sub < 2; ++sub)
      for (int j = 0; j < n; ++j)
        for (int jp = 0; jp < n; ++jp) {
          double v, d;
          lagrange(n, zl, jp, 0.5 * (sub + zl[j]), v, d);
          t64[p].H[(sub * n + j) * n + jp] = v;
        }
    for (int k = 0; k < 2 * kMaxN * kMaxN; ++k) t32[p].H[k] = (float)t64[p].H[k];
    for (int k = 0; k < kMaxN * kMaxN; ++k) {
      t32[p].S[k] = (float)t64[p].S[k];
      t32[p].D[k] = (float)t64[p].D[k];
      t32[p].Dc[k] = (float)t64[p].Dc[k];
    }
    for (int k = 0; k < kMaxN; ++k) {
      t32[p].w[k] = (float)t64[p].w[k];
      t32[p].x[k] = (float)t64[p].x[k];
    }
    even_odd(n, t64[p].S, false, t64[p].eS);
    even_odd(n, t64[p].S, true, t64[p].eSt);
    even_odd(n, t64[p].Dc, false, t64[p].eDc);
    even_odd(n, t64[p].Dc, true, t64[p].eDct);
    even_odd(n, t64[p].S, false, t32[p].eS);
    even_odd(n, t64[p].S, true, t32[p].eSt);
    even_odd(n, t64[p].Dc, false, t32[p].eDc);
    even_odd(n, t64[p].Dc, true, t32[p].eDct);
  }
  MPDG_CUDA(cudaMemcpyToSymbol(c_tab64, t64, sizeof(t64)));
  MPDG_CUDA(cudaMemcpyToSymbol(c_tab32, t32, sizeof(t32)));
  g_tables_ready = true;
}

}  // namespace

void shape_1d(int p, double *S, double *D, double *w, double *x)
{
  const int n = p + 1;
  double zl[kMaxN];
  gauss(n, x, w);
  lobatto(n, zl);
  for (int q = 0; q < n; ++q)
    for (int i = 0; i < n; ++i) lagrange(n, zl, i, x[q], S[q * n + i], D[q * n + i]);
}

// ------------------------------------------------------------ kernel params

// MODE_SUPG: MODE_LINEAR plus the advection-diffusion SUPG flux
// tau_K u (c_mass u + c_vel u.grad u - c_diff lap u) (advection_diffusion_operator.cpp:450-495)
enum { MODE_LINEAR = 0, MODE_HEAT_RESIDUAL = 1, MODE_SUPG = 2 };
constexpr int kMaxMultiVec = 4;
enum { GEOM_UNIFORM = 0, GEOM_GENERAL = 1 };

template <typename Real>
struct KP {
  const Real *src;        // LINEAR: operand (or phi_old for the advdiff rhs); RESIDUAL: T_old
  Real *dst;
  const Real *T;          // k(T) field (LINEAR) / current T (RESIDUAL)
  const Real *q_src;      // RESIDUAL: nodal heat source (may be null)
  const Real *metric;     // GENERAL: [cell][7][n^3] = JxW, G00 G01 G02 G11 G12 G22
  const Real *velb;       // GENERAL + velocity: [cell][3][n^3] = JxW J^-1 u
  const Real *trig;       // UNIFORM vortex: sin(pi x), cos(pi x), sin(pi y), cos(pi y)
  const Real *tau;        // SUPG: per colour-major cell tau_K
  // heat material law (MPDG_MAT_*); LINEAR uses c_mass, c_vel, c_diff, k_alpha
  int mat, two_phase_sharp, solid_sharp, vol_specific;
  Real mrho[3], mcp[3], mk[3], solidus, liquidus, inv_mushy, dt_inv;
  Real latent;  // latent heat of fusion (0: no apparent capacity)
  int ac_type;  // its apparent-capacity profile (MPDG_AC_*)
  const Real *Told;       // T_old (laws with a solid phase), or T - T_old when told_inc
  int told_inc;
  // mapped mesh: cell->DoF map [colour-major cell][n^3]; skip the cells that
  // touch a constrained DoF in the diagonal kernel
  const int *cmap;
  int skip_constrained;
  // host side only: restrict the colour launches to cell layers [zlo, zhi)
  int zlo, zhi;
  // coefficient stream copies carry an L2 evict-first hint
  int stream_evict_first;
  // launched as a programmatic dependent of the previous colour launch
  int pdl;
  // multi-vector apply: nvec operands msrc[v] -> mdst[v]
  int nvec;
  const Real *msrc[kMaxMultiVec];
  Real *mdst[kMaxMultiVec];
  const Real *Hs;         // level-set heaviside (two-phase laws)
  int supg_lap;           // SUPG with diffusion: the Laplacian term
  const Real *lam;        // SUPG with diffusion, general cells: [cell][3][n^3] curvature term (lam_kernel)
  const uint8_t *dmask;
  const uint8_t *cell_flags;
  const uint4 *cell_mask;
  const uint4 *cell_first;  // mapped meshes: first-touch local DoFs per cell (null: every cell adds)
  long NX, NY;
  int nc[3];
  int trig_stride;
  int par[3], cn[3];
  // exact division of a colour-local cell index by cn[0] and cn[0]*cn[1]:
  // q = (x * magic) >> 40 with magic = ceil(2^40 / d), exact for x * d < 2^40
  unsigned long long div0_magic, div01_magic;
  long ccount, cfirst;
  // uniform geometry: 1/h, 1/h^2 and the cell volume, so the kernels divide nothing
  Real ih[3], ih2[3], hvol;
  Real h[3], origin[3];
  Real c_mass, c_vel, c_diff, k_alpha;
  int vel_kind;
  Real vel_param[3];
  int masked_read, masked_write, full_tangent;
  // fine block of a two-level mesh: the hanging DoFs (cells ix = 0, i = 0) read
  // the coarse face through the interpolation H and stage their contributions
  const Real *hsrc;      // coarse block's values (null: no hanging DoFs)
  Real *hstage;          // [fine interface cell iz*hnc1 + iy][k' n + j']
  const uint8_t *hmask;  // coarse block's Dirichlet mask (or null)
  long hNXc, hNYc;       // coarse lattice
  int hnc1;              // fine cells in y
};

// mapped meshes (mapped.cuh)
template <typename Real>
void launch_mapped_apply(Op &op, Real *dst, const Real *src);
template <typename Real>
void mapped_condense(Op &op, Real *dst);
void launch_mapped_diagonal(Op &op, double *diag);

template <int n>
struct Cfg {
  static constexpr int cpb = (n == 2) ? 32 : (n == 3) ? 14 : (n == 4) ? 8 : 5;
};

// ---------------------------------------------------- contraction helpers
// tile layout: t[k*n*n + j*n + i]

template <int n, typename Real, bool TR>
__device__ __forceinline__ void cz(const Real *M, const Real (&in)[n], Real (&out)[n])
{
#pragma unroll
  for (int q = 0; q < n; ++q) {
    Real s = 0;
#pragma unroll
    for (int k = 0; k < n; ++k) s += (TR ? M[k * n + q] : M[q * n + k]) * in[k];
    out[q] = s;
  }
}

// out = M in through the even-odd form of M (ANTI: M[n-1-q][n-1-k] = -M[q][k]):
// n = 5 takes 21 (20) instructions instead of 25
template <int n, typename Real, bool ANTI>
__device__ __forceinline__ void ceo(const EO<Real> &M, const Real (&in)[n], Real (&out)[n])
{
  constexpr int h = n / 2;
  Real e[h], o[h];
#pragma unroll
  for (int k = 0; k < h; ++k) {
    e[k] = in[k] + in[n - 1 - k];
    o[k] = in[k] - in[n - 1 - k];
  }
#pragma unroll
  for (int q = 0; q < h; ++q) {
    Real a = M.e[q * kMaxH] * e[0];
#pragma unroll
    for (int k = 1; k < h; ++k) a += M.e[q * kMaxH + k] * e[k];
    if (n & 1) a += M.cm[q] * in[h];
    Real b = M.o[q * kMaxH] * o[0];
#pragma unroll
    for (int k = 1; k < h; ++k) b += M.o[q * kMaxH + k] * o[k];
    out[q] = a + b;
    out[n - 1 - q] = ANTI ? b - a : a - b;
  }
  if (n & 1) {
    if (ANTI) {
      Real s = M.rm[0] * o[0];
#pragma unroll
      for (int k = 1; k < h; ++k) s += M.rm[k] * o[k];
      out[h] = s;
    } else {
      Real s = M.mm * in[h];
#pragma unroll
      for (int k = 0; k < h; ++k) s += M.rm[k] * e[k];
      out[h] = s;
    }
  }
}

// the 1D contractions of the warp-per-cell apply: the even-odd form where it
// saves instructions (n = 5), the plain product otherwise
template <int n, typename Real, bool TR, bool ANTI>
__device__ __forceinline__ void c1(const Real *M, const EO<Real> &eo, const Real (&in)[n], Real (&out)[n])
{
  if constexpr (n == 5)
    ceo<n, Real, ANTI>(eo, in, out);
  else
    cz<n, Real, TR>(M, in, out);
}

template <int n, typename Real, bool TR>
__device__ __forceinline__ void cx(const Real *M, const Real *t, int i, int j, Real (&out)[n])
{
#pragma unroll
  for (int k = 0; k < n; ++k) {
    Real s = 0;
#pragma unroll
    for (int r = 0; r < n; ++r) s += (TR ? M[r * n + i] : M[i * n + r]) * t[k * n * n + j * n + r];
    out[k] = s;
  }
}

template <int n, typename Real, bool TR>
__device__ __forceinline__ void cy(const Real *M, const Real *t, int i, int j, Real (&out)[n])
{
#pragma unroll
  for (int k = 0; k < n; ++k) {
    Real s = 0;
#pragma unroll
    for (int r = 0; r < n; ++r) s += (TR ? M[r * n + j] : M[j * n + r]) * t[k * n * n + r * n + i];
    out[k] = s;
  }
}

template <int n, typename Real>
__device__ __forceinline__ void put(Real *t, int i, int j, const Real (&v)[n])
{
#pragma unroll
  for (int k = 0; k < n; ++k) t[k * n * n + j * n + i] = v[k];
}

// nodal column -> values at the Gauss points (thread (i,j) ends with qp (i,j,*))
template <int n, typename Real>
__device__ __forceinline__ void to_qp(const Real *S, Real *t, int i, int j, const Real (&u)[n],
                                      Real (&v)[n])
{
  Real a[n];
  cz<n, Real, false>(S, u, a);
  put<n>(t, i, j, a);
  __syncthreads();
  cy<n, Real, false>(S, t, i, j, v);
  __syncthreads();
  put<n>(t, i, j, v);
  __syncthreads();
  cx<n, Real, false>(S, t, i, j, a);
  __syncthreads();
#pragma unroll
  for (int k = 0; k < n; ++k) v[k] = a[k];
}

// values at the Gauss points -> reference gradients (collocation)
template <int n, typename Real>
__device__ __forceinline__ void grad_qp(const Real *Dc, Real *t, int i, int j, const Real (&v)[n],
                                        Real (&gx)[n], Real (&gy)[n], Real (&gz)[n])
{
  put<n>(t, i, j, v);
  __syncthreads();
  cx<n, Real, false>(Dc, t, i, j, gx);
  cy<n, Real, false>(Dc, t, i, j, gy);
  cz<n, Real, false>(Dc, v, gz);
  __syncthreads();
}

// test with (value, reference gradient) and return the nodal column
template <int n, typename Real>
__device__ __forceinline__ void from_qp(const Real *S, const Real *Dc, Real *t0, Real *t1, int i,
                                        int j, const Real (&val)[n], const Real (&fx)[n],
                                        const Real (&fy)[n], const Real (&fz)[n], Real (&out)[n])
{
  Real a[n], b[n];
  put<n>(t0, i, j, fx);
  put<n>(t1, i, j, fy);
  __syncthreads();
  cx<n, Real, true>(Dc, t0, i, j, a);
  cy<n, Real, true>(Dc, t1, i, j, b);
  cz<n, Real, true>(Dc, fz, out);
#pragma unroll
  for (int k = 0; k < n; ++k) a[k] += b[k] + out[k] + val[k];
  __syncthreads();
  put<n>(t0, i, j, a);
  __syncthreads();
  cx<n, Real, true>(S, t0, i, j, b);
  __syncthreads();
  put<n>(t0, i, j, b);
  __syncthreads();
  cy<n, Real, true>(S, t0, i, j, a);
  cz<n, Real, true>(S, a, out);
}

template <typename Real, int n>
__device__ __forceinline__ void uniform_velocity(const KP<Real> &p, const Tables<Real> &T, int ix,
                                                 int iy, int iz, int i, int j, int k, Real u[3])
{
  if (p.vel_kind == MPDG_VEL_VORTEX) {
    const Real sx = p.trig[ix * n + i], cxv = p.trig[p.trig_stride + ix * n + i];
    const Real sy = p.trig[2 * p.trig_stride + iy * n + j],
               cyv = p.trig[3 * p.trig_stride + iy * n + j];
    u[0] = sx * cyv;
    u[1] = -cxv * sy;
    u[2] = 0;
  } else if (p.vel_kind == MPDG_VEL_ROTATION) {
    const Real x = p.origin[0] + (ix + T.x[i]) * p.h[0];
    const Real z = p.origin[2] + (iz + T.x[k]) * p.h[2];
    u[0] = p.vel_param[0] * z;
    u[1] = 0;
    u[2] = -p.vel_param[0] * x;
  } else {
    u[0] = p.vel_param[0];
    u[1] = p.vel_param[1];
    u[2] = p.vel_param[2];
  }
}

// --------------------------------------------------------- material laws
// (rho c_p / dt, rho c_p, k) at a quadrature point and their T derivatives
// (Material::compute_parameters_internal, material.templates.hpp:213-760; the
// solid fraction of :748-760, the cubic solid/liquid interpolation of :546-600,
// the gas weight of :513-523; rho c_p by the product rule,
// heat_diffuse_operator.cpp:1176-1199)
template <typename Real>
__device__ __forceinline__ Real ls_value(Real fs, Real vl, Real vs)
{
  if (fs == Real(0)) return vl;
  if (fs == Real(1)) return vs;
  return vl + (vs - vl) * (Real(-2) * fs * fs * fs + Real(3) * fs * fs);
}

template <typename Real>
__device__ __forceinline__ Real ls_deriv(Real fs, Real inv_mushy, Real vl, Real vs)
{
  if (fs == Real(0) || fs == Real(1)) return Real(0);
  return -inv_mushy * (vs - vl) * (Real(-6) * fs * fs + Real(6) * fs);
}

// apparent heat capacity of the latent heat of fusion L over the mushy zone
// [Ts, Tl] as a function of the solid fraction fs, and its T derivative
// (ApparentCapacity::evaluate / compute_temperature_derivative,
// source/heat/apparent_capacity.cpp); 0 outside 0 < fs < 1.  constant: L/(Tl-Ts);
// poly4_bell: L r b(xi), r = 2/(Tl-Ts), xi = 1 - 2 fs, b(x) = 15/16 (x^2-1)^2;
// qlq: at T = Tl - fs (Tl-Ts) two ramps 0 -> 2L/(Tl-Ts) -> 0 over the halves of
// the zone, each quadratic with zero end slope over (Tl-Ts)/6 and linear between
template <typename Real>
__device__ __forceinline__ void qlq_ramp(Real x, Real x1, Real x2, Real y1, Real y2, Real delta, Real &f, Real &df)
{
  const Real s = (y2 - y1) / (x2 - x1 - delta);
  if (x < x1 + delta) {
    f = y1 + Real(0.5) * s / delta * (x - x1) * (x - x1);
    df = s * (x - x1) / delta;
  } else if (x > x2 - delta) {
    f = y2 - Real(0.5) * s / delta * (x2 - x) * (x2 - x);
    df = s * (x2 - x) / delta;
  } else {
    f = y1 + Real(0.5) * s * delta + s * (x - x1 - delta);
    df = s;
  }
}

template <typename Real>
__device__ __forceinline__ void apparent_capacity(const KP<Real> &p, Real fs, Real &c, Real &dc)
{
  c = dc = Real(0);
  if (!(p.latent > Real(0)) || fs <= Real(0) || fs >= Real(1)) return;
  const Real dT = p.liquidus - p.solidus;
  if (p.ac_type == MPDG_AC_CONSTANT) {
    c = p.latent / dT;
  } else if (p.ac_type == MPDG_AC_POLY4_BELL) {
    const Real r = Real(2) / dT, xi = Real(1) - Real(2) * fs, x2 = xi * xi;
    c = p.latent * r * (Real(15.0 / 16.0) * x2 * x2 - Real(15.0 / 8.0) * x2 + Real(15.0 / 16.0));
    dc = p.latent * r * r * (Real(15.0 / 4.0) * x2 * xi - Real(15.0 / 4.0) * xi);
  } else {
    const Real T = p.liquidus - fs * dT, Tp = Real(0.5) * (p.solidus + p.liquidus), Cp = Real(2) * p.latent / dT,
               delta = dT / Real(6);
    if (T <= Tp) qlq_ramp<Real>(T, p.solidus, Tp, Real(0), Cp, delta, c, dc);
    else qlq_ramp<Real>(T, Tp, p.liquidus, Cp, Real(0), delta, c, dc);
  }
}

template <typename Real>
__device__ __forceinline__ void law_eval(const KP<Real> &p, Real T, Real H, Real &cm, Real &cv, Real &kq,
                                         Real &dcm, Real &dcv, Real &dk)
{
  if (p.mat == MPDG_MAT_LINEAR) {
    cm = p.c_mass;
    cv = p.c_vel;
    kq = p.c_diff * (Real(1) + p.k_alpha * T);
    dk = p.c_diff * p.k_alpha;
    dcm = dcv = Real(0);
    return;
  }
  const bool gas = p.mat == MPDG_MAT_GAS_LIQUID || p.mat == MPDG_MAT_GAS_LIQUID_SOLID;
  const bool sol = p.mat == MPDG_MAT_LIQUID_SOLID || p.mat == MPDG_MAT_GAS_LIQUID_SOLID;
  Real fs = 0;
  if (sol) {
    fs = p.solid_sharp ? (T < p.solidus ? Real(1) : Real(0))
                       : fmin(fmax((p.liquidus - T) * p.inv_mushy, Real(0)), Real(1));
  }
  const Real w = gas ? (p.two_phase_sharp ? (H > Real(0.5) ? Real(1) : Real(0)) : H) : Real(1);
  Real v[4], dv[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const Real vl = (e == 0) ? p.mrho[1] : (e == 1) ? p.mcp[1] : (e == 2) ? p.mk[1] : p.mrho[1] * p.mcp[1];
    const Real vs = (e == 0) ? p.mrho[2] : (e == 1) ? p.mcp[2] : (e == 2) ? p.mk[2] : p.mrho[2] * p.mcp[2];
    const Real vg = (e == 0) ? p.mrho[0] : (e == 1) ? p.mcp[0] : (e == 2) ? p.mk[0] : p.mrho[0] * p.mcp[0];
    v[e] = sol ? ls_value(fs, vl, vs) : vl;
    dv[e] = sol ? ls_deriv(fs, p.inv_mushy, vl, vs) : Real(0);
    if (sol && e == 1) {
      // latent heat: the solid/liquid c_p gains the apparent capacity
      // (material.templates.hpp:566-578, 604-616), before the gas weighting
      Real c, dc;
      apparent_capacity<Real>(p, fs, c, dc);
      v[1] += c;
      dv[1] += dc;
    }
    if (gas) {
      v[e] = (Real(1) - w) * vg + w * v[e];
      dv[e] = w * dv[e];
    }
  }
  const Real rc = p.vol_specific ? v[3] : v[0] * v[1];
  const Real drc = p.vol_specific ? dv[3] : dv[1] * v[0] + dv[0] * v[1];
  cm = rc * p.dt_inv;
  cv = rc;
  kq = v[2];
  dcm = drc * p.dt_inv;
  dcv = drc;
  dk = dv[2];
}

#include "apply_warp.cuh"
#include "apply_lane.cuh"
#include "batch_apply.cuh"

// ------------------------------------------------------------ the cell kernel

template <int P, typename Real, int GEOM, int MODE, bool KT>
__global__ void __launch_bounds__(128) cell_kernel(const KP<Real> p)
{
  constexpr int n = P + 1, n2 = n * n, n3 = n2 * n, CPB = Cfg<n>::cpb;
  __shared__ Real sm[CPB][2][n3];
  __shared__ Real sS[n2], sDc[n2];
  const Tables<Real> &T = tab<Real>(P);
  const int tid = threadIdx.x, slot = threadIdx.y;
  const int i = tid % n, j = tid / n;
  // 1D tables in shared memory: rows are indexed by the thread's i/j, which
  // the constant cache would serialise
  if (slot == 0) {
    sS[tid] = T.S[tid];
    sDc[tid] = T.Dc[tid];
  }
  __syncthreads();
  const long cidx = (long)blockIdx.x * CPB + slot;
  const bool active = cidx < p.ccount;
  int ix = 0, iy = 0, iz = 0;
  if (active) {
    const long a = cidx % p.cn[0], b = (cidx / p.cn[0]) % p.cn[1], c = cidx / ((long)p.cn[0] * p.cn[1]);
    ix = 2 * (int)a + p.par[0];
    iy = 2 * (int)b + p.par[1];
    iz = 2 * (int)c + p.par[2];
  }
  const long cell = p.cfirst + cidx;
  const long zs = p.NX * p.NY;
  const long g0 = ((long)(iz * P) * p.NY + (iy * P + j)) * p.NX + (ix * P + i);
  // global DoFs of the thread's column: the lattice, or the cell->DoF map of a
  // mapped mesh
  long gk[n];
#pragma unroll
  for (int k = 0; k < n; ++k) gk[k] = (p.cmap && active) ? (long)p.cmap[cell * n3 + k * n2 + j * n + i] : g0 + k * zs;
  const bool bflag = active && p.cell_flags && (p.cell_flags[cell] & 1);
  Real *t0 = sm[slot][0], *t1 = sm[slot][1];

  Real u[n], uq[n], gx[n], gy[n], gz[n];
#pragma unroll
  for (int k = 0; k < n; ++k) {
    Real v = 0;
    if (active) {
      v = p.src[gk[k]];
      if (MODE != MODE_HEAT_RESIDUAL && p.masked_read && bflag && p.dmask[gk[k]]) v = 0;
    }
    u[k] = v;
  }

  // temperature field at the Gauss points (k(T) law, Newton residual)
  Real Tq[n], Tgx[n], Tgy[n], Tgz[n];
  const bool needT = KT || MODE == MODE_HEAT_RESIDUAL;
  if (needT) {
    Real tl[n];
#pragma unroll
    for (int k = 0; k < n; ++k) tl[k] = active ? p.T[gk[k]] : Real(0);
    to_qp<n>(sS, t1, i, j, tl, Tq);
    if (MODE == MODE_HEAT_RESIDUAL || p.full_tangent) grad_qp<n>(sDc, t1, i, j, Tq, Tgx, Tgy, Tgz);
  }
  // material-law fields at the Gauss points: heaviside (two-phase laws), T_old
  // (Newton terms of laws with a solid phase)
  Real Hq[n], Oq[n];
  if (needT && p.Hs) {
    Real hl[n];
#pragma unroll
    for (int k = 0; k < n; ++k) hl[k] = active ? p.Hs[gk[k]] : Real(0);
    to_qp<n>(sS, t1, i, j, hl, Hq);
  }
  if (KT && MODE != MODE_HEAT_RESIDUAL && p.full_tangent && p.Told) {
    Real ol[n];
#pragma unroll
    for (int k = 0; k < n; ++k) ol[k] = active ? p.Told[gk[k]] : Real(0);
    to_qp<n>(sS, t1, i, j, ol, Oq);
  }
  Real oq[n], hq[n];
  if (MODE == MODE_HEAT_RESIDUAL) {
    // u holds T_old here; the residual is evaluated at T
    to_qp<n>(sS, t0, i, j, u, oq);
    Real ql[n];
#pragma unroll
    for (int k = 0; k < n; ++k) ql[k] = (active && p.q_src) ? p.q_src[gk[k]] : Real(0);
    to_qp<n>(sS, t0, i, j, ql, hq);
#pragma unroll
    for (int k = 0; k < n; ++k) {
      uq[k] = Tq[k];
      gx[k] = Tgx[k];
      gy[k] = Tgy[k];
      gz[k] = Tgz[k];
    }
  } else {
    to_qp<n>(sS, t0, i, j, u, uq);
    grad_qp<n>(sDc, t0, i, j, uq, gx, gy, gz);
  }

  // SUPG with diffusion: second reference derivatives d2/dxi_d^2 at the Gauss
  // points, by collocation differentiation of the gradient along its own axis
  // and, on general cells, the mixed ones (d/dy of the x-gradient, d/dz of the
  // x- and y-gradients)
  Real gxx[n], gyy[n], gzz[n], gxy[n], gxz[n], gyz[n];
  if (MODE == MODE_SUPG && p.supg_lap) {
    put<n>(t0, i, j, gx);
    put<n>(t1, i, j, gy);
    __syncthreads();
    cx<n, Real, false>(sDc, t0, i, j, gxx);
    cy<n, Real, false>(sDc, t1, i, j, gyy);
    cz<n, Real, false>(sDc, gz, gzz);
    if (GEOM == GEOM_GENERAL) {
      cy<n, Real, false>(sDc, t0, i, j, gxy);
      cz<n, Real, false>(sDc, gx, gxz);
      cz<n, Real, false>(sDc, gy, gyz);
    }
    __syncthreads();
  }

  // quadrature-point kernel
  Real val[n], fx[n], fy[n], fz[n];
#pragma unroll
  for (int k = 0; k < n; ++k) {
    Real JxW, G00, G01, G02, G11, G12, G22, b0 = 0, b1 = 0, b2 = 0;
    if (GEOM == GEOM_GENERAL) {
      const Real *m = p.metric + cell * metric_stride(n) + k * n2 + j * n + i;
      if (active) {
        JxW = m[0];
        G00 = m[n3];
        G01 = m[2 * n3];
        G02 = m[3 * n3];
        G11 = m[4 * n3];
        G12 = m[5 * n3];
        G22 = m[6 * n3];
        if (p.vel_kind != MPDG_VEL_NONE) {
          const Real *vb = p.velb + cell * velb_stride(n) + k * n2 + j * n + i;
          b0 = vb[0];
          b1 = vb[n3];
          b2 = vb[2 * n3];
        }
      } else {
        JxW = G00 = G11 = G22 = 1;
        G01 = G02 = G12 = 0;
      }
    } else {
      JxW = p.h[0] * p.h[1] * p.h[2] * T.w[i] * T.w[j] * T.w[k];
      G00 = JxW / (p.h[0] * p.h[0]);
      G11 = JxW / (p.h[1] * p.h[1]);
      G22 = JxW / (p.h[2] * p.h[2]);
      G01 = G02 = G12 = 0;
      if (p.vel_kind == MPDG_VEL_NODAL) {
        if (active) {  // the stream JxW J^-1 u of the velocity field
          const Real *vb = p.velb + cell * velb_stride(n) + k * n2 + j * n + i;
          b0 = vb[0];
          b1 = vb[n3];
          b2 = vb[2 * n3];
        }
      } else if (p.vel_kind != MPDG_VEL_NONE) {
        Real uv[3];
        uniform_velocity<Real, n>(p, T, ix, iy, iz, i, j, k, uv);
        b0 = JxW * uv[0] / p.h[0];
        b1 = JxW * uv[1] / p.h[1];
        b2 = JxW * uv[2] / p.h[2];
      }
    }
    Real cm = p.c_mass, cv = p.c_vel, kq = p.c_diff, dcm = 0, dcv = 0, dk = 0;
    if (needT) law_eval<Real>(p, Tq[k], p.Hs ? Hq[k] : Real(0), cm, cv, kq, dcm, dcv, dk);
    const Real adv = b0 * gx[k] + b1 * gy[k] + b2 * gz[k];
    Real f0, f1, f2;
    if (GEOM == GEOM_GENERAL) {
      f0 = G00 * gx[k] + G01 * gy[k] + G02 * gz[k];
      f1 = G01 * gx[k] + G11 * gy[k] + G12 * gz[k];
      f2 = G02 * gx[k] + G12 * gy[k] + G22 * gz[k];
    } else {
      f0 = G00 * gx[k];
      f1 = G11 * gy[k];
      f2 = G22 * gz[k];
    }
    if (MODE == MODE_HEAT_RESIDUAL) {
      // -( rho_cp/dt (T - T_old) - q + rho_cp vel.grad T ) N - k(T) grad T . grad N
      val[k] = -(cm * JxW * (uq[k] - oq[k]) - JxW * hq[k] + cv * adv);
      fx[k] = -kq * f0;
      fy[k] = -kq * f1;
      fz[k] = -kq * f2;
    } else {
      val[k] = cm * JxW * uq[k] + cv * adv;
      fx[k] = kq * f0;
      fy[k] = kq * f1;
      fz[k] = kq * f2;
      if (MODE == MODE_SUPG) {
        // tau_K u r tested with grad N: reference flux tau_K r JxW J^-1 u = tau_K r b,
        // with u.grad u = adv / JxW and lap u = G : H_xi / JxW - lam . grad_xi u
        // (G = JxW J^-1 J^-T, lam from lam_kernel; lam = 0 and G diagonal on
        // axis-aligned cells)
        const Real tau = active ? p.tau[cell] : Real(0);
        Real r = p.c_mass * uq[k] + p.c_vel * adv / JxW;
        if (p.supg_lap) {
          Real lap;
          if (GEOM == GEOM_GENERAL) {
            lap = (G00 * gxx[k] + G11 * gyy[k] + G22 * gzz[k] +
                   Real(2) * (G01 * gxy[k] + G02 * gxz[k] + G12 * gyz[k])) / JxW;
            if (active) {
              const Real *lm = p.lam + cell * 3 * n3 + k * n2 + j * n + i;
              lap -= lm[0] * gx[k] + lm[n3] * gy[k] + lm[2 * n3] * gz[k];
            }
          } else {
            lap = p.ih2[0] * gxx[k] + p.ih2[1] * gyy[k] + p.ih2[2] * gzz[k];
          }
          r -= p.c_diff * lap;
        }
        const Real tr = tau * r;
        fx[k] += tr * b0;
        fy[k] += tr * b1;
        fz[k] += tr * b2;
      }
      if (KT && p.full_tangent) {
        // dk/dT grad T du, tested with grad N: G (reference grad T) scaled by u
        const Real du = dk * uq[k];
        if (GEOM == GEOM_GENERAL) {
          fx[k] += du * (G00 * Tgx[k] + G01 * Tgy[k] + G02 * Tgz[k]);
          fy[k] += du * (G01 * Tgx[k] + G11 * Tgy[k] + G12 * Tgz[k]);
          fz[k] += du * (G02 * Tgx[k] + G12 * Tgy[k] + G22 * Tgz[k]);
        } else {
          fx[k] += du * G00 * Tgx[k];
          fy[k] += du * G11 * Tgy[k];
          fz[k] += du * G22 * Tgz[k];
        }
        // d(rho c_p)/dT ((T - T_old)/dt + u.grad T) du tested with N
        if (p.Told) {
          const Real dT = p.told_inc ? Oq[k] : Tq[k] - Oq[k];
          val[k] += (dcm * dT * JxW + dcv * (b0 * Tgx[k] + b1 * Tgy[k] + b2 * Tgz[k])) * uq[k];
        }
      }
    }
  }

  Real out[n];
  from_qp<n>(sS, sDc, t0, t1, i, j, val, fx, fy, fz, out);

  if (active) {
#pragma unroll
    for (int k = 0; k < n; ++k) {
      const long g = gk[k];
      if (p.masked_write && bflag && p.dmask[g]) continue;
      p.dst[g] += out[k];
    }
  }
}

// --------------------------------------------------------- diagonal kernel
// diag_i = sum_q F_t(q) A_x[qx][ix] A_y[qy][iy] A_z[qz][iz] over the terms t of
// the element matrix diagonal (mass, the six G components, the three velocity
// components), each a product of squared/mixed 1D tables: the same entries
// MatrixFreeTools::compute_diagonal extracts by unit-vector sweeps.

template <int P, int GEOM, bool KT>
__global__ void __launch_bounds__(128) diag_kernel(const KP<double> p)
{
  using Real = double;
  constexpr int n = P + 1, n2 = n * n, n3 = n2 * n, CPB = Cfg<n>::cpb;
  __shared__ Real sm[6][CPB][n3];  // one tile per term group of the y sweep
  __shared__ Real tb[5][n2];  // S^2, D^2, S*D, S, Dc
  const Tables<Real> &T = tab<Real>(P);
  const int tid = threadIdx.x, slot = threadIdx.y;
  const int lin = slot * blockDim.x + tid;
  if (lin < n2) {
    const Real s = T.S[lin], d = T.D[lin];
    tb[0][lin] = s * s;
    tb[1][lin] = d * d;
    tb[2][lin] = s * d;
    tb[3][lin] = s;
    tb[4][lin] = T.Dc[lin];
  }
  __syncthreads();
  const Real *SS = tb[0], *DD = tb[1], *SD = tb[2];
  const int i = tid % n, j = tid / n;
  const long cidx = (long)blockIdx.x * CPB + slot;
  const bool active = cidx < p.ccount;
  int ix = 0, iy = 0, iz = 0;
  if (active) {
    const long a = cidx % p.cn[0], b = (cidx / p.cn[0]) % p.cn[1], c = cidx / ((long)p.cn[0] * p.cn[1]);
    ix = 2 * (int)a + p.par[0];
    iy = 2 * (int)b + p.par[1];
    iz = 2 * (int)c + p.par[2];
  }
  const long cell = p.cfirst + cidx;
  const long zs = p.NX * p.NY;
  const long g0 = ((long)(iz * P) * p.NY + (iy * P + j)) * p.NX + (ix * P + i);
  long gk[n];
#pragma unroll
  for (int k = 0; k < n; ++k) gk[k] = (p.cmap && active) ? (long)p.cmap[cell * n3 + k * n2 + j * n + i] : g0 + k * zs;
  const bool bflag = active && p.cell_flags && (p.cell_flags[cell] & 1);
  // cells of a mapped mesh that touch a constrained DoF get their diagonal share
  // from their element matrices (skip_constrained)
  const bool wr = active && !(p.skip_constrained && p.cell_flags && (p.cell_flags[cell] & 2));
  Real *t = sm[0][slot];

  Real Tq[n], Tgx[n], Tgy[n], Tgz[n];
  if (KT) {
    Real tl[n];
#pragma unroll
    for (int k = 0; k < n; ++k) tl[k] = active ? p.T[gk[k]] : Real(0);
    to_qp<n>(tb[3], t, i, j, tl, Tq);
    if (p.full_tangent) grad_qp<n>(tb[4], t, i, j, Tq, Tgx, Tgy, Tgz);
  }
  Real Hq[n], Oq[n];
  if (KT && p.Hs) {
    Real hl[n];
#pragma unroll
    for (int k = 0; k < n; ++k) hl[k] = active ? p.Hs[gk[k]] : Real(0);
    to_qp<n>(tb[3], t, i, j, hl, Hq);
  }
  if (KT && p.full_tangent && p.Told) {
    Real ol[n];
#pragma unroll
    for (int k = 0; k < n; ++k) ol[k] = active ? p.Told[gk[k]] : Real(0);
    to_qp<n>(tb[3], t, i, j, ol, Oq);
  }
  Real Fm[n], F00[n], F11[n], F22[n], F01[n], F02[n], F12[n], Fb0[n], Fb1[n], Fb2[n];
#pragma unroll
  for (int k = 0; k < n; ++k) {
    Real JxW, G00, G01, G02, G11, G12, G22, b0 = 0, b1 = 0, b2 = 0;
    if (GEOM == GEOM_GENERAL) {
      const Real *m = p.metric + cell * metric_stride(n) + k * n2 + j * n + i;
      JxW = active ? m[0] : 0;
      G00 = active ? m[n3] : 0;
      G01 = active ? m[2 * n3] : 0;
      G02 = active ? m[3 * n3] : 0;
      G11 = active ? m[4 * n3] : 0;
      G12 = active ? m[5 * n3] : 0;
      G22 = active ? m[6 * n3] : 0;
      if (p.vel_kind != MPDG_VEL_NONE && active) {
        const Real *vb = p.velb + cell * velb_stride(n) + k * n2 + j * n + i;
        b0 = vb[0];
        b1 = vb[n3];
        b2 = vb[2 * n3];
      }
    } else {
      JxW = p.h[0] * p.h[1] * p.h[2] * T.w[i] * T.w[j] * T.w[k];
      G00 = JxW / (p.h[0] * p.h[0]);
      G11 = JxW / (p.h[1] * p.h[1]);
      G22 = JxW / (p.h[2] * p.h[2]);
      G01 = G02 = G12 = 0;
      if (p.vel_kind == MPDG_VEL_NODAL) {
        if (active) {  // the stream JxW J^-1 u of the velocity field
          const Real *vb = p.velb + cell * velb_stride(n) + k * n2 + j * n + i;
          b0 = vb[0];
          b1 = vb[n3];
          b2 = vb[2 * n3];
        }
      } else if (p.vel_kind != MPDG_VEL_NONE) {
        Real uv[3];
        uniform_velocity<Real, n>(p, T, ix, iy, iz, i, j, k, uv);
        b0 = JxW * uv[0] / p.h[0];
        b1 = JxW * uv[1] / p.h[1];
        b2 = JxW * uv[2] / p.h[2];
      }
    }
    Real cm = p.c_mass, cv = p.c_vel, kq = p.c_diff, dcm = 0, dcv = 0, dk = 0;
    if (KT) law_eval<Real>(p, Tq[k], p.Hs ? Hq[k] : Real(0), cm, cv, kq, dcm, dcv, dk);
    Fm[k] = cm * JxW;
    if (KT && p.full_tangent && p.Told)
      Fm[k] += dcm * (Tq[k] - Oq[k]) * JxW + dcv * (b0 * Tgx[k] + b1 * Tgy[k] + b2 * Tgz[k]);
    F00[k] = kq * G00;
    F11[k] = kq * G11;
    F22[k] = kq * G22;
    F01[k] = 2 * kq * G01;
    F02[k] = 2 * kq * G02;
    F12[k] = 2 * kq * G12;
    // velocity term phi_i (b . grad phi_i), plus the full-tangent term
    // grad phi_i . (dk G gradT) phi_i, which has the same table structure
    Real e0 = cv * b0, e1 = cv * b1, e2 = cv * b2;
    if (KT && p.full_tangent) {
      e0 += dk * (G00 * Tgx[k] + G01 * Tgy[k] + G02 * Tgz[k]);
      e1 += dk * (G01 * Tgx[k] + G11 * Tgy[k] + G12 * Tgz[k]);
      e2 += dk * (G02 * Tgx[k] + G12 * Tgy[k] + G22 * Tgz[k]);
    }
    Fb0[k] = e0;
    Fb1[k] = e1;
    Fb2[k] = e2;
  }
  // The terms grouped by their (x, y) tables: a group's z contractions are
  // summed in registers, and the y contractions of the groups that share an x
  // table are summed before the one x contraction of each x table.  Groups:
  // 0 (S2,S2): mass, F22, b2   1 (D2,S2): F00   2 (S2,D2): F11
  // 3 (SD,S2): b0, F02         4 (S2,SD): b1, F12   5 (SD,SD): F01
  constexpr int NG = GEOM == GEOM_GENERAL ? 6 : 5;
  {
    Real g[NG][n], a[n];
    cz<n, Real, true>(SS, Fm, g[0]);
    cz<n, Real, true>(DD, F22, a);
#pragma unroll
    for (int k = 0; k < n; ++k) g[0][k] += a[k];
    cz<n, Real, true>(SD, Fb2, a);
#pragma unroll
    for (int k = 0; k < n; ++k) g[0][k] += a[k];
    cz<n, Real, true>(SS, F00, g[1]);
    cz<n, Real, true>(SS, F11, g[2]);
    cz<n, Real, true>(SS, Fb0, g[3]);
    cz<n, Real, true>(SS, Fb1, g[4]);
    if constexpr (GEOM == GEOM_GENERAL) {
      cz<n, Real, true>(SD, F02, a);
#pragma unroll
      for (int k = 0; k < n; ++k) g[3][k] += a[k];
      cz<n, Real, true>(SD, F12, a);
#pragma unroll
      for (int k = 0; k < n; ++k) g[4][k] += a[k];
      cz<n, Real, true>(SS, F01, g[NG - 1]);
    }
    __syncthreads();  // the tiles of the quadrature-point interpolations are free
#pragma unroll
    for (int gi = 0; gi < NG; ++gi) put<n>(sm[gi][slot], i, j, g[gi]);
  }
  __syncthreads();
  Real xs[3][n];  // by x table: S2, D2, SD
  {
    Real b[n];
    cy<n, Real, true>(SS, sm[0][slot], i, j, xs[0]);
    cy<n, Real, true>(DD, sm[2][slot], i, j, b);
#pragma unroll
    for (int k = 0; k < n; ++k) xs[0][k] += b[k];
    cy<n, Real, true>(SD, sm[4][slot], i, j, b);
#pragma unroll
    for (int k = 0; k < n; ++k) xs[0][k] += b[k];
    cy<n, Real, true>(SS, sm[1][slot], i, j, xs[1]);
    cy<n, Real, true>(SS, sm[3][slot], i, j, xs[2]);
    if constexpr (GEOM == GEOM_GENERAL) {
      cy<n, Real, true>(SD, sm[NG - 1][slot], i, j, b);
#pragma unroll
      for (int k = 0; k < n; ++k) xs[2][k] += b[k];
    }
  }
  __syncthreads();
#pragma unroll
  for (int gi = 0; gi < 3; ++gi) put<n>(sm[gi][slot], i, j, xs[gi]);
  __syncthreads();
  Real acc[n];
  {
    Real b[n];
    cx<n, Real, true>(SS, sm[0][slot], i, j, acc);
    cx<n, Real, true>(DD, sm[1][slot], i, j, b);
#pragma unroll
    for (int k = 0; k < n; ++k) acc[k] += b[k];
    cx<n, Real, true>(SD, sm[2][slot], i, j, b);
#pragma unroll
    for (int k = 0; k < n; ++k) acc[k] += b[k];
  }
  if (wr) {
#pragma unroll
    for (int k = 0; k < n; ++k) {
      const long g = gk[k];
      if (p.masked_write && bflag && p.dmask[g]) continue;
      p.dst[g] += acc[k];
    }
  }
}

// ----------------------------------------------------- coefficient merge
// coef[cell][0][q] = c_mass JxW, coef[cell][1+e][q] = c_diff k(T_q) G_e: the
// per-quadrature-point data of the general-geometry apply, rebuilt whenever T
// or dt change (T is constant during a linear solve)

struct ColourSet {
  Colour c[8];
};

template <int P, bool KT>
__global__ void __launch_bounds__(128) merge_kernel(const KP<double> p, const ColourSet cs,
                                                    long n_cells, double *coef64, float *coef32)
{
  constexpr int n = P + 1, n2 = n * n, n3 = n2 * n, CPB = Cfg<n>::cpb, MS = metric_stride(n);
  __shared__ double sm[CPB][n3];
  __shared__ double sS[n2];
  const Tables<double> &T = tab<double>(P);
  const int tid = threadIdx.x, slot = threadIdx.y;
  const int i = tid % n, j = tid / n;
  if (slot == 0) sS[tid] = T.S[tid];
  __syncthreads();
  const long cell = (long)blockIdx.x * CPB + slot;
  const bool active = cell < n_cells;
  int c = 0;
  while (c < 7 && cell >= cs.c[c + 1].first) ++c;
  const Colour &C = cs.c[c];
  const long cidx = active ? cell - C.first : 0;
  const int ix = 2 * (int)(cidx % C.cn[0]) + C.par[0];
  const int iy = 2 * (int)((cidx / C.cn[0]) % C.cn[1]) + C.par[1];
  const int iz = 2 * (int)(cidx / ((long)C.cn[0] * C.cn[1])) + C.par[2];
  double Tq[n];
  if (KT) {
    const long zs = p.NX * p.NY;
    const long g0 = ((long)(iz * P) * p.NY + (iy * P + j)) * p.NX + (ix * P + i);
    double tl[n];
#pragma unroll
    for (int k = 0; k < n; ++k) tl[k] = active ? p.T[g0 + k * zs] : 0.0;
    to_qp<n>(sS, sm[slot], i, j, tl, Tq);
  }
  if (!active) return;
#pragma unroll
  for (int k = 0; k < n; ++k) {
    const int q = k * n2 + j * n + i;
    const double *m = p.metric + cell * MS + q;
    const double kq = KT ? p.c_diff * (1.0 + p.k_alpha * Tq[k]) : p.c_diff;
    double v[7];
    v[0] = p.c_mass * m[0];
#pragma unroll
    for (int e = 1; e < 7; ++e) v[e] = kq * m[e * n3];
#pragma unroll
    for (int e = 0; e < 7; ++e) {
      coef64[cell * MS + e * n3 + q] = v[e];
      if (coef32) coef32[cell * MS + e * n3 + q] = (float)v[e];
    }
  }
}

// ------------------------------------------------------ geometry kernels

// per (cell, qp): JxW and G = JxW J^-1 J^-T of the trilinear map, colour-major
// corners of colour-major cell `cell`: from the vertex lattice, or, on a
// mapped mesh, from the per-cell corners (cellvert, [cell][8][3])
__device__ __forceinline__ void cell_corners(const double *vert, int nc0, int nc1, const Colour *colours,
                                             const double *cellvert, long cell, double V[8][3])
{
  if (cellvert) {
    for (int v = 0; v < 8; ++v)
      for (int a = 0; a < 3; ++a) V[v][a] = cellvert[(cell * 8 + v) * 3 + a];
    return;
  }
  int c = 0;
  while (c < 7 && cell >= colours[c + 1].first) ++c;
  const Colour &C = colours[c];
  const long cidx = cell - C.first;
  const int ix = 2 * (int)(cidx % C.cn[0]) + C.par[0];
  const int iy = 2 * (int)((cidx / C.cn[0]) % C.cn[1]) + C.par[1];
  const int iz = 2 * (int)(cidx / ((long)C.cn[0] * C.cn[1])) + C.par[2];
  for (int v = 0; v < 8; ++v) {
    const long vid = ((long)(iz + ((v >> 2) & 1)) * (nc1 + 1) + (iy + ((v >> 1) & 1))) * (nc0 + 1) + (ix + (v & 1));
    for (int a = 0; a < 3; ++a) V[v][a] = vert[vid * 3 + a];
  }
}

__global__ void metric_kernel(const double *vert, int nc0, int nc1, long n_cells, int P,
                              const Colour *colours, const double *cellvert, double *metric, float *metric32,
                              const double *xq_all, const double *wq_all)
{
  const int n = P + 1, n3 = n * n * n;
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= n_cells * n3) return;
  const long cell = gid / n3;
  const int q = (int)(gid % n3);
  double V[8][3];
  cell_corners(vert, nc0, nc1, colours, cellvert, cell, V);
  const int qi = q % n, qj = (q / n) % n, qk = q / (n * n);
  const double xi[3] = {xq_all[qi], xq_all[qj], xq_all[qk]};
  const double w = wq_all[qi] * wq_all[qj] * wq_all[qk];
  double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int v = 0; v < 8; ++v) {
    const int bx = v & 1, by = (v >> 1) & 1, bz = (v >> 2) & 1;
    const double f[3] = {bx ? xi[0] : 1 - xi[0], by ? xi[1] : 1 - xi[1], bz ? xi[2] : 1 - xi[2]};
    const double df[3] = {bx ? 1.0 : -1.0, by ? 1.0 : -1.0, bz ? 1.0 : -1.0};
    const double dB[3] = {df[0] * f[1] * f[2], f[0] * df[1] * f[2], f[0] * f[1] * df[2]};
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) J[a][b] += V[v][a] * dB[b];
  }
  const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                     J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                     J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
  const double id = 1.0 / det;
  double Ji[3][3];
  Ji[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) * id;
  Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
  Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
  Ji[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) * id;
  Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
  Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
  Ji[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) * id;
  Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
  Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
  const double JxW = det * w;
  double G[6];
  const int ab[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
  for (int e = 0; e < 6; ++e) {
    double s = 0;
    for (int c2 = 0; c2 < 3; ++c2) s += Ji[ab[e][0]][c2] * Ji[ab[e][1]][c2];
    G[e] = JxW * s;
  }
  double *m = metric + cell * metric_stride(n) + q;
  m[0] = JxW;
  for (int e = 0; e < 6; ++e) m[(e + 1) * n3] = G[e];
  if (metric32) {
    float *m32 = metric32 + cell * metric_stride(n) + q;
    m32[0] = (float)JxW;
    for (int e = 0; e < 6; ++e) m32[(e + 1) * n3] = (float)G[e];
  }
}

// per (cell, qp): the curvature term lam of the physical Laplacian on a
// trilinear cell, lap u = sum_ab Gt_ab d2u/dxi_a dxi_b - lam . grad_xi u with
// Gt = J^-1 J^-T, K_j[a][b] = d2 x_j / dxi_a dxi_b (mixed only) and
// lam_a = sum_j (J^-1)_aj sum_bc Gt_bc K_j[b][c]: the chain rule through
// d(J^-1)/dxi_c = -J^-1 (dJ/dxi_c) J^-1.  It is the Laplacian
// FEEvaluation::get_laplacian returns on non-affine cells (SUPG with
// diffusion, advection_diffusion_operator.cpp:483-486).  Layout [cell][3][n^3].
__global__ void lam_kernel(const double *vert, int nc0, int nc1, long n_cells, int P, const Colour *colours,
                           const double *cellvert, const double *xq_all, double *lam, float *lam32)
{
  const int n = P + 1, n3 = n * n * n;
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= n_cells * n3) return;
  const long cell = gid / n3;
  const int q = (int)(gid % n3);
  double V[8][3];
  cell_corners(vert, nc0, nc1, colours, cellvert, cell, V);
  const double xi[3] = {xq_all[q % n], xq_all[(q / n) % n], xq_all[q / (n * n)]};
  double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, K[3][3][3];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      for (int c = 0; c < 3; ++c) K[a][b][c] = 0.0;
  for (int v = 0; v < 8; ++v) {
    double f[3], df[3];
    for (int d = 0; d < 3; ++d) {
      const int bit = (v >> d) & 1;
      f[d] = bit ? xi[d] : 1.0 - xi[d];
      df[d] = bit ? 1.0 : -1.0;
    }
    const double dB[3] = {df[0] * f[1] * f[2], f[0] * df[1] * f[2], f[0] * f[1] * df[2]};
    // mixed second derivatives: (xy) f_z, (xz) f_y, (yz) f_x
    const double d2[3] = {df[0] * df[1] * f[2], df[0] * f[1] * df[2], f[0] * df[1] * df[2]};
    for (int a = 0; a < 3; ++a) {
      for (int b = 0; b < 3; ++b) J[a][b] += V[v][a] * dB[b];
      K[a][0][1] += V[v][a] * d2[0];
      K[a][0][2] += V[v][a] * d2[1];
      K[a][1][2] += V[v][a] * d2[2];
    }
  }
  const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                     J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                     J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
  const double id = 1.0 / det;
  double Ji[3][3];
  Ji[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) * id;
  Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
  Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
  Ji[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) * id;
  Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
  Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
  Ji[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) * id;
  Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
  Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
  double Gt[3][3];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) Gt[a][b] = Ji[a][0] * Ji[b][0] + Ji[a][1] * Ji[b][1] + Ji[a][2] * Ji[b][2];
  double kap[3];
  for (int j = 0; j < 3; ++j) kap[j] = 2.0 * (Gt[0][1] * K[j][0][1] + Gt[0][2] * K[j][0][2] + Gt[1][2] * K[j][1][2]);
  for (int a = 0; a < 3; ++a) {
    const double l = Ji[a][0] * kap[0] + Ji[a][1] * kap[1] + Ji[a][2] * kap[2];
    lam[(cell * 3 + a) * n3 + q] = l;
    if (lam32) lam32[(cell * 3 + a) * n3 + q] = (float)l;
  }
}

// per (cell, qp): b = JxW J^-1 u(x_q) for a prescribed velocity on a general mesh
__global__ void velb_kernel(const double *vert, int nc0, int nc1, long n_cells, int P,
                            const Colour *colours, const double *cellvert, int vel_kind, double s0, double s1,
                            double s2, double *velb, float *velb32, const double *xq_all,
                            const double *wq_all)
{
  const int n = P + 1, n3 = n * n * n;
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= n_cells * n3) return;
  const long cell = gid / n3;
  const int q = (int)(gid % n3);
  double V[8][3];
  cell_corners(vert, nc0, nc1, colours, cellvert, cell, V);
  const int qi = q % n, qj = (q / n) % n, qk = q / (n * n);
  const double xi[3] = {xq_all[qi], xq_all[qj], xq_all[qk]};
  const double w = wq_all[qi] * wq_all[qj] * wq_all[qk];
  double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, x[3] = {0, 0, 0};
  for (int v = 0; v < 8; ++v) {
    const int bx = v & 1, by = (v >> 1) & 1, bz = (v >> 2) & 1;
    const double f[3] = {bx ? xi[0] : 1 - xi[0], by ? xi[1] : 1 - xi[1], bz ? xi[2] : 1 - xi[2]};
    const double df[3] = {bx ? 1.0 : -1.0, by ? 1.0 : -1.0, bz ? 1.0 : -1.0};
    const double dB[3] = {df[0] * f[1] * f[2], f[0] * df[1] * f[2], f[0] * f[1] * df[2]};
    const double B = f[0] * f[1] * f[2];
    for (int a = 0; a < 3; ++a) {
      x[a] += V[v][a] * B;
      for (int b = 0; b < 3; ++b) J[a][b] += V[v][a] * dB[b];
    }
  }
  double u[3] = {0, 0, 0};
  if (vel_kind == MPDG_VEL_VORTEX) {
    u[0] = sin(M_PI * x[0]) * cos(M_PI * x[1]);
    u[1] = -cos(M_PI * x[0]) * sin(M_PI * x[1]);
  } else if (vel_kind == MPDG_VEL_ROTATION) {
    u[0] = s0 * x[2];
    u[2] = -s0 * x[0];
  } else {
    u[0] = s0;
    u[1] = s1;
    u[2] = s2;
  }
  // JxW J^-1 = w adj(J)
  double A[3][3];
  A[0][0] = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  A[0][1] = J[0][2] * J[2][1] - J[0][1] * J[2][2];
  A[0][2] = J[0][1] * J[1][2] - J[0][2] * J[1][1];
  A[1][0] = J[1][2] * J[2][0] - J[1][0] * J[2][2];
  A[1][1] = J[0][0] * J[2][2] - J[0][2] * J[2][0];
  A[1][2] = J[0][2] * J[1][0] - J[0][0] * J[1][2];
  A[2][0] = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  A[2][1] = J[0][1] * J[2][0] - J[0][0] * J[2][1];
  A[2][2] = J[0][0] * J[1][1] - J[0][1] * J[1][0];
  for (int a = 0; a < 3; ++a) {
    const double b = w * (A[a][0] * u[0] + A[a][1] * u[1] + A[a][2] * u[2]);
    velb[cell * velb_stride(n) + a * n3 + q] = b;
    if (velb32) velb32[cell * velb_stride(n) + a * n3 + q] = (float)b;
  }
}

// per (cell, qp) of a colour-major cell: the nodal velocity field U
// (component-major [3][N], the vector the reference operators read with
// read_dof_values_plain, heat_diffuse_operator.cpp:975-980,
// advection_diffusion_operator.cpp:461-465) interpolated to the Gauss point
// with the Gauss-Lobatto basis, u_q = sum_{a,b,c} S(q_x,a) S(q_y,b) S(q_z,c)
// U(dof(a,b,c)); then the apply's stream value w adj(J) u_q = JxW J^-1 u_q (as
// velb_kernel) and, for tau_K, |u_q|.  Lattice cells find their DoFs from their
// position, mapped cells through the cell->DoF map.
__global__ void nodal_velb_kernel(const double *vert, int nc0, int nc1, long NX, long NY, long N, long n_cells,
                                  int P, const Colour *colours, const double *cellvert, const int *cmap,
                                  const double *U, double *velb, float *velb32, double *umag)
{
  const int n = P + 1, n3 = n * n * n;
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= n_cells * n3) return;
  const long cell = gid / n3;
  const int q = (int)(gid % n3);
  const Tables<double> &T = tab<double>(P);
  const int qi = q % n, qj = (q / n) % n, qk = q / (n * n);
  long base = 0;
  if (!cmap) {
    int c = 0;
    while (c < 7 && cell >= colours[c + 1].first) ++c;
    const Colour &C = colours[c];
    const long cidx = cell - C.first;
    const long ix = 2 * (cidx % C.cn[0]) + C.par[0];
    const long iy = 2 * ((cidx / C.cn[0]) % C.cn[1]) + C.par[1];
    const long iz = 2 * (cidx / ((long)C.cn[0] * C.cn[1])) + C.par[2];
    base = (iz * P * NY + iy * P) * NX + ix * P;
  }
  double u[3] = {0, 0, 0};
  for (int c = 0; c < n; ++c) {
    const double sc = T.S[qk * n + c];
    for (int b = 0; b < n; ++b) {
      const double sbc = sc * T.S[qj * n + b];
      for (int a = 0; a < n; ++a) {
        const double wgt = sbc * T.S[qi * n + a];
        const long g = cmap ? (long)cmap[cell * n3 + (c * n + b) * n + a] : base + ((long)c * NY + b) * NX + a;
        u[0] += wgt * U[g];
        u[1] += wgt * U[N + g];
        u[2] += wgt * U[2 * N + g];
      }
    }
  }
  double V[8][3];
  cell_corners(vert, nc0, nc1, colours, cellvert, cell, V);
  const double xi[3] = {T.x[qi], T.x[qj], T.x[qk]};
  const double w = T.w[qi] * T.w[qj] * T.w[qk];
  double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int v = 0; v < 8; ++v) {
    const int bx = v & 1, by = (v >> 1) & 1, bz = (v >> 2) & 1;
    const double f[3] = {bx ? xi[0] : 1 - xi[0], by ? xi[1] : 1 - xi[1], bz ? xi[2] : 1 - xi[2]};
    const double df[3] = {bx ? 1.0 : -1.0, by ? 1.0 : -1.0, bz ? 1.0 : -1.0};
    const double dB[3] = {df[0] * f[1] * f[2], f[0] * df[1] * f[2], f[0] * f[1] * df[2]};
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) J[a][b] += V[v][a] * dB[b];
  }
  double A[3][3];
  A[0][0] = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  A[0][1] = J[0][2] * J[2][1] - J[0][1] * J[2][2];
  A[0][2] = J[0][1] * J[1][2] - J[0][2] * J[1][1];
  A[1][0] = J[1][2] * J[2][0] - J[1][0] * J[2][2];
  A[1][1] = J[0][0] * J[2][2] - J[0][2] * J[2][0];
  A[1][2] = J[0][2] * J[1][0] - J[0][0] * J[1][2];
  A[2][0] = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  A[2][1] = J[0][1] * J[2][0] - J[0][0] * J[2][1];
  A[2][2] = J[0][0] * J[1][1] - J[0][1] * J[1][0];
  for (int a = 0; a < 3; ++a) {
    const double b = w * (A[a][0] * u[0] + A[a][1] * u[1] + A[a][2] * u[2]);
    velb[cell * velb_stride(n) + a * n3 + q] = b;
    if (velb32) velb32[cell * velb_stride(n) + a * n3 + q] = (float)b;
  }
  if (umag) umag[gid] = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
}

// per colour-major cell: the SUPG parameter tau_K (compute_stabilization_parameter,
// advection_diffusion_operator.cpp:499-533): coefficient h_K, or, for a negative
// coefficient, h_K / max_q |u(x_q)| (0 when that maximum is below 1e-6), with the
// cell size h_K = diameter / sqrt(3) (scratch_data.cpp:249-266); the diameter of
// a hexahedron is its longest main diagonal
__global__ void tau_kernel(const double *vert, int nc0, int nc1, long n_cells, int P, const Colour *colours,
                           const double *cellvert, int vel_kind, double s0, double s1, double s2, double coef,
                           const double *xq_all, double *tau64, float *tau32, const double *umag)
{
  const int n = P + 1;
  const long cell = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= n_cells) return;
  double V[8][3];
  cell_corners(vert, nc0, nc1, colours, cellvert, cell, V);
  double diam = 0.0;
  for (int d = 0; d < 4; ++d) {
    double s = 0.0;
    for (int a = 0; a < 3; ++a) s += (V[d][a] - V[7 - d][a]) * (V[d][a] - V[7 - d][a]);
    diam = fmax(diam, sqrt(s));
  }
  const double h = diam / sqrt(3.0);
  double tau;
  if (coef >= 0.0) {
    tau = coef * h;
  } else {
    double umax = 0.0;
    for (int q = 0; q < n * n * n; ++q) {
      if (umag) {  // velocity given as a DoF vector: |u| at the Gauss points
        umax = fmax(umax, umag[cell * n * n * n + q]);
        continue;
      }
      const double xi[3] = {xq_all[q % n], xq_all[(q / n) % n], xq_all[q / (n * n)]};
      double x[3] = {0, 0, 0};
      for (int v = 0; v < 8; ++v) {
        const double B = ((v & 1) ? xi[0] : 1 - xi[0]) * (((v >> 1) & 1) ? xi[1] : 1 - xi[1]) *
                         (((v >> 2) & 1) ? xi[2] : 1 - xi[2]);
        for (int a = 0; a < 3; ++a) x[a] += V[v][a] * B;
      }
      double u[3] = {0, 0, 0};
      if (vel_kind == MPDG_VEL_VORTEX) {
        u[0] = sin(M_PI * x[0]) * cos(M_PI * x[1]);
        u[1] = -cos(M_PI * x[0]) * sin(M_PI * x[1]);
      } else if (vel_kind == MPDG_VEL_ROTATION) {
        u[0] = s0 * x[2];
        u[2] = -s0 * x[0];
      } else if (vel_kind == MPDG_VEL_CONST) {
        u[0] = s0;
        u[1] = s1;
        u[2] = s2;
      }
      umax = fmax(umax, sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]));
    }
    tau = (umax >= 1e-6) ? h / umax : 0.0;
  }
  tau64[cell] = tau;
  if (tau32) tau32[cell] = (float)tau;
}

// probing of the diagonal: x = 1 at the DoFs of one residue class (X, Y, Z) mod
// n = (a, b, c), else 0.  Two such DoFs are n apart in some direction and share
// no cell, so A x holds each probed DoF's exact diagonal entry there.
__global__ void lattice_probe_kernel(double *x, long N, long NX, long NY, int n, int a, int b, int c)
{
  for (long g = (long)blockIdx.x * blockDim.x + threadIdx.x; g < N; g += (long)gridDim.x * blockDim.x) {
    const long X = g % NX, Y = (g / NX) % NY, Z = g / (NX * NY);
    x[g] = (X % n == a && Y % n == b && Z % n == c) ? 1.0 : 0.0;
  }
}

__global__ void lattice_take_kernel(double *diag, const double *y, long N, long NX, long NY, int n, int a, int b,
                                    int c)
{
  for (long g = (long)blockIdx.x * blockDim.x + threadIdx.x; g < N; g += (long)gridDim.x * blockDim.x) {
    const long X = g % NX, Y = (g / NX) % NY, Z = g / (NX * NY);
    if (X % n == a && Y % n == b && Z % n == c) diag[g] = y[g];
  }
}

__global__ void cast_kernel(const double *a, float *b, long n)
{
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}

// inverse diagonal with the reference's thresholds; constrained entries -> 1
__global__ void invert_kernel(double *d, long n, const uint8_t *mask, double thr)
{
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (mask && mask[i]) {
    d[i] = 1.0;
    return;
  }
  const double v = d[i];
  d[i] = (fabs(v) > thr) ? 1.0 / v : 1.0;
}

__global__ void set_masked_kernel(double *d, long n, const uint8_t *mask, double value)
{
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && mask[i]) d[i] = value;
}

// ------------------------------------------------------------- host side

namespace {

void colour_layout(Mesh &m)
{
  long first = 0;
  for (int c = 0; c < 8; ++c) {
    Colour &C = m.colour[c];
    C.par[0] = c & 1;
    C.par[1] = (c >> 1) & 1;
    C.par[2] = (c >> 2) & 1;
    for (int d = 0; d < 3; ++d) C.cn[d] = (m.nc[d] - C.par[d] + 1) / 2;
    C.count = (long)C.cn[0] * C.cn[1] * C.cn[2];
    C.first = first;
    first += C.count;
  }
}

template <typename T>
T *dev_alloc(size_t count, size_t &bytes)
{
  T *p = nullptr;
  if (count == 0) return nullptr;
  cudaError_t e = tracked_malloc(&p, count * sizeof(T));
  if (e != cudaSuccess) throw Error{MPDG_ERR_ALLOC, std::string("cudaMalloc: ") + cudaGetErrorString(e)};
  bytes += count * sizeof(T);
  return p;
}

unsigned grid_for(long n, int block) { return (unsigned)((n + block - 1) / block); }

}  // namespace

void build_mesh_device_data(Mesh &m, const uint8_t *host_mask, bool force_general)
{
  upload_tables();
  colour_layout(m);
  const int p = m.degree, n = p + 1, n3 = n * n * n;
  // uniform axis-aligned box detection
  const int nv0 = m.nc[0] + 1, nv1 = m.nc[1] + 1, nv2 = m.nc[2] + 1;
  const double *V = m.vertices.data();
  for (int d = 0; d < 3; ++d) {
    m.origin[d] = V[d];
    const long last = (d == 0) ? (nv0 - 1) : (d == 1) ? (long)(nv1 - 1) * nv0 : (long)(nv2 - 1) * nv0 * nv1;
    m.h[d] = (V[last * 3 + d] - V[d]) / m.nc[d];
  }
  bool uniform = !force_general;
  double scale = 0.0;
  for (int d = 0; d < 3; ++d) scale = std::fmax(scale, std::fabs(m.h[d]) * m.nc[d]);
  for (long v = 0; uniform && v < (long)nv0 * nv1 * nv2; ++v) {
    const long c[3] = {v % nv0, (v / nv0) % nv1, v / ((long)nv0 * nv1)};
    for (int d = 0; d < 3; ++d)
      if (std::fabs(V[v * 3 + d] - (m.origin[d] + c[d] * m.h[d])) > 1e-14 * scale) {
        uniform = false;
        break;
      }
  }
  m.uniform = uniform;

  m.d_vert = dev_alloc<double>(m.vertices.size(), m.device_bytes);
  MPDG_CUDA(cudaMemcpy(m.d_vert, V, m.vertices.size() * sizeof(double), cudaMemcpyHostToDevice));

  if (!uniform) {
    Colour *d_col = nullptr;
    MPDG_CUDA(tracked_malloc(&d_col, sizeof(m.colour)));
    MPDG_CUDA(cudaMemcpy(d_col, m.colour, sizeof(m.colour), cudaMemcpyHostToDevice));
    double *d_xw = nullptr;
    double xw[2 * kMaxN];
    {
      double xq[kMaxN], wq[kMaxN];
      gauss(n, xq, wq);
      for (int q = 0; q < n; ++q) {
        xw[q] = xq[q];
        xw[kMaxN + q] = wq[q];
      }
    }
    MPDG_CUDA(tracked_malloc(&d_xw, sizeof(xw)));
    MPDG_CUDA(cudaMemcpy(d_xw, xw, sizeof(xw), cudaMemcpyHostToDevice));
    m.d_metric64 = dev_alloc<double>((size_t)m.n_cells * metric_stride(n), m.device_bytes);
    MPDG_CUDA(cudaMemset(m.d_metric64, 0, sizeof(double) * m.n_cells * metric_stride(n)));
    const long total = m.n_cells * n3;
    metric_kernel<<<grid_for(total, 256), 256>>>(m.d_vert, m.nc[0], m.nc[1], m.n_cells, p, d_col, nullptr,
                                                 m.d_metric64, nullptr, d_xw, d_xw + kMaxN);
    MPDG_LAUNCHED();
    MPDG_CUDA(cudaDeviceSynchronize());
    cudaFree(d_col);
    cudaFree(d_xw);
  }

  // Dirichlet mask and per-cell flags
  if (host_mask) {
    std::vector<uint8_t> flags(m.n_cells, 0);
    std::vector<uint32_t> cmask(4 * (size_t)m.n_cells, 0u);
    bool any = false;
    for (int c = 0; c < 8; ++c) {
      const Colour &C = m.colour[c];
      for (long k = 0; k < C.count; ++k) {
        const int ix = 2 * (int)(k % C.cn[0]) + C.par[0];
        const int iy = 2 * (int)((k / C.cn[0]) % C.cn[1]) + C.par[1];
        const int iz = 2 * (int)(k / ((long)C.cn[0] * C.cn[1])) + C.par[2];
        uint8_t f = 0;
        for (int kk = 0; kk <= p; ++kk)
          for (int jj = 0; jj <= p; ++jj)
            for (int ii = 0; ii <= p; ++ii) {
              const long g = ((long)(iz * p + kk) * m.NY + (iy * p + jj)) * m.NX + (ix * p + ii);
              if (host_mask[g]) {
                f = 1;
                const int bit = (kk * n + jj) * n + ii;
                cmask[4 * (C.first + k) + bit / 32] |= 1u << (bit % 32);
              }
            }
        flags[C.first + k] = f;
        any = any || f;
      }
    }
    m.has_dirichlet = any;
    if (any) {
      m.d_dmask = dev_alloc<uint8_t>(m.N, m.device_bytes);
      MPDG_CUDA(cudaMemcpy(m.d_dmask, host_mask, m.N, cudaMemcpyHostToDevice));
      m.d_cell_flags = dev_alloc<uint8_t>(m.n_cells, m.device_bytes);
      MPDG_CUDA(cudaMemcpy(m.d_cell_flags, flags.data(), m.n_cells, cudaMemcpyHostToDevice));
      m.d_cell_mask = dev_alloc<uint32_t>(4 * (size_t)m.n_cells, m.device_bytes);
      MPDG_CUDA(cudaMemcpy(m.d_cell_mask, cmask.data(), sizeof(uint32_t) * cmask.size(),
                           cudaMemcpyHostToDevice));
    }
  }
}

void ensure_metric32(Mesh &m, cudaStream_t s)
{
  if (m.uniform || m.metric32_ready) return;
  const int n = m.degree + 1;
  const long total = m.n_cells * metric_stride(n);
  m.d_metric32 = dev_alloc<float>(total, m.device_bytes);
  cast_kernel<<<grid_for(total, 256), 256, 0, s>>>(m.d_metric64, m.d_metric32, total);
  MPDG_LAUNCHED();
  m.metric32_ready = true;
}

void build_op_device_data(Op &op)
{
  Mesh &m = *op.mesh;
  const int p = m.degree, n = p + 1, n3 = n * n * n;
  const bool want32 = (op.d.precision_mask & (1 << MPDG_FP32)) != 0;
  op.d_err = dev_alloc<int>(1, op.device_bytes);
  MPDG_CUDA(cudaMemset(op.d_err, 0, sizeof(int)));
  if (op.d.kind == MPDG_OP_ADVDIFF && op.d.supg) {
    Colour *d_col = nullptr;
    double *d_xq = nullptr;
    double xq[kMaxN], wq[kMaxN];
    gauss(n, xq, wq);
    MPDG_CUDA(tracked_malloc(&d_col, sizeof(m.colour)));
    MPDG_CUDA(cudaMemcpy(d_col, m.colour, sizeof(m.colour), cudaMemcpyHostToDevice));
    MPDG_CUDA(tracked_malloc(&d_xq, sizeof(xq)));
    MPDG_CUDA(cudaMemcpy(d_xq, xq, sizeof(xq), cudaMemcpyHostToDevice));
    op.d_tau64 = dev_alloc<double>((size_t)m.n_cells, op.device_bytes);
    if (want32) op.d_tau32 = dev_alloc<float>((size_t)m.n_cells, op.device_bytes);
    if (op.d.vel_kind == MPDG_VEL_NODAL && op.d.supg_coefficient < 0.0) {
      // tau_K = h_K / max |u| follows the velocity field (build_nodal_velocity)
      MPDG_CUDA(cudaMemset(op.d_tau64, 0, sizeof(double) * m.n_cells));
      if (op.d_tau32) MPDG_CUDA(cudaMemset(op.d_tau32, 0, sizeof(float) * m.n_cells));
    } else {
      tau_kernel<<<grid_for(m.n_cells, 128), 128>>>(m.d_vert, m.nc[0], m.nc[1], m.n_cells, p, d_col,
                                                    m.d_cellvert, op.d.vel_kind, op.d.vel_param[0], op.d.vel_param[1],
                                                    op.d.vel_param[2], op.d.supg_coefficient, d_xq, op.d_tau64,
                                                    op.d_tau32, nullptr);
      MPDG_LAUNCHED();
    }
    if (op.d.diffusivity != 0.0 && !m.uniform) {
      // the Laplacian of the SUPG residual on general cells needs the
      // curvature of the map at every quadrature point
      const size_t cnt = (size_t)m.n_cells * 3 * n3;
      op.d_lam64 = dev_alloc<double>(cnt, op.device_bytes);
      if (want32) op.d_lam32 = dev_alloc<float>(cnt, op.device_bytes);
      lam_kernel<<<grid_for(m.n_cells * n3, 256), 256>>>(m.d_vert, m.nc[0], m.nc[1], m.n_cells, p, d_col,
                                                         m.d_cellvert, d_xq, op.d_lam64, op.d_lam32);
      MPDG_LAUNCHED();
    }
    MPDG_CUDA(cudaDeviceSynchronize());
    cudaFree(d_col);
    cudaFree(d_xq);
  }
  if (op.d.vel_kind == MPDG_VEL_NONE || op.d.vel_kind == MPDG_VEL_NODAL) return;  // nodal: at set_field
  if (!m.uniform) {
    Colour *d_col = nullptr;
    MPDG_CUDA(tracked_malloc(&d_col, sizeof(m.colour)));
    MPDG_CUDA(cudaMemcpy(d_col, m.colour, sizeof(m.colour), cudaMemcpyHostToDevice));
    double xw[2 * kMaxN], xq[kMaxN], wq[kMaxN];
    gauss(n, xq, wq);
    for (int q = 0; q < n; ++q) {
      xw[q] = xq[q];
      xw[kMaxN + q] = wq[q];
    }
    double *d_xw = nullptr;
    MPDG_CUDA(tracked_malloc(&d_xw, sizeof(xw)));
    MPDG_CUDA(cudaMemcpy(d_xw, xw, sizeof(xw), cudaMemcpyHostToDevice));
    const long total = m.n_cells * n3;
    op.d_velb64 = dev_alloc<double>((size_t)m.n_cells * velb_stride(n), op.device_bytes);
    MPDG_CUDA(cudaMemset(op.d_velb64, 0, sizeof(double) * m.n_cells * velb_stride(n)));
    if (want32) {
      op.d_velb32 = dev_alloc<float>((size_t)m.n_cells * velb_stride(n), op.device_bytes);
      MPDG_CUDA(cudaMemset(op.d_velb32, 0, sizeof(float) * m.n_cells * velb_stride(n)));
    }
    velb_kernel<<<grid_for(total, 256), 256>>>(m.d_vert, m.nc[0], m.nc[1], m.n_cells, p, d_col, m.d_cellvert,
                                               op.d.vel_kind, op.d.vel_param[0], op.d.vel_param[1],
                                               op.d.vel_param[2], op.d_velb64, op.d_velb32, d_xw,
                                               d_xw + kMaxN);
    MPDG_LAUNCHED();
    MPDG_CUDA(cudaDeviceSynchronize());
    cudaFree(d_col);
    cudaFree(d_xw);
  } else if (op.d.vel_kind == MPDG_VEL_VORTEX) {
    // separable velocity: sin/cos of pi x at every Gauss point position per axis
    double xq[kMaxN], wq[kMaxN];
    gauss(n, xq, wq);
    const int stride = std::max(m.nc[0], m.nc[1]) * n;
    std::vector<double> t(4 * (size_t)stride, 0.0);
    for (int c = 0; c < m.nc[0]; ++c)
      for (int q = 0; q < n; ++q) {
        const double x = m.origin[0] + (c + xq[q]) * m.h[0];
        t[c * n + q] = std::sin(M_PI * x);
        t[stride + c * n + q] = std::cos(M_PI * x);
      }
    for (int c = 0; c < m.nc[1]; ++c)
      for (int q = 0; q < n; ++q) {
        const double y = m.origin[1] + (c + xq[q]) * m.h[1];
        t[2 * stride + c * n + q] = std::sin(M_PI * y);
        t[3 * stride + c * n + q] = std::cos(M_PI * y);
      }
    op.d_trig64 = dev_alloc<double>(t.size(), op.device_bytes);
    MPDG_CUDA(cudaMemcpy(op.d_trig64, t.data(), t.size() * sizeof(double), cudaMemcpyHostToDevice));
    std::vector<float> t32(t.begin(), t.end());
    op.d_trig32 = dev_alloc<float>(t.size(), op.device_bytes);
    MPDG_CUDA(cudaMemcpy(op.d_trig32, t32.data(), t32.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
}

void build_nodal_velocity(Op &op)
{
  Mesh &m = *op.mesh;
  if (op.d.vel_kind != MPDG_VEL_NODAL)
    throw Error{MPDG_ERR_ARG, "MPDG_FIELD_VELOCITY needs an operator created with vel_kind MPDG_VEL_NODAL"};
  if (!op.U64) return;
  const int p = m.degree, n = p + 1, n3 = n * n * n;
  const bool want32 = (op.d.precision_mask & (1 << MPDG_FP32)) != 0;
  const size_t count = (size_t)m.n_cells * velb_stride(n);
  if (!op.d_velb64) {
    op.d_velb64 = dev_alloc<double>(count, op.device_bytes);
    MPDG_CUDA(cudaMemsetAsync(op.d_velb64, 0, sizeof(double) * count, op.stream));
  }
  if (want32 && !op.d_velb32) {
    op.d_velb32 = dev_alloc<float>(count, op.device_bytes);
    MPDG_CUDA(cudaMemsetAsync(op.d_velb32, 0, sizeof(float) * count, op.stream));
  }
  const bool with_tau = op.d.kind == MPDG_OP_ADVDIFF && op.d.supg && op.d.supg_coefficient < 0.0;
  Colour *d_col = nullptr;
  double *umag = nullptr, *d_xq = nullptr;
  auto cleanup = [&]() {
    cudaStreamSynchronize(op.stream);
    if (d_col) cudaFree(d_col);
    if (umag) cudaFree(umag);
    if (d_xq) cudaFree(d_xq);
  };
  try {
    MPDG_CUDA(tracked_malloc(&d_col, sizeof(m.colour)));
    MPDG_CUDA(cudaMemcpyAsync(d_col, m.colour, sizeof(m.colour), cudaMemcpyHostToDevice, op.stream));
    if (with_tau) MPDG_CUDA(tracked_malloc(&umag, sizeof(double) * (size_t)m.n_cells * n3));
    const long total = m.n_cells * n3;
    nodal_velb_kernel<<<grid_for(total, 256), 256, 0, op.stream>>>(
        m.d_vert, m.nc[0], m.nc[1], m.NX, m.NY, m.N, m.n_cells, p, d_col, m.d_cellvert, m.d_cmap, op.U64,
        op.d_velb64, want32 ? op.d_velb32 : nullptr, umag);
    MPDG_LAUNCHED();
    if (with_tau) {
      double xq[kMaxN], wq[kMaxN];
      gauss(n, xq, wq);
      MPDG_CUDA(tracked_malloc(&d_xq, sizeof(xq)));
      MPDG_CUDA(cudaMemcpyAsync(d_xq, xq, sizeof(xq), cudaMemcpyHostToDevice, op.stream));
      tau_kernel<<<grid_for(m.n_cells, 128), 128, 0, op.stream>>>(m.d_vert, m.nc[0], m.nc[1], m.n_cells, p, d_col,
                                                                 m.d_cellvert, op.d.vel_kind, 0.0, 0.0, 0.0,
                                                                 op.d.supg_coefficient, d_xq, op.d_tau64,
                                                                 op.d_tau32, umag);
      MPDG_LAUNCHED();
    }
  } catch (...) {
    cleanup();
    throw;
  }
  cleanup();
}

__global__ void diff_cast_kernel(const double *a, const double *b, float *c, long n)
{
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) c[i] = (float)(a[i] - b[i]);
}

__global__ void shift_cast_kernel(const double *a, double shift, float *c, long n)
{
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) c[i] = (float)(a[i] - shift);
}

// FP32 copies of the fields the FP32 form reads: T, the heaviside, and the
// increment T - T_old (formed in FP64: the float copies of T and T_old would
// lose its digits to cancellation)
void ensure_T32(Op &op)
{
  const long N = op.mesh->N;
  const double *src[2] = {op.T64, op.H64};
  float **dst[2] = {&op.T32, &op.H32};
  for (int f = 0; f < 2; ++f) {
    if (!src[f]) continue;
    if (!*dst[f]) *dst[f] = dev_alloc<float>(N, op.device_bytes);
    cast_kernel<<<grid_for(N, 256), 256, 0, op.stream>>>(src[f], *dst[f], N);
    MPDG_LAUNCHED();
  }
  if (op.T64 && op.Told64) {
    if (!op.Told32) op.Told32 = dev_alloc<float>(N, op.device_bytes);
    diff_cast_kernel<<<grid_for(N, 256), 256, 0, op.stream>>>(op.T64, op.Told64, op.Told32, N);
    MPDG_LAUNCHED();
  }
  // laws with a solid phase read T - solidus: within the mushy zone the
  // solid fraction and the apparent capacity vary on the scale of
  // liquidus - solidus, far finer than a float's resolution of T itself
  if (op.T64 && op.d.kind == MPDG_OP_HEAT && law_has_solid(op.d.material)) {
    if (!op.Ts32) op.Ts32 = dev_alloc<float>(N, op.device_bytes);
    shift_cast_kernel<<<grid_for(N, 256), 256, 0, op.stream>>>(op.T64, op.d.solidus, op.Ts32, N);
    MPDG_LAUNCHED();
  }
}

namespace {

template <typename Real>
KP<Real> base_params(Op &op)
{
  Mesh &m = *op.mesh;
  KP<Real> k{};
  k.NX = m.NX;
  k.NY = m.NY;
  k.hsrc = (const Real *)op.hang_src;
  k.hstage = (Real *)op.d_stage;
  k.hmask = op.hang_mask;
  k.hNXc = op.hang_NXc;
  k.hNYc = op.hang_NYc;
  k.hnc1 = m.nc[1];
  for (int d = 0; d < 3; ++d) k.nc[d] = m.nc[d];
  for (int d = 0; d < 3; ++d) {
    k.h[d] = (Real)m.h[d];
    k.origin[d] = (Real)m.origin[d];
    k.vel_param[d] = (Real)op.d.vel_param[d];
  }
  k.vel_kind = op.d.vel_kind;
  if (op.d.vel_kind == MPDG_VEL_NODAL && !op.d_velb64)
    throw Error{MPDG_ERR_ARG, "the operator needs the velocity field (MPDG_FIELD_VELOCITY)"};
  if (op.d.vel_kind == MPDG_VEL_NODAL && sizeof(Real) == 4 && !op.d_velb32)
    throw Error{MPDG_ERR_ARG, "the FP32 form was not prepared for this operator (precision_mask)"};
  for (int d = 0; d < 3; ++d) {
    k.ih[d] = (Real)(1.0 / m.h[d]);
    k.ih2[d] = (Real)(1.0 / (m.h[d] * m.h[d]));
  }
  k.hvol = (Real)(m.h[0] * m.h[1] * m.h[2]);
  if constexpr (sizeof(Real) == 8) {
    k.metric = m.d_metric64;
    k.velb = op.d_velb64;
    k.trig = op.d_trig64;
    k.T = op.T64;
    k.tau = op.d_tau64;
    k.lam = op.d_lam64;
  } else {
    k.metric = m.d_metric32;
    k.velb = op.d_velb32;
    k.trig = op.d_trig32;
    k.T = op.T32;
    k.tau = op.d_tau32;
    k.lam = op.d_lam32;
  }
  k.supg_lap = op.d.kind == MPDG_OP_ADVDIFF && op.d.supg && op.d.diffusivity != 0.0;
  k.cmap = m.d_cmap;
  k.nvec = 1;
  k.trig_stride = std::max(m.nc[0], m.nc[1]) * m.n;
  k.dmask = m.d_dmask;
  k.cell_flags = m.d_cell_flags;
  k.cell_mask = reinterpret_cast<const uint4 *>(m.d_cell_mask);
  k.cell_first = reinterpret_cast<const uint4 *>(m.d_cell_first);
  const bool heat = op.d.kind == MPDG_OP_HEAT;
  k.c_mass = (Real)(heat ? op.d.rho_cp / op.d.dt : 1.0 / op.d.dt);
  k.c_vel = (Real)(heat ? op.d.rho_cp : op.d.theta);
  k.c_diff = (Real)(heat ? op.d.k0 : op.d.theta * op.d.diffusivity);
  k.k_alpha = (Real)(heat ? op.d.k_alpha : 0.0);
  k.full_tangent = heat && op.d.full_tangent;
  // heat material law
  const bool law = heat && op.d.material != MPDG_MAT_LINEAR;
  const bool law_T = law && law_has_solid(op.d.material), law_H = law && law_two_phase(op.d.material);
  k.mat = law ? op.d.material : MPDG_MAT_LINEAR;
  k.two_phase_sharp = op.d.two_phase_sharp;
  k.solid_sharp = op.d.solid_liquid_sharp;
  k.vol_specific = op.d.volume_specific;
  for (int e = 0; e < 3; ++e) {
    k.mrho[e] = (Real)op.d.mat_rho[e];
    k.mcp[e] = (Real)op.d.mat_cp[e];
    k.mk[e] = (Real)op.d.mat_k[e];
  }
  k.solidus = (Real)op.d.solidus;
  k.liquidus = (Real)op.d.liquidus;
  k.inv_mushy = law_T ? (Real)(1.0 / (op.d.liquidus - op.d.solidus)) : Real(0);
  k.latent = law_T ? (Real)op.d.latent_heat : Real(0);
  k.ac_type = op.d.apparent_capacity;
  k.dt_inv = (Real)(1.0 / op.d.dt);
  if (law_T) k.full_tangent = 1;  // heat_diffuse_operator.cpp:1040-1055 (do_solidification)
  if constexpr (sizeof(Real) == 8) {
    k.Told = law_T ? op.Told64 : nullptr;
    k.Hs = law_H ? op.H64 : nullptr;
  } else {
    k.Told = law_T ? op.Told32 : nullptr;  // T - T_old
    k.told_inc = 1;
    k.Hs = law_H ? op.H32 : nullptr;
    if (law_T) {
      // T - solidus against the shifted zone [0, liquidus - solidus] (ensure_T32)
      if (!op.Ts32) throw Error{MPDG_ERR_ARG, "the FP32 form was not prepared for this operator (precision_mask)"};
      k.T = op.Ts32;
      k.solidus = Real(0);
      k.liquidus = (Real)(op.d.liquidus - op.d.solidus);
    }
  }
  const bool mask = op.use_dirichlet && m.has_dirichlet;
  k.masked_read = mask;
  k.masked_write = mask;
  return k;
}

// the colours of a mesh: the 8 parity colours of a lattice, or a mapped
// mesh's greedy colours
inline int n_colours(const Mesh &m) { return m.mapped ? (int)m.mcol.size() : 8; }
inline const Colour *colours(const Mesh &m) { return m.mapped ? m.mcol.data() : m.colour; }

template <typename Real>
void colour_params(KP<Real> &k, const Colour &C)
{
  for (int d = 0; d < 3; ++d) {
    k.par[d] = C.par[d];
    k.cn[d] = C.cn[d];
  }
  k.ccount = C.count;
  k.cfirst = C.first;
  const unsigned long long two40 = 1ull << 40;
  const unsigned long long d0 = (unsigned long long)std::max(1, C.cn[0]);
  const unsigned long long d01 = d0 * (unsigned long long)std::max(1, C.cn[1]);
  k.div0_magic = (two40 + d0 - 1) / d0;
  k.div01_magic = (two40 + d01 - 1) / d01;
  // exactness of the magic division: x * d < 2^40 for every cell index x
  if ((unsigned long long)C.count * d01 >= two40)
    throw Error{MPDG_ERR_SIZE, "mesh too large for the colour index arithmetic"};
}

template <int P, typename Real, int MODE, bool KT>
void run_cells(Op &op, KP<Real> k)
{
  Mesh &m = *op.mesh;
  constexpr int n = P + 1, CPB = Cfg<n>::cpb;
  const dim3 block(n * n, CPB);
  for (int c = 0; c < n_colours(m); ++c) {
    const Colour &C = colours(m)[c];
    if (C.count == 0) continue;
    colour_params(k, C);
    const unsigned grid = (unsigned)((C.count + CPB - 1) / CPB);
    if (m.uniform)
      cell_kernel<P, Real, GEOM_UNIFORM, MODE, KT><<<grid, block, 0, op.stream>>>(k);
    else
      cell_kernel<P, Real, GEOM_GENERAL, MODE, KT><<<grid, block, 0, op.stream>>>(k);
    MPDG_LAUNCHED();
  }
}

template <typename Real, int MODE, bool KT>
void dispatch_degree(Op &op, const KP<Real> &k)
{
  switch (op.mesh->degree) {
    case 1: run_cells<1, Real, MODE, KT>(op, k); break;
    case 2: run_cells<2, Real, MODE, KT>(op, k); break;
    case 3: run_cells<3, Real, MODE, KT>(op, k); break;
    case 4: run_cells<4, Real, MODE, KT>(op, k); break;
    default: throw Error{MPDG_ERR_UNSUPPORTED, "degree must be 1..4"};
  }
}

bool supg(const Op &op) { return op.d.kind == MPDG_OP_ADVDIFF && op.d.supg; }

bool uses_kT(const Op &op)
{
  return op.d.kind == MPDG_OP_HEAT && (op.d.k_alpha != 0.0 || op.d.full_tangent || op.d.material != MPDG_MAT_LINEAR);
}

bool uses_law(const Op &op) { return op.d.kind == MPDG_OP_HEAT && op.d.material != MPDG_MAT_LINEAR; }

// the fields a material law reads must be set before it is applied
template <typename Real>
void check_law_fields(const Op &op, const KP<Real> &k)
{
  if (!uses_law(op)) return;
  if (law_has_solid(op.d.material) && !k.Told)
    throw Error{MPDG_ERR_ARG, "this material law needs the T_old field (MPDG_FIELD_TEMPERATURE_OLD)"};
  if (law_two_phase(op.d.material) && !k.Hs)
    throw Error{MPDG_ERR_ARG, "this material law needs the heaviside field (MPDG_FIELD_HEAVISIDE)"};
}

}  // namespace

namespace {

int g_num_sms = 0;

// slabs of the resident apply in one precision: the operator's setting, or 1
// (one launch per colour over all layers)
int apply_slabs(const Op &op, int precision)
{
  const Mesh &m = *op.mesh;
  if (m.mapped || op.fine) return 1;
  const int S = op.sched[precision].slabs > 0 ? op.sched[precision].slabs : 1;
  return std::max(1, std::min(S, std::min(kMaxApplySlabs, m.nc[2] / 2)));
}

int num_sms()
{
  if (g_num_sms == 0) {
    int dev = 0;
    MPDG_CUDA(cudaGetDevice(&dev));
    MPDG_CUDA(cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev));
  }
  return g_num_sms;
}

template <int P, typename Real, int GEOM, bool HANG, bool MULTI = false, bool MAPPED = false, int GROUP = 32>
void run_warp_apply(Op &op, KP<Real> k)
{
  Mesh &m = *op.mesh;
  constexpr int n = P + 1, CPW = GROUP / (n * n), GPC = kWarpsPerCTA * 32 / GROUP;
  const bool gvel = GEOM == GEOM_GENERAL && op.d.vel_kind != MPDG_VEL_NONE;
  const size_t per_warp = sizeof(Real) * warp_smem_elems<P, Real, GEOM, GROUP>(gvel);
  const size_t smem = per_warp * GPC + kSmemAlign;
  // bulk-copy alignment contract, checked before any launch: 16-byte aligned
  // shared destinations, global sources and sizes
  static_assert((metric_stride(n) * sizeof(Real)) % 16 == 0, "metric stride");
  static_assert((velb_stride(n) * sizeof(Real)) % 16 == 0, "velocity stride");
  if (per_warp % 16 != 0) throw Error{MPDG_ERR_ARG, "per-warp shared memory not 16-byte aligned"};
  if (GEOM == GEOM_GENERAL && ((uintptr_t)k.metric % 16 != 0 || (gvel && (uintptr_t)k.velb % 16 != 0)))
    throw Error{MPDG_ERR_ARG, "coefficient stream not 16-byte aligned"};
  if (GEOM == GEOM_GENERAL && (!k.metric || (gvel && !k.velb)))
    throw Error{MPDG_ERR_ARG, "coefficient stream missing"};
  if (m.N >= (1L << 32)) throw Error{MPDG_ERR_UNSUPPORTED, "the warp apply indexes DoFs with 32 bits"};
  auto kern = warp_apply_kernel<P, Real, GEOM, HANG, MULTI, MAPPED, GROUP>;
  static int configured_smem = -1, blocks_per_sm = 0;  // per instantiation
  if (configured_smem != (int)smem) {
    MPDG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    MPDG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, kern, kWarpsPerCTA * 32, smem));
    if (blocks_per_sm < 1) blocks_per_sm = 1;
    configured_smem = (int)smem;
  }
  const long resident = (long)num_sms() * blocks_per_sm;
  constexpr int prec = sizeof(Real) == 4 ? MPDG_FP32 : MPDG_FP64;
  k.stream_evict_first = op.sched[prec].evict_first;
  const bool use_pdl = op.sched[prec].pdl != 0 && !HANG;
  int launched = 0;
  // the colour launches of cell layers [k.zlo, k.zhi) (all layers when empty)
  auto colour_launches = [&](KP<Real> k) {
    for (int c = 0; c < n_colours(m); ++c) {
      const Colour &C = colours(m)[c];
      if (C.count == 0) continue;
      colour_params(k, C);
      if (k.zhi > k.zlo) {
        // the colour's cells are z-major: layers [zlo, zhi) are a contiguous
        // run of colour-local indices, and the z parity absorbs the offset
        const long plane = (long)C.cn[0] * C.cn[1];
        const long m_lo = (k.zlo - C.par[2] + 1) / 2, m_hi = (k.zhi - C.par[2] + 1) / 2;
        const long c_lo = std::min((long)C.count, m_lo * plane), c_hi = std::min((long)C.count, m_hi * plane);
        if (c_hi <= c_lo) continue;
        k.cfirst = C.first + c_lo;
        k.ccount = c_hi - c_lo;
        k.par[2] = C.par[2] + 2 * (int)m_lo;
      }
      const long groups = (k.ccount + CPW - 1) / CPW;
      const long blocks = std::min(resident, (groups + GPC - 1) / GPC);
      // colours after the first of an apply start as programmatic dependents of
      // the previous colour: src and the coefficients are not written by it,
      // and the kernel reads dst only after griddepcontrol.wait.  The first
      // colour is ordered fully after whatever produced src.
      const bool pdl = use_pdl && launched > 0;
      k.pdl = pdl ? 1 : 0;
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3((unsigned)blocks);
      cfg.blockDim = dim3(kWarpsPerCTA * 32);
      cfg.dynamicSmemBytes = smem;
      cfg.stream = op.stream;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      attr[0].val.programmaticStreamSerializationAllowed = 1;
      cfg.attrs = attr;
      cfg.numAttrs = pdl ? 1 : 0;
      MPDG_CUDA(cudaLaunchKernelEx(&cfg, kern, k, op.d_err));
      MPDG_LAUNCHED();
      ++launched;
    }
  };
  // slab order: the 8 colours of one z-slab of cell layers before the next
  // slab's, so that a slab's DoF vectors stay in L2 across its colours (the
  // first-touch rule holds across slabs: interior slab ends are odd)
  const int S = (k.zhi > k.zlo || HANG || MAPPED) ? 1 : apply_slabs(op, prec);
  if (S <= 1) {
    colour_launches(k);
    return;
  }
  int bounds[kMaxApplySlabs + 1];
  const int ns = slab_bounds(m.nc[2], S, bounds);
  for (int sl = 0; sl < ns; ++sl) {
    KP<Real> ks = k;
    ks.zlo = bounds[sl];
    ks.zhi = bounds[sl + 1];
    colour_launches(ks);
  }
}

// the lane apply serves uniform lattices of degree 1 or 2 with one operand, no
// hanging DoFs and a velocity it evaluates in-kernel
template <typename Real>
bool lane_apply_eligible(const Op &op, const KP<Real> &k)
{
  const Mesh &m = *op.mesh;
  return m.uniform && !m.mapped && (m.degree == 1 || m.degree == 2) && k.hsrc == nullptr &&
         k.vel_kind != MPDG_VEL_NODAL;
}

// the per-quadrature-point coefficient tables of the lane apply (degree P,
// velocity kind VK) for the operator's constants
template <int P, typename Real, int VK>
LaneCoef<Real> lane_coef(const KP<Real> &k)
{
  constexpr int n = P + 1, n2 = n * n, n3 = n2 * n;
  double xq[kMaxN], wq[kMaxN], Dc[kMaxN * kMaxN];
  gauss(n, xq, wq);
  for (int q = 0; q < n; ++q)
    for (int r = 0; r < n; ++r) {
      double v, d;
      lagrange(n, xq, r, xq[q], v, d);
      Dc[q * n + r] = d;
    }
  const double hvol = (double)k.hvol;
  double vf[3] = {1.0, 1.0, 1.0};  // the velocity factor the kernel does not evaluate
  if (VK == LANE_VEL_CONST) for (int d = 0; d < 3; ++d) vf[d] = (double)k.vel_param[d];
  if (VK == LANE_VEL_VORTEX) vf[1] = -1.0;
  if (VK == LANE_VEL_ROTATION) vf[0] = (double)k.vel_param[0], vf[2] = -(double)k.vel_param[0];
  LaneCoef<Real> c{};
  for (int q = 0; q < n3; ++q) {
    const double W = wq[q % n] * wq[(q / n) % n] * wq[q / n2];
    c.mass[q] = (Real)((double)k.c_mass * hvol * W);
    for (int d = 0; d < 3; ++d) {
      c.diff[d][q] = (Real)((double)k.c_diff * hvol * (double)k.ih2[d] * W);
      c.adv[d][q] = (Real)((double)k.c_vel * hvol * (double)k.ih[d] * W * vf[d]);
    }
  }
  for (int d = 0; d < 3; ++d)
    for (int b = 0; b < n; ++b)
      for (int a = 0; a < n; ++a) c.line[d][b * n + a] = (Real)((double)k.c_diff * hvol * (double)k.ih2[d] * wq[a] * wq[b]);
  for (int r = 0; r < n; ++r)
    for (int s = 0; s < n; ++s) {
      double acc = 0.0;
      for (int t = 0; t < n; ++t) acc += Dc[t * n + r] * wq[t] * Dc[t * n + s];
      c.K[r * n + s] = (Real)acc;
    }
  return c;
}

template <int P, typename Real, int VK, int OCC>
void run_lane_apply(Op &op, KP<Real> k)
{
  const LaneCoef<Real> coef = lane_coef<P, Real, VK>(k);
  Mesh &m = *op.mesh;
  if (m.N >= (1L << 32)) throw Error{MPDG_ERR_UNSUPPORTED, "the lane apply indexes DoFs with 32 bits"};
  constexpr int prec = sizeof(Real) == 4 ? MPDG_FP32 : MPDG_FP64;
  const bool use_pdl = op.sched[prec].pdl != 0;
  LaneColour lc{};
  for (int c = 0; c < 8; ++c) {
    lc.pfirst[c] = m.colour[c].first;
    lc.pcn0[c] = m.colour[c].cn[0];
    lc.pcn1[c] = m.colour[c].cn[1];
  }
  const int nseg = (m.nc[0] + kLaneSeg - 1) / kLaneSeg;
  int launched = 0;
  // the colour launches of cell layers [zlo, zhi) (all layers when empty), in
  // the order x-segment parity, then y, then z parity
  auto colour_launches = [&](int zlo, int zhi) {
    for (int c = 0; c < 8; ++c) {
      lc.sx = c & 1;
      lc.py = (c >> 1) & 1;
      lc.pz = (c >> 2) & 1;
      lc.nsx = (nseg - lc.sx + 1) / 2;
      lc.cny = (m.nc[1] - lc.py + 1) / 2;
      const int zi0 = (zlo - lc.pz + 1) / 2, zi1 = (zhi - lc.pz + 1) / 2;
      lc.zi0 = zi0;
      lc.nwarps = (long)lc.nsx * lc.cny * std::max(0, zi1 - zi0);
      if (lc.nwarps == 0) continue;
      const bool pdl = use_pdl && launched > 0;
      k.pdl = pdl ? 1 : 0;
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3((unsigned)((lc.nwarps + 3) / 4));
      cfg.blockDim = dim3(128);
      cfg.dynamicSmemBytes = 0;
      cfg.stream = op.stream;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      attr[0].val.programmaticStreamSerializationAllowed = 1;
      cfg.attrs = attr;
      cfg.numAttrs = pdl ? 1 : 0;
      MPDG_CUDA(cudaLaunchKernelEx(&cfg, lane_apply_kernel<P, Real, VK, OCC>, k, lc, coef));
      MPDG_LAUNCHED();
      ++launched;
    }
  };
  if (k.zhi > k.zlo) {
    colour_launches(k.zlo, k.zhi);
    return;
  }
  // z-slabs with odd interior ends keep the first-touch rule across slabs
  int bounds[kMaxApplySlabs + 1];
  const int ns = slab_bounds(m.nc[2], apply_slabs(op, prec), bounds);
  for (int sl = 0; sl < ns; ++sl) colour_launches(bounds[sl], bounds[sl + 1]);
}

template <int P, typename Real, int OCC>
void lane_apply_velocity(Op &op, const KP<Real> &k)
{
  switch (k.vel_kind) {
    case MPDG_VEL_NONE: run_lane_apply<P, Real, LANE_VEL_NONE, OCC>(op, k); break;
    case MPDG_VEL_CONST: run_lane_apply<P, Real, LANE_VEL_CONST, OCC>(op, k); break;
    case MPDG_VEL_VORTEX: run_lane_apply<P, Real, LANE_VEL_VORTEX, OCC>(op, k); break;
    case MPDG_VEL_ROTATION: run_lane_apply<P, Real, LANE_VEL_ROTATION, OCC>(op, k); break;
    default: throw Error{MPDG_ERR_UNSUPPORTED, "velocity kind not evaluated by the lane apply"};
  }
}

template <typename Real, int GEOM>
void warp_apply_degree(Op &op, const KP<Real> &k)
{
  if constexpr (GEOM == GEOM_UNIFORM) {
    const int lane = op.sched[sizeof(Real) == 4 ? MPDG_FP32 : MPDG_FP64].lane;
    if (lane && lane_apply_eligible(op, k)) {
      // a uniform lattice streams no coefficients, so a multi-vector apply
      // loses nothing by applying its vectors in turn (and then returns the
      // bits of the single applies)
      for (int v = 0; v < std::max(1, k.nvec); ++v) {
        KP<Real> kv = k;
        kv.src = k.nvec > 1 ? k.msrc[v] : k.src;
        kv.dst = k.nvec > 1 ? k.mdst[v] : k.dst;
        kv.nvec = 1;
        // Q1 fits either bound without spilling: one variant; lane 2 is the
        // variant with more resident CTAs per SM
        if (op.mesh->degree == 1) lane_apply_velocity<1, Real, 0>(op, kv);
        else if (lane == 2) lane_apply_velocity<2, Real, 1>(op, kv);
        else lane_apply_velocity<2, Real, 0>(op, kv);
      }
      return;
    }
  }
  const bool hang = k.hsrc != nullptr;
  if constexpr (GEOM == GEOM_GENERAL) {
    if (op.mesh->mapped) {
      switch (op.mesh->degree) {
        case 1: run_warp_apply<1, Real, GEOM, false, false, true>(op, k); break;
        case 2: run_warp_apply<2, Real, GEOM, false, false, true>(op, k); break;
        case 3: run_warp_apply<3, Real, GEOM, false, false, true>(op, k); break;
        case 4: run_warp_apply<4, Real, GEOM, false, false, true>(op, k); break;
        default: throw Error{MPDG_ERR_UNSUPPORTED, "degree must be 1..4"};
      }
      return;
    }
  }
  if (k.nvec > 1) {
    switch (op.mesh->degree) {
      case 1: run_warp_apply<1, Real, GEOM, false, true>(op, k); break;
      case 2: run_warp_apply<2, Real, GEOM, false, true>(op, k); break;
      case 3: run_warp_apply<3, Real, GEOM, false, true>(op, k); break;
      case 4: run_warp_apply<4, Real, GEOM, false, true>(op, k); break;
      default: throw Error{MPDG_ERR_UNSUPPORTED, "degree must be 1..4"};
    }
    return;
  }
  // CTA-wide cell groups (fewer idle lanes) where the schedule asks for them;
  // they only differ from warp groups for Q2 and Q4
  const bool cta = op.sched[sizeof(Real) == 4 ? MPDG_FP32 : MPDG_FP64].cta && !hang;
  switch (op.mesh->degree) {
    case 1: hang ? run_warp_apply<1, Real, GEOM, true>(op, k) : run_warp_apply<1, Real, GEOM, false>(op, k); break;
    case 2:
      if (cta) run_warp_apply<2, Real, GEOM, false, false, false, 128>(op, k);
      else if (hang) run_warp_apply<2, Real, GEOM, true>(op, k);
      else run_warp_apply<2, Real, GEOM, false>(op, k);
      break;
    case 3: hang ? run_warp_apply<3, Real, GEOM, true>(op, k) : run_warp_apply<3, Real, GEOM, false>(op, k); break;
    case 4:
      if (cta) run_warp_apply<4, Real, GEOM, false, false, false, 128>(op, k);
      else if (hang) run_warp_apply<4, Real, GEOM, true>(op, k);
      else run_warp_apply<4, Real, GEOM, false>(op, k);
      break;
    default: throw Error{MPDG_ERR_UNSUPPORTED, "degree must be 1..4"};
  }
}

template <int P, bool KT>
void run_merge(Op &op, KP<double> k, double *c64, float *c32)
{
  Mesh &m = *op.mesh;
  constexpr int n = P + 1, CPB = Cfg<n>::cpb;
  ColourSet cs;
  for (int c = 0; c < 8; ++c) cs.c[c] = m.colour[c];
  const unsigned grid = (unsigned)((m.n_cells + CPB - 1) / CPB);
  merge_kernel<P, KT><<<grid, dim3(n * n, CPB), 0, op.stream>>>(k, cs, m.n_cells, c64, c32);
  MPDG_LAUNCHED();
}

// builds the merged coefficient stream of `op` in the requested precision
void ensure_coef(Op &op, bool want32)
{
  Mesh &m = *op.mesh;
  if (op.coef64_ok && (!want32 || op.coef32_ok)) return;
  const size_t count = (size_t)m.n_cells * metric_stride(m.n);
  if (!op.d_coef64) {
    op.d_coef64 = dev_alloc<double>(count, op.device_bytes);
    MPDG_CUDA(cudaMemsetAsync(op.d_coef64, 0, sizeof(double) * count, op.stream));
  }
  if (want32 && !op.d_coef32) {
    op.d_coef32 = dev_alloc<float>(count, op.device_bytes);
    MPDG_CUDA(cudaMemsetAsync(op.d_coef32, 0, sizeof(float) * count, op.stream));
  }
  KP<double> k = base_params<double>(op);
  const bool kt = uses_kT(op);
  if (kt && !k.T) throw Error{MPDG_ERR_ARG, "k(T) operator needs the temperature field"};
  float *c32 = want32 ? op.d_coef32 : nullptr;
  switch (m.degree) {
    case 1: kt ? run_merge<1, true>(op, k, op.d_coef64, c32) : run_merge<1, false>(op, k, op.d_coef64, c32); break;
    case 2: kt ? run_merge<2, true>(op, k, op.d_coef64, c32) : run_merge<2, false>(op, k, op.d_coef64, c32); break;
    case 3: kt ? run_merge<3, true>(op, k, op.d_coef64, c32) : run_merge<3, false>(op, k, op.d_coef64, c32); break;
    case 4: kt ? run_merge<4, true>(op, k, op.d_coef64, c32) : run_merge<4, false>(op, k, op.d_coef64, c32); break;
    default: throw Error{MPDG_ERR_UNSUPPORTED, "degree must be 1..4"};
  }
  op.coef64_ok = true;
  op.coef32_ok = want32;
}

}  // namespace

// ---------------------------------------------------------- Robin boundary faces
// Heat operator faces with a convective condition (heat_diffuse_operator.cpp:1088-1129):
// tangent alpha u v, residual -alpha (T - T_inf) v, on the box faces flagged in
// robin_faces (bit 2 d + s: direction d, side s).  One warp per face; lane
// (a, b) owns the face DoF at tangential positions (a, b) and the face
// quadrature point (q_a, q_b) = (a, b) of QGauss(p+1)^2 with the surface element
// |dx/dxi_t0 x dx/dxi_t1| of the trilinear map.  The 2D face mass is sum
// factorised through a per-warp shared tile.  Faces of one plane run in four
// parity colours, so the scatter adds without atomics.
enum { ROBIN_APPLY = 0, ROBIN_RESIDUAL = 1, ROBIN_DIAGONAL = 2 };

// the terms of one boundary face (local face (d, s) of the cell with corners
// V) for the warp that owns it: lane (a, b) < n^2 (on) holds face DoF g
template <int P, typename Real>
__device__ __forceinline__ void robin_face(const double (&V)[8][3], int d, int s, long g, bool on, int a, int b,
                                           Real *t, int conv, double alpha, double t_inf, int rad, double es,
                                           double t_rad, int mode, const Real *src, const Real *Tf, Real *dst,
                                           const uint8_t *rmask, const uint8_t *wmask)
{
  constexpr int n = P + 1;
  const Tables<Real> &T = tab<Real>(P);
  const int t0 = (d == 0) ? 1 : 0, t1 = (d == 2) ? 1 : 2;
  // surface element at the lane's face quadrature point
  double xi[3];
  xi[d] = s ? 1.0 : 0.0;
  xi[t0] = (double)T.x[a];
  xi[t1] = (double)T.x[b];
  double Ja[3] = {0, 0, 0}, Jb[3] = {0, 0, 0};
  for (int v = 0; v < 8; ++v) {
    const int bv[3] = {v & 1, (v >> 1) & 1, (v >> 2) & 1};
    double fv[3], dfv[3];
    for (int e = 0; e < 3; ++e) {
      fv[e] = bv[e] ? xi[e] : 1.0 - xi[e];
      dfv[e] = bv[e] ? 1.0 : -1.0;
    }
    double da = dfv[t0], db = dfv[t1];
    for (int e = 0; e < 3; ++e)
      if (e != t0) da *= fv[e];
    for (int e = 0; e < 3; ++e)
      if (e != t1) db *= fv[e];
    for (int e = 0; e < 3; ++e) {
      Ja[e] += V[v][e] * da;
      Jb[e] += V[v][e] * db;
    }
  }
  const double cr[3] = {Ja[1] * Jb[2] - Ja[2] * Jb[1], Ja[2] * Jb[0] - Ja[0] * Jb[2],
                        Ja[0] * Jb[1] - Ja[1] * Jb[0]};
  const double jxw = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]) * (double)T.w[a] * (double)T.w[b];
  // face interpolation: lane (a, b) holds a nodal value and receives the value
  // at face quadrature point (a, b), along t0 then t1
  const auto interp = [&](Real v) -> Real {
    if (on) t[b * n + a] = v;
    __syncwarp();
    Real w = 0;
    for (int r = 0; r < n; ++r) w += T.S[a * n + r] * t[b * n + r];
    __syncwarp();
    if (on) t[b * n + a] = w;
    __syncwarp();
    Real q = 0;
    for (int r = 0; r < n; ++r) q += T.S[b * n + r] * t[r * n + a];
    __syncwarp();
    return q;
  };
  // T at the point: the residual's argument, or the linearisation point of the
  // radiative tangent
  Real Tq = 0;
  if (rad || mode == ROBIN_RESIDUAL) {
    const Real *Ts = (mode == ROBIN_RESIDUAL) ? src : Tf;
    Tq = interp(on ? Ts[g] : Real(0));
  }
  const Real coef = (conv ? (Real)alpha : Real(0)) + (rad ? Real(4) * (Real)es * Tq * Tq * Tq : Real(0));
  Real out;
  if (mode == ROBIN_DIAGONAL) {
    if (on) t[b * n + a] = coef * (Real)jxw;
    __syncwarp();
    out = 0;
    for (int qb = 0; qb < n; ++qb)
      for (int qa = 0; qa < n; ++qa) {
        const Real sa = T.S[qa * n + a], sb = T.S[qb * n + b];
        out += sa * sa * sb * sb * t[qb * n + qa];
      }
  } else {
    Real val;
    if (mode == ROBIN_RESIDUAL) {
      const Real tr = (Real)t_rad, T2 = Tq * Tq;
      val = -(conv ? (Real)alpha * (Tq - (Real)t_inf) : Real(0)) -
            (rad ? (Real)es * (T2 * T2 - tr * tr * tr * tr) : Real(0));
    } else {
      val = coef * interp(on ? ((rmask && rmask[g]) ? Real(0) : src[g]) : Real(0));
    }
    // tested with the face shape functions: transposed passes
    if (on) t[b * n + a] = val * (Real)jxw;
    __syncwarp();
    Real w = 0;
    for (int r = 0; r < n; ++r) w += T.S[r * n + a] * t[b * n + r];
    __syncwarp();
    if (on) t[b * n + a] = w;
    __syncwarp();
    out = 0;
    for (int r = 0; r < n; ++r) out += T.S[r * n + b] * t[r * n + a];
  }
  if (on && !(wmask && wmask[g])) dst[g] += out;
}

template <int P, typename Real>
__global__ void __launch_bounds__(128) robin_kernel(const double *vert, int nc0, int nc1, int nc2, int d, int s,
                                                    int colour, long NX, long NY, int conv, double alpha,
                                                    double t_inf, int rad, double es, double t_rad, int mode,
                                                    const Real *src, const Real *Tf, Real *dst,
                                                    const uint8_t *rmask, const uint8_t *wmask)
{
  constexpr int n = P + 1, n2 = n * n;
  __shared__ Real tile[4][n2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nc[3] = {nc0, nc1, nc2};
  const int t0 = (d == 0) ? 1 : 0, t1 = (d == 2) ? 1 : 2;
  const int pa = colour & 1, pb = (colour >> 1) & 1;
  const int ca = (nc[t0] - pa + 1) / 2, cb = (nc[t1] - pb + 1) / 2;
  const long f = (long)blockIdx.x * 4 + warp;
  if (f >= (long)ca * cb) return;  // warp-uniform
  const int fa = 2 * (int)(f % ca) + pa, fb = 2 * (int)(f / ca) + pb;
  int cell[3];
  cell[d] = s ? nc[d] - 1 : 0;
  cell[t0] = fa;
  cell[t1] = fb;
  const bool on = lane < n2;
  const int a = on ? lane % n : 0, b = on ? lane / n : 0;
  int loc[3];
  loc[d] = s ? P : 0;
  loc[t0] = a;
  loc[t1] = b;
  const long g = ((long)(cell[2] * P + loc[2]) * NY + (cell[1] * P + loc[1])) * NX + (cell[0] * P + loc[0]);
  double V[8][3];
  for (int v = 0; v < 8; ++v) {
    const long vid = ((long)(cell[2] + ((v >> 2) & 1)) * (nc1 + 1) + (cell[1] + ((v >> 1) & 1))) * (nc0 + 1) +
                     (cell[0] + (v & 1));
    for (int e = 0; e < 3; ++e) V[v][e] = vert[vid * 3 + e];
  }
  robin_face<P, Real>(V, d, s, g, on, a, b, tile[warp], conv, alpha, t_inf, rad, es, t_rad, mode, src, Tf, dst,
                      rmask, wmask);
}

// boundary faces of a mapped mesh (cells' local faces with a boundary id
// whose bit conv_bits / rad_bits selects), one warp per face of one face
// colour: the faces of a colour share no DoF, so the scatter adds without atomics
template <int P, typename Real>
__global__ void __launch_bounds__(128) mapped_face_kernel(const int *fcell, const int8_t *fface, const int8_t *fid,
                                                          long first, long count, const int *cmap,
                                                          const double *cellvert, int conv_bits, double alpha,
                                                          double t_inf, int rad_bits, double es, double t_rad,
                                                          int mode, const Real *src, const Real *Tf, Real *dst,
                                                          const uint8_t *rmask, const uint8_t *wmask,
                                                          const uint8_t *cell_flags)
{
  constexpr int n = P + 1, n2 = n * n, n3 = n2 * n;
  __shared__ Real tile[4][n2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long f = (long)blockIdx.x * 4 + warp;
  if (f >= count) return;  // warp-uniform
  const long e = first + f;
  const long slot = fcell[e];
  // the diagonal of a cell with constrained DoFs comes from its element
  // matrix, face matrices included
  if (mode == ROBIN_DIAGONAL && cell_flags && (cell_flags[slot] & 2)) return;  // warp-uniform
  const int face = fface[e], id = fid[e];
  const int conv = (conv_bits >> id) & 1, rad = (rad_bits >> id) & 1;
  if (!conv && !rad) return;  // warp-uniform
  const int d = face >> 1, s = face & 1;
  const int t0 = (d == 0) ? 1 : 0, t1 = (d == 2) ? 1 : 2;
  const bool on = lane < n2;
  const int a = on ? lane % n : 0, b = on ? lane / n : 0;
  int loc[3];
  loc[d] = s ? P : 0;
  loc[t0] = a;
  loc[t1] = b;
  const long g = cmap[slot * n3 + (loc[2] * n + loc[1]) * n + loc[0]];
  double V[8][3];
  for (int v = 0; v < 8; ++v)
    for (int c = 0; c < 3; ++c) V[v][c] = cellvert[(slot * 8 + v) * 3 + c];
  robin_face<P, Real>(V, d, s, g, on, a, b, tile[warp], conv, alpha, t_inf, rad, es, t_rad, mode, src, Tf, dst,
                      rmask, wmask);
}

template <typename Real>
void launch_robin(Op &op, Real *dst, const Real *src, int mode)
{
  const mpdg_op_desc &D = op.d;
  if (D.kind != MPDG_OP_HEAT) return;
  const bool any_conv = D.robin_faces && D.robin_alpha != 0.0, any_rad = D.rad_faces && D.rad_emissivity != 0.0;
  if (!any_conv && !any_rad) return;
  Mesh &m = *op.mesh;
  const Real *Tf = nullptr;
  if constexpr (sizeof(Real) == 8) Tf = op.T64;
  else Tf = op.T32;
  if (any_rad && !Tf) throw Error{MPDG_ERR_ARG, "radiative faces need the temperature field"};
  const double es = D.rad_emissivity * 5.670374419e-8;  // Stefan-Boltzmann constant
  upload_tables();
  const bool mask = op.use_dirichlet && m.has_dirichlet;
  const uint8_t *rmask = (mode == ROBIN_APPLY && mask) ? m.d_dmask : nullptr;
  const uint8_t *wmask = mask ? m.d_dmask : nullptr;
  if (m.mapped) {
    // the cells' faces with a selected boundary id, colour by colour
    const int conv_bits = any_conv ? D.robin_faces : 0, rad_bits = any_rad ? D.rad_faces : 0;
    for (size_t c = 0; c + 1 < m.mface_first.size(); ++c) {
      const long first = m.mface_first[c], count = m.mface_first[c + 1] - first;
      if (count == 0) continue;
      const unsigned grid = (unsigned)((count + 3) / 4);
#define MPDG_MFACE(PP)                                                                                            \
  mapped_face_kernel<PP, Real><<<grid, 128, 0, op.stream>>>(m.d_mface_cell, m.d_mface_f, m.d_mface_id, first, count, \
                                                            m.d_cmap, m.d_cellvert, conv_bits, D.robin_alpha,        \
                                                            D.robin_t_inf, rad_bits, es, D.rad_t_inf, mode, src, Tf, \
                                                            dst, rmask, wmask, m.d_cell_flags)
      switch (m.degree) {
        case 1: MPDG_MFACE(1); break;
        case 2: MPDG_MFACE(2); break;
        case 3: MPDG_MFACE(3); break;
        default: MPDG_MFACE(4); break;
      }
#undef MPDG_MFACE
      MPDG_LAUNCHED();
    }
    return;
  }
  for (int d = 0; d < 3; ++d)
    for (int s = 0; s < 2; ++s) {
      const int bit = 1 << (2 * d + s);
      const int conv = any_conv && (D.robin_faces & bit), rad = any_rad && (D.rad_faces & bit);
      if (!conv && !rad) continue;
      const int t0 = (d == 0) ? 1 : 0, t1 = (d == 2) ? 1 : 2;
      for (int c = 0; c < 4; ++c) {
        const long ca = (m.nc[t0] - (c & 1) + 1) / 2, cb = (m.nc[t1] - ((c >> 1) & 1) + 1) / 2;
        const long faces = ca * cb;
        if (faces == 0) continue;
        const unsigned grid = (unsigned)((faces + 3) / 4);
#define MPDG_ROBIN(PP)                                                                                   \
  robin_kernel<PP, Real><<<grid, 128, 0, op.stream>>>(m.d_vert, m.nc[0], m.nc[1], m.nc[2], d, s, c, m.NX, \
                                                      m.NY, conv, D.robin_alpha, D.robin_t_inf, rad, es,   \
                                                      D.rad_t_inf, mode, src, Tf, dst, rmask, wmask)
        switch (m.degree) {
          case 1: MPDG_ROBIN(1); break;
          case 2: MPDG_ROBIN(2); break;
          case 3: MPDG_ROBIN(3); break;
          default: MPDG_ROBIN(4); break;
        }
#undef MPDG_ROBIN
        MPDG_LAUNCHED();
      }
    }
}

void invalidate_coef(Op &op)
{
  op.coef64_ok = false;
  op.coef32_ok = false;
}

// ------------------------------------------------------------ hanging nodes
// Adds the staged contributions of the fine interface cells to the coarse DoFs
// of the interface plane: one thread per coarse DoF (Y, Z) sums, in a fixed
// order, the stage entries of the (up to 4) coarse faces containing it times
// their 4 subfaces, so the result is deterministic.
template <typename Real>
__global__ void hang_fold_kernel(const Real *stage, Real *dst, long NXc, long NYc, long NZc, int P, int ncc1,
                                 int ncc2, int ncf1, const uint8_t *cmask)
{
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= NYc * NZc) return;
  const int Y = (int)(t % NYc), Z = (int)(t / NYc);
  const int n = P + 1;
  int cys[2], czs[2], ny = 0, nz = 0;
  const int qy = Y / P, qz = Z / P;
  if (Y % P == 0) {
    if (qy >= 1) cys[ny++] = qy - 1;
    if (qy < ncc1) cys[ny++] = qy;
  } else {
    cys[ny++] = qy;
  }
  if (Z % P == 0) {
    if (qz >= 1) czs[nz++] = qz - 1;
    if (qz < ncc2) czs[nz++] = qz;
  } else {
    czs[nz++] = qz;
  }
  Real sum = 0;
  for (int b = 0; b < nz; ++b)
    for (int a = 0; a < ny; ++a) {
      const int cy = cys[a], cz = czs[b], jp = Y - cy * P, kp = Z - cz * P;
      for (int sz = 0; sz < 2; ++sz)
        for (int sy = 0; sy < 2; ++sy) {
          const long fi = (long)(2 * cz + sz) * ncf1 + (2 * cy + sy);
          sum += stage[fi * n * n + kp * n + jp];
        }
    }
  const long g = ((long)Z * NYc + Y) * NXc + (NXc - 1);
  if (!(cmask && cmask[g])) dst[g] += sum;
}

// probe of the interface plane for the diagonal: x = 1 at the coarse interface
// DoFs (Y, Z) with Y % n == a and Z % n == b, 0 elsewhere
__global__ void hang_probe_kernel(double *x, long N, long NXc, long NYc, long NZc, int n, int a, int b)
{
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < N; t += (long)gridDim.x * blockDim.x) {
    double v = 0.0;
    if (t < NXc * NYc * NZc && t % NXc == NXc - 1) {
      const long Y = (t / NXc) % NYc, Z = t / (NXc * NYc);
      v = (Y % n == a && Z % n == b) ? 1.0 : 0.0;
    }
    x[t] = v;
  }
}

__global__ void hang_probe_take_kernel(double *diag, const double *y, long NXc, long NYc, long NZc, int n, int a,
                                       int b)
{
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= NYc * NZc) return;
  const long Y = t % NYc, Z = t / NYc;
  if (Y % n != a || Z % n != b) return;
  const long g = (Z * NYc + Y) * NXc + (NXc - 1);
  diag[g] = y[g];
}

template <typename Real>
void launch_cells(Op &op, Real *dst, const Real *src);

// the fine block of a two-level mesh, after the coarse block: its hanging DoFs
// read the coarse values of src, their contributions fold into dst's coarse part
template <typename Real>
void launch_fine_block(Op &op, Real *dst, const Real *src)
{
  Op &f = *op.fine;
  Mesh &m = *op.mesh;
  const bool mask = op.use_dirichlet && m.has_dirichlet;
  f.use_dirichlet = op.use_dirichlet;
  // the fine block runs in the apply's stream, which may be a capture stream
  // that is destroyed after the capture: the fine op's own stream comes back
  const cudaStream_t fine_stream = f.stream;
  f.stream = op.stream;
  f.hang_src = src;
  f.hang_mask = mask ? m.d_dmask : nullptr;
  try {
    launch_cells<Real>(f, dst + m.N_own, src + m.N_own);
  } catch (...) {
    f.hang_src = nullptr;
    f.stream = fine_stream;
    throw;
  }
  f.hang_src = nullptr;
  f.stream = fine_stream;
  const Mesh &fm = *f.mesh;
  const long cnt = m.NY * m.NZ;
  hang_fold_kernel<Real><<<grid_for(cnt, 256), 256, 0, op.stream>>>(
      (const Real *)f.d_stage, dst, m.NX, m.NY, m.NZ, m.degree, m.nc[1], m.nc[2], fm.nc[1], mask ? m.d_dmask : nullptr);
  MPDG_LAUNCHED();
}



template <typename Real>
__global__ void io_pre_kernel(Real *tmp, const Real *src, const uint8_t *io, long n)
{
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    tmp[i] = io[i] ? Real(0) : src[i];
}

template <typename Real>
__global__ void io_post_kernel(Real *dst, const Real *src, const uint8_t *io, long n)
{
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    if (io[i]) dst[i] = src[i];
}

template <typename Real>
void launch_apply(Op &op, Real *dst, const Real *src)
{
  const Real *in = src;
  const long N = op.mesh->N;
  const unsigned grid = (unsigned)std::min(grid_for(N, 256), (unsigned)(148 * 16));
  if (op.d_io) {
    // do_pre_vmult: the constrained entries of src read as 0 (in a copy; the
    // caller's src is not modified)
    const size_t bytes = sizeof(Real) * (size_t)N;
    if (op.io_tmp_bytes < bytes) {
      if (op.io_tmp) cudaFree(op.io_tmp);
      op.io_tmp = nullptr;
      op.io_tmp_bytes = 0;
      MPDG_CUDA(tracked_malloc(&op.io_tmp, bytes));
      op.io_tmp_bytes = bytes;
    }
    io_pre_kernel<Real><<<grid, 256, 0, op.stream>>>((Real *)op.io_tmp, src, op.d_io, N);
    MPDG_LAUNCHED();
    in = (const Real *)op.io_tmp;
  }
  if (op.mesh->mapped) {
    launch_mapped_apply<Real>(op, dst, in);
  } else {
    launch_cells<Real>(op, dst, in);
    launch_robin<Real>(op, dst, in, ROBIN_APPLY);
    if (op.fine) launch_fine_block<Real>(op, dst, in);
  }
  if (op.d_io) {
    // do_post_vmult: identity rows
    io_post_kernel<Real><<<grid, 256, 0, op.stream>>>(dst, src, op.d_io, N);
    MPDG_LAUNCHED();
  }
}

template <typename Real>
void launch_cells(Op &op, Real *dst, const Real *src)
{
  Mesh &m = *op.mesh;
  const bool kt = uses_kT(op);
  const bool full = op.d.kind == MPDG_OP_HEAT && op.d.full_tangent;
  if (!m.uniform && op.d.vel_kind != MPDG_VEL_NONE && sizeof(Real) == 4 && !op.d_velb32)
    throw Error{MPDG_ERR_ARG, "the FP32 form was not prepared for this operator (precision_mask)"};
  KP<Real> k = base_params<Real>(op);
  k.src = src;
  k.dst = dst;
  if (kt && !k.T) throw Error{MPDG_ERR_ARG, "k(T) operator needs the temperature field"};
  check_law_fields(op, k);
  if (supg(op)) {
    // SUPG: block kernel with the stabilisation flux (raw geometry on general meshes)
    if (!k.tau) throw Error{MPDG_ERR_ARG, "the FP32 form was not prepared for this operator (precision_mask)"};
    if (!m.uniform && sizeof(Real) == 4) {
      ensure_metric32(m, op.stream);
      k.metric = (const Real *)(const void *)m.d_metric32;
    }
    MPDG_CUDA(cudaMemsetAsync(dst, 0, sizeof(Real) * m.N_own, op.stream));
    dispatch_degree<Real, MODE_SUPG, false>(op, k);
    return;
  }
  const bool law = uses_law(op);
  if (!full && !law && !m.uniform) {
    // general geometry: merged coefficient stream (k(T), c_mass, c_diff folded in)
    ensure_coef(op, sizeof(Real) == 4);
    if constexpr (sizeof(Real) == 8) k.metric = op.d_coef64;
    else k.metric = op.d_coef32;
    warp_apply_degree<Real, GEOM_GENERAL>(op, k);
    return;
  }
  if (!full && !kt) {
    warp_apply_degree<Real, GEOM_UNIFORM>(op, k);
    return;
  }
  // full Newton tangent, material laws, or k(T) on a uniform mesh: block kernel on raw geometry
  if (!m.uniform && sizeof(Real) == 4) {
    ensure_metric32(m, op.stream);
    k.metric = (const Real *)(const void *)m.d_metric32;
  }
  MPDG_CUDA(cudaMemsetAsync(dst, 0, sizeof(Real) * m.N_own, op.stream));
  if (kt) dispatch_degree<Real, MODE_LINEAR, true>(op, k);
  else dispatch_degree<Real, MODE_LINEAR, false>(op, k);
}

template void launch_apply<double>(Op &, double *, const double *);
template void launch_apply<float>(Op &, float *, const float *);

bool plain_warp_apply(const Op &op)
{
  const Mesh &m = *op.mesh;
  const mpdg_op_desc &D = op.d;
  const bool heat = D.kind == MPDG_OP_HEAT;
  const bool faces = heat && ((D.robin_faces && D.robin_alpha != 0.0) || (D.rad_faces && D.rad_emissivity != 0.0));
  const bool full = heat && D.full_tangent;
  return !op.fine && !m.mapped && !op.d_io && !faces && !supg(op) && !full && !uses_law(op) &&
         (!m.uniform || !uses_kT(op));
}

void set_wait_first_polls(long long polls)
{
  const long long v = polls < 0 ? (long long)kMbarSpinLimit : polls;
  MPDG_CUDA(cudaMemcpyToSymbol(c_wait_first_polls, &v, sizeof(v)));
}

int slab_bounds(int nz, int S, int *bounds)
{
  S = std::max(1, std::min(S, std::min(kMaxApplySlabs, nz / 2)));
  bounds[0] = 0;
  for (int i = 1; i < S; ++i) {
    const int b = (int)((long)i * nz / S) | 1;
    bounds[i] = std::min(std::max(b, bounds[i - 1] + 1), nz - 1);
  }
  bounds[S] = nz;
  for (int i = 1; i < S; ++i)
    if (bounds[i] % 2 == 0 || bounds[i] <= bounds[i - 1] || bounds[i] >= nz)
      throw Error{MPDG_ERR_ARG, "slab bounds"};
  return S;
}

void autotune_apply(Op &op, int precision, int reps, ApplySchedule &best, double &best_ms,
                    std::vector<double> *all_ms)
{
  Mesh &m = *op.mesh;
  const size_t esz = precision == MPDG_FP32 ? sizeof(float) : sizeof(double);
  const size_t bytes = esz * (size_t)m.N;
  reps = std::max(1, reps);
  // candidates: slabs 1, 2, 4, 8, 16 (as many as the layers allow), each with and
  // without the evict-first hint where a coefficient stream exists
  std::vector<ApplySchedule> cand;
  const bool stream = !m.uniform || m.mapped;
  const bool cta_differs = (m.degree == 2 || m.degree == 4) && !m.mapped && !op.fine;
  // the lane apply: uniform lattices of degree 1 or 2 whose vmult takes the
  // constant-coefficient path with an in-kernel velocity
  const bool lane_ok = m.uniform && !m.mapped && !op.fine && (m.degree == 1 || m.degree == 2) &&
                       plain_warp_apply(op) && !uses_kT(op) && op.d.vel_kind != MPDG_VEL_NODAL;
  const int lane_max = lane_ok ? (m.degree == 2 ? 2 : 1) : 0;
  for (int S : {1, 2}) {
    if (S > 1 && (S > m.nc[2] / 2 || m.mapped || op.fine)) continue;
    for (int h = 0; h <= (stream ? 1 : 0); ++h)
      for (int d = 0; d <= 1; ++d) {
        for (int g = 0; g <= (cta_differs ? 1 : 0); ++g) {
          ApplySchedule c;
          c.slabs = S;
          c.evict_first = h;
          c.pdl = d;
          c.cta = g;
          cand.push_back(c);
        }
        for (int l = 1; l <= lane_max; ++l) {
          ApplySchedule c;
          c.slabs = S;
          c.evict_first = h;
          c.pdl = d;
          c.lane = l;
          cand.push_back(c);
        }
      }
  }
  void *x = nullptr, *y = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  const ApplySchedule saved = op.sched[precision];
  MPDG_CUDA(tracked_malloc(&x, bytes));
  auto cleanup = [&]() {
    cudaStreamSynchronize(op.stream);
    if (x) cudaFree(x);
    if (y) cudaFree(y);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  };
  try {
    MPDG_CUDA(tracked_malloc(&y, bytes));
    MPDG_CUDA(cudaEventCreate(&e0));
    MPDG_CUDA(cudaEventCreate(&e1));
    MPDG_CUDA(cudaMemsetAsync(x, 0, bytes, op.stream));
    best_ms = -1.0;
    if (all_ms) all_ms->clear();
    for (const ApplySchedule &c : cand) {
      op.sched[precision] = c;
      auto apply = [&]() {
        if (precision == MPDG_FP32) launch_apply<float>(op, (float *)y, (const float *)x);
        else launch_apply<double>(op, (double *)y, (const double *)x);
      };
      apply();  // warm-up (first use of the schedule)
      MPDG_CUDA(cudaEventRecord(e0, op.stream));
      for (int r = 0; r < reps; ++r) apply();
      MPDG_CUDA(cudaEventRecord(e1, op.stream));
      MPDG_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      MPDG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      const double per = ms / reps;
      if (all_ms) all_ms->push_back(per);
      if (best_ms < 0.0 || per < best_ms) {
        best_ms = per;
        best = c;
      }
    }
    op.sched[precision] = best;
  } catch (...) {
    op.sched[precision] = saved;
    cleanup();
    throw;
  }
  cleanup();
}

void launch_apply_zrange(Op &op, double *dst, const double *src, int z0, int z1)
{
  Mesh &m = *op.mesh;
  if (!plain_warp_apply(op)) throw Error{MPDG_ERR_UNSUPPORTED, "layer-range apply: plain warp operators only"};
  KP<double> k = base_params<double>(op);
  if (uses_kT(op) && !k.T) throw Error{MPDG_ERR_ARG, "k(T) operator needs the temperature field"};
  k.src = src;
  k.dst = dst;
  k.zlo = z0;
  k.zhi = z1;
  if (m.uniform) {
    warp_apply_degree<double, GEOM_UNIFORM>(op, k);
  } else {
    ensure_coef(op, false);
    k.metric = op.d_coef64;
    warp_apply_degree<double, GEOM_GENERAL>(op, k);
  }
}

// dst[v] = A src[v] for nvec vectors.  Operators whose apply is the plain warp
// kernel (no faces, constraints rows, hanging nodes, SUPG or phase law) take up
// to kMaxMultiVec vectors per pass, reading each cell's coefficients once;
// the others apply the vectors one after the other.
template <typename Real>
void launch_apply_multi(Op &op, int nvec, Real *const *dst, const Real *const *src)
{
  Mesh &m = *op.mesh;
  const long N = m.N;
  for (int a = 0; a < nvec; ++a) {
    if (!dst[a] || !src[a]) throw Error{MPDG_ERR_ARG, "null vector"};
    for (int b = 0; b < nvec; ++b) {
      const bool over_ds = dst[a] < src[b] + N && src[b] < dst[a] + N;
      const bool over_dd = a != b && dst[a] < dst[b] + N && dst[b] < dst[a] + N;
      if (over_ds || over_dd) throw Error{MPDG_ERR_ARG, "multi-vector apply: destinations overlap a vector"};
    }
  }
  if (!plain_warp_apply(op)) {
    for (int v = 0; v < nvec; ++v) launch_apply<Real>(op, dst[v], src[v]);
    return;
  }
  if (!m.uniform && op.d.vel_kind != MPDG_VEL_NONE && sizeof(Real) == 4 && !op.d_velb32)
    throw Error{MPDG_ERR_ARG, "the FP32 form was not prepared for this operator (precision_mask)"};
  KP<Real> k = base_params<Real>(op);
  if (uses_kT(op) && !k.T) throw Error{MPDG_ERR_ARG, "k(T) operator needs the temperature field"};
  if (!m.uniform) {
    ensure_coef(op, sizeof(Real) == 4);
    if constexpr (sizeof(Real) == 8) k.metric = op.d_coef64;
    else k.metric = op.d_coef32;
  }
  for (int c = 0; c < nvec; c += kMaxMultiVec) {
    const int cnt = std::min(kMaxMultiVec, nvec - c);
    k.src = src[c];
    k.dst = dst[c];
    k.nvec = cnt;
    for (int v = 0; v < cnt; ++v) {
      k.msrc[v] = src[c + v];
      k.mdst[v] = dst[c + v];
    }
    if (m.uniform) warp_apply_degree<Real, GEOM_UNIFORM>(op, k);
    else warp_apply_degree<Real, GEOM_GENERAL>(op, k);
  }
}

template void launch_apply_multi<double>(Op &, int, double *const *, const double *const *);
template void launch_apply_multi<float>(Op &, int, float *const *, const float *const *);

void launch_rhs(Op &op, double *dst, const double *src, const double *heat_source)
{
  if (op.fine) throw Error{MPDG_ERR_UNSUPPORTED, "create_rhs on two-level meshes"};
  KP<double> k = base_params<double>(op);
  k.src = src;
  k.dst = dst;
  k.masked_read = 0;  // read_dof_values_plain
  if (op.d.kind == MPDG_OP_HEAT) {
    if (!op.T64) throw Error{MPDG_ERR_ARG, "heat residual needs the temperature field"};
    check_law_fields(op, k);
    k.q_src = heat_source;
    dispatch_degree<double, MODE_HEAT_RESIDUAL, false>(op, k);
    launch_robin<double>(op, dst, op.T64, ROBIN_RESIDUAL);
  } else {
    if (heat_source) throw Error{MPDG_ERR_ARG, "advection-diffusion rhs takes no heat source"};
    // phi_old/dt N - (1-theta) vel.grad phi_old N - (1-theta) D grad phi_old . grad N
    k.c_mass = 1.0 / op.d.dt;
    k.c_vel = -(1.0 - op.d.theta);
    k.c_diff = -(1.0 - op.d.theta) * op.d.diffusivity;
    k.k_alpha = 0.0;
    k.full_tangent = 0;
    // SUPG: + tau_K u (phi_old/dt - (1-theta) u.grad phi_old + (1-theta) D lap phi_old)
    // tested with grad N (advection_diffusion_operator.cpp:336-346)
    if (supg(op)) dispatch_degree<double, MODE_SUPG, false>(op, k);
    else dispatch_degree<double, MODE_LINEAR, false>(op, k);
  }
  // integrate_scatter through the constraints: the constrained rows go to their masters
  if (op.mesh->mapped) mapped_condense<double>(op, dst);
}

namespace {
template <int P, bool KT>
void run_diag(Op &op, KP<double> k)
{
  Mesh &m = *op.mesh;
  constexpr int n = P + 1, CPB = Cfg<n>::cpb;
  const dim3 block(n * n, CPB);
  for (int c = 0; c < n_colours(m); ++c) {
    const Colour &C = colours(m)[c];
    if (C.count == 0) continue;
    colour_params(k, C);
    const unsigned grid = (unsigned)((C.count + CPB - 1) / CPB);
    if (m.uniform) diag_kernel<P, GEOM_UNIFORM, KT><<<grid, block, 0, op.stream>>>(k);
    else diag_kernel<P, GEOM_GENERAL, KT><<<grid, block, 0, op.stream>>>(k);
    MPDG_LAUNCHED();
  }
}
}  // namespace

#include "mapped.cuh"

void launch_block_diagonal(Op &op, double *diag);

// Diagonal of a two-level mesh: each block's local diagonal, then the coarse
// interface DoFs by probing.  A probe sets 1 at the interface DoFs with
// (Y % n, Z % n) = (a, b).  Two such DoFs are at least n apart in Y or Z, so
// they share neither a coarse cell nor a coarse face (and so no fine interface
// cell): the full apply returns each probed DoF's exact diagonal entry.
// n^2 probes, each one apply.
void launch_composite_diagonal(Op &op, double *diag)
{
  Mesh &m = *op.mesh;
  launch_block_diagonal(op, diag);
  Op &f = *op.fine;
  f.use_dirichlet = op.use_dirichlet;
  launch_block_diagonal(f, diag + m.N_own);
  double *x = nullptr, *y = nullptr;
  MPDG_CUDA(tracked_malloc(&x, sizeof(double) * m.N));
  const cudaError_t e = tracked_malloc(&y, sizeof(double) * m.N);
  if (e != cudaSuccess) {
    cudaFree(x);
    throw Error{MPDG_ERR_ALLOC, "diagonal probes"};
  }
  try {
    const int n = m.degree + 1;
    const long cnt = m.NY * m.NZ;
    for (int b = 0; b < n; ++b)
      for (int a = 0; a < n; ++a) {
        hang_probe_kernel<<<grid_for(std::min(m.N, 148L * 1024), 256), 256, 0, op.stream>>>(x, m.N, m.NX, m.NY,
                                                                                           m.NZ, n, a, b);
        MPDG_LAUNCHED();
        launch_apply<double>(op, y, x);
        hang_probe_take_kernel<<<grid_for(cnt, 256), 256, 0, op.stream>>>(diag, y, m.NX, m.NY, m.NZ, n, a, b);
        MPDG_LAUNCHED();
      }
    const uint8_t *tm = op.use_dirichlet ? m.d_tmask_dir : m.d_tmask_hang;
    set_masked_kernel<<<grid_for(m.N, 256), 256, 0, op.stream>>>(diag, m.N, tm, 1.0);
    MPDG_LAUNCHED();
    MPDG_CUDA(cudaStreamSynchronize(op.stream));
  } catch (...) {
    cudaStreamSynchronize(op.stream);
    cudaFree(x);
    cudaFree(y);
    throw;
  }
  cudaFree(x);
  cudaFree(y);
}

void launch_diagonal(Op &op, double *diag)
{
  if (op.mesh->mapped) {
    launch_mapped_diagonal(op, diag);
    return;
  }
  if (op.fine) {
    launch_composite_diagonal(op, diag);
    return;
  }
  launch_block_diagonal(op, diag);
}

// Diagonal of a SUPG operator by probing: n^3 residue classes, one apply each
// (the SUPG element matrix has no product-of-1D-tables diagonal of the kind
// diag_kernel sums; MatrixFreeTools::compute_diagonal does the same unit sweeps
// cell by cell)
void launch_probe_diagonal(Op &op, double *diag)
{
  Mesh &m = *op.mesh;
  double *x = nullptr, *y = nullptr;
  MPDG_CUDA(tracked_malloc(&x, sizeof(double) * m.N));
  const cudaError_t e = tracked_malloc(&y, sizeof(double) * m.N);
  if (e != cudaSuccess) {
    cudaFree(x);
    throw Error{MPDG_ERR_ALLOC, "diagonal probes"};
  }
  try {
    const int n = m.degree + 1;
    const unsigned grid = grid_for(std::min(m.N, 148L * 1024), 256);
    for (int c = 0; c < n; ++c)
      for (int b = 0; b < n; ++b)
        for (int a = 0; a < n; ++a) {
          lattice_probe_kernel<<<grid, 256, 0, op.stream>>>(x, m.N, m.NX, m.NY, n, a, b, c);
          MPDG_LAUNCHED();
          launch_cells<double>(op, y, x);
          lattice_take_kernel<<<grid, 256, 0, op.stream>>>(diag, y, m.N, m.NX, m.NY, n, a, b, c);
          MPDG_LAUNCHED();
        }
    if (op.use_dirichlet && m.has_dirichlet) {
      set_masked_kernel<<<grid_for(m.N, 256), 256, 0, op.stream>>>(diag, m.N, m.d_dmask, 1.0);
      MPDG_LAUNCHED();
    }
    MPDG_CUDA(cudaStreamSynchronize(op.stream));
  } catch (...) {
    cudaStreamSynchronize(op.stream);
    cudaFree(x);
    cudaFree(y);
    throw;
  }
  cudaFree(x);
  cudaFree(y);
}

void launch_block_diagonal(Op &op, double *diag)
{
  Mesh &m = *op.mesh;
  if (supg(op)) {
    launch_probe_diagonal(op, diag);
    return;
  }
  KP<double> k = base_params<double>(op);
  k.dst = diag;
  const bool kt = uses_kT(op);
  if (kt && !k.T) throw Error{MPDG_ERR_ARG, "k(T) operator needs the temperature field"};
  check_law_fields(op, k);
  MPDG_CUDA(cudaMemsetAsync(diag, 0, sizeof(double) * m.N_own, op.stream));

  switch (m.degree) {
    case 1: kt ? run_diag<1, true>(op, k) : run_diag<1, false>(op, k); break;
    case 2: kt ? run_diag<2, true>(op, k) : run_diag<2, false>(op, k); break;
    case 3: kt ? run_diag<3, true>(op, k) : run_diag<3, false>(op, k); break;
    case 4: kt ? run_diag<4, true>(op, k) : run_diag<4, false>(op, k); break;
    default: throw Error{MPDG_ERR_UNSUPPORTED, "degree must be 1..4"};
  }
  launch_robin<double>(op, diag, nullptr, ROBIN_DIAGONAL);
  if (op.use_dirichlet && m.has_dirichlet) {
    set_masked_kernel<<<grid_for(m.N_own, 256), 256, 0, op.stream>>>(diag, m.N_own, m.d_dmask, 1.0);
    MPDG_LAUNCHED();
  }
}

// DoFs whose diagonal (and inverse) is 1: Dirichlet DoFs when selected, and the
// hanging DoFs of a two-level mesh always
const uint8_t *constraint_mask(const Op &op)
{
  const Mesh &m = *op.mesh;
  if (m.fine || m.mapped) return op.use_dirichlet ? m.d_tmask_dir : m.d_tmask_hang;
  return (op.use_dirichlet && m.has_dirichlet) ? m.d_dmask : nullptr;
}

void launch_invert_diagonal(Op &op, double *diag)
{
  Mesh &m = *op.mesh;
  double thr = 1e-10;  // heat_diffuse_operator.cpp:283
  if (op.d.kind == MPDG_OP_ADVDIFF) {
    // advection_diffusion_operator.cpp:436-439
    thr = 1e-14 * std::fmax(1.0, linf(diag, m.N, op.stream));
  }
  invert_kernel<<<grid_for(m.N, 256), 256, 0, op.stream>>>(diag, m.N, constraint_mask(op), thr);
  MPDG_LAUNCHED();
  if (op.d_io) {  // advection_diffusion_operator.cpp:438-445
    set_masked_kernel<<<grid_for(m.N, 256), 256, 0, op.stream>>>(diag, m.N, op.d_io, 1.0);
    MPDG_LAUNCHED();
  }
}

void launch_invert_with_threshold(Op &op, double *diag, double thr)
{
  Mesh &m = *op.mesh;
  invert_kernel<<<grid_for(m.N, 256), 256, 0, op.stream>>>(diag, m.N, constraint_mask(op), thr);
  MPDG_LAUNCHED();
  if (op.d_io) {  // identity rows: inverse diagonal 1 (advection_diffusion_operator.cpp:438-445)
    set_masked_kernel<<<grid_for(m.N, 256), 256, 0, op.stream>>>(diag, m.N, op.d_io, 1.0);
    MPDG_LAUNCHED();
  }
}

const char *noalloc_unready_reason(const Op &op)
{
  const Mesh &m = *op.mesh;
  const bool full = op.d.kind == MPDG_OP_HEAT && op.d.full_tangent;
  if (op.fine) return "two-level meshes are not supported (their diagonal probes allocate)";
  if (supg(op)) return "SUPG operators are not supported (their diagonal probes allocate)";
  if (op.d_io && op.io_tmp_bytes < sizeof(double) * (size_t)m.N)
    return "the inflow/outflow copy of the operand is not built yet: call mpdg_vmult once first";
  if (m.mapped) {
    if (m.n_cons != 0) return "mapped meshes with constraints are not supported (operand copy, element matrices)";
    if (uses_kT(op) || uses_law(op)) return nullptr;  // block kernel through the map
    return op.coef64_ok ? nullptr : "the coefficient stream is not built yet: call mpdg_vmult once first";
  }
  if (uses_law(op)) return nullptr;  // block kernel on raw geometry
  if (!full && !m.uniform && !op.coef64_ok)
    return "the coefficient stream is not built yet: call mpdg_vmult once first";
  return nullptr;  // nothing is built lazily on the other paths
}

}  // namespace mpdg

namespace mpdg {

// per-cell integrated L2 norm squared (one thread per cell), summed per block
template <int P>
__global__ void l2_cells_kernel(const double *u, long NX, long NY, int nc0, int nc1, long n_cells,
                                const Colour *colours, const int *cmap, const double *metric, double hx,
                                double hy, double hz, double *partial)
{
  constexpr int n = P + 1, n3 = n * n * n;
  const Tables<double> &T = tab<double>(P);
  double s = 0.0;
  for (long cell = (long)blockIdx.x * blockDim.x + threadIdx.x; cell < n_cells;
       cell += (long)gridDim.x * blockDim.x) {
    double a[n3], b[n3];
    if (cmap) {
      // mapped mesh: the cell's DoFs through its cell->DoF map
      for (int t = 0; t < n3; ++t) a[t] = u[cmap[cell * n3 + t]];
    } else {
      int c = 0;
      while (c < 7 && cell >= colours[c + 1].first) ++c;
      const Colour &C = colours[c];
      const long cidx = cell - C.first;
      const int ix = 2 * (int)(cidx % C.cn[0]) + C.par[0];
      const int iy = 2 * (int)((cidx / C.cn[0]) % C.cn[1]) + C.par[1];
      const int iz = 2 * (int)(cidx / ((long)C.cn[0] * C.cn[1])) + C.par[2];
      for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
          for (int i = 0; i < n; ++i)
            a[(k * n + j) * n + i] = u[((long)(iz * P + k) * NY + (iy * P + j)) * NX + (ix * P + i)];
    }
    // x, y, z interpolation to the Gauss points
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        for (int q = 0; q < n; ++q) {
          double t = 0;
          for (int i = 0; i < n; ++i) t += T.S[q * n + i] * a[(k * n + j) * n + i];
          b[(k * n + j) * n + q] = t;
        }
    for (int k = 0; k < n; ++k)
      for (int q = 0; q < n; ++q)
        for (int i = 0; i < n; ++i) {
          double t = 0;
          for (int j = 0; j < n; ++j) t += T.S[q * n + j] * b[(k * n + j) * n + i];
          a[(k * n + q) * n + i] = t;
        }
    for (int q = 0; q < n; ++q)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          double t = 0;
          for (int k = 0; k < n; ++k) t += T.S[q * n + k] * a[(k * n + j) * n + i];
          b[(q * n + j) * n + i] = t;
        }
    for (int q = 0; q < n3; ++q) {
      const int qi = q % n, qj = (q / n) % n, qk = q / (n * n);
      const double JxW = metric ? metric[cell * metric_stride(n) + q] : hx * hy * hz * T.w[qi] * T.w[qj] * T.w[qk];
      s += b[q] * b[q] * JxW;
    }
  }
  __shared__ double ws[256];
  ws[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) ws[threadIdx.x] += ws[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = ws[0];
}

double l2_norm_integrated(Op &op, const double *u)
{
  if (op.fine) throw Error{MPDG_ERR_UNSUPPORTED, "integrated norms on two-level meshes"};
  Mesh &m = *op.mesh;
  const int blocks = 256;
  Colour *d_col = nullptr;
  double *partial = nullptr;
  MPDG_CUDA(tracked_malloc(&d_col, sizeof(m.colour)));
  MPDG_CUDA(cudaMemcpy(d_col, m.colour, sizeof(m.colour), cudaMemcpyHostToDevice));
  MPDG_CUDA(tracked_malloc(&partial, sizeof(double) * blocks));
  const double *met = m.uniform ? nullptr : m.d_metric64;
  switch (m.degree) {
    case 1: l2_cells_kernel<1><<<blocks, 256, 0, op.stream>>>(u, m.NX, m.NY, m.nc[0], m.nc[1], m.n_cells, d_col, m.d_cmap, met, m.h[0], m.h[1], m.h[2], partial); break;
    case 2: l2_cells_kernel<2><<<blocks, 256, 0, op.stream>>>(u, m.NX, m.NY, m.nc[0], m.nc[1], m.n_cells, d_col, m.d_cmap, met, m.h[0], m.h[1], m.h[2], partial); break;
    case 3: l2_cells_kernel<3><<<blocks, 256, 0, op.stream>>>(u, m.NX, m.NY, m.nc[0], m.nc[1], m.n_cells, d_col, m.d_cmap, met, m.h[0], m.h[1], m.h[2], partial); break;
    case 4: l2_cells_kernel<4><<<blocks, 256, 0, op.stream>>>(u, m.NX, m.NY, m.nc[0], m.nc[1], m.n_cells, d_col, m.d_cmap, met, m.h[0], m.h[1], m.h[2], partial); break;
    default: throw Error{MPDG_ERR_UNSUPPORTED, "degree must be 1..4"};
  }
  MPDG_LAUNCHED();
  std::vector<double> h(blocks);
  MPDG_CUDA(cudaMemcpyAsync(h.data(), partial, sizeof(double) * blocks, cudaMemcpyDeviceToHost, op.stream));
  MPDG_CUDA(cudaStreamSynchronize(op.stream));
  cudaFree(partial);
  cudaFree(d_col);
  double s = 0.0;
  for (double v : h) s += v;
  return std::sqrt(s);
}

}  // namespace mpdg

namespace mpdg {

int cells_per_warp(int degree)
{
  switch (degree) {
    case 1: return WCfg<2>::cpw;
    case 2: return WCfg<3>::cpw;
    case 3: return WCfg<4>::cpw;
    case 4: return WCfg<5>::cpw;
    default: return 1;
  }
}

namespace {
template <typename Real, int WPC, bool TUNED>
int batch_occupancy()
{
  static int blocks_per_sm = 0;
  if (!blocks_per_sm) {
    upload_tables();
    MPDG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, batch_apply_kernel<Real, WPC, TUNED>,
                                                            WPC * 32, 0));
    if (blocks_per_sm < 1) blocks_per_sm = 1;
  }
  return blocks_per_sm;
}

template <typename Real, int WPC, bool TUNED>
void launch_batch_shape(const BatchSchedule &sched, const SlotInfo *info, const BatchSlotParams *params,
                        Real *const *src, Real *const *dst, const int *mask, int cap, cudaStream_t s)
{
  const int occ = batch_occupancy<Real, WPC, TUNED>();  // tables uploaded before any launch (and capture)
  const int blocks = num_sms() * ((cap > 0) ? std::min(cap, occ) : occ);
  for (int c = 0; c < 8; ++c) {
    batch_apply_kernel<Real, WPC, TUNED><<<(unsigned)blocks, WPC * 32, 0, s>>>(
        c, sched.hdr, sched.seg_slot + (size_t)c * sched.cap, sched.seg_prefix + (size_t)c * sched.cap, info,
        params, src, dst, mask);
    MPDG_LAUNCHED();
  }
}

template <typename Real>
void batch_setup_all()
{
  batch_occupancy<Real, 2, true>();
  batch_occupancy<Real, 4, true>();
  batch_occupancy<Real, 8, true>();
  batch_occupancy<Real, 2, false>();
  batch_occupancy<Real, 4, false>();
  batch_occupancy<Real, 8, false>();
}
}  // namespace

void batch_apply_setup()
{
  batch_setup_all<float>();
  batch_setup_all<double>();
}

template <typename Real>
void launch_batch_apply(const BatchSchedule &sched, const SlotInfo *info, const BatchSlotParams *params,
                        Real *const *src, Real *const *dst, const int *mask, const BatchShape &shape,
                        cudaStream_t s)
{
  const int cap = shape.ctas_per_sm;
  switch (shape.warps_per_cta * 2 + (shape.tuned_tiles ? 1 : 0)) {
    case 4: launch_batch_shape<Real, 2, false>(sched, info, params, src, dst, mask, cap, s); break;
    case 5: launch_batch_shape<Real, 2, true>(sched, info, params, src, dst, mask, cap, s); break;
    case 8: launch_batch_shape<Real, 4, false>(sched, info, params, src, dst, mask, cap, s); break;
    case 9: launch_batch_shape<Real, 4, true>(sched, info, params, src, dst, mask, cap, s); break;
    case 16: launch_batch_shape<Real, 8, false>(sched, info, params, src, dst, mask, cap, s); break;
    case 17: launch_batch_shape<Real, 8, true>(sched, info, params, src, dst, mask, cap, s); break;
    default: throw Error{MPDG_ERR_ARG, "batched apply: warps per CTA must be 2, 4 or 8"};
  }
}
template void launch_batch_apply<double>(const BatchSchedule &, const SlotInfo *, const BatchSlotParams *,
                                         double *const *, double *const *, const int *, const BatchShape &,
                                         cudaStream_t);
template void launch_batch_apply<float>(const BatchSchedule &, const SlotInfo *, const BatchSlotParams *,
                                        float *const *, float *const *, const int *, const BatchShape &,
                                        cudaStream_t);

}  // namespace mpdg
