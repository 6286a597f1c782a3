// Lane-per-cell operator apply for low degrees (Q1, Q2) on uniform lattices
// with constant coefficients (the vmult of heat_diffuse_operator.cpp:179-197
// and advection_diffusion_operator.cpp:238-272 on an axis-aligned box).
// Included by operator_kernels.cu after apply_warp.cuh.
//
// Why a second apply for these degrees: a Q2 cell has 27 DoFs, so its whole
// sum factorisation fits in one thread's registers.  The warp apply spends
// most of its time exchanging lines through shared memory (the l1tex pipe);
// here every contraction is a register FMA with a constant-bank operand and
// shared memory is not used at all.
//
// Layout and schedule:
//  * the 32 lanes of a warp own 32 consecutive cells of one x-row of cells
//    (an x-segment); the x-face a lane shares with the next lane is added into
//    that lane's column by one warp shuffle per face DoF, so x-neighbours
//    inside a segment need no colouring and every such DoF is written once;
//  * launches are coloured by x-segment parity and the y and z cell parities
//    (8 colours, 4 when a row has a single segment), run in that order with
//    the first-touch rule of the warp apply: the cell whose parity bits are
//    zero in all directions in which a DoF is shared stores it, later colours
//    add.  A colour touches half of the x-segments, so the DoF vectors' lines
//    are read about half as often as under cell-parity colours;
//  * per cell: values at the Gauss points (z, x, y sweeps), then per direction
//    the collocation gradient of every line, its diffusion flux and advection
//    term, and the transposed gradient; then the test-function sweeps back to
//    the nodes.  Registers: two 27-value arrays (values, residual).
//  * colour launches after the first are programmatic dependents of the one
//    before: gathers and arithmetic overlap the previous colour's tail, reads
//    of dst wait for it (griddepcontrol.wait).

constexpr int kLaneSeg = 32;  // cells of an x-segment: the lanes of a warp
constexpr int kLaneN2 = 9, kLaneN3 = 27;  // tables sized for Q2

// one colour launch of the lane apply
struct LaneColour {
  int sx, py, pz;  // x-segment parity, y and z cell parities
  int nsx;         // segments of parity sx per row of cells
  int cny;         // cell rows of parity py per z-layer
  int zi0;         // first z index of this launch: iz = 2 (zi0 + zi) + pz
  long nwarps;     // segments (= warps) of this launch
  // the mesh's parity colours: colour-major index of a cell's Dirichlet mask
  long pfirst[8];
  int pcn0[8], pcn1[8];
};

// velocity kinds the lane apply evaluates in-kernel
enum { LANE_VEL_NONE = 0, LANE_VEL_CONST = 1, LANE_VEL_VORTEX = 2, LANE_VEL_ROTATION = 3 };

// resident CTAs of 128 threads per SM the register allocation is bounded for:
// OCC = 0 gives a Q2 cell's sum factorisation registers enough not to spill
// (FP64 166, FP32 96 registers); OCC = 1 trades a few spilled values for one
// more resident CTA per SM (FP64 128, FP32 80 registers)
template <int P, typename Real, int OCC>
struct LaneOcc {
  static constexpr int min_blocks =
      (sizeof(Real) == 8) ? (P == 2 ? (OCC ? 4 : 3) : 6) : (P == 2 ? (OCC ? 6 : 5) : 8);
};

// per-quadrature-point coefficients of a uniform lattice, the same for every
// cell (JxW = hvol w_x w_y w_z, J^-1 = diag(1/h)), kernel parameters so that
// every product reads a constant-bank operand
template <typename Real>
struct LaneCoef {
  Real mass[kLaneN3];     // c_mass JxW
  Real diff[3][kLaneN3];  // c_diff JxW / h_d^2
  Real adv[3][kLaneN3];   // c_vel JxW / h_d times the constant factor of u_d
  Real line[3][kLaneN2];  // c_diff hvol / h_d^2 times the weights off the line
  Real K[kLaneN2];        // Dc^T diag(w) Dc
};

template <int P, typename Real, int VK, int OCC>
__global__ void __launch_bounds__(128, LaneOcc<P, Real, OCC>::min_blocks)
    lane_apply_kernel(const KP<Real> p, const LaneColour lc, const LaneCoef<Real> c)
{
  constexpr int n = P + 1, n2 = n * n, n3 = n2 * n;
  static_assert(n3 <= 32, "the lane apply keeps one 32-bit Dirichlet mask word per cell");
  static_assert(n3 <= kLaneN3, "coefficient tables sized for Q2");
  const Tables<Real> &T = tab<Real>(P);
  if (p.pdl) grid_dep_launch_dependents();
  const long w = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (w >= lc.nwarps) return;  // whole warps only: the shuffles below need all 32 lanes
  const int lane = threadIdx.x & 31;
  const int sxi = (int)(w % lc.nsx);
  const long r = w / lc.nsx;
  const int yi = (int)(r % lc.cny), zi = (int)(r / lc.cny) + lc.zi0;
  const int ix = (2 * sxi + lc.sx) * kLaneSeg + lane, iy = 2 * yi + lc.py, iz = 2 * zi + lc.pz;
  // lanes past the end of the row take part in the shuffles with a zero cell
  const bool act = ix < p.nc[0];
  const int ixc = act ? ix : p.nc[0] - 1;
  const unsigned NXu = (unsigned)p.NX, NYu = (unsigned)p.NY, zs = NXu * NYu;
  const unsigned g0 = ((unsigned)(iz * P) * NYu + (unsigned)(iy * P)) * NXu + (unsigned)(ixc * P);

  // constrained DoFs of the cell (bit (k n + j) n + i)
  unsigned rmask = 0u, wmask = 0u;
  if (p.cell_mask && (p.masked_read || p.masked_write) && act) {
    const int pc = (ix & 1) + 2 * (iy & 1) + 4 * (iz & 1);
    const long ci = lc.pfirst[pc] + ((long)(iz >> 1) * lc.pcn1[pc] + (iy >> 1)) * lc.pcn0[pc] + (ix >> 1);
    const unsigned bits = p.cell_mask[ci].x;
    rmask = p.masked_read ? bits : 0u;
    wmask = p.masked_write ? bits : 0u;
  }

  // gather: u[(k n + j) n + i] = src at DoF (i, j, k) of the cell
  Real u[n3];
#pragma unroll
  for (int k = 0; k < n; ++k)
#pragma unroll
    for (int j = 0; j < n; ++j)
#pragma unroll
      for (int i = 0; i < n; ++i) {
        const int q = (k * n + j) * n + i;
        u[q] = (act && !((rmask >> q) & 1u)) ? __ldg(p.src + g0 + k * zs + j * NXu + i) : Real(0);
      }

  // values at the Gauss points: S along z, x, y (in place)
#pragma unroll
  for (int j = 0; j < n; ++j)
#pragma unroll
    for (int i = 0; i < n; ++i) {
      Real a[n], b[n];
#pragma unroll
      for (int k = 0; k < n; ++k) a[k] = u[(k * n + j) * n + i];
      cz<n, Real, false>(T.S, a, b);
#pragma unroll
      for (int k = 0; k < n; ++k) u[(k * n + j) * n + i] = b[k];
    }
#pragma unroll
  for (int k = 0; k < n; ++k)
#pragma unroll
    for (int j = 0; j < n; ++j) {
      Real a[n], b[n];
#pragma unroll
      for (int i = 0; i < n; ++i) a[i] = u[(k * n + j) * n + i];
      cz<n, Real, false>(T.S, a, b);
#pragma unroll
      for (int i = 0; i < n; ++i) u[(k * n + j) * n + i] = b[i];
    }
#pragma unroll
  for (int k = 0; k < n; ++k)
#pragma unroll
    for (int i = 0; i < n; ++i) {
      Real a[n], b[n];
#pragma unroll
      for (int j = 0; j < n; ++j) a[j] = u[(k * n + j) * n + i];
      cz<n, Real, false>(T.S, a, b);
#pragma unroll
      for (int j = 0; j < n; ++j) u[(k * n + j) * n + i] = b[j];
    }

  // velocity factors at the Gauss coordinates of the cell: vx0, vx1 along x,
  // vy0, vy1 along y, vz along z.  Vortex: u = (sin(pi x) cos(pi y),
  // -cos(pi x) sin(pi y), 0) from the trigonometric table; rotation:
  // u = (w z, 0, -w x) (w folded into the advection table)
  Real vx0[n], vx1[n], vy0[n], vy1[n], vz[n];
#pragma unroll
  for (int q = 0; q < n; ++q) {
    vx0[q] = vx1[q] = vy0[q] = vy1[q] = vz[q] = Real(0);
    if constexpr (VK == LANE_VEL_VORTEX) {
      vx0[q] = p.trig[ixc * n + q];                        // sin(pi x)
      vx1[q] = p.trig[p.trig_stride + ixc * n + q];        // cos(pi x)
      vy0[q] = p.trig[2 * p.trig_stride + iy * n + q];     // sin(pi y)
      vy1[q] = p.trig[3 * p.trig_stride + iy * n + q];     // cos(pi y)
    } else if constexpr (VK == LANE_VEL_ROTATION) {
      vx0[q] = p.origin[0] + (ixc + T.x[q]) * p.h[0];
      vz[q] = p.origin[2] + (iz + T.x[q]) * p.h[2];
    }
  }
  // velocity component d at Gauss point (qx, qy, qz), without the factors the
  // advection table holds (a constant velocity, the rotation rate and sign)
  auto vel = [&](int d, int qx, int qy, int qz) -> Real {
    if constexpr (VK == LANE_VEL_VORTEX) return d == 0 ? vx0[qx] * vy1[qy] : vx1[qx] * vy0[qy];
    else if constexpr (VK == LANE_VEL_ROTATION) return d == 0 ? vz[qz] : vx0[qx];
    else return Real(1);
  };

  // residual at the Gauss points: mass term, then per direction the
  // advection term b_d g_d and the transposed collocation derivative of the
  // diffusion flux, line by line.  Directions without advection apply the
  // line stiffness K = Dc^T diag(w) Dc to the values at once.
  Real R[n3];
#pragma unroll
  for (int q = 0; q < n3; ++q) R[q] = c.mass[q] * u[q];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    // directions in which the velocity vanishes identically carry no advection term
    const bool adv = VK != LANE_VEL_NONE && !(VK == LANE_VEL_VORTEX && d == 2) && !(VK == LANE_VEL_ROTATION && d == 1);
#pragma unroll
    for (int a = 0; a < n; ++a)
#pragma unroll
      for (int b = 0; b < n; ++b) {
        // line along d through the other two indices (a, b)
        int idx[n];
#pragma unroll
        for (int t = 0; t < n; ++t)
          idx[t] = d == 0 ? (b * n + a) * n + t : d == 1 ? (b * n + t) * n + a : (t * n + b) * n + a;
        Real line[n], back[n];
#pragma unroll
        for (int t = 0; t < n; ++t) line[t] = u[idx[t]];
        if (adv) {
          Real g[n], f[n];
          cz<n, Real, false>(T.Dc, line, g);
#pragma unroll
          for (int t = 0; t < n; ++t) {
            const int q = idx[t];
            const int qx = q % n, qy = (q / n) % n, qz = q / n2;
            f[t] = c.diff[d][q] * g[t];
            R[q] += (c.adv[d][q] * vel(d, qx, qy, qz)) * g[t];
          }
          cz<n, Real, true>(T.Dc, f, back);
#pragma unroll
          for (int t = 0; t < n; ++t) R[idx[t]] += back[t];
        } else {
          cz<n, Real, false>(c.K, line, back);
#pragma unroll
          for (int t = 0; t < n; ++t) R[idx[t]] += c.line[d][b * n + a] * back[t];
        }
      }
  }

  // test functions: S^T along y, x, z (in place on R)
#pragma unroll
  for (int k = 0; k < n; ++k)
#pragma unroll
    for (int i = 0; i < n; ++i) {
      Real a[n], b[n];
#pragma unroll
      for (int j = 0; j < n; ++j) a[j] = R[(k * n + j) * n + i];
      cz<n, Real, true>(T.S, a, b);
#pragma unroll
      for (int j = 0; j < n; ++j) R[(k * n + j) * n + i] = b[j];
    }
#pragma unroll
  for (int k = 0; k < n; ++k)
#pragma unroll
    for (int j = 0; j < n; ++j) {
      Real a[n], b[n];
#pragma unroll
      for (int i = 0; i < n; ++i) a[i] = R[(k * n + j) * n + i];
      cz<n, Real, true>(T.S, a, b);
#pragma unroll
      for (int i = 0; i < n; ++i) R[(k * n + j) * n + i] = b[i];
    }
#pragma unroll
  for (int j = 0; j < n; ++j)
#pragma unroll
    for (int i = 0; i < n; ++i) {
      Real a[n], b[n];
#pragma unroll
      for (int k = 0; k < n; ++k) a[k] = R[(k * n + j) * n + i];
      cz<n, Real, true>(T.S, a, b);
#pragma unroll
      for (int k = 0; k < n; ++k) R[(k * n + j) * n + i] = b[k];
    }

  // x-neighbours inside the segment: lane l adds lane l-1's i = P face into
  // its i = 0 face (lane l-1 is active whenever lane l is)
#pragma unroll
  for (int k = 0; k < n; ++k)
#pragma unroll
    for (int j = 0; j < n; ++j) {
      const Real v = __shfl_up_sync(0xffffffffu, R[(k * n + j) * n + P], 1);
      if (lane > 0) R[(k * n + j) * n] += v;
    }
  if (!act) return;

  // first-touch scatter.  Lane l writes its faces i < P; the i = P face only at
  // the end of the segment or of the row.  A DoF shared with another launch is
  // stored by the launch whose parities are zero in the shared directions and
  // added to by the others (odd segments and odd cell rows / layers add).
  const bool xend = lane == kLaneSeg - 1 || ix == p.nc[0] - 1;
  const bool odd_seg = lc.sx != 0;
  unsigned first_bits = 0u, write_bits = 0u;
#pragma unroll
  for (int k = 0; k < n; ++k)
#pragma unroll
    for (int j = 0; j < n; ++j)
#pragma unroll
      for (int i = 0; i < n; ++i) {
        const int q = (k * n + j) * n + i;
        const bool wr = i < P || xend;
        const bool xl = odd_seg && ((i == 0 && lane == 0 && ix > 0) || (i == P && lane == kLaneSeg - 1 && ix < p.nc[0] - 1));
        const bool yl = (iy & 1) && ((j == 0 && iy > 0) || (j == P && iy < p.nc[1] - 1));
        const bool zl = (iz & 1) && ((k == 0 && iz > 0) || (k == P && iz < p.nc[2] - 1));
        first_bits |= (unsigned)!(xl || yl || zl) << q;
        write_bits |= (unsigned)wr << q;
      }
  if (p.pdl) grid_dep_wait();
  Real dpre[n3];
#pragma unroll
  for (int k = 0; k < n; ++k)
#pragma unroll
    for (int j = 0; j < n; ++j)
#pragma unroll
      for (int i = 0; i < n; ++i) {
        const int q = (k * n + j) * n + i;
        const bool add = ((write_bits >> q) & 1u) && !((first_bits >> q) & 1u) && !((wmask >> q) & 1u);
        dpre[q] = add ? p.dst[g0 + k * zs + j * NXu + i] : Real(0);
      }
#pragma unroll
  for (int k = 0; k < n; ++k)
#pragma unroll
    for (int j = 0; j < n; ++j)
#pragma unroll
      for (int i = 0; i < n; ++i) {
        const int q = (k * n + j) * n + i;
        if (!((write_bits >> q) & 1u)) continue;
        const bool first = (first_bits >> q) & 1u, masked = (wmask >> q) & 1u;
        Real *d = p.dst + g0 + k * zs + j * NXu + i;
        if (first) *d = masked ? Real(0) : R[q];
        else if (!masked) *d = dpre[q] + R[q];
      }
}
