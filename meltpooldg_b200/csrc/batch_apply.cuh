// Batched operator apply over many independent solves (included by
// operator_kernels.cu).  One launch per colour covers that colour's cells of
// every scheduled solve, of any degree: the device schedule (rebuilt every
// Krylov step from the solves' running flags) lists the solves with cells of
// the colour and the prefix of their warp groups; persistent warps walk the
// group index, find their solve by binary search in the prefix and apply the
// cell with that solve's degree (a warp-uniform switch into the templated cell
// body) and parameters.  Converged solves are not in the schedule and cost
// nothing.  Meshes are uniform boxes (unit cube, nc^3 cells), so there is no
// coefficient stream; homogeneous Dirichlet on all faces is evaluated from the
// DoF index.  Same warp-per-cell contraction scheme and first-touch scatter as
// warp_apply_kernel.
#pragma once

#include <type_traits>

constexpr int kBatchTileElems = 320;   // at least the largest warp_tile_elems over P

__device__ __forceinline__ int batch_find(const int *__restrict__ prefix, int n, int g)
{
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (prefix[mid] <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// what a warp needs of the solve whose groups it is walking, for one colour;
// cached in shared memory and reloaded only when the warp crosses into the
// next solve's segment
template <typename Real>
struct WarpSlot {
  const Real *src;
  Real *dst;
  long NX;
  unsigned long long m0, m01;
  double c_mass, c_vel, c_diff, hvol, ih, ih2, h;
  int ok, degree, nc, count, cn0, cn1, vel_kind, dirichlet;
};

template <typename Real>
__device__ __forceinline__ void load_warp_slot(WarpSlot<Real> &W, int colour, int s, const SlotInfo *info,
                                               const BatchSlotParams *params, Real *const *src_ptrs,
                                               Real *const *dst_ptrs, const int *mask, int lane)
{
  if (lane == 0) {
    const SlotInfo &I = info[s];
    const SlotColour &C = I.col[colour];
    const BatchSlotParams &Q = params[s];
    W.src = src_ptrs[s];
    W.dst = dst_ptrs[s];
    W.NX = I.NX;
    W.m0 = C.m0;
    W.m01 = C.m01;
    W.c_mass = Q.c_mass;
    W.c_vel = Q.c_vel;
    W.c_diff = Q.c_diff;
    W.hvol = Q.hvol;
    W.ih = Q.ih;
    W.ih2 = Q.ih2;
    W.h = Q.h;
    W.ok = mask[s];
    W.degree = I.degree;
    W.nc = I.nc;
    W.count = C.count;
    W.cn0 = C.cn0;
    W.cn1 = C.cn1;
    W.vel_kind = Q.vel_kind;
    W.dirichlet = Q.dirichlet;
  }
  __syncwarp();
}

// cell of colour-local group lg and the lane's position in it
template <int P>
struct BatchLanePos {
  bool lane_ok, act, gact, bxy;  // gact: gathers (idle lanes copy their mirror lane)
  int i, j, s_sub, ix, iy, iz;
  long NX, g0;
};

template <int P, typename Real>
__device__ __forceinline__ BatchLanePos<P> batch_pos(int colour, int lg, const WarpSlot<Real> &W, int lane)
{
  constexpr int n = P + 1, n2 = n * n, CPW = WCfg<n>::cpw;
  BatchLanePos<P> q;
  // idle lanes copy an active lane of their own half-warp (see warp_apply_kernel)
  q.lane_ok = lane < CPW * n2;
  const int mlane = q.lane_ok ? lane : lane - (32 - CPW * n2);
  const int sub = mlane / n2, l = mlane % n2;
  q.i = l % n;
  q.j = l / n;
  q.s_sub = sub;
  const int cidx = lg * CPW + sub;
  q.gact = cidx < W.count;
  q.act = q.lane_ok && q.gact;
  q.ix = q.iy = q.iz = 0;
  if (q.gact) {
    const unsigned x = (unsigned)cidx;
    const unsigned q0 = (unsigned)(((unsigned long long)x * W.m0) >> 40);
    const unsigned q01 = (unsigned)(((unsigned long long)x * W.m01) >> 40);
    q.ix = 2 * (int)(x - q0 * (unsigned)W.cn0) + (colour & 1);
    q.iy = 2 * (int)(q0 - q01 * (unsigned)W.cn1) + ((colour >> 1) & 1);
    q.iz = 2 * (int)q01 + ((colour >> 2) & 1);
  }
  q.NX = W.NX;
  const int X = q.ix * P + q.i, Y = q.iy * P + q.j;
  q.g0 = ((long)(q.iz * P) * q.NX + Y) * q.NX + X;
  q.bxy = W.dirichlet && (X == 0 || X == q.NX - 1 || Y == 0 || Y == q.NX - 1);
  return q;
}

// the lane's src column of the cell (zero at Dirichlet DoFs); only loads, so
// the values stay in flight while the previous group computes
template <int P, typename Real>
__device__ __forceinline__ void batch_gather(int colour, int lg, const WarpSlot<Real> &W, int lane,
                                             Real (&u)[kMaxN])
{
  constexpr int n = P + 1;
  const BatchLanePos<P> q = batch_pos<P>(colour, lg, W, lane);
  const long zs = q.NX * q.NX;
  const Real *src = W.src;
  const bool dir = W.dirichlet;
#pragma unroll
  for (int k = 0; k < n; ++k) {
    const int Z = q.iz * P + k;
    const bool masked = q.bxy || (dir && (Z == 0 || Z == q.NX - 1));
    u[k] = (q.gact && !masked) ? src[q.g0 + k * zs] : Real(0);
  }
}

// TUNED: the conflict-minimal tile layouts of the warp apply, else the plain one
template <int P, typename Real, bool TUNED>
__device__ __forceinline__ void batch_cell(int colour, int local_group, const WarpSlot<Real> &W,
                                           const Real (&uin)[kMaxN], Real *tiles, int lane)
{
  constexpr int n = P + 1;
  using L = typename std::conditional<TUNED, TileLayout<n, Real, 32>, PlainTileLayout<n, Real>>::type;
  static_assert(L::elems <= kBatchTileElems, "tile area");
  const Tables<Real> &T = tab<Real>(P);
  const BatchLanePos<P> q = batch_pos<P>(colour, local_group, W, lane);
  const int i = q.i, j = q.j, ix = q.ix, iy = q.iy, iz = q.iz;
  Real *t0 = tiles + q.s_sub * L::sc0;
  Real *t1 = tiles + L::t0_elems + q.s_sub * L::sc1;
  const long NX = q.NX, zs = NX * NX, g0 = q.g0;
  Real *dst = W.dst;
  const bool dir = W.dirichlet;
  // store-or-add decision and the early loads of the values to add to
  const int nc = W.nc;
  const bool sx = (i == 0 && ix > 0) || (i == P && ix < nc - 1);
  const bool sy = (j == 0 && iy > 0) || (j == P && iy < nc - 1);
  const bool later_xy = (sx && (ix & 1)) || (sy && (iy & 1));
  unsigned first_bits = 0, mask_bits = 0;
  Real dpre[n];
#pragma unroll
  for (int k = 0; k < n; ++k) {
    const int Z = iz * P + k;
    const bool sz = (k == 0 && iz > 0) || (k == P && iz < nc - 1);
    const bool first = !(later_xy || (sz && (iz & 1)));
    const bool masked = q.bxy || (dir && (Z == 0 || Z == NX - 1));
    first_bits |= (unsigned)first << k;
    mask_bits |= (unsigned)masked << k;
    dpre[k] = (q.act && !first && !masked) ? dst[g0 + k * zs] : Real(0);
  }
  Real u[n];
#pragma unroll
  for (int k = 0; k < n; ++k) u[k] = uin[k];
  Real uq[n], gx[n], gy[n], gz[n];
  l_forward<n, Real, L, false>(T, t0, t1, true, i, j, u, uq, gx, gy, gz);
  Real val[n], fx[n], fy[n], fz[n];
  const Real hvol = (Real)W.hvol, ih = (Real)W.ih, ih2 = (Real)W.ih2;
  const Real c_mass = (Real)W.c_mass, c_vel = (Real)W.c_vel, c_diff = (Real)W.c_diff;
  Real b0f = 0, b1f = 0;
  if (W.vel_kind == MPDG_VEL_VORTEX) {
    Real sxv, cxv, syv, cyv;
    const Real xq = ((Real)ix + T.x[i]) * (Real)W.h, yq = ((Real)iy + T.x[j]) * (Real)W.h;
    sincospi(xq, &sxv, &cxv);
    sincospi(yq, &syv, &cyv);
    b0f = c_vel * ih * sxv * cyv;
    b1f = -c_vel * ih * cxv * syv;
  }
  const Real wij = hvol * T.w[i] * T.w[j];
#pragma unroll
  for (int k = 0; k < n; ++k) {
    const Real JxW = wij * T.w[k];
    val[k] = JxW * (c_mass * uq[k] + b0f * gx[k] + b1f * gy[k]);
    const Real kd = c_diff * JxW * ih2;
    fx[k] = kd * gx[k];
    fy[k] = kd * gy[k];
    fz[k] = kd * gz[k];
  }
  Real out[n];
  l_backward<n, Real, L, false>(T, t0, t1, true, i, j, val, fx, fy, fz, out);
  if (q.act) {
#pragma unroll
    for (int k = 0; k < n; ++k) {
      const long gg = g0 + k * zs;
      if ((first_bits >> k) & 1) dst[gg] = ((mask_bits >> k) & 1) ? Real(0) : out[k];
      else if (!((mask_bits >> k) & 1)) dst[gg] = dpre[k] + out[k];
    }
  }
}

template <typename Real, int WPC>
struct BatchOcc {  // register budget: 16 (FP32) or 12 (FP64) resident warps per SM
  static constexpr int warps = sizeof(Real) == 8 ? 12 : 16;
  static constexpr int min_blocks = warps / WPC > 0 ? warps / WPC : 1;
};

// WPC warps per CTA and the tile layout (TUNED) are the block and tile shapes
// the batch's autotuner picks from (mpdg_batch_autotune)
template <typename Real, int WPC, bool TUNED>
__global__ void __launch_bounds__(WPC * 32, BatchOcc<Real, WPC>::min_blocks)
    batch_apply_kernel(int colour, const BatchScheduleHeader *__restrict__ hdr,
                       const int *__restrict__ seg_slot, const int *__restrict__ seg_prefix,
                       const SlotInfo *__restrict__ info, const BatchSlotParams *__restrict__ params,
                       Real *const *__restrict__ src_ptrs, Real *const *__restrict__ dst_ptrs,
                       const int *__restrict__ mask)
{
  __shared__ Real tiles_all[WPC][kBatchTileElems];
  __shared__ WarpSlot<Real> wslot[WPC][2];
  const int total = hdr->total_groups[colour], nseg = hdr->n_seg[colour];
  if (total == 0) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  Real *tiles = tiles_all[warp];
  // each warp walks a contiguous range of groups: one binary search per launch,
  // then the segment index only advances (neighbouring groups are neighbouring
  // cells of the same solve)
  const int nwarps = gridDim.x * WPC, wid = blockIdx.x * WPC + warp;
  const int per = (total + nwarps - 1) / nwarps;
  const int gbeg = min(total, wid * per), gend = min(total, gbeg + per);
  if (gbeg >= gend) return;
  int kseg = batch_find(seg_prefix, nseg, gbeg);
  int buf = 0;
  load_warp_slot(wslot[warp][buf], colour, seg_slot[kseg], info, params, src_ptrs, dst_ptrs, mask, lane);
  auto gather = [&](int lg, const WarpSlot<Real> &W, Real (&u)[kMaxN]) {
    if (!W.ok) return;
    switch (W.degree) {
      case 1: batch_gather<1, Real>(colour, lg, W, lane, u); break;
      case 2: batch_gather<2, Real>(colour, lg, W, lane, u); break;
      case 3: batch_gather<3, Real>(colour, lg, W, lane, u); break;
      default: batch_gather<4, Real>(colour, lg, W, lane, u); break;
    }
  };
  int g = gbeg, lg = gbeg - seg_prefix[kseg];
  int next_start = (kseg + 1 < nseg) ? seg_prefix[kseg + 1] : total;
  Real u[kMaxN];
  gather(lg, wslot[warp][buf], u);
  while (g < gend) {
    // next group's column first: its loads overlap this group's computation
    const int gn = g + 1;
    int bn = buf, lgn = lg + 1;
    Real un[kMaxN];
    if (gn < gend) {
      if (gn >= next_start) {  // the next group starts the next solve's segment
        while (kseg + 1 < nseg && seg_prefix[kseg + 1] <= gn) ++kseg;
        next_start = (kseg + 1 < nseg) ? seg_prefix[kseg + 1] : total;
        bn = buf ^ 1;
        load_warp_slot(wslot[warp][bn], colour, seg_slot[kseg], info, params, src_ptrs, dst_ptrs, mask, lane);
        lgn = gn - seg_prefix[kseg];
      }
      gather(lgn, wslot[warp][bn], un);
    }
    const WarpSlot<Real> &W = wslot[warp][buf];
    if (W.ok) {
      switch (W.degree) {
        case 1: batch_cell<1, Real, TUNED>(colour, lg, W, u, tiles, lane); break;
        case 2: batch_cell<2, Real, TUNED>(colour, lg, W, u, tiles, lane); break;
        case 3: batch_cell<3, Real, TUNED>(colour, lg, W, u, tiles, lane); break;
        default: batch_cell<4, Real, TUNED>(colour, lg, W, u, tiles, lane); break;
      }
    }
    __syncwarp();  // the slot buffer of this group may be reloaded for the group after next
    g = gn;
    lg = lgn;
    buf = bn;
#pragma unroll
    for (int k = 0; k < kMaxN; ++k) u[k] = un[k];
  }
}
