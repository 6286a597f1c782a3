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

constexpr int kBatchTileElems = 256;   // max over P of 2 * cells_per_warp * (P+1)^3

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

template <int P, typename Real>
__device__ __forceinline__ void batch_cell(int colour, int local_group, const SlotInfo &I,
                                           const BatchSlotParams &Q, const Real *__restrict__ src,
                                           Real *__restrict__ dst, Real *tiles, int lane)
{
  constexpr int n = P + 1, n2 = n * n, n3 = n2 * n, CPW = WCfg<n>::cpw;
  static_assert(2 * CPW * n3 <= kBatchTileElems, "tile area");
  const Tables<Real> &T = tab<Real>(P);
  const int sub = lane / n2, l = lane % n2, i = l % n, j = l / n;
  const bool lane_ok = sub < CPW;
  const int s_sub = lane_ok ? sub : 0;
  Real *t0 = tiles + s_sub * n3;
  Real *t1 = tiles + (CPW + s_sub) * n3;
  const SlotColour &C = I.col[colour];
  const int par0 = colour & 1, par1 = (colour >> 1) & 1, par2 = (colour >> 2) & 1;
  const int cidx = local_group * CPW + sub;
  const bool act = lane_ok && cidx < C.count;
  int ix = 0, iy = 0, iz = 0;
  if (act) {
    const unsigned x = (unsigned)cidx;
    const unsigned q0 = (unsigned)(((unsigned long long)x * C.m0) >> 40);
    const unsigned q01 = (unsigned)(((unsigned long long)x * C.m01) >> 40);
    ix = 2 * (int)(x - q0 * (unsigned)C.cn0) + par0;
    iy = 2 * (int)(q0 - q01 * (unsigned)C.cn1) + par1;
    iz = 2 * (int)q01 + par2;
  }
  const long NX = I.NX, zs = NX * NX;
  const int X = ix * P + i, Y = iy * P + j;
  const long g0 = ((long)(iz * P) * NX + Y) * NX + X;
  const bool bxy = Q.dirichlet && (X == 0 || X == NX - 1 || Y == 0 || Y == NX - 1);
  Real u[n];
#pragma unroll
  for (int k = 0; k < n; ++k) {
    const int Z = iz * P + k;
    const bool masked = bxy || (Q.dirichlet && (Z == 0 || Z == NX - 1));
    u[k] = (act && !masked) ? src[g0 + k * zs] : Real(0);
  }
  Real uq[n], gx[n], gy[n], gz[n];
  l_forward<n>(T.S, T.Dc, t0, t1, lane_ok, i, j, u, uq, gx, gy, gz);
  Real val[n], fx[n], fy[n], fz[n];
  const Real hvol = (Real)Q.hvol, ih = (Real)Q.ih, ih2 = (Real)Q.ih2;
  const Real c_mass = (Real)Q.c_mass, c_vel = (Real)Q.c_vel, c_diff = (Real)Q.c_diff;
  Real b0f = 0, b1f = 0;
  if (Q.vel_kind == MPDG_VEL_VORTEX) {
    Real sx, cx, sy, cy;
    const Real xq = ((Real)ix + T.x[i]) * (Real)Q.h, yq = ((Real)iy + T.x[j]) * (Real)Q.h;
    sincospi(xq, &sx, &cx);
    sincospi(yq, &sy, &cy);
    b0f = c_vel * ih * sx * cy;
    b1f = -c_vel * ih * cx * sy;
  }
#pragma unroll
  for (int k = 0; k < n; ++k) {
    const Real JxW = hvol * T.w[i] * T.w[j] * T.w[k];
    val[k] = JxW * (c_mass * uq[k] + b0f * gx[k] + b1f * gy[k]);
    const Real kd = c_diff * JxW * ih2;
    fx[k] = kd * gx[k];
    fy[k] = kd * gy[k];
    fz[k] = kd * gz[k];
  }
  Real out[n];
  l_backward<n>(T.S, T.Dc, t0, t1, lane_ok, i, j, val, fx, fy, fz, out);
  if (act) {
    const int nc = I.nc;
    const bool sx = (i == 0 && ix > 0) || (i == P && ix < nc - 1);
    const bool sy = (j == 0 && iy > 0) || (j == P && iy < nc - 1);
    const bool later_xy = (sx && (ix & 1)) || (sy && (iy & 1));
#pragma unroll
    for (int k = 0; k < n; ++k) {
      const long gg = g0 + k * zs;
      const int Z = iz * P + k;
      const bool sz = (k == 0 && iz > 0) || (k == P && iz < nc - 1);
      const bool first = !(later_xy || (sz && (iz & 1)));
      const bool masked = bxy || (Q.dirichlet && (Z == 0 || Z == NX - 1));
      if (first) dst[gg] = masked ? Real(0) : out[k];
      else if (!masked) dst[gg] += out[k];
    }
  }
}

template <typename Real>
__global__ void __launch_bounds__(kWarpsPerCTA * 32, 4)
    batch_apply_kernel(int colour, const BatchScheduleHeader *__restrict__ hdr,
                       const int *__restrict__ seg_slot, const int *__restrict__ seg_prefix,
                       const SlotInfo *__restrict__ info, const BatchSlotParams *__restrict__ params,
                       Real *const *__restrict__ src_ptrs, Real *const *__restrict__ dst_ptrs,
                       const int *__restrict__ mask)
{
  __shared__ Real tiles_all[kWarpsPerCTA][kBatchTileElems];
  const int total = hdr->total_groups[colour], nseg = hdr->n_seg[colour];
  if (total == 0) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  Real *tiles = tiles_all[warp];
  for (int g = blockIdx.x * kWarpsPerCTA + warp; g < total; g += gridDim.x * kWarpsPerCTA) {
    const int k = batch_find(seg_prefix, nseg, g);
    const int s = seg_slot[k];
    if (!mask[s]) continue;  // warp-uniform
    const SlotInfo &I = info[s];
    const BatchSlotParams &Q = params[s];
    const Real *src = src_ptrs[s];
    Real *dst = dst_ptrs[s];
    const int lg = g - seg_prefix[k];
    switch (I.degree) {
      case 1: batch_cell<1, Real>(colour, lg, I, Q, src, dst, tiles, lane); break;
      case 2: batch_cell<2, Real>(colour, lg, I, Q, src, dst, tiles, lane); break;
      case 3: batch_cell<3, Real>(colour, lg, I, Q, src, dst, tiles, lane); break;
      default: batch_cell<4, Real>(colour, lg, I, Q, src, dst, tiles, lane); break;
    }
  }
}
