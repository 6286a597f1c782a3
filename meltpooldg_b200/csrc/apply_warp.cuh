// Warp-per-cell operator apply (the hot path of vmult), included by
// operator_kernels.cu after the shared tables and kernel parameters.
//
// Layout and schedule:
//  * a warp owns CPW = 32 / n^2 cells (n = degree + 1; one cell for Q4, two
//    for Q3, three for Q2, eight for Q1); lane (i, j) of a cell keeps the DoF
//    column (i, j, 0..n-1) in registers, so z-contractions are register FMAs
//    and x/y contractions go through a per-cell shared tile with __syncwarp
//    only -- no block-wide barrier anywhere in the cell pipeline;
//  * warps are persistent over the cells of one parity colour; the per-cell
//    geometry stream (JxW and the six entries of JxW J^-1 J^-T per quadrature
//    point, padded to 16 bytes per cell) of the warp's next cells is brought
//    into shared memory by one TMA bulk copy (cp.async.bulk + mbarrier
//    complete_tx) issued before the gather and the interpolation, which hide
//    its latency;
//  * scatter is atomic-free: the colours run in order 0..7 and, for every DoF,
//    the cell whose parity bits are zero in all directions in which the DoF is
//    shared with a neighbour is the first to touch it; that cell stores, later
//    colours add.  dst needs no clearing pass.
#pragma once

constexpr int kWarpsPerCTA = 4;
constexpr long kMbarSpinLimit = 1L << 26;  // bounded wait on a bulk copy

template <int n>
struct WCfg {
  static constexpr int cpw = (n == 2) ? 8 : (n == 3) ? 3 : (n == 4) ? 2 : 1;
};

__device__ __forceinline__ unsigned smem_u32(const void *p)
{
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar)
{
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned phase)
{
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// bounded wait: on expiry the error word is set and the wait is retried once
// (also bounded) so that no copy is left targeting this CTA's shared memory
__device__ __forceinline__ void mbar_wait_bounded(uint64_t *bar, unsigned phase, int *err)
{
  long spins = 0;
  while (!mbar_try_wait(bar, phase)) {
    if (++spins > kMbarSpinLimit) {
      if (err) atomicExch(err, 1);
      long again = 0;
      while (!mbar_try_wait(bar, phase) && ++again < kMbarSpinLimit) {
      }
      return;
    }
  }
}

// ---- warp-synchronous contraction passes (tile layout t[k*n*n + j*n + i])

template <int n, typename Real>
__device__ __forceinline__ void w_to_qp(const Real *S, Real *t, int i, int j, const Real (&u)[n],
                                        Real (&v)[n])
{
  Real a[n];
  cz<n, Real, false>(S, u, a);
  put<n>(t, i, j, a);
  __syncwarp();
  cy<n, Real, false>(S, t, i, j, v);
  __syncwarp();
  put<n>(t, i, j, v);
  __syncwarp();
  cx<n, Real, false>(S, t, i, j, a);
  __syncwarp();
#pragma unroll
  for (int k = 0; k < n; ++k) v[k] = a[k];
}

template <int n, typename Real>
__device__ __forceinline__ void w_grad_qp(const Real *Dc, Real *t, int i, int j, const Real (&v)[n],
                                          Real (&gx)[n], Real (&gy)[n], Real (&gz)[n])
{
  put<n>(t, i, j, v);
  __syncwarp();
  cx<n, Real, false>(Dc, t, i, j, gx);
  cy<n, Real, false>(Dc, t, i, j, gy);
  cz<n, Real, false>(Dc, v, gz);
  __syncwarp();
}

template <int n, typename Real>
__device__ __forceinline__ void w_from_qp(const Real *S, const Real *Dc, Real *t0, Real *t1, int i,
                                          int j, const Real (&val)[n], const Real (&fx)[n],
                                          const Real (&fy)[n], const Real (&fz)[n], Real (&out)[n])
{
  Real a[n], b[n];
  put<n>(t0, i, j, fx);
  put<n>(t1, i, j, fy);
  __syncwarp();
  cx<n, Real, true>(Dc, t0, i, j, a);
  cy<n, Real, true>(Dc, t1, i, j, b);
  cz<n, Real, true>(Dc, fz, out);
#pragma unroll
  for (int k = 0; k < n; ++k) a[k] += b[k] + out[k] + val[k];
  __syncwarp();
  put<n>(t0, i, j, a);
  __syncwarp();
  cx<n, Real, true>(S, t0, i, j, b);
  __syncwarp();
  put<n>(t0, i, j, b);
  __syncwarp();
  cy<n, Real, true>(S, t0, i, j, a);
  cz<n, Real, true>(S, a, out);
  __syncwarp();
}

// dynamic shared memory per warp, in units of Real
template <int P, typename Real, int GEOM>
__host__ __device__ constexpr int warp_smem_elems(bool vel)
{
  constexpr int n = P + 1, n3 = n * n * n, CPW = WCfg<n>::cpw;
  return (GEOM == GEOM_GENERAL ? CPW * (metric_stride(n) + (vel ? velb_stride(n) : 0)) : 0) +
         2 * (CPW + 1) * n3;
}

template <int P, typename Real, int GEOM, bool KT>
__global__ void __launch_bounds__(kWarpsPerCTA * 32) warp_apply_kernel(const KP<Real> p, int *err)
{
  constexpr int n = P + 1, n2 = n * n, n3 = n2 * n, CPW = WCfg<n>::cpw;
  constexpr int MS = metric_stride(n), VS = velb_stride(n);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bars[kWarpsPerCTA];
  __shared__ Real sS[n2], sDc[n2];
  const Tables<Real> &T = tab<Real>(P);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool has_vel = p.vel_kind != MPDG_VEL_NONE;
  const bool gvel = GEOM == GEOM_GENERAL && has_vel;

  for (int t = threadIdx.x; t < n2; t += blockDim.x) {
    sS[t] = T.S[t];
    sDc[t] = T.Dc[t];
  }
  if (lane == 0) mbar_init(&bars[warp], 1);
  fence_mbar_init();
  __syncthreads();

  Real *wsm = reinterpret_cast<Real *>(smem_raw) + warp * warp_smem_elems<P, Real, GEOM>(gvel);
  Real *stage = wsm;                                    // CPW * MS
  Real *vstage = wsm + (GEOM == GEOM_GENERAL ? CPW * MS : 0);  // CPW * VS
  Real *tiles = wsm + (GEOM == GEOM_GENERAL ? CPW * (MS + (gvel ? VS : 0)) : 0);

  const int sub = lane / n2, l = lane % n2, i = l % n, j = l / n;
  const bool lane_ok = sub < CPW;
  Real *t0 = tiles + sub * n3;               // idle lanes get the scratch tile CPW
  Real *t1 = tiles + (CPW + 1 + sub) * n3;
  const long zs = p.NX * p.NY;
  unsigned phase = 0;

  for (long group = (long)blockIdx.x * kWarpsPerCTA + warp; group * CPW < p.ccount;
       group += (long)gridDim.x * kWarpsPerCTA) {
    const long c0 = group * CPW;
    const int ncell = (int)min((long)CPW, p.ccount - c0);
    if (GEOM == GEOM_GENERAL && lane == 0) {
      fence_proxy_async();
      const unsigned mb = ncell * MS * sizeof(Real), vb = gvel ? ncell * VS * sizeof(Real) : 0;
      mbar_expect_tx(&bars[warp], mb + vb);
      bulk_g2s(stage, p.metric + (p.cfirst + c0) * MS, mb, &bars[warp]);
      if (gvel) bulk_g2s(vstage, p.velb + (p.cfirst + c0) * VS, vb, &bars[warp]);
    }
    const long cidx = c0 + sub;
    const bool active = lane_ok && sub < ncell;
    int ix = 0, iy = 0, iz = 0;
    if (active) {
      const long a = cidx % p.cn[0], b = (cidx / p.cn[0]) % p.cn[1], c = cidx / ((long)p.cn[0] * p.cn[1]);
      ix = 2 * (int)a + p.par[0];
      iy = 2 * (int)b + p.par[1];
      iz = 2 * (int)c + p.par[2];
    }
    const long cell = p.cfirst + cidx;
    const long g0 = ((long)(iz * P) * p.NY + (iy * P + j)) * p.NX + (ix * P + i);
    const bool bflag = active && p.cell_flags && (p.cell_flags[cell] & 1);

    Real u[n];
#pragma unroll
    for (int k = 0; k < n; ++k) {
      Real v = 0;
      if (active) {
        v = p.src[g0 + k * zs];
        if (p.masked_read && bflag && p.dmask[g0 + k * zs]) v = 0;
      }
      u[k] = v;
    }
    Real Tq[n], Tgx[n], Tgy[n], Tgz[n];
    if (KT) {
      Real tl[n];
#pragma unroll
      for (int k = 0; k < n; ++k) tl[k] = active ? p.T[g0 + k * zs] : Real(0);
      w_to_qp<n>(sS, t1, i, j, tl, Tq);
      if (p.full_tangent) w_grad_qp<n>(sDc, t1, i, j, Tq, Tgx, Tgy, Tgz);
    }
    Real uq[n], gx[n], gy[n], gz[n];
    w_to_qp<n>(sS, t0, i, j, u, uq);
    w_grad_qp<n>(sDc, t0, i, j, uq, gx, gy, gz);

    if (GEOM == GEOM_GENERAL) {
      mbar_wait_bounded(&bars[warp], phase, err);
      phase ^= 1;
    }

    Real val[n], fx[n], fy[n], fz[n];
    const Real *ms = stage + (lane_ok ? sub : 0) * MS + j * n + i;
    const Real *vs = vstage + (lane_ok ? sub : 0) * VS + j * n + i;
#pragma unroll
    for (int k = 0; k < n; ++k) {
      Real JxW, G00, G01, G02, G11, G12, G22, b0 = 0, b1 = 0, b2 = 0;
      if (GEOM == GEOM_GENERAL) {
        const Real *m = ms + k * n2;
        JxW = m[0];
        G00 = m[n3];
        G01 = m[2 * n3];
        G02 = m[3 * n3];
        G11 = m[4 * n3];
        G12 = m[5 * n3];
        G22 = m[6 * n3];
        if (gvel) {
          b0 = vs[k * n2];
          b1 = vs[k * n2 + n3];
          b2 = vs[k * n2 + 2 * n3];
        }
      } else {
        JxW = p.h[0] * p.h[1] * p.h[2] * T.w[i] * T.w[j] * T.w[k];
        G00 = JxW / (p.h[0] * p.h[0]);
        G11 = JxW / (p.h[1] * p.h[1]);
        G22 = JxW / (p.h[2] * p.h[2]);
        G01 = G02 = G12 = 0;
        if (has_vel) {
          Real uv[3];
          uniform_velocity<Real, n>(p, T, ix, iy, iz, i, j, k, uv);
          b0 = JxW * uv[0] / p.h[0];
          b1 = JxW * uv[1] / p.h[1];
          b2 = JxW * uv[2] / p.h[2];
        }
      }
      const Real kq = KT ? p.c_diff * (Real(1) + p.k_alpha * Tq[k]) : p.c_diff;
      val[k] = p.c_mass * JxW * uq[k] + p.c_vel * (b0 * gx[k] + b1 * gy[k] + b2 * gz[k]);
      if (GEOM == GEOM_GENERAL) {
        fx[k] = kq * (G00 * gx[k] + G01 * gy[k] + G02 * gz[k]);
        fy[k] = kq * (G01 * gx[k] + G11 * gy[k] + G12 * gz[k]);
        fz[k] = kq * (G02 * gx[k] + G12 * gy[k] + G22 * gz[k]);
      } else {
        fx[k] = kq * G00 * gx[k];
        fy[k] = kq * G11 * gy[k];
        fz[k] = kq * G22 * gz[k];
      }
      if (KT && p.full_tangent) {
        const Real dk = p.c_diff * p.k_alpha * uq[k];
        if (GEOM == GEOM_GENERAL) {
          fx[k] += dk * (G00 * Tgx[k] + G01 * Tgy[k] + G02 * Tgz[k]);
          fy[k] += dk * (G01 * Tgx[k] + G11 * Tgy[k] + G12 * Tgz[k]);
          fz[k] += dk * (G02 * Tgx[k] + G12 * Tgy[k] + G22 * Tgz[k]);
        } else {
          fx[k] += dk * G00 * Tgx[k];
          fy[k] += dk * G11 * Tgy[k];
          fz[k] += dk * G22 * Tgz[k];
        }
      }
    }

    Real out[n];
    w_from_qp<n>(sS, sDc, t0, t1, i, j, val, fx, fy, fz, out);

    if (active) {
      const bool sx = (i == 0 && ix > 0) || (i == P && ix < p.nc[0] - 1);
      const bool sy = (j == 0 && iy > 0) || (j == P && iy < p.nc[1] - 1);
      const bool later_xy = (sx && (ix & 1)) || (sy && (iy & 1));
#pragma unroll
      for (int k = 0; k < n; ++k) {
        const long g = g0 + k * zs;
        const bool sz = (k == 0 && iz > 0) || (k == P && iz < p.nc[2] - 1);
        const bool first = !(later_xy || (sz && (iz & 1)));
        const bool masked = p.masked_write && bflag && p.dmask[g];
        if (first) p.dst[g] = masked ? Real(0) : out[k];
        else if (!masked) p.dst[g] += out[k];
      }
    }
  }
}
