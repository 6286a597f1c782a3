// FP32 warp-per-cell apply with z-plane pairs in packed FP32x2 arithmetic
// (included by operator_kernels.cu after apply_warp.cuh).
//
// Same schedule, scatter and bulk-copied coefficient stream as
// warp_apply_kernel, but the lane's DoF column is held as NP = ceil(n/2)
// float2 pairs (planes k, k+1).  Every register contraction, every shared
// tile read (one 64-bit load fetches both planes) and every quadrature-point
// FMA then serves two planes: __ffma2_rn (sm_100 packed FP32 FMA) halves the
// instruction count of the FP32 form, which is issue-bound.  The coefficient
// stream keeps the FP32 layout of warp_apply_kernel (no padding in HBM).
#pragma once

template <int n>
struct PairCfg {
  static constexpr int np = (n + 1) / 2;  // plane pairs (the last one half empty for odd n)
};

// (S[2q][k], S[2q+1][k]) etc.: row pairs of the 1D tables for the register passes
struct PairTables {
  float2 S[kMaxN * kMaxN];    // [qp][k] = (S[2qp][k], S[2qp+1][k])
  float2 St[kMaxN * kMaxN];   // [qp][k] = (S[k][2qp], S[k][2qp+1])
  float2 Dc[kMaxN * kMaxN];
  float2 Dct[kMaxN * kMaxN];
  float2 w[kMaxN];            // (w[2qp], w[2qp+1]) Gauss weights
};
__constant__ PairTables c_pair[kMaxDegree + 1];

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 fmul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fadd2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float lo_hi(const float2 &v, int h) { return h ? v.y : v.x; }

// out[qp] = sum_k A[qp][k] * in_k   (A = paired constant table, in_k scalar plane k)
template <int n>
__device__ __forceinline__ void cz2(const float2 *A, const float2 (&in)[PairCfg<n>::np],
                                    float2 (&out)[PairCfg<n>::np])
{
  constexpr int NP = PairCfg<n>::np;
#pragma unroll
  for (int q = 0; q < NP; ++q) {
    float2 s = make_float2(0.f, 0.f);
#pragma unroll
    for (int k = 0; k < n; ++k) s = ffma2(A[q * n + k], f2(lo_hi(in[k / 2], k & 1)), s);
    out[q] = s;
  }
}

// x-pass: out[kp] = sum_r M[i][r] (TR: M[r][i]) * t[kp][j][r]
template <int n, bool TR>
__device__ __forceinline__ void cx2(const float *M, const float2 *t, int i, int j,
                                    float2 (&out)[PairCfg<n>::np])
{
  constexpr int NP = PairCfg<n>::np;
  float m[n];
#pragma unroll
  for (int r = 0; r < n; ++r) m[r] = TR ? M[r * n + i] : M[i * n + r];
#pragma unroll
  for (int kp = 0; kp < NP; ++kp) {
    float2 s = make_float2(0.f, 0.f);
#pragma unroll
    for (int r = 0; r < n; ++r) s = ffma2(f2(m[r]), t[(kp * n + j) * n + r], s);
    out[kp] = s;
  }
}

template <int n, bool TR>
__device__ __forceinline__ void cy2(const float *M, const float2 *t, int i, int j,
                                    float2 (&out)[PairCfg<n>::np])
{
  constexpr int NP = PairCfg<n>::np;
  float m[n];
#pragma unroll
  for (int r = 0; r < n; ++r) m[r] = TR ? M[r * n + j] : M[j * n + r];
#pragma unroll
  for (int kp = 0; kp < NP; ++kp) {
    float2 s = make_float2(0.f, 0.f);
#pragma unroll
    for (int r = 0; r < n; ++r) s = ffma2(f2(m[r]), t[(kp * n + r) * n + i], s);
    out[kp] = s;
  }
}

template <int n>
__device__ __forceinline__ void put2(float2 *t, int i, int j, const float2 (&v)[PairCfg<n>::np])
{
#pragma unroll
  for (int kp = 0; kp < PairCfg<n>::np; ++kp) t[(kp * n + j) * n + i] = v[kp];
}

template <int P, int GEOM>
__host__ __device__ constexpr int pair_smem_floats(bool vel)
{
  constexpr int n = P + 1, CPW = WCfg<n>::cpw, NP = PairCfg<n>::np;
  return (((GEOM == GEOM_GENERAL ? CPW * (metric_stride(n) + (vel ? velb_stride(n) : 0)) : 0) +
           2 * CPW * NP * n * n * 2) + 7) / 8 * 8;
}

template <int P, int GEOM>
__global__ void __launch_bounds__(kWarpsPerCTA * 32, (P == 4 ? 5 : P == 3 ? 6 : 8))
    warp_apply_f2_kernel(const KP<float> p, int *err)
{
  constexpr int n = P + 1, n2 = n * n, n3 = n2 * n, CPW = WCfg<n>::cpw, NP = PairCfg<n>::np;
  constexpr int MS = metric_stride(n), VS = velb_stride(n);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bars[kWarpsPerCTA];
  __shared__ float sS[n2], sDc[n2];
  const Tables<float> &T = tab<float>(P);
  const PairTables &PT = c_pair[P];
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

  unsigned char *base = smem_raw + ((kSmemAlign - (smem_u32(smem_raw) & (kSmemAlign - 1))) & (kSmemAlign - 1));
  float *wsm = reinterpret_cast<float *>(base) + warp * pair_smem_floats<P, GEOM>(gvel);
  float *stage = wsm;
  float *vstage = wsm + (GEOM == GEOM_GENERAL ? CPW * MS : 0);
  float2 *tiles = reinterpret_cast<float2 *>(wsm + (GEOM == GEOM_GENERAL ? CPW * (MS + (gvel ? VS : 0)) : 0));

  const int sub = lane / n2, l = lane % n2, i = l % n, j = l / n;
  const bool lane_ok = sub < CPW;
  const int s_sub = lane_ok ? sub : 0;
  float2 *t0 = tiles + s_sub * NP * n2;
  float2 *t1 = tiles + (CPW + s_sub) * NP * n2;
  const long zs = p.NX * p.NY;
  const int count = (int)p.ccount;
  const int gstride = gridDim.x * kWarpsPerCTA;
  unsigned phase = 0;

  auto issue_stage = [&](int grp) {
    const int c0 = grp * CPW;
    const int ncell = min(CPW, count - c0);
    const unsigned mb = ncell * MS * sizeof(float), vb = gvel ? ncell * VS * sizeof(float) : 0;
    fence_proxy_async();
    mbar_expect_tx(&bars[warp], mb + vb);
    bulk_g2s(stage, p.metric + (p.cfirst + c0) * (long)MS, mb, &bars[warp]);
    if (gvel) bulk_g2s(vstage, p.velb + (p.cfirst + c0) * (long)VS, vb, &bars[warp]);
  };
  const bool use_mask = p.cell_mask != nullptr && (p.masked_read || p.masked_write);
  auto gather = [&](int grp, float (&A)[n], uint4 &cm) {
    const int cidx = grp * CPW + sub;
    const bool act = lane_ok && grp * CPW < count && cidx < count;
    int ix = 0, iy = 0, iz = 0;
    if (act) colour_cell(cidx, p, ix, iy, iz);
    const long g0 = ((long)(iz * P) * p.NY + (iy * P + j)) * p.NX + (ix * P + i);
#pragma unroll
    for (int k = 0; k < n; ++k) A[k] = act ? p.src[g0 + k * zs] : 0.f;
    cm = (act && use_mask) ? p.cell_mask[p.cfirst + cidx] : make_uint4(0u, 0u, 0u, 0u);
  };
  auto mask_bit = [&](const uint4 &cm, int k) -> bool {
    const int b = k * n2 + l;
    const unsigned w = (b < 32) ? cm.x : (b < 64) ? cm.y : (b < 96) ? cm.z : cm.w;
    return (w >> (b & 31)) & 1u;
  };

  int group = blockIdx.x * kWarpsPerCTA + warp;
  if (GEOM == GEOM_GENERAL && lane == 0 && group * CPW < count) issue_stage(group);
  float A[n];
  uint4 cmA;
  gather(group, A, cmA);

  for (; group * CPW < count; group += gstride) {
    const int gnext = group + gstride;
    const bool has_next = gnext * CPW < count;
    const int cidx = group * CPW + sub;
    const bool active = lane_ok && cidx < count;
    int ix = 0, iy = 0, iz = 0;
    if (active) colour_cell(cidx, p, ix, iy, iz);
    const long g0 = ((long)(iz * P) * p.NY + (iy * P + j)) * p.NX + (ix * P + i);
    const uint4 cm = cmA;

    const bool sx = (i == 0 && ix > 0) || (i == P && ix < p.nc[0] - 1);
    const bool sy = (j == 0 && iy > 0) || (j == P && iy < p.nc[1] - 1);
    const bool later_xy = (sx && (ix & 1)) || (sy && (iy & 1));
    float dpre[n];
    unsigned first_bits = 0, mask_bits = 0;
#pragma unroll
    for (int k = 0; k < n; ++k) {
      const long g = g0 + k * zs;
      const bool sz = (k == 0 && iz > 0) || (k == P && iz < p.nc[2] - 1);
      const bool first = !(later_xy || (sz && (iz & 1)));
      const bool masked = p.masked_write && mask_bit(cm, k);
      first_bits |= (unsigned)first << k;
      mask_bits |= (unsigned)masked << k;
      dpre[k] = (active && !first && !masked) ? p.dst[g] : 0.f;
    }

    float2 u[NP];
#pragma unroll
    for (int kp = 0; kp < NP; ++kp) {
      const int k0 = 2 * kp, k1 = 2 * kp + 1;
      const float a0 = (p.masked_read && mask_bit(cm, k0)) ? 0.f : A[k0];
      const float a1 = (k1 < n) ? ((p.masked_read && mask_bit(cm, k1)) ? 0.f : A[k1 < n ? k1 : 0]) : 0.f;
      u[kp] = make_float2(a0, a1);
    }
    if (has_next) gather(gnext, A, cmA);

    // values and reference gradients at the Gauss points
    float2 a[NP], uq[NP], gx[NP], gy[NP], gz[NP];
    cz2<n>(PT.S, u, a);
    if (lane_ok) put2<n>(t0, i, j, a);
    __syncwarp();
    cy2<n, false>(sS, t0, i, j, uq);
    __syncwarp();
    if (lane_ok) put2<n>(t0, i, j, uq);
    __syncwarp();
    cx2<n, false>(sS, t0, i, j, a);
    __syncwarp();
#pragma unroll
    for (int kp = 0; kp < NP; ++kp) uq[kp] = a[kp];
    if (lane_ok) put2<n>(t0, i, j, uq);
    __syncwarp();
    cx2<n, false>(sDc, t0, i, j, gx);
    cy2<n, false>(sDc, t0, i, j, gy);
    cz2<n>(PT.Dc, uq, gz);
    __syncwarp();

    if (GEOM == GEOM_GENERAL) {
      mbar_wait_bounded(&bars[warp], phase, err);
      phase ^= 1;
    }

    // quadrature-point kernel, two planes per instruction
    float2 val[NP], fx[NP], fy[NP], fz[NP];
    const float *ms = stage + s_sub * MS + j * n + i;
    const float *vs = vstage + s_sub * VS + j * n + i;
#pragma unroll
    for (int kp = 0; kp < NP; ++kp) {
      const int k0 = 2 * kp, k1 = (2 * kp + 1 < n) ? 2 * kp + 1 : 2 * kp;
      const bool has1 = 2 * kp + 1 < n;
      auto pick = [&](const float *m, int e) {
        return make_float2(m[e * n3 + k0 * n2], has1 ? m[e * n3 + k1 * n2] : 0.f);
      };
      float2 b0 = make_float2(0.f, 0.f), b1 = b0, b2 = b0;
      if (GEOM == GEOM_GENERAL) {
        const float2 cm2 = pick(ms, 0), G00 = pick(ms, 1), G01 = pick(ms, 2), G02 = pick(ms, 3),
                     G11 = pick(ms, 4), G12 = pick(ms, 5), G22 = pick(ms, 6);
        if (gvel) {
          const float2 cv = f2(p.c_vel);
          b0 = fmul2(cv, pick(vs, 0));
          b1 = fmul2(cv, pick(vs, 1));
          b2 = fmul2(cv, pick(vs, 2));
        }
        val[kp] = ffma2(cm2, uq[kp], ffma2(b0, gx[kp], ffma2(b1, gy[kp], fmul2(b2, gz[kp]))));
        fx[kp] = ffma2(G00, gx[kp], ffma2(G01, gy[kp], fmul2(G02, gz[kp])));
        fy[kp] = ffma2(G01, gx[kp], ffma2(G11, gy[kp], fmul2(G12, gz[kp])));
        fz[kp] = ffma2(G02, gx[kp], ffma2(G12, gy[kp], fmul2(G22, gz[kp])));
      } else {
        const float2 JxW = fmul2(f2(p.hvol * T.w[i] * T.w[j]), PT.w[kp]);
        if (has_vel) {
          float uv0[3], uv1[3];
          uniform_velocity<float, n>(p, T, ix, iy, iz, i, j, k0, uv0);
          uniform_velocity<float, n>(p, T, ix, iy, iz, i, j, k1, uv1);
          const float2 cj = fmul2(f2(p.c_vel), JxW);
          b0 = fmul2(cj, make_float2(uv0[0] * p.ih[0], uv1[0] * p.ih[0]));
          b1 = fmul2(cj, make_float2(uv0[1] * p.ih[1], uv1[1] * p.ih[1]));
          b2 = fmul2(cj, make_float2(uv0[2] * p.ih[2], uv1[2] * p.ih[2]));
        }
        val[kp] = ffma2(fmul2(f2(p.c_mass), JxW), uq[kp],
                        ffma2(b0, gx[kp], ffma2(b1, gy[kp], fmul2(b2, gz[kp]))));
        const float2 kd = fmul2(f2(p.c_diff), JxW);
        fx[kp] = fmul2(fmul2(kd, f2(p.ih2[0])), gx[kp]);
        fy[kp] = fmul2(fmul2(kd, f2(p.ih2[1])), gy[kp]);
        fz[kp] = fmul2(fmul2(kd, f2(p.ih2[2])), gz[kp]);
      }
      if (!has1) {  // the empty half of the last pair stays zero
        val[kp].y = 0.f;
        fx[kp].y = 0.f;
        fy[kp].y = 0.f;
        fz[kp].y = 0.f;
      }
    }
    if (GEOM == GEOM_GENERAL) {
      __syncwarp();
      if (lane == 0 && has_next) issue_stage(gnext);
    }

    // test with values and gradients, back to the nodal column
    float2 b[NP], c[NP];
    if (lane_ok) {
      put2<n>(t0, i, j, fx);
      put2<n>(t1, i, j, fy);
    }
    __syncwarp();
    cx2<n, true>(sDc, t0, i, j, b);
    cy2<n, true>(sDc, t1, i, j, c);
    cz2<n>(PT.Dct, fz, a);
#pragma unroll
    for (int kp = 0; kp < NP; ++kp) b[kp] = fadd2(fadd2(b[kp], c[kp]), fadd2(a[kp], val[kp]));
    __syncwarp();
    if (lane_ok) put2<n>(t0, i, j, b);
    __syncwarp();
    cx2<n, true>(sS, t0, i, j, c);
    __syncwarp();
    if (lane_ok) put2<n>(t0, i, j, c);
    __syncwarp();
    cy2<n, true>(sS, t0, i, j, b);
    // z: out_k = sum_q S[q][k] b_q; the empty half of the last pair is zero in b
    float2 outp[NP];
    cz2<n>(PT.St, b, outp);
    __syncwarp();

    if (active) {
#pragma unroll
      for (int k = 0; k < n; ++k) {
        const long g = g0 + k * zs;
        const float o = lo_hi(outp[k / 2], k & 1);
        if ((first_bits >> k) & 1) p.dst[g] = ((mask_bits >> k) & 1) ? 0.f : o;
        else if (!((mask_bits >> k) & 1)) p.dst[g] = dpre[k] + o;
      }
    }
  }
}
