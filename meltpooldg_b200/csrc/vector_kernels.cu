// Vector kernels of the Krylov solvers: deterministic FP64 reductions (warp
// shuffles, then a fixed-order block pass) and the fused CG / Chebyshev / GMRES
// updates.  All reductions accumulate in FP64 whatever the vector precision.
#include <cuda_runtime.h>

#include <cmath>

#include "mpdg_internal.h"
#include "vector_kernels.cuh"

namespace mpdg {

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

// block-wide sum of v (blockDim.x == kRedThreads); result valid in thread 0
__device__ __forceinline__ double block_sum(double v)
{
  __shared__ double ws[kRedThreads / 32];
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) ws[w] = v;
  __syncthreads();
  double s = 0.0;
  if (w == 0) {
    s = (lane < kRedThreads / 32) ? ws[lane] : 0.0;
    s = warp_sum(s);
  }
  __syncthreads();
  return s;
}

// Grid-stride loops take kU elements per thread per pass (i, i + stride, ...,
// loaded before any is used), so that each thread keeps kU loads of every
// operand in flight; the per-thread order of a sum is the plain grid-stride
// order, so reductions do not depend on kU.
constexpr int kU = 4;

template <typename A, typename B>
__global__ void __launch_bounds__(kRedThreads) dot_partial_kernel(const A *a, const B *b, long n,
                                                                  double *partial)
{
  double s = 0.0;
  const long stride = (long)gridDim.x * blockDim.x;
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  for (; i + (kU - 1) * stride < n; i += kU * stride) {
    A va[kU];
    B vb[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      va[u] = a[i + u * stride];
      vb[u] = b[i + u * stride];
    }
#pragma unroll
    for (int u = 0; u < kU; ++u) s += (double)va[u] * (double)vb[u];
  }
  for (; i < n; i += stride) s += (double)a[i] * (double)b[i];
  s = block_sum(s);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kRedThreads) linf_partial_kernel(const double *a, long n, double *partial)
{
  __shared__ double ws[kRedThreads / 32];
  double s = 0.0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    s = fmax(s, fabs(a[i]));
  s = warp_max(s);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) ws[w] = s;
  __syncthreads();
  if (w == 0) {
    s = (lane < kRedThreads / 32) ? ws[lane] : 0.0;
    s = warp_max(s);
    if (lane == 0) partial[blockIdx.x] = s;
  }
}

// sums (or max-reduces) `count` groups of kRedBlocks partials into out[0..count)
__global__ void __launch_bounds__(kRedThreads) finish_kernel(const double *partial, int count,
                                                             double *out, int use_max)
{
  const int g = blockIdx.x;
  if (g >= count) return;
  double s = 0.0;
  for (int i = threadIdx.x; i < kRedBlocks; i += blockDim.x) {
    const double v = partial[(long)g * kRedBlocks + i];
    s = use_max ? fmax(s, v) : s + v;
  }
  if (use_max) {
    __shared__ double ws[kRedThreads / 32];
    s = warp_max(s);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) ws[w] = s;
    __syncthreads();
    if (w == 0) {
      s = (lane < kRedThreads / 32) ? ws[lane] : 0.0;
      s = warp_max(s);
      if (lane == 0) out[g] = s;
    }
  } else {
    s = block_sum(s);
    if (threadIdx.x == 0) out[g] = s;
  }
}

// V_k . u and (HAS_W) V_k . w for k0 <= k < k0 + CNT: partial groups k and
// m + k.  CNT is a compile-time width, so every load of an element's row is
// issued before the first product that uses one.
template <typename R, bool HAS_W, int CNT>
__device__ __forceinline__ void mdot2_chunk(const R *V, long n, int m, int k0, const R *u, const R *w,
                                            double *partial)
{
  double su[CNT], sw[CNT];
#pragma unroll
  for (int c = 0; c < CNT; ++c) su[c] = sw[c] = 0.0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double ui = (double)u[i];
    const double wi = HAS_W ? (double)w[i] : 0.0;
    double vk[CNT];
#pragma unroll
    for (int c = 0; c < CNT; ++c) vk[c] = (double)V[(long)(k0 + c) * n + i];
#pragma unroll
    for (int c = 0; c < CNT; ++c) {
      su[c] += vk[c] * ui;
      if (HAS_W) sw[c] += vk[c] * wi;
    }
  }
#pragma unroll
  for (int c = 0; c < CNT; ++c) {
    const double t = block_sum(su[c]);
    if (threadIdx.x == 0) partial[(long)(k0 + c) * kRedBlocks + blockIdx.x] = t;
    if (HAS_W) {
      const double t2 = block_sum(sw[c]);
      if (threadIdx.x == 0) partial[(long)(m + k0 + c) * kRedBlocks + blockIdx.x] = t2;
    }
  }
}

// V_k . u and (HAS_W) V_k . w for k < m in one pass, 8 basis vectors at a
// time (u and w are read once per 8)
template <typename R, bool HAS_W>
__global__ void __launch_bounds__(kRedThreads, 4) mdot2_partial_kernel(const R *V, long n, int m, const R *u,
                                                                    const R *w, double *partial)
{
  for (int k0 = 0; k0 < m; k0 += 8) {
    switch (min(8, m - k0)) {
      case 8: mdot2_chunk<R, HAS_W, 8>(V, n, m, k0, u, w, partial); break;
      case 7: mdot2_chunk<R, HAS_W, 7>(V, n, m, k0, u, w, partial); break;
      case 6: mdot2_chunk<R, HAS_W, 6>(V, n, m, k0, u, w, partial); break;
      case 5: mdot2_chunk<R, HAS_W, 5>(V, n, m, k0, u, w, partial); break;
      case 4: mdot2_chunk<R, HAS_W, 4>(V, n, m, k0, u, w, partial); break;
      case 3: mdot2_chunk<R, HAS_W, 3>(V, n, m, k0, u, w, partial); break;
      case 2: mdot2_chunk<R, HAS_W, 2>(V, n, m, k0, u, w, partial); break;
      default: mdot2_chunk<R, HAS_W, 1>(V, n, m, k0, u, w, partial); break;
    }
  }
}

// One sweep of delayed classical Gram-Schmidt over the basis columns 0..j+1:
//   q_j     = (V_j - sum_{k<j} s_k V_k) / alpha          (written over V_j)
//   u_{j+1} = V_{j+1} / alpha - sum_{k<j} c_k V_k - c_j q_j   (over V_{j+1})
// V_{j+1} holds w = B u_j on entry; s and c come as kernel parameters.
template <typename R>
__global__ void dcgs2_sweep_kernel(R *V, long n, int j, double inv_alpha, const DcgsCoef cf)
{
  R *vj = V + (long)j * n, *vn = V + (long)(j + 1) * n;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double q = (double)vj[i], u = (double)vn[i] * inv_alpha;
    for (int k = 0; k < j; ++k) {
      const double vk = (double)V[(long)k * n + i];
      q -= cf.s[k] * vk;
      u -= cf.c[k] * vk;
    }
    const R qr = (R)(q * inv_alpha);
    vj[i] = qr;
    vn[i] = (R)(u - cf.c[j] * (double)qr);
  }
}

// x = sum_k y[k] V_k
template <typename R>
__global__ void combine_kernel(const R *V, long n, int m, const double *y, R *x)
{
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < m; ++k) s += y[k] * (double)V[(long)k * n + i];
    x[i] = (R)s;
  }
}

template <typename R>
__global__ void axpby_kernel(long n, double a, const R *x, double b, R *y)
{
  const long stride = (long)gridDim.x * blockDim.x;
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  for (; i + (kU - 1) * stride < n; i += kU * stride) {
    R vx[kU], vy[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      vx[u] = x[i + u * stride];
      vy[u] = y[i + u * stride];
    }
#pragma unroll
    for (int u = 0; u < kU; ++u) y[i + u * stride] = (R)(a * (double)vx[u] + b * (double)vy[u]);
  }
  for (; i < n; i += stride) y[i] = (R)(a * (double)x[i] + b * (double)y[i]);
}

// y = b - y
__global__ void residual_kernel(long n, const double *b, double *y)
{
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    y[i] = b[i] - y[i];
}

template <typename R>
__global__ void scale_copy_kernel(long n, double a, const double *x, R *y)
{
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    y[i] = (R)(a * x[i]);
}

template <typename R>
__global__ void add_scaled_kernel(long n, double a, const R *x, double *y)
{
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    y[i] += a * (double)x[i];
}

template <typename R>
__global__ void mul_kernel(long n, const R *d, const R *x, R *y)
{
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    y[i] = d[i] * x[i];
}

// CG step part 1: alpha = s[RZ] / s[PAP]; x += alpha p; r -= alpha Ap;
// with jacobi: z = invd r; partials of r.r (slot 0) and r.z (slot 1)
template <typename R, typename RX, bool LAG = false>
__global__ void __launch_bounds__(kRedThreads) cg_update_kernel(long n, const double *s, RX *x,
                                                                R *r, const R *p, const R *Ap,
                                                                const R *invd, R *z,
                                                                double *partial, double xscale)
{
  if (LAG && s[kDONE] != 0.0) return;  // grid-uniform: the solve stopped
  const double alpha = s[kRZ] / s[kPAP];
  const double xa = alpha * xscale;
  double rr = 0.0, rz = 0.0;
  auto one = [&](long i, RX xi, R pi, R r0, R api, R di) {
    x[i] = (RX)((double)xi + xa * (double)pi);
    const R ri = (R)((double)r0 - alpha * (double)api);
    r[i] = ri;
    rr += (double)ri * (double)ri;
    if (invd) {
      const R zi = di * ri;
      z[i] = zi;
      rz += (double)ri * (double)zi;
    }
  };
  const long stride = (long)gridDim.x * blockDim.x;
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  for (; i + (kU - 1) * stride < n; i += kU * stride) {
    RX vx[kU];
    R vp[kU], vr[kU], va[kU], vd[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const long j = i + u * stride;
      vx[u] = x[j];
      vp[u] = p[j];
      vr[u] = r[j];
      va[u] = Ap[j];
      vd[u] = invd ? invd[j] : R(0);
    }
#pragma unroll
    for (int u = 0; u < kU; ++u) one(i + u * stride, vx[u], vp[u], vr[u], va[u], vd[u]);
  }
  for (; i < n; i += stride) one(i, x[i], p[i], r[i], Ap[i], invd ? invd[i] : R(0));
  rr = block_sum(rr);
  if (threadIdx.x == 0) partial[blockIdx.x] = rr;
  if (invd) {
    rz = block_sum(rz);
    if (threadIdx.x == 0) partial[kRedBlocks + blockIdx.x] = rz;
  }
}

// CG step part 2: beta = s[RZNEW] / s[RZ]; p = z + beta p; s[RZ] <- s[RZNEW] (block 0)
template <typename R, bool LAG = false>
__global__ void cg_direction_kernel(long n, double *s, R *p, const R *z)
{
  if (LAG && s[kDONE] != 0.0) return;
  const double beta = s[kRZNEW] / s[kRZ];
  const long stride = (long)gridDim.x * blockDim.x;
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  for (; i + (kU - 1) * stride < n; i += kU * stride) {
    R vz[kU], vp[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      vz[u] = z[i + u * stride];
      vp[u] = p[i + u * stride];
    }
#pragma unroll
    for (int u = 0; u < kU; ++u) p[i + u * stride] = (R)((double)vz[u] + beta * (double)vp[u]);
  }
  for (; i < n; i += stride) p[i] = (R)((double)z[i] + beta * (double)p[i]);
}

__global__ void shift_scalar_kernel(double *s)
{
  s[kRZ] = s[kRZNEW];
}

__global__ void shift_scalar_lagged_kernel(double *s)
{
  if (s[kDONE] == 0.0) s[kRZ] = s[kRZNEW];
}

// after each iteration: counts it (s[kCONV]) and runs the host loop's test
// |r| <= tol (sqrt correctly rounded, so the decision is the host's) and the
// non-finite check, once; r.r is kept, since later (skipped) iterations reuse
// the partials.  The iteration number lives on the device, so a batch of
// iterations is the same launch sequence every time (a graph replays it).
__global__ void cg_check_kernel(double *s)
{
  if (s[kDONE] != 0.0) return;
  s[kCONV] += 1.0;
  const double rr = s[kRR], res = sqrt(rr);
  if (!isfinite(res)) {
    s[kDONE] = 2.0;
  } else if (res <= s[kTOL]) {
    s[kDONE] = 1.0;
  } else {
    return;
  }
  s[kRRCONV] = rr;
}

// Chebyshev start: d = invd r / theta; z = d
template <typename R>
__global__ void cheb_start_kernel(long n, double inv_theta, const R *invd, const R *r, R *d, R *z)
{
  const long stride = (long)gridDim.x * blockDim.x;
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  for (; i + (kU - 1) * stride < n; i += kU * stride) {
    R vi[kU], vr[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      vi[u] = invd[i + u * stride];
      vr[u] = r[i + u * stride];
    }
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const R v = (R)(inv_theta * (double)(vi[u] * vr[u]));
      d[i + u * stride] = v;
      z[i + u * stride] = v;
    }
  }
  for (; i < n; i += stride) {
    const R v = (R)(inv_theta * (double)(invd[i] * r[i]));
    d[i] = v;
    z[i] = v;
  }
}

// Chebyshev step: d = c1 d + c2 invd (r - t); z += d
template <typename R>
__global__ void cheb_step_kernel(long n, double c1, double c2, const R *invd, const R *r, const R *t,
                                 R *d, R *z)
{
  const long stride = (long)gridDim.x * blockDim.x;
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  for (; i + (kU - 1) * stride < n; i += kU * stride) {
    R vi[kU], vr[kU], vt[kU], vd[kU], vz[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const long j = i + u * stride;
      vi[u] = invd[j];
      vr[u] = r[j];
      vt[u] = t[j];
      vd[u] = d[j];
      vz[u] = z[j];
    }
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const R v = (R)(c1 * (double)vd[u] + c2 * (double)(vi[u] * (vr[u] - vt[u])));
      d[i + u * stride] = v;
      z[i + u * stride] = vz[u] + v;
    }
  }
  for (; i < n; i += stride) {
    const R v = (R)(c1 * (double)d[i] + c2 * (double)(invd[i] * (r[i] - t[i])));
    d[i] = v;
    z[i] += v;
  }
}

// ------------------------------------------------------------------ host side

namespace {
unsigned vgrid(long n)
{
  long g = (n + 255) / 256;
  if (g > 148L * 16) g = 148L * 16;
  if (g < 1) g = 1;
  return (unsigned)g;
}
// blocks of 256 threads for an unrolled elementwise kernel: one pass of kU
// elements per thread where n allows, at most 16 blocks per SM
unsigned vgrid4(long n)
{
  long g = (n + 256 * kU - 1) / (256 * kU);
  if (g > 148L * 16) g = 148L * 16;
  if (g < 1) g = 1;
  return (unsigned)g;
}
}  // namespace

void dev_dot(const double *a, const double *b, long n, double *partial, double *out, cudaStream_t s)
{
  dot_partial_kernel<double, double><<<kRedBlocks, kRedThreads, 0, s>>>(a, b, n, partial);
  MPDG_LAUNCHED();
  finish_kernel<<<1, kRedThreads, 0, s>>>(partial, 1, out, 0);
  MPDG_LAUNCHED();
}

void dev_dot_f(const float *a, const float *b, long n, double *partial, double *out, cudaStream_t s)
{
  dot_partial_kernel<float, float><<<kRedBlocks, kRedThreads, 0, s>>>(a, b, n, partial);
  MPDG_LAUNCHED();
  finish_kernel<<<1, kRedThreads, 0, s>>>(partial, 1, out, 0);
  MPDG_LAUNCHED();
}

void dev_linf(const double *a, long n, double *partial, double *out, cudaStream_t s)
{
  linf_partial_kernel<<<kRedBlocks, kRedThreads, 0, s>>>(a, n, partial);
  MPDG_LAUNCHED();
  finish_kernel<<<1, kRedThreads, 0, s>>>(partial, 1, out, 1);
  MPDG_LAUNCHED();
}

template <typename R>
void dev_mdot2(const R *V, long n, int m, const R *u, const R *w, double *partial, double *out, cudaStream_t s)
{
  if (w)
    mdot2_partial_kernel<R, true><<<kRedBlocks, kRedThreads, 0, s>>>(V, n, m, u, w, partial);
  else
    mdot2_partial_kernel<R, false><<<kRedBlocks, kRedThreads, 0, s>>>(V, n, m, u, w, partial);
  MPDG_LAUNCHED();
  const int groups = w ? 2 * m : m;
  finish_kernel<<<groups, kRedThreads, 0, s>>>(partial, groups, out, 0);
  MPDG_LAUNCHED();
}
template void dev_mdot2<double>(const double *, long, int, const double *, const double *, double *, double *,
                                cudaStream_t);
template void dev_mdot2<float>(const float *, long, int, const float *, const float *, double *, double *,
                               cudaStream_t);

template <typename R>
void dev_dcgs2_sweep(R *V, long n, int j, double inv_alpha, const DcgsCoef &cf, cudaStream_t s)
{
  dcgs2_sweep_kernel<R><<<vgrid(n), 256, 0, s>>>(V, n, j, inv_alpha, cf);
  MPDG_LAUNCHED();
}
template void dev_dcgs2_sweep<double>(double *, long, int, double, const DcgsCoef &, cudaStream_t);
template void dev_dcgs2_sweep<float>(float *, long, int, double, const DcgsCoef &, cudaStream_t);

template <typename R>
void dev_combine(const R *V, long n, int m, const double *y, R *x, cudaStream_t s)
{
  combine_kernel<R><<<vgrid(n), 256, 0, s>>>(V, n, m, y, x);
  MPDG_LAUNCHED();
}
template void dev_combine<double>(const double *, long, int, const double *, double *, cudaStream_t);
template void dev_combine<float>(const float *, long, int, const double *, float *, cudaStream_t);

template <typename R>
void dev_axpby(long n, double a, const R *x, double b, R *y, cudaStream_t s)
{
  axpby_kernel<R><<<vgrid4(n), 256, 0, s>>>(n, a, x, b, y);
  MPDG_LAUNCHED();
}
template void dev_axpby<double>(long, double, const double *, double, double *, cudaStream_t);
template void dev_axpby<float>(long, double, const float *, double, float *, cudaStream_t);

void dev_residual(long n, const double *b, double *y, cudaStream_t s)
{
  residual_kernel<<<vgrid(n), 256, 0, s>>>(n, b, y);
  MPDG_LAUNCHED();
}

template <typename R>
void dev_scale_copy(long n, double a, const double *x, R *y, cudaStream_t s)
{
  scale_copy_kernel<R><<<vgrid(n), 256, 0, s>>>(n, a, x, y);
  MPDG_LAUNCHED();
}
template void dev_scale_copy<double>(long, double, const double *, double *, cudaStream_t);
template void dev_scale_copy<float>(long, double, const double *, float *, cudaStream_t);

template <typename R>
void dev_add_scaled(long n, double a, const R *x, double *y, cudaStream_t s)
{
  add_scaled_kernel<R><<<vgrid(n), 256, 0, s>>>(n, a, x, y);
  MPDG_LAUNCHED();
}
template void dev_add_scaled<double>(long, double, const double *, double *, cudaStream_t);
template void dev_add_scaled<float>(long, double, const float *, double *, cudaStream_t);

template <typename R>
void dev_mul(long n, const R *d, const R *x, R *y, cudaStream_t s)
{
  mul_kernel<R><<<vgrid(n), 256, 0, s>>>(n, d, x, y);
  MPDG_LAUNCHED();
}
template void dev_mul<double>(long, const double *, const double *, double *, cudaStream_t);
template void dev_mul<float>(long, const float *, const float *, float *, cudaStream_t);

template <typename R, typename RX>
void dev_cg_update(long n, double *s, RX *x, R *r, const R *p, const R *Ap, const R *invd, R *z,
                   double *partial, cudaStream_t st, double xscale)
{
  cg_update_kernel<R, RX><<<kRedBlocks, kRedThreads, 0, st>>>(n, s, x, r, p, Ap, invd, z, partial,
                                                              xscale);
  MPDG_LAUNCHED();
  // rr -> s[kRR]; rz -> s[kRZNEW]
  finish_kernel<<<1, kRedThreads, 0, st>>>(partial, 1, s + kRR, 0);
  MPDG_LAUNCHED();
  if (invd) {
    finish_kernel<<<1, kRedThreads, 0, st>>>(partial + kRedBlocks, 1, s + kRZNEW, 0);
    MPDG_LAUNCHED();
  }
}
template void dev_cg_update<double, double>(long, double *, double *, double *, const double *,
                                            const double *, const double *, double *, double *,
                                            cudaStream_t, double);
template void dev_cg_update<float, float>(long, double *, float *, float *, const float *,
                                          const float *, const float *, float *, double *,
                                          cudaStream_t, double);
template void dev_cg_update<float, double>(long, double *, double *, float *, const float *,
                                           const float *, const float *, float *, double *,
                                           cudaStream_t, double);

template <typename R>
void dev_cg_direction(long n, double *s, R *p, const R *z, cudaStream_t st)
{
  cg_direction_kernel<R><<<vgrid4(n), 256, 0, st>>>(n, s, p, z);
  MPDG_LAUNCHED();
  shift_scalar_kernel<<<1, 1, 0, st>>>(s);
  MPDG_LAUNCHED();
}
template void dev_cg_direction<double>(long, double *, double *, const double *, cudaStream_t);
template void dev_cg_direction<float>(long, double *, float *, const float *, cudaStream_t);

template <typename R, typename RX>
void dev_cg_update_lagged(long n, double *s, RX *x, R *r, const R *p, const R *Ap, const R *invd, R *z,
                          double *partial, cudaStream_t st)
{
  cg_update_kernel<R, RX, true><<<kRedBlocks, kRedThreads, 0, st>>>(n, s, x, r, p, Ap, invd, z, partial, 1.0);
  MPDG_LAUNCHED();
  finish_kernel<<<1, kRedThreads, 0, st>>>(partial, 1, s + kRR, 0);
  MPDG_LAUNCHED();
  if (invd) {
    finish_kernel<<<1, kRedThreads, 0, st>>>(partial + kRedBlocks, 1, s + kRZNEW, 0);
    MPDG_LAUNCHED();
  }
}
template void dev_cg_update_lagged<double, double>(long, double *, double *, double *, const double *,
                                                   const double *, const double *, double *, double *,
                                                   cudaStream_t);
template void dev_cg_update_lagged<float, float>(long, double *, float *, float *, const float *,
                                                 const float *, const float *, float *, double *,
                                                 cudaStream_t);

template <typename R>
void dev_cg_direction_lagged(long n, double *s, R *p, const R *z, cudaStream_t st)
{
  cg_direction_kernel<R, true><<<vgrid4(n), 256, 0, st>>>(n, s, p, z);
  MPDG_LAUNCHED();
  shift_scalar_lagged_kernel<<<1, 1, 0, st>>>(s);
  MPDG_LAUNCHED();
}
template void dev_cg_direction_lagged<double>(long, double *, double *, const double *, cudaStream_t);
template void dev_cg_direction_lagged<float>(long, double *, float *, const float *, cudaStream_t);

__global__ void cg_check_init_kernel(double *s, double tol)
{
  s[kDONE] = 0.0;
  s[kCONV] = 0.0;
  s[kRRCONV] = 0.0;
  s[kTOL] = tol;
}

void dev_cg_check_init(double *s, double tol, cudaStream_t st)
{
  cg_check_init_kernel<<<1, 1, 0, st>>>(s, tol);
  MPDG_LAUNCHED();
}

void dev_cg_check(double *s, cudaStream_t st)
{
  cg_check_kernel<<<1, 1, 0, st>>>(s);
  MPDG_LAUNCHED();
}

template <typename R>
void dev_cheb_start(long n, double inv_theta, const R *invd, const R *r, R *d, R *z, cudaStream_t s)
{
  cheb_start_kernel<R><<<vgrid4(n), 256, 0, s>>>(n, inv_theta, invd, r, d, z);
  MPDG_LAUNCHED();
}
template void dev_cheb_start<double>(long, double, const double *, const double *, double *,
                                     double *, cudaStream_t);
template void dev_cheb_start<float>(long, double, const float *, const float *, float *, float *,
                                    cudaStream_t);

template <typename R>
void dev_cheb_step(long n, double c1, double c2, const R *invd, const R *r, const R *t, R *d, R *z,
                   cudaStream_t s)
{
  cheb_step_kernel<R><<<vgrid4(n), 256, 0, s>>>(n, c1, c2, invd, r, t, d, z);
  MPDG_LAUNCHED();
}
template void dev_cheb_step<double>(long, double, double, const double *, const double *,
                                    const double *, double *, double *, cudaStream_t);
template void dev_cheb_step<float>(long, double, double, const float *, const float *, const float *,
                                   float *, float *, cudaStream_t);

template <typename R>
__global__ void copy_kernel(long n, const R *x, R *y)
{
  const long stride = (long)gridDim.x * blockDim.x;
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  for (; i + (kU - 1) * stride < n; i += kU * stride) {
    R v[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) v[u] = x[i + u * stride];
#pragma unroll
    for (int u = 0; u < kU; ++u) y[i + u * stride] = v[u];
  }
  for (; i < n; i += stride) y[i] = x[i];
}

template <typename R>
void dev_copy(long n, const R *x, R *y, cudaStream_t s)
{
  copy_kernel<R><<<vgrid4(n), 256, 0, s>>>(n, x, y);
  MPDG_LAUNCHED();
}
template void dev_copy<double>(long, const double *, double *, cudaStream_t);
template void dev_copy<float>(long, const float *, float *, cudaStream_t);

}  // namespace mpdg
