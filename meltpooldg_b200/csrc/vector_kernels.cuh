// Host launchers of the solver vector kernels (vector_kernels.cu).
#pragma once

#include <cuda_runtime.h>

namespace mpdg {

constexpr int kRedThreads = 256;  // threads per reduction block
constexpr int kRedBlocks = 592;   // 4 blocks per SM on 148 SMs: fixed, so sums are deterministic

// slots of the device scalar array used by the CG kernels
enum { kRZ = 0, kRZNEW = 1, kPAP = 2, kRR = 3, kNScalars = 8 };
// CG with the convergence test on the device (dev_cg_check): the solve's state
// (0 running, 1 converged, 2 not finite), the iteration it stopped at, r.r
// there, and the tolerance on |r|
enum { kDONE = 4, kCONV = 5, kRRCONV = 6, kTOL = 7 };

void dev_dot(const double *a, const double *b, long n, double *partial, double *out, cudaStream_t s);
void dev_dot_f(const float *a, const float *b, long n, double *partial, double *out, cudaStream_t s);
void dev_linf(const double *a, long n, double *partial, double *out, cudaStream_t s);
// delayed classical Gram-Schmidt (GMRES): the dots V_k.u and, when w is given,
// V_k.w for k < m (out[k], out[m + k]), one pass over the basis
template <typename R>
void dev_mdot2(const R *V, long n, int m, const R *u, const R *w, double *partial, double *out, cudaStream_t s);
// coefficients of one sweep, passed by value (restart length <= 60)
struct DcgsCoef {
  double s[64];
  double c[64];
};
// q_j = (V_j - V s) / alpha over V_j; V_{j+1} = V_{j+1} / alpha - V c - c_j q_j
template <typename R>
void dev_dcgs2_sweep(R *V, long n, int j, double inv_alpha, const DcgsCoef &cf, cudaStream_t s);

template <typename R>
void dev_combine(const R *V, long n, int m, const double *y, R *x, cudaStream_t s);
template <typename R>
void dev_axpby(long n, double a, const R *x, double b, R *y, cudaStream_t s);
void dev_residual(long n, const double *b, double *y, cudaStream_t s);
template <typename R>
void dev_scale_copy(long n, double a, const double *x, R *y, cudaStream_t s);
template <typename R>
void dev_add_scaled(long n, double a, const R *x, double *y, cudaStream_t s);
template <typename R>
void dev_mul(long n, const R *d, const R *x, R *y, cudaStream_t s);
template <typename R, typename RX>
void dev_cg_update(long n, double *s, RX *x, R *r, const R *p, const R *Ap, const R *invd, R *z,
                   double *partial, cudaStream_t st, double xscale = 1.0);
template <typename R>
void dev_cg_direction(long n, double *s, R *p, const R *z, cudaStream_t st);
// the same two steps, skipped once s[kDONE] is set, and the device-side test
// that counts the iteration in s[kCONV] and sets s[kDONE] (|r| <= s[kTOL], or
// r.r not finite)
template <typename R, typename RX>
void dev_cg_update_lagged(long n, double *s, RX *x, R *r, const R *p, const R *Ap, const R *invd, R *z,
                          double *partial, cudaStream_t st);
template <typename R>
void dev_cg_direction_lagged(long n, double *s, R *p, const R *z, cudaStream_t st);
void dev_cg_check(double *s, cudaStream_t st);
// resets the state slots and sets the tolerance
void dev_cg_check_init(double *s, double tol, cudaStream_t st);
template <typename R>
void dev_cheb_start(long n, double inv_theta, const R *invd, const R *r, R *d, R *z, cudaStream_t s);
template <typename R>
void dev_cheb_step(long n, double c1, double c2, const R *invd, const R *r, const R *t, R *d, R *z,
                   cudaStream_t s);
template <typename R>
void dev_copy(long n, const R *x, R *y, cudaStream_t s);

}  // namespace mpdg
