// Least-squares-projection predictor (LeastSquaresProjection::vmult,
// include/meltpooldg/linear_algebra/predictor.hpp:37-80) on the device.
//
// The initial guess of a time step is the combination of the k old solutions
// x_s whose image A x_s comes closest to the right-hand side b.  The k images
// come from one multi-vector apply (the coefficient stream is read once per
// pass of up to four vectors instead of once per vector), then they are
// orthogonalised in place by the reference's modified Gram-Schmidt recurrence
// (P(0,s) = w_s.w_0; w_s -= P(j,s)/P(j,j) w_j, P(j+1,s) = w_s.w_{j+1}; stop when
// P(s,s) < 1e-16 P(0,0)), the coefficients follow by back substitution of
// P c = (w_s.b), and x = sum_s c_s x_s.  Dot products use the deterministic
// fixed-grid reductions of the solvers; the k x k recurrence runs on the host.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "mpdg_internal.h"
#include "vector_kernels.cuh"

namespace mpdg {

namespace {

struct DotScratch {
  double *partial = nullptr, *out = nullptr;
  ~DotScratch()
  {
    if (partial) cudaFree(partial);
    if (out) cudaFree(out);
  }
};

double dot(const double *a, const double *b, long n, DotScratch &d, cudaStream_t s)
{
  double h = 0.0;
  dev_dot(a, b, n, d.partial, d.out, s);
  MPDG_CUDA(cudaMemcpyAsync(&h, d.out, sizeof(double), cudaMemcpyDeviceToHost, s));
  MPDG_CUDA(cudaStreamSynchronize(s));
  return h;
}

}  // namespace

int predict_lsq(Op &op, int n_old, const double *const *old, const double *rhs, double *solution)
{
  const long N = op.mesh->N;
  const cudaStream_t s = op.stream;
  if (n_old < 1 || n_old > kMaxLsqVectors) throw Error{MPDG_ERR_ARG, "1 to 32 old solutions"};
  if (!rhs || !solution) throw Error{MPDG_ERR_ARG, "null vector"};
  for (int i = 0; i < n_old; ++i)
    if (!old[i]) throw Error{MPDG_ERR_ARG, "null old solution"};
  if (op.lsq_cols < n_old) {
    MPDG_CUDA(cudaStreamSynchronize(s));
    if (op.lsq_buf) cudaFree(op.lsq_buf);
    op.lsq_buf = nullptr;
    op.lsq_cols = 0;
    const cudaError_t e = tracked_malloc(&op.lsq_buf, sizeof(double) * (size_t)N * n_old);
    if (e != cudaSuccess) throw Error{MPDG_ERR_ALLOC, "predictor images"};
    op.lsq_cols = n_old;
    op.device_bytes += sizeof(double) * (size_t)N * n_old;
  }
  DotScratch d;
  MPDG_CUDA(tracked_malloc(&d.partial, sizeof(double) * kRedBlocks));
  MPDG_CUDA(tracked_malloc(&d.out, sizeof(double)));
  std::vector<double *> w(n_old);
  for (int i = 0; i < n_old; ++i) w[i] = op.lsq_buf + (size_t)i * N;
  // images of every old solution in passes of up to four vectors
  launch_apply_multi<double>(op, n_old, w.data(), old);

  // modified Gram-Schmidt on the images (predictor.hpp:47-62)
  std::vector<double> P((size_t)n_old * n_old, 0.0);
  auto Pm = [&](int r, int c) -> double & { return P[(size_t)r * n_old + c]; };
  int step = 0;
  for (; step < n_old; ++step) {
    Pm(0, step) = dot(w[step], w[0], N, d, s);
    for (int j = 0; j < step; ++j) {
      dev_axpby<double>(N, -Pm(j, step) / Pm(j, j), w[j], 1.0, w[step], s);
      Pm(j + 1, step) = dot(w[step], w[j + 1], N, d, s);
    }
    if (Pm(step, step) < 1e-16 * Pm(0, 0)) break;
  }
  // least-squares coefficients by back substitution (predictor.hpp:64-75)
  std::vector<double> c(step > 0 ? step : 1, 0.0);
  for (int k = 0; k < step; ++k) c[k] = dot(w[k], rhs, N, d, s);
  for (int k = step - 1; k >= 0; --k) {
    double sum = c[k];
    for (int j = k + 1; j < step; ++j) sum -= c[j] * Pm(k, j);
    c[k] = sum / Pm(k, k);
  }
  // extrapolation from the old solutions (predictor.hpp:77-80)
  if (step == 0) {
    MPDG_CUDA(cudaMemsetAsync(solution, 0, sizeof(double) * N, s));
  } else {
    dev_scale_copy<double>(N, c[0], old[0], solution, s);
    for (int k = 1; k < step; ++k) dev_add_scaled<double>(N, c[k], old[k], solution, s);
  }
  MPDG_CUDA(cudaStreamSynchronize(s));
  return step;
}

}  // namespace mpdg
