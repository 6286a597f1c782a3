// Krylov solvers on the device: preconditioned CG and right-preconditioned
// restarted GMRES with deal.II ReductionControl semantics
// (include/meltpooldg/linear_algebra/linear_solver.hpp:26-134: converged when
// |r_k|_2 <= max(abs_tol, rel_tol |r_0|_2)), the Jacobi preconditioner of
// include/meltpooldg/linear_algebra/preconditioner_jacobi.hpp:50-69, a Chebyshev
// smoother over it, and the FP32-inner / FP64-defect-correction driver.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <random>
#include <vector>

#include "mpdg_internal.h"
#include "vector_kernels.cuh"

namespace mpdg {

struct Workspace {
  long N = 0;
  // FP64 vectors
  double *r = nullptr, *z = nullptr, *p = nullptr, *Ap = nullptr, *invd = nullptr, *cd = nullptr,
         *ct = nullptr;
  // FP32 vectors
  float *r32 = nullptr, *z32 = nullptr, *p32 = nullptr, *Ap32 = nullptr, *x32 = nullptr,
        *invd32 = nullptr, *cd32 = nullptr, *ct32 = nullptr;
  double *V = nullptr;  // GMRES basis (FP64)
  int V_cols = 0;
  float *V32 = nullptr;  // GMRES basis (FP32 inner solves)
  int V32_cols = 0;
  double *partial = nullptr;  // reduction partials: 128 groups of kRedBlocks
  double *scal = nullptr;     // device scalars (kNScalars) + GMRES dots (128)
  double *host = nullptr;     // pinned host mirror
  size_t bytes = 0;
};

namespace {

template <typename T>
T *walloc(Workspace &w, size_t count)
{
  T *p = nullptr;
  cudaError_t e = tracked_malloc(&p, count * sizeof(T));
  if (e != cudaSuccess) throw Error{MPDG_ERR_ALLOC, std::string("cudaMalloc: ") + cudaGetErrorString(e)};
  w.bytes += count * sizeof(T);
  return p;
}

Workspace &ws64(Op &op)
{
  if (!op.ws) op.ws = new Workspace();
  Workspace &w = *op.ws;
  const long N = op.mesh->N;
  w.N = N;
  if (!w.r) {
    w.r = walloc<double>(w, N);
    w.z = walloc<double>(w, N);
    w.p = walloc<double>(w, N);
    w.Ap = walloc<double>(w, N);
    w.invd = walloc<double>(w, N);
    w.cd = walloc<double>(w, N);
    w.ct = walloc<double>(w, N);
    w.partial = walloc<double>(w, 128L * kRedBlocks);
    w.scal = walloc<double>(w, kNScalars + 128);
    MPDG_CUDA(tracked_malloc_host(&w.host, sizeof(double) * (kNScalars + 128)));
  }
  return w;
}

Workspace &ws32(Op &op)
{
  Workspace &w = ws64(op);
  const long N = op.mesh->N;
  if (!w.r32) {
    w.r32 = walloc<float>(w, N);
    w.z32 = walloc<float>(w, N);
    w.p32 = walloc<float>(w, N);
    w.Ap32 = walloc<float>(w, N);
    w.x32 = walloc<float>(w, N);
    w.invd32 = walloc<float>(w, N);
    w.cd32 = walloc<float>(w, N);
    w.ct32 = walloc<float>(w, N);
  }
  return w;
}

double fetch(Op &op, Workspace &w, const double *dev, int count = 1)
{
  MPDG_CUDA(cudaMemcpyAsync(w.host, dev, sizeof(double) * count, cudaMemcpyDeviceToHost, op.stream));
  MPDG_CUDA(cudaStreamSynchronize(op.stream));
  return w.host[0];
}

struct Prec {
  int kind = MPDG_PREC_JACOBI;
  int degree = 5;
  double lmin = 0, lmax = 0;
};

template <typename R>
struct V {
  R *r, *z, *p, *Ap, *invd, *cd, *ct;
};

V<double> vecs(Workspace &w, double *) { return {w.r, w.z, w.p, w.Ap, w.invd, w.cd, w.ct}; }
V<float> vecs(Workspace &w, float *) { return {w.r32, w.z32, w.p32, w.Ap32, w.invd32, w.cd32, w.ct32}; }

template <typename R>
void prec_apply(Op &op, const Prec &P, const V<R> &v, const R *r, R *z, int &applies)
{
  const long N = op.mesh->N;
  if (P.kind == MPDG_PREC_IDENTITY) {
    dev_copy<R>(N, r, z, op.stream);
    return;
  }
  if (P.kind == MPDG_PREC_JACOBI) {
    dev_mul<R>(N, v.invd, r, z, op.stream);
    return;
  }
  // Chebyshev semi-iteration on D^-1 A over [lmin, lmax], zero start
  const double theta = 0.5 * (P.lmax + P.lmin), delta = 0.5 * (P.lmax - P.lmin);
  const double sigma = theta / delta;
  double rho = 1.0 / sigma;
  dev_cheb_start<R>(N, 1.0 / theta, v.invd, r, v.cd, z, op.stream);
  for (int k = 1; k < P.degree; ++k) {
    launch_apply<R>(op, v.ct, z);
    ++applies;
    const double rho_new = 1.0 / (2.0 * sigma - rho);
    dev_cheb_step<R>(N, rho_new * rho, 2.0 * rho_new / delta, v.invd, r, v.ct, v.cd, z, op.stream);
    rho = rho_new;
  }
}

// preconditioned CG; returns MPDG_OK / error; deal.II SolverCG recurrence
template <typename R>
int pcg(Op &op, Workspace &w, const Prec &P, const R *b, R *x, bool x_is_zero, double rel_tol,
        double abs_tol, int max_it, int &iters, double &res0, double &res, int &applies)
{
  const long N = op.mesh->N;
  V<R> v = vecs(w, (R *)nullptr);
  cudaStream_t s = op.stream;
  double *sc = w.scal;
  if (x_is_zero) {
    dev_copy<R>(N, b, v.r, s);
  } else {
    launch_apply<R>(op, v.Ap, x);
    ++applies;
    dev_copy<R>(N, b, v.r, s);
    dev_axpby<R>(N, -1.0, v.Ap, 1.0, v.r, s);
  }
  if (sizeof(R) == 8)
    dev_dot((const double *)v.r, (const double *)v.r, N, w.partial, sc + kRR, s);
  else
    dev_dot_f((const float *)v.r, (const float *)v.r, N, w.partial, sc + kRR, s);
  res0 = std::sqrt(fetch(op, w, sc + kRR));
  res = res0;
  iters = 0;
  if (!std::isfinite(res0)) return MPDG_ERR_NAN;
  const double tol = std::fmax(abs_tol, rel_tol * res0);
  if (res0 <= tol) return MPDG_OK;
  prec_apply<R>(op, P, v, v.r, v.z, applies);
  auto dot_into = [&](const R *a, const R *bb, double *out) {
    if (sizeof(R) == 8)
      dev_dot((const double *)a, (const double *)bb, N, w.partial, out, s);
    else
      dev_dot_f((const float *)a, (const float *)bb, N, w.partial, out, s);
  };
  dot_into(v.r, v.z, sc + kRZ);
  dev_copy<R>(N, v.z, v.p, s);
  const bool fused_jacobi = P.kind == MPDG_PREC_JACOBI;
  // The test |r| <= tol runs on the device after every iteration
  // (dev_cg_check); the host reads its verdict every K iterations.  On small
  // problems the round trip costs more than the iterations launched past
  // convergence, whose updates are skipped (x, r, p stay those of the
  // converged iteration: the result, the iteration count and the residual are
  // the per-iteration test's).
  const int K = (N <= (4L << 20)) ? 4 : 1;
  dev_cg_check_init(sc, tol, s);
  const int applies0 = applies;
  int prec_count = 0, launched = 0;
  auto report = [&](int it) {
    iters = it;
    applies = applies0 + it + (it > 0 ? (it - 1) * prec_count : 0);
  };
  auto run_batch = [&](int batch) {
    for (int bi = 0; bi < batch; ++bi) {
      launch_apply<R>(op, v.Ap, v.p);
      dot_into(v.p, v.Ap, sc + kPAP);
      dev_cg_update_lagged<R, R>(N, sc, x, v.r, v.p, v.Ap, fused_jacobi ? v.invd : nullptr, v.z, w.partial, s);
      dev_cg_check(sc, s);
      if (!fused_jacobi) {
        int pa = 0;
        prec_apply<R>(op, P, v, v.r, v.z, pa);
        prec_count = pa;
        dot_into(v.r, v.z, sc + kRZNEW);
      }
      dev_cg_direction_lagged<R>(N, sc, v.p, v.z, s);
    }
  };
  // Batches after the first replay one CUDA graph of K iterations (the launch
  // sequence is the same every time: pointers fixed, scalars and the
  // iteration count on the device), which removes the per-kernel launch cost
  // that dominates small solves.  Captured on a stream of its own; if the
  // capture fails, the batches run launch by launch.
  cudaGraphExec_t gexec = nullptr;
  int64_t graph_kernels = 0;
  bool graph_tried = false;
  struct GraphGuard {
    cudaGraphExec_t &g;
    ~GraphGuard()
    {
      if (g) cudaGraphExecDestroy(g);
    }
  } guard{gexec};
  auto capture = [&]() {
    graph_tried = true;
    cudaStream_t cap = nullptr;
    if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    const cudaStream_t saved = op.stream;
    const int64_t k0 = mpdg_kernel_launches();
    cudaGraph_t g = nullptr;
    bool ok = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
      op.stream = cap;
      s = cap;
      try {
        run_batch(K);
      } catch (...) {
        ok = false;
      }
      op.stream = saved;
      s = saved;
      ok = (cudaStreamEndCapture(cap, &g) == cudaSuccess) && ok && g != nullptr;
      if (ok) ok = cudaGraphInstantiate(&gexec, g, 0) == cudaSuccess;
      if (g) cudaGraphDestroy(g);
    }
    cudaStreamDestroy(cap);
    cudaGetLastError();  // a failed capture leaves no sticky error
    graph_kernels = mpdg_kernel_launches() - k0;
    count_launch((int)-graph_kernels);  // captured, not run: counted at each replay
    if (!ok && gexec) {
      cudaGraphExecDestroy(gexec);
      gexec = nullptr;
    }
  };
  while (true) {
    const int batch = std::min(K, max_it - launched);
    if (K > 1 && batch == K && launched > 0 && !graph_tried) capture();
    if (gexec && batch == K) {
      MPDG_CUDA(cudaGraphLaunch(gexec, op.stream));
      count_launch((int)graph_kernels);
    } else {
      run_batch(batch);
    }
    launched += batch;
    fetch(op, w, sc + kDONE, 3);
    const double done = w.host[0], conv = w.host[1], rr = w.host[2];
    if (done == 1.0) {
      report((int)conv);
      res = std::sqrt(rr);
      return MPDG_OK;
    }
    if (done != 0.0) {
      report((int)conv);
      res = std::sqrt(rr);
      return MPDG_ERR_NAN;
    }
    if (launched >= max_it) {
      report(launched);
      res = std::sqrt(fetch(op, w, sc + kRR));
      return MPDG_ERR_NOT_CONVERGED;
    }
  }
}

// FP32-inner CG with reliable updates: one FP32 CG recurrence (operator and
// preconditioner in FP32, dot products accumulated in FP64) on the system
// scaled by 1/|r0|; the solution is accumulated in FP64 (x += |r0| alpha p),
// and whenever the iterated FP32 residual has dropped by `delta` since the
// last true residual, the FP64 defect b - A x is computed and replaces it.
// The search direction is kept, so no Krylov information is lost to restarts.
int pcg_reliable(Op &op, Workspace &w, const Prec &P, const double *b, double *x, double rel_tol,
                 double abs_tol, int max_it, double delta, int &iters, int &updates, double &res0,
                 double &res, int &applies)
{
  const long N = op.mesh->N;
  cudaStream_t s = op.stream;
  V<float> v = vecs(w, (float *)nullptr);
  double *sc = w.scal;
  auto true_residual = [&]() {
    launch_apply<double>(op, w.Ap, x);
    ++applies;
    dev_copy<double>(N, b, w.r, s);
    dev_axpby<double>(N, -1.0, w.Ap, 1.0, w.r, s);
    dev_dot(w.r, w.r, N, w.partial, sc + kRR, s);
    return std::sqrt(fetch(op, w, sc + kRR));
  };
  res0 = true_residual();
  res = res0;
  iters = 0;
  updates = 0;
  if (!std::isfinite(res0)) return MPDG_ERR_NAN;
  const double tol = std::fmax(abs_tol, rel_tol * res0);
  if (res0 <= tol) return MPDG_OK;
  const double scale = res0;
  dev_scale_copy<float>(N, 1.0 / scale, w.r, v.r, s);
  auto precondition = [&]() {
    prec_apply<float>(op, P, v, v.r, v.z, applies);
    dev_dot_f(v.r, v.z, N, w.partial, sc + kRZNEW, s);
  };
  precondition();
  dev_copy<float>(N, v.z, v.p, s);
  // rz <- rz_new
  MPDG_CUDA(cudaMemcpyAsync(sc + kRZ, sc + kRZNEW, sizeof(double), cudaMemcpyDeviceToDevice, s));
  double rmax = 1.0;  // iterated residual at the last true residual, scaled
  const bool fused_jacobi = P.kind == MPDG_PREC_JACOBI;
  while (true) {
    launch_apply<float>(op, v.Ap, v.p);
    ++applies;
    dev_dot_f(v.p, v.Ap, N, w.partial, sc + kPAP, s);
    dev_cg_update<float, double>(N, sc, x, v.r, v.p, v.Ap, fused_jacobi ? v.invd : nullptr, v.z,
                                 w.partial, s, scale);
    ++iters;
    const double rel = std::sqrt(fetch(op, w, sc + kRR));
    if (!std::isfinite(rel)) return MPDG_ERR_NAN;
    bool replaced = false;
    if (rel * scale <= tol || rel < delta * rmax) {
      res = true_residual();
      ++updates;
      if (!std::isfinite(res)) return MPDG_ERR_NAN;
      if (res <= tol) return MPDG_OK;
      dev_scale_copy<float>(N, 1.0 / scale, w.r, v.r, s);
      rmax = res / scale;
      replaced = true;
    } else {
      res = rel * scale;
    }
    if (iters >= max_it) return MPDG_ERR_NOT_CONVERGED;
    if (!fused_jacobi || replaced) precondition();
    dev_cg_direction<float>(N, sc, v.p, v.z, s);
  }
}

template <typename R>
R *&gmres_basis(Workspace &w, int *&cols);
template <>
double *&gmres_basis<double>(Workspace &w, int *&cols)
{
  cols = &w.V_cols;
  return w.V;
}
template <>
float *&gmres_basis<float>(Workspace &w, int *&cols)
{
  cols = &w.V32_cols;
  return w.V32;
}

template <typename R>
void dot_any(const R *a, const R *b, long n, double *partial, double *out, cudaStream_t s)
{
  if constexpr (sizeof(R) == 8) dev_dot(a, b, n, partial, out, s);
  else dev_dot_f(a, b, n, partial, out, s);
}

// Right-preconditioned restarted GMRES, vectors in R, Hessenberg and dot
// products in FP64.  The Arnoldi basis is orthogonalised by delayed classical
// Gram-Schmidt with re-orthogonalisation (DCGS2: Swirydowicz, Langou,
// Ananthan, Yang and Thomas, "Low synchronization Gram-Schmidt and generalized
// minimal residual algorithms", Numer. Linear Algebra Appl. 28, 2021).  Step j
// holds q_0..q_{j-1} final and u_j, the once-projected candidate for q_j:
//   w = B u_j                               (B = A M^-1; one apply)
//   s = Q_{j-1}^T u_j, t = u_j.u_j, z = Q_{j-1}^T w, y = u_j.w   (one pass)
//   alpha = |u_j - Q_{j-1} s| = sqrt(t - s.s)
//   column j-1 of H gets + s and alpha below the diagonal: its Givens
//   rotation gives the residual estimate of step j-1
//   c = Q_j^T w / alpha (q_j.w = (y - s.z) / alpha)
//   H[:, j] = c - H_{j-1} s / alpha   (B Q_{j-1} = Q_j H_{j-1})
//   q_j = (u_j - Q_{j-1} s) / alpha, u_{j+1} = w / alpha - Q_j c   (one sweep)
// which is two passes of classical Gram-Schmidt with the second pass of each
// vector made in the next step: one read of the basis for the dots and one for
// the update per iteration, and one host round trip.  The residual estimate
// lags by one apply, so each cycle applies B once more than it iterates.
template <typename R>
int gmres(Op &op, Workspace &w, const Prec &P, const R *b, R *x, bool x_is_zero, double rel_tol,
          double abs_tol, int max_it, int restart, int &iters, double &res0, double &res,
          int &applies)
{
  const long N = op.mesh->N;
  cudaStream_t s = op.stream;
  V<R> v = vecs(w, (R *)nullptr);
  const int m = std::max(1, std::min(restart, 60));
  int *cols = nullptr;
  R *&VB = gmres_basis<R>(w, cols);
  if (!VB || *cols < m + 1) {
    if (VB) cudaFree(VB);
    VB = walloc<R>(w, (size_t)N * (m + 1));
    *cols = m + 1;
  }
  // H: the Arnoldi Hessenberg; Hr: its Givens-rotated copy (least squares)
  std::vector<double> H((m + 1) * m, 0.0), Hr((m + 1) * m, 0.0), cs(m), sn(m), g(m + 1), y(m);
  DcgsCoef cf;
  double *dsc = w.scal + kNScalars;
  iters = 0;
  double tol = -1.0;
  int status = MPDG_ERR_NOT_CONVERGED;
  bool first = true;
  while (true) {
    if (first && x_is_zero) {
      dev_copy<R>(N, b, VB, s);
    } else {
      launch_apply<R>(op, v.Ap, x);
      ++applies;
      dev_copy<R>(N, b, VB, s);
      dev_axpby<R>(N, -1.0, v.Ap, 1.0, VB, s);
    }
    first = false;
    dot_any<R>(VB, VB, N, w.partial, w.scal + kRR, s);
    const double beta = std::sqrt(fetch(op, w, w.scal + kRR));
    if (tol < 0.0) {
      res0 = beta;
      tol = std::fmax(abs_tol, rel_tol * beta);
    }
    res = beta;
    if (!std::isfinite(beta)) return MPDG_ERR_NAN;
    if (beta <= tol) {
      status = MPDG_OK;
      break;
    }
    if (iters >= max_it) break;
    dev_axpby<R>(N, 0.0, VB, 1.0 / beta, VB, s);
    std::fill(g.begin(), g.end(), 0.0);
    std::fill(H.begin(), H.end(), 0.0);
    g[0] = beta;
    const int it0 = iters;
    int k = 0;  // final columns of this cycle
    bool done = false;
    for (int j = 0;; ++j) {
      R *uj = VB + (long)j * N, *wn = VB + (long)(j + 1) * N;
      // no further apply once the cycle or the iteration budget is full: the
      // step only completes column j-1
      const bool last = j == m || it0 + j >= max_it;
      if (!last) {
        prec_apply<R>(op, P, v, uj, v.z, applies);
        launch_apply<R>(op, wn, v.z);
        ++applies;
      }
      dev_mdot2<R>(VB, N, j + 1, uj, last ? nullptr : wn, w.partial, dsc, s);
      const int cnt = last ? j + 1 : 2 * (j + 1);
      MPDG_CUDA(cudaMemcpyAsync(w.host, dsc, sizeof(double) * cnt, cudaMemcpyDeviceToHost, s));
      MPDG_CUDA(cudaStreamSynchronize(s));
      const double *hs = w.host, *hz = w.host + (j + 1);
      double ss = 0.0, sz = 0.0;
      for (int i = 0; i < j; ++i) {
        ss += hs[i] * hs[i];
        if (!last) sz += hs[i] * hz[i];
      }
      const double t = hs[j], a2 = t - ss;
      if (!std::isfinite(t) || !std::isfinite(a2) || !std::isfinite(sz)) return MPDG_ERR_NAN;
      const double alpha = a2 > 1e-28 * t ? std::sqrt(a2) : 0.0;
      if (j > 0) {
        // column j-1 is final: + s, alpha below the diagonal; its rotation
        const int jc = j - 1;
        for (int i = 0; i < j; ++i) H[i * m + jc] += hs[i];
        H[j * m + jc] = alpha;
        for (int i = 0; i <= j; ++i) Hr[i * m + jc] = H[i * m + jc];
        for (int i = 0; i < jc; ++i) {
          const double a = Hr[i * m + jc], c = Hr[(i + 1) * m + jc];
          Hr[i * m + jc] = cs[i] * a + sn[i] * c;
          Hr[(i + 1) * m + jc] = -sn[i] * a + cs[i] * c;
        }
        const double a = Hr[jc * m + jc], c = Hr[j * m + jc], rr = std::sqrt(a * a + c * c);
        cs[jc] = a / rr;
        sn[jc] = c / rr;
        Hr[jc * m + jc] = rr;
        Hr[j * m + jc] = 0.0;
        g[j] = -sn[jc] * g[jc];
        g[jc] = cs[jc] * g[jc];
        ++iters;
        res = std::fabs(g[j]);
        if (!std::isfinite(res)) return MPDG_ERR_NAN;
        if (res <= tol) {
          k = j;
          done = true;
          break;
        }
      }
      if (last || alpha == 0.0) {
        k = j;
        break;
      }
      // column j from the first pass; the sweep makes q_j and u_{j+1}
      const double ia = 1.0 / alpha;
      for (int i = 0; i < j; ++i) {
        cf.s[i] = hs[i];
        cf.c[i] = hz[i] * ia;
      }
      cf.c[j] = (hz[j] - sz) * ia * ia;
      for (int i = 0; i <= j; ++i) {
        double hsum = 0.0;
        for (int l = std::max(0, i - 1); l < j; ++l) hsum += H[i * m + l] * hs[l];
        H[i * m + j] = cf.c[i] - hsum * ia;
      }
      dev_dcgs2_sweep<R>(VB, N, j, ia, cf, s);
    }
    if (k > 0) {
      for (int i = k - 1; i >= 0; --i) {
        double t = g[i];
        for (int l = i + 1; l < k; ++l) t -= Hr[i * m + l] * y[l];
        y[i] = t / Hr[i * m + i];
      }
      MPDG_CUDA(cudaMemcpyAsync(dsc, y.data(), sizeof(double) * k, cudaMemcpyHostToDevice, s));
      // V y into p: the Chebyshev smoother keeps its A z in ct
      dev_combine<R>(VB, N, k, dsc, v.p, s);
      prec_apply<R>(op, P, v, v.p, v.z, applies);
      dev_axpby<R>(N, 1.0, v.z, 1.0, x, s);
      MPDG_CUDA(cudaStreamSynchronize(s));  // y is read from pageable memory
    }
    if (done) {
      status = MPDG_OK;
      break;
    }
    if (iters >= max_it) break;
  }
  return status;
}

// deterministic start vector in [-1, 1) (splitmix64 of the index and the
// seed), zero on constrained DoFs, whose rows of A are zero
__global__ void lanczos_start_kernel(double *v, long n, const uint8_t *mask, unsigned long long seed)
{
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    unsigned long long z = seed + 0x9e3779b97f4a7c15ull * (unsigned long long)(i + 1);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    const double u = (double)(z >> 11) * (1.0 / 9007199254740992.0);  // [0,1)
    v[i] = (mask && mask[i]) ? 0.0 : 2.0 * u - 1.0;
  }
}

// largest eigenvalue of D^-1 A from CG-Lanczos on A x = start
double lanczos_lmax(Op &op, Workspace &w, int steps, int &applies)
{
  const long N = op.mesh->N;
  cudaStream_t s = op.stream;
  double *start = w.cd;
  const uint8_t *mask = (op.use_dirichlet && op.mesh->has_dirichlet) ? op.mesh->d_dmask : nullptr;
  lanczos_start_kernel<<<1184, 256, 0, s>>>(start, N, mask, 4ull);
  MPDG_LAUNCHED();
  double *r = w.r, *z = w.z, *p = w.p, *Ap = w.Ap, *sc = w.scal;
  dev_copy<double>(N, start, r, s);
  dev_mul<double>(N, w.invd, r, z, s);
  dev_copy<double>(N, z, p, s);
  dev_dot(r, z, N, w.partial, sc + kRZ, s);
  std::vector<double> al, be;
  double *xdummy = w.ct;
  MPDG_CUDA(cudaMemsetAsync(xdummy, 0, sizeof(double) * N, s));
  for (int k = 0; k < steps; ++k) {
    launch_apply<double>(op, Ap, p);
    ++applies;
    dev_dot(p, Ap, N, w.partial, sc + kPAP, s);
    dev_cg_update<double, double>(N, sc, xdummy, r, p, Ap, w.invd, z, w.partial, s);
    MPDG_CUDA(cudaMemcpyAsync(w.host, sc, sizeof(double) * 4, cudaMemcpyDeviceToHost, s));
    MPDG_CUDA(cudaStreamSynchronize(s));
    const double rz = w.host[kRZ], rz_new = w.host[kRZNEW], pap = w.host[kPAP];
    if (!(pap > 0) || !(rz > 0)) break;
    al.push_back(rz / pap);
    be.push_back(rz_new / rz);
    dev_cg_direction<double>(N, sc, p, z, s);
    if (!(rz_new > 0)) break;
  }
  const int k = (int)al.size();
  if (k == 0) return 1.0;
  std::vector<double> dg(k), of(k, 0.0);
  for (int j = 0; j < k; ++j) {
    dg[j] = 1.0 / al[j] + (j > 0 ? be[j - 1] / al[j - 1] : 0.0);
    of[j] = (j + 1 < k) ? std::sqrt(be[j]) / al[j] : 0.0;
  }
  double lo = 0.0, hi = 0.0;
  for (int j = 0; j < k; ++j) hi = std::fmax(hi, dg[j] + std::fabs(of[j]) + (j > 0 ? std::fabs(of[j - 1]) : 0.0));
  for (int it = 0; it < 200; ++it) {
    const double mid = 0.5 * (lo + hi);
    int cnt = 0;
    double q = 1.0;
    for (int j = 0; j < k; ++j) {
      q = dg[j] - mid - (j > 0 ? of[j - 1] * of[j - 1] / q : 0.0);
      if (q == 0.0) q = -1e-300;
      if (q < 0.0) ++cnt;
    }
    if (cnt >= k) hi = mid;
    else lo = mid;
  }
  return hi;
}

__global__ void cast_down_kernel(const double *a, float *b, long n)
{
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

}  // namespace

int solve(Op &op, const mpdg_solver_desc &d, double *x, const double *b, mpdg_solve_report &rep)
{
  const auto t0 = std::chrono::steady_clock::now();
  Workspace &w = ws64(op);
  const long N = op.mesh->N;
  cudaStream_t s = op.stream;
  rep = mpdg_solve_report{};
  int applies = 0;
  Prec P;
  P.kind = d.preconditioner;
  P.degree = d.chebyshev_degree > 0 ? d.chebyshev_degree : 5;
  if (P.kind != MPDG_PREC_IDENTITY) {
    launch_diagonal(op, w.invd);
    launch_invert_diagonal(op, w.invd);
  }
  if (P.kind == MPDG_PREC_CHEBYSHEV) {
    const double lam = lanczos_lmax(op, w, d.lanczos_steps > 0 ? d.lanczos_steps : 10, applies);
    const double range = d.chebyshev_range > 0 ? d.chebyshev_range : 30.0;
    const double safety = d.chebyshev_safety > 0 ? d.chebyshev_safety : 1.2;
    P.lmax = safety * lam;
    P.lmin = lam / range;
    rep.lambda_max = lam;
  }
  const double rel = d.rel_tolerance, abs_tol = d.abs_tolerance;
  const int max_it = d.max_iterations > 0 ? d.max_iterations : 10000;
  int status = MPDG_OK;
  double res0 = 0, res = 0;
  if (!d.mixed_precision) {
    int it = 0;
    if (d.solver == MPDG_SOLVER_CG)
      status = pcg<double>(op, w, P, b, x, false, rel, abs_tol, max_it, it, res0, res, applies);
    else
      status = gmres<double>(op, w, P, b, x, false, rel, abs_tol, max_it,
                             d.gmres_restart > 0 ? d.gmres_restart : 30, it, res0, res, applies);
    rep.iterations = it;
  } else {
    Workspace &w32 = ws32(op);
    if (op.T64) ensure_T32(op);
    cast_down_kernel<<<1184, 256, 0, s>>>(w.invd, w32.invd32, N);
    MPDG_LAUNCHED();
    if (d.solver == MPDG_SOLVER_CG) {
      // CG: reliable updates (one FP32 Krylov recurrence, FP64 defects)
      int it = 0, upd = 0;
      status = pcg_reliable(op, w32, P, b, x, rel, abs_tol, max_it,
                            (d.reliable_delta > 0 && d.reliable_delta < 1) ? d.reliable_delta : 0.1, it,
                            upd, res0, res, applies);
      rep.iterations = it;
      rep.outer_iterations = upd;
      MPDG_CUDA(cudaStreamSynchronize(s));
      rep.status = status;
      rep.operator_applies = applies;
      rep.initial_residual = res0;
      rep.final_residual = res;
      rep.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      return status;
    }
    // FP64 defect: r = b - A x
    launch_apply<double>(op, w.Ap, x);
    ++applies;
    dev_copy<double>(N, b, w.r, s);
    dev_axpby<double>(N, -1.0, w.Ap, 1.0, w.r, s);
    dev_dot(w.r, w.r, N, w.partial, w.scal + kRR, s);
    res0 = std::sqrt(fetch(op, w, w.scal + kRR));
    res = res0;
    const double tol = std::fmax(abs_tol, rel * res0);
    const double inner = d.inner_tolerance > 0 ? d.inner_tolerance : 3e-6;
    const int max_outer = d.max_outer > 0 ? d.max_outer : 20;
    int outer = 0, total = 0;
    status = std::isfinite(res0) ? MPDG_OK : MPDG_ERR_NAN;
    while (status == MPDG_OK && res > tol) {
      if (outer >= max_outer || total >= max_it) {
        status = MPDG_ERR_NOT_CONVERGED;
        break;
      }
      // unit-norm FP32 defect, FP32 correction, FP64 update
      dev_scale_copy<float>(N, 1.0 / res, w.r, w32.r32, s);
      MPDG_CUDA(cudaMemsetAsync(w32.x32, 0, sizeof(float) * N, s));
      int it = 0;
      double r0i = 0, ri = 0;
      // the inner GMRES reads its rhs from r32, which it uses for nothing else
      // (z32 holds the preconditioner's output)
      int st = gmres<float>(op, w32, P, w32.r32, w32.x32, true, inner, 0.0,
                            std::max(1, max_it - total), d.gmres_restart > 0 ? d.gmres_restart : 30,
                            it, r0i, ri, applies);
      total += it;
      if (st == MPDG_ERR_NAN) {
        status = st;
        break;
      }
      dev_add_scaled<float>(N, res, w32.x32, x, s);
      launch_apply<double>(op, w.Ap, x);
      ++applies;
      dev_copy<double>(N, b, w.r, s);
      dev_axpby<double>(N, -1.0, w.Ap, 1.0, w.r, s);
      dev_dot(w.r, w.r, N, w.partial, w.scal + kRR, s);
      res = std::sqrt(fetch(op, w, w.scal + kRR));
      ++outer;
      if (!std::isfinite(res)) status = MPDG_ERR_NAN;
    }
    rep.iterations = total;
    rep.outer_iterations = outer;
  }
  MPDG_CUDA(cudaStreamSynchronize(s));
  rep.status = status;
  rep.operator_applies = applies;
  rep.initial_residual = res0;
  rep.final_residual = res;
  rep.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return status;
}

void free_workspace(Op &op)
{
  if (!op.ws) return;
  Workspace &w = *op.ws;
  for (void *p : {(void *)w.r, (void *)w.z, (void *)w.p, (void *)w.Ap, (void *)w.invd, (void *)w.cd,
                  (void *)w.ct, (void *)w.r32, (void *)w.z32, (void *)w.p32, (void *)w.Ap32,
                  (void *)w.x32, (void *)w.invd32, (void *)w.cd32, (void *)w.ct32, (void *)w.V,
                  (void *)w.V32,
                  (void *)w.partial, (void *)w.scal})
    if (p) cudaFree(p);
  if (w.host) cudaFreeHost(w.host);
  delete op.ws;
  op.ws = nullptr;
}

double linf(const double *a, long n, cudaStream_t s)
{
  double *partial = nullptr, *out = nullptr, h = 0.0;
  MPDG_CUDA(tracked_malloc(&partial, sizeof(double) * (kRedBlocks + 1)));
  out = partial + kRedBlocks;
  dev_linf(a, n, partial, out, s);
  MPDG_CUDA(cudaMemcpyAsync(&h, out, sizeof(double), cudaMemcpyDeviceToHost, s));
  MPDG_CUDA(cudaStreamSynchronize(s));
  cudaFree(partial);
  return h;
}

}  // namespace mpdg
