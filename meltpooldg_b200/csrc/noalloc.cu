// Jacobi-preconditioned CG that allocates nothing (mpdg_solve_cg_noalloc).
//
// Some callers cannot allocate device memory at solve time: a host that runs
// the solve inside its own memory pool or arena (allocating outside it would
// defeat the pool's accounting and can fail once the pool owns the free
// memory), a time loop that must not synchronise the device (cudaMalloc and
// cudaFree synchronise), or an application that forbids driver allocations
// after start-up.  For them this entry point keeps its scratch -- the CG
// vectors r, z, p, Ap, the inverse diagonal, the reduction partials and the
// device scalars -- in one file-scope __device__ array of fixed size, which
// every GPU that loads the library holds until the process exits.
//
// The array is shared by every call on a device and keeps the last call's
// contents; everything that must start at zero is cleared by the call itself.
// Two calls whose work overlaps on the GPU (different streams, or different
// host threads without ordering) race on the array: the caller serialises them.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <mutex>

#include "mpdg_internal.h"
#include "vector_kernels.cuh"

namespace mpdg {

// capacity: problems of up to kNoAllocMaxDofs DoFs (five FP64 vectors)
constexpr long kNoAllocMaxDofs = 1L << 18;  // 262,144 DoFs, 10.5 MB of scratch
constexpr long kNoAllocPartials = 4L * kRedBlocks;
constexpr long kNoAllocScalars = 64;
constexpr long kNoAllocElems = 5 * kNoAllocMaxDofs + kNoAllocPartials + kNoAllocScalars;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocElems];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
double *g_noalloc_ptr[kMaxDevices] = {nullptr};

// device address of the scratch array for the current device; the host-side
// name of a __device__ array is not a device address, so it is resolved once
// per device with that device current
double *scratch_for_current_device()
{
  int dev = 0;
  MPDG_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) throw Error{MPDG_ERR_ARG, "device index out of range"};
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess)
      throw Error{MPDG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e)};
    g_noalloc_ptr[dev] = static_cast<double *>(ptr);
  }
  return g_noalloc_ptr[dev];
}

double read_scalar(const double *dev, cudaStream_t s)
{
  double h = 0.0;
  MPDG_CUDA(cudaMemcpyAsync(&h, dev, sizeof(double), cudaMemcpyDeviceToHost, s));
  MPDG_CUDA(cudaStreamSynchronize(s));
  return h;
}

void read_scalars(const double *dev, double *h, int count, cudaStream_t s)
{
  MPDG_CUDA(cudaMemcpyAsync(h, dev, sizeof(double) * count, cudaMemcpyDeviceToHost, s));
  MPDG_CUDA(cudaStreamSynchronize(s));
}

}  // namespace

int solve_cg_noalloc(Op &op, double *x, const double *b, double rel_tol, double abs_tol, int max_it,
                     mpdg_solve_report &rep)
{
  const auto t0 = std::chrono::steady_clock::now();
  const long N = op.mesh->N;
  if (N > kNoAllocMaxDofs)
    throw Error{MPDG_ERR_SIZE, "problem has " + std::to_string(N) + " DoFs; the allocation-free CG "
                "holds scratch for at most " + std::to_string(kNoAllocMaxDofs)};
  if (const char *why = noalloc_unready_reason(op))
    throw Error{MPDG_ERR_ARG, std::string("mpdg_solve_cg_noalloc: ") + why};
  double *base = scratch_for_current_device();
  double *r = base, *z = base + N, *p = base + 2 * N, *Ap = base + 3 * N, *invd = base + 4 * N;
  double *partial = base + 5 * kNoAllocMaxDofs;
  double *sc = partial + kNoAllocPartials;
  cudaStream_t s = op.stream;
  MPDG_CUDA(cudaMemsetAsync(sc, 0, sizeof(double) * kNoAllocScalars, s));

  // Jacobi: inverse diagonal with the operator's threshold rule
  launch_diagonal(op, invd);
  double thr = 1e-10;  // heat_diffuse_operator.cpp:283
  if (op.d.kind == MPDG_OP_ADVDIFF) {
    dev_linf(invd, N, partial, sc + 8, s);  // advection_diffusion_operator.cpp:436-439
    thr = 1e-14 * std::fmax(1.0, read_scalar(sc + 8, s));
  }
  launch_invert_with_threshold(op, invd, thr);

  // CG (deal.II SolverCG + ReductionControl semantics), x holds the start
  int applies = 0;
  launch_apply<double>(op, Ap, x);
  ++applies;
  dev_copy<double>(N, b, r, s);
  dev_axpby<double>(N, -1.0, Ap, 1.0, r, s);
  dev_dot(r, r, N, partial, sc + kRR, s);
  const double res0 = std::sqrt(read_scalar(sc + kRR, s));
  double res = res0;
  int it = 0, status = MPDG_OK;
  const double tol = std::fmax(abs_tol, rel_tol * res0);
  if (!std::isfinite(res0)) status = MPDG_ERR_NAN;
  else if (res0 > tol) {
    dev_mul<double>(N, invd, r, z, s);
    dev_dot(r, z, N, partial, sc + kRZ, s);
    dev_copy<double>(N, z, p, s);
    // the convergence test on the device after every iteration, read every 4
    // iterations (updates past convergence are skipped: results and counts
    // are the per-iteration test's)
    constexpr int K = 4;
    dev_cg_check_init(sc, tol, s);
    int launched = 0;
    while (true) {
      const int batch = std::min(K, max_it - launched);
      for (int bi = 0; bi < batch; ++bi) {
        launch_apply<double>(op, Ap, p);
        dev_dot(p, Ap, N, partial, sc + kPAP, s);
        dev_cg_update_lagged<double, double>(N, sc, x, r, p, Ap, invd, z, partial, s);
        ++launched;
        dev_cg_check(sc, s);
        dev_cg_direction_lagged<double>(N, sc, p, z, s);
      }
      double h[3];
      read_scalars(sc + kDONE, h, 3, s);
      if (h[0] != 0.0) {
        it = (int)h[1];
        res = std::sqrt(h[2]);
        if (h[0] != 1.0) status = MPDG_ERR_NAN;
        break;
      }
      if (launched >= max_it) {
        it = launched;
        res = std::sqrt(read_scalar(sc + kRR, s));
        status = MPDG_ERR_NOT_CONVERGED;
        break;
      }
    }
    applies += it;
  }
  MPDG_CUDA(cudaStreamSynchronize(s));
  rep = mpdg_solve_report{};
  rep.status = status;
  rep.iterations = it;
  rep.operator_applies = applies;
  rep.initial_residual = res0;
  rep.final_residual = res;
  rep.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return status;
}

}  // namespace mpdg
