// Measured FMA throughput of this GPU in FP64 and FP32 (mpdg_fma_peak), the
// denominator of the apply's arithmetic-rate roofline.  Each thread runs 8
// independent FMA chains (enough in flight to hide the pipe latency) for a
// fixed number of steps; the result is stored so that nothing is eliminated.
#include <cuda_runtime.h>

#include <algorithm>

#include "mpdg_internal.h"

namespace mpdg {

namespace {

template <typename Real>
__global__ void fma_burn_kernel(Real *out, int steps, Real a, Real b)
{
  Real x[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) x[c] = (Real)(threadIdx.x + c) * Real(1e-3);
  for (int s = 0; s < steps; ++s) {
#pragma unroll
    for (int r = 0; r < 16; ++r) {
#pragma unroll
      for (int c = 0; c < 8; ++c) x[c] = x[c] * a + b;
    }
  }
  Real acc = 0;
#pragma unroll
  for (int c = 0; c < 8; ++c) acc += x[c];
  out[(long)blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

template <typename Real>
double measure(int sms)
{
  const int threads = 256, blocks = sms * 8, steps = 2048;
  Real *out = nullptr;
  MPDG_CUDA(tracked_malloc(&out, sizeof(Real) * (size_t)threads * blocks));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double best = 0.0;
  for (int rep = 0; rep < 4; ++rep) {
    cudaEventRecord(e0);
    fma_burn_kernel<Real><<<blocks, threads>>>(out, steps, Real(0.9999999), Real(1e-7));
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    const double flops = 2.0 * 8 * 16 * (double)steps * threads * blocks;
    if (rep > 0 && ms > 0.f) best = std::max(best, flops / (ms * 1e-3) / 1e9);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const cudaError_t e = cudaGetLastError();
  cudaFree(out);
  if (e != cudaSuccess) throw Error{MPDG_ERR_CUDA, cudaGetErrorString(e)};
  return best;
}

}  // namespace

void fma_peak(double &gflops64, double &gflops32)
{
  int dev = 0, sms = 0;
  MPDG_CUDA(cudaGetDevice(&dev));
  MPDG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  gflops64 = measure<double>(sms);
  gflops32 = measure<float>(sms);
}

}  // namespace mpdg
