// Batched and served solves: many independent heat / advection-diffusion
// problems (uniform unit-cube meshes, FE_Q(1..4)) advanced together, one CUDA
// graph launch per Krylov step for all of them.
//
// Each admitted problem owns a slot: FP64 x, b and defect vectors, FP32 r, z,
// p, Ap (and the BiCGStab vectors) and its FP32 inverse diagonal.  One step of
// the graph runs, for every active slot at once,
//   * the batched FP32 operator apply (one launch per degree and colour over a
//     segment table of all slots' cells, batch_apply.cuh);
//   * chunked vector kernels whose per-slot scalars live on the device, with
//     per-slot reductions over fixed chunks (deterministic, so a problem gives
//     the same result alone and in any mix);
//   * the reliable-update decision, and for the slots that take it the FP64
//     apply and defect b - A x that replaces the FP32 residual.
// Heat problems (symmetric) use CG, advection-diffusion problems BiCGStab,
// both with Jacobi preconditioning, FP32 operator and FP64 solution, defects,
// dots and norms.  The host only replays the graph and polls how many slots
// are still running; membership changes rebuild the tables and the graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <string>
#include <thread>
#include <vector>

#include "mpdg_internal.h"
#include "vector_kernels.cuh"

namespace mpdg {

constexpr int kChunk = 8192;  // vector elements per reduction chunk

struct BatchChunk {
  int slot, begin, end;
};

enum { SL_RUNNING = 0, SL_CONVERGED = 1, SL_NOT_CONVERGED = 2, SL_BREAKDOWN = 3, SL_NAN = 4 };

// per-slot device scalars
struct SlotScalars {
  double rz, rz_new, pap, rr;          // CG
  double rho, rho_new, alpha, omega;   // BiCGStab
  double tv, tt, ts;                   // BiCGStab dots (t.v... see kernels)
  double scale, tol, rmax, res, res0;
  int active, need_defect, iters, defects, status, max_it, kind, pad;
};

struct BatchSlot {
  bool used = false;
  int64_t ticket = -1;
  mpdg_problem_desc desc{};
  long N = 0;
  size_t bytes = 0;
  double *x = nullptr, *b = nullptr, *r64 = nullptr;
  float *r = nullptr, *z = nullptr, *p = nullptr, *Ap = nullptr, *invd = nullptr;
  float *rh = nullptr, *v = nullptr, *sv = nullptr, *t = nullptr;  // BiCGStab: r-hat, v, s, t
  double t_admit = 0;
  int first_chunk = 0, n_chunks = 0;
};

struct Batch {
  int device = 0;
  int64_t budget = 0, used = 0;
  int capacity = 0;
  double delta = 0.1;
  int max_it = 20000;
  cudaStream_t stream = nullptr;
  cudaMemPool_t pool = nullptr;  // slot vectors: stream-ordered, kept by the pool after release
  std::vector<BatchSlot> slots;
  int64_t next_ticket = 0;
  // device tables (capacity entries)
  SlotScalars *d_sc = nullptr;
  BatchSlotParams *d_params = nullptr;
  int *d_active = nullptr;  // [2][capacity]: running flags, then the per-kind masks of a step
  int *d_defect = nullptr;
  double **d_x = nullptr, **d_b = nullptr, **d_r64 = nullptr;
  float **d_r = nullptr, **d_z = nullptr, **d_p = nullptr, **d_Ap = nullptr, **d_invd = nullptr;
  float **d_rh = nullptr, **d_v = nullptr, **d_sv = nullptr, **d_t = nullptr;
  int *d_running = nullptr;     // number of running slots (polled by the host)
  int *h_running = nullptr;     // pinned
  SlotScalars *h_sc = nullptr;  // pinned copy of the scalars (polling)
  double *d_adm = nullptr;      // admission scratch: reduction partials and |b|^2
  // membership-dependent
  BatchChunk *d_chunks = nullptr;
  int n_chunks = 0;
  int *d_slot_chunk = nullptr;  // [capacity][2]: first chunk, count
  double *d_part = nullptr;     // chunk partials, 4 per chunk
  BatchApplyPlan plan;
  std::vector<void *> plan_allocs;
  cudaGraphExec_t graph = nullptr;
  int64_t step_kernels = 0;     // kernels of one graph step
  bool dirty = true;
  int tuned_cap = 0;            // resident CTAs per SM of the batched apply (0 = occupancy maximum)
  double tuned_ms = 0;
};

namespace {

template <typename T>
T *balloc(size_t n)
{
  T *p = nullptr;
  if (n == 0) return nullptr;
  cudaError_t e = cudaMalloc(&p, n * sizeof(T));
  if (e != cudaSuccess) throw Error{MPDG_ERR_ALLOC, std::string("cudaMalloc: ") + cudaGetErrorString(e)};
  return p;
}

unsigned grid1(long n, int b = 256) { return (unsigned)std::max(1L, std::min(4096L, (n + b - 1) / b)); }

// ------------------------------------------------------------------ kernels

__device__ __forceinline__ double bwarp_sum(double v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// block sum for 256 threads; valid in thread 0
__device__ __forceinline__ double bblock_sum(double v)
{
  __shared__ double ws[8];
  v = bwarp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) ws[w] = v;
  __syncthreads();
  double s = 0.0;
  if (w == 0) {
    s = (lane < 8) ? ws[lane] : 0.0;
    s = bwarp_sum(s);
  }
  __syncthreads();
  return s;
}

// deterministic [-1,1) values per (seed, index), zero on the boundary DoFs
__global__ void bk_rhs(double *b, long N, long NX, int dirichlet, unsigned long long seed)
{
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    unsigned long long z = seed * 0x9e3779b97f4a7c15ull + 0xbf58476d1ce4e5b9ull * (unsigned long long)(i + 1);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    const double u = (double)(z >> 11) * (1.0 / 9007199254740992.0);
    const long X = i % NX, Y = (i / NX) % NX, Z = i / (NX * NX);
    const bool bd = dirichlet && (X == 0 || Y == 0 || Z == 0 || X == NX - 1 || Y == NX - 1 || Z == NX - 1);
    b[i] = bd ? 0.0 : 2.0 * u - 1.0;
  }
}

__global__ void bk_set_boundary(double *d, long N, long NX, double value)
{
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const long X = i % NX, Y = (i / NX) % NX, Z = i / (NX * NX);
    if (X == 0 || Y == 0 || Z == 0 || X == NX - 1 || Y == NX - 1 || Z == NX - 1) d[i] = value;
  }
}

// slot initialisation from b with |b|^2 in *bb: scale = |b|, r = b / scale
// (FP32), x = 0, z = invd r; CG: p = z and partials of r.z; BiCGStab (rh
// given): rh = p = r and partials of r.r
__global__ void bk_init_vectors(const double *b, const double *bb, double *x, float *r, float *z, float *p,
                                const float *invd, float *rh, long N, double *part)
{
  const double nb = sqrt(*bb);
  const double inv_scale = nb > 0.0 ? 1.0 / nb : 1.0;
  double s = 0.0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    x[i] = 0.0;
    const float ri = (float)(b[i] * inv_scale);
    r[i] = ri;
    const float zi = invd[i] * ri;
    z[i] = zi;
    if (rh) {
      rh[i] = ri;
      p[i] = ri;
      s += (double)ri * (double)ri;
    } else {
      p[i] = zi;
      s += (double)ri * (double)zi;
    }
  }
  s = bblock_sum(s);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// per-slot scalars, parameters and flags of a newly admitted problem
__global__ void bk_init_scalars(SlotScalars *sc, int *active, int *defect, BatchSlotParams *params, int slot,
                                const double *part, int nparts, const double *bb, int kind, int max_it,
                                double rel_tol, double abs_tol, BatchSlotParams prm)
{
  double v = 0.0;
  for (int k = threadIdx.x; k < nparts; k += blockDim.x) v += part[k];
  v = bblock_sum(v);
  if (threadIdx.x != 0) return;
  SlotScalars q{};
  q.kind = kind;
  q.max_it = max_it;
  q.res0 = sqrt(*bb);
  q.res = q.res0;
  q.scale = q.res0 > 0.0 ? q.res0 : 1.0;
  q.tol = fmax(abs_tol, rel_tol * q.res0);
  q.rmax = 1.0;
  q.rz = v;
  q.rz_new = v;
  q.rho = v;
  q.rho_new = v;
  q.alpha = 1.0;
  q.omega = 1.0;
  const bool done = !(q.res0 > q.tol);
  q.status = done ? SL_CONVERGED : SL_RUNNING;
  q.active = done ? 0 : 1;
  sc[slot] = q;
  active[slot] = q.active;
  defect[slot] = 0;
  params[slot] = prm;
}

// Jacobi diagonal of a uniform unit-cube problem.  On the box every term of
// the cell operator is a product of 1D factors, and the cells that share a
// DoF form a Cartesian product of per-direction cell sets, so the assembled
// diagonal is a product of per-direction sums:
//   d = c_mass h^3 Mx My Mz + c_diff h (Ax My Mz + Mx Ay Mz + Mx My Az)
//       + c_vel h^2 (SDx CSy - CSx SDy) Mz            (vortex velocity)
// with, over the cells c sharing index X (local index i) and Gauss points q,
//   M = sum w S_qi^2,  A = sum w D_qi^2,
//   SD = sum w sin(pi x_q) D_qi S_qi,  CS = sum w cos(pi x_q) S_qi^2.
struct DiagTab {
  double S[kMaxN * kMaxN], D[kMaxN * kMaxN], w[kMaxN], x[kMaxN];
};

__global__ void bk_diag_factors(DiagTab t, int p, int nc, double h, double *F, long NX)
{
  const long X = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (X >= NX) return;
  const int n = p + 1;
  long cells[2];
  int loc[2], m = 0;
  const long c = X / p;
  const int r = (int)(X % p);
  if (r) {
    cells[m] = c;
    loc[m++] = r;
  } else {
    if (c >= 1) {
      cells[m] = c - 1;
      loc[m++] = p;
    }
    if (c < nc) {
      cells[m] = c;
      loc[m++] = 0;
    }
  }
  double M = 0.0, A = 0.0, SD = 0.0, CS = 0.0;
  for (int e = 0; e < m; ++e)
    for (int q = 0; q < n; ++q) {
      const double sv = t.S[q * n + loc[e]], dv = t.D[q * n + loc[e]], w = t.w[q];
      double sn, cs;
      sincospi(((double)cells[e] + t.x[q]) * h, &sn, &cs);
      M += w * sv * sv;
      A += w * dv * dv;
      SD += w * sn * dv * sv;
      CS += w * cs * sv * sv;
    }
  F[X] = M;
  F[NX + X] = A;
  F[2 * NX + X] = SD;
  F[3 * NX + X] = CS;
}

__global__ void bk_diag_invd(const double *F, long NX, long N, double c_mass, double c_diff, double c_vel,
                             double h, int vortex, int dirichlet, double thr, float *invd)
{
  for (long g = (long)blockIdx.x * blockDim.x + threadIdx.x; g < N; g += (long)gridDim.x * blockDim.x) {
    const long X = g % NX, Y = (g / NX) % NX, Z = g / (NX * NX);
    const double Mx = F[X], My = F[Y], Mz = F[Z];
    double d = c_mass * h * h * h * Mx * My * Mz + c_diff * h * (F[NX + X] * My * Mz + Mx * F[NX + Y] * Mz + Mx * My * F[NX + Z]);
    if (vortex) d += c_vel * h * h * (F[2 * NX + X] * F[3 * NX + Y] - F[3 * NX + X] * F[2 * NX + Y]) * Mz;
    if (dirichlet && (X == 0 || Y == 0 || Z == 0 || X == NX - 1 || Y == NX - 1 || Z == NX - 1)) d = 1.0;
    invd[g] = (float)(fabs(d) > thr ? 1.0 / d : 1.0);
  }
}

// diagonal in FP64 (tests compare it with the single-problem operator)
__global__ void bk_diag_values(const double *F, long NX, long N, double c_mass, double c_diff, double c_vel,
                               double h, int vortex, int dirichlet, double *out)
{
  for (long g = (long)blockIdx.x * blockDim.x + threadIdx.x; g < N; g += (long)gridDim.x * blockDim.x) {
    const long X = g % NX, Y = (g / NX) % NX, Z = g / (NX * NX);
    const double Mx = F[X], My = F[Y], Mz = F[Z];
    double d = c_mass * h * h * h * Mx * My * Mz + c_diff * h * (F[NX + X] * My * Mz + Mx * F[NX + Y] * Mz + Mx * My * F[NX + Z]);
    if (vortex) d += c_vel * h * h * (F[2 * NX + X] * F[3 * NX + Y] - F[3 * NX + X] * F[2 * NX + Y]) * Mz;
    if (dirichlet && (X == 0 || Y == 0 || Z == 0 || X == NX - 1 || Y == NX - 1 || Z == NX - 1)) d = 1.0;
    out[g] = d;
  }
}

#define FOR_CHUNK(ch)                                                            \
  for (int ci = blockIdx.x; ci < n_chunks; ci += gridDim.x) {                    \
    const BatchChunk ch = chunks[ci];

#define END_FOR_CHUNK }

// p.Ap partials (CG) / rh.v partials (BiCGStab), per chunk of active slots
__global__ void bk_dot_pap(const BatchChunk *chunks, int n_chunks, const int *active, float *const *A,
                           float *const *B, double *part)
{
  FOR_CHUNK(ch)
    double s = 0.0;
    if (active[ch.slot]) {
      const float *a = A[ch.slot], *bb = B[ch.slot];
      for (int i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) s += (double)a[i] * (double)bb[i];
    }
    s = bblock_sum(s);
    if (threadIdx.x == 0) part[4 * ci] = s;
  END_FOR_CHUNK
}

// sums per slot: out[slot-field] = sum over the slot's chunks of part[4c + k]
template <int K>
__device__ double slot_sum(const double *part, const int *slot_chunk, int s)
{
  const int c0 = slot_chunk[2 * s], nc = slot_chunk[2 * s + 1];
  double v = 0.0;
  for (int c = c0; c < c0 + nc; ++c) v += part[4 * c + K];
  return v;
}

__global__ void bk_finish_pap(SlotScalars *sc, const int *active, const double *part, const int *slot_chunk,
                              int n_slots)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_slots || !active[s]) return;
  sc[s].pap = slot_sum<0>(part, slot_chunk, s);
}

// CG: alpha = rz / pap; x += scale alpha p; r -= alpha Ap; z = invd r; partials r.r, r.z
__global__ void bk_cg_update(const BatchChunk *chunks, int n_chunks, const int *active,
                             const SlotScalars *sc, double *const *X, float *const *R, float *const *Z,
                             float *const *Pv, float *const *APv, float *const *ID, double *part)
{
  FOR_CHUNK(ch)
    double rr = 0.0, rz = 0.0;
    const int s = ch.slot;
    if (active[s] && sc[s].kind == MPDG_OP_HEAT) {
      const double alpha = sc[s].rz / sc[s].pap, xa = alpha * sc[s].scale;
      double *x = X[s];
      float *r = R[s], *z = Z[s];
      const float *p = Pv[s], *ap = APv[s], *id = ID[s];
      for (int i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) {
        x[i] += xa * (double)p[i];
        const float ri = (float)((double)r[i] - alpha * (double)ap[i]);
        r[i] = ri;
        const float zi = id[i] * ri;
        z[i] = zi;
        rr += (double)ri * (double)ri;
        rz += (double)ri * (double)zi;
      }
    }
    rr = bblock_sum(rr);
    rz = bblock_sum(rz);
    if (threadIdx.x == 0) {
      part[4 * ci + 1] = rr;
      part[4 * ci + 2] = rz;
    }
  END_FOR_CHUNK
}

// per-slot bookkeeping after the FP32 update; decides the FP64 defect
__global__ void bk_cg_decide(SlotScalars *sc, int *active, int *defect, const double *part,
                             const int *slot_chunk, int n_slots, double delta)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_slots) return;
  defect[s] = 0;
  if (!active[s] || sc[s].kind != MPDG_OP_HEAT) return;
  SlotScalars &q = sc[s];
  if (!(q.pap > 0.0)) {
    q.status = SL_BREAKDOWN;
    active[s] = 0;
    return;
  }
  q.rr = slot_sum<1>(part, slot_chunk, s);
  q.rz_new = slot_sum<2>(part, slot_chunk, s);
  q.iters += 1;
  const double rel = sqrt(q.rr);
  if (!isfinite(rel)) {
    q.status = SL_NAN;
    active[s] = 0;
    return;
  }
  q.res = rel * q.scale;
  if (q.res <= q.tol || rel < delta * q.rmax || q.iters >= q.max_it) defect[s] = 1;
}

// defect b - A x (A x already in r64) for flagged slots, partials of |d|^2
__global__ void bk_defect(const BatchChunk *chunks, int n_chunks, const int *defect,
                          double *const *B, double *const *R64, double *part)
{
  FOR_CHUNK(ch)
    double s = 0.0;
    if (defect[ch.slot]) {
      const double *b = B[ch.slot];
      double *r = R64[ch.slot];
      for (int i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) {
        const double d = b[i] - r[i];
        r[i] = d;
        s += d * d;
      }
    }
    s = bblock_sum(s);
    if (threadIdx.x == 0) part[4 * ci + 3] = s;
  END_FOR_CHUNK
}

__global__ void bk_defect_decide(SlotScalars *sc, int *active, int *defect, const double *part,
                                 const int *slot_chunk, int n_slots)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_slots || !defect[s]) return;
  SlotScalars &q = sc[s];
  q.res = sqrt(slot_sum<3>(part, slot_chunk, s));
  q.defects += 1;
  if (!isfinite(q.res)) {
    q.status = SL_NAN;
    active[s] = 0;
    defect[s] = 0;
  } else if (q.res <= q.tol) {
    q.status = SL_CONVERGED;
    active[s] = 0;
    defect[s] = 0;
  } else if (q.iters >= q.max_it) {
    q.status = SL_NOT_CONVERGED;
    active[s] = 0;
    defect[s] = 0;
  } else {
    q.rmax = q.res / q.scale;
  }
}

// replacement of the FP32 residual by the FP64 defect (CG), partials of r.z
__global__ void bk_cg_replace(const BatchChunk *chunks, int n_chunks, const int *defect,
                              const SlotScalars *sc, double *const *R64, float *const *R, float *const *Z,
                              float *const *ID, double *part)
{
  FOR_CHUNK(ch)
    double rz = 0.0;
    const int s = ch.slot;
    if (defect[s] && sc[s].kind == MPDG_OP_HEAT) {
      const double is = 1.0 / sc[s].scale;
      const double *d = R64[s];
      float *r = R[s], *z = Z[s];
      const float *id = ID[s];
      for (int i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) {
        const float ri = (float)(d[i] * is);
        r[i] = ri;
        const float zi = id[i] * ri;
        z[i] = zi;
        rz += (double)ri * (double)zi;
      }
    }
    rz = bblock_sum(rz);
    if (threadIdx.x == 0) part[4 * ci + 2] = rz;
  END_FOR_CHUNK
}

__global__ void bk_cg_replace_finish(SlotScalars *sc, const int *defect, const double *part,
                                     const int *slot_chunk, int n_slots)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_slots || !defect[s] || sc[s].kind != MPDG_OP_HEAT) return;
  sc[s].rz_new = slot_sum<2>(part, slot_chunk, s);
}

// p = z + beta p
__global__ void bk_cg_direction(const BatchChunk *chunks, int n_chunks, const int *active,
                                const SlotScalars *sc, float *const *Z, float *const *Pv)
{
  FOR_CHUNK(ch)
    const int s = ch.slot;
    if (active[s] && sc[s].kind == MPDG_OP_HEAT) {
      const double beta = sc[s].rz_new / sc[s].rz;
      const float *z = Z[s];
      float *p = Pv[s];
      for (int i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x)
        p[i] = (float)((double)z[i] + beta * (double)p[i]);
    }
  END_FOR_CHUNK
}

__global__ void bk_cg_shift(SlotScalars *sc, const int *active, int n_slots)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_slots || !active[s] || sc[s].kind != MPDG_OP_HEAT) return;
  sc[s].rz = sc[s].rz_new;
}

__global__ void bk_count_running(const int *active, int n_slots, int *out)
{
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  int c = 0;
  for (int s = threadIdx.x; s < n_slots; s += blockDim.x) c += active[s] ? 1 : 0;
  atomicAdd(&cnt, c);
  __syncthreads();
  if (threadIdx.x == 0) *out = cnt;
}

// ---------------- BiCGStab (right-preconditioned by Jacobi), advection-diffusion slots
// state: r (residual, scaled), rh (shadow), p, v = A M p, s, t = A M s; M = diag(invd)
// phase A (after v = A (invd p) in Ap): alpha = rho / (rh . v)
__global__ void bk_bicg_alpha_partials(const BatchChunk *chunks, int n_chunks, const int *active,
                                       const SlotScalars *sc, float *const *RH, float *const *V,
                                       double *part)
{
  FOR_CHUNK(ch)
    double s = 0.0;
    if (active[ch.slot] && sc[ch.slot].kind == MPDG_OP_ADVDIFF) {
      const float *rh = RH[ch.slot], *v = V[ch.slot];
      for (int i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) s += (double)rh[i] * (double)v[i];
    }
    s = bblock_sum(s);
    if (threadIdx.x == 0) part[4 * ci] = s;
  END_FOR_CHUNK
}

__global__ void bk_bicg_alpha(SlotScalars *sc, int *active, const double *part, const int *slot_chunk,
                              int n_slots)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_slots || !active[s] || sc[s].kind != MPDG_OP_ADVDIFF) return;
  const double rv = slot_sum<0>(part, slot_chunk, s);
  if (!(rv != 0.0) || !isfinite(rv)) {
    sc[s].status = SL_BREAKDOWN;
    active[s] = 0;
    return;
  }
  sc[s].alpha = sc[s].rho / rv;
}

// s = r - alpha v, (into sv); z = invd s (into z) for the second apply
__global__ void bk_bicg_s(const BatchChunk *chunks, int n_chunks, const int *active, const SlotScalars *sc,
                          float *const *R, float *const *V, float *const *SV, float *const *Z,
                          float *const *ID)
{
  FOR_CHUNK(ch)
    const int s = ch.slot;
    if (active[s] && sc[s].kind == MPDG_OP_ADVDIFF) {
      const double a = sc[s].alpha;
      const float *r = R[s], *v = V[s], *id = ID[s];
      float *sv = SV[s], *z = Z[s];
      for (int i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) {
        const float si = (float)((double)r[i] - a * (double)v[i]);
        sv[i] = si;
        z[i] = id[i] * si;
      }
    }
  END_FOR_CHUNK
}

// after t = A z: partials t.s and t.t
__global__ void bk_bicg_omega_partials(const BatchChunk *chunks, int n_chunks, const int *active,
                                       const SlotScalars *sc, float *const *T, float *const *SV,
                                       double *part)
{
  FOR_CHUNK(ch)
    double ts = 0.0, tt = 0.0;
    const int s = ch.slot;
    if (active[s] && sc[s].kind == MPDG_OP_ADVDIFF) {
      const float *t = T[s], *sv = SV[s];
      for (int i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) {
        ts += (double)t[i] * (double)sv[i];
        tt += (double)t[i] * (double)t[i];
      }
    }
    ts = bblock_sum(ts);
    tt = bblock_sum(tt);
    if (threadIdx.x == 0) {
      part[4 * ci] = ts;
      part[4 * ci + 1] = tt;
    }
  END_FOR_CHUNK
}

__global__ void bk_bicg_omega(SlotScalars *sc, int *active, const double *part, const int *slot_chunk,
                              int n_slots)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_slots || !active[s] || sc[s].kind != MPDG_OP_ADVDIFF) return;
  const double ts = slot_sum<0>(part, slot_chunk, s), tt = slot_sum<1>(part, slot_chunk, s);
  sc[s].omega = (tt > 0.0) ? ts / tt : 0.0;
}

// x += scale (alpha invd p + omega invd s); r = s - omega t; partials r.r and rh.r
__global__ void bk_bicg_update(const BatchChunk *chunks, int n_chunks, const int *active,
                               const SlotScalars *sc, double *const *X, float *const *R, float *const *Pv,
                               float *const *SV, float *const *T, float *const *RH, float *const *ID,
                               double *part)
{
  FOR_CHUNK(ch)
    double rr = 0.0, rhr = 0.0;
    const int s = ch.slot;
    if (active[s] && sc[s].kind == MPDG_OP_ADVDIFF) {
      const double a = sc[s].alpha, w = sc[s].omega, scl = sc[s].scale;
      double *x = X[s];
      float *r = R[s];
      const float *p = Pv[s], *sv = SV[s], *t = T[s], *rh = RH[s], *id = ID[s];
      for (int i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) {
        x[i] += scl * (a * (double)(id[i] * p[i]) + w * (double)(id[i] * sv[i]));
        const float ri = (float)((double)sv[i] - w * (double)t[i]);
        r[i] = ri;
        rr += (double)ri * (double)ri;
        rhr += (double)rh[i] * (double)ri;
      }
    }
    rr = bblock_sum(rr);
    rhr = bblock_sum(rhr);
    if (threadIdx.x == 0) {
      part[4 * ci + 1] = rr;
      part[4 * ci + 2] = rhr;
    }
  END_FOR_CHUNK
}

__global__ void bk_bicg_decide(SlotScalars *sc, int *active, int *defect, const double *part,
                               const int *slot_chunk, int n_slots, double delta)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_slots) return;
  if (!active[s] || sc[s].kind != MPDG_OP_ADVDIFF) return;
  SlotScalars &q = sc[s];
  q.rr = slot_sum<1>(part, slot_chunk, s);
  q.rho_new = slot_sum<2>(part, slot_chunk, s);
  q.iters += 1;
  const double rel = sqrt(q.rr);
  if (!isfinite(rel)) {
    q.status = SL_NAN;
    active[s] = 0;
    return;
  }
  q.res = rel * q.scale;
  if (q.res <= q.tol || rel < delta * q.rmax || q.iters >= q.max_it || !(q.omega != 0.0)) defect[s] = 1;
}

// restart from the FP64 defect: r = rh = d / scale, p = r, rho = r.r
__global__ void bk_bicg_replace(const BatchChunk *chunks, int n_chunks, const int *defect,
                                const SlotScalars *sc, double *const *R64, float *const *R,
                                float *const *RH, float *const *Pv, double *part)
{
  FOR_CHUNK(ch)
    double rr = 0.0;
    const int s = ch.slot;
    if (defect[s] && sc[s].kind == MPDG_OP_ADVDIFF) {
      const double is = 1.0 / sc[s].scale;
      const double *d = R64[s];
      float *r = R[s], *rh = RH[s], *p = Pv[s];
      for (int i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) {
        const float ri = (float)(d[i] * is);
        r[i] = ri;
        rh[i] = ri;
        p[i] = ri;
        rr += (double)ri * (double)ri;
      }
    }
    rr = bblock_sum(rr);
    if (threadIdx.x == 0) part[4 * ci + 2] = rr;
  END_FOR_CHUNK
}

__global__ void bk_bicg_replace_finish(SlotScalars *sc, const int *defect, const double *part,
                                       const int *slot_chunk, int n_slots)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_slots || !defect[s] || sc[s].kind != MPDG_OP_ADVDIFF) return;
  sc[s].rho = slot_sum<2>(part, slot_chunk, s);
  sc[s].rho_new = sc[s].rho;
}

// p = r + beta (p - omega v), beta = (rho_new / rho) (alpha / omega); skipped right after a restart
__global__ void bk_bicg_direction(const BatchChunk *chunks, int n_chunks, const int *active,
                                  const int *defect, const SlotScalars *sc, float *const *R,
                                  float *const *Pv, float *const *V)
{
  FOR_CHUNK(ch)
    const int s = ch.slot;
    if (active[s] && !defect[s] && sc[s].kind == MPDG_OP_ADVDIFF) {
      const double beta = (sc[s].rho_new / sc[s].rho) * (sc[s].alpha / sc[s].omega), w = sc[s].omega;
      const float *r = R[s], *v = V[s];
      float *p = Pv[s];
      for (int i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x)
        p[i] = (float)((double)r[i] + beta * ((double)p[i] - w * (double)v[i]));
    }
  END_FOR_CHUNK
}

__global__ void bk_bicg_shift(SlotScalars *sc, const int *active, int n_slots)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_slots || !active[s] || sc[s].kind != MPDG_OP_ADVDIFF) return;
  sc[s].rho = sc[s].rho_new;
}

// z = invd p for the first BiCGStab apply (right preconditioning)
__global__ void bk_bicg_precond_p(const BatchChunk *chunks, int n_chunks, const int *active,
                                  const SlotScalars *sc, float *const *Pv, float *const *Z,
                                  float *const *ID)
{
  FOR_CHUNK(ch)
    const int s = ch.slot;
    if (active[s] && sc[s].kind == MPDG_OP_ADVDIFF) {
      const float *p = Pv[s], *id = ID[s];
      float *z = Z[s];
      for (int i = ch.begin + threadIdx.x; i < ch.end; i += blockDim.x) z[i] = id[i] * p[i];
    }
  END_FOR_CHUNK
}

// active mask restricted to one kind (for the applies of the BiCGStab phases)
__global__ void bk_kind_mask(const SlotScalars *sc, const int *active, int *out, int kind, int n_slots)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n_slots) out[s] = (active[s] && sc[s].kind == kind) ? 1 : 0;
}

}  // namespace
}  // namespace mpdg


namespace mpdg {
namespace {

// admission scratch layout (doubles): [0, R) reduction partials, [R] |b|^2,
// [R+8, 2R+8) initialisation partials, [2R+16] |x|^2
constexpr int kAdmDoubles = 2 * kRedBlocks + 32;
constexpr int kAdmBB = kRedBlocks, kAdmInit = kRedBlocks + 8, kAdmNorm = 2 * kRedBlocks + 16;

size_t slot_bytes(long N, int kind)
{
  // x, b, r64 (FP64) + r, z, p, Ap, invd (FP32) [+ rh, v, s, t for BiCGStab]
  return (size_t)N * (3 * 8 + 5 * 4 + (kind == MPDG_OP_ADVDIFF ? 4 * 4 : 0));
}

long problem_dofs(const mpdg_problem_desc &d)
{
  const long NX = (long)d.nc * d.degree + 1;
  return NX * NX * NX;
}

void check_desc(const mpdg_problem_desc &d)
{
  if (d.kind != MPDG_OP_HEAT && d.kind != MPDG_OP_ADVDIFF) throw Error{MPDG_ERR_ARG, "unknown problem kind"};
  if (d.degree < 1 || d.degree > kMaxDegree) throw Error{MPDG_ERR_UNSUPPORTED, "degree must be 1..4"};
  if (d.nc < 2 || d.nc > 400) throw Error{MPDG_ERR_ARG, "cells per direction must be 2..400"};
  if (!(d.dt > 0.0)) throw Error{MPDG_ERR_ARG, "time increment must be positive"};
  if (d.kind == MPDG_OP_HEAT && d.vel_kind != MPDG_VEL_NONE)
    throw Error{MPDG_ERR_UNSUPPORTED, "batched heat problems have no velocity"};
  if (d.kind == MPDG_OP_ADVDIFF && d.vel_kind != MPDG_VEL_NONE && d.vel_kind != MPDG_VEL_VORTEX)
    throw Error{MPDG_ERR_UNSUPPORTED, "batched advection uses the vortex velocity"};
  if (problem_dofs(d) > (1L << 31) - 2L * kChunk)
    throw Error{MPDG_ERR_SIZE, "a batched problem holds at most 2^31 - 16384 DoFs"};
  if (d.rel_tolerance < 0.0 || d.abs_tolerance < 0.0 || d.max_iterations < 0)
    throw Error{MPDG_ERR_ARG, "negative tolerance or iteration limit"};
}

// operator coefficients of the batched apply: same meaning as the single
// problem's (heat: rho_cp/dt, rho_cp, k0; advection-diffusion: 1/dt, theta, theta D)
BatchSlotParams slot_params(const mpdg_problem_desc &d)
{
  BatchSlotParams prm{};
  const double h = 1.0 / d.nc;
  prm.h = h;
  prm.hvol = h * h * h;
  prm.ih = 1.0 / h;
  prm.ih2 = 1.0 / (h * h);
  prm.vel_kind = d.vel_kind;
  prm.dirichlet = d.dirichlet ? 1 : 0;
  if (d.kind == MPDG_OP_HEAT) {
    prm.c_mass = d.rho_cp / d.dt;
    prm.c_vel = d.rho_cp;
    prm.c_diff = d.k0;
  } else {
    prm.c_mass = 1.0 / d.dt;
    prm.c_vel = d.theta;
    prm.c_diff = d.theta * d.diffusivity;
  }
  return prm;
}

DiagTab diag_tables(int p)
{
  DiagTab t;
  std::memset(&t, 0, sizeof(t));
  shape_1d(p, t.S, t.D, t.w, t.x);
  return t;
}

// the 1D factors of the diagonal into F (4 NX doubles), then invd or the FP64 diagonal
void enqueue_diagonal(const mpdg_problem_desc &d, double *F, float *invd, double *diag, cudaStream_t st)
{
  const long NX = (long)d.nc * d.degree + 1, N = NX * NX * NX;
  const BatchSlotParams prm = slot_params(d);
  bk_diag_factors<<<(unsigned)((NX + 127) / 128), 128, 0, st>>>(diag_tables(d.degree), d.degree, d.nc, prm.h, F, NX);
  MPDG_LAUNCHED();
  const int vortex = d.vel_kind == MPDG_VEL_VORTEX;
  if (invd) {
    // inversion thresholds of the single-problem operators
    const double thr = d.kind == MPDG_OP_HEAT ? 1e-10 : 1e-14;
    bk_diag_invd<<<grid1(N), 256, 0, st>>>(F, NX, N, prm.c_mass, prm.c_diff, prm.c_vel, prm.h, vortex,
                                           prm.dirichlet, thr, invd);
    MPDG_LAUNCHED();
  }
  if (diag) {
    bk_diag_values<<<grid1(N), 256, 0, st>>>(F, NX, N, prm.c_mass, prm.c_diff, prm.c_vel, prm.h, vortex,
                                             prm.dirichlet, diag);
    MPDG_LAUNCHED();
  }
}

// host copy of bk_rhs (same integer arithmetic, exact double conversion)
void rhs_host(const mpdg_problem_desc &d, double *b)
{
  const long NX = (long)d.nc * d.degree + 1, N = NX * NX * NX;
  const unsigned long long seed = d.rhs_seed;
  for (long i = 0; i < N; ++i) {
    unsigned long long z = seed * 0x9e3779b97f4a7c15ull + 0xbf58476d1ce4e5b9ull * (unsigned long long)(i + 1);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    const double u = (double)(z >> 11) * (1.0 / 9007199254740992.0);
    const long X = i % NX, Y = (i / NX) % NX, Z = i / (NX * NX);
    const bool bd = d.dirichlet && (X == 0 || Y == 0 || Z == 0 || X == NX - 1 || Y == NX - 1 || Z == NX - 1);
    b[i] = bd ? 0.0 : 2.0 * u - 1.0;
  }
}

template <typename T>
T *palloc(Batch &B, size_t n)
{
  void *p = nullptr;
  const cudaError_t e = cudaMallocFromPoolAsync(&p, n * sizeof(T), B.pool, B.stream);
  if (e != cudaSuccess) throw Error{MPDG_ERR_ALLOC, std::string("device pool: ") + cudaGetErrorString(e)};
  return (T *)p;
}

void free_slot_vectors(Batch &B, BatchSlot &S)
{
  for (void *p : {(void *)S.x, (void *)S.b, (void *)S.r64, (void *)S.r, (void *)S.z, (void *)S.p,
                  (void *)S.Ap, (void *)S.invd, (void *)S.rh, (void *)S.v, (void *)S.sv, (void *)S.t})
    if (p) cudaFreeAsync(p, B.stream);
}

template <typename T>
void ptr_table(Batch &B, T *BatchSlot::*field, T **dev)
{
  std::vector<T *> h(B.capacity, nullptr);
  for (int s = 0; s < B.capacity; ++s)
    if (B.slots[s].used) h[s] = B.slots[s].*field;
  MPDG_CUDA(cudaMemcpyAsync(dev, h.data(), sizeof(T *) * B.capacity, cudaMemcpyHostToDevice, B.stream));
  MPDG_CUDA(cudaStreamSynchronize(B.stream));  // h is a temporary
}

void drop_graph(Batch &B)
{
  if (B.graph) {
    cudaGraphExecDestroy(B.graph);
    B.graph = nullptr;
  }
}

void free_plan(Batch &B)
{
  for (void *p : B.plan_allocs) cudaFree(p);
  B.plan_allocs.clear();
  B.plan = BatchApplyPlan{};
  if (B.d_chunks) cudaFree(B.d_chunks);
  if (B.d_part) cudaFree(B.d_part);
  B.d_chunks = nullptr;
  B.d_part = nullptr;
  B.n_chunks = 0;
  drop_graph(B);
}

// tables of the current membership: chunks, per-slot chunk ranges, apply segments, pointers
void rebuild_tables(Batch &B)
{
  MPDG_CUDA(cudaStreamSynchronize(B.stream));
  free_plan(B);
  std::vector<BatchChunk> chunks;
  std::vector<int> slot_chunk(2 * (size_t)B.capacity, 0);
  for (int s = 0; s < B.capacity; ++s) {
    BatchSlot &S = B.slots[s];
    if (!S.used) continue;
    S.first_chunk = (int)chunks.size();
    for (long b = 0; b < S.N; b += kChunk) chunks.push_back({s, (int)b, (int)std::min(S.N, b + kChunk)});
    S.n_chunks = (int)chunks.size() - S.first_chunk;
    slot_chunk[2 * s] = S.first_chunk;
    slot_chunk[2 * s + 1] = S.n_chunks;
  }
  B.n_chunks = (int)chunks.size();
  if (B.n_chunks) {
    B.d_chunks = balloc<BatchChunk>(B.n_chunks);
    MPDG_CUDA(cudaMemcpy(B.d_chunks, chunks.data(), sizeof(BatchChunk) * B.n_chunks, cudaMemcpyHostToDevice));
    B.d_part = balloc<double>(4 * (size_t)B.n_chunks);
  }
  MPDG_CUDA(cudaMemcpy(B.d_slot_chunk, slot_chunk.data(), sizeof(int) * 2 * B.capacity, cudaMemcpyHostToDevice));
  for (int p = 1; p <= kMaxDegree; ++p) {
    const int cpw = cells_per_warp(p);
    for (int c = 0; c < 8; ++c) {
      std::vector<BatchSeg> segs;
      std::vector<int> prefix;
      long groups = 0;
      for (int s = 0; s < B.capacity; ++s) {
        const BatchSlot &S = B.slots[s];
        if (!S.used || S.desc.degree != p) continue;
        BatchSeg g{};
        g.slot = s;
        g.nc = S.desc.nc;
        long count = 1;
        for (int d = 0; d < 3; ++d) {
          g.par[d] = (c >> d) & 1;
          g.cn[d] = (S.desc.nc - g.par[d] + 1) / 2;
          count *= g.cn[d];
        }
        if (count == 0) continue;
        g.count = (int)count;
        const unsigned long long d0 = (unsigned long long)g.cn[0], d01 = d0 * (unsigned long long)g.cn[1];
        g.div0_magic = ((1ull << 40) + d0 - 1) / d0;
        g.div01_magic = ((1ull << 40) + d01 - 1) / d01;
        g.NX = (long)S.desc.nc * p + 1;
        prefix.push_back((int)groups);
        segs.push_back(g);
        groups += (count + cpw - 1) / cpw;
      }
      if (segs.empty()) continue;
      if (groups > INT32_MAX / 2) throw Error{MPDG_ERR_SIZE, "batch too large for one apply launch"};
      BatchSeg *ds = balloc<BatchSeg>(segs.size());
      B.plan_allocs.push_back(ds);
      int *dp = balloc<int>(prefix.size());
      B.plan_allocs.push_back(dp);
      MPDG_CUDA(cudaMemcpy(ds, segs.data(), sizeof(BatchSeg) * segs.size(), cudaMemcpyHostToDevice));
      MPDG_CUDA(cudaMemcpy(dp, prefix.data(), sizeof(int) * prefix.size(), cudaMemcpyHostToDevice));
      B.plan.segs[p][c] = ds;
      B.plan.prefix[p][c] = dp;
      B.plan.nseg[p][c] = (int)segs.size();
      B.plan.groups[p][c] = (int)groups;
    }
  }
  ptr_table<double>(B, &BatchSlot::x, B.d_x);
  ptr_table<double>(B, &BatchSlot::b, B.d_b);
  ptr_table<double>(B, &BatchSlot::r64, B.d_r64);
  ptr_table<float>(B, &BatchSlot::r, B.d_r);
  ptr_table<float>(B, &BatchSlot::z, B.d_z);
  ptr_table<float>(B, &BatchSlot::p, B.d_p);
  ptr_table<float>(B, &BatchSlot::Ap, B.d_Ap);
  ptr_table<float>(B, &BatchSlot::invd, B.d_invd);
  ptr_table<float>(B, &BatchSlot::rh, B.d_rh);
  ptr_table<float>(B, &BatchSlot::v, B.d_v);
  ptr_table<float>(B, &BatchSlot::sv, B.d_sv);
  ptr_table<float>(B, &BatchSlot::t, B.d_t);
  B.dirty = false;
}

// one Krylov step of every running slot (the body of the graph)
void enqueue_step(Batch &B, int cap)
{
  cudaStream_t st = B.stream;
  const int S = B.capacity, nc = B.n_chunks;
  const unsigned gs = (unsigned)((S + 255) / 256), gc = (unsigned)std::max(1, std::min(nc, 148 * 8));
  int *kmask = B.d_active + S;
#define BK(kernel, grid, ...)                            \
  do {                                                   \
    kernel<<<grid, 256, 0, st>>>(__VA_ARGS__);           \
    MPDG_LAUNCHED();                                     \
  } while (0)
  // CG on the heat problems: Ap = A p (FP32), alpha, x/r/z update
  BK(bk_kind_mask, gs, B.d_sc, B.d_active, kmask, MPDG_OP_HEAT, S);
  launch_batch_apply<float>(B.plan, B.d_params, B.d_p, B.d_Ap, kmask, cap, st);
  BK(bk_dot_pap, gc, B.d_chunks, nc, kmask, B.d_p, B.d_Ap, B.d_part);
  BK(bk_finish_pap, gs, B.d_sc, kmask, B.d_part, B.d_slot_chunk, S);
  BK(bk_cg_update, gc, B.d_chunks, nc, kmask, B.d_sc, B.d_x, B.d_r, B.d_z, B.d_p, B.d_Ap, B.d_invd, B.d_part);
  BK(bk_cg_decide, gs, B.d_sc, B.d_active, B.d_defect, B.d_part, B.d_slot_chunk, S, B.delta);
  // BiCGStab on the advection-diffusion problems: v = A M p, alpha, s, t = A M s, omega, update
  BK(bk_kind_mask, gs, B.d_sc, B.d_active, kmask, MPDG_OP_ADVDIFF, S);
  BK(bk_bicg_precond_p, gc, B.d_chunks, nc, kmask, B.d_sc, B.d_p, B.d_z, B.d_invd);
  launch_batch_apply<float>(B.plan, B.d_params, B.d_z, B.d_v, kmask, cap, st);
  BK(bk_bicg_alpha_partials, gc, B.d_chunks, nc, kmask, B.d_sc, B.d_rh, B.d_v, B.d_part);
  BK(bk_bicg_alpha, gs, B.d_sc, B.d_active, B.d_part, B.d_slot_chunk, S);
  BK(bk_kind_mask, gs, B.d_sc, B.d_active, kmask, MPDG_OP_ADVDIFF, S);
  BK(bk_bicg_s, gc, B.d_chunks, nc, kmask, B.d_sc, B.d_r, B.d_v, B.d_sv, B.d_z, B.d_invd);
  launch_batch_apply<float>(B.plan, B.d_params, B.d_z, B.d_t, kmask, cap, st);
  BK(bk_bicg_omega_partials, gc, B.d_chunks, nc, kmask, B.d_sc, B.d_t, B.d_sv, B.d_part);
  BK(bk_bicg_omega, gs, B.d_sc, B.d_active, B.d_part, B.d_slot_chunk, S);
  BK(bk_bicg_update, gc, B.d_chunks, nc, kmask, B.d_sc, B.d_x, B.d_r, B.d_p, B.d_sv, B.d_t, B.d_rh, B.d_invd,
     B.d_part);
  BK(bk_bicg_decide, gs, B.d_sc, B.d_active, B.d_defect, B.d_part, B.d_slot_chunk, S, B.delta);
  // FP64 defects b - A x of the slots whose FP32 residual dropped by delta (or that look converged)
  launch_batch_apply<double>(B.plan, B.d_params, B.d_x, B.d_r64, B.d_defect, cap, st);
  BK(bk_defect, gc, B.d_chunks, nc, B.d_defect, B.d_b, B.d_r64, B.d_part);
  BK(bk_defect_decide, gs, B.d_sc, B.d_active, B.d_defect, B.d_part, B.d_slot_chunk, S);
  BK(bk_cg_replace, gc, B.d_chunks, nc, B.d_defect, B.d_sc, B.d_r64, B.d_r, B.d_z, B.d_invd, B.d_part);
  BK(bk_cg_replace_finish, gs, B.d_sc, B.d_defect, B.d_part, B.d_slot_chunk, S);
  BK(bk_bicg_replace, gc, B.d_chunks, nc, B.d_defect, B.d_sc, B.d_r64, B.d_r, B.d_rh, B.d_p, B.d_part);
  BK(bk_bicg_replace_finish, gs, B.d_sc, B.d_defect, B.d_part, B.d_slot_chunk, S);
  // search directions and scalar shifts
  BK(bk_cg_direction, gc, B.d_chunks, nc, B.d_active, B.d_sc, B.d_z, B.d_p);
  BK(bk_bicg_direction, gc, B.d_chunks, nc, B.d_active, B.d_defect, B.d_sc, B.d_r, B.d_p, B.d_v);
  BK(bk_cg_shift, gs, B.d_sc, B.d_active, S);
  BK(bk_bicg_shift, gs, B.d_sc, B.d_active, S);
  BK(bk_count_running, 1, B.d_active, S, B.d_running);
#undef BK
}

void ensure_graph(Batch &B)
{
  if (B.dirty) rebuild_tables(B);
  if (B.graph) return;
  // one-time launcher set-up (tables, occupancy) must not happen inside the capture
  launch_batch_apply<float>(BatchApplyPlan{}, nullptr, nullptr, nullptr, nullptr, 0, B.stream);
  launch_batch_apply<double>(BatchApplyPlan{}, nullptr, nullptr, nullptr, nullptr, 0, B.stream);
  const int64_t before = mpdg_kernel_launches();
  cudaGraph_t g = nullptr;
  MPDG_CUDA(cudaStreamBeginCapture(B.stream, cudaStreamCaptureModeThreadLocal));
  try {
    enqueue_step(B, B.tuned_cap);
  } catch (...) {
    cudaStreamEndCapture(B.stream, &g);
    if (g) cudaGraphDestroy(g);
    count_launch(-(int)(mpdg_kernel_launches() - before));
    throw;
  }
  MPDG_CUDA(cudaStreamEndCapture(B.stream, &g));
  B.step_kernels = mpdg_kernel_launches() - before;
  count_launch(-(int)B.step_kernels);  // captured, not launched
  const cudaError_t e = cudaGraphInstantiate(&B.graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    B.graph = nullptr;
    throw Error{MPDG_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e)};
  }
}

double now_s()
{
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int find_slot(const Batch &B, int64_t ticket)
{
  for (int s = 0; s < B.capacity; ++s)
    if (B.slots[s].used && B.slots[s].ticket == ticket) return s;
  return -1;
}

// admission of one problem: slot vectors from the pool, Jacobi diagonal,
// right-hand side, initial state.  Only enqueues work on the batch stream.
int admit(Batch &B, const mpdg_problem_desc &d, const double *b_host, int64_t &ticket)
{
  check_desc(d);
  const long N = problem_dofs(d);
  const size_t bytes = slot_bytes(N, d.kind);
  if (B.used + (int64_t)bytes > B.budget) return MPDG_ERR_BUDGET;
  int s = -1;
  for (int k = 0; k < B.capacity; ++k)
    if (!B.slots[k].used) {
      s = k;
      break;
    }
  if (s < 0) return MPDG_ERR_BUDGET;
  BatchSlot &S = B.slots[s];
  S = BatchSlot{};
  S.desc = d;
  S.N = N;
  S.bytes = bytes;
  try {
    S.x = palloc<double>(B, N);
    S.b = palloc<double>(B, N);
    S.r64 = palloc<double>(B, N);
    S.r = palloc<float>(B, N);
    S.z = palloc<float>(B, N);
    S.p = palloc<float>(B, N);
    S.Ap = palloc<float>(B, N);
    S.invd = palloc<float>(B, N);
    if (d.kind == MPDG_OP_ADVDIFF) {
      S.rh = palloc<float>(B, N);
      S.v = palloc<float>(B, N);
      S.sv = palloc<float>(B, N);
      S.t = palloc<float>(B, N);
    }
  } catch (...) {
    free_slot_vectors(B, S);
    S = BatchSlot{};
    throw;
  }
  S.used = true;
  B.used += (int64_t)bytes;
  cudaStream_t st = B.stream;
  const long NX = (long)d.nc * d.degree + 1;
  enqueue_diagonal(d, S.r64, S.invd, nullptr, st);  // r64 is free scratch until the first defect
  if (b_host) {
    MPDG_CUDA(cudaMemcpyAsync(S.b, b_host, sizeof(double) * N, cudaMemcpyHostToDevice, st));
    if (d.dirichlet) {
      bk_set_boundary<<<grid1(N), 256, 0, st>>>(S.b, N, NX, 0.0);
      MPDG_LAUNCHED();
    }
  } else {
    bk_rhs<<<grid1(N), 256, 0, st>>>(S.b, N, NX, d.dirichlet, (unsigned long long)d.rhs_seed);
    MPDG_LAUNCHED();
  }
  dev_dot(S.b, S.b, N, B.d_adm, B.d_adm + kAdmBB, st);
  bk_init_vectors<<<kRedBlocks, 256, 0, st>>>(S.b, B.d_adm + kAdmBB, S.x, S.r, S.z, S.p, S.invd, S.rh, N,
                                              B.d_adm + kAdmInit);
  MPDG_LAUNCHED();
  const double rel = (d.rel_tolerance > 0.0 || d.abs_tolerance > 0.0) ? d.rel_tolerance : 1e-10;
  bk_init_scalars<<<1, 256, 0, st>>>(B.d_sc, B.d_active, B.d_defect, B.d_params, s, B.d_adm + kAdmInit,
                                     kRedBlocks, B.d_adm + kAdmBB, d.kind,
                                     d.max_iterations > 0 ? d.max_iterations : B.max_it, rel, d.abs_tolerance,
                                     slot_params(d));
  MPDG_LAUNCHED();
  S.ticket = B.next_ticket++;
  S.t_admit = now_s();
  ticket = S.ticket;
  B.dirty = true;
  return MPDG_OK;
}

void release(Batch &B, int s)
{
  BatchSlot &S = B.slots[s];
  free_slot_vectors(B, S);
  B.used -= (int64_t)S.bytes;
  S = BatchSlot{};
  MPDG_CUDA(cudaMemsetAsync(B.d_active + s, 0, sizeof(int), B.stream));
  MPDG_CUDA(cudaMemsetAsync(B.d_defect + s, 0, sizeof(int), B.stream));
  B.dirty = true;
}

void report_of(const SlotScalars &q, mpdg_solve_report &rep)
{
  rep = mpdg_solve_report{};
  rep.status = q.status == SL_RUNNING         ? 1
               : q.status == SL_CONVERGED     ? MPDG_OK
               : q.status == SL_NOT_CONVERGED ? MPDG_ERR_NOT_CONVERGED
               : q.status == SL_NAN           ? MPDG_ERR_NAN
                                              : MPDG_ERR_BREAKDOWN;
  rep.iterations = q.iters;
  rep.outer_iterations = q.defects;
  rep.operator_applies = (q.kind == MPDG_OP_ADVDIFF ? 2 : 1) * q.iters + q.defects;
  rep.initial_residual = q.res0;
  rep.final_residual = q.res;
}

void fetch_scalars(Batch &B)
{
  MPDG_CUDA(cudaMemcpyAsync(B.h_sc, B.d_sc, sizeof(SlotScalars) * B.capacity, cudaMemcpyDeviceToHost, B.stream));
  MPDG_CUDA(cudaStreamSynchronize(B.stream));
}

int used_slots(const Batch &B)
{
  int k = 0;
  for (const BatchSlot &S : B.slots) k += S.used ? 1 : 0;
  return k;
}

// up to max_steps graph launches, reading the running count every poll steps
int run_steps(Batch &B, int max_steps, int poll, int &running)
{
  running = 0;
  if (used_slots(B) == 0 || max_steps <= 0) return 0;
  ensure_graph(B);
  if (B.n_chunks == 0) return 0;
  poll = std::max(1, poll);
  int steps = 0;
  while (steps < max_steps) {
    const int k = std::min(poll, max_steps - steps);
    for (int i = 0; i < k; ++i) MPDG_CUDA(cudaGraphLaunch(B.graph, B.stream));
    count_launch((int)(k * B.step_kernels));
    steps += k;
    MPDG_CUDA(cudaMemcpyAsync(B.h_running, B.d_running, sizeof(int), cudaMemcpyDeviceToHost, B.stream));
    MPDG_CUDA(cudaStreamSynchronize(B.stream));
    running = *B.h_running;
    if (running == 0) break;
  }
  return steps;
}

double slot_norm(Batch &B, const BatchSlot &S)
{
  dev_dot(S.x, S.x, S.N, B.d_adm, B.d_adm + kAdmNorm, B.stream);
  double v = 0.0;
  MPDG_CUDA(cudaMemcpyAsync(&v, B.d_adm + kAdmNorm, sizeof(double), cudaMemcpyDeviceToHost, B.stream));
  MPDG_CUDA(cudaStreamSynchronize(B.stream));
  return std::sqrt(v);
}

void destroy_batch(Batch &B)
{
  if (B.stream) cudaStreamSynchronize(B.stream);
  for (int s = 0; s < B.capacity; ++s)
    if (B.slots[s].used) free_slot_vectors(B, B.slots[s]);
  if (B.stream) cudaStreamSynchronize(B.stream);
  free_plan(B);
  for (void *p : {(void *)B.d_sc, (void *)B.d_params, (void *)B.d_active, (void *)B.d_defect, (void *)B.d_x,
                  (void *)B.d_b, (void *)B.d_r64, (void *)B.d_r, (void *)B.d_z, (void *)B.d_p, (void *)B.d_Ap,
                  (void *)B.d_invd, (void *)B.d_rh, (void *)B.d_v, (void *)B.d_sv, (void *)B.d_t,
                  (void *)B.d_running, (void *)B.d_adm, (void *)B.d_slot_chunk})
    if (p) cudaFree(p);
  if (B.h_running) cudaFreeHost(B.h_running);
  if (B.h_sc) cudaFreeHost(B.h_sc);
  if (B.pool) cudaMemPoolDestroy(B.pool);
  if (B.stream) cudaStreamDestroy(B.stream);
}

}  // namespace
}  // namespace mpdg

struct mpdg_batch {
  mpdg::Batch b;
};

using namespace mpdg;

extern "C" {

mpdg_status mpdg_batch_create(int64_t budget_bytes, int capacity, double reliable_delta, mpdg_batch **out)
{
  return guarded([&]() -> int {
    if (!out) throw Error{MPDG_ERR_ARG, "null argument"};
    if (budget_bytes <= 0 || capacity < 1 || capacity > 65536)
      throw Error{MPDG_ERR_ARG, "budget must be positive and capacity 1..65536"};
    if (!(reliable_delta > 0.0 && reliable_delta < 1.0)) throw Error{MPDG_ERR_ARG, "reliable_delta must be in (0,1)"};
    auto *h = new mpdg_batch();
    Batch &B = h->b;
    try {
      B.budget = budget_bytes;
      B.capacity = capacity;
      B.delta = reliable_delta;
      MPDG_CUDA(cudaGetDevice(&B.device));
      MPDG_CUDA(cudaStreamCreateWithFlags(&B.stream, cudaStreamNonBlocking));
      cudaMemPoolProps props{};
      props.allocType = cudaMemAllocationTypePinned;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = B.device;
      MPDG_CUDA(cudaMemPoolCreate(&B.pool, &props));
      uint64_t keep = UINT64_MAX;
      MPDG_CUDA(cudaMemPoolSetAttribute(B.pool, cudaMemPoolAttrReleaseThreshold, &keep));
      B.slots.resize(capacity);
      B.d_sc = balloc<SlotScalars>(capacity);
      B.d_params = balloc<BatchSlotParams>(capacity);
      B.d_active = balloc<int>(2 * (size_t)capacity);
      B.d_defect = balloc<int>(capacity);
      B.d_x = balloc<double *>(capacity);
      B.d_b = balloc<double *>(capacity);
      B.d_r64 = balloc<double *>(capacity);
      B.d_r = balloc<float *>(capacity);
      B.d_z = balloc<float *>(capacity);
      B.d_p = balloc<float *>(capacity);
      B.d_Ap = balloc<float *>(capacity);
      B.d_invd = balloc<float *>(capacity);
      B.d_rh = balloc<float *>(capacity);
      B.d_v = balloc<float *>(capacity);
      B.d_sv = balloc<float *>(capacity);
      B.d_t = balloc<float *>(capacity);
      B.d_running = balloc<int>(1);
      B.d_adm = balloc<double>(kAdmDoubles);
      B.d_slot_chunk = balloc<int>(2 * (size_t)capacity);
      MPDG_CUDA(cudaMemset(B.d_sc, 0, sizeof(SlotScalars) * capacity));
      MPDG_CUDA(cudaMemset(B.d_active, 0, sizeof(int) * 2 * capacity));
      MPDG_CUDA(cudaMemset(B.d_defect, 0, sizeof(int) * capacity));
      MPDG_CUDA(cudaMemset(B.d_slot_chunk, 0, sizeof(int) * 2 * capacity));
      MPDG_CUDA(cudaHostAlloc((void **)&B.h_running, sizeof(int), cudaHostAllocDefault));
      MPDG_CUDA(cudaHostAlloc((void **)&B.h_sc, sizeof(SlotScalars) * capacity, cudaHostAllocDefault));
    } catch (...) {
      destroy_batch(B);
      delete h;
      throw;
    }
    *out = h;
    return MPDG_OK;
  });
}

mpdg_status mpdg_batch_destroy(mpdg_batch *batch)
{
  if (!batch) return MPDG_OK;
  destroy_batch(batch->b);
  delete batch;
  return MPDG_OK;
}

mpdg_status mpdg_problem_bytes(const mpdg_problem_desc *desc, int64_t *bytes, int64_t *n_dofs)
{
  return guarded([&]() -> int {
    if (!desc) throw Error{MPDG_ERR_ARG, "null argument"};
    check_desc(*desc);
    const long N = problem_dofs(*desc);
    if (bytes) *bytes = (int64_t)slot_bytes(N, desc->kind);
    if (n_dofs) *n_dofs = N;
    return MPDG_OK;
  });
}

mpdg_status mpdg_problem_rhs_host(const mpdg_problem_desc *desc, double *b_host)
{
  return guarded([&]() -> int {
    if (!desc || !b_host) throw Error{MPDG_ERR_ARG, "null argument"};
    check_desc(*desc);
    rhs_host(*desc, b_host);
    return MPDG_OK;
  });
}

mpdg_status mpdg_problem_diagonal_host(const mpdg_problem_desc *desc, double *diag_host)
{
  return guarded([&]() -> int {
    if (!desc || !diag_host) throw Error{MPDG_ERR_ARG, "null argument"};
    check_desc(*desc);
    const long N = problem_dofs(*desc), NX = (long)desc->nc * desc->degree + 1;
    double *F = balloc<double>(4 * (size_t)NX), *d = nullptr;
    try {
      d = balloc<double>(N);
      enqueue_diagonal(*desc, F, nullptr, d, 0);
      MPDG_CUDA(cudaMemcpy(diag_host, d, sizeof(double) * N, cudaMemcpyDeviceToHost));
    } catch (...) {
      cudaFree(F);
      if (d) cudaFree(d);
      throw;
    }
    cudaFree(F);
    cudaFree(d);
    return MPDG_OK;
  });
}

mpdg_status mpdg_batch_submit(mpdg_batch *batch, const mpdg_problem_desc *desc, const double *rhs, int64_t *ticket)
{
  return guarded([&]() -> int {
    if (!batch || !desc || !ticket) throw Error{MPDG_ERR_ARG, "null argument"};
    const int rc = admit(batch->b, *desc, rhs, *ticket);
    if (rc == MPDG_ERR_BUDGET) set_last_error("problem does not fit the free budget or no slot is free");
    return rc;
  });
}

mpdg_status mpdg_batch_run(mpdg_batch *batch, int max_steps, int poll_steps, int *steps, int *running)
{
  return guarded([&]() -> int {
    if (!batch) throw Error{MPDG_ERR_ARG, "null argument"};
    int r = 0;
    const int k = run_steps(batch->b, max_steps, poll_steps, r);
    if (steps) *steps = k;
    if (running) *running = r;
    return MPDG_OK;
  });
}

mpdg_status mpdg_batch_poll(mpdg_batch *batch, int64_t ticket, mpdg_solve_report *report)
{
  return guarded([&]() -> int {
    if (!batch || !report) throw Error{MPDG_ERR_ARG, "null argument"};
    Batch &B = batch->b;
    const int s = find_slot(B, ticket);
    if (s < 0) throw Error{MPDG_ERR_ARG, "unknown ticket"};
    MPDG_CUDA(cudaMemcpyAsync(B.h_sc + s, B.d_sc + s, sizeof(SlotScalars), cudaMemcpyDeviceToHost, B.stream));
    MPDG_CUDA(cudaStreamSynchronize(B.stream));
    report_of(B.h_sc[s], *report);
    return MPDG_OK;
  });
}

mpdg_status mpdg_batch_take(mpdg_batch *batch, int64_t ticket, double *x_host, mpdg_solve_report *report)
{
  return guarded([&]() -> int {
    if (!batch) throw Error{MPDG_ERR_ARG, "null argument"};
    Batch &B = batch->b;
    const int s = find_slot(B, ticket);
    if (s < 0) throw Error{MPDG_ERR_ARG, "unknown ticket"};
    MPDG_CUDA(cudaMemcpyAsync(B.h_sc + s, B.d_sc + s, sizeof(SlotScalars), cudaMemcpyDeviceToHost, B.stream));
    MPDG_CUDA(cudaStreamSynchronize(B.stream));
    if (B.h_sc[s].status == SL_RUNNING) throw Error{MPDG_ERR_ARG, "problem still running"};
    const BatchSlot &S = B.slots[s];
    if (x_host) {
      MPDG_CUDA(cudaMemcpyAsync(x_host, S.x, sizeof(double) * S.N, cudaMemcpyDeviceToHost, B.stream));
      MPDG_CUDA(cudaStreamSynchronize(B.stream));
    }
    if (report) report_of(B.h_sc[s], *report);
    release(B, s);
    return MPDG_OK;
  });
}

mpdg_status mpdg_batch_autotune(mpdg_batch *batch, int *ctas_per_sm, double *apply_ms)
{
  return guarded([&]() -> int {
    if (!batch) throw Error{MPDG_ERR_ARG, "null argument"};
    Batch &B = batch->b;
    if (used_slots(B) == 0) throw Error{MPDG_ERR_ARG, "autotuning needs admitted problems"};
    if (B.dirty) rebuild_tables(B);
    std::vector<int> ones(B.capacity, 0);
    for (int s = 0; s < B.capacity; ++s) ones[s] = B.slots[s].used ? 1 : 0;
    int *d_all = balloc<int>(B.capacity);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int best_cap = 0;
    double best = 1e30;
    try {
      MPDG_CUDA(cudaMemcpy(d_all, ones.data(), sizeof(int) * B.capacity, cudaMemcpyHostToDevice));
      MPDG_CUDA(cudaEventCreate(&e0));
      MPDG_CUDA(cudaEventCreate(&e1));
      for (int cap : {1, 2, 3, 4, 6, 8, 0}) {
        launch_batch_apply<float>(B.plan, B.d_params, B.d_p, B.d_Ap, d_all, cap, B.stream);
        MPDG_CUDA(cudaEventRecord(e0, B.stream));
        const int reps = 5;
        for (int r = 0; r < reps; ++r) launch_batch_apply<float>(B.plan, B.d_params, B.d_p, B.d_Ap, d_all, cap, B.stream);
        MPDG_CUDA(cudaEventRecord(e1, B.stream));
        MPDG_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        MPDG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        const double t = ms / reps;
        if (t < best * 0.98) {  // prefer the earlier (smaller) cap unless clearly faster
          best = t;
          best_cap = cap;
        }
      }
    } catch (...) {
      cudaFree(d_all);
      if (e0) cudaEventDestroy(e0);
      if (e1) cudaEventDestroy(e1);
      throw;
    }
    cudaFree(d_all);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    B.tuned_cap = best_cap;
    B.tuned_ms = best;
    drop_graph(B);
    if (ctas_per_sm) *ctas_per_sm = best_cap;
    if (apply_ms) *apply_ms = best;
    return MPDG_OK;
  });
}

mpdg_status mpdg_batch_used_bytes(mpdg_batch *batch, int64_t *bytes)
{
  if (!batch || !bytes) return MPDG_ERR_ARG;
  *bytes = batch->b.used;
  return MPDG_OK;
}

mpdg_status mpdg_serve(mpdg_batch *batch, const mpdg_problem_desc *req, const double *arrival_s, int n,
                       int poll_steps, double **x_host, double *latency_s, double *x_norm,
                       mpdg_solve_report *reports, double *wall_s)
{
  return guarded([&]() -> int {
    if (!batch || (!req && n > 0) || (!arrival_s && n > 0) || n < 0) throw Error{MPDG_ERR_ARG, "null argument"};
    Batch &B = batch->b;
    if (used_slots(B) != 0) throw Error{MPDG_ERR_ARG, "serving starts on an empty batch"};
    long max_n = 0;
    for (int i = 0; i < n; ++i) {
      check_desc(req[i]);
      if (i && arrival_s[i] < arrival_s[i - 1]) throw Error{MPDG_ERR_ARG, "arrival times must ascend"};
      const long N = problem_dofs(req[i]);
      if ((int64_t)slot_bytes(N, req[i].kind) > B.budget)
        throw Error{MPDG_ERR_BUDGET, "a request is larger than the whole budget"};
      max_n = std::max(max_n, N);
    }
    double *staging = nullptr;
    if (max_n) MPDG_CUDA(cudaHostAlloc((void **)&staging, sizeof(double) * max_n, cudaHostAllocDefault));
    std::vector<int> slot_req(B.capacity, -1);
    int next = 0, done = 0;
    const double t0 = now_s();
    double t_last = t0;
    try {
      while (done < n) {
        const double t = now_s() - t0;
        while (next < n && arrival_s[next] <= t) {
          int64_t tk = -1;
          if (admit(B, req[next], nullptr, tk) != MPDG_OK) break;  // waits for memory or a slot
          slot_req[find_slot(B, tk)] = next;
          ++next;
        }
        if (used_slots(B) == 0) {
          if (next < n) {
            const double wait = arrival_s[next] - (now_s() - t0);
            if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 0.05)));
          }
          continue;
        }
        int running = 0;
        run_steps(B, std::max(1, poll_steps), std::max(1, poll_steps), running);
        fetch_scalars(B);
        for (int s = 0; s < B.capacity; ++s) {
          if (!B.slots[s].used || B.h_sc[s].status == SL_RUNNING) continue;
          const int i = slot_req[s];
          const BatchSlot &S = B.slots[s];
          if (x_norm) x_norm[i] = slot_norm(B, S);
          double *dst = (x_host && x_host[i]) ? x_host[i] : staging;
          MPDG_CUDA(cudaMemcpyAsync(dst, S.x, sizeof(double) * S.N, cudaMemcpyDeviceToHost, B.stream));
          MPDG_CUDA(cudaStreamSynchronize(B.stream));
          t_last = now_s();
          if (latency_s) latency_s[i] = (t_last - t0) - arrival_s[i];
          if (reports) report_of(B.h_sc[s], reports[i]);
          release(B, s);
          slot_req[s] = -1;
          ++done;
        }
      }
    } catch (...) {
      if (staging) cudaFreeHost(staging);
      throw;
    }
    if (staging) cudaFreeHost(staging);
    if (wall_s) *wall_s = t_last - t0;
    return MPDG_OK;
  });
}

}  // extern "C"
