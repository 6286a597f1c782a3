// Internal declarations of libmpdg (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <new>
#include <string>
#include <vector>

#include "../../include/mpdg.h"

namespace mpdg {

constexpr int kMaxDegree = 4;
constexpr int kMaxN = kMaxDegree + 1;

// Per-cell strides of the streamed geometry (7 metric values, 3 velocity
// values per quadrature point), padded to 4 elements so that every cell block
// starts on a 16-byte boundary in both precisions (bulk-copy requirement).
__host__ __device__ constexpr int metric_stride(int n) { return ((7 * n * n * n + 3) / 4) * 4; }
__host__ __device__ constexpr int velb_stride(int n) { return ((3 * n * n * n + 3) / 4) * 4; }

// thrown inside the library, converted to a status code at the C boundary
struct Error {
  int status;
  std::string msg;
};

void set_last_error(const std::string &msg);
void count_launch(int n = 1);

// Every device and pinned-host allocation of the library goes through these
// wrappers, which count them (mpdg_allocations): tests use the count to show
// that an entry point allocated nothing.
void count_allocation();
inline cudaError_t tracked_malloc_raw(void **p, size_t bytes)
{
  count_allocation();
  return cudaMalloc(p, bytes);
}
template <typename T>
inline cudaError_t tracked_malloc(T **p, size_t bytes)
{
  return tracked_malloc_raw(reinterpret_cast<void **>(p), bytes);
}
template <typename T>
inline cudaError_t tracked_malloc_async(T **p, size_t bytes, cudaStream_t s)
{
  count_allocation();
  return cudaMallocAsync(reinterpret_cast<void **>(p), bytes, s);
}
template <typename T>
inline cudaError_t tracked_malloc_pool_async(T **p, size_t bytes, cudaMemPool_t pool, cudaStream_t s)
{
  count_allocation();
  return cudaMallocFromPoolAsync(reinterpret_cast<void **>(p), bytes, pool, s);
}
template <typename T>
inline cudaError_t tracked_malloc_host(T **p, size_t bytes)
{
  count_allocation();
  return cudaMallocHost(reinterpret_cast<void **>(p), bytes);
}

// runs the body of an extern "C" entry: internal errors become status codes
template <typename F>
int guarded(F &&f)
{
  try {
    return f();
  } catch (const Error &e) {
    set_last_error(e.msg);
    return e.status;
  } catch (const std::bad_alloc &) {
    set_last_error("host allocation failed");
    return MPDG_ERR_ALLOC;
  } catch (...) {
    set_last_error("unknown error");
    return MPDG_ERR_ARG;
  }
}

#define MPDG_CUDA(call)                                                               \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                            \
      throw ::mpdg::Error{MPDG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
  } while (0)

#define MPDG_LAUNCHED()                                      \
  do {                                                       \
    cudaError_t e_ = cudaGetLastError();                     \
    if (e_ != cudaSuccess)                                   \
      throw ::mpdg::Error{MPDG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e_)}; \
    ::mpdg::count_launch();                                  \
  } while (0)

// Cells are processed in 8 parity colours (ix%2, iy%2, iz%2): two cells of one
// colour never share a DoF, so a colour's cells add into dst without atomics.
struct Colour {
  int par[3];
  int cn[3];     // cells per direction in this colour
  long count;    // cells in this colour
  long first;    // index of its first cell in colour-major order
};

struct Mesh {
  int degree = 1, n = 2;
  int nc[3] = {1, 1, 1};
  long NX = 0, NY = 0, NZ = 0, N = 0, n_cells = 0;
  bool uniform = false;
  double h[3] = {0, 0, 0}, origin[3] = {0, 0, 0};
  Colour colour[8];
  std::vector<double> vertices;        // host copy
  double *d_vert = nullptr;            // device vertices
  double *d_metric64 = nullptr;        // general geometry: [colour-major cell][7][n^3]
  float *d_metric32 = nullptr;
  uint8_t *d_dmask = nullptr;          // Dirichlet mask per DoF (nullptr: none)
  uint8_t *d_cell_flags = nullptr;     // per colour-major cell: bit0 touches a constrained DoF
  uint32_t *d_cell_mask = nullptr;     // per colour-major cell: 128-bit mask of its constrained
                                       // local DoFs (bit k*n*n + j*n + i)
  // mapped meshes: per colour-major cell, 128-bit mask of the local DoFs it
  // touches first in colour order (it stores them; later colours add)
  uint32_t *d_cell_first = nullptr;
  bool all_dofs_touched = false;       // mapped meshes: every DoF lies in some cell
  // mapped meshes: cells' local faces with a boundary id, grouped by face
  // colour (faces of a colour share no DoF), colour c at [mface_first[c], [c+1])
  int *d_mface_cell = nullptr;
  int8_t *d_mface_f = nullptr, *d_mface_id = nullptr;
  int8_t *d_cell_fids = nullptr;       // per colour-major cell: its 6 faces' boundary ids
  std::vector<long> mface_first;
  bool has_dirichlet = false;
  size_t device_bytes = 0;
  bool metric32_ready = false;
  // Two-level mesh (hanging nodes): this mesh is the coarse block and `fine`
  // the fine block, refined 2:1 in y and z, meeting at the coarse block's
  // x = max face.  Vectors hold the coarse block's N_own DoFs, then the fine
  // block's; N is their sum.  The fine DoFs on the interface plane hang on the
  // coarse faces (read through the interpolation, never written).
  Mesh *fine = nullptr;
  long N_own = 0;
  // Mapped mesh (mpdg_mesh_create_mapped): cells given by their corners and
  // their cell->DoF map, coloured greedily so that no two cells of a colour
  // share a DoF; homogeneous affine constraints distributed before and
  // condensed after the cell loop.
  bool mapped = false;
  std::vector<Colour> mcol;          // count and first of each colour (cn = {count, 1, 1})
  int *d_cmap = nullptr;             // [colour-major cell][n^3] global DoFs
  double *d_cellvert = nullptr;      // [colour-major cell][8][3] corners
  long n_cons = 0, n_masters = 0;
  long *d_cons_dof = nullptr, *d_cons_ptr = nullptr, *d_cons_mast = nullptr;  // per constraint
  double *d_cons_w = nullptr;
  long *d_mast_dof = nullptr, *d_mast_ptr = nullptr, *d_mast_cons = nullptr;  // per master
  double *d_mast_w = nullptr;
  int *d_cons_of = nullptr;          // per DoF: its constraint index, or -1
  std::vector<long> ccells;          // colour-major cells that touch a constrained DoF
  long *d_ccells = nullptr;
  uint8_t *d_tmask_dir = nullptr;   // whole vector: Dirichlet or hanging
  uint8_t *d_tmask_hang = nullptr;  // whole vector: hanging only
};

struct Workspace;  // solver vectors (solvers.cu)

constexpr int kPipeSlabs = 8;       // z-slabs of the pipelined host-buffer apply
constexpr int kMaxApplySlabs = 32;  // z-slabs of the resident apply

// schedule of the resident warp apply (mpdg_op_set_schedule, mpdg_op_autotune);
// the defaults are the fastest measured at the benchmark configurations on a
// B200 (colour overlap: FP64 Q4 64^3 0.519 -> 0.488 ms, FP32 0.327 -> 0.294 ms
// with the evict-first hint; z-slabs only add launch tails there)
struct ApplySchedule {
  int slabs = 1;        // z-slabs of cell layers, each running its 8 colours
  int evict_first = 0;  // L2 evict-first hint on the coefficient stream
  int pdl = 1;          // colour launches as programmatic dependents of the previous one
  int cta = 0;          // cell groups of a whole CTA (Q2, Q4) instead of a warp
  int lane = 0;         // one thread per cell (Q1, Q2 on uniform lattices, constant coefficients)
};

struct Op {
  Mesh *mesh = nullptr;
  mpdg_op_desc d{};
  bool use_dirichlet = true;
  cudaStream_t stream = nullptr;
  const double *T64 = nullptr;         // temperature (device): caller-owned, or T_own
  double *T_own = nullptr;             // operator-owned copy set from host values
  float *T32 = nullptr;                // FP32 copy of T
  // material-law fields: T_old (laws with a solid phase) and the level-set
  // heaviside (two-phase laws), caller-owned or set from host values
  const double *Told64 = nullptr, *H64 = nullptr;
  double *Told_own = nullptr, *H_own = nullptr;
  float *Told32 = nullptr, *H32 = nullptr;  // FP32: T - T_old and the heaviside
  float *Ts32 = nullptr;                    // FP32, laws with a solid phase: T - solidus
  // velocity as a DoF vector (MPDG_VEL_NODAL): component-major [3][N],
  // caller-owned or set from host values
  const double *U64 = nullptr;
  double *U_own = nullptr;
  double *d_velb64 = nullptr;          // general geometry or nodal velocity: [cell][3][n^3]
  float *d_velb32 = nullptr;
  float *d_trig32 = nullptr;           // uniform vortex velocity: sin/cos tables
  double *d_tau64 = nullptr;           // SUPG: tau_K per colour-major cell
  double *d_lam64 = nullptr;           // SUPG with diffusion on general cells: Laplacian curvature term
  float *d_lam32 = nullptr;
  float *d_tau32 = nullptr;
  double *d_trig64 = nullptr;
  Workspace *ws = nullptr;
  int *d_err = nullptr;                // device error word (bounded waits that expired)
  // merged per-quadrature-point coefficients for the general-geometry apply:
  // [cell][7][n^3] = c_mass JxW, c_diff k(T_q) G (G = JxW J^-1 J^-T, 6 entries)
  double *d_coef64 = nullptr;
  float *d_coef32 = nullptr;
  bool coef64_ok = false, coef32_ok = false;
  size_t device_bytes = 0;
  // two-level mesh: the fine block's operator and the per-interface-cell stage
  // of the hanging DoFs' contributions to the coarse DoFs
  Op *fine = nullptr;
  void *d_stage = nullptr;
  // set on the fine block's operator for one apply: where the hanging DoFs read from
  const void *hang_src = nullptr;
  const uint8_t *hang_mask = nullptr;
  long hang_NXc = 0, hang_NYc = 0;  // the coarse lattice the hanging DoFs read from
  // inflow/outflow constraints (advection_diffusion_operator.cpp:545-578): identity
  // rows at the flagged DoFs; the source there is read as 0 and copied to the result
  uint8_t *d_io = nullptr;
  // device copies of the host vectors of mpdg_vmult_host (src, dst)
  double *host_stage = nullptr;
  // z-slab pipeline of the host-buffer apply: copy-in and copy-out streams and
  // one event per slab and stage (created on first use)
  cudaStream_t pipe_in = nullptr, pipe_out = nullptr;
  cudaEvent_t pipe_ev[2 * kPipeSlabs] = {};
  // least-squares predictor: images of the old solutions (lsq_cols vectors of N)
  double *lsq_buf = nullptr;
  int lsq_cols = 0;
  void *io_tmp = nullptr;
  size_t io_tmp_bytes = 0;
  ApplySchedule sched[2] = {ApplySchedule{1, 0, 1, 0}, ApplySchedule{1, 1, 1, 0}};  // [MPDG_FP64], [MPDG_FP32]
};

// ---- batched apply over many solves (batch_apply.cuh / batch.cu)
// per problem and colour: cells of the colour, cells per direction in x and y,
// warp groups (cells per warp packed), magic divisors of cn0 and cn0*cn1
struct SlotColour {
  int count, cn0, cn1, groups;
  unsigned long long m0, m01;
};

// static description of a batch slot (written when a problem is admitted)
struct SlotInfo {
  int degree, nc, kind, n_chunks;
  long NX, N;
  SlotColour col[8];
};

struct BatchSlotParams {
  double c_mass, c_vel, c_diff;    // heat: rho_cp/dt, rho_cp, k0; advdiff: 1/dt, theta, theta D
  double hvol, ih, ih2, h;
  int vel_kind, dirichlet;
};

// compacted work list of the flagged slots, rebuilt on the device every step:
// per colour the flagged slots with cells of that colour and the prefix of
// their warp groups; the flagged slots with the prefix of their vector chunks
struct BatchScheduleHeader {
  int n_seg[8], total_groups[8];
  int n_slots, total_chunks;
};

struct BatchSchedule {
  BatchScheduleHeader *hdr = nullptr;
  int *seg_slot = nullptr;    // [8][cap]
  int *seg_prefix = nullptr;  // [8][cap]
  int *act_slot = nullptr;    // [cap]
  int *chunk_prefix = nullptr;  // [cap]
  int cap = 0;
};

// cells per warp of the warp-per-cell kernels for degree p (32 / (p+1)^2)
int cells_per_warp(int degree);
// one-time set-up of the batched apply (tables, occupancy): before any graph capture
void batch_apply_setup();
// block and tile shape of the batched apply (picked by mpdg_batch_autotune):
// warps per CTA (2, 4, 8), the conflict-minimal or the plain tile layout, and
// the resident CTAs per SM of its persistent grid (0: the occupancy maximum)
struct BatchShape {
  int warps_per_cta = 4;
  bool tuned_tiles = true;
  int ctas_per_sm = 0;
};
// one launch per colour over the scheduled slots whose mask entry is set; persistent
// grid of SMs x min(ctas_per_sm, occupancy) CTAs
template <typename Real>
void launch_batch_apply(const BatchSchedule &sched, const SlotInfo *info, const BatchSlotParams *params,
                        Real *const *src, Real *const *dst, const int *mask, const BatchShape &shape,
                        cudaStream_t s);

// ---- operator kernels (operator_kernels.cu)
// 1D tables of degree p on [0,1]: GLL Lagrange basis values S[q*(p+1)+i] and
// derivatives D at the p+1 Gauss points x with weights w
void shape_1d(int p, double *S, double *D, double *w, double *x);

void build_mesh_device_data(Mesh &m, const uint8_t *host_mask, bool force_general);
void ensure_metric32(Mesh &m, cudaStream_t s);
void build_op_device_data(Op &op);
// interpolates the nodal velocity field op.U64 to the quadrature points: the
// stream JxW J^-1 u of the apply (both precisions) and, with SUPG, tau_K
void build_nodal_velocity(Op &op);
void ensure_T32(Op &op);
void fma_peak(double &gflops64, double &gflops32);
void build_mapped_mesh(Mesh &m, const mpdg_mapped_mesh_desc &d);
inline bool law_has_solid(int mat) { return mat == MPDG_MAT_LIQUID_SOLID || mat == MPDG_MAT_GAS_LIQUID_SOLID; }
inline bool law_two_phase(int mat) { return mat == MPDG_MAT_GAS_LIQUID || mat == MPDG_MAT_GAS_LIQUID_SOLID; }
// marks the merged coefficient stream stale (new temperature field or dt)
void invalidate_coef(Op &op);

template <typename Real>
void launch_apply(Op &op, Real *dst, const Real *src);
template <typename Real>
void launch_apply_multi(Op &op, int nvec, Real *const *dst, const Real *const *src);
// the operator's apply is the warp kernel alone (no faces, identity rows,
// hanging nodes, SUPG, Newton tangent or phase law; a lattice mesh)
bool plain_warp_apply(const Op &op);
// the cells of z-layers [z0, z1) of a plain warp apply; dst holds the first
// stores of their DoFs (layer ranges must be applied in increasing order and
// end after an even layer, so that every DoF's first toucher runs first)
void launch_apply_zrange(Op &op, double *dst, const double *src, int z0, int z1);
// bounds[0..S] of S z-slabs of nz cell layers (interior bounds odd); returns S,
// limited to nz / 2 and kMaxApplySlabs
int slab_bounds(int nz, int S, int *bounds);
// times the resident apply of `op` in one precision over the candidate
// schedules and keeps the fastest (mpdg_op_autotune)
void autotune_apply(Op &op, int precision, int reps, ApplySchedule &best, double &best_ms,
                    std::vector<double> *all_ms);
constexpr int kMaxLsqVectors = 32;
// returns the number of old solutions used (predictor.cu)
int predict_lsq(Op &op, int n_old, const double *const *old, const double *rhs, double *solution);
void launch_rhs(Op &op, double *dst, const double *src, const double *heat_source);
void launch_diagonal(Op &op, double *diag);
void launch_invert_diagonal(Op &op, double *diag);
// inversion with a given threshold (no reduction, no allocation)
void launch_invert_with_threshold(Op &op, double *diag, double thr);
// polls of a bounded device wait before it reports expiry (< 0: the default)
void set_wait_first_polls(long long polls);
// nullptr when an FP64 apply and the diagonal of `op` build nothing lazily (no
// device allocation); else why not
const char *noalloc_unready_reason(const Op &op);
double l2_norm_integrated(Op &op, const double *u);

// ---- vector kernels (vector_kernels.cu)
template <typename Real>
struct Reducer;  // deterministic two-pass reductions into FP64

double dot(const double *a, const double *b, long n, cudaStream_t s);
double dot_f(const float *a, const float *b, long n, cudaStream_t s);
double norm2(const double *a, long n, cudaStream_t s);
double linf(const double *a, long n, cudaStream_t s);

// ---- solvers (solvers.cu)
int solve(Op &op, const mpdg_solver_desc &desc, double *x, const double *b, mpdg_solve_report &rep);
void free_workspace(Op &op);
int solve_cg_noalloc(Op &op, double *x, const double *b, double rel_tol, double abs_tol, int max_it,
                     mpdg_solve_report &rep);

}  // namespace mpdg
