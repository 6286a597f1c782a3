// extern "C" entry points of libmpdg (declared in include/mpdg.h).  Every call
// converts internal errors into a status code; no exception crosses the ABI.
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "mpdg_internal.h"
#include "vector_kernels.cuh"

struct mpdg_mesh {
  mpdg::Mesh m;
};
struct mpdg_op {
  mpdg::Op o;
};

namespace mpdg {

namespace {
thread_local std::string g_last_error;
std::atomic<int64_t> g_launches{0};
}  // namespace

void set_last_error(const std::string &msg) { g_last_error = msg; }
void count_launch(int n) { g_launches += n; }

}  // namespace mpdg

using namespace mpdg;

extern "C" {

const char *mpdg_last_error(void) { return g_last_error.c_str(); }
int mpdg_version(void) { return 1; }
int64_t mpdg_kernel_launches(void) { return g_launches.load(); }

mpdg_status mpdg_mesh_create(const mpdg_mesh_desc *desc, mpdg_mesh **out)
{
  return guarded([&]() -> int {
    if (!desc || !out || !desc->vertices) throw Error{MPDG_ERR_ARG, "null argument"};
    if (desc->dim != 3) throw Error{MPDG_ERR_UNSUPPORTED, "the device path is three-dimensional"};
    if (desc->degree < 1 || desc->degree > kMaxDegree) throw Error{MPDG_ERR_UNSUPPORTED, "degree must be 1..4"};
    for (int d = 0; d < 3; ++d)
      if (desc->nc[d] < 1) throw Error{MPDG_ERR_ARG, "cell counts must be positive"};
    auto *h = new mpdg_mesh();
    Mesh &m = h->m;
    m.degree = desc->degree;
    m.n = desc->degree + 1;
    for (int d = 0; d < 3; ++d) m.nc[d] = desc->nc[d];
    m.NX = (long)m.nc[0] * m.degree + 1;
    m.NY = (long)m.nc[1] * m.degree + 1;
    m.NZ = (long)m.nc[2] * m.degree + 1;
    m.N = m.NX * m.NY * m.NZ;
    m.n_cells = (long)m.nc[0] * m.nc[1] * m.nc[2];
    const long nv = (long)(m.nc[0] + 1) * (m.nc[1] + 1) * (m.nc[2] + 1);
    m.vertices.assign(desc->vertices, desc->vertices + nv * 3);
    try {
      build_mesh_device_data(m, desc->dirichlet_mask, desc->geometry == MPDG_GEOM_GENERAL);
    } catch (...) {
      mpdg_mesh_destroy(h);
      throw;
    }
    *out = h;
    return MPDG_OK;
  });
}

mpdg_status mpdg_mesh_destroy(mpdg_mesh *mesh)
{
  if (!mesh) return MPDG_OK;
  Mesh &m = mesh->m;
  for (void *p : {(void *)m.d_vert, (void *)m.d_metric64, (void *)m.d_metric32, (void *)m.d_dmask,
                  (void *)m.d_cell_flags, (void *)m.d_cell_mask})
    if (p) cudaFree(p);
  delete mesh;
  return MPDG_OK;
}

mpdg_status mpdg_mesh_n_dofs(const mpdg_mesh *mesh, int64_t *n)
{
  if (!mesh || !n) return MPDG_ERR_ARG;
  *n = mesh->m.N;
  return MPDG_OK;
}

mpdg_status mpdg_mesh_device_bytes(const mpdg_mesh *mesh, int64_t *bytes)
{
  if (!mesh || !bytes) return MPDG_ERR_ARG;
  *bytes = (int64_t)mesh->m.device_bytes;
  return MPDG_OK;
}

mpdg_status mpdg_op_create(mpdg_mesh *mesh, const mpdg_op_desc *desc, mpdg_op **out)
{
  return guarded([&]() -> int {
    if (!mesh || !desc || !out) throw Error{MPDG_ERR_ARG, "null argument"};
    if (desc->kind != MPDG_OP_HEAT && desc->kind != MPDG_OP_ADVDIFF) throw Error{MPDG_ERR_ARG, "unknown operator kind"};
    if (!(desc->dt > 0.0)) throw Error{MPDG_ERR_ARG, "time increment must be positive"};
    if (desc->vel_kind < MPDG_VEL_NONE || desc->vel_kind > MPDG_VEL_CONST) throw Error{MPDG_ERR_ARG, "unknown velocity kind"};
    auto *h = new mpdg_op();
    Op &o = h->o;
    o.mesh = &mesh->m;
    o.d = *desc;
    if (o.d.precision_mask == 0) o.d.precision_mask = 1 << MPDG_FP64;
    try {
      build_op_device_data(o);
    } catch (...) {
      mpdg_op_destroy(h);
      throw;
    }
    *out = h;
    return MPDG_OK;
  });
}

mpdg_status mpdg_op_destroy(mpdg_op *op)
{
  if (!op) return MPDG_OK;
  Op &o = op->o;
  free_workspace(o);
  for (void *p : {(void *)o.T_own, (void *)o.d_err, (void *)o.d_coef64, (void *)o.d_coef32, (void *)o.T32, (void *)o.d_velb64, (void *)o.d_velb32, (void *)o.d_trig32,
                  (void *)o.d_trig64})
    if (p) cudaFree(p);
  delete op;
  return MPDG_OK;
}

mpdg_status mpdg_op_reset_time_increment(mpdg_op *op, double dt)
{
  if (!op || !(dt > 0.0)) return MPDG_ERR_ARG;
  if (op->o.d.dt != dt) invalidate_coef(op->o);
  op->o.d.dt = dt;
  return MPDG_OK;
}

mpdg_status mpdg_op_use_dirichlet(mpdg_op *op, int use_dirichlet)
{
  if (!op) return MPDG_ERR_ARG;
  op->o.use_dirichlet = use_dirichlet != 0;
  return MPDG_OK;
}

mpdg_status mpdg_op_set_field(mpdg_op *op, int field, const double *values)
{
  return guarded([&]() -> int {
    if (!op) throw Error{MPDG_ERR_ARG, "null operator"};
    if (field != MPDG_FIELD_TEMPERATURE) throw Error{MPDG_ERR_ARG, "unknown field"};
    op->o.T64 = values;
    invalidate_coef(op->o);
    if (values && (op->o.d.precision_mask & (1 << MPDG_FP32))) ensure_T32(op->o);
    return MPDG_OK;
  });
}

mpdg_status mpdg_op_set_field_host(mpdg_op *op, int field, const double *values)
{
  return guarded([&]() -> int {
    if (!op || !values) throw Error{MPDG_ERR_ARG, "null argument"};
    if (field != MPDG_FIELD_TEMPERATURE) throw Error{MPDG_ERR_ARG, "unknown field"};
    Op &o = op->o;
    const size_t bytes = sizeof(double) * o.mesh->N;
    if (!o.T_own) {
      MPDG_CUDA(cudaMalloc(&o.T_own, bytes));
      o.device_bytes += bytes;
    }
    MPDG_CUDA(cudaMemcpyAsync(o.T_own, values, bytes, cudaMemcpyHostToDevice, o.stream));
    MPDG_CUDA(cudaStreamSynchronize(o.stream));
    o.T64 = o.T_own;
    invalidate_coef(o);
    if (o.d.precision_mask & (1 << MPDG_FP32)) ensure_T32(o);
    return MPDG_OK;
  });
}

mpdg_status mpdg_op_device_error(mpdg_op *op, int *flag)
{
  return guarded([&]() -> int {
    if (!op || !flag) throw Error{MPDG_ERR_ARG, "null argument"};
    MPDG_CUDA(cudaStreamSynchronize(op->o.stream));
    MPDG_CUDA(cudaMemcpy(flag, op->o.d_err, sizeof(int), cudaMemcpyDeviceToHost));
    MPDG_CUDA(cudaMemset(op->o.d_err, 0, sizeof(int)));
    return MPDG_OK;
  });
}

mpdg_status mpdg_op_set_stream(mpdg_op *op, void *stream)
{
  if (!op) return MPDG_ERR_ARG;
  op->o.stream = (cudaStream_t)stream;
  return MPDG_OK;
}

mpdg_status mpdg_vmult(mpdg_op *op, double *dst, const double *src)
{
  return guarded([&]() -> int {
    if (!op || !dst || !src) throw Error{MPDG_ERR_ARG, "null argument"};
    launch_apply<double>(op->o, dst, src);
    return MPDG_OK;
  });
}

mpdg_status mpdg_vmult_f32(mpdg_op *op, float *dst, const float *src)
{
  return guarded([&]() -> int {
    if (!op || !dst || !src) throw Error{MPDG_ERR_ARG, "null argument"};
    Op &o = op->o;
    if (o.T64 && !o.T32) ensure_T32(o);
    launch_apply<float>(o, dst, src);
    return MPDG_OK;
  });
}

mpdg_status mpdg_vmult_host(mpdg_op *op, double *dst_host, const double *src_host)
{
  return guarded([&]() -> int {
    if (!op || !dst_host || !src_host) throw Error{MPDG_ERR_ARG, "null argument"};
    Op &o = op->o;
    const size_t bytes = sizeof(double) * o.mesh->N;
    double *d_src = nullptr, *d_dst = nullptr;
    MPDG_CUDA(cudaMallocAsync(&d_src, bytes, o.stream));
    MPDG_CUDA(cudaMallocAsync(&d_dst, bytes, o.stream));
    MPDG_CUDA(cudaMemcpyAsync(d_src, src_host, bytes, cudaMemcpyHostToDevice, o.stream));
    launch_apply<double>(o, d_dst, d_src);
    MPDG_CUDA(cudaMemcpyAsync(dst_host, d_dst, bytes, cudaMemcpyDeviceToHost, o.stream));
    MPDG_CUDA(cudaFreeAsync(d_src, o.stream));
    MPDG_CUDA(cudaFreeAsync(d_dst, o.stream));
    MPDG_CUDA(cudaStreamSynchronize(o.stream));
    return MPDG_OK;
  });
}

mpdg_status mpdg_compute_diagonal(mpdg_op *op, double *diag)
{
  return guarded([&]() -> int {
    if (!op || !diag) throw Error{MPDG_ERR_ARG, "null argument"};
    launch_diagonal(op->o, diag);
    return MPDG_OK;
  });
}

mpdg_status mpdg_compute_inverse_diagonal(mpdg_op *op, double *inv_diag)
{
  return guarded([&]() -> int {
    if (!op || !inv_diag) throw Error{MPDG_ERR_ARG, "null argument"};
    launch_diagonal(op->o, inv_diag);
    launch_invert_diagonal(op->o, inv_diag);
    return MPDG_OK;
  });
}

namespace {
// device staging of host vectors for the *_host entry points
struct HostStage {
  explicit HostStage(Op &o) : o(o) {}
  double *up(const double *h)
  {
    if (!h) return nullptr;
    double *d = nullptr;
    const size_t bytes = sizeof(double) * o.mesh->N;
    MPDG_CUDA(cudaMallocAsync(&d, bytes, o.stream));
    bufs.push_back(d);
    MPDG_CUDA(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, o.stream));
    return d;
  }
  void down(double *h, const double *d)
  {
    MPDG_CUDA(cudaMemcpyAsync(h, d, sizeof(double) * o.mesh->N, cudaMemcpyDeviceToHost, o.stream));
  }
  ~HostStage()
  {
    for (double *d : bufs) cudaFreeAsync(d, o.stream);
    cudaStreamSynchronize(o.stream);
  }
  Op &o;
  std::vector<double *> bufs;
};
}  // namespace

mpdg_status mpdg_compute_inverse_diagonal_host(mpdg_op *op, double *inv_diag_host)
{
  return guarded([&]() -> int {
    if (!op || !inv_diag_host) throw Error{MPDG_ERR_ARG, "null argument"};
    HostStage st(op->o);
    double *d = st.up(inv_diag_host);
    launch_diagonal(op->o, d);
    launch_invert_diagonal(op->o, d);
    st.down(inv_diag_host, d);
    return MPDG_OK;
  });
}

mpdg_status mpdg_create_rhs_host(mpdg_op *op, double *dst_host, const double *src_host,
                                 const double *heat_source_host)
{
  return guarded([&]() -> int {
    if (!op || !dst_host || !src_host) throw Error{MPDG_ERR_ARG, "null argument"};
    HostStage st(op->o);
    double *d = st.up(dst_host);
    const double *s = st.up(src_host);
    const double *q = st.up(heat_source_host);
    launch_rhs(op->o, d, s, q);
    st.down(dst_host, d);
    return MPDG_OK;
  });
}

mpdg_status mpdg_create_rhs(mpdg_op *op, double *dst, const double *src, const double *heat_source)
{
  return guarded([&]() -> int {
    if (!op || !dst || !src) throw Error{MPDG_ERR_ARG, "null argument"};
    launch_rhs(op->o, dst, src, heat_source);
    return MPDG_OK;
  });
}

void mpdg_solver_desc_default(mpdg_solver_desc *d)
{
  if (!d) return;
  std::memset(d, 0, sizeof(*d));
  d->solver = MPDG_SOLVER_GMRES;            // LinearSolverData defaults, linear_solver_data.hpp:38-51
  d->preconditioner = MPDG_PREC_JACOBI;     // "Diagonal" in heat_data.cpp:11-12
  d->max_iterations = 10000;
  d->rel_tolerance = 1e-12;
  d->abs_tolerance = 1e-20;
  d->gmres_restart = 30;
  d->chebyshev_degree = 5;
  d->lanczos_steps = 10;
  d->chebyshev_range = 30.0;
  d->chebyshev_safety = 1.2;
  d->mixed_precision = 0;
  d->inner_tolerance = 3e-6;  // two defect-correction steps reach 1e-10
  d->max_outer = 20;
  d->reliable_delta = 0.1;
}

mpdg_status mpdg_solve(mpdg_op *op, const mpdg_solver_desc *desc, double *x, const double *b,
                       mpdg_solve_report *report)
{
  mpdg_solve_report local{};
  int st = guarded([&]() -> int {
    if (!op || !desc || !x || !b) throw Error{MPDG_ERR_ARG, "null argument"};
    return solve(op->o, *desc, x, b, local);
  });
  local.status = st;
  if (report) *report = local;
  return st;
}

mpdg_status mpdg_solve_host(mpdg_op *op, const mpdg_solver_desc *desc, double *x_host,
                            const double *b_host, mpdg_solve_report *report)
{
  mpdg_solve_report local{};
  int st = guarded([&]() -> int {
    if (!op || !desc || !x_host || !b_host) throw Error{MPDG_ERR_ARG, "null argument"};
    Op &o = op->o;
    const size_t bytes = sizeof(double) * o.mesh->N;
    double *d_x = nullptr, *d_b = nullptr;
    MPDG_CUDA(cudaMalloc(&d_x, bytes));
    MPDG_CUDA(cudaMalloc(&d_b, bytes));
    MPDG_CUDA(cudaMemcpyAsync(d_x, x_host, bytes, cudaMemcpyHostToDevice, o.stream));
    MPDG_CUDA(cudaMemcpyAsync(d_b, b_host, bytes, cudaMemcpyHostToDevice, o.stream));
    int s = solve(o, *desc, d_x, d_b, local);
    MPDG_CUDA(cudaMemcpyAsync(x_host, d_x, bytes, cudaMemcpyDeviceToHost, o.stream));
    MPDG_CUDA(cudaStreamSynchronize(o.stream));
    cudaFree(d_x);
    cudaFree(d_b);
    return s;
  });
  local.status = st;
  if (report) *report = local;
  return st;
}

mpdg_status mpdg_solve_cg_noalloc(mpdg_op *op, double *x, const double *b, double rel_tolerance,
                                  double abs_tolerance, int max_iterations,
                                  mpdg_solve_report *report)
{
  mpdg_solve_report local{};
  int st = guarded([&]() -> int {
    if (!op || !x || !b) throw Error{MPDG_ERR_ARG, "null argument"};
    if (max_iterations < 1) throw Error{MPDG_ERR_ARG, "max_iterations must be positive"};
    return solve_cg_noalloc(op->o, x, b, rel_tolerance, abs_tolerance, max_iterations, local);
  });
  local.status = st;
  if (report) *report = local;
  return st;
}

mpdg_status mpdg_l2_norm(mpdg_op *op, const double *u, double *norm)
{
  return guarded([&]() -> int {
    if (!op || !u || !norm) throw Error{MPDG_ERR_ARG, "null argument"};
    *norm = l2_norm_integrated(op->o, u);
    return MPDG_OK;
  });
}

}  // extern "C"
