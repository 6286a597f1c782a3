// extern "C" entry points of libmpdg (declared in include/mpdg.h).  Every call
// converts internal errors into a status code; no exception crosses the ABI.
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
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
std::atomic<int64_t> g_allocations{0};
}  // namespace

void set_last_error(const std::string &msg) { g_last_error = msg; }
void count_launch(int n) { g_launches += n; }
void count_allocation() { ++g_allocations; }

}  // namespace mpdg

using namespace mpdg;

extern "C" {

const char *mpdg_last_error(void) { return g_last_error.c_str(); }
int mpdg_version(void) { return 1; }
int64_t mpdg_kernel_launches(void) { return g_launches.load(); }
int64_t mpdg_allocations(void) { return g_allocations.load(); }

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
    m.N_own = m.N;
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

mpdg_status mpdg_mesh_create_mapped(const mpdg_mapped_mesh_desc *desc, mpdg_mesh **out)
{
  return guarded([&]() -> int {
    if (!desc || !out || !desc->cell_vertices || !desc->cell_dofs) throw Error{MPDG_ERR_ARG, "null argument"};
    if (desc->degree < 1 || desc->degree > kMaxDegree) throw Error{MPDG_ERR_UNSUPPORTED, "degree must be 1..4"};
    if (desc->n_cells < 1 || desc->n_dofs < 1) throw Error{MPDG_ERR_ARG, "empty mesh"};
    if (desc->n_constraints < 0 ||
        (desc->n_constraints > 0 && (!desc->constrained_dofs || !desc->constraint_offsets ||
                                     !desc->constraint_masters || !desc->constraint_weights)))
      throw Error{MPDG_ERR_ARG, "constraint arrays missing"};
    auto *h = new mpdg_mesh();
    try {
      build_mapped_mesh(h->m, *desc);
    } catch (...) {
      mpdg_mesh_destroy(h);
      throw;
    }
    *out = h;
    return MPDG_OK;
  });
}

mpdg_status mpdg_mesh_create_two_level(const mpdg_mesh_desc *coarse, const mpdg_mesh_desc *fine, mpdg_mesh **out)
{
  return guarded([&]() -> int {
    if (!coarse || !fine || !out || !coarse->vertices || !fine->vertices) throw Error{MPDG_ERR_ARG, "null argument"};
    if (coarse->degree != fine->degree) throw Error{MPDG_ERR_ARG, "both blocks carry the same degree"};
    if (fine->nc[1] != 2 * coarse->nc[1] || fine->nc[2] != 2 * coarse->nc[2])
      throw Error{MPDG_ERR_ARG, "the fine block refines the coarse interface 2:1 in y and z"};
    // the fine block's interface plane hangs on the coarse faces: it is not part
    // of the fine block's Dirichlet set
    const long NXf = (long)fine->nc[0] * fine->degree + 1, NYf = (long)fine->nc[1] * fine->degree + 1,
               NZf = (long)fine->nc[2] * fine->degree + 1;
    std::vector<uint8_t> fmask;
    mpdg_mesh_desc fd = *fine;
    if (fine->dirichlet_mask) {
      fmask.assign(fine->dirichlet_mask, fine->dirichlet_mask + NXf * NYf * NZf);
      for (long r = 0; r < NYf * NZf; ++r) fmask[r * NXf] = 0;
      fd.dirichlet_mask = fmask.data();
    }
    mpdg_mesh *hc = nullptr, *hf = nullptr;
    int st = mpdg_mesh_create(coarse, &hc);
    if (st != MPDG_OK) return st;
    st = mpdg_mesh_create(&fd, &hf);
    if (st != MPDG_OK) {
      mpdg_mesh_destroy(hc);
      return st;
    }
    Mesh &m = hc->m;
    Mesh *f = new Mesh(std::move(hf->m));
    hf->m = Mesh{};
    delete hf;
    m.fine = f;
    try {
      // the fine interface vertices must lie on the coarse faces (bilinear face
      // map at the half points)
      const int c0 = coarse->nc[0], c1 = coarse->nc[1], c2 = coarse->nc[2];
      auto cv = [&](int vy, int vz, int a) {
        return m.vertices[(((long)vz * (c1 + 1) + vy) * (c0 + 1) + c0) * 3 + a];
      };
      double scale = 0.0;
      for (double v : m.vertices) scale = std::fmax(scale, std::fabs(v));
      for (int vz = 0; vz <= 2 * c2; ++vz)
        for (int vy = 0; vy <= 2 * c1; ++vy) {
          const int cy = std::min(vy / 2, c1 - 1), cz = std::min(vz / 2, c2 - 1);
          const double ty = 0.5 * (vy - 2 * cy), tz = 0.5 * (vz - 2 * cz);
          for (int a = 0; a < 3; ++a) {
            const double want = (1 - ty) * (1 - tz) * cv(cy, cz, a) + ty * (1 - tz) * cv(cy + 1, cz, a) +
                                (1 - ty) * tz * cv(cy, cz + 1, a) + ty * tz * cv(cy + 1, cz + 1, a);
            const double got = f->vertices[(((long)vz * (2 * c1 + 1) + vy) * (fine->nc[0] + 1)) * 3 + a];
            if (std::fabs(got - want) > 1e-12 * std::fmax(1.0, scale))
              throw Error{MPDG_ERR_ARG, "fine interface vertices do not lie on the coarse faces"};
          }
        }
      // whole-vector masks: Dirichlet (both blocks) or hanging, and hanging only
      const long Nc = m.N_own, Nf = f->N_own, N = Nc + Nf;
      std::vector<uint8_t> tdir(N, 0), thang(N, 0);
      if (coarse->dirichlet_mask)
        for (long i = 0; i < Nc; ++i) tdir[i] = coarse->dirichlet_mask[i] ? 1 : 0;
      if (fd.dirichlet_mask)
        for (long i = 0; i < Nf; ++i) tdir[Nc + i] = fd.dirichlet_mask[i] ? 1 : 0;
      for (long r = 0; r < NYf * NZf; ++r) tdir[Nc + r * NXf] = thang[Nc + r * NXf] = 1;
      MPDG_CUDA(tracked_malloc(&m.d_tmask_dir, N));
      MPDG_CUDA(tracked_malloc(&m.d_tmask_hang, N));
      MPDG_CUDA(cudaMemcpy(m.d_tmask_dir, tdir.data(), N, cudaMemcpyHostToDevice));
      MPDG_CUDA(cudaMemcpy(m.d_tmask_hang, thang.data(), N, cudaMemcpyHostToDevice));
      m.device_bytes += 2 * N + f->device_bytes;
      m.N = N;
    } catch (...) {
      mpdg_mesh_destroy(hc);
      throw;
    }
    *out = hc;
    return MPDG_OK;
  });
}

namespace {
void free_mesh_arrays(Mesh &m)
{
  for (void *p : {(void *)m.d_vert, (void *)m.d_metric64, (void *)m.d_metric32, (void *)m.d_dmask,
                  (void *)m.d_cell_flags, (void *)m.d_cell_mask, (void *)m.d_tmask_dir, (void *)m.d_tmask_hang,
                  (void *)m.d_cmap, (void *)m.d_cell_first, (void *)m.d_mface_cell, (void *)m.d_mface_f, (void *)m.d_mface_id, (void *)m.d_cell_fids, (void *)m.d_cellvert, (void *)m.d_cons_dof, (void *)m.d_cons_ptr,
                  (void *)m.d_cons_mast, (void *)m.d_cons_w, (void *)m.d_mast_dof, (void *)m.d_mast_ptr,
                  (void *)m.d_mast_cons, (void *)m.d_mast_w, (void *)m.d_cons_of, (void *)m.d_ccells})
    if (p) cudaFree(p);
}

}  // namespace

mpdg_status mpdg_mesh_destroy(mpdg_mesh *mesh)
{
  if (!mesh) return MPDG_OK;
  Mesh &m = mesh->m;
  free_mesh_arrays(m);
  if (m.fine) {
    free_mesh_arrays(*m.fine);
    delete m.fine;
  }
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
    if (desc->vel_kind < MPDG_VEL_NONE || desc->vel_kind > MPDG_VEL_NODAL) throw Error{MPDG_ERR_ARG, "unknown velocity kind"};
    Mesh &mm = mesh->m;
    if (mm.fine && (desc->k_alpha != 0.0 || desc->full_tangent || (desc->robin_faces && desc->robin_alpha != 0.0)))
      throw Error{MPDG_ERR_UNSUPPORTED,
                  "two-level meshes take constant coefficients: no k(T) law, full tangent or Robin faces"};
    if (desc->material < MPDG_MAT_LINEAR || desc->material > MPDG_MAT_GAS_LIQUID_SOLID)
      throw Error{MPDG_ERR_ARG, "unknown material law"};
    if (desc->material != MPDG_MAT_LINEAR && desc->kind != MPDG_OP_HEAT)
      throw Error{MPDG_ERR_ARG, "material laws apply to the heat operator"};
    if (law_has_solid(desc->material) && !desc->solid_liquid_sharp && !(desc->liquidus > desc->solidus))
      throw Error{MPDG_ERR_ARG, "the mushy zone needs liquidus > solidus"};
    if (!(desc->latent_heat >= 0.0)) throw Error{MPDG_ERR_ARG, "latent heat of fusion must be >= 0"};
    if (desc->apparent_capacity < MPDG_AC_POLY4_BELL || desc->apparent_capacity > MPDG_AC_QLQ)
      throw Error{MPDG_ERR_ARG, "unknown apparent capacity profile"};
    if (desc->latent_heat > 0.0 && law_has_solid(desc->material)) {
      // ApparentCapacity asserts liquidus > solidus (apparent_capacity.cpp:160-165) and
      // Material refuses it with the volume-specific capacity (material.templates.hpp:322-328)
      if (!(desc->liquidus > desc->solidus))
        throw Error{MPDG_ERR_ARG, "the apparent capacity needs liquidus > solidus"};
      if (desc->volume_specific)
        throw Error{MPDG_ERR_UNSUPPORTED, "the apparent capacity is not defined for the volume-specific heat capacity"};
    }
    if (mm.fine && (desc->material != MPDG_MAT_LINEAR || (desc->rad_faces && desc->rad_emissivity != 0.0)))
      throw Error{MPDG_ERR_UNSUPPORTED, "two-level meshes take constant coefficients: no material law or radiation"};
    if (desc->supg && desc->kind != MPDG_OP_ADVDIFF)
      throw Error{MPDG_ERR_ARG, "SUPG stabilisation applies to the advection-diffusion operator"};
    if (desc->supg && mm.fine) throw Error{MPDG_ERR_UNSUPPORTED, "SUPG on two-level meshes"};
    if (desc->vel_kind == MPDG_VEL_NODAL && mm.fine)
      throw Error{MPDG_ERR_UNSUPPORTED, "two-level meshes take no fields (velocity as a DoF vector)"};
    auto *h = new mpdg_op();
    Op &o = h->o;
    o.mesh = &mm;
    o.d = *desc;
    if (o.d.precision_mask == 0) o.d.precision_mask = 1 << MPDG_FP64;
    // CTA-wide cell groups measured faster for Q2 (both precisions) and Q4 in
    // FP64 on a B200 (128^3 Q2: 0.664 -> 0.638 ms FP64, 0.399 -> 0.390 ms FP32;
    // 64^3 Q4 FP64 0.490 -> 0.485 ms; Q4 FP32 0.294 -> 0.299 ms, kept on warps)
    o.sched[MPDG_FP64].cta = (mm.degree == 2 || mm.degree == 4) ? 1 : 0;
    o.sched[MPDG_FP32].cta = mm.degree == 2 ? 1 : 0;
    // the lane apply (uniform lattices, constant coefficients; other operators
    // keep the warp apply) measured faster for Q2 on a B200: 128^3 advection-
    // diffusion 0.664 -> 0.372 ms FP64, 0.431 -> 0.216 ms FP32; 64^3 heat
    // 0.092 -> 0.052 ms FP64.  Below ~20^3 cells the warp apply is a little
    // faster (16^3: 19.6 vs 20.5 us), so the default starts at 32^3 cells;
    // the autotuner decides case by case.
    const int lane_default = (mm.degree == 2 && mm.n_cells >= 32768) ? 1 : 0;
    o.sched[MPDG_FP64].lane = lane_default;
    o.sched[MPDG_FP32].lane = lane_default;
    try {
      build_op_device_data(o);
      if (mm.fine) {
        o.fine = new Op();
        Op &f = *o.fine;
        f.mesh = mm.fine;
        f.d = o.d;
        f.stream = o.stream;
        f.hang_NXc = mm.NX;
        f.hang_NYc = mm.NY;
        build_op_device_data(f);
        const int n = mm.degree + 1;
        const size_t bytes = sizeof(double) * (size_t)mm.fine->nc[1] * mm.fine->nc[2] * n * n;
        MPDG_CUDA(tracked_malloc(&f.d_stage, bytes));
        MPDG_CUDA(cudaMemset(f.d_stage, 0, bytes));
        f.device_bytes += bytes;
      }
    } catch (...) {
      mpdg_op_destroy(h);
      throw;
    }
    *out = h;
    return MPDG_OK;
  });
}

namespace {
void free_op_arrays(Op &o)
{
  free_workspace(o);
  for (void *p : {(void *)o.T_own, (void *)o.d_err, (void *)o.d_coef64, (void *)o.d_coef32, (void *)o.T32, (void *)o.Ts32,
                  (void *)o.d_velb64, (void *)o.d_velb32, (void *)o.d_trig32, (void *)o.d_trig64, o.d_stage,
                  (void *)o.d_tau64, (void *)o.d_tau32, (void *)o.d_lam64, (void *)o.d_lam32, (void *)o.Told_own, (void *)o.H_own, (void *)o.Told32,
                  (void *)o.H32, (void *)o.lsq_buf, (void *)o.host_stage,
                  (void *)o.d_io, o.io_tmp, (void *)o.U_own})
    if (p) cudaFree(p);
  if (o.pipe_in) {
    cudaStreamSynchronize(o.pipe_in);
    cudaStreamSynchronize(o.pipe_out);
    cudaStreamDestroy(o.pipe_in);
    cudaStreamDestroy(o.pipe_out);
    for (auto &e : o.pipe_ev)
      if (e) cudaEventDestroy(e);
    o.pipe_in = o.pipe_out = nullptr;
  }
}
}  // namespace

mpdg_status mpdg_op_destroy(mpdg_op *op)
{
  if (!op) return MPDG_OK;
  Op &o = op->o;
  free_op_arrays(o);
  if (o.fine) {
    free_op_arrays(*o.fine);
    delete o.fine;
  }
  delete op;
  return MPDG_OK;
}

mpdg_status mpdg_op_reset_time_increment(mpdg_op *op, double dt)
{
  if (!op || !(dt > 0.0)) return MPDG_ERR_ARG;
  if (op->o.d.dt != dt) invalidate_coef(op->o);
  op->o.d.dt = dt;
  if (op->o.fine) {
    if (op->o.fine->d.dt != dt) invalidate_coef(*op->o.fine);
    op->o.fine->d.dt = dt;
  }
  return MPDG_OK;
}

mpdg_status mpdg_op_use_dirichlet(mpdg_op *op, int use_dirichlet)
{
  if (!op) return MPDG_ERR_ARG;
  op->o.use_dirichlet = use_dirichlet != 0;
  if (op->o.fine) op->o.fine->use_dirichlet = use_dirichlet != 0;
  return MPDG_OK;
}

namespace {
// the device pointer slot and the operator-owned buffer of a field
void field_slots(Op &o, int field, const double **&slot, double **&own)
{
  switch (field) {
    case MPDG_FIELD_TEMPERATURE: slot = &o.T64; own = &o.T_own; return;
    case MPDG_FIELD_TEMPERATURE_OLD: slot = &o.Told64; own = &o.Told_own; return;
    case MPDG_FIELD_HEAVISIDE: slot = &o.H64; own = &o.H_own; return;
    case MPDG_FIELD_VELOCITY:
      if (o.d.vel_kind != MPDG_VEL_NODAL)
        throw Error{MPDG_ERR_ARG, "MPDG_FIELD_VELOCITY needs an operator created with vel_kind MPDG_VEL_NODAL"};
      slot = &o.U64;
      own = &o.U_own;
      return;
    default: throw Error{MPDG_ERR_ARG, "unknown field"};
  }
}

// values of a field: n_dofs, or 3 n_dofs for the velocity
size_t field_count(const Op &o, int field) { return (field == MPDG_FIELD_VELOCITY ? 3 : 1) * (size_t)o.mesh->N; }

// what setting a field rebuilds
void field_changed(Op &o, int field)
{
  if (field == MPDG_FIELD_VELOCITY) {
    build_nodal_velocity(o);
    return;
  }
  invalidate_coef(o);
  if (o.d.precision_mask & (1 << MPDG_FP32)) ensure_T32(o);
}
}  // namespace

mpdg_status mpdg_op_set_field(mpdg_op *op, int field, const double *values)
{
  return guarded([&]() -> int {
    if (!op) throw Error{MPDG_ERR_ARG, "null operator"};
    const double **slot = nullptr;
    double **own = nullptr;
    field_slots(op->o, field, slot, own);
    if (op->o.fine) throw Error{MPDG_ERR_UNSUPPORTED, "two-level meshes take no fields"};
    *slot = values;
    if (values || field != MPDG_FIELD_VELOCITY) field_changed(op->o, field);
    return MPDG_OK;
  });
}

mpdg_status mpdg_op_set_field_host(mpdg_op *op, int field, const double *values)
{
  return guarded([&]() -> int {
    if (!op || !values) throw Error{MPDG_ERR_ARG, "null argument"};
    Op &o = op->o;
    const double **slot = nullptr;
    double **own = nullptr;
    field_slots(o, field, slot, own);
    if (o.fine) throw Error{MPDG_ERR_UNSUPPORTED, "two-level meshes take no fields"};
    const size_t bytes = sizeof(double) * field_count(o, field);
    if (!*own) {
      MPDG_CUDA(tracked_malloc(own, bytes));
      o.device_bytes += bytes;
    }
    MPDG_CUDA(cudaMemcpyAsync(*own, values, bytes, cudaMemcpyHostToDevice, o.stream));
    MPDG_CUDA(cudaStreamSynchronize(o.stream));
    *slot = *own;
    field_changed(o, field);
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

mpdg_status mpdg_op_set_inflow_outflow(mpdg_op *op, const uint8_t *host_mask)
{
  return guarded([&]() -> int {
    if (!op) throw Error{MPDG_ERR_ARG, "null operator"};
    Op &o = op->o;
    if (o.d_io) {
      MPDG_CUDA(cudaStreamSynchronize(o.stream));
      cudaFree(o.d_io);
      o.d_io = nullptr;
    }
    if (!host_mask) return MPDG_OK;
    const long N = o.mesh->N;
    bool any = false;
    for (long i = 0; i < N && !any; ++i) any = host_mask[i] != 0;
    if (!any) return MPDG_OK;
    MPDG_CUDA(tracked_malloc(&o.d_io, N));
    MPDG_CUDA(cudaMemcpy(o.d_io, host_mask, N, cudaMemcpyHostToDevice));
    return MPDG_OK;
  });
}

mpdg_status mpdg_op_set_stream(mpdg_op *op, void *stream)
{
  if (!op) return MPDG_ERR_ARG;
  op->o.stream = (cudaStream_t)stream;
  if (op->o.fine) op->o.fine->stream = (cudaStream_t)stream;
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

mpdg_status mpdg_debug_set_wait_polls(int64_t polls)
{
  return guarded([&]() -> int {
    set_wait_first_polls((long long)polls);
    return MPDG_OK;
  });
}

mpdg_status mpdg_op_set_schedule(mpdg_op *op, int precision, const mpdg_schedule *sched)
{
  return guarded([&]() -> int {
    if (!op || !sched) throw Error{MPDG_ERR_ARG, "null argument"};
    if (precision != MPDG_FP64 && precision != MPDG_FP32) throw Error{MPDG_ERR_ARG, "precision"};
    if (sched->slabs < 1 || sched->slabs > kMaxApplySlabs) throw Error{MPDG_ERR_ARG, "slabs must be 1..32"};
    op->o.sched[precision].slabs = sched->slabs;
    op->o.sched[precision].evict_first = sched->l2_evict_first ? 1 : 0;
    op->o.sched[precision].pdl = sched->overlap_colours ? 1 : 0;
    op->o.sched[precision].cta = sched->cta_cell_groups ? 1 : 0;
    if (sched->lane_cells < 0 || sched->lane_cells > 2) throw Error{MPDG_ERR_ARG, "lane_cells must be 0, 1 or 2"};
    op->o.sched[precision].lane = sched->lane_cells;
    return MPDG_OK;
  });
}

mpdg_status mpdg_op_get_schedule(mpdg_op *op, int precision, mpdg_schedule *sched)
{
  return guarded([&]() -> int {
    if (!op || !sched) throw Error{MPDG_ERR_ARG, "null argument"};
    if (precision != MPDG_FP64 && precision != MPDG_FP32) throw Error{MPDG_ERR_ARG, "precision"};
    sched->slabs = op->o.sched[precision].slabs;
    sched->l2_evict_first = op->o.sched[precision].evict_first;
    sched->overlap_colours = op->o.sched[precision].pdl;
    sched->cta_cell_groups = op->o.sched[precision].cta;
    sched->lane_cells = op->o.sched[precision].lane;
    return MPDG_OK;
  });
}

mpdg_status mpdg_op_autotune(mpdg_op *op, int precision, int reps, mpdg_schedule *best, double *apply_ms,
                             double *candidate_ms, int n_candidate_ms)
{
  return guarded([&]() -> int {
    if (!op) throw Error{MPDG_ERR_ARG, "null argument"};
    if (precision != MPDG_FP64 && precision != MPDG_FP32) throw Error{MPDG_ERR_ARG, "precision"};
    Op &o = op->o;
    if (precision == MPDG_FP32 && o.T64 && !o.T32) ensure_T32(o);
    ApplySchedule b;
    double ms = 0.0;
    std::vector<double> all;
    autotune_apply(o, precision, reps, b, ms, &all);
    if (best) {
      best->slabs = b.slabs;
      best->l2_evict_first = b.evict_first;
      best->overlap_colours = b.pdl;
      best->cta_cell_groups = b.cta;
      best->lane_cells = b.lane;
    }
    if (apply_ms) *apply_ms = ms;
    if (candidate_ms)
      for (int i = 0; i < n_candidate_ms; ++i) candidate_ms[i] = i < (int)all.size() ? all[i] : -1.0;
    return MPDG_OK;
  });
}

mpdg_status mpdg_fma_peak(double *gflops64, double *gflops32)
{
  return guarded([&]() -> int {
    if (!gflops64 || !gflops32) throw Error{MPDG_ERR_ARG, "null argument"};
    fma_peak(*gflops64, *gflops32);
    return MPDG_OK;
  });
}

mpdg_status mpdg_vmult_multi(mpdg_op *op, int n_vectors, double *const *dst, const double *const *src)
{
  return guarded([&]() -> int {
    if (!op || !dst || !src || n_vectors < 1) throw Error{MPDG_ERR_ARG, "null argument or no vectors"};
    launch_apply_multi<double>(op->o, n_vectors, dst, src);
    return MPDG_OK;
  });
}

mpdg_status mpdg_vmult_multi_f32(mpdg_op *op, int n_vectors, float *const *dst, const float *const *src)
{
  return guarded([&]() -> int {
    if (!op || !dst || !src || n_vectors < 1) throw Error{MPDG_ERR_ARG, "null argument or no vectors"};
    Op &o = op->o;
    if (o.T64 && !o.T32) ensure_T32(o);
    launch_apply_multi<float>(o, n_vectors, dst, src);
    return MPDG_OK;
  });
}

mpdg_status mpdg_predict_lsq(mpdg_op *op, int n_old, const double *const *old_solutions, const double *rhs,
                             double *solution, int *n_used)
{
  return guarded([&]() -> int {
    if (!op || !old_solutions) throw Error{MPDG_ERR_ARG, "null argument"};
    const int used = predict_lsq(op->o, n_old, old_solutions, rhs, solution);
    if (n_used) *n_used = used;
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
    // device staging kept by the operator between calls: a vmult from host
    // buffers costs its two PCIe copies and the apply, no allocation
    if (!o.host_stage) {
      MPDG_CUDA(tracked_malloc(&o.host_stage, 2 * bytes));
      o.device_bytes += 2 * bytes;
    }
    double *d_src = o.host_stage, *d_dst = o.host_stage + o.mesh->N;
    const Mesh &m = *o.mesh;
    const int nz = m.nc[2], S = std::min(kPipeSlabs, nz / 2);
    if (!plain_warp_apply(o) || S < 2) {
      MPDG_CUDA(cudaMemcpyAsync(d_src, src_host, bytes, cudaMemcpyHostToDevice, o.stream));
      launch_apply<double>(o, d_dst, d_src);
      MPDG_CUDA(cudaMemcpyAsync(dst_host, d_dst, bytes, cudaMemcpyDeviceToHost, o.stream));
      MPDG_CUDA(cudaStreamSynchronize(o.stream));
      return MPDG_OK;
    }
    // z-slab pipeline: the copy-in of slab s+1, the apply of slab s and the
    // copy-out of slab s-1 overlap (the two copy directions run at once).  A
    // slab of cell layers [za, zb) reads the DoF planes [za P, zb P] and
    // completes the planes below zb P; interior slab ends zb are odd, so the
    // layer below every slab boundary is even and its cells store the shared
    // plane before the next slab's cells add to it (the first-touch rule)
    if (!o.pipe_in) {
      MPDG_CUDA(cudaStreamCreateWithFlags(&o.pipe_in, cudaStreamNonBlocking));
      MPDG_CUDA(cudaStreamCreateWithFlags(&o.pipe_out, cudaStreamNonBlocking));
      for (auto &e : o.pipe_ev) MPDG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    const long plane = m.NX * m.NY, P = m.degree, NZ = m.NZ;
    int bounds[kPipeSlabs + 1];
    bounds[0] = 0;
    for (int i = 1; i < S; ++i) {
      int b = (int)((long)i * nz / S) | 1;
      bounds[i] = std::min(std::max(b, bounds[i - 1] + 1), nz - 1);
    }
    bounds[S] = nz;
    for (int i = 1; i < S; ++i)
      if (bounds[i] % 2 == 0 || bounds[i] <= bounds[i - 1])
        throw Error{MPDG_ERR_ARG, "host apply pipeline: slab bounds"};
    // all copies in first: they depend on nothing, and the copy-in stream
    // then never waits for the host to enqueue the applies
    long in_next = 0, out_next = 0;  // first plane not yet copied in / out
    for (int sl = 0; sl < S; ++sl) {
      const long in_end = std::min(NZ, (long)bounds[sl + 1] * P + 1);
      if (in_end > in_next)
        MPDG_CUDA(cudaMemcpyAsync(d_src + in_next * plane, src_host + in_next * plane,
                                  sizeof(double) * (in_end - in_next) * plane, cudaMemcpyHostToDevice, o.pipe_in));
      in_next = std::max(in_next, in_end);
      MPDG_CUDA(cudaEventRecord(o.pipe_ev[2 * sl], o.pipe_in));
    }
    for (int sl = 0; sl < S; ++sl) {
      const int za = bounds[sl], zb = bounds[sl + 1];
      MPDG_CUDA(cudaStreamWaitEvent(o.stream, o.pipe_ev[2 * sl], 0));
      launch_apply_zrange(o, d_dst, d_src, za, zb);
      MPDG_CUDA(cudaEventRecord(o.pipe_ev[2 * sl + 1], o.stream));
      MPDG_CUDA(cudaStreamWaitEvent(o.pipe_out, o.pipe_ev[2 * sl + 1], 0));
      const long out_end = (zb == nz) ? NZ : (long)zb * P;
      if (out_end > out_next)
        MPDG_CUDA(cudaMemcpyAsync(dst_host + out_next * plane, d_dst + out_next * plane,
                                  sizeof(double) * (out_end - out_next) * plane, cudaMemcpyDeviceToHost, o.pipe_out));
      out_next = std::max(out_next, out_end);
    }
    MPDG_CUDA(cudaStreamSynchronize(o.pipe_out));
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
    MPDG_CUDA(tracked_malloc_async(&d, bytes, o.stream));
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
    // device copies of x and b, freed on every exit (a failed solve throws)
    struct Buffers {
      double *x = nullptr, *b = nullptr;
      cudaStream_t st = nullptr;
      ~Buffers()
      {
        if (st) cudaStreamSynchronize(st);
        if (x) cudaFree(x);
        if (b) cudaFree(b);
      }
    } d;
    d.st = o.stream;
    MPDG_CUDA(tracked_malloc(&d.x, bytes));
    MPDG_CUDA(tracked_malloc(&d.b, bytes));
    MPDG_CUDA(cudaMemcpyAsync(d.x, x_host, bytes, cudaMemcpyHostToDevice, o.stream));
    MPDG_CUDA(cudaMemcpyAsync(d.b, b_host, bytes, cudaMemcpyHostToDevice, o.stream));
    int s = solve(o, *desc, d.x, d.b, local);
    MPDG_CUDA(cudaMemcpyAsync(x_host, d.x, bytes, cudaMemcpyDeviceToHost, o.stream));
    MPDG_CUDA(cudaStreamSynchronize(o.stream));
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
