/*
 * mpdg.h -- C ABI of the B200 matrix-free heat / advection-diffusion operator
 * library (libmpdg.so, CUDA sm_100a).
 *
 * Every entry point returns an int status (MPDG_OK = 0, negative = error) and
 * never throws.  Vectors passed to the apply/solve calls are DEVICE pointers
 * (unless the name says _host), laid out in the library's lexicographic DoF
 * numbering (x fastest):
 *     g = (Z * NY + Y) * NX + X,   X = ix * degree + i  in [0, nc[0] * degree]
 * Constrained (Dirichlet) DoFs are read as zero by the operator apply and are
 * never written by it, as in MeltPoolDG's MatrixFree cell loops.
 *
 * Each entry point names the MeltPoolDG interface it replaces.  Calls on one
 * operator must be serialised by the caller; they are queued on the
 * operator's stream (set with mpdg_op_set_stream, default: the legacy stream).
 */
#ifndef MPDG_H
#define MPDG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int mpdg_status;
enum {
  MPDG_OK = 0,
  MPDG_ERR_ARG = -1,            /* invalid argument */
  MPDG_ERR_CUDA = -2,           /* CUDA runtime error (see mpdg_last_error) */
  MPDG_ERR_ALLOC = -3,          /* device allocation failed */
  MPDG_ERR_NOT_CONVERGED = -4,  /* iteration limit reached (SolverControl::NoConvergence) */
  MPDG_ERR_BREAKDOWN = -5,      /* CG breakdown: p.Ap <= 0 or rz <= 0 */
  MPDG_ERR_NAN = -6,            /* non-finite residual */
  MPDG_ERR_UNSUPPORTED = -7,    /* configuration not implemented on the device */
  MPDG_ERR_BUDGET = -8,         /* request exceeds the memory budget (serving) */
  MPDG_ERR_SIZE = -9            /* problem larger than a fixed capacity */
};

enum { MPDG_OP_HEAT = 0, MPDG_OP_ADVDIFF = 1 };
enum { MPDG_FP64 = 0, MPDG_FP32 = 1 };
enum {
  MPDG_VEL_NONE = 0,
  MPDG_VEL_ROTATION = 1, /* u = s (z, 0, -x): advection_diffusion_vortex.hpp:93-115 (dim 3) */
  MPDG_VEL_VORTEX = 2,   /* u = (sin pi x cos pi y, -cos pi x sin pi y, 0) */
  MPDG_VEL_CONST = 3,    /* u = vel_param */
  /* u given as a DoF vector (MPDG_FIELD_VELOCITY): the velocity field the
   * reference operators read with read_dof_values_plain
   * (heat_diffuse_operator.cpp:975-980, advection_diffusion_operator.cpp:461-465) */
  MPDG_VEL_NODAL = 4
};
enum { MPDG_GEOM_AUTO = 0, MPDG_GEOM_GENERAL = 1 };
enum { MPDG_SOLVER_CG = 0, MPDG_SOLVER_GMRES = 1 };
enum { MPDG_PREC_IDENTITY = 0, MPDG_PREC_JACOBI = 1, MPDG_PREC_CHEBYSHEV = 2 };
/* MPDG_FIELD_VELOCITY: 3 n_dofs values, component-major (u_x of every DoF,
 * then u_y, then u_z), for operators with vel_kind MPDG_VEL_NODAL */
enum { MPDG_FIELD_TEMPERATURE = 0, MPDG_FIELD_TEMPERATURE_OLD = 1, MPDG_FIELD_HEAVISIDE = 2,
       MPDG_FIELD_VELOCITY = 3 };
/* heat material laws (MaterialTypes; Material::compute_parameters_internal,
 * include/meltpooldg/core/material.templates.hpp:213-760).  LINEAR: rho_cp and
 * k(T) = k0 (1 + k_alpha T).  The phase laws interpolate the gas / liquid / solid
 * properties by the level-set heaviside H (MPDG_FIELD_HEAVISIDE; weight H, or
 * H > 0.5 when two_phase_sharp) and the solid fraction
 * f_s = clamp((liquidus - T) / (liquidus - solidus), 0, 1) (or T < solidus when
 * solid_liquid_sharp) with the cubic 3 f_s^2 - 2 f_s^3; rho c_p = rho * c_p, or
 * the interpolated rho*c_p when volume_specific.  Laws with a solid phase add
 * the Newton terms d(rho c_p)/dT ((T - T_old)/dt + u.grad T) du and
 * dk/dT grad T du (heat_diffuse_operator.cpp:1040-1062) and read
 * MPDG_FIELD_TEMPERATURE_OLD.  Latent heat (apparent capacity) is not offered. */
enum { MPDG_MAT_LINEAR = 0, MPDG_MAT_GAS_LIQUID = 1, MPDG_MAT_LIQUID_SOLID = 2, MPDG_MAT_GAS_LIQUID_SOLID = 3 };
/* apparent heat capacity profiles of the latent heat of fusion
 * (ApparentCapacityType, include/meltpooldg/core/material_data.hpp:43-113) */
enum { MPDG_AC_POLY4_BELL = 0, MPDG_AC_CONSTANT = 1, MPDG_AC_QLQ = 2 };

typedef struct mpdg_mesh mpdg_mesh;
typedef struct mpdg_op mpdg_op;

/* Structured hexahedral mesh of nc[0] x nc[1] x nc[2] trilinear cells carrying
 * FE_Q(degree) on Gauss-Lobatto points with QGauss(degree+1) quadrature
 * (source/utilities/fe_util.cpp:18-57). */
typedef struct {
  int dim;                         /* must be 3 */
  int degree;                      /* 1..4 */
  int nc[3];
  const double *vertices;          /* host, (nc0+1)(nc1+1)(nc2+1) x 3, x fastest */
  const uint8_t *dirichlet_mask;   /* host, n_dofs entries (1 = constrained) or NULL */
  int geometry;                    /* MPDG_GEOM_AUTO: uniform boxes skip the metric stream */
} mpdg_mesh_desc;

/* Operator parameters (names follow MeltPoolDG's HeatData / AdvectionDiffusionData). */
typedef struct {
  int kind;                 /* MPDG_OP_HEAT or MPDG_OP_ADVDIFF */
  double dt;                /* time increment (OperatorBase::reset_time_increment) */
  /* heat: v = rho_cp/dt u + rho_cp vel.grad u, g = k(T) grad u, k(T) = k0 (1 + k_alpha T) */
  double rho_cp, k0, k_alpha;
  int full_tangent;         /* add dk/dT grad(T) u to the flux (non-symmetric tangent) */
  /* advection-diffusion: v = u/dt + theta vel.grad u, g = theta D grad u */
  double theta, diffusivity;
  int vel_kind;
  double vel_param[3];
  int precision_mask;       /* bit MPDG_FP64 / bit MPDG_FP32: forms to prepare (0 = FP64) */
  /* heat: convective (Robin) faces, heat_diffuse_operator.cpp:1088-1129: tangent alpha u v,
   * residual -alpha (T - t_inf) v on the box faces with bit 2*direction + side set
   * (side 0: the low face, 1: the high face); 0 = none */
  double robin_alpha, robin_t_inf;
  int robin_faces;
  /* advection-diffusion: SUPG stabilisation (AdvectionDiffusionData::conv_stab,
   * advection_diffusion_operator.cpp:276-358, 450-533): the flux gains
   * tau_K u (u/dt + theta u.grad u - theta D lap u) (right-hand side:
   * tau_K u (phi/dt - (1-theta) u.grad phi + (1-theta) D lap phi)), with
   * tau_K = supg_coefficient h_K, or h_K / max_q |u| when supg_coefficient < 0,
   * h_K = cell diameter / sqrt(3).  lap u is the physical Laplacian on every
   * cell shape, the trilinear map's curvature included (get_laplacian,
   * advection_diffusion_operator.cpp:483-486).  The diagonal is built by
   * probing (n^3 applies). */
  int supg;
  double supg_coefficient;
  /* heat: radiative faces (heat_diffuse_operator.cpp:766-772, 1122-1124): tangent
   * 4 eps sigma T^3 u v, residual -eps sigma (T^4 - rad_t_inf^4) v on the faces
   * flagged as in robin_faces; sigma = 5.670374419e-8 */
  double rad_emissivity, rad_t_inf;
  int rad_faces;
  /* heat: material law (MPDG_MAT_*); phase properties indexed gas, liquid, solid */
  int material;
  double mat_rho[3], mat_cp[3], mat_k[3];
  double solidus, liquidus;
  int two_phase_sharp, solid_liquid_sharp, volume_specific;
  /* heat, laws with a solid phase: latent heat of fusion (> 0 adds the
   * apparent capacity of profile MPDG_AC_* to c_p in the mushy zone, and its
   * T derivative to the Newton terms: Material, material.templates.hpp:566-616;
   * ApparentCapacity, source/heat/apparent_capacity.cpp).  Not defined with
   * volume_specific, as in the reference. */
  double latent_heat;
  int apparent_capacity;
} mpdg_op_desc;

typedef struct {
  int solver;               /* MPDG_SOLVER_CG or MPDG_SOLVER_GMRES (right preconditioned) */
  int preconditioner;       /* MPDG_PREC_* */
  int max_iterations;       /* LinearSolverData::max_iterations */
  double rel_tolerance;     /* LinearSolverData::rel_tolerance */
  double abs_tolerance;     /* LinearSolverData::abs_tolerance */
  int gmres_restart;        /* Krylov basis size, default 30 */
  int chebyshev_degree;     /* residual polynomial degree (degree-1 applies), default 5 */
  int lanczos_steps;        /* eigenvalue estimate steps, default 10 */
  double chebyshev_range;   /* lambda_min = lambda_max / range, default 30 */
  double chebyshev_safety;  /* lambda_max scaled by this, default 1.2 */
  int mixed_precision;      /* 1: FP32 operator/preconditioner, FP64 defects, dots and update */
  double inner_tolerance;   /* GMRES: relative reduction of each inner FP32 solve, default 3e-6 */
  int max_outer;            /* GMRES: defect-correction steps, default 20 */
  double reliable_delta;    /* CG: FP64 defect whenever the FP32 residual fell by this, default 0.1 */
} mpdg_solver_desc;

typedef struct {
  int status;               /* MPDG_OK or an error code */
  int iterations;           /* Krylov iterations (sum of inner ones when mixed) */
  int outer_iterations;     /* mixed: FP64 defect evaluations (CG) / correction steps (GMRES) */
  int operator_applies;     /* all operator applies, any precision */
  double initial_residual;  /* |b - A x0|_2 */
  double final_residual;    /* |b - A x|_2 in FP64 */
  double lambda_max;        /* Chebyshev estimate (0 if unused) */
  double seconds;           /* wall time of the solve */
} mpdg_solve_report;

/* ------------------------------------------------------------------ general */
const char *mpdg_last_error(void);
int mpdg_version(void);

/* ------------------------------------------------------------------ meshes */
/* replaces ScratchData::build / MatrixFree::reinit: source/core/scratch_data.cpp:191-268 */
mpdg_status mpdg_mesh_create(const mpdg_mesh_desc *desc, mpdg_mesh **mesh);
/* Two-level mesh with hanging nodes: a coarse block and a fine block that
 * refines it 2:1 in y and z (fine->nc[1] = 2 coarse->nc[1], fine->nc[2] =
 * 2 coarse->nc[2]), meeting at the coarse block's x = max face, on which the
 * fine block's x = min face lies (its interface vertices on the coarse faces'
 * bilinear maps at the half points).  The fine DoFs on that plane hang on the
 * coarse faces: their values are the coarse faces' interpolants, as deal.II's
 * hanging-node constraints on a 2:1 refined face (read_dof_values /
 * distribute_local_to_global with constraints, matrix_free cell loops of
 * heat_diffuse_operator.cpp:199-241).  Vectors hold the coarse block's DoFs,
 * then the fine block's (both lexicographic); the hanging DoFs are constrained
 * like Dirichlet DoFs (read through the interpolation, output 0, diagonal 1).
 * Operators on it take constant coefficients (no k(T), Robin faces or full
 * tangent) and support vmult, the diagonal and the solvers. */
mpdg_status mpdg_mesh_create_two_level(const mpdg_mesh_desc *coarse, const mpdg_mesh_desc *fine,
                                       mpdg_mesh **mesh);
/* Mapped mesh: the ingestion form of an unstructured hexahedral mesh, as a
 * deal.II host holds it (DoFHandler cell->DoF maps, AffineConstraints;
 * utilities/amr.hpp:55, utilities/constraints.hpp:117-135).  Each cell gives its
 * 8 corners (trilinear map, corner v = x-bit + 2 y-bit + 4 z-bit) and its
 * (degree+1)^3 global DoFs, lexicographic within the cell (x fastest).  The
 * homogeneous affine constraints (hanging nodes) read
 * x[constrained_dofs[c]] = sum_{e in [offsets[c], offsets[c+1])} weights[e] x[masters[e]],
 * masters unconstrained.  The operator is sum_K C_K^T A_K C_K as the reference's
 * cell loops with constraints form it: constrained DoFs are read through their
 * constraint, written to their masters and stay 0; diagonal 1 there.  Cells are
 * coloured greedily (no two cells of a colour share a DoF; at most 64 colours),
 * so the scatter is atomic-free and deterministic.  Operators on it: the heat
 * operator (k(T), the phase laws and the full tangent; fields read plain) and the
 * advection-diffusion operator (prescribed velocity or a velocity vector,
 * SUPG, inflow/outflow rows), convective and radiative faces selected by the
 * cells' face_ids; vmult, the diagonal,
 * create_rhs, the solvers and the integrated L2 norm. */
typedef struct {
  int degree;                        /* 1..4 */
  int64_t n_cells, n_dofs;
  const double *cell_vertices;       /* host, n_cells x 8 x 3 */
  const int64_t *cell_dofs;          /* host, n_cells x (degree+1)^3 */
  const uint8_t *dirichlet_mask;     /* host, n_dofs entries (1 = constrained) or NULL */
  int64_t n_constraints;
  const int64_t *constrained_dofs;   /* n_constraints */
  const int64_t *constraint_offsets; /* n_constraints + 1 */
  const int64_t *constraint_masters;
  const double *constraint_weights;
  /* host, n_cells x 6 or NULL: boundary id of each cell's local face 2 d + s
   * (-1 interior; 0..5 selects the face by bit id of mpdg_op_desc.robin_faces
   * and rad_faces, as the box faces of a lattice do) */
  const int8_t *face_ids;
} mpdg_mapped_mesh_desc;
mpdg_status mpdg_mesh_create_mapped(const mpdg_mapped_mesh_desc *desc, mpdg_mesh **mesh);
mpdg_status mpdg_mesh_destroy(mpdg_mesh *mesh);
/* n_dofs of the mesh (ScratchData::get_dof_handler(idx).n_dofs()) */
mpdg_status mpdg_mesh_n_dofs(const mpdg_mesh *mesh, int64_t *n_dofs);
/* device bytes held by the mesh (geometry stream, masks) */
mpdg_status mpdg_mesh_device_bytes(const mpdg_mesh *mesh, int64_t *bytes);

/* ---------------------------------------------------------------- operators */
/* replaces the constructors of HeatDiffuseMultiPhaseOperator
 * (include/meltpooldg/heat/heat_diffuse_operator.hpp:110) and
 * AdvectionDiffusionOperator (source/level_set/advection_diffusion_operator.cpp:17-41) */
mpdg_status mpdg_op_create(mpdg_mesh *mesh, const mpdg_op_desc *desc, mpdg_op **op);
mpdg_status mpdg_op_destroy(mpdg_op *op);
/* OperatorBase::reset_time_increment, include/meltpooldg/core/operator_base.hpp:41-46 */
mpdg_status mpdg_op_reset_time_increment(mpdg_op *op, double dt);
/* OperatorBase::reset_dof_index, operator_base.hpp:31-35: use_dirichlet = 0 selects
 * the constraint set without Dirichlet rows (used for the lifting of
 * include/meltpooldg/linear_algebra/utilities_matrixfree.hpp:39-101) */
mpdg_status mpdg_op_use_dirichlet(mpdg_op *op, int use_dirichlet);
/* state vectors the operator reads (temperature for k(T) and the Newton residual);
 * device pointer, FP64, n_dofs; an FP32 copy is made for the FP32 form.  The
 * operator folds k(T) into its per-quadrature-point coefficients when this is
 * called: a caller that changes the field's values in place calls it again
 * before the next vmult (the reference re-reads T in every vmult,
 * heat_diffuse_operator.cpp:1000-1012).  MPDG_FIELD_VELOCITY (3 n_dofs values)
 * is interpolated to the quadrature points when set, into the stream
 * JxW J^-1 u the apply reads (and tau_K with SUPG); the same rule applies. */
mpdg_status mpdg_op_set_field(mpdg_op *op, int field, const double *device_values);
/* the same with host values, copied into operator-owned device memory */
mpdg_status mpdg_op_set_field_host(mpdg_op *op, int field, const double *host_values);
mpdg_status mpdg_op_set_stream(mpdg_op *op, void *cuda_stream);
/* inflow/outflow constraints of the advection-diffusion operator
 * (AdvectionDiffusionOperator::set_inflow_outflow_bc / do_pre_vmult /
 * do_post_vmult, advection_diffusion_operator.cpp:537-578): identity rows at
 * the flagged DoFs (host mask, n_dofs bytes; NULL clears).  vmult reads src as
 * 0 there and returns src there; the inverse diagonal is 1 there
 * (:438-445).  src is not modified (the reference zeroes it in place). */
mpdg_status mpdg_op_set_inflow_outflow(mpdg_op *op, const uint8_t *host_mask);
/* reads and clears the operator's device error word: nonzero when a bounded
 * device-side wait (bulk-copy completion) expired; synchronises the stream */
mpdg_status mpdg_op_device_error(mpdg_op *op, int *flag);
/* test hook: the number of polls after which a bounded device wait of the
 * apply reports expiry on the current device (polls < 0 restores the default,
 * 2^26).  An expired wait sets the operator's error word and then waits for
 * its copy with the full limit, so results are unchanged.  No reference
 * counterpart (the reference has no device code). */
mpdg_status mpdg_debug_set_wait_polls(int64_t polls);

/* OperatorMatrixFree::vmult, operator_base.hpp:239-243
 * (heat: source/heat/heat_diffuse_operator.cpp:179-197;
 *  advection-diffusion: source/level_set/advection_diffusion_operator.cpp:238-272) */
mpdg_status mpdg_vmult(mpdg_op *op, double *dst, const double *src);
/* the same operator applied in FP32 (operator data and vectors in FP32) */
mpdg_status mpdg_vmult_f32(mpdg_op *op, float *dst, const float *src);
/* dst[v] = A src[v] for n_vectors device vectors (host arrays of device
 * pointers; no destination may overlap any vector).  Operators whose apply is
 * the plain cell kernel (no boundary faces, inflow rows, hanging nodes, SUPG or
 * phase law) read each cell's coefficients once per pass of up to 4 vectors;
 * the others apply the vectors in turn.  Replaces the n vmult calls of
 * LeastSquaresProjection::vmult (include/meltpooldg/linear_algebra/predictor.hpp:37-46). */
mpdg_status mpdg_vmult_multi(mpdg_op *op, int n_vectors, double *const *dst, const double *const *src);
/* Schedule of the resident apply, per precision.  slabs > 1 runs the colour
 * launches z-slab by z-slab (cell layers split into `slabs` runs with odd
 * interior ends, each running its 8 colours before the next), so that a slab's
 * DoF vectors stay in L2 across its colours; l2_evict_first marks the streamed
 * per-quadrature-point coefficients evict-first in L2; overlap_colours launches
 * every colour after an apply's first as a programmatic dependent of the one
 * before, so that its start (coefficient copies, src gathers, the first cells'
 * arithmetic) overlaps the previous colour's last cells and only its reads of
 * dst wait for it; cta_cell_groups lets the four warps of a CTA share their
 * cells (5 Q4 cells or 14 Q2 cells per 128 threads instead of 4 or 12, so
 * fewer lanes idle; the tile exchanges become CTA barriers), for degrees 2
 * and 4 on lattice meshes.  lane_cells (uniform lattices of degree 1 or 2,
 * constant coefficients, one operand, velocities other than MPDG_VEL_NODAL)
 * gives every cell one thread that keeps its whole sum factorisation in
 * registers; 32 lanes own a row segment of cells and add their shared x-faces
 * by warp shuffles, so these launches colour by segment parity in x.  Results
 * are identical for every schedule without lane_cells, and agree with them to
 * rounding with it.  No reference
 * counterpart: the schedule of deal.II's MatrixFree::cell_loop
 * (heat_diffuse_operator.cpp:183) is internal to it. */
typedef struct {
  int slabs;            /* 1..32 (capped at half the cell layers) */
  int l2_evict_first;   /* 0 or 1 */
  int overlap_colours;  /* 0 or 1 */
  int cta_cell_groups;  /* 0 or 1 */
  int lane_cells;       /* 0: warp apply; 1, 2: lane apply, 2 with more resident CTAs per SM */
} mpdg_schedule;
mpdg_status mpdg_op_set_schedule(mpdg_op *op, int precision, const mpdg_schedule *schedule);
mpdg_status mpdg_op_get_schedule(mpdg_op *op, int precision, mpdg_schedule *schedule);
/* Autotuner of the resident apply: times `reps` applies (after one warm-up) of
 * each candidate schedule -- slabs 1, 2, 4, 8, 16, each with and without the
 * evict-first hint where the mesh streams coefficients, each with and without
 * overlap_colours -- in the given
 * precision (MPDG_FP64 / MPDG_FP32), keeps the fastest on the operator and
 * returns it with its time per apply.  candidate_ms (may be NULL) receives up to
 * n_candidate_ms per-candidate times in that order (-1 past the last).
 * Allocates two scratch vectors for the duration of the call. */
mpdg_status mpdg_op_autotune(mpdg_op *op, int precision, int reps, mpdg_schedule *best, double *apply_ms,
                             double *candidate_ms, int n_candidate_ms);
/* measured FMA throughput of the current GPU (GFLOP/s, 2 flops per FMA) in
 * FP64 and FP32: the arithmetic ceiling the apply's flop rate is reported against */
mpdg_status mpdg_fma_peak(double *gflops64, double *gflops32);
mpdg_status mpdg_vmult_multi_f32(mpdg_op *op, int n_vectors, float *const *dst, const float *const *src);
/* LeastSquaresProjection::vmult (predictor.hpp:37-80): solution = sum_s c_s old[s]
 * minimising |A sum_s c_s old[s] - rhs| over the first old solutions whose images
 * stay independent (modified Gram-Schmidt, stop when the new image's squared norm
 * falls below 1e-16 of the first's).  n_old = 1..32 device vectors; *n_used (may
 * be NULL) receives how many were used (0: the first image is zero, solution = 0). */
mpdg_status mpdg_predict_lsq(mpdg_op *op, int n_old, const double *const *old_solutions, const double *rhs,
                             double *solution, int *n_used);
/* host-buffer form: copies src to the device, applies, copies dst back.  For a
 * plain warp-kernel operator (no faces, identity rows, hanging nodes, SUPG,
 * Newton tangent or phase law) on a lattice of >= 4 cell layers the three
 * steps overlap over up to 8 z-slabs of cell layers (copy-in, apply and
 * copy-out on separate streams); dst_host is complete when the call returns.
 * Pinned host buffers let the two copy directions run at once. */
mpdg_status mpdg_vmult_host(mpdg_op *op, double *dst_host, const double *src_host);

/* OperatorMatrixFree::compute_inverse_diagonal_from_matrixfree, operator_base.hpp:268-272
 * (heat: heat_diffuse_operator.cpp:271-284, threshold 1e-10;
 *  advection-diffusion: advection_diffusion_operator.cpp:401-446, threshold 1e-14 max(1,|d|inf)) */
mpdg_status mpdg_compute_inverse_diagonal(mpdg_op *op, double *inv_diag);
mpdg_status mpdg_compute_inverse_diagonal_host(mpdg_op *op, double *inv_diag_host);
/* the diagonal itself (before inversion; constrained entries 1) */
mpdg_status mpdg_compute_diagonal(mpdg_op *op, double *diag);

/* OperatorMatrixFree::create_rhs, operator_base.hpp:208-212: dst += rhs contribution.
 * heat (heat_diffuse_operator.cpp:783-806): src = T_old, the operator's temperature
 *   field is T, heat_source may be NULL; Dirichlet DoFs are not written.
 * advection-diffusion (advection_diffusion_operator.cpp:276-358): src = phi_old,
 *   heat_source must be NULL; written to all DoFs unless Dirichlet rows are selected. */
mpdg_status mpdg_create_rhs(mpdg_op *op, double *dst, const double *src, const double *heat_source);
/* host-buffer form of mpdg_create_rhs (dst_host in/out) */
mpdg_status mpdg_create_rhs_host(mpdg_op *op, double *dst_host, const double *src_host,
                                 const double *heat_source_host);

/* LinearSolver::solve, include/meltpooldg/linear_algebra/linear_solver.hpp:26-134,
 * with the Jacobi preconditioner of preconditioner_jacobi.hpp:29-88 (or the
 * Chebyshev smoother on top of it).  x holds the initial guess on entry.
 * GMRES is right-preconditioned with restart gmres_restart (default 30, at
 * most 60); its Arnoldi basis is orthogonalised by delayed classical
 * Gram-Schmidt with re-orthogonalisation, which builds the Krylov basis and
 * residual estimates of modified Gram-Schmidt in exact arithmetic, and applies
 * the operator once more than it iterates in each cycle that converges.  CG
 * tests convergence on the device after every iteration; the report counts
 * the iterations up to the one that converged. */
mpdg_status mpdg_solve(mpdg_op *op, const mpdg_solver_desc *desc, double *x, const double *b,
                       mpdg_solve_report *report);
/* host-buffer form of mpdg_solve (x_host in/out, b_host in) */
mpdg_status mpdg_solve_host(mpdg_op *op, const mpdg_solver_desc *desc, double *x_host,
                            const double *b_host, mpdg_solve_report *report);
void mpdg_solver_desc_default(mpdg_solver_desc *desc);

/* Jacobi-preconditioned CG (FP64) that allocates no device or pinned host
 * memory: for callers that cannot allocate while they solve -- a host whose
 * device memory is owned by its own pool or arena, a time loop that must not
 * synchronise the device (cudaMalloc/cudaFree do), an application that allows
 * no driver allocation after start-up.  It has no counterpart in the
 * reference (which allocates its solver vectors per solve).
 *
 * Scratch (the CG vectors, the inverse diagonal, reduction partials and
 * scalars) lives in one fixed __device__ array that every GPU loading the
 * library holds until exit; problems larger than 262,144 DoFs are rejected
 * with MPDG_ERR_SIZE.  The first call on a device resolves the array's device
 * address (cudaGetSymbolAddress) with that device current: make that first
 * call before any stream capture.  On a general (non-uniform) mesh, and with
 * inflow/outflow rows, the operator's coefficient stream and operand copy
 * must exist already (one mpdg_vmult first), else MPDG_ERR_ARG; operators
 * whose diagonal needs probe vectors (two-level meshes, SUPG) and mapped
 * meshes with constraints are rejected with MPDG_ERR_ARG.  All calls on a device share the array: calls whose work
 * overlaps on the GPU race and must be serialised by the caller.  Semantics as
 * mpdg_solve with solver CG and preconditioner Jacobi; x holds the start. */
mpdg_status mpdg_solve_cg_noalloc(mpdg_op *op, double *x, const double *b, double rel_tolerance,
                                  double abs_tolerance, int max_iterations,
                                  mpdg_solve_report *report);

/* integrated L2 norm of a DoF vector (VectorTools::compute_norm,
 * source/utilities/vector_tools.cpp:170-201), FP64 */
mpdg_status mpdg_l2_norm(mpdg_op *op, const double *u, double *norm);

/* number of kernels this library launched since load (its own kernels only) */
int64_t mpdg_kernel_launches(void);
/* number of device and pinned-host allocations (cudaMalloc, cudaMallocAsync,
 * pool and host allocations) this library made since load */
int64_t mpdg_allocations(void);

/* ------------------------------------------------------- batched solves
 * Many independent problems advanced together on one GPU.  The reference
 * solves one problem per process (LinearSolver::solve, linear_solver.hpp:26-134,
 * called from heat_transfer_operation.cpp:300-330 and
 * advection_diffusion_operation.cpp:228-262); a batch holds each admitted
 * problem's vectors resident in device memory and advances every running
 * problem by one Krylov step per CUDA-graph launch: one batched FP32 operator
 * apply per degree and colour over all problems' cells, per-problem FP64 dots
 * and norms, FP64 solution, and FP64 defects b - A x (FP64 operator) that
 * replace the FP32 residual whenever it has dropped by the reliable-update
 * factor, so the reported residual is an FP64 one.  Heat problems run CG,
 * advection-diffusion problems BiCGStab, both Jacobi-preconditioned.  A
 * problem's result does not depend on which other problems share the batch. */
typedef struct mpdg_batch mpdg_batch;

typedef struct {
  int kind;              /* MPDG_OP_HEAT (CG) or MPDG_OP_ADVDIFF (BiCGStab) */
  int degree;            /* 1..4 */
  int nc;                /* cells per direction of the unit cube, 2..400 */
  int dirichlet;         /* homogeneous Dirichlet on all faces (1) or none (0) */
  int vel_kind;          /* advection-diffusion: MPDG_VEL_VORTEX or MPDG_VEL_NONE */
  int max_iterations;    /* 0: the batch default */
  double dt;             /* time increment */
  double rho_cp, k0;     /* heat: rho c_p and conductivity */
  double theta, diffusivity;         /* advection-diffusion */
  double rel_tolerance, abs_tolerance;
  uint64_t rhs_seed;     /* right-hand side: values in [-1,1) from this seed (0 on Dirichlet DoFs) */
} mpdg_problem_desc;

/* budget_bytes bounds the device memory of all admitted problems' vectors;
 * capacity is the maximum number of problems held at once */
mpdg_status mpdg_batch_create(int64_t budget_bytes, int capacity, double reliable_delta,
                              mpdg_batch **batch);
mpdg_status mpdg_batch_destroy(mpdg_batch *batch);
/* device bytes a problem takes in a batch (its admission footprint) and its DoF count */
mpdg_status mpdg_problem_bytes(const mpdg_problem_desc *desc, int64_t *bytes, int64_t *n_dofs);
/* the seeded right-hand side of a problem, on the host (the values a batch uses) */
mpdg_status mpdg_problem_rhs_host(const mpdg_problem_desc *desc, double *b_host);
/* the FP64 Jacobi diagonal a batch uses for a problem (constrained entries 1) */
mpdg_status mpdg_problem_diagonal_host(const mpdg_problem_desc *desc, double *diag_host);
/* admits a problem: MPDG_ERR_BUDGET when its footprint does not fit the free
 * budget or no slot is free (nothing is admitted then).  rhs_host may be NULL
 * (seeded right-hand side) or n_dofs values.  Admission only enqueues work. */
mpdg_status mpdg_batch_submit(mpdg_batch *batch, const mpdg_problem_desc *desc, const double *rhs_host,
                              int64_t *ticket);
/* runs up to max_steps Krylov steps (graph launches), checking every
 * poll_steps steps whether problems are still running; returns the steps run
 * and the problems still running */
mpdg_status mpdg_batch_run(mpdg_batch *batch, int max_steps, int poll_steps, int *steps, int *running);
/* state of one problem: report->status is 1 while it runs, else its final status */
mpdg_status mpdg_batch_poll(mpdg_batch *batch, int64_t ticket, mpdg_solve_report *report);
/* copies a finished problem's solution to the host (x_host may be NULL), fills
 * the report and releases the problem's slot and memory */
mpdg_status mpdg_batch_take(mpdg_batch *batch, int64_t ticket, double *x_host, mpdg_solve_report *report);
/* the batch's autotuner: times the batched FP32 apply of the current
 * membership (call once problems are admitted) over its block and tile shapes
 * -- 2, 4 or 8 warps per CTA, the conflict-minimal or the plain tile layout,
 * and 1, 2, 3, 4, 6, 8 or the occupancy maximum of resident CTAs per SM --
 * and keeps the fastest; returns its CTAs per SM and time (mpdg_batch_shape
 * reads the whole shape).  No reference counterpart (the reference has no
 * batched solves). */
mpdg_status mpdg_batch_autotune(mpdg_batch *batch, int *ctas_per_sm, double *apply_ms);
/* the shape the batched apply runs with: warps per CTA, tile layout (1: the
 * conflict-minimal one) and resident CTAs per SM (0: occupancy maximum) */
mpdg_status mpdg_batch_shape(mpdg_batch *batch, int *warps_per_cta, int *tuned_tiles, int *ctas_per_sm);
/* device bytes admitted now */
mpdg_status mpdg_batch_used_bytes(mpdg_batch *batch, int64_t *bytes);
/* counters of the last mpdg_serve call (n <= 9 values): host seconds spent in
 * admission, in result copies, waiting for the GPU and in graph launches;
 * graph steps launched; requests admitted and finished; most problems
 * resident at once; polls of the running flags */
mpdg_status mpdg_batch_stats(mpdg_batch *batch, double *stats, int n);

/* Serving loop: requests arrive at arrival_s[i] seconds after the call starts
 * (ascending).  Each arrived request is admitted as soon as its footprint fits
 * the batch's budget and a slot is free (first come, first served), joins the
 * running problems at the next step, and leaves the batch when it finishes:
 * its solution is copied to the host (into x_host[i] when x_host and
 * x_host[i] are not NULL, else into a staging buffer) and its latency
 * (completion - arrival) recorded.  poll_steps graph steps run between checks
 * of finished problems.  latency_s, x_norm (|x|_2, FP64) and reports may be
 * NULL; wall_s receives the time from the start to the last completion. */
mpdg_status mpdg_serve(mpdg_batch *batch, const mpdg_problem_desc *requests, const double *arrival_s,
                       int n_requests, int poll_steps, double **x_host, double *latency_s,
                       double *x_norm, mpdg_solve_report *reports, double *wall_s);

#ifdef __cplusplus
}
#endif
#endif
