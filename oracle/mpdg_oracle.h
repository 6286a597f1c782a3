/*
 * mpdg_oracle.h -- CPU oracle for the matrix-free heat / advection-diffusion
 * operators.  TEST INFRASTRUCTURE ONLY: the tests, the smoke check and the
 * CPU-baseline leg of bench.py use it as the checker; no product code path
 * links or calls it.
 *
 * It restates, in plain FP64 C, the arithmetic that MeltPoolDG performs
 * through deal.II's MatrixFree/FEEvaluation on the operator path:
 *   - heat tangent      source/heat/heat_diffuse_operator.cpp:179-197,955-1086
 *   - heat Robin faces  source/heat/heat_diffuse_operator.cpp:1088-1129
 *   - heat residual     source/heat/heat_diffuse_operator.cpp:393-529,726-806
 *   - heat diagonal     source/heat/heat_diffuse_operator.cpp:271-284
 *   - advdiff tangent   source/level_set/advection_diffusion_operator.cpp:238-272,450-495
 *   - advdiff rhs       source/level_set/advection_diffusion_operator.cpp:276-358
 *   - advdiff diagonal  source/level_set/advection_diffusion_operator.cpp:401-446
 *   - discretisation    source/utilities/fe_util.cpp:18-57 (FE_Q(p) on Gauss-Lobatto
 *                       support points, MappingQGeneric, QGauss(p+1))
 *   - Krylov solvers    include/meltpooldg/linear_algebra/linear_solver.hpp:26-134
 *                       (ReductionControl semantics)
 *
 * Meshes are structured boxes of nc[0] x nc[1] (x nc[2]) multilinear cells
 * whose vertices are given explicitly (so they may be perturbed).  Global
 * DoFs are numbered lexicographically, x fastest:
 *   g = (Z * NY + Y) * NX + X,  X = ix*p + i in [0, nc[0]*p], ...
 */
#ifndef MPDG_ORACLE_H
#define MPDG_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_HEAT = 0, ORC_ADVDIFF = 1 };

enum {
  ORC_VEL_NONE = 0,
  ORC_VEL_ROTATION = 1, /* u = s * (x_{dim-1}, 0.., -x_0): advection_diffusion_vortex.hpp:93-115 */
  ORC_VEL_VORTEX = 2,   /* u = (sin pi x cos pi y, -cos pi x sin pi y, 0) */
  ORC_VEL_CONST = 3,    /* u = vel_param */
  ORC_VEL_NODAL = 4     /* u interpolated from a dim x N nodal field (component-major) */
};

enum { ORC_PREC_IDENTITY = 0, ORC_PREC_JACOBI = 1, ORC_PREC_CHEBYSHEV = 2 };
/* heat material laws (MaterialTypes, Material::compute_parameters_internal,
 * include/meltpooldg/core/material.templates.hpp:213-500): LINEAR is rho_cp and
 * k(T) = k0 (1 + k_alpha T); the phase laws interpolate gas / liquid / solid
 * properties by the level-set heaviside H and the solid fraction f_s(T) */
enum { ORC_MAT_LINEAR = 0, ORC_MAT_GAS_LIQUID = 1, ORC_MAT_LIQUID_SOLID = 2, ORC_MAT_GAS_LIQUID_SOLID = 3 };
/* apparent heat capacity profiles of the latent heat of fusion (ApparentCapacityType) */
enum { ORC_AC_POLY4_BELL = 0, ORC_AC_CONSTANT = 1, ORC_AC_QLQ = 2 };
#define ORC_STEFAN_BOLTZMANN 5.670374419e-8

typedef struct {
  int dim;             /* 2 or 3 */
  int degree;          /* p >= 1 */
  int nc[3];           /* cells per direction (nc[2] ignored for dim 2) */
  const double *vert;  /* (nc0+1)(nc1+1)(nc2+1) x dim vertex coordinates, x fastest */
} orc_mesh;

typedef struct {
  int kind;                  /* ORC_HEAT or ORC_ADVDIFF */
  double dt;                 /* time increment */
  /* heat */
  double rho_cp;             /* volumetric heat capacity rho*c_p */
  double k0, k_alpha;        /* conductivity law k(T) = k0 * (1 + k_alpha * T) */
  int full_tangent;          /* add dk/dT * grad(T) * du to the flux (non-symmetric) */
  const double *temperature; /* nodal T for k(T) and the residual; NULL means T = 0 */
  double robin_alpha;        /* convection coefficient on Robin faces */
  double robin_t_inf;        /* ambient temperature of the Robin condition (residual only) */
  int robin_faces;           /* bit (2*d + side): box face with normal along d, side 0 = min */
  /* advection-diffusion */
  double theta, diffusivity;
  /* velocity, both operators */
  int vel_kind;
  double vel_param[3];
  const double *vel_nodal;
  /* homogeneous Dirichlet mask: constrained DoFs are read as 0 and never written */
  const unsigned char *dirichlet;
  /* advection-diffusion SUPG (advection_diffusion_operator.cpp:450-533): flux
   * += tau_K vel (residual), tau_K = h_K / max_q |vel| (coefficient < 0) or
   * coefficient h_K, h_K = cell diameter / sqrt(dim); axis-aligned cells */
  int supg;
  double supg_coefficient;
  /* heat: radiative faces (heat_diffuse_operator.cpp:766-772, 1122-1124): tangent
   * 4 eps sigma T^3 u v, residual -eps sigma (T^4 - T_inf^4) v; bits as robin_faces */
  double rad_emissivity, rad_t_inf;
  int rad_faces;
  /* heat: material law (ORC_MAT_*); phase properties index 0 gas, 1 liquid, 2 solid */
  int material;
  double mat_rho[3], mat_cp[3], mat_k[3];
  double solidus, liquidus;
  int two_phase_sharp;      /* weight heaviside(H, 0.5) instead of H */
  int solid_liquid_sharp;   /* f_s = T < solidus instead of the mushy-zone ramp */
  int volume_specific;      /* interpolate rho*c_p itself instead of rho and c_p */
  const double *temperature_old; /* T_old: solidification terms of the tangent */
  const double *heaviside;       /* level set as heaviside, nodal (two-phase laws) */
  /* latent heat of fusion (> 0: the apparent capacity of profile ORC_AC_* is
   * added to c_p in the mushy zone of laws with a solid phase) */
  double latent_heat;
  int apparent_capacity;
} orc_op;

typedef struct {
  int type;                 /* ORC_PREC_* */
  const double *inv_diag;   /* Jacobi / Chebyshev diagonal */
  int degree;               /* Chebyshev: residual polynomial degree (degree-1 operator applies) */
  double lambda_min, lambda_max;
} orc_prec;

long orc_n_dofs(const orc_mesh *m);
void orc_gauss_legendre(int n, double *x, double *w);  /* on [0,1] */
void orc_gauss_lobatto(int n, double *x);              /* on [0,1] */
/* S[q*n+i] = phi_i(xq), D[q*n+i] = phi_i'(xq), phi on the n Gauss-Lobatto nodes */
void orc_shape_tables(int n, const double *xq, int nq, double *S, double *D);
void orc_dof_coordinates(const orc_mesh *m, double *xyz);   /* N x dim */

void orc_vmult(const orc_mesh *m, const orc_op *op, double *dst, const double *src);
void orc_vmult_brute(const orc_mesh *m, const orc_op *op, double *dst, const double *src);
void orc_vmult_cells(const orc_mesh *m, const orc_op *op, double *dst, const double *src,
                     long cell_begin, long cell_end);
void orc_diagonal(const orc_mesh *m, const orc_op *op, double *diag);
void orc_invert_diagonal(const orc_mesh *m, const orc_op *op, double *diag);
void orc_rhs_heat(const orc_mesh *m, const orc_op *op, double *dst, const double *t_old,
                  const double *heat_source, const unsigned char *scatter_mask);
void orc_rhs_advdiff(const orc_mesh *m, const orc_op *op, double *dst, const double *phi_old,
                     const unsigned char *scatter_mask);
double orc_l2_norm(const orc_mesh *m, const double *u);
void orc_l2_norm_cells(const orc_mesh *m, const double *u, double *cell_norms);

int orc_cg(const orc_mesh *m, const orc_op *op, const orc_prec *P, const double *b, double *x,
           double rel_tol, double abs_tol, int max_it, int *n_it, double *res_hist);
int orc_gmres(const orc_mesh *m, const orc_op *op, const orc_prec *P, const double *b, double *x,
              double rel_tol, double abs_tol, int max_it, int restart, int *n_it,
              double *res_hist);
double orc_estimate_lambda_max(const orc_mesh *m, const orc_op *op, const double *inv_diag,
                               const double *start, int n_steps);
void orc_prec_apply(const orc_mesh *m, const orc_op *op, const orc_prec *P, double *z,
                    const double *r);

/* ------------------------------------------------------------ hanging nodes
 * Two-level mesh: a coarse block and a fine block refined 2:1 in y and z,
 * meeting at the plane normal to x where the coarse block ends (coarse cells
 * ix = nc[0]-1, fine cells ix = 0).  fine.nc[1] = 2 coarse.nc[1], fine.nc[2] =
 * 2 coarse.nc[2]; the fine interface vertices lie on the coarse faces.
 * Global vector: the coarse block's DoFs (lexicographic), then the fine
 * block's (lexicographic, all of its lattice).  The fine DoFs on the interface
 * plane hang on the coarse face (deal.II hanging-node constraints of a 2:1
 * refined face): the value of fine DoF (j, k) of subface (sy, sz) is the coarse
 * face interpolant  sum_{j',k'} P[sy][j][j'] P[sz][k][k'] u_c(j', k'),
 * P[s][j][j'] = coarse Lagrange basis j' at (s + z_j) / 2.  The operator is
 * sum_K C_K^T A_K C_K; the hanging DoFs are constrained like Dirichlet DoFs
 * (read through the constraint, output 0, diagonal 1).  dim 3, constant
 * coefficients (no k(T) field, no Robin faces, analytic velocities). */
typedef struct {
  orc_mesh coarse, fine;
} orc_mesh2;

long orc2_n_dofs(const orc_mesh2 *m);
/* P[s][j][j'] of degree p (2 x n x n) */
void orc2_hanging_matrix(int degree, double *P);
void orc2_vmult(const orc_mesh2 *m, const orc_op *op, double *dst, const double *src);
void orc2_diagonal(const orc_mesh2 *m, const orc_op *op, double *diag);
/* values of the hanging fine DoFs from the coarse DoFs (the constraint distribution) */
void orc2_distribute(const orc_mesh2 *m, double *u);
void orc2_dof_coordinates(const orc_mesh2 *m, double *xyz);

/* ------------------------------------------------------------- mapped meshes
 * Unstructured hexahedra: each cell's 8 corners (x fastest) and its cell->DoF
 * map (n^3 per cell, lexicographic), homogeneous affine constraints as CSR over
 * all DoFs (cons_ptr[N+1]; an empty range = unconstrained).  dim 3, constant
 * coefficients or fields read through the map; no faces, no SUPG. */
typedef struct {
  int degree;
  long n_cells, n_dofs;
  const double *cell_vertices;
  const long *cell_dofs;
  const long *cons_ptr;
  const long *cons_idx;
  const double *cons_w;
  /* boundary id of each cell's local face 2 d + s ([n_cells][6]; -1 interior,
   * 0..5 the bit of robin_faces / rad_faces that selects it), or NULL */
  const signed char *face_ids;
} orc_mapped;

void orcm_vmult(const orc_mapped *m, const orc_op *op, double *dst, const double *src);
/* apparent capacity of op's latent heat at temperature T and its T derivative
 * (solid fraction from op's solidus/liquidus, clamped to [0, 1]) */
void orc_apparent_capacity(const orc_op *op, double T, double *c, double *dc);
void orcm_diagonal(const orc_mapped *m, const orc_op *op, double *diag);

#ifdef __cplusplus
}
#endif
#endif
