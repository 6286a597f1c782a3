"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, the smoke check and the CPU-baseline leg of bench.py import this
module; it is the checker of the CUDA path, never part of it.  The C side
(mpdg_oracle.c) restates MeltPoolDG's operator arithmetic; this file adds mesh
and boundary-mask builders and thin wrappers.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmpdg_oracle.so")

HEAT, ADVDIFF = 0, 1
VEL_NONE, VEL_ROTATION, VEL_VORTEX, VEL_CONST, VEL_NODAL = 0, 1, 2, 3, 4
PREC_IDENTITY, PREC_JACOBI, PREC_CHEBYSHEV = 0, 1, 2
MAT_LINEAR, MAT_GAS_LIQUID, MAT_LIQUID_SOLID, MAT_GAS_LIQUID_SOLID = 0, 1, 2, 3
AC_POLY4_BELL, AC_CONSTANT, AC_QLQ = 0, 1, 2

_dp = C.POINTER(C.c_double)
_u8p = C.POINTER(C.c_uint8)


class _Mesh(C.Structure):
    _fields_ = [("dim", C.c_int), ("degree", C.c_int), ("nc", C.c_int * 3), ("vert", _dp)]


class _Op(C.Structure):
    _fields_ = [
        ("kind", C.c_int), ("dt", C.c_double),
        ("rho_cp", C.c_double), ("k0", C.c_double), ("k_alpha", C.c_double),
        ("full_tangent", C.c_int), ("temperature", _dp),
        ("robin_alpha", C.c_double), ("robin_t_inf", C.c_double), ("robin_faces", C.c_int),
        ("theta", C.c_double), ("diffusivity", C.c_double),
        ("vel_kind", C.c_int), ("vel_param", C.c_double * 3), ("vel_nodal", _dp),
        ("dirichlet", _u8p),
        ("supg", C.c_int), ("supg_coefficient", C.c_double),
        ("rad_emissivity", C.c_double), ("rad_t_inf", C.c_double), ("rad_faces", C.c_int),
        ("material", C.c_int), ("mat_rho", C.c_double * 3), ("mat_cp", C.c_double * 3),
        ("mat_k", C.c_double * 3), ("solidus", C.c_double), ("liquidus", C.c_double),
        ("two_phase_sharp", C.c_int), ("solid_liquid_sharp", C.c_int), ("volume_specific", C.c_int),
        ("temperature_old", _dp), ("heaviside", _dp),
        ("latent_heat", C.c_double), ("apparent_capacity", C.c_int),
    ]


class _Mesh2(C.Structure):
    _fields_ = [("coarse", _Mesh), ("fine", _Mesh)]


_lp = C.POINTER(C.c_long)


class _Mapped(C.Structure):
    _fields_ = [("degree", C.c_int), ("n_cells", C.c_long), ("n_dofs", C.c_long), ("cell_vertices", _dp),
                ("cell_dofs", _lp), ("cons_ptr", _lp), ("cons_idx", _lp), ("cons_w", _dp),
                ("face_ids", C.POINTER(C.c_int8))]


class _Prec(C.Structure):
    _fields_ = [("type", C.c_int), ("inv_diag", _dp), ("degree", C.c_int),
                ("lambda_min", C.c_double), ("lambda_max", C.c_double)]


def build():
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P_m, P_o, P_p = C.POINTER(_Mesh), C.POINTER(_Op), C.POINTER(_Prec)
        L.orc_n_dofs.restype = C.c_long
        L.orc_n_dofs.argtypes = [P_m]
        for name in ("orc_vmult", "orc_vmult_brute"):
            getattr(L, name).argtypes = [P_m, P_o, _dp, _dp]
        L.orc_vmult_cells.argtypes = [P_m, P_o, _dp, _dp, C.c_long, C.c_long]
        L.orc_diagonal.argtypes = [P_m, P_o, _dp]
        L.orc_invert_diagonal.argtypes = [P_m, P_o, _dp]
        L.orc_rhs_heat.argtypes = [P_m, P_o, _dp, _dp, _dp, _u8p]
        L.orc_rhs_advdiff.argtypes = [P_m, P_o, _dp, _dp, _u8p]
        L.orc_l2_norm.restype = C.c_double
        L.orc_l2_norm.argtypes = [P_m, _dp]
        L.orc_dof_coordinates.argtypes = [P_m, _dp]
        L.orc_cg.argtypes = [P_m, P_o, P_p, _dp, _dp, C.c_double, C.c_double, C.c_int,
                             C.POINTER(C.c_int), _dp]
        L.orc_gmres.argtypes = [P_m, P_o, P_p, _dp, _dp, C.c_double, C.c_double, C.c_int,
                                C.c_int, C.POINTER(C.c_int), _dp]
        L.orc_estimate_lambda_max.restype = C.c_double
        L.orc_estimate_lambda_max.argtypes = [P_m, P_o, _dp, _dp, C.c_int]
        L.orc_prec_apply.argtypes = [P_m, P_o, P_p, _dp, _dp]
        L.orc_gauss_legendre.argtypes = [C.c_int, _dp, _dp]
        L.orc_gauss_lobatto.argtypes = [C.c_int, _dp]
        P_m2 = C.POINTER(_Mesh2)
        L.orc2_n_dofs.restype = C.c_long
        L.orc2_n_dofs.argtypes = [P_m2]
        L.orc2_hanging_matrix.argtypes = [C.c_int, _dp]
        L.orc2_vmult.argtypes = [P_m2, P_o, _dp, _dp]
        L.orc2_diagonal.argtypes = [P_m2, P_o, _dp]
        L.orc2_distribute.argtypes = [P_m2, _dp]
        L.orc2_dof_coordinates.argtypes = [P_m2, _dp]
        P_mm = C.POINTER(_Mapped)
        L.orcm_vmult.argtypes = [P_mm, P_o, _dp, _dp]
        L.orcm_diagonal.argtypes = [P_mm, P_o, _dp]
        L.orc_apparent_capacity.argtypes = [P_o, C.c_double, _dp, _dp]
        _lib = L
    return _lib


def _ptr(a, t=_dp):
    return None if a is None else a.ctypes.data_as(t)


# ----------------------------------------------------------------- meshes

def box_vertices(dim, nc, lo, hi, perturb=0.0, seed=None):
    """Vertices of a structured box mesh, x fastest; interior vertices moved by
    U[-perturb*h, perturb*h] per coordinate when perturb > 0 (boundary fixed)."""
    nc = list(nc)[:dim]
    axes = [np.linspace(lo[d], hi[d], nc[d] + 1) for d in range(dim)]
    grids = np.meshgrid(*axes[::-1], indexing="ij")[::-1]  # slowest axis first
    V = np.stack([g.reshape(-1) for g in grids], axis=1).astype(np.float64)
    if perturb > 0.0:
        rng = np.random.Generator(np.random.PCG64(seed))
        h = np.array([(hi[d] - lo[d]) / nc[d] for d in range(dim)])
        disp = rng.uniform(-1.0, 1.0, size=V.shape) * perturb * h
        idx = np.stack(np.meshgrid(*[np.arange(n + 1) for n in nc[::-1]], indexing="ij")[::-1],
                       axis=-1).reshape(-1, dim)
        interior = np.all((idx > 0) & (idx < np.array(nc)), axis=1)
        V[interior] += disp[interior]
    return np.ascontiguousarray(V)


class Mesh:
    def __init__(self, dim, degree, nc, vertices):
        self.dim, self.degree = dim, degree
        self.nc = (list(nc) + [1, 1, 1])[:3]
        if dim == 2:
            self.nc[2] = 1
        self.vert = np.ascontiguousarray(vertices, dtype=np.float64)
        self._c = _Mesh(dim, degree, (C.c_int * 3)(*self.nc), _ptr(self.vert))
        self.shape = tuple(self.nc[d] * degree + 1 for d in range(dim))  # (NX, NY[, NZ])
        self.n_dofs = int(np.prod(self.shape))
        self.n_cells = int(np.prod(self.nc[:dim]))

    @classmethod
    def box(cls, dim, degree, nc, lo=None, hi=None, perturb=0.0, seed=None):
        lo = lo if lo is not None else [0.0] * dim
        hi = hi if hi is not None else [1.0] * dim
        return cls(dim, degree, nc, box_vertices(dim, nc, lo, hi, perturb, seed))

    def dof_coordinates(self):
        x = np.zeros((self.n_dofs, self.dim))
        lib().orc_dof_coordinates(C.byref(self._c), _ptr(x))
        return x

    def grid_index(self):
        """Integer grid coordinates (X, Y[, Z]) of each DoF."""
        idx = np.indices(self.shape[::-1]).reshape(self.dim, -1)[::-1]
        return idx.T

    def boundary_face_mask(self, faces=None):
        """uint8 mask of DoFs on the selected box faces (default: all faces);
        faces = iterable of (direction, side)."""
        gi = self.grid_index()
        mask = np.zeros(self.n_dofs, dtype=bool)
        if faces is None:
            faces = [(d, s) for d in range(self.dim) for s in (0, 1)]
        for d, s in faces:
            mask |= gi[:, d] == (0 if s == 0 else self.shape[d] - 1)
        return mask.astype(np.uint8)


def _arr(a, dtype=np.float64):
    return None if a is None else np.ascontiguousarray(a, dtype)


class Operator:
    """Parameters of one heat or advection-diffusion operator (oracle side).

    `material` selects a phase law of the heat operator: a dict with `kind`
    (MAT_GAS_LIQUID, MAT_LIQUID_SOLID, MAT_GAS_LIQUID_SOLID), `rho`, `cp`, `k`
    (each (gas, liquid, solid)), `solidus`, `liquidus` and the flags
    `two_phase_sharp`, `solid_liquid_sharp`, `volume_specific`, and the latent
    heat of fusion `latent_heat` with its `apparent_capacity` profile (AC_*,
    default AC_QLQ as in MaterialData); None keeps
    rho_cp and k(T) = k0 (1 + k_alpha T).  `temperature_old` and `heaviside` are
    the nodal fields those laws read."""

    def __init__(self, kind, dt, rho_cp=1.0, k0=1.0, k_alpha=0.0, full_tangent=False,
                 temperature=None, robin_alpha=0.0, robin_t_inf=0.0, robin_faces=0,
                 theta=0.5, diffusivity=0.0, vel_kind=VEL_NONE, vel_param=(0.0, 0.0, 0.0),
                 vel_nodal=None, dirichlet=None, supg=False, supg_coefficient=-1.0,
                 rad_emissivity=0.0, rad_t_inf=0.0, rad_faces=0, material=None,
                 temperature_old=None, heaviside=None):
        self.temperature = _arr(temperature)
        self.vel_nodal = _arr(vel_nodal)
        self.dirichlet = _arr(dirichlet, np.uint8)
        self.temperature_old = _arr(temperature_old)
        self.heaviside = _arr(heaviside)
        self.kind, self.dt = kind, dt
        mat = material or {}
        three = C.c_double * 3
        self._c = _Op(kind, dt, rho_cp, k0, k_alpha, int(full_tangent), _ptr(self.temperature),
                      robin_alpha, robin_t_inf, robin_faces, theta, diffusivity, vel_kind,
                      three(*vel_param), _ptr(self.vel_nodal),
                      _ptr(self.dirichlet, _u8p), int(bool(supg)), float(supg_coefficient),
                      rad_emissivity, rad_t_inf, rad_faces, int(mat.get("kind", MAT_LINEAR)),
                      three(*mat.get("rho", (0, 0, 0))), three(*mat.get("cp", (0, 0, 0))),
                      three(*mat.get("k", (0, 0, 0))), float(mat.get("solidus", 0.0)),
                      float(mat.get("liquidus", 0.0)), int(bool(mat.get("two_phase_sharp", False))),
                      int(bool(mat.get("solid_liquid_sharp", False))),
                      int(bool(mat.get("volume_specific", False))),
                      _ptr(self.temperature_old), _ptr(self.heaviside),
                      float(mat.get("latent_heat", 0.0)), int(mat.get("apparent_capacity", AC_QLQ)))
        self.params = dict(kind=kind, dt=dt, rho_cp=rho_cp, k0=k0, k_alpha=k_alpha,
                           full_tangent=full_tangent, robin_alpha=robin_alpha,
                           robin_t_inf=robin_t_inf, robin_faces=robin_faces, theta=theta,
                           diffusivity=diffusivity, vel_kind=vel_kind, vel_param=vel_param, supg=supg,
                           supg_coefficient=supg_coefficient, rad_emissivity=rad_emissivity,
                           rad_t_inf=rad_t_inf, rad_faces=rad_faces, material=material)
        self.fields = dict(temperature=self.temperature, vel_nodal=self.vel_nodal, dirichlet=self.dirichlet,
                           temperature_old=self.temperature_old, heaviside=self.heaviside)

    def _with(self, **kw):
        f = dict(self.fields)
        f.update(kw)
        return Operator(**self.params, **f)

    def with_dirichlet(self, mask):
        return self._with(dirichlet=mask)

    def with_temperature(self, T):
        return self._with(temperature=T)

    def with_fields(self, **kw):
        return self._with(**kw)


# ----------------------------------------------------------- operations

def vmult(mesh, op, src, brute=False):
    src = np.ascontiguousarray(src, np.float64)
    dst = np.zeros(mesh.n_dofs)
    f = lib().orc_vmult_brute if brute else lib().orc_vmult
    f(C.byref(mesh._c), C.byref(op._c), _ptr(dst), _ptr(src))
    return dst


def vmult_cells(mesh, op, src, cell_begin, cell_end):
    """Apply of a contiguous range of cells only (CPU-baseline sampling)."""
    src = np.ascontiguousarray(src, np.float64)
    dst = np.zeros(mesh.n_dofs)
    lib().orc_vmult_cells(C.byref(mesh._c), C.byref(op._c), _ptr(dst), _ptr(src),
                          int(cell_begin), int(cell_end))
    return dst


def diagonal(mesh, op):
    d = np.zeros(mesh.n_dofs)
    lib().orc_diagonal(C.byref(mesh._c), C.byref(op._c), _ptr(d))
    return d


def inverse_diagonal(mesh, op):
    d = diagonal(mesh, op)
    lib().orc_invert_diagonal(C.byref(mesh._c), C.byref(op._c), _ptr(d))
    return d


def rhs_heat(mesh, op, t_old, heat_source=None, scatter_mask=None, dst=None):
    dst = np.zeros(mesh.n_dofs) if dst is None else dst
    t_old = np.ascontiguousarray(t_old, np.float64)
    hs = None if heat_source is None else np.ascontiguousarray(heat_source, np.float64)
    sm = None if scatter_mask is None else np.ascontiguousarray(scatter_mask, np.uint8)
    lib().orc_rhs_heat(C.byref(mesh._c), C.byref(op._c), _ptr(dst), _ptr(t_old), _ptr(hs),
                       _ptr(sm, _u8p))
    return dst


def rhs_advdiff(mesh, op, phi_old, scatter_mask=None, dst=None):
    dst = np.zeros(mesh.n_dofs) if dst is None else dst
    phi_old = np.ascontiguousarray(phi_old, np.float64)
    sm = None if scatter_mask is None else np.ascontiguousarray(scatter_mask, np.uint8)
    lib().orc_rhs_advdiff(C.byref(mesh._c), C.byref(op._c), _ptr(dst), _ptr(phi_old),
                          _ptr(sm, _u8p))
    return dst


def apparent_capacity(op, T):
    """(apparent capacity, its T derivative) of the operator's latent heat at
    temperature T (ApparentCapacity, source/heat/apparent_capacity.cpp)."""
    c, dc = C.c_double(), C.c_double()
    lib().orc_apparent_capacity(C.byref(op._c), float(T), C.byref(c), C.byref(dc))
    return c.value, dc.value


def l2_norm(mesh, u):
    u = np.ascontiguousarray(u, np.float64)
    return lib().orc_l2_norm(C.byref(mesh._c), _ptr(u))


def _prec(kind, inv_diag=None, degree=0, lmin=0.0, lmax=0.0):
    return _Prec(kind, _ptr(inv_diag), degree, lmin, lmax)


def cg(mesh, op, b, x0=None, inv_diag=None, rel_tol=1e-12, abs_tol=1e-20, max_it=10000,
       chebyshev=None):
    """Returns (x, iterations, residual history, converged)."""
    x = np.zeros(mesh.n_dofs) if x0 is None else np.array(x0, dtype=np.float64)
    b = np.ascontiguousarray(b, np.float64)
    if chebyshev is not None:
        P = _prec(PREC_CHEBYSHEV, inv_diag, chebyshev["degree"], chebyshev["lambda_min"],
                  chebyshev["lambda_max"])
    elif inv_diag is not None:
        P = _prec(PREC_JACOBI, inv_diag)
    else:
        P = _prec(PREC_IDENTITY)
    it = C.c_int(0)
    hist = np.zeros(max_it + 1)
    st = lib().orc_cg(C.byref(mesh._c), C.byref(op._c), C.byref(P), _ptr(b), _ptr(x), rel_tol,
                      abs_tol, max_it, C.byref(it), _ptr(hist))
    return x, it.value, hist[: it.value + 1], st == 0


def gmres(mesh, op, b, x0=None, inv_diag=None, rel_tol=1e-12, abs_tol=1e-20, max_it=10000,
          restart=30):
    x = np.zeros(mesh.n_dofs) if x0 is None else np.array(x0, dtype=np.float64)
    b = np.ascontiguousarray(b, np.float64)
    P = _prec(PREC_JACOBI, inv_diag) if inv_diag is not None else _prec(PREC_IDENTITY)
    it = C.c_int(0)
    hist = np.zeros(max_it + 1)
    st = lib().orc_gmres(C.byref(mesh._c), C.byref(op._c), C.byref(P), _ptr(b), _ptr(x), rel_tol,
                         abs_tol, max_it, restart, C.byref(it), _ptr(hist))
    return x, it.value, hist[: it.value + 1], st == 0


def lambda_max(mesh, op, inv_diag, start, n_steps=10):
    start = np.ascontiguousarray(start, np.float64)
    return lib().orc_estimate_lambda_max(C.byref(mesh._c), C.byref(op._c), _ptr(inv_diag),
                                         _ptr(start), n_steps)


def chebyshev_apply(mesh, op, inv_diag, r, degree, lmin, lmax):
    z = np.zeros(mesh.n_dofs)
    r = np.ascontiguousarray(r, np.float64)
    P = _prec(PREC_CHEBYSHEV, inv_diag, degree, lmin, lmax)
    lib().orc_prec_apply(C.byref(mesh._c), C.byref(op._c), C.byref(P), _ptr(z), _ptr(r))
    return z


def gauss_legendre(n):
    x, w = np.zeros(n), np.zeros(n)
    lib().orc_gauss_legendre(n, _ptr(x), _ptr(w))
    return x, w


def gauss_lobatto(n):
    x = np.zeros(n)
    lib().orc_gauss_lobatto(n, _ptr(x))
    return x


# ------------------------------------------------------------ hanging nodes

class Mesh2:
    """Two-level mesh (orc_mesh2): a coarse block of nc cells on
    [lo, (xm, hi_y, hi_z)] and a fine block of (ncf_x, 2 nc_y, 2 nc_z) cells on
    [(xm, lo_y, lo_z), hi]; the fine DoFs on the plane x = xm hang on the coarse
    faces.  Interior vertices of each block may be perturbed; boundary vertices
    (the interface included) stay on the regular lattice."""

    def __init__(self, degree, nc, ncf_x, lo=(0.0, 0.0, 0.0), xm=0.5, hi=(1.0, 1.0, 1.0), perturb=0.0,
                 seed=None):
        nc = tuple(int(v) for v in nc)
        ncf = (int(ncf_x), 2 * nc[1], 2 * nc[2])
        Vc = box_vertices(3, nc, lo, (xm, hi[1], hi[2]), perturb, seed)
        Vf = box_vertices(3, ncf, (xm, lo[1], lo[2]), hi, perturb, None if seed is None else seed + 1)
        self.degree = degree
        self.coarse = Mesh(3, degree, nc, Vc)
        self.fine = Mesh(3, degree, ncf, Vf)
        self._c = _Mesh2(self.coarse._c, self.fine._c)
        self.n_coarse = self.coarse.n_dofs
        self.n_dofs = self.coarse.n_dofs + self.fine.n_dofs

    def hanging_mask(self):
        """uint8 mask of the hanging fine DoFs (the fine block's x = xm plane)."""
        m = np.zeros(self.n_dofs, dtype=np.uint8)
        m[self.n_coarse:] = (self.fine.grid_index()[:, 0] == 0)
        return m

    def boundary_face_mask(self, faces=None):
        """Dirichlet mask of the outer box faces ((direction, side) pairs; default
        all six): x = lo on the coarse block, x = hi on the fine block, the
        y and z faces on both.  The hanging plane is not part of it."""
        if faces is None:
            faces = [(d, s) for d in range(3) for s in (0, 1)]
        fc = [f for f in faces if f != (0, 1)]
        ff = [f for f in faces if f != (0, 0)]
        mc = self.coarse.boundary_face_mask(fc) if fc else np.zeros(self.n_coarse, np.uint8)
        mf = self.fine.boundary_face_mask(ff) if ff else np.zeros(self.fine.n_dofs, np.uint8)
        return np.concatenate([mc, mf]).astype(np.uint8)

    def dof_coordinates(self):
        x = np.zeros((self.n_dofs, 3))
        lib().orc2_dof_coordinates(C.byref(self._c), _ptr(x))
        return x


def hanging_matrix(degree):
    """P[s, j, j'] = coarse Lagrange basis j' at the fine node (s + z_j) / 2."""
    n = degree + 1
    P = np.zeros(2 * n * n)
    lib().orc2_hanging_matrix(degree, _ptr(P))
    return P.reshape(2, n, n)


def vmult2(mesh2, op, src):
    src = np.ascontiguousarray(src, np.float64)
    dst = np.zeros(mesh2.n_dofs)
    lib().orc2_vmult(C.byref(mesh2._c), C.byref(op._c), _ptr(dst), _ptr(src))
    return dst


def diagonal2(mesh2, op):
    d = np.zeros(mesh2.n_dofs)
    lib().orc2_diagonal(C.byref(mesh2._c), C.byref(op._c), _ptr(d))
    return d


def distribute2(mesh2, u):
    """u with its hanging fine DoFs set to the coarse face interpolant."""
    u = np.array(u, dtype=np.float64)
    lib().orc2_distribute(C.byref(mesh2._c), _ptr(u))
    return u


# ------------------------------------------------------ least-squares predictor

def lsq_projection(mesh, op, old_solutions, rhs):
    """LeastSquaresProjection::vmult (include/meltpooldg/linear_algebra/predictor.hpp:37-80):
    images w_s = A x_s orthogonalised in place by modified Gram-Schmidt
    (P(0,s) = w_s.w_0; w_s -= P(j,s)/P(j,j) w_j, P(j+1,s) = w_s.w_{j+1}), stop
    when P(s,s) < 1e-16 P(0,0); back substitution of P c = (w_s.b); returns
    (sum_s c_s x_s, number of old solutions used)."""
    k = len(old_solutions)
    w = [vmult(mesh, op, x) for x in old_solutions]
    P = np.zeros((k, k))
    step = 0
    while step < k:
        P[0, step] = w[step] @ w[0]
        for j in range(step):
            w[step] = w[step] + (-P[j, step] / P[j, j]) * w[j]
            P[j + 1, step] = w[step] @ w[j + 1]
        if P[step, step] < 1e-16 * P[0, 0]:
            break
        step += 1
    c = [w[s] @ rhs for s in range(step)]
    for s in range(step - 1, -1, -1):
        acc = c[s]
        for j in range(s + 1, step):
            acc -= c[j] * P[s, j]
        c[s] = acc / P[s, s]
    x = np.zeros_like(rhs)
    for s in range(step):
        x = x + c[s] * old_solutions[s]
    return x, step


# ------------------------------------------------------------- mapped meshes

def _cell_corners(vert, nc, ix, iy, iz):
    V = vert.reshape(nc[2] + 1, nc[1] + 1, nc[0] + 1, 3)
    return np.array([V[iz + (v >> 2 & 1), iy + (v >> 1 & 1), ix + (v & 1)] for v in range(8)])


class MappedMesh:
    """Unstructured hexahedral mesh in the ingestion form (orc_mapped): each
    cell's 8 corners (x fastest), its n^3 global DoFs (lexicographic within the
    cell), homogeneous constraints {dof: [(master, weight), ...]}, and optionally
    the boundary id of each cell's local face 2 d + s (`face_ids`, shape
    (n_cells, 6), -1 interior; id b is selected by bit b of robin_faces /
    rad_faces)."""

    def __init__(self, degree, cell_vertices, cell_dofs, n_dofs, constraints=None, face_ids=None):
        self.degree = int(degree)
        n = degree + 1
        self.cell_vertices = np.ascontiguousarray(cell_vertices, np.float64).reshape(-1, 8, 3)
        self.cell_dofs = np.ascontiguousarray(cell_dofs, np.int64).reshape(-1, n ** 3)
        self.n_cells = self.cell_dofs.shape[0]
        self.n_dofs = int(n_dofs)
        self.constraints = dict(constraints or {})
        ptr = np.zeros(self.n_dofs + 1, np.int64)
        idx, w = [], []
        for g in range(self.n_dofs):
            ent = self.constraints.get(g, [])
            ptr[g + 1] = ptr[g] + len(ent)
            idx += [m for m, _ in ent]
            w += [x for _, x in ent]
        self.cons_ptr = ptr
        self.cons_idx = np.ascontiguousarray(idx if idx else [0], np.int64)
        self.cons_w = np.ascontiguousarray(w if w else [0.0], np.float64)
        self.face_ids = None if face_ids is None else np.ascontiguousarray(face_ids, np.int8).reshape(-1, 6)
        self._c = _Mapped(self.degree, self.n_cells, self.n_dofs, _ptr(self.cell_vertices),
                          self.cell_dofs.ctypes.data_as(_lp), ptr.ctypes.data_as(_lp),
                          self.cons_idx.ctypes.data_as(_lp), _ptr(self.cons_w),
                          None if self.face_ids is None else self.face_ids.ctypes.data_as(C.POINTER(C.c_int8)))

    def constrained_mask(self):
        m = np.zeros(self.n_dofs, np.uint8)
        m[list(self.constraints)] = 1
        return m


def mapped_from_mesh(mesh, perm=None, cell_order=None):
    """The structured 3D mesh `mesh` in the ingestion form; `perm[g]` renumbers
    DoF g, `cell_order` lists the cells (lexicographic index) in the order given;
    the box faces carry boundary ids 2 d + s (as the lattice's robin_faces bits)."""
    p, nc = mesh.degree, mesh.nc
    n = p + 1
    NX, NY = mesh.shape[0], mesh.shape[1]
    cells = list(cell_order) if cell_order is not None else range(nc[0] * nc[1] * nc[2])
    verts, dofs, fids = [], [], []
    for c in cells:
        ix, iy, iz = c % nc[0], (c // nc[0]) % nc[1], c // (nc[0] * nc[1])
        verts.append(_cell_corners(mesh.vert, nc, ix, iy, iz))
        ic = (ix, iy, iz)
        fids.append([2 * d + s if ic[d] == (nc[d] - 1 if s else 0) else -1 for d in range(3) for s in range(2)])
        k, j, i = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
        g = ((iz * p + k) * NY + (iy * p + j)) * NX + (ix * p + i)
        g = g.reshape(-1)
        dofs.append(g if perm is None else np.asarray(perm)[g])
    return MappedMesh(p, np.array(verts), np.array(dofs), mesh.n_dofs, face_ids=np.array(fids, np.int8))


def mapped_from_mesh2(m2):
    """The two-level mesh `m2` in the ingestion form: its cells (coarse, then
    fine), its DoF numbering, and the hanging constraints of the fine DoFs on
    the interface plane (weights: the coarse face's Lagrange basis at the fine
    node, hanging_matrix)."""
    p = m2.degree
    n = p + 1
    mc = mapped_from_mesh(m2.coarse)
    mf = mapped_from_mesh(m2.fine)
    P = hanging_matrix(p)
    NXc, NYc = m2.coarse.shape[0], m2.coarse.shape[1]
    NXf, NYf, NZf = m2.fine.shape
    ncf = m2.fine.nc
    cons = {}
    for Zf in range(NZf):
        for Yf in range(NYf):
            iy, iz = min(Yf // p, ncf[1] - 1), min(Zf // p, ncf[2] - 1)
            j, k = Yf - iy * p, Zf - iz * p
            sy, cy, sz, cz = iy % 2, iy // 2, iz % 2, iz // 2
            ent = []
            for kp in range(n):
                for jp in range(n):
                    w = P[sy, j, jp] * P[sz, k, kp]
                    if abs(w) > 1e-14:
                        ent.append((((cz * p + kp) * NYc + (cy * p + jp)) * NXc + (NXc - 1), float(w)))
            cons[m2.n_coarse + (Zf * NYf + Yf) * NXf] = ent
    return MappedMesh(p, np.concatenate([mc.cell_vertices, mf.cell_vertices]),
                      np.concatenate([mc.cell_dofs, mf.cell_dofs + m2.n_coarse]), m2.n_dofs, cons)


def mapped_vmult(mm, op, src):
    src = np.ascontiguousarray(src, np.float64)
    dst = np.zeros(mm.n_dofs)
    lib().orcm_vmult(C.byref(mm._c), C.byref(op._c), _ptr(dst), _ptr(src))
    return dst


def mapped_diagonal(mm, op):
    d = np.zeros(mm.n_dofs)
    lib().orcm_diagonal(C.byref(mm._c), C.byref(op._c), _ptr(d))
    return d
