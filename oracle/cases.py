"""Replays of the reference's golden integration cases with the CPU oracle
(TEST INFRASTRUCTURE ONLY).

Each driver rebuilds a reference application case from its parameter file and
case source and returns the quantity the reference prints per time step, so
that the oracle can be pinned against the committed .output digits:

* advection_diffusion_vortex (applications/mp-advec-diff/cases/advection_diffusion_vortex.hpp):
  domain [-1,1]^dim refined `refinements` times, FE_Q(1); tanh level set
  around a sphere of radius 0.25 (:33-73); rotating velocity s*(y,-x) with
  s = 4 (:75-100, :291); inflow faces selected by face centre (:170-193) with
  Dirichlet value -1 (:158); Crank-Nicolson (theta = 0.5), D = 0, dt = 0.01,
  GMRES + Diagonal at rel. tol. 1e-12 (advection_diffusion_data.cpp:11-12,
  linear_solver_data.hpp:38-51); the per-step solve follows
  source/level_set/advection_diffusion_operation.cpp:227-367 with the
  Dirichlet lifting of include/meltpooldg/linear_algebra/utilities_matrixfree.hpp:39-101;
  printed value: the integrated L2 norm of the advected field (:331-342).
* unidirectional_heat_transfer
  (applications/mp-heat-transfer/cases/unidirectional_heat_transfer/unidirectional_heat_transfer.cpp):
  [0,0.1]^2 refined 5 times, FE_Q(1), T0 = x (LinearTemp(0, 0.1), :27-47),
  single-phase material, Newton-Raphson (source/linear_algebra/newton_raphson_solver.cpp:24-80)
  with GMRES + Diagonal (heat_data.cpp:11-12); optional convective (Robin)
  boundary on the right face (:217-221) with T0 = 1000 (:233-236); printed
  value: integrated L2 norm of T after Newton convergence.
"""
from __future__ import annotations

import numpy as np

from . import oracle as O


def vortex_inflow_mask(mesh: O.Mesh, lo=-1.0, hi=1.0):
    """DoFs on faces whose centre satisfies the inflow rule of
    advection_diffusion_vortex.hpp:170-193."""
    dim, p = mesh.dim, mesh.degree
    coords = mesh.vert
    nc = mesh.nc
    nv = [nc[d] + 1 for d in range(dim)]
    gi = mesh.grid_index()
    mask = np.zeros(mesh.n_dofs, dtype=bool)
    half = 0.5 * (lo + hi)

    def vid(c):
        v = 0
        for d in reversed(range(dim)):
            v = v * nv[d] + c[d]
        return v

    for d in range(dim):
        for s in (0, 1):
            # enumerate boundary faces orthogonal to d on side s
            tang = [t for t in range(dim) if t != d]
            ranges = [range(nc[t]) for t in tang]
            for cell_t in np.ndindex(*[len(r) for r in ranges]):
                corners = []
                for off in np.ndindex(*([2] * len(tang))):
                    c = [0] * dim
                    c[d] = 0 if s == 0 else nc[d]
                    for a, t in enumerate(tang):
                        c[t] = cell_t[a] + off[a]
                    corners.append(coords[vid(c)])
                centre = np.mean(corners, axis=0)
                inflow = ((centre[0] == lo and centre[dim - 1] >= half)
                          or (centre[0] == hi and centre[dim - 1] <= half)
                          or (centre[dim - 1] == hi and centre[0] >= half)
                          or (centre[dim - 1] == lo and centre[0] <= half))
                if not inflow:
                    continue
                sel = gi[:, d] == (0 if s == 0 else mesh.shape[d] - 1)
                for a, t in enumerate(tang):
                    sel &= (gi[:, t] >= cell_t[a] * p) & (gi[:, t] <= (cell_t[a] + 1) * p)
                mask |= sel
    return mask.astype(np.uint8)


def vortex_io_mask(mesh: O.Mesh, velocity_scale=4.0):
    """Inflow/outflow constraint set of advection_diffusion_operation.cpp:371-499
    for the vortex case with "inflow outflow bc" (both boundary labels carry the
    condition, advection_diffusion_vortex.hpp:159-166): every DoF at a support
    point of a boundary face where u . n <= 0, u = s (y, .., -x) with y the last
    coordinate (PrescribedVelocityField, advection_diffusion_vortex.hpp:88-104)."""
    dim = mesh.dim
    x = mesh.dof_coordinates()
    gi = mesh.grid_index()
    u = np.zeros((mesh.n_dofs, dim))
    u[:, 0] = velocity_scale * x[:, dim - 1]
    u[:, dim - 1] = -velocity_scale * x[:, 0]
    mask = np.zeros(mesh.n_dofs, dtype=bool)
    for d in range(dim):
        for s, sign in ((0, -1.0), (1, 1.0)):
            on = gi[:, d] == (0 if s == 0 else mesh.shape[d] - 1)
            mask |= on & (sign * u[:, d] <= 0.0)
    return mask.astype(np.uint8)


def vortex_setup(dim, refinements, degree=1):
    n = 2 ** refinements
    mesh = O.Mesh.box(dim, degree, [n] * dim, lo=[-1.0] * dim, hi=[1.0] * dim)
    h = 2.0 / n
    eps = 0.5 * (h * np.sqrt(dim)) / np.sqrt(dim)  # 0.5 * minimal diameter / sqrt(dim)
    centre = np.zeros(dim)
    centre[dim - 1] = 0.5
    x = mesh.dof_coordinates()
    sd = 0.25 - np.linalg.norm(x - centre, axis=1)
    phi0 = np.tanh(sd / (2.0 * eps))
    mask = vortex_inflow_mask(mesh)
    return mesh, phi0, mask


def vortex_case(dim, refinements, n_steps=5, dt=0.01, velocity_scale=4.0, theta=0.5,
                diffusivity=0.0, solver=None, inflow_outflow=False, supg=False):
    """Returns the per-step integrated L2 norms.  `solver(op, rhs, x0, inv)` can
    replace the oracle GMRES (used to drive the GPU path through the same case).
    With `inflow_outflow` the constrained set is the u . n <= 0 boundary DoFs and
    the initial field keeps its values there until the first solve sets them
    (the constraint is applied after each solve,
    advection_diffusion_operation.cpp:286-294).  `supg` switches on the SUPG
    terms with the automatic parameter h_K / max |u| (coefficient -1)."""
    mesh, phi, mask = vortex_setup(dim, refinements)
    phi = phi.copy()
    if inflow_outflow:
        mask = vortex_io_mask(mesh, velocity_scale)
    else:
        phi[mask == 1] = -1.0
    op_nobc = O.Operator(O.ADVDIFF, dt, theta=theta, diffusivity=diffusivity,
                         vel_kind=O.VEL_ROTATION, vel_param=(velocity_scale, 0.0, 0.0), supg=supg)
    op = op_nobc.with_dirichlet(mask)
    bc = np.where(mask == 1, -1.0, 0.0)
    norms = []
    for _ in range(n_steps):
        temp = -O.vmult(mesh, op_nobc, bc)
        O.rhs_advdiff(mesh, op_nobc, phi, dst=temp)
        temp[mask == 1] = 0.0
        inv = O.inverse_diagonal(mesh, op)
        x, it, hist, ok = O.gmres(mesh, op, temp, x0=phi, inv_diag=inv, rel_tol=1e-12,
                                  abs_tol=1e-20)
        assert ok
        x[mask == 1] = -1.0
        norms.append(O.l2_norm(mesh, x))
        phi = x
    return norms


def smoothed_heaviside(distance, eps):
    """CharacteristicFunctions::smoothed_heaviside (utilities/characteristic_functions.hpp:18-28)."""
    d = np.asarray(distance, np.float64)
    mid = (d + eps) / (2.0 * eps) + np.sin(np.pi * d / eps) / (2.0 * np.pi)
    return np.where(d > eps, 1.0, np.where(d <= -eps, 0.0, mid))


def unidirectional_heat_case(n_steps=5, dt=1e-4, k=1.0, rho=1.0, cp=1.0, convection=0.0,
                             t_inf=300.0, refinements=5, emissivity=0.0, rad_t_inf=300.0, velocity=0.0,
                             material=None, two_phase=False, solidification=False,
                             residual_tolerance=5e-9, solver=None, mesh=None):
    """Returns the per-step integrated L2 norms of T after Newton convergence
    (newton_raphson_solver.cpp:24-80 with field_correction_tolerance 1e-10,
    nonlinear_solver_data.hpp:13-18).

    The case (unidirectional_heat_transfer.cpp): [0,0.1]^2, convective and
    radiative faces at x = 0.1 (:196-209); T0 = LinearTemp(1960, 1980) with
    solidification, 1000 with a convective or radiative face, else
    LinearTemp(0, 0.1) (:213-227); velocity (-v, 0) (:51-67); with two phases
    the heaviside of the level set 0.05 - y (:73-90), or with solidification
    the covected 0.2/3 - x - v t (:98-116), both with eps = 0.01, interpolated
    at the nodes at the new time each step (heat_transfer_application.cpp:67-70).
    `material` is an oracle phase-law dict; None is the single-phase (k, rho, cp).
    `solver(op, rhs, T_old)` can replace the oracle GMRES; `mesh` the default mesh."""
    n = 2 ** refinements
    mesh = mesh or O.Mesh.box(2, 1, [n, n], lo=[0.0, 0.0], hi=[0.1, 0.1])
    x = mesh.dof_coordinates()
    if solidification:
        T = 1960.0 + 20.0 * x[:, 0] / 0.1
    elif convection > 0.0 or emissivity > 0.0:
        T = np.full(mesh.n_dofs, 1000.0)
    else:
        T = x[:, 0].copy()
    faces = 1 << (2 * 0 + 1)
    kw = dict(rho_cp=rho * cp, k0=k, robin_alpha=convection, robin_t_inf=t_inf,
              robin_faces=faces if convection > 0.0 else 0, rad_emissivity=emissivity,
              rad_t_inf=rad_t_inf, rad_faces=faces if emissivity > 0.0 else 0, material=material)
    if velocity != 0.0:
        kw.update(vel_kind=O.VEL_CONST, vel_param=(-velocity, 0.0, 0.0))
    norms = []
    t = 0.0
    for _ in range(n_steps):
        t += dt
        H = None
        if two_phase:
            H = smoothed_heaviside(0.1 * 2.0 / 3.0 - x[:, 0] - velocity * t, 0.01) if solidification \
                else smoothed_heaviside(0.05 - x[:, 1], 0.01)
        T_old = T.copy()
        op = O.Operator(O.HEAT, dt, temperature=T, temperature_old=T_old, heaviside=H, **kw)
        inv = O.inverse_diagonal(mesh, op)
        for _it in range(10):
            op = op.with_temperature(T)
            rhs = O.rhs_heat(mesh, op, T_old)
            if solver is None:
                dx, _, _, ok = O.gmres(mesh, op, rhs, inv_diag=inv, rel_tol=1e-12, abs_tol=1e-20)
                assert ok
            else:
                dx = solver(op, rhs, T_old)
            if np.linalg.norm(rhs) < residual_tolerance and np.linalg.norm(dx) < 1e-10:
                break
            T = T + dx
        else:
            raise RuntimeError("Newton did not converge")
        norms.append(O.l2_norm(mesh, T))
    return norms



# Parameters of the reference's unidirectional heat-transfer test cases
# (applications/mp-heat-transfer/cases/unidirectional_heat_transfer/tests/*.json):
# material "gas" is the single phase; phase laws index (gas, liquid, solid).
_STEEL = dict(k=55.563, rho=7850.0, cp=460.0)
_GAS_LIQUID = dict(kind=O.MAT_GAS_LIQUID, rho=(3925.0, 7850.0, 0.0), cp=(230.0, 460.0, 0.0),
                   k=(27.7815, 55.563, 0.0))
_LIQUID_SOLID = dict(kind=O.MAT_LIQUID_SOLID, rho=(0.0, 7850.0, 7850.0), cp=(0.0, 460.0, 700.0),
                     k=(0.0, 55.563, 17.0), solidus=1966.0, liquidus=1974.0)
_GAS_LIQUID_SOLID = dict(kind=O.MAT_GAS_LIQUID_SOLID, rho=(3925.0, 7850.0, 7850.0), cp=(230.0, 460.0, 700.0),
                         k=(27.7815, 55.563, 17.0), solidus=1966.0, liquidus=1974.0, two_phase_sharp=True)
HEAT_CASES = {
    "unidirectional_heat_transfer_with_radiation": dict(dt=0.01, emissivity=0.98, **_STEEL),
    "unidirectional_heat_transfer_with_radiation_and_convection":
        dict(dt=0.01, emissivity=0.98, convection=25.0, **_STEEL),
    "unidirectional_heat_transfer_with_velocity":
        dict(dt=0.001, emissivity=0.98, convection=25.0, velocity=0.01, residual_tolerance=1e-6, **_STEEL),
    "unidirectional_heat_transfer_with_two_phase":
        dict(dt=0.001, emissivity=0.98, convection=25.0, velocity=0.01, residual_tolerance=1e-6,
             material=_GAS_LIQUID, two_phase=True),
    "unidirectional_heat_transfer_with_two_phase_rho_times_cp":
        dict(dt=0.001, emissivity=0.98, convection=25.0, velocity=0.01, residual_tolerance=1e-6,
             material=dict(_GAS_LIQUID, volume_specific=True), two_phase=True),
    "unidirectional_heat_transfer_with_velocity_and_solidification":
        dict(dt=0.01, velocity=0.005, residual_tolerance=1e-7, material=_LIQUID_SOLID, solidification=True),
    "unidirectional_heat_transfer_with_two_phase_and_solidification":
        dict(dt=1.0, velocity=1e-4, residual_tolerance=1e-7, material=_GAS_LIQUID_SOLID, two_phase=True,
             solidification=True),
}


def printed_match(got, printed):
    """The reference prints ||T|| with 6 digits of a norm it sums from float cell
    norms (source/utilities/vector_tools.cpp:151): a value matches when it is
    within half a unit of the last printed digit plus that float noise (5e-8)."""
    ref = float(printed)
    half = 0.5 * 10.0 ** (int(printed.lower().split("e")[1]) - 5)
    return abs(got - ref) <= half + 5e-8 * abs(ref)
