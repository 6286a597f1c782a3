"""Time-step drivers around the operators: the callers of the hot path, restated
from MeltPoolDG's operation classes.

* AdvectionDiffusionOperation.solve follows
  source/level_set/advection_diffusion_operation.cpp:227-367 (matrix-free branch):
  Dirichlet lifting rhs = create_rhs(phi_old) - A_noBC x_D with constrained rows
  zeroed (include/meltpooldg/linear_algebra/utilities_matrixfree.hpp:39-101),
  Jacobi update, Krylov solve, distribute constraints.
* HeatDiffuseOperation.solve follows source/heat/heat_diffuse_operation.cpp:261-289
  with NewtonRaphsonSolver::solve (source/linear_algebra/newton_raphson_solver.cpp:24-80):
  residual -> linear solve -> convergence test on |r| and |dx| -> update.

The per-step bookkeeping on vectors (negation, masking) is torch glue; every
operator apply, diagonal, residual and Krylov iteration runs in libmpdg.
"""
from __future__ import annotations

import numpy as np
import torch

from .operators import (AdvectionDiffusionOperator, HeatDiffuseOperator, LinearSolver,
                        LinearSolverData)


class AdvectionDiffusionOperation:
    """`inflow_outflow` = (mask, values): DoFs fixed to values after each solve
    through identity rows of the operator instead of Dirichlet constraints
    (create_inflow_outflow_constraints and solve,
    advection_diffusion_operation.cpp:227-294, 371-499).  `supg`,
    `supg_coefficient`: the "convection stabilization" settings
    (AdvectionDiffusionData::conv_stab)."""

    def __init__(self, mesh, dt, theta=0.5, diffusivity=0.0, velocity=None, dirichlet_values=None,
                 linear_solver: LinearSolverData = None, device="cuda", inflow_outflow=None, supg=False,
                 supg_coefficient=-1.0, velocity_field=None):
        self.mesh = mesh
        self.op = AdvectionDiffusionOperator(mesh, dt, theta=theta, diffusivity=diffusivity,
                                             velocity="nodal" if velocity_field is not None else velocity,
                                             supg=supg, supg_coefficient=supg_coefficient)
        if velocity_field is not None:
            # the velocity as a DoF vector (3 n_dofs, component-major), e.g. the flow solver's
            self.velocity = torch.tensor(np.asarray(velocity_field, np.float64).reshape(-1), device=device)
            self.op.set_velocity(self.velocity)
        self.io = None
        if inflow_outflow is not None:
            io_mask, io_vals = inflow_outflow
            io_mask = np.asarray(io_mask, np.uint8)
            self.io = (torch.tensor(io_mask.astype(bool), device=device),
                       torch.tensor(np.where(io_mask == 1, np.asarray(io_vals, np.float64), 0.0), device=device))
        self.data = linear_solver or LinearSolverData(solver_type="GMRES", preconditioner_type="Diagonal")
        self.device = device
        N = mesh.n_dofs
        mask = mesh.mask if mesh.mask is not None else np.zeros(N, np.uint8)
        self.mask = torch.tensor(mask.astype(bool), device=device)
        vals = np.zeros(N) if dirichlet_values is None else np.asarray(dirichlet_values, np.float64)
        self.bc_values = torch.tensor(np.where(mask == 1, vals, 0.0), device=device)
        self.solution = torch.zeros(N, dtype=torch.float64, device=device)
        self.iterations = []

    def set_initial_condition(self, values):
        """VectorTools::interpolate + constraints.distribute
        (advection_diffusion_operation.cpp:76-94)."""
        s = torch.tensor(np.asarray(values, np.float64), device=self.device)
        s[self.mask] = self.bc_values[self.mask]
        self.solution = s

    def solve(self):
        op = self.op
        old = self.solution.clone()
        rhs = torch.empty_like(old)
        bc = self.bc_values
        if self.io is not None:
            # the lifting includes the inflow values; the identity rows are off
            # while it is computed (utilities_matrixfree.hpp:39-101)
            bc = bc.clone()
            bc[self.io[0]] = self.io[1][self.io[0]]
            op.set_inflow_outflow(None)
        op.reset_dof_index(with_dirichlet=False)
        op.vmult(rhs, bc)
        rhs.neg_()
        op.create_rhs(rhs, old)
        op.reset_dof_index(with_dirichlet=True)
        rhs[self.mask] = 0.0
        if self.io is not None:
            rhs[self.io[0]] = 0.0
            op.set_inflow_outflow(self.io[0].cpu().numpy().astype(np.uint8))
        x = old.clone()
        it = LinearSolver.solve(op, x, rhs, self.data)
        self.iterations.append(it)
        x[self.mask] = self.bc_values[self.mask]
        if self.io is not None:
            x[self.io[0]] = self.io[1][self.io[0]]
        self.solution = x
        return x

    def l2_norm(self):
        return self.op.l2_norm(self.solution)


class HeatDiffuseOperation:
    """One heat time step with Newton-Raphson (HeatDiffuseOperation::solve,
    source/heat/heat_diffuse_operation.cpp; newton_raphson_solver.cpp:24-80).
    `heaviside(t)` returns the nodal level-set heaviside at time t for the
    two-phase laws (re-interpolated before every step,
    heat_transfer_application.cpp:67-70)."""

    def __init__(self, mesh, dt, rho_cp=1.0, k0=1.0, k_alpha=0.0, full_tangent=False,
                 linear_solver: LinearSolverData = None, residual_tolerance=1e-9,
                 field_correction_tolerance=1e-10, max_nonlinear_iterations=10, device="cuda",
                 robin_alpha=0.0, robin_t_inf=0.0, robin_faces=(), rad_emissivity=0.0, rad_t_inf=0.0,
                 rad_faces=(), velocity=None, material=None, heaviside=None, velocity_field=None):
        self.mesh = mesh
        self.op = HeatDiffuseOperator(mesh, dt, rho_cp=rho_cp, k0=k0, k_alpha=k_alpha,
                                      full_tangent=full_tangent, robin_alpha=robin_alpha,
                                      robin_t_inf=robin_t_inf, robin_faces=robin_faces,
                                      rad_emissivity=rad_emissivity, rad_t_inf=rad_t_inf, rad_faces=rad_faces,
                                      velocity="nodal" if velocity_field is not None else velocity,
                                      material=material)
        if velocity_field is not None:
            # the velocity as a DoF vector (3 n_dofs, component-major), e.g. the flow solver's
            self.velocity = torch.tensor(np.asarray(velocity_field, np.float64).reshape(-1), device=device)
            self.op.set_velocity(self.velocity)
        self.dt = dt
        self.time = 0.0
        self.heaviside = heaviside
        self.H = None
        self.data = linear_solver or LinearSolverData(solver_type="GMRES", preconditioner_type="Diagonal")
        self.res_tol = residual_tolerance
        self.dx_tol = field_correction_tolerance
        self.max_nl = max_nonlinear_iterations
        self.device = device
        N = mesh.n_dofs
        self.temperature = torch.zeros(N, dtype=torch.float64, device=device)
        self.op.set_temperature(self.temperature)
        self.newton_iterations = []
        self.linear_iterations = []

    def set_initial_condition(self, values):
        self.temperature.copy_(torch.tensor(np.asarray(values, np.float64), device=self.device))

    def solve(self):
        T = self.temperature
        self.time += self.dt
        if self.heaviside is not None:
            self.H = torch.tensor(np.asarray(self.heaviside(self.time), np.float64), device=self.device)
            self.op.set_heaviside(self.H)
        self.op.set_temperature(T)
        T_old = T.clone()
        self.op.set_temperature_old(T_old)
        rhs = torch.empty_like(T)
        dx = torch.empty_like(T)
        for i in range(self.max_nl):
            rhs.zero_()
            self.op.create_rhs(rhs, T_old)
            dx.zero_()
            it = LinearSolver.solve(self.op, dx, rhs, self.data)
            self.linear_iterations.append(it)
            if float(torch.linalg.vector_norm(rhs)) < self.res_tol and \
                    float(torch.linalg.vector_norm(dx)) < self.dx_tol:
                self.newton_iterations.append(i)
                return T
            T.add_(dx)
            self.op.set_temperature(T)  # the operator linearises about the updated T
        raise RuntimeError("Newton-Raphson did not converge (ExcNewtonDidNotConverge)")

    def l2_norm(self):
        return self.op.l2_norm(self.temperature)
