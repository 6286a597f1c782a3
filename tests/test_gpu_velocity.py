"""Velocity given as a DoF vector (MPDG_VEL_NODAL, MPDG_FIELD_VELOCITY): the
coupling path of the reference, whose operators read the flow solver's
velocity with read_dof_values_plain (heat_diffuse_operator.cpp:975-980,
1038-1041; advection_diffusion_operator.cpp:461-465, 477-480).  Checked
against the oracle's nodal velocity (ORC_VEL_NODAL): vmult (FP64 to 1e-12,
FP32 to 2e-5), the diagonal and create_rhs, on uniform and perturbed cells and
a mapped mesh with renumbered DoFs; SUPG with tau_K from the field; a constant
field equals the prescribed constant velocity; and the reference's
unidirectional_heat_transfer_with_velocity golden with the velocity given as
a vector."""
import json
import os

import numpy as np
import pytest

from gpu_helpers import dev, meshes, relerr, rng
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-5
GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_outputs.json")))


def _field(om, seed):
    """A smooth velocity field at the DoFs plus noise (3 n_dofs, component-major)."""
    x = om.dof_coordinates()
    R = rng(seed)
    U = np.stack([np.sin(2.0 * x[:, 1]) + 0.3, np.cos(1.5 * x[:, 0]) * x[:, 2], x[:, 0] - 0.5 * x[:, 1]])
    return (U + 0.05 * R.uniform(-1, 1, U.shape)).reshape(-1)


@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("perturb", [0.0, 0.1])
@pytest.mark.parametrize("kind", ["heat", "advdiff"])
def test_nodal_velocity_parity(cuda, p, perturb, kind):
    import torch
    import meltpooldg_b200 as M
    nc = (4, 5, 3)
    mask = M.boundary_mask(nc, p, faces=[(0, 0), (2, 1)])
    gm, om = meshes(nc, p, perturb, seed=8, mask=mask)
    U = _field(om, 30 + p)
    if kind == "heat":
        op = M.HeatDiffuseOperator(gm, 1e-3, rho_cp=2.0, k0=1.5, velocity="nodal", precisions=("fp64", "fp32"))
        oop = O.Operator(O.HEAT, 1e-3, rho_cp=2.0, k0=1.5, vel_kind=O.VEL_NODAL, vel_nodal=U, dirichlet=mask)
    else:
        op = M.AdvectionDiffusionOperator(gm, 1e-3, theta=0.5, diffusivity=1e-2, velocity="nodal",
                                          precisions=("fp64", "fp32"))
        oop = O.Operator(O.ADVDIFF, 1e-3, theta=0.5, diffusivity=1e-2, vel_kind=O.VEL_NODAL, vel_nodal=U,
                         dirichlet=mask)
    src = rng(p).uniform(-1, 1, gm.n_dofs)
    x = torch.empty(gm.n_dofs, dtype=torch.float64, device="cuda")
    with pytest.raises(M.MpdgError, match="velocity"):
        op.vmult(x, dev(src))  # no field yet
    op.set_velocity(dev(U))
    op.vmult(x, dev(src))
    ref = O.vmult(om, oop, src)
    assert relerr(x.cpu().numpy(), ref) < TOL64
    x32 = torch.empty(gm.n_dofs, dtype=torch.float32, device="cuda")
    op.vmult(x32, dev(src, torch.float32))
    assert relerr(x32.double().cpu().numpy(), ref) < TOL32
    d = torch.empty_like(x)
    op.compute_diagonal(d)
    assert relerr(d.cpu().numpy(), O.diagonal(om, oop)) < TOL64
    rhs = torch.zeros_like(x)
    if kind == "heat":
        T = rng(5).uniform(0.0, 1.0, gm.n_dofs)
        T_old = T - 0.01 * rng(6).uniform(-1, 1, gm.n_dofs)
        op.set_temperature(dev(T))
        op.create_rhs(rhs, dev(T_old))
        want = O.rhs_heat(om, oop.with_temperature(T), T_old, scatter_mask=mask)
    else:
        # Dirichlet rows selected: constrained DoFs are not written
        op.create_rhs(rhs, dev(src))
        want = O.rhs_advdiff(om, oop, src, scatter_mask=mask)
    assert relerr(rhs.cpu().numpy(), want) < TOL64
    # a new field value takes effect when set again
    op.set_velocity(dev(2.0 * U))
    op.vmult(x, dev(src))
    assert relerr(x.cpu().numpy(), O.vmult(om, oop.with_fields(vel_nodal=2.0 * U), src)) < TOL64


def test_constant_field_equals_prescribed_velocity(cuda):
    import torch
    import meltpooldg_b200 as M
    nc, p = (5, 4, 4), 3
    gm, om = meshes(nc, p, 0.1, seed=3)
    vel = (0.4, -0.7, 0.25)
    U = np.concatenate([np.full(gm.n_dofs, v) for v in vel])
    a = M.AdvectionDiffusionOperator(gm, 1e-3, theta=0.5, diffusivity=1e-3, velocity=vel)
    b = M.AdvectionDiffusionOperator(gm, 1e-3, theta=0.5, diffusivity=1e-3, velocity="nodal")
    b.set_velocity(dev(U))
    src = dev(rng(2).uniform(-1, 1, gm.n_dofs))
    ya, yb = torch.empty_like(src), torch.empty_like(src)
    a.vmult(ya, src)
    b.vmult(yb, src)
    assert float((ya - yb).abs().max() / ya.abs().max()) < 1e-13


@pytest.mark.parametrize("p", [2, 4])
def test_nodal_velocity_supg(cuda, p):
    """SUPG (D = 0) with tau_K = h_K / max_q |u| from the field's values at the
    Gauss points, on perturbed cells."""
    import torch
    import meltpooldg_b200 as M
    nc = (4, 4, 3)
    gm, om = meshes(nc, p, 0.1, seed=12)
    U = _field(om, 44)
    op = M.AdvectionDiffusionOperator(gm, 1e-2, theta=0.5, diffusivity=0.0, velocity="nodal", supg=True,
                                      supg_coefficient=-1.0)
    op.set_velocity(dev(U))
    oop = O.Operator(O.ADVDIFF, 1e-2, theta=0.5, diffusivity=0.0, vel_kind=O.VEL_NODAL, vel_nodal=U, supg=True,
                     supg_coefficient=-1.0)
    src = rng(9).uniform(-1, 1, gm.n_dofs)
    y = torch.empty(gm.n_dofs, dtype=torch.float64, device="cuda")
    op.vmult(y, dev(src))
    assert relerr(y.cpu().numpy(), O.vmult(om, oop, src)) < TOL64


def test_nodal_velocity_on_a_mapped_mesh(cuda):
    """The same operator through a mapped mesh with renumbered DoFs: the field
    is read through the cell->DoF map."""
    import torch
    import meltpooldg_b200 as M
    nc, p = (4, 3, 5), 2
    gm, om = meshes(nc, p, 0.1, seed=21)
    perm = rng(4).permutation(om.n_dofs)
    mm = O.mapped_from_mesh(om, perm=perm)
    gmm = M.MappedMesh(mm.cell_vertices, mm.cell_dofs, mm.n_dofs, mm.degree)
    U = _field(om, 50).reshape(3, -1)
    Up = np.zeros_like(U)
    Up[:, perm] = U
    a = M.HeatDiffuseOperator(gm, 1e-2, rho_cp=2.0, k0=1.5, velocity="nodal")
    b = M.HeatDiffuseOperator(gmm, 1e-2, rho_cp=2.0, k0=1.5, velocity="nodal")
    a.set_velocity(dev(U.reshape(-1)))
    b.set_velocity(dev(Up.reshape(-1)))
    src = rng(3).uniform(-1, 1, om.n_dofs)
    srcp = np.zeros_like(src)
    srcp[perm] = src
    ya = torch.empty(om.n_dofs, dtype=torch.float64, device="cuda")
    yb = torch.empty_like(ya)
    a.vmult(ya, dev(src))
    b.vmult(yb, dev(srcp))
    ref = O.vmult(om, O.Operator(O.HEAT, 1e-2, rho_cp=2.0, k0=1.5, vel_kind=O.VEL_NODAL, vel_nodal=U.reshape(-1)),
                  src)
    assert relerr(ya.cpu().numpy(), ref) < TOL64
    assert relerr(yb.cpu().numpy()[perm], ref) < TOL64


def test_velocity_golden_with_the_velocity_as_a_vector(cuda):
    """unidirectional_heat_transfer_with_velocity (2D Q1 32^2, extruded to one
    layer of unit depth) with the velocity (-v, 0, 0) handed over as a DoF
    vector instead of a constant: all printed values match."""
    import meltpooldg_b200 as M
    from meltpooldg_b200.operations import HeatDiffuseOperation
    from oracle import cases
    name = "unidirectional_heat_transfer_with_velocity"
    c = dict(cases.HEAT_CASES[name])
    nc = (32, 32, 1)
    V = M.box_vertices(nc, (0.0, 0.0, 0.0), (0.1, 0.1, 1.0))
    mesh = M.Mesh(V, nc, 1)
    N = mesh.n_dofs
    U = np.concatenate([np.full(N, -c["velocity"]), np.zeros(N), np.zeros(N)])
    opn = HeatDiffuseOperation(mesh, c["dt"], residual_tolerance=c.get("residual_tolerance", 5e-9),
                               linear_solver=M.LinearSolverData(rel_tolerance=1e-12),
                               rho_cp=c["rho"] * c["cp"], k0=c["k"], robin_alpha=c["convection"],
                               robin_t_inf=300.0, robin_faces=[(0, 1)], rad_emissivity=c["emissivity"],
                               rad_t_inf=300.0, rad_faces=[(0, 1)], velocity_field=U)
    opn.set_initial_condition(np.full(N, 1000.0))
    for printed in GOLDEN[name]["printed"]:
        opn.solve()
        assert cases.printed_match(opn.l2_norm(), printed), (opn.l2_norm(), printed)
