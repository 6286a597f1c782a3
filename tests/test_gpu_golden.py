"""The reference's golden integration cases driven through the CUDA path."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_outputs.json")))


def test_vortex_3d_golden_on_gpu(cuda):
    """advection_diffusion_vortex_mf_3d: Q1, 8^3 cells on [-1,1]^3, CN, GMRES + Diagonal."""
    import meltpooldg_b200 as M
    from meltpooldg_b200.operations import AdvectionDiffusionOperation
    from oracle import cases
    om, phi0, mask = cases.vortex_setup(3, 3)
    mesh = M.Mesh(om.vert, (8, 8, 8), 1, mask)
    opn = AdvectionDiffusionOperation(mesh, 0.01, theta=0.5, diffusivity=0.0,
                                      velocity=("rotation", 4.0),
                                      dirichlet_values=np.full(mesh.n_dofs, -1.0))
    opn.set_initial_condition(phi0)
    ref = GOLDEN["advection_diffusion_vortex_mf_3d"]["values"]
    for r in ref:
        opn.solve()
        assert abs(opn.l2_norm() - r) / r < 5e-8


def test_unidirectional_heat_golden_on_gpu(cuda):
    """unidirectional_heat_transfer (2D, Q1, 32^2) extruded to one layer of
    hexahedra of unit depth: the solution is z-independent, so the 3D L2 norm
    equals the 2D one."""
    import meltpooldg_b200 as M
    from meltpooldg_b200.operations import HeatDiffuseOperation
    nc = (32, 32, 1)
    V = M.box_vertices(nc, (0.0, 0.0, 0.0), (0.1, 0.1, 1.0))
    mesh = M.Mesh(V, nc, 1)
    opn = HeatDiffuseOperation(mesh, 1e-4, rho_cp=1.0, k0=1.0, residual_tolerance=5e-9,
                               linear_solver=M.LinearSolverData(rel_tolerance=1e-12))
    X = np.tile(np.linspace(0.0, 0.1, 33), 33 * 2)
    opn.set_initial_condition(X)
    got = []
    for _ in range(5):
        opn.solve()
        got.append("%.5e" % opn.l2_norm())
    assert got == GOLDEN["unidirectional_heat_transfer"]["printed"]


def test_unidirectional_heat_convection_golden_on_gpu(cuda):
    """unidirectional_heat_transfer_with_convection (2D Q1 32^2, Robin face at
    x = 0.1 with alpha = 25, T_inf = 300, steel properties, dt = 0.01) extruded
    to one layer of unit depth: the Robin face terms run on the device."""
    import meltpooldg_b200 as M
    from meltpooldg_b200.operations import HeatDiffuseOperation
    nc = (32, 32, 1)
    V = M.box_vertices(nc, (0.0, 0.0, 0.0), (0.1, 0.1, 1.0))
    mesh = M.Mesh(V, nc, 1)
    opn = HeatDiffuseOperation(mesh, 0.01, rho_cp=7850.0 * 460.0, k0=55.563, residual_tolerance=5e-9,
                               linear_solver=M.LinearSolverData(rel_tolerance=1e-12),
                               robin_alpha=25.0, robin_t_inf=300.0, robin_faces=[(0, 1)])
    opn.set_initial_condition(np.full(mesh.n_dofs, 1000.0))
    got = []
    for _ in range(5):
        opn.solve()
        got.append("%.5e" % opn.l2_norm())
    assert got == GOLDEN["unidirectional_heat_transfer_with_convection"]["printed"]


@pytest.mark.parametrize("name", ["advection_diffusion_vortex_mf_inflow_outflow_3d"])
def test_vortex_inflow_outflow_golden_on_gpu(cuda, name):
    """advection_diffusion_vortex_mf_inflow_outflow_3d: the u . n <= 0 boundary
    DoFs carry identity rows in the operator (mpdg_op_set_inflow_outflow) and are
    set to -1 after each solve; no Dirichlet constraints."""
    import meltpooldg_b200 as M
    from meltpooldg_b200.operations import AdvectionDiffusionOperation
    from oracle import cases
    om, phi0, _ = cases.vortex_setup(3, 3)
    io = cases.vortex_io_mask(om, 4.0)
    mesh = M.Mesh(om.vert, (8, 8, 8), 1, None)
    opn = AdvectionDiffusionOperation(mesh, 0.01, theta=0.5, diffusivity=0.0, velocity=("rotation", 4.0),
                                      inflow_outflow=(io, np.full(mesh.n_dofs, -1.0)))
    opn.set_initial_condition(phi0)
    for r in GOLDEN[name]["values"]:
        opn.solve()
        assert abs(opn.l2_norm() - r) / r < 5e-8
