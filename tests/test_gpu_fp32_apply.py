"""The FP32 form of the apply against the oracle (2e-5) on meshes whose colour
counts leave the warps' last cell groups partly empty (including single-cell
and one-layer meshes), with Dirichlet masks, every degree, k(T) on general
geometry, and the analytic velocities on uniform meshes and on general
geometry."""
import numpy as np
import pytest

from gpu_helpers import dev, meshes, relerr, rng
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL32 = 2e-5


@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("nc", [(5, 3, 7), (1, 1, 1), (2, 3, 1), (9, 4, 3)])
@pytest.mark.parametrize("perturb", [0.0, 0.1])
def test_fp32_heat_apply(cuda, p, nc, perturb):
    import torch
    import meltpooldg_b200 as M
    mask = M.boundary_mask(nc, p, faces=[(0, 0), (2, 1)])
    gm, om = meshes(nc, p, perturb, seed=p, mask=mask)
    T = rng(p).uniform(300, 3000, gm.n_dofs)
    op = M.HeatDiffuseOperator(gm, 1e-3, rho_cp=2.0, k0=1.5, k_alpha=1e-3 if perturb else 0.0,
                               precisions=("fp64", "fp32"))
    op.set_temperature(dev(T))
    oop = O.Operator(O.HEAT, 1e-3, rho_cp=2.0, k0=1.5, k_alpha=1e-3 if perturb else 0.0, temperature=T,
                     dirichlet=mask)
    src = rng(10 + p).uniform(-1, 1, gm.n_dofs)
    d32 = torch.empty(gm.n_dofs, dtype=torch.float32, device="cuda")
    op.vmult(d32, dev(src, torch.float32))
    assert relerr(d32.double().cpu().numpy(), O.vmult(om, oop, src)) < TOL32


@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("vel,okind,oparam", [("vortex", O.VEL_VORTEX, (0, 0, 0)),
                                              (("rotation", 4.0), O.VEL_ROTATION, (4.0, 0, 0)),
                                              ((0.3, -0.7, 1.1), O.VEL_CONST, (0.3, -0.7, 1.1))])
def test_fp32_advdiff_uniform_apply(cuda, p, vel, okind, oparam):
    import torch
    import meltpooldg_b200 as M
    nc = (5, 4, 3)
    mask = M.boundary_mask(nc, p, faces=[(1, 0)])
    gm, om = meshes(nc, p, 0.0, seed=1, mask=mask, lo=(-1, -1, -1), hi=(1, 1, 1))
    op = M.AdvectionDiffusionOperator(gm, 1e-3, theta=0.5, diffusivity=1e-3, velocity=vel,
                                      precisions=("fp64", "fp32"))
    oop = O.Operator(O.ADVDIFF, 1e-3, theta=0.5, diffusivity=1e-3, vel_kind=okind, vel_param=oparam,
                     dirichlet=mask)
    src = rng(20 + p).uniform(-1, 1, gm.n_dofs)
    d32 = torch.empty(gm.n_dofs, dtype=torch.float32, device="cuda")
    op.vmult(d32, dev(src, torch.float32))
    assert relerr(d32.double().cpu().numpy(), O.vmult(om, oop, src)) < TOL32


@pytest.mark.parametrize("p", [2, 4])
def test_fp32_general_with_velocity(cuda, p):
    import torch
    import meltpooldg_b200 as M
    nc = (4, 3, 5)
    gm, om = meshes(nc, p, 0.1, seed=3, lo=(-1, -1, -1), hi=(1, 1, 1))
    op = M.AdvectionDiffusionOperator(gm, 1e-3, theta=0.5, diffusivity=1e-3, velocity="vortex",
                                      precisions=("fp64", "fp32"))
    oop = O.Operator(O.ADVDIFF, 1e-3, theta=0.5, diffusivity=1e-3, vel_kind=O.VEL_VORTEX)
    src = rng(30 + p).uniform(-1, 1, gm.n_dofs)
    d32 = torch.empty(gm.n_dofs, dtype=torch.float32, device="cuda")
    op.vmult(d32, dev(src, torch.float32))
    assert relerr(d32.double().cpu().numpy(), O.vmult(om, oop, src)) < TOL32
