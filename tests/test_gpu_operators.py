"""Parity of the CUDA operator kernels (called through the C ABI) with the CPU
oracle on seeded inputs: FP64 to 1e-12 relative (max norm), FP32 to 2e-5."""
import numpy as np
import pytest

from gpu_helpers import dev, meshes, relerr, rng
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-5


def _heat(gm, dt=1e-3, rho_cp=1.0, k0=1.0, k_alpha=0.0, full=False, vel=None, prec=("fp64",)):
    import meltpooldg_b200 as M
    return M.HeatDiffuseOperator(gm, dt, rho_cp=rho_cp, k0=k0, k_alpha=k_alpha, full_tangent=full,
                                 velocity=vel, precisions=prec)


@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("perturb", [0.0, 0.1])
def test_heat_vmult_parity(cuda, p, perturb):
    import torch
    nc = (5, 4, 3)
    import meltpooldg_b200 as M
    mask = M.boundary_mask(nc, p)
    gm, om = meshes(nc, p, perturb, seed=2, mask=mask)
    R = rng(p)
    T = R.uniform(300, 3000, gm.n_dofs)
    src = R.uniform(-1, 1, gm.n_dofs)
    op = _heat(gm, rho_cp=2.0, k0=1.5, k_alpha=1e-3, prec=("fp64", "fp32"))
    op.set_temperature(dev(T))
    dst = torch.empty(gm.n_dofs, dtype=torch.float64, device="cuda")
    op.vmult(dst, dev(src))
    ref = O.vmult(om, O.Operator(O.HEAT, 1e-3, rho_cp=2.0, k0=1.5, k_alpha=1e-3, temperature=T,
                                 dirichlet=mask), src)
    assert relerr(dst.cpu().numpy(), ref) < TOL64
    d32 = torch.empty(gm.n_dofs, dtype=torch.float32, device="cuda")
    op.vmult(d32, dev(src, torch.float32))
    assert relerr(d32.double().cpu().numpy(), ref) < TOL32


@pytest.mark.parametrize("p", [2, 4])
def test_heat_full_tangent_and_velocity(cuda, p):
    import torch
    nc = (3, 4, 3)
    gm, om = meshes(nc, p, 0.1, seed=3)
    R = rng(11)
    T = R.uniform(300, 3000, gm.n_dofs)
    src = R.uniform(-1, 1, gm.n_dofs)
    op = _heat(gm, rho_cp=3.0, k0=2.0, k_alpha=1e-3, full=True, vel=(0.5, -1.0, 2.0))
    op.set_temperature(dev(T))
    dst = torch.empty(gm.n_dofs, dtype=torch.float64, device="cuda")
    op.vmult(dst, dev(src))
    oop = O.Operator(O.HEAT, 1e-3, rho_cp=3.0, k0=2.0, k_alpha=1e-3, full_tangent=True,
                     temperature=T, vel_kind=O.VEL_CONST, vel_param=(0.5, -1.0, 2.0))
    assert relerr(dst.cpu().numpy(), O.vmult(om, oop, src)) < TOL64
    diag = torch.empty_like(dst)
    op.compute_diagonal(diag)
    assert relerr(diag.cpu().numpy(), O.diagonal(om, oop)) < TOL64


@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("geometry", ["uniform", "general"])
def test_advdiff_vmult_parity(cuda, p, geometry):
    import torch
    import meltpooldg_b200 as M
    nc = (4, 3, 4)
    mask = M.boundary_mask(nc, p, faces=[(0, 0), (1, 1)])
    perturb = 0.1 if geometry == "general" else 0.0
    gm, om = meshes(nc, p, perturb, seed=4, mask=mask, lo=(-1, -1, -1), hi=(1, 1, 1))
    R = rng(20 + p)
    src = R.uniform(-1, 1, gm.n_dofs)
    for vel, okind, oparam in [("vortex", O.VEL_VORTEX, (0, 0, 0)),
                               (("rotation", 4.0), O.VEL_ROTATION, (4.0, 0, 0))]:
        op = M.AdvectionDiffusionOperator(gm, 1e-3, theta=0.5, diffusivity=1e-3, velocity=vel,
                                          precisions=("fp64", "fp32"))
        dst = torch.empty(gm.n_dofs, dtype=torch.float64, device="cuda")
        op.vmult(dst, dev(src))
        oop = O.Operator(O.ADVDIFF, 1e-3, theta=0.5, diffusivity=1e-3, vel_kind=okind,
                         vel_param=oparam, dirichlet=mask)
        ref = O.vmult(om, oop, src)
        assert relerr(dst.cpu().numpy(), ref) < TOL64
        d32 = torch.empty(gm.n_dofs, dtype=torch.float32, device="cuda")
        op.vmult(d32, dev(src, torch.float32))
        assert relerr(d32.double().cpu().numpy(), ref) < TOL32
        # without the Dirichlet rows (lifting form)
        op.reset_dof_index(with_dirichlet=False)
        op.vmult(dst, dev(src))
        oop2 = O.Operator(O.ADVDIFF, 1e-3, theta=0.5, diffusivity=1e-3, vel_kind=okind, vel_param=oparam)
        assert relerr(dst.cpu().numpy(), O.vmult(om, oop2, src)) < TOL64
        op.reset_dof_index(with_dirichlet=True)
        # inverse diagonal with the 1e-14 max(1,|d|) rule
        inv = torch.empty_like(dst)
        op.compute_inverse_diagonal_from_matrixfree(inv)
        assert relerr(inv.cpu().numpy(), O.inverse_diagonal(om, oop)) < TOL64
        # rhs (plain read, written everywhere)
        rhs = torch.zeros_like(dst)
        op.reset_dof_index(with_dirichlet=False)
        op.create_rhs(rhs, dev(src))
        op.reset_dof_index(with_dirichlet=True)
        assert relerr(rhs.cpu().numpy(), O.rhs_advdiff(om, oop2, src)) < TOL64


@pytest.mark.parametrize("p", [1, 2, 4])
def test_heat_diagonal_and_rhs(cuda, p):
    import torch
    import meltpooldg_b200 as M
    nc = (4, 3, 3)
    mask = M.boundary_mask(nc, p, faces=[(2, 0)])
    gm, om = meshes(nc, p, 0.1, seed=5, mask=mask)
    R = rng(30 + p)
    T = R.uniform(300, 3000, gm.n_dofs)
    T_old = R.uniform(300, 3000, gm.n_dofs)
    q = R.uniform(-5, 5, gm.n_dofs)
    op = _heat(gm, dt=1e-2, rho_cp=4.0, k0=3.0, k_alpha=1e-3)
    op.set_temperature(dev(T))
    oop = O.Operator(O.HEAT, 1e-2, rho_cp=4.0, k0=3.0, k_alpha=1e-3, temperature=T, dirichlet=mask)
    inv = torch.empty(gm.n_dofs, dtype=torch.float64, device="cuda")
    op.compute_inverse_diagonal_from_matrixfree(inv)
    assert relerr(inv.cpu().numpy(), O.inverse_diagonal(om, oop)) < TOL64
    rhs = torch.zeros_like(inv)
    op.create_rhs(rhs, dev(T_old), dev(q))
    ref = O.rhs_heat(om, oop, T_old, heat_source=q, scatter_mask=mask)
    assert relerr(rhs.cpu().numpy(), ref) < TOL64


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_heat_robin_faces(cuda, p):
    """Convective faces (heat_diffuse_operator.cpp:1088-1129) on a perturbed mesh:
    tangent, diagonal and Newton residual against the oracle, FP64 and FP32.
    Three Robin planes, one of them meeting a Dirichlet plane."""
    import torch
    import meltpooldg_b200 as M
    nc = (5, 4, 3)
    faces = [(0, 1), (1, 0), (2, 1)]
    bits = sum(1 << (2 * d + s) for d, s in faces)
    mask = M.boundary_mask(nc, p, faces=[(0, 0)])
    gm, om = meshes(nc, p, 0.1, seed=7, mask=mask)
    R = rng(50 + p)
    T = R.uniform(300, 3000, gm.n_dofs)
    T_old = R.uniform(300, 3000, gm.n_dofs)
    src = R.uniform(-1, 1, gm.n_dofs)
    op = M.HeatDiffuseOperator(gm, 1e-2, rho_cp=4.0, k0=3.0, precisions=("fp64", "fp32"),
                               robin_alpha=250.0, robin_t_inf=300.0, robin_faces=faces)
    op.set_temperature(dev(T))
    oop = O.Operator(O.HEAT, 1e-2, rho_cp=4.0, k0=3.0, temperature=T, dirichlet=mask,
                     robin_alpha=250.0, robin_t_inf=300.0, robin_faces=bits)
    dst = torch.empty(gm.n_dofs, dtype=torch.float64, device="cuda")
    op.vmult(dst, dev(src))
    ref = O.vmult(om, oop, src)
    assert relerr(dst.cpu().numpy(), ref) < TOL64
    # without the faces the result differs: the test sees the face term
    assert relerr(O.vmult(om, O.Operator(O.HEAT, 1e-2, rho_cp=4.0, k0=3.0, temperature=T,
                                         dirichlet=mask), src), ref) > 1e-6
    d32 = torch.empty(gm.n_dofs, dtype=torch.float32, device="cuda")
    op.vmult(d32, dev(src, torch.float32))
    assert relerr(d32.double().cpu().numpy(), ref) < TOL32
    inv = torch.empty(gm.n_dofs, dtype=torch.float64, device="cuda")
    op.compute_inverse_diagonal_from_matrixfree(inv)
    assert relerr(inv.cpu().numpy(), O.inverse_diagonal(om, oop)) < TOL64
    rhs = torch.zeros_like(inv)
    op.create_rhs(rhs, dev(T_old))
    ref = O.rhs_heat(om, oop, T_old, scatter_mask=mask)
    assert relerr(rhs.cpu().numpy(), ref) < TOL64


def test_inflow_outflow_identity_rows(cuda):
    """Identity rows (do_pre_vmult / do_post_vmult): src read as 0 at the
    flagged DoFs, result there equal to src; inverse diagonal 1 there."""
    import torch
    import meltpooldg_b200 as M
    nc, p = (4, 3, 3), 2
    gm, om = meshes(nc, p, 0.1, seed=9)
    R = rng(77)
    io = (R.uniform(size=gm.n_dofs) < 0.2).astype(np.uint8)
    src = R.uniform(-1, 1, gm.n_dofs)
    op = M.AdvectionDiffusionOperator(gm, 1e-2, theta=0.5, diffusivity=0.02, velocity="vortex",
                                      precisions=("fp64", "fp32"))
    oop = O.Operator(O.ADVDIFF, 1e-2, theta=0.5, diffusivity=0.02, vel_kind=O.VEL_VORTEX)
    ref = O.vmult(om, oop, np.where(io == 1, 0.0, src))
    ref[io == 1] = src[io == 1]
    d_src = dev(src)
    op.set_inflow_outflow(io)
    dst = torch.empty_like(d_src)
    op.vmult(dst, d_src)
    assert relerr(dst.cpu().numpy(), ref) < TOL64
    assert torch.equal(d_src, dev(src))  # src is not modified
    d32 = torch.empty(gm.n_dofs, dtype=torch.float32, device="cuda")
    op.vmult(d32, dev(src, torch.float32))
    assert relerr(d32.double().cpu().numpy(), ref) < TOL32
    inv = torch.empty_like(d_src)
    op.compute_inverse_diagonal_from_matrixfree(inv)
    want = O.inverse_diagonal(om, oop)
    want[io == 1] = 1.0
    assert relerr(inv.cpu().numpy(), want) < TOL64
    op.set_inflow_outflow(None)
    op.vmult(dst, d_src)
    assert relerr(dst.cpu().numpy(), O.vmult(om, oop, src)) < TOL64


def test_c1_vmult_full_size(cuda):
    """Config 1: 16^3 Q2 unit cube, Dirichlet on all faces, src ~ U[-1,1] seed 0."""
    import torch
    import meltpooldg_b200 as M
    nc, p = (16, 16, 16), 2
    mask = M.boundary_mask(nc, p)
    gm, om = meshes(nc, p, mask=mask)
    assert gm.n_dofs == 35937
    src = rng(0).uniform(-1, 1, gm.n_dofs)
    op = _heat(gm, dt=1e-3)
    dst = torch.empty(gm.n_dofs, dtype=torch.float64, device="cuda")
    op.vmult(dst, dev(src))
    ref = O.vmult(om, O.Operator(O.HEAT, 1e-3, dirichlet=mask), src)
    assert relerr(dst.cpu().numpy(), ref) < TOL64
    host = np.empty(gm.n_dofs)
    op.vmult_host(host, src)
    assert relerr(host, ref) < TOL64


def test_l2_norm_and_linearity(cuda):
    import torch
    gm, om = meshes((6, 5, 4), 3, 0.1, seed=6)
    R = rng(40)
    a, b = R.uniform(-1, 1, gm.n_dofs), R.uniform(-1, 1, gm.n_dofs)
    op = _heat(gm, k0=2.0, k_alpha=0.0, vel=(1.0, 0.0, -1.0))
    assert abs(op.l2_norm(dev(a)) - O.l2_norm(om, a)) < 1e-12 * O.l2_norm(om, a)
    x = torch.empty(gm.n_dofs, dtype=torch.float64, device="cuda")
    y, z = torch.empty_like(x), torch.empty_like(x)
    op.vmult(x, dev(a))
    op.vmult(y, dev(b))
    op.vmult(z, dev(2.0 * a - 3.0 * b))
    assert float((z - (2 * x - 3 * y)).abs().max() / z.abs().max()) < 1e-13


def test_errors_are_status_codes(cuda):
    import meltpooldg_b200 as M
    with pytest.raises(M.MpdgError):
        M.Mesh(M.box_vertices((2, 2, 2)), (2, 2, 2), 7)
    gm, _ = meshes((2, 2, 2), 2)
    op = _heat(gm, k_alpha=1e-3)
    import torch
    x = torch.zeros(gm.n_dofs, dtype=torch.float64, device="cuda")
    with pytest.raises(M.MpdgError):  # k(T) without a temperature field
        op.vmult(x, x)
