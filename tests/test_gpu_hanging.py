"""Hanging nodes on the device (two-level meshes, mpdg_mesh_create_two_level)
against the oracle's constrained operator: vmult (FP64 to 1e-12, FP32 to
2e-5), the diagonal (1e-12), CG + Jacobi iteration counts and solutions."""
import numpy as np
import pytest

from gpu_helpers import dev, relerr
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-5


def two_level(p, nc=(2, 2, 2), ncf_x=3, perturb=0.0, seed=1, dirichlet=True, geometry="auto"):
    import meltpooldg_b200 as M
    om = O.Mesh2(p, nc, ncf_x, perturb=perturb, seed=seed)
    mask = om.boundary_face_mask() if dirichlet else np.zeros(om.n_dofs, np.uint8)
    nc_f = (ncf_x, 2 * nc[1], 2 * nc[2])
    gm = M.TwoLevelMesh(om.coarse.vert, nc, om.fine.vert, nc_f, p, mask[:om.n_coarse], mask[om.n_coarse:],
                        geometry=geometry)
    assert gm.n_dofs == om.n_dofs
    return gm, om, mask


def _ops(gm, kind, mask, prec=("fp64", "fp32")):
    import meltpooldg_b200 as M
    if kind == "heat":
        op = M.HeatDiffuseOperator(gm, 1e-2, rho_cp=2.0, k0=1.5, precisions=prec)
        oop = O.Operator(O.HEAT, 1e-2, rho_cp=2.0, k0=1.5, dirichlet=mask)
    else:
        op = M.AdvectionDiffusionOperator(gm, 1e-2, theta=0.5, diffusivity=0.05, velocity="vortex",
                                          precisions=prec)
        oop = O.Operator(O.ADVDIFF, 1e-2, theta=0.5, diffusivity=0.05, vel_kind=O.VEL_VORTEX, dirichlet=mask)
    return op, oop


@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("kind", ["heat", "advdiff"])
@pytest.mark.parametrize("perturb", [0.0, 0.1])
def test_two_level_vmult_parity(cuda, p, kind, perturb):
    import torch
    gm, om, mask = two_level(p, perturb=perturb, seed=10 + p)
    op, oop = _ops(gm, kind, mask)
    R = np.random.default_rng(p)
    src = R.uniform(-1, 1, gm.n_dofs)
    src[om.hanging_mask().astype(bool)] = 0.0
    ref = O.vmult2(om, oop, src)
    dst = torch.empty(gm.n_dofs, dtype=torch.float64, device="cuda")
    op.vmult(dst, dev(src))
    assert relerr(dst.cpu().numpy(), ref) < TOL64
    d32 = torch.empty(gm.n_dofs, dtype=torch.float32, device="cuda")
    op.vmult(d32, dev(src, torch.float32))
    assert relerr(d32.double().cpu().numpy(), ref) < TOL32


@pytest.mark.parametrize("p", [1, 2, 4])
def test_two_level_values_at_hanging_slots_are_ignored(cuda, p):
    """The hanging DoFs are read through the interpolation: whatever the vector
    holds there does not change the result, and the output there is 0."""
    import torch
    gm, om, mask = two_level(p, dirichlet=False)
    op, oop = _ops(gm, "heat", mask, prec=("fp64",))
    hm = om.hanging_mask().astype(bool)
    R = np.random.default_rng(5)
    a = R.uniform(-1, 1, gm.n_dofs)
    b = a.copy()
    b[hm] = R.uniform(-9, 9, int(hm.sum()))
    ya = torch.empty(gm.n_dofs, dtype=torch.float64, device="cuda")
    yb = torch.empty_like(ya)
    op.vmult(ya, dev(a))
    op.vmult(yb, dev(b))
    assert torch.equal(ya, yb)
    assert float(ya.cpu().numpy()[hm].__abs__().max()) == 0.0


@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("kind", ["heat", "advdiff"])
def test_two_level_diagonal(cuda, p, kind):
    import torch
    gm, om, mask = two_level(p, perturb=0.1, seed=20 + p)
    op, oop = _ops(gm, kind, mask, prec=("fp64",))
    d = torch.empty(gm.n_dofs, dtype=torch.float64, device="cuda")
    op.compute_diagonal(d)
    assert relerr(d.cpu().numpy(), O.diagonal2(om, oop)) < TOL64


def _oracle_cg(om, oop, b, diag, rel_tol, max_it=2000):
    """deal.II SolverCG recurrence with Jacobi, on the oracle's constrained operator."""
    inv = 1.0 / diag
    x = np.zeros_like(b)
    r = b.copy()
    res0 = np.linalg.norm(r)
    z = inv * r
    p = z.copy()
    rz = r @ z
    for it in range(1, max_it + 1):
        Ap = O.vmult2(om, oop, p)
        alpha = rz / (p @ Ap)
        x += alpha * p
        r -= alpha * Ap
        if np.linalg.norm(r) <= rel_tol * res0:
            return x, it
        z = inv * r
        rz_new = r @ z
        p = z + (rz_new / rz) * p
        rz = rz_new
    raise RuntimeError("oracle CG did not converge")


@pytest.mark.parametrize("p", [2, 3])
def test_two_level_cg_iterations_match_oracle(cuda, p):
    import torch
    import meltpooldg_b200 as M
    gm, om, mask = two_level(p, nc=(2, 3, 2), ncf_x=2, perturb=0.1, seed=30 + p)
    op, oop = _ops(gm, "heat", mask, prec=("fp64",))
    hm = om.hanging_mask().astype(bool) | mask.astype(bool)
    R = np.random.default_rng(7)
    xs = R.uniform(-1, 1, gm.n_dofs)
    xs[hm] = 0.0
    b = O.vmult2(om, oop, xs)
    x_ref, its_ref = _oracle_cg(om, oop, b, O.diagonal2(om, oop), 1e-10)
    x = torch.zeros(gm.n_dofs, dtype=torch.float64, device="cuda")
    its = M.LinearSolver.solve(op, x, dev(b), M.LinearSolverData(solver_type="CG", preconditioner_type="Diagonal",
                                                                 rel_tolerance=1e-10, abs_tolerance=0.0))
    assert abs(its - its_ref) <= 1, (its, its_ref)
    assert np.linalg.norm(x.cpu().numpy() - x_ref) <= 1e-8 * np.linalg.norm(x_ref)
    # the FP32 operator with FP64 reliable updates reaches the same FP64 residual
    x2 = torch.zeros_like(x)
    M.LinearSolver.solve(op, x2, dev(b), M.LinearSolverData(solver_type="CG", preconditioner_type="Diagonal",
                                                            rel_tolerance=1e-10, abs_tolerance=0.0,
                                                            mixed_precision=True))
    r = b - O.vmult2(om, oop, x2.cpu().numpy())
    assert np.linalg.norm(r) <= 1.01e-10 * np.linalg.norm(b)


@pytest.mark.parametrize("p", [1, 2])
def test_two_level_inflow_outflow_identity_rows(cuda, p):
    """Identity rows (advection_diffusion_operator.cpp:537-578) across both
    blocks of a two-level mesh: src read as 0 at the flagged DoFs, the result
    there equal to src (hanging DoFs never flagged: they are not unknowns)."""
    import torch
    gm, om, mask = two_level(p, perturb=0.1, seed=30 + p, dirichlet=False)
    op, oop = _ops(gm, "advdiff", mask)
    R = np.random.default_rng(40 + p)
    hm = om.hanging_mask().astype(bool)
    io = (R.uniform(size=gm.n_dofs) < 0.2).astype(np.uint8)
    io[hm] = 0
    src = R.uniform(-1, 1, gm.n_dofs)
    src[hm] = 0.0
    ref = O.vmult2(om, oop, np.where(io == 1, 0.0, src))
    ref[io == 1] = src[io == 1]
    op.set_inflow_outflow(io)
    dst = torch.empty(gm.n_dofs, dtype=torch.float64, device="cuda")
    op.vmult(dst, dev(src))
    assert relerr(dst.cpu().numpy(), ref) < TOL64
    d32 = torch.empty(gm.n_dofs, dtype=torch.float32, device="cuda")
    op.vmult(d32, dev(src, torch.float32))
    assert relerr(d32.double().cpu().numpy(), ref) < TOL32
