"""Device Krylov solvers against the oracle's: CG iteration counts, GMRES
solutions, Chebyshev and the FP32-inner / FP64-defect-correction form."""
import numpy as np
import pytest

from gpu_helpers import dev, meshes, relerr, rng
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_c1_cg_jacobi_iteration_parity(cuda):
    """Config 1: CG + Jacobi to 1e-10, rhs = A x*, x* ~ U[-1,1] seed 1 on free DoFs."""
    import torch
    import meltpooldg_b200 as M
    nc, p = (16, 16, 16), 2
    mask = M.boundary_mask(nc, p)
    gm, om = meshes(nc, p, mask=mask)
    xs = rng(1).uniform(-1, 1, gm.n_dofs)
    xs[mask == 1] = 0.0
    oop = O.Operator(O.HEAT, 1e-3, dirichlet=mask)
    b = O.vmult(om, oop, xs)
    inv = O.inverse_diagonal(om, oop)
    xo, it_o, hist_o, ok = O.cg(om, oop, b, inv_diag=inv, rel_tol=1e-10, abs_tol=1e-20)
    assert ok
    op = M.HeatDiffuseOperator(gm, 1e-3)
    x = torch.zeros(gm.n_dofs, dtype=torch.float64, device="cuda")
    it = M.LinearSolver.solve(op, x, dev(b), M.LinearSolverData(
        solver_type="CG", preconditioner_type="Diagonal", rel_tolerance=1e-10, abs_tolerance=1e-20))
    rep = M.LinearSolver.last_report
    assert it == it_o, (it, it_o)
    assert rep["final_residual"] <= 1e-10 * rep["initial_residual"]
    assert abs(rep["initial_residual"] - hist_o[0]) < 1e-12 * hist_o[0]
    assert relerr(x.cpu().numpy(), xo) < 1e-9


def test_gmres_advdiff_matches_oracle(cuda):
    import torch
    import meltpooldg_b200 as M
    nc, p = (6, 6, 6), 2
    mask = M.boundary_mask(nc, p, faces=[(0, 0)])
    gm, om = meshes(nc, p, 0.1, seed=9, mask=mask, lo=(-1, -1, -1), hi=(1, 1, 1))
    b = rng(2).uniform(-1, 1, gm.n_dofs)
    b[mask == 1] = 0.0
    oop = O.Operator(O.ADVDIFF, 1e-2, theta=0.5, diffusivity=1e-2, vel_kind=O.VEL_VORTEX, dirichlet=mask)
    inv = O.inverse_diagonal(om, oop)
    xo, it_o, _, ok = O.gmres(om, oop, b, inv_diag=inv, rel_tol=1e-12)
    assert ok
    op = M.AdvectionDiffusionOperator(gm, 1e-2, theta=0.5, diffusivity=1e-2, velocity="vortex")
    x = torch.zeros(gm.n_dofs, dtype=torch.float64, device="cuda")
    it = M.LinearSolver.solve(op, x, dev(b), M.LinearSolverData(rel_tolerance=1e-12))
    assert relerr(x.cpu().numpy(), xo) < 1e-9
    assert abs(it - it_o) <= 2


def _advdiff_system(nc=(6, 6, 6), p=2):
    import meltpooldg_b200 as M
    mask = M.boundary_mask(nc, p, faces=[(0, 0)])
    gm, om = meshes(nc, p, 0.1, seed=9, mask=mask, lo=(-1, -1, -1), hi=(1, 1, 1))
    b = rng(2).uniform(-1, 1, gm.n_dofs)
    b[mask == 1] = 0.0
    oop = O.Operator(O.ADVDIFF, 1e-2, theta=0.5, diffusivity=1e-2, vel_kind=O.VEL_VORTEX, dirichlet=mask)
    return gm, om, b, oop


@pytest.mark.parametrize("restart", [2, 5])
@pytest.mark.parametrize("mixed", [False, True])
def test_gmres_restarted_matches_oracle(cuda, restart, mixed):
    """Restart cycles: each ends with the step that only completes the last
    Hessenberg column (no apply), then a fresh residual."""
    import torch
    import meltpooldg_b200 as M
    gm, om, b, oop = _advdiff_system()
    inv = O.inverse_diagonal(om, oop)
    xo, it_o, _, ok = O.gmres(om, oop, b, inv_diag=inv, rel_tol=1e-10, restart=restart)
    assert ok
    op = M.AdvectionDiffusionOperator(gm, 1e-2, theta=0.5, diffusivity=1e-2, velocity="vortex",
                                      precisions=("fp64", "fp32") if mixed else ("fp64",))
    x = torch.zeros(gm.n_dofs, dtype=torch.float64, device="cuda")
    it = M.LinearSolver.solve(op, x, dev(b), M.LinearSolverData(rel_tolerance=1e-10, gmres_restart=restart,
                                                                mixed_precision=mixed))
    rep = M.LinearSolver.last_report
    assert rep["final_residual"] <= 1e-10 * rep["initial_residual"]
    assert relerr(x.cpu().numpy(), xo) < (1e-7 if mixed else 1e-8)
    if not mixed:
        assert abs(it - it_o) <= 2, (it, it_o)
    # the true residual under the oracle's operator
    r = b - O.vmult(om, oop, x.cpu().numpy())
    assert np.linalg.norm(r) <= 2e-10 * np.linalg.norm(b)


def test_gmres_iteration_limit_inside_a_cycle(cuda):
    """max_iterations that ends a restart cycle early: NOT_CONVERGED after
    exactly that many iterations, with the solution updated from them."""
    import torch
    import meltpooldg_b200 as M
    from meltpooldg_b200._capi import NoConvergence
    gm, om, b, oop = _advdiff_system()
    op = M.AdvectionDiffusionOperator(gm, 1e-2, theta=0.5, diffusivity=1e-2, velocity="vortex")
    x = torch.zeros(gm.n_dofs, dtype=torch.float64, device="cuda")
    with pytest.raises(NoConvergence):
        M.LinearSolver.solve(op, x, dev(b), M.LinearSolverData(rel_tolerance=1e-14, gmres_restart=3,
                                                               max_iterations=7))
    rep = M.LinearSolver.last_report
    assert rep["iterations"] == 7
    r = b - O.vmult(om, oop, x.cpu().numpy())
    assert np.linalg.norm(r) < np.linalg.norm(b)


def _c2_like(nc, p):
    """Config 2 shape at a small size: perturbed vertices (10% h, seed 2),
    T ~ U[300,3000] (seed 3), k = k0 (1 + 1e-3 T), Dirichlet on all faces."""
    import meltpooldg_b200 as M
    mask = M.boundary_mask(nc, p)
    gm, om = meshes(nc, p, 0.1, seed=2, mask=mask)
    T = rng(3).uniform(300, 3000, gm.n_dofs)
    xs = rng(5).uniform(-1, 1, gm.n_dofs)
    xs[mask == 1] = 0.0
    oop = O.Operator(O.HEAT, 1e-3, k0=1.0, k_alpha=1e-3, temperature=T, dirichlet=mask)
    b = O.vmult(om, oop, xs)
    return gm, om, mask, T, xs, oop, b


def test_chebyshev_cg_and_mixed_precision(cuda):
    import torch
    import meltpooldg_b200 as M
    gm, om, mask, T, xs, oop, b = _c2_like((8, 8, 8), 4)
    op = M.HeatDiffuseOperator(gm, 1e-3, k0=1.0, k_alpha=1e-3, precisions=("fp64", "fp32"))
    op.set_temperature(dev(T))
    data = M.LinearSolverData(solver_type="CG", preconditioner_type="Chebyshev", rel_tolerance=1e-10,
                              abs_tolerance=1e-20)
    x64 = torch.zeros(gm.n_dofs, dtype=torch.float64, device="cuda")
    M.LinearSolver.solve(op, x64, dev(b), data)
    r64 = M.LinearSolver.last_report
    assert r64["final_residual"] <= 1e-10 * r64["initial_residual"]
    assert relerr(x64.cpu().numpy(), xs) < 1e-7
    data.mixed_precision = True
    x32 = torch.zeros_like(x64)
    M.LinearSolver.solve(op, x32, dev(b), data)
    r32 = M.LinearSolver.last_report
    assert r32["final_residual"] <= 1e-10 * r32["initial_residual"], r32
    assert r32["outer_iterations"] >= 1
    # the stated error of the mixed form against the FP64 solve
    assert relerr(x32.cpu().numpy(), x64.cpu().numpy()) < 1e-8
    # Jacobi-preconditioned CG agrees as well
    data2 = M.LinearSolverData(solver_type="CG", preconditioner_type="Diagonal", rel_tolerance=1e-10)
    x3 = torch.zeros_like(x64)
    M.LinearSolver.solve(op, x3, dev(b), data2)
    assert relerr(x3.cpu().numpy(), x64.cpu().numpy()) < 1e-8


@pytest.mark.parametrize("solver", ["CG", "GMRES"])
@pytest.mark.parametrize("mixed", [False, True])
def test_solves_from_a_nonzero_initial_guess(cuda, solver, mixed):
    """The Newton loop starts each solve from the previous increment: the
    relative tolerance is taken against the residual of that start (deal.II
    ReductionControl), as in the oracle started from the same vector."""
    import torch
    import meltpooldg_b200 as M
    if solver == "CG":
        gm, om, mask, T, xs, oop, b = _c2_like((6, 6, 6), 2)
        op = M.HeatDiffuseOperator(gm, 1e-3, k0=1.0, k_alpha=1e-3, precisions=("fp64", "fp32"))
        op.set_temperature(dev(T))
    else:
        gm, om, b, oop = _advdiff_system()
        mask = M.boundary_mask((6, 6, 6), 2, faces=[(0, 0)])
        op = M.AdvectionDiffusionOperator(gm, 1e-2, theta=0.5, diffusivity=1e-2, velocity="vortex",
                                          precisions=("fp64", "fp32"))
    x0 = rng(21).uniform(-1, 1, gm.n_dofs)
    x0[np.asarray(mask) == 1] = 0.0
    inv = O.inverse_diagonal(om, oop)
    if solver == "CG":
        xo, it_o, _, ok = O.cg(om, oop, b, x0=x0, inv_diag=inv, rel_tol=1e-10, abs_tol=1e-20)
    else:
        xo, it_o, _, ok = O.gmres(om, oop, b, x0=x0, inv_diag=inv, rel_tol=1e-10, restart=5)
    assert ok
    x = dev(x0.copy())
    it = M.LinearSolver.solve(op, x, dev(b), M.LinearSolverData(solver_type=solver, rel_tolerance=1e-10,
                                                                abs_tolerance=1e-20, gmres_restart=5,
                                                                mixed_precision=mixed))
    rep = M.LinearSolver.last_report
    r0 = np.linalg.norm(b - O.vmult(om, oop, x0))
    assert abs(rep["initial_residual"] - r0) <= 1e-12 * r0
    assert rep["final_residual"] <= 1e-10 * rep["initial_residual"]
    assert relerr(x.cpu().numpy(), xo) < (1e-7 if mixed else 1e-8)
    if not mixed:
        assert abs(it - it_o) <= (0 if solver == "CG" else 2), (it, it_o)


@pytest.mark.parametrize("mixed", [False, True])
def test_gmres_chebyshev_restarted(cuda, mixed):
    """GMRES with the Chebyshev smoother as its right preconditioner, over
    several restart cycles: each cycle's correction V y goes through the
    smoother, whose own scratch vectors must not hold it."""
    import torch
    import meltpooldg_b200 as M
    gm, om, mask, T, xs, oop, b = _c2_like((6, 6, 6), 3)
    op = M.HeatDiffuseOperator(gm, 1e-3, k0=1.0, k_alpha=1e-3, precisions=("fp64", "fp32"))
    op.set_temperature(dev(T))
    data = M.LinearSolverData(solver_type="GMRES", preconditioner_type="Chebyshev", rel_tolerance=1e-10,
                              abs_tolerance=1e-20, gmres_restart=3, mixed_precision=mixed)
    x = torch.zeros(gm.n_dofs, dtype=torch.float64, device="cuda")
    it = M.LinearSolver.solve(op, x, dev(b), data)
    rep = M.LinearSolver.last_report
    assert rep["final_residual"] <= 1e-10 * rep["initial_residual"], rep
    assert it > 3  # more than one cycle
    r = b - O.vmult(om, oop, x.cpu().numpy())
    assert np.linalg.norm(r) <= 2e-10 * np.linalg.norm(b)
    assert relerr(x.cpu().numpy(), xs) < 1e-7


def test_solver_failure_modes_are_reported(cuda):
    import torch
    import meltpooldg_b200 as M
    gm, om, mask, T, xs, oop, b = _c2_like((4, 4, 4), 2)
    op = M.HeatDiffuseOperator(gm, 1e-3, k0=1.0, k_alpha=1e-3)
    op.set_temperature(dev(T))
    x = torch.zeros(gm.n_dofs, dtype=torch.float64, device="cuda")
    with pytest.raises(M.NoConvergence):
        M.LinearSolver.solve(op, x, dev(b), M.LinearSolverData(solver_type="CG", max_iterations=2,
                                                               rel_tolerance=1e-14))
    bad = b.copy()
    bad[len(bad) // 2] = np.nan
    x.zero_()
    with pytest.raises(M.MpdgError) as e:
        M.LinearSolver.solve(op, x, dev(bad), M.LinearSolverData(solver_type="CG"))
    assert e.value.status == -6


@pytest.mark.parametrize("solver", ["CG", "GMRES"])
def test_solve_with_host_buffers_equals_device_solve(cuda, solver):
    """mpdg_solve_host (host x and b, device copies inside the call) runs the
    same loop as mpdg_solve: the same iterates, bit for bit; a failing solve
    reports its error and leaves the operator usable."""
    import torch
    import meltpooldg_b200 as M
    if solver == "CG":
        gm, om, mask, T, xs, oop, b = _c2_like((5, 5, 5), 2)
        op = M.HeatDiffuseOperator(gm, 1e-3, k0=1.0, k_alpha=1e-3)
        op.set_temperature(dev(T))
    else:
        gm, om, b, oop = _advdiff_system()
        op = M.AdvectionDiffusionOperator(gm, 1e-2, theta=0.5, diffusivity=1e-2, velocity="vortex")
    data = M.LinearSolverData(solver_type=solver, rel_tolerance=1e-10, abs_tolerance=1e-20)
    x = torch.zeros(gm.n_dofs, dtype=torch.float64, device="cuda")
    it = M.LinearSolver.solve(op, x, dev(b), data)
    xh = np.zeros(gm.n_dofs)
    it_h = M.LinearSolver.solve_host(op, xh, np.ascontiguousarray(b), data)
    assert it_h == it
    assert np.array_equal(xh, x.cpu().numpy())
    bad = b.copy()
    bad[len(bad) // 2] = np.nan
    with pytest.raises(M.MpdgError):
        M.LinearSolver.solve_host(op, np.zeros(gm.n_dofs), bad, data)
    xh2 = np.zeros(gm.n_dofs)
    assert M.LinearSolver.solve_host(op, xh2, np.ascontiguousarray(b), data) == it
    assert np.array_equal(xh2, xh)
