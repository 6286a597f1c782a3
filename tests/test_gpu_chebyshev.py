"""CG + Chebyshev(5)/Jacobi on the device: iteration counts and solutions as
the oracle's (given the device's largest-eigenvalue estimate) on uniform and
perturbed meshes, and the lattice path against a mapped mesh of the same
lattice (the two sum the cell contributions in different orders), in FP64
and in the FP32-inner form."""
import numpy as np
import pytest

from gpu_helpers import dev, meshes, relerr, rng
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _data(mixed=False):
    import meltpooldg_b200 as M
    return M.LinearSolverData(solver_type="CG", preconditioner_type="Chebyshev", rel_tolerance=1e-10,
                              abs_tolerance=1e-20, mixed_precision=mixed)


@pytest.mark.parametrize("p,perturb", [(2, 0.0), (3, 0.1), (4, 0.1), (4, 0.0)])
def test_chebyshev_cg_matches_oracle(cuda, p, perturb):
    import torch
    import meltpooldg_b200 as M
    nc = (6, 5, 4)
    mask = M.boundary_mask(nc, p)
    gm, om = meshes(nc, p, perturb, seed=2, mask=mask)
    xs = rng(5).uniform(-1, 1, gm.n_dofs)
    xs[mask == 1] = 0.0
    if perturb > 0.0:
        T = rng(3).uniform(300, 3000, gm.n_dofs)
        op = M.HeatDiffuseOperator(gm, 1e-3, k0=1.0, k_alpha=1e-3)
        op.set_temperature(dev(T))
        oop = O.Operator(O.HEAT, 1e-3, k0=1.0, k_alpha=1e-3, temperature=T, dirichlet=mask)
    else:
        op = M.HeatDiffuseOperator(gm, 1e-3, rho_cp=2.0, k0=1.5)
        oop = O.Operator(O.HEAT, 1e-3, rho_cp=2.0, k0=1.5, dirichlet=mask)
    b = O.vmult(om, oop, xs)
    x = torch.zeros(gm.n_dofs, dtype=torch.float64, device="cuda")
    it = M.LinearSolver.solve(op, x, dev(b), _data())
    rep = M.LinearSolver.last_report
    lam = rep["lambda_max"]
    inv = O.inverse_diagonal(om, oop)
    xo, it_o, _, ok = O.cg(om, oop, b, inv_diag=inv, rel_tol=1e-10, abs_tol=1e-20,
                           chebyshev={"degree": 5, "lambda_min": lam / 30, "lambda_max": 1.2 * lam})
    assert ok
    assert it == it_o, (it, it_o)
    assert relerr(x.cpu().numpy(), xo) < 1e-9


@pytest.mark.parametrize("p", [2, 4])
@pytest.mark.parametrize("mixed", [False, True])
def test_lattice_and_mapped_chebyshev_solves_agree(cuda, p, mixed):
    """A mapped mesh of the same lattice (identity numbering) applies the same
    operator through the cell->DoF map."""
    import torch
    import meltpooldg_b200 as M
    nc = (5, 4, 6)
    mask = M.boundary_mask(nc, p)
    gm, om = meshes(nc, p, 0.1, seed=7, mask=mask)
    mm = O.mapped_from_mesh(om)
    gmm = M.MappedMesh(mm.cell_vertices, mm.cell_dofs, mm.n_dofs, mm.degree, dirichlet_mask=mask)
    prec = ("fp64", "fp32")
    b = rng(11).uniform(-1, 1, gm.n_dofs)
    b[mask == 1] = 0.0
    out = []
    for mesh in (gm, gmm):
        op = M.HeatDiffuseOperator(mesh, 1e-3, rho_cp=2.0, k0=1.5, precisions=prec)
        x = torch.zeros(gm.n_dofs, dtype=torch.float64, device="cuda")
        it = M.LinearSolver.solve(op, x, dev(b), _data(mixed))
        out.append((it, x.cpu().numpy(), dict(M.LinearSolver.last_report)))
    (it_f, x_f, rep_f), (it_s, x_s, rep_s) = out
    # the two paths sum the cell contributions in different orders
    assert abs(it_f - it_s) <= (1 if mixed else 0), (it_f, it_s)
    assert rep_f["final_residual"] <= 1e-10 * rep_f["initial_residual"]
    assert relerr(x_f, x_s) < (1e-6 if mixed else 1e-10)
