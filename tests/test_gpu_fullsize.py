"""Parity at the benchmark configurations themselves, through the C ABI.

* Config 2 at full size: 64^3 hexahedra with interior vertices displaced by
  U[-0.1h, 0.1h] (seed 2), FE_Q(4) (16,974,593 DoFs), heat operator with
  k(T) = k0 (1 + 1e-3 T), T ~ U[300, 3000] (seed 3), Dirichlet on all faces;
  src ~ U[-1, 1] (seed 0).  FP64 apply to 1e-12, FP32 to 2e-5 against the
  oracle's vmult (heat_diffuse_operator.cpp:179-197, 955-1086).
* Config 3 at full size: 128^3 uniform cells, FE_Q(2), advection-diffusion
  with the vortex velocity, theta = 0.5, D = 1e-3, dt = 1e-3
  (advection_diffusion_operator.cpp:238-272, 450-495).
* Every schedule of the resident apply (z-slabs, L2 hint, colour overlap, CTA
  cell groups) returns the same bits as the one-launch-per-colour apply; the
  lane apply of config 3 (one thread per cell) matches the oracle likewise.
* CG + Chebyshev(5)/Jacobi at 32^3 Q4 (perturbed, k(T)): the device's Lanczos
  estimate of lambda_max equals the oracle's own estimate from the same start
  vector to 1e-10, and CG with the oracle's own Chebyshev interval takes as
  many iterations as the device (linear_solver.hpp:36-38 semantics).
"""
import numpy as np
import pytest

from gpu_helpers import dev, meshes, relerr, rng
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-5


def _c2_problem(nc):
    import meltpooldg_b200 as M
    p = 4
    mask = M.boundary_mask(nc, p)
    gm, om = meshes(nc, p, 0.1, seed=2, mask=mask)
    T = rng(3).uniform(300.0, 3000.0, gm.n_dofs)
    op = M.HeatDiffuseOperator(gm, 1e-3, rho_cp=1.0, k0=1.0, k_alpha=1e-3, precisions=("fp64", "fp32"))
    Td = dev(T)
    op.set_temperature(Td)
    op._keep_T = Td
    oop = O.Operator(O.HEAT, 1e-3, rho_cp=1.0, k0=1.0, k_alpha=1e-3, temperature=T, dirichlet=mask)
    return gm, om, op, oop, mask


def _schedules_bit_identical(op, src, dtype):
    import torch
    prec = "fp32" if dtype == torch.float32 else "fp64"
    ref = torch.empty_like(src)
    op.set_schedule(1, False, prec, overlap_colours=False)
    op.vmult(ref, src)
    for slabs, hint, overlap, cta in [(1, False, True, False), (2, False, False, False), (8, True, True, True),
                                      (16, False, True, False), (1, True, True, True)]:
        op.set_schedule(slabs, hint, prec, overlap_colours=overlap, cta_cell_groups=cta)
        out = torch.empty_like(src)
        op.vmult(out, src)
        assert torch.equal(out, ref), (slabs, hint, overlap, cta)
    op.set_schedule(1, False, prec, overlap_colours=False)
    return ref


def test_config2_full_size_vmult_parity(cuda):
    import torch
    gm, om, op, oop, _ = _c2_problem((64, 64, 64))
    assert gm.n_dofs == 16974593
    src = rng(0).uniform(-1.0, 1.0, gm.n_dofs)
    ref = O.vmult(om, oop, src)
    d64 = _schedules_bit_identical(op, dev(src), torch.float64)
    assert relerr(d64.cpu().numpy(), ref) < TOL64
    d32 = _schedules_bit_identical(op, dev(src, torch.float32), torch.float32)
    assert relerr(d32.double().cpu().numpy(), ref) < TOL32


def test_config3_full_size_vmult_parity(cuda):
    import torch
    import meltpooldg_b200 as M
    nc, p = (128, 128, 128), 2
    gm, om = meshes(nc, p)
    assert gm.n_dofs == 16974593
    op = M.AdvectionDiffusionOperator(gm, 1e-3, theta=0.5, diffusivity=1e-3, velocity="vortex",
                                      precisions=("fp64", "fp32"))
    oop = O.Operator(O.ADVDIFF, 1e-3, theta=0.5, diffusivity=1e-3, vel_kind=O.VEL_VORTEX)
    src = rng(0).uniform(-1.0, 1.0, gm.n_dofs)
    ref = O.vmult(om, oop, src)
    d64 = _schedules_bit_identical(op, dev(src), torch.float64)
    assert relerr(d64.cpu().numpy(), ref) < TOL64
    d32 = _schedules_bit_identical(op, dev(src, torch.float32), torch.float32)
    assert relerr(d32.double().cpu().numpy(), ref) < TOL32
    # the lane apply (one thread per cell; 4 x-segments per row of cells), in
    # both register variants, one launch per colour and in z-slabs
    for prec, dtype, tol in (("fp64", torch.float64, TOL64), ("fp32", torch.float32, TOL32)):
        s = dev(src, dtype)
        for lane, slabs in ((1, 1), (2, 1), (2, 4)):
            op.set_schedule(slabs, False, prec, overlap_colours=True, lane_cells=lane)
            out = torch.full_like(s, float("nan"))
            op.vmult(out, s)
            assert relerr(out.double().cpu().numpy(), ref) < tol, (prec, lane, slabs)
    assert op.device_error() == 0


def lanczos_start(n, mask, seed=4):
    """The device's deterministic Lanczos start vector (splitmix64 of the DoF
    index and the seed, in [-1, 1), 0 on constrained DoFs), in numpy."""
    i = np.arange(1, n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + np.uint64(0x9E3779B97F4A7C15) * i
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    u = (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    v = 2.0 * u - 1.0
    if mask is not None:
        v[np.asarray(mask) != 0] = 0.0
    return v


@pytest.mark.parametrize("mixed", [False, True])
def test_config2_midsize_chebyshev_cg_with_oracle_lambda(cuda, mixed):
    import torch
    import meltpooldg_b200 as M
    gm, om, op, oop, mask = _c2_problem((32, 32, 32))
    xs = rng(5).uniform(-1.0, 1.0, gm.n_dofs)
    xs[mask == 1] = 0.0
    b = O.vmult(om, oop, xs)
    data = M.LinearSolverData(solver_type="CG", preconditioner_type="Chebyshev", rel_tolerance=1e-10,
                              abs_tolerance=1e-20, mixed_precision=mixed)
    x = torch.zeros(gm.n_dofs, dtype=torch.float64, device="cuda")
    it = M.LinearSolver.solve(op, x, dev(b), data)
    rep = dict(M.LinearSolver.last_report)
    inv = O.inverse_diagonal(om, oop)
    lam_o = O.lambda_max(om, oop, inv, lanczos_start(gm.n_dofs, mask), 10)
    assert abs(rep["lambda_max"] - lam_o) <= 1e-10 * lam_o, (rep["lambda_max"], lam_o)
    xo, it_o, _, ok = O.cg(om, oop, b, inv_diag=inv, rel_tol=1e-10, abs_tol=1e-20,
                           chebyshev={"degree": 5, "lambda_min": lam_o / 30, "lambda_max": 1.2 * lam_o})
    assert ok
    if mixed:
        # FP32 inner iterations with FP64 defects: the same Krylov recurrence up
        # to rounding, so the count may differ by a step
        assert abs(it - it_o) <= 2, (it, it_o)
        assert relerr(x.cpu().numpy(), xo) < 1e-8
    else:
        assert it == it_o, (it, it_o)
        assert relerr(x.cpu().numpy(), xo) < 1e-9
    # the true FP64 residual of the device solution, by the oracle's operator
    r = b - O.vmult(om, oop, x.cpu().numpy())
    assert np.linalg.norm(r) <= 1.05e-10 * np.linalg.norm(b)
