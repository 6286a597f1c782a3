"""Operator and batch state set through the C ABI: a new time increment
(OperatorBase::reset_time_increment), a caller's CUDA stream, the batch's poll
of a running problem and the mesh's device footprint."""
import numpy as np
import pytest

from gpu_helpers import dev, meshes, relerr, rng
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _heat_case(nc, p, perturb):
    import meltpooldg_b200 as M
    mask = M.boundary_mask(nc, p)
    gm, om = meshes(nc, p, perturb, seed=2, mask=mask)
    T = rng(3).uniform(300, 3000, gm.n_dofs)
    return M, gm, om, mask, T


@pytest.mark.parametrize("case", ["heat_q3_perturbed_kT", "heat_q2_uniform", "advdiff_q2_uniform"])
def test_reset_time_increment_equals_a_fresh_operator(cuda, case):
    """Every cached coefficient that holds 1/dt is rebuilt: the FP64 and FP32
    applies after the reset equal those of an operator made with the new dt."""
    import torch
    import meltpooldg_b200 as M
    dt1, dt2 = 1e-3, 3.7e-2
    if case == "heat_q3_perturbed_kT":
        nc, p = (5, 4, 3), 3
        mask = M.boundary_mask(nc, p)
        gm, om = meshes(nc, p, 0.1, seed=2, mask=mask)
        T = rng(3).uniform(300, 3000, gm.n_dofs)

        def make(dt):
            op = M.HeatDiffuseOperator(gm, dt, k0=1.0, k_alpha=1e-3, precisions=("fp64", "fp32"))
            op.set_temperature(dev(T))
            return op
        oop = O.Operator(O.HEAT, dt2, k0=1.0, k_alpha=1e-3, temperature=T, dirichlet=mask)
    elif case == "heat_q2_uniform":
        nc, p = (40, 40, 24), 2  # enough cells for the lane apply
        mask = M.boundary_mask(nc, p)
        gm, om = meshes(nc, p, mask=mask)

        def make(dt):
            return M.HeatDiffuseOperator(gm, dt, rho_cp=2.0, k0=1.5, precisions=("fp64", "fp32"))
        oop = O.Operator(O.HEAT, dt2, rho_cp=2.0, k0=1.5, dirichlet=mask)
    else:
        nc, p = (40, 40, 24), 2
        mask = M.boundary_mask(nc, p)
        gm, om = meshes(nc, p, mask=mask, lo=(-1, -1, -1), hi=(1, 1, 1))

        def make(dt):
            return M.AdvectionDiffusionOperator(gm, dt, theta=0.5, diffusivity=1e-3, velocity="vortex",
                                                precisions=("fp64", "fp32"))
        oop = O.Operator(O.ADVDIFF, dt2, theta=0.5, diffusivity=1e-3, vel_kind=O.VEL_VORTEX, dirichlet=mask)
    src = dev(rng(8).uniform(-1, 1, gm.n_dofs))
    op = make(dt1)
    out = torch.empty_like(src)
    op.vmult(out, src)                       # builds the dt1 caches
    op.vmult(out.float(), src.float())
    op.reset_time_increment(dt2)
    fresh = make(dt2)
    got, ref = torch.empty_like(src), torch.empty_like(src)
    op.vmult(got, src)
    fresh.vmult(ref, src)
    assert torch.equal(got, ref)
    got32, ref32 = torch.empty_like(src, dtype=torch.float32), torch.empty_like(src, dtype=torch.float32)
    op.vmult(got32, src.float())
    fresh.vmult(ref32, src.float())
    assert torch.equal(got32, ref32)
    if gm.n_dofs <= 200000:
        assert relerr(got.cpu().numpy(), O.vmult(om, oop, src.cpu().numpy())) < 1e-12


def test_operator_on_a_caller_stream(cuda):
    """Applies and solves launched on a caller's stream give the results of
    the default stream, bit for bit."""
    import torch
    M, gm, om, mask, T = _heat_case((6, 5, 4), 2, 0.1)
    op = M.HeatDiffuseOperator(gm, 1e-3, k0=1.0, k_alpha=1e-3)
    op.set_temperature(dev(T))
    src = dev(rng(9).uniform(-1, 1, gm.n_dofs))
    ref = torch.empty_like(src)
    op.vmult(ref, src)
    b = ref.clone()
    x_ref = torch.zeros_like(src)
    data = M.LinearSolverData(solver_type="CG", rel_tolerance=1e-10)
    it_ref = M.LinearSolver.solve(op, x_ref, b, data)
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    op.set_stream(s)
    got = torch.empty_like(src)
    x = torch.zeros_like(src)
    with torch.cuda.stream(s):
        op.vmult(got, src)
        it = M.LinearSolver.solve(op, x, b, data)
    s.synchronize()
    op.set_stream(None)
    assert torch.equal(got, ref)
    assert it == it_ref
    assert torch.equal(x, x_ref)


def test_batch_poll_follows_a_problem(cuda):
    """poll reports a submitted problem as running (status 1) until the
    batch has advanced it to convergence, then its final report."""
    from meltpooldg_b200 import batch as B
    prob = B.Problem(kind=B.OP_HEAT, degree=2, nc=6, k0=3.0, dt=1e-3, rho_cp=1.0, rel_tolerance=1e-10,
                     rhs_seed=5)
    with B.Batch(1 << 30, capacity=4) as bt:
        t = bt.submit(prob)
        assert bt.poll(t)["status"] == 1
        steps, running = bt.run(max_steps=2, poll_steps=1)
        rep = bt.poll(t)
        assert rep["status"] == 1 and running == 1
        bt.run()
        rep = bt.poll(t)
        assert rep["status"] == 0
        assert rep["iterations"] > 2
        assert rep["final_residual"] <= 1e-10 * rep["initial_residual"]
        x, rep2 = bt.take(t, prob.n_dofs)
        assert rep2["iterations"] == rep["iterations"]
        assert np.all(np.isfinite(x))


def test_mesh_device_bytes_grow_with_the_mesh(cuda):
    import meltpooldg_b200 as M
    small = M.Mesh(M.box_vertices((4, 4, 4)), (4, 4, 4), 2, M.boundary_mask((4, 4, 4), 2))
    large = M.Mesh(M.box_vertices((12, 12, 12)), (12, 12, 12), 2, M.boundary_mask((12, 12, 12), 2))
    assert 0 < small.device_bytes() < large.device_bytes()
    small.close()
    large.close()
