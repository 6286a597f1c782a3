"""Batched and served solves (mpdg_batch_* / mpdg_serve) against the FP64 oracle.

Each problem's residual is recomputed with the oracle's FP64 operator; the
Jacobi diagonal the batch builds is compared with the oracle's; a problem's
solution must be bit-identical alone and in any mix of other problems, in the
batch and in the serving loop."""
import numpy as np
import pytest

from gpu_helpers import relerr
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# residual tolerance of a batched solve, checked with the oracle's FP64 operator:
# the batch stops at |b - A x| <= 1e-10 |b| by its own FP64 defect; the oracle's
# operator differs from the batch's FP64 apply by rounding only
RES_TOL = 1.05e-10
DIAG_TOL = 1e-12


def _B():
    from meltpooldg_b200 import batch as B
    return B


def oracle_problem(p):
    """Oracle mesh and operator of a batched problem (unit cube, uniform)."""
    from meltpooldg_b200 import box_vertices
    B = _B()
    V = box_vertices((p.nc,) * 3)
    om = O.Mesh(3, p.degree, (p.nc,) * 3, V)
    mask = om.boundary_face_mask() if p.dirichlet else None
    if p.kind == B.OP_HEAT:
        op = O.Operator(O.HEAT, p.dt, rho_cp=p.rho_cp, k0=p.k0, dirichlet=mask)
    else:
        op = O.Operator(O.ADVDIFF, p.dt, theta=p.theta, diffusivity=p.diffusivity,
                        vel_kind=O.VEL_VORTEX if p.vortex else O.VEL_NONE, dirichlet=mask)
    return om, op


def oracle_relres(p, x):
    om, op = oracle_problem(p)
    b = p.rhs()
    r = b - O.vmult(om, op, x)
    return float(np.linalg.norm(r) / np.linalg.norm(b))


def heat(nc, degree, k0=1.0, seed=0, **kw):
    B = _B()
    return B.Problem(kind=B.OP_HEAT, degree=degree, nc=nc, k0=k0, rhs_seed=seed, **kw)


def advdiff(nc, degree, seed=0, **kw):
    B = _B()
    return B.Problem(kind=B.OP_ADVDIFF, degree=degree, nc=nc, rhs_seed=seed, **kw)


@pytest.mark.parametrize("make", [lambda: heat(5, 2, k0=7.0), lambda: heat(4, 4, k0=30.0),
                                  lambda: advdiff(5, 3, diffusivity=1e-2)])
def test_batch_diagonal_matches_oracle(make):
    p = make()
    om, op = oracle_problem(p)
    ref = O.diagonal(om, op)
    got = p.diagonal()
    assert relerr(got, ref) <= DIAG_TOL


def test_batch_rhs_host_matches_device():
    """The host copy of the seeded right-hand side is the one the batch solves."""
    B = _B()
    p = heat(4, 2, seed=11)
    b = p.rhs()
    with B.Batch(10**9, capacity=4) as bt:
        t1 = bt.submit(p)
        t2 = bt.submit(p, rhs=b)
        bt.run()
        x1, r1 = bt.take(t1, p.n_dofs)
        x2, r2 = bt.take(t2, p.n_dofs)
    assert np.array_equal(x1, x2)
    assert r1["iterations"] == r2["iterations"]


@pytest.mark.parametrize("make", [lambda: heat(6, 2, k0=3.0, seed=1), lambda: heat(4, 3, k0=80.0, seed=2),
                                  lambda: heat(3, 4, seed=3), lambda: heat(8, 1, seed=4),
                                  lambda: advdiff(6, 2, seed=5), lambda: advdiff(4, 3, seed=6,
                                                                                 diffusivity=1e-2)])
def test_batched_solve_residual_against_oracle(make):
    B = _B()
    p = make()
    (x,), (rep,) = B.solve_batch([p])
    assert rep["status"] == 0, rep
    assert rep["final_residual"] <= 1e-10 * rep["initial_residual"] * (1 + 1e-12)
    assert oracle_relres(p, x) <= RES_TOL


def test_batched_heat_matches_single_fp64_cg():
    """Same problem through the single-problem FP64 CG + Jacobi path."""
    import torch
    import meltpooldg_b200 as M
    B = _B()
    p = heat(6, 3, k0=5.0, seed=9)
    (xb,), (rep,) = B.solve_batch([p])
    mesh = M.Mesh(M.box_vertices((p.nc,) * 3), (p.nc,) * 3, p.degree,
                  M.boundary_mask((p.nc,) * 3, p.degree))
    op = M.HeatDiffuseOperator(mesh, p.dt, rho_cp=p.rho_cp, k0=p.k0)
    b = torch.tensor(p.rhs(), device="cuda")
    x = torch.zeros_like(b)
    its = M.LinearSolver.solve(op, x, b, M.LinearSolverData(solver_type="CG", rel_tolerance=1e-10))
    xs = x.cpu().numpy()
    assert np.linalg.norm(xb - xs) <= 1e-7 * np.linalg.norm(xs)
    # mixed precision with reliable updates keeps the FP64 iteration count within a few steps
    assert abs(rep["iterations"] - its) <= max(3, its // 10), (rep["iterations"], its)


def test_alone_equals_in_mix():
    """A problem's solution does not depend on the other problems in the batch."""
    B = _B()
    target = heat(5, 3, k0=12.0, seed=21)
    target_a = advdiff(5, 2, seed=22)
    others = [heat(7, 2, seed=30), advdiff(4, 4, seed=31), heat(3, 4, k0=90.0, seed=32),
              heat(9, 1, seed=33), advdiff(6, 3, seed=34)]
    alone, ralone = B.solve_batch([target, target_a])
    mixed, rmixed = B.solve_batch(others[:2] + [target] + others[2:4] + [target_a] + others[4:])
    assert np.array_equal(alone[0], mixed[2])
    assert np.array_equal(alone[1], mixed[5])
    assert ralone[0]["iterations"] == rmixed[2]["iterations"]
    assert ralone[1]["iterations"] == rmixed[5]["iterations"]
    for p, x in zip(others, [mixed[0], mixed[1], mixed[3], mixed[4], mixed[6]]):
        assert oracle_relres(p, x) <= RES_TOL


def test_budget_admission_and_release():
    from meltpooldg_b200 import MpdgError
    from meltpooldg_b200 import _capi
    B = _B()
    p = heat(6, 2, seed=1)
    nb = p.bytes()
    with B.Batch(int(nb * 2.5), capacity=8) as bt:
        t1 = bt.submit(p)
        t2 = bt.submit(p)
        assert bt.used_bytes == 2 * nb
        with pytest.raises(MpdgError) as e:
            bt.submit(p)
        assert e.value.status == _capi.ERR_BUDGET
        assert bt.try_submit(p) is None
        bt.run()
        x1, _ = bt.take(t1, p.n_dofs)
        assert bt.used_bytes == nb
        t3 = bt.submit(p)  # memory freed by take is admitted again
        bt.run()
        x2, _ = bt.take(t2, p.n_dofs)
        x3, _ = bt.take(t3, p.n_dofs)
        assert bt.used_bytes == 0
    assert np.array_equal(x1, x2) and np.array_equal(x1, x3)


def test_autotune_keeps_results():
    B = _B()
    ps = [heat(6, 2, seed=41), heat(4, 4, seed=42), advdiff(5, 3, seed=43)]
    ref, _ = B.solve_batch(ps)
    with B.Batch(10**10, capacity=8) as bt:
        ts = [bt.submit(p) for p in ps]
        cap, ms = bt.autotune()
        assert cap in (0, 1, 2, 3, 4, 6, 8) and ms > 0
        shape = bt.shape()
        assert shape["warps_per_cta"] in (2, 4, 8) and shape["ctas_per_sm"] == cap
        assert shape["tile_layout"] in ("conflict-minimal", "plain")
        bt.run()
        got = [bt.take(t, p.n_dofs)[0] for t, p in zip(ts, ps)]
    for a, b in zip(ref, got):
        assert np.array_equal(a, b)


def test_serve_results_equal_alone():
    """Requests arriving over time, admitted while others run, give the same
    solutions as each problem alone."""
    B = _B()
    rng = np.random.default_rng(5)
    probs = []
    for i in range(14):
        if i % 2:
            probs.append(advdiff(int(rng.integers(3, 7)), int(rng.integers(2, 5)), seed=100 + i))
        else:
            probs.append(heat(int(rng.integers(3, 8)), int(rng.integers(2, 5)),
                              k0=float(np.exp(rng.uniform(0, np.log(100)))), seed=100 + i))
    arrivals = np.cumsum(rng.exponential(0.01, size=len(probs)))
    budget = int(sum(p.bytes() for p in probs) * 0.4)  # forces waiting for memory
    budget = max(budget, max(p.bytes() for p in probs))
    with B.Batch(budget, capacity=6) as bt:
        out = bt.serve(probs, arrivals, poll_steps=2, keep_solutions=True)
    assert all(r["status"] == 0 for r in out["reports"])
    assert np.all(out["latency_s"] > 0)
    for i, p in enumerate(probs):
        (x,), (r,) = B.solve_batch([p])
        assert np.array_equal(out["solutions"][i], x), i
        assert out["reports"][i]["iterations"] == r["iterations"]
        assert out["x_norm"][i] == pytest.approx(np.linalg.norm(x), rel=1e-12)
    for i in (0, 1):
        assert oracle_relres(probs[i], out["solutions"][i]) <= RES_TOL
