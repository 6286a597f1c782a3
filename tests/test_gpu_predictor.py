"""Multi-vector apply (mpdg_vmult_multi) and the least-squares-projection
predictor (mpdg_predict_lsq, predictor.hpp:37-80) on the device.

* every vector of a multi-vector apply equals its own vmult (the same cell
  arithmetic; FP64 and FP32, merged-stream and uniform kernels, Dirichlet
  masks, passes of 4 and a remainder, and the per-vector fallback for
  operators with faces);
* the predictor matches the oracle's restatement (1e-9) with the same number
  of old solutions used, also when a dependent old solution stops it."""
import numpy as np
import pytest

from gpu_helpers import dev, meshes, relerr, rng
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _ops(kind, p):
    import meltpooldg_b200 as M
    nc = (5, 4, 3)
    mask = M.boundary_mask(nc, p, faces=[(0, 0), (1, 1)])
    if kind == "heat_general_kT":
        gm, om = meshes(nc, p, 0.1, seed=3, mask=mask)
        op = M.HeatDiffuseOperator(gm, 1e-3, rho_cp=2.0, k0=1.5, k_alpha=1e-3, precisions=("fp64", "fp32"))
        T = rng(4).uniform(300, 3000, gm.n_dofs)
        op.set_temperature(dev(T))
        oop = O.Operator(O.HEAT, 1e-3, rho_cp=2.0, k0=1.5, k_alpha=1e-3, temperature=T, dirichlet=mask)
        return gm, om, op, oop, T
    if kind == "advdiff_uniform":
        gm, om = meshes(nc, p, 0.0, seed=3, mask=mask, lo=(-1, -1, -1), hi=(1, 1, 1))
        op = M.AdvectionDiffusionOperator(gm, 1e-3, theta=0.5, diffusivity=1e-3, velocity="vortex",
                                          precisions=("fp64", "fp32"))
        oop = O.Operator(O.ADVDIFF, 1e-3, theta=0.5, diffusivity=1e-3, vel_kind=O.VEL_VORTEX, dirichlet=mask)
        return gm, om, op, oop, None
    gm, om = meshes(nc, p, 0.1, seed=3, mask=mask)
    op = M.HeatDiffuseOperator(gm, 1e-3, rho_cp=2.0, k0=1.5, robin_alpha=3.0, robin_t_inf=1.0,
                               robin_faces=[(2, 1)], precisions=("fp64", "fp32"))
    oop = O.Operator(O.HEAT, 1e-3, rho_cp=2.0, k0=1.5, robin_alpha=3.0, robin_t_inf=1.0, robin_faces=1 << 5,
                     dirichlet=mask)
    return gm, om, op, oop, None


@pytest.mark.parametrize("p", [1, 2, 4])
@pytest.mark.parametrize("kind", ["heat_general_kT", "advdiff_uniform", "heat_robin_fallback"])
@pytest.mark.parametrize("nvec", [2, 4, 5])
def test_vmult_multi_equals_single_applies(cuda, p, kind, nvec):
    import torch
    gm, om, op, oop, _ = _ops(kind, p)
    R = rng(10 + nvec)
    for dtype in (torch.float64, torch.float32):
        srcs = [dev(R.uniform(-1, 1, gm.n_dofs), dtype) for _ in range(nvec)]
        dsts = [torch.empty_like(s) for s in srcs]
        op.vmult_multi(dsts, srcs)
        for s, d in zip(srcs, dsts):
            one = torch.empty_like(s)
            op.vmult(one, s)
            assert relerr(d.double().cpu().numpy(), one.double().cpu().numpy()) <= 1e-14
    # and against the oracle in FP64
    x = R.uniform(-1, 1, gm.n_dofs)
    y = R.uniform(-1, 1, gm.n_dofs)
    d0, d1 = torch.empty(gm.n_dofs, dtype=torch.float64, device="cuda"), torch.empty(gm.n_dofs,
                                                                                    dtype=torch.float64,
                                                                                    device="cuda")
    op.vmult_multi([d0, d1], [dev(x), dev(y)])
    assert relerr(d0.cpu().numpy(), O.vmult(om, oop, x)) < 1e-12
    assert relerr(d1.cpu().numpy(), O.vmult(om, oop, y)) < 1e-12


def test_vmult_multi_rejects_overlap(cuda):
    import torch
    gm, om, op, oop, _ = _ops("heat_general_kT", 2)
    a = dev(np.ones(gm.n_dofs))
    b = torch.empty_like(a)
    with pytest.raises(Exception, match="overlap"):
        op.vmult_multi([a, b], [a, b])


@pytest.mark.parametrize("p", [1, 2, 4])
@pytest.mark.parametrize("kind", ["heat_general_kT", "advdiff_uniform"])
def test_predictor_matches_oracle(cuda, p, kind):
    import torch
    import meltpooldg_b200 as M
    gm, om, op, oop, _ = _ops(kind, p)
    R = rng(30 + p)
    old = [R.uniform(-1, 1, gm.n_dofs) for _ in range(5)]
    b = R.uniform(-1, 1, gm.n_dofs)
    x_ref, used_ref = O.lsq_projection(om, oop, old, b)
    x = torch.empty(gm.n_dofs, dtype=torch.float64, device="cuda")
    lsp = M.LeastSquaresProjection([dev(v) for v in old])
    used = lsp.vmult(op, x, dev(b))
    assert used == used_ref == 5
    assert relerr(x.cpu().numpy(), x_ref) < 1e-9
    # a right-hand side in the image of the span is predicted exactly
    c = np.array([0.3, -1.1, 0.7, 2.0, -0.4])
    xt = sum(ci * v for ci, v in zip(c, old))
    lsp.vmult(op, x, dev(O.vmult(om, oop, xt)))
    assert relerr(x.cpu().numpy(), xt) < 1e-9


def test_predictor_stops_at_dependent_solution(cuda):
    import torch
    import meltpooldg_b200 as M
    gm, om, op, oop, _ = _ops("heat_general_kT", 2)
    R = rng(40)
    a, b_ = R.uniform(-1, 1, gm.n_dofs), R.uniform(-1, 1, gm.n_dofs)
    old = [a, b_, a - 2.0 * b_, R.uniform(-1, 1, gm.n_dofs)]
    rhs = R.uniform(-1, 1, gm.n_dofs)
    x_ref, used_ref = O.lsq_projection(om, oop, old, rhs)
    x = torch.empty(gm.n_dofs, dtype=torch.float64, device="cuda")
    used = M.LeastSquaresProjection([dev(v) for v in old]).vmult(op, x, dev(rhs))
    assert used == used_ref == 2
    assert relerr(x.cpu().numpy(), x_ref) < 1e-9
