"""CPU checks of the oracle's SUPG terms (advection_diffusion_operator.cpp:276-358,
450-533) by known answers that need no implementation detail:

* with a constant velocity u = (1, 0, 0) on the unit box of cubes of edge h,
  tau_K = h (automatic parameter h_K / max |u|, h_K = diameter / sqrt(dim)),
  and for phi = x^2 and the test function w = x (u . grad w = 1) the SUPG part
  of w^T A phi is  h * int (phi/dt + theta u.grad phi - theta D lap phi)
  = h (1/(3 dt) + theta - 2 theta D);  the right-hand side's SUPG part is
  h * int (phi/dt - (1-theta) u.grad phi + (1-theta) D lap phi)
  = h (1/(3 dt) - (1-theta) + 2 (1-theta) D);
* the sum-factorised apply equals the brute-force element matrices (which
  take the Laplacian of each basis function from second derivatives rather than
  by differentiating interpolated gradients), and the diagonal equals probing;
* coefficient 0 switches the stabilisation off.
"""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("p", [2, 3])
@pytest.mark.parametrize("D", [0.0, 0.05])
def test_supg_known_answer(dim, p, D):
    nc = [4] * dim
    m = O.Mesh.box(dim, p, nc, lo=[0.0] * dim, hi=[1.0] * dim)
    h, dt, th = 0.25, 1e-2, 0.5
    x = m.dof_coordinates()
    phi, w = x[:, 0] ** 2, x[:, 0].copy()
    kw = dict(theta=th, diffusivity=D, vel_kind=O.VEL_CONST, vel_param=(1.0, 0.0, 0.0))
    a_s = O.Operator(O.ADVDIFF, dt, supg=True, **kw)
    a_0 = O.Operator(O.ADVDIFF, dt, **kw)
    got = w @ (O.vmult(m, a_s, phi) - O.vmult(m, a_0, phi))
    want = h * (1.0 / (3.0 * dt) + th - 2.0 * th * D)
    assert abs(got - want) <= 1e-12 * abs(want)
    got_rhs = w @ (O.rhs_advdiff(m, a_s, phi) - O.rhs_advdiff(m, a_0, phi))
    want_rhs = h * (1.0 / (3.0 * dt) - (1.0 - th) + 2.0 * (1.0 - th) * D)
    assert abs(got_rhs - want_rhs) <= 1e-12 * abs(want_rhs)


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("perturb,D", [(0.0, 0.05), (0.1, 0.0)])
@pytest.mark.parametrize("coef", [-1.0, 0.7])
def test_supg_apply_matches_element_matrices(dim, p, perturb, D, coef):
    m = O.Mesh.box(dim, p, [3] * dim if dim == 3 else [4, 4], perturb=perturb, seed=3)
    op = O.Operator(O.ADVDIFF, 1e-2, theta=0.5, diffusivity=D, vel_kind=O.VEL_VORTEX, supg=True,
                    supg_coefficient=coef)
    u = np.random.default_rng(p).uniform(-1, 1, m.n_dofs)
    a, b = O.vmult(m, op, u), O.vmult(m, op, u, brute=True)
    assert np.abs(a - b).max() <= 1e-13 * np.abs(a).max()
    d = O.diagonal(m, op)
    for i in range(0, m.n_dofs, max(1, m.n_dofs // 15)):
        e = np.zeros(m.n_dofs)
        e[i] = 1.0
        assert abs(O.vmult(m, op, e)[i] - d[i]) <= 1e-13 * abs(d[i])


def test_supg_coefficient_zero_is_plain():
    m = O.Mesh.box(3, 2, [3, 3, 3], perturb=0.1, seed=1)
    kw = dict(theta=0.5, diffusivity=0.0, vel_kind=O.VEL_VORTEX)
    u = np.random.default_rng(0).uniform(-1, 1, m.n_dofs)
    a = O.vmult(m, O.Operator(O.ADVDIFF, 1e-2, supg=True, supg_coefficient=0.0, **kw), u)
    b = O.vmult(m, O.Operator(O.ADVDIFF, 1e-2, **kw), u)
    assert np.array_equal(a, b)
