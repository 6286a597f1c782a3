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
* coefficient 0 switches the stabilisation off;
* on perturbed (non-affine) cells the SUPG Laplacian is the physical one, the
  map's curvature included: with u = (1, 0, 0), w = x and the Laplacian term
  isolated by the difference of two diffusivities, an interpolated linear
  function has Laplacian 0 and a physical quadratic (exact in Q2 and Q3 under
  a trilinear map) its constant; the tau-weighted cell volumes come from
  phi = 1, whose Laplacian and gradient vanish.
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
@pytest.mark.parametrize("perturb,D", [(0.0, 0.05), (0.1, 0.0), (0.15, 0.05)])
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


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("p", [2, 3])
@pytest.mark.parametrize("coef", [-1.0, 0.6])
def test_supg_laplacian_on_perturbed_cells_known_answer(dim, p, coef):
    nc = [3] * dim
    m = O.Mesh.box(dim, p, nc, lo=[0.0] * dim, hi=[1.0] * dim, perturb=0.2, seed=11)
    x = m.dof_coordinates()
    dt, th, D1, D2 = 1e-2, 0.5, 0.3, 0.1
    w = x[:, 0].copy()

    def supg_part(D, phi):
        kw = dict(theta=th, diffusivity=D, vel_kind=O.VEL_CONST, vel_param=(1.0, 0.0, 0.0))
        return w @ (O.vmult(m, O.Operator(O.ADVDIFF, dt, supg=True, supg_coefficient=coef, **kw), phi) -
                    O.vmult(m, O.Operator(O.ADVDIFF, dt, **kw), phi))

    # sum_K tau_K |K| (u.grad w = 1): phi = 1 leaves only phi/dt in the residual
    one = np.ones(m.n_dofs)
    tau_vol = dt * supg_part(D1, one)
    assert tau_vol > 0.0
    if dim == 3:
        lin = 0.3 * x[:, 0] - 1.2 * x[:, 1] + 0.7 * x[:, 2]
        quad, lap = x[:, 0] ** 2 + 2 * x[:, 1] ** 2 + 3 * x[:, 2] ** 2 + x[:, 0] * x[:, 1] + x[:, 1] * x[:, 2], 12.0
    else:
        lin = 0.3 * x[:, 0] - 1.2 * x[:, 1]
        quad, lap = x[:, 0] ** 2 + 2 * x[:, 1] ** 2 + x[:, 0] * x[:, 1], 6.0
    scale = abs(supg_part(D1, quad))
    # the Laplacian term alone: -theta (D1 - D2) sum_K tau_K int_K lap phi
    got_lin = supg_part(D1, lin) - supg_part(D2, lin)
    assert abs(got_lin) <= 1e-12 * scale
    got = supg_part(D1, quad) - supg_part(D2, quad)
    want = -th * (D1 - D2) * lap * tau_vol
    assert abs(got - want) <= 1e-11 * abs(want)
    # the sum-factorised apply and the element matrices agree on these cells
    op = O.Operator(O.ADVDIFF, dt, theta=th, diffusivity=D1, vel_kind=O.VEL_VORTEX, supg=True,
                    supg_coefficient=coef)
    u = np.random.default_rng(p).uniform(-1, 1, m.n_dofs)
    a, b = O.vmult(m, op, u), O.vmult(m, op, u, brute=True)
    assert np.abs(a - b).max() <= 1e-13 * np.abs(a).max()
