"""CPU checks of the oracle's hanging-node (two-level mesh) operator.

Known answers, independent of any implementation detail:
* the hanging interpolation reproduces every coarse polynomial of degree p
  (the constraint weights are the coarse Lagrange basis at the fine nodes);
* the constrained operator is symmetric and writes nothing at hanging DoFs;
* a global linear field lies in the kernel of the interior Laplacian rows
  (the constrained space is conforming);
* the constrained mass matrix sums to the volume (partition of unity);
* the diagonal equals unit-vector probing.
"""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.mark.parametrize("p", [1, 2, 3])
def test_hanging_interpolation_reproduces_coarse_polynomials(p):
    m2 = O.Mesh2(p, (2, 2, 2), 2)
    x = m2.dof_coordinates()
    hm = m2.hanging_mask().astype(bool)
    u = x[:, 1] ** p + 0.3 * x[:, 2] ** p * x[:, 1] ** (p - 1) - 2.0 * x[:, 2]
    ud = O.distribute2(m2, np.where(hm, 0.0, u))
    assert np.abs(ud[hm] - u[hm]).max() < 1e-13
    P = O.hanging_matrix(p)
    assert np.allclose(P.sum(axis=2), 1.0, atol=1e-14)  # partition of unity per fine node


@pytest.mark.parametrize("p", [1, 2, 3])
def test_hanging_operator_properties(p):
    m2 = O.Mesh2(p, (2, 2, 2), 2, perturb=0.1, seed=3)
    hm = m2.hanging_mask().astype(bool)
    N = m2.n_dofs
    R = np.random.default_rng(p)
    a, b = R.uniform(-1, 1, N), R.uniform(-1, 1, N)
    a[hm] = b[hm] = 0.0
    op = O.Operator(O.HEAT, 1e-2, rho_cp=2.0, k0=1.5)
    Aa, Ab = O.vmult2(m2, op, a), O.vmult2(m2, op, b)
    assert abs(b @ Aa - a @ Ab) <= 1e-13 * abs(b @ Aa)
    assert np.all(Aa[hm] == 0.0)
    # mass only: the constrained basis sums to one, so 1^T M 1 is the volume
    mass = O.Operator(O.HEAT, 1.0, rho_cp=1.0, k0=0.0)
    one = np.where(hm, 0.0, 1.0)
    assert abs(O.vmult2(m2, mass, one).sum() - 1.0) < 1e-12
    # diagonal = unit-vector probing
    d = O.diagonal2(m2, op)
    for i in np.flatnonzero(~hm)[:: max(1, N // 25)]:
        e = np.zeros(N)
        e[i] = 1.0
        assert abs(O.vmult2(m2, op, e)[i] - d[i]) <= 1e-13 * abs(d[i])


@pytest.mark.parametrize("p", [1, 2, 3])
def test_linear_field_in_kernel_of_interior_rows(p):
    m2 = O.Mesh2(p, (2, 2, 2), 2, perturb=0.1, seed=4)
    hm = m2.hanging_mask().astype(bool)
    bd = m2.boundary_face_mask().astype(bool)
    x = m2.dof_coordinates()
    lap = O.Operator(O.HEAT, 1e300, rho_cp=0.0, k0=1.0)
    u = np.where(hm, 0.0, 1.0 + 2.0 * x[:, 0] - x[:, 1] + 0.5 * x[:, 2])
    r = O.vmult2(m2, lap, u)
    assert np.abs(r[~bd & ~hm]).max() < 1e-12
