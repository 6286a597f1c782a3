"""CPU checks of the oracle's least-squares-projection predictor
(predictor.hpp:37-80) by known answers: a right-hand side that is the image
of a combination of the old solutions is predicted exactly; a dependent old
solution stops the recurrence; the prediction minimises |A x - b| over the
span (normal equations)."""
import numpy as np

from oracle import oracle as O


def _setup(k, seed):
    m = O.Mesh.box(3, 2, [3, 3, 3], perturb=0.1, seed=seed)
    op = O.Operator(O.HEAT, 1e-2, rho_cp=2.0, k0=1.5)
    R = np.random.default_rng(seed)
    return m, op, [R.uniform(-1, 1, m.n_dofs) for _ in range(k)], R


def test_lsq_reproduces_a_combination():
    m, op, old, R = _setup(4, 1)
    c = np.array([0.5, -1.25, 2.0, 0.75])
    x_true = sum(ci * xi for ci, xi in zip(c, old))
    x, used = O.lsq_projection(m, op, old, O.vmult(m, op, x_true))
    assert used == 4
    assert np.abs(x - x_true).max() <= 1e-10 * np.abs(x_true).max()


def test_lsq_stops_at_a_dependent_solution():
    m, op, old, R = _setup(3, 2)
    old = old[:2] + [old[0] - 2.0 * old[1]] + [R.uniform(-1, 1, m.n_dofs)]
    x, used = O.lsq_projection(m, op, old, R.uniform(-1, 1, m.n_dofs))
    assert used == 2


def test_lsq_satisfies_normal_equations():
    m, op, old, R = _setup(3, 3)
    b = R.uniform(-1, 1, m.n_dofs)
    x, used = O.lsq_projection(m, op, old, b)
    r = O.vmult(m, op, x) - b
    for xi in old:
        w = O.vmult(m, op, xi)
        assert abs(w @ r) <= 1e-10 * np.linalg.norm(w) * np.linalg.norm(b)
