"""Locally refined meshes (meltpooldg_b200.refine.refine_box) with face and edge
hanging nodes, checked on the CPU oracle by known answers: the constraints
reproduce every polynomial of degree p, the constrained heat operator is
symmetric, its mass sums to the volume, and linear fields lie in the kernel of
the interior Laplace rows.  Perturbed coarse vertices included."""
import numpy as np
import pytest

from meltpooldg_b200.refine import refine_box
from oracle import oracle as O

PATTERNS = {"column": [13, 4, 22], "corner_L": [0, 1, 3], "single": [13]}


def _mesh(p, pattern, perturb):
    nc = (3, 3, 3)
    V = O.box_vertices(3, nc, [0.0] * 3, [1.0] * 3, perturb, 7) if perturb else None
    r = refine_box(nc, p, PATTERNS[pattern], vertices=V)
    mm = O.MappedMesh(p, r["cell_vertices"], r["cell_dofs"], r["n_dofs"], r["constraints"])
    return r, mm


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("pattern", sorted(PATTERNS))
@pytest.mark.parametrize("perturb", [0.0, 0.1])
def test_refined_mesh_known_answers(p, pattern, perturb):
    r, mm = _mesh(p, pattern, perturb)
    x = r["coordinates"]
    cm = mm.constrained_mask().astype(bool)
    assert cm.sum() > 0
    if perturb == 0.0:  # on affine cells the interpolant of a polynomial of degree p is exact
        f = x[:, 0] ** p + 0.3 * x[:, 1] ** p * x[:, 2] - x[:, 2] ** p + 0.1
        for g, ent in r["constraints"].items():
            assert abs(sum(w * f[m] for m, w in ent) - f[g]) < 1e-12
    # trilinear fields are interpolated exactly on any mesh
    f1 = 1.0 + 2.0 * x[:, 0] - x[:, 1] + 0.5 * x[:, 2]
    for g, ent in r["constraints"].items():
        assert abs(sum(w * f1[m] for m, w in ent) - f1[g]) < 1e-12
    heat = O.Operator(O.HEAT, 1e-2, rho_cp=2.0, k0=1.5)
    R = np.random.default_rng(p)
    a, b = R.uniform(-1, 1, mm.n_dofs), R.uniform(-1, 1, mm.n_dofs)
    a[cm] = b[cm] = 0.0
    Aa, Ab = O.mapped_vmult(mm, heat, a), O.mapped_vmult(mm, heat, b)
    assert abs(b @ Aa - a @ Ab) <= 1e-13 * abs(b @ Aa)
    mass = O.Operator(O.HEAT, 1.0, rho_cp=1.0, k0=0.0)
    assert abs(O.mapped_vmult(mm, mass, np.where(cm, 0.0, 1.0)).sum() - 1.0) < 1e-12
    lap = O.Operator(O.HEAT, 1e300, rho_cp=0.0, k0=1.0)
    rr = O.mapped_vmult(mm, lap, np.where(cm, 0.0, f1))
    interior = ~(r["boundary"].astype(bool) | cm)
    assert np.abs(rr[interior]).max() < 1e-12
