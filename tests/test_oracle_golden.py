"""The CPU oracle against the reference's own golden outputs and against
itself (two independent evaluation routes).  No GPU needed."""
import json
import os

import numpy as np
import pytest

from oracle import cases
from oracle import oracle as O

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_outputs.json")))

# The reference prints ||phi||_L2 through VectorTools::integrate_difference, which
# stores per-cell norms in a Vector<float> (source/utilities/vector_tools.cpp:151)
# and sums them in float: its 11 printed digits carry float noise of a few 1e-8.
VORTEX_RTOL = 5e-8


@pytest.mark.parametrize("name,dim,refinements", [
    ("advection_diffusion_vortex_mf", 2, 5),
    ("advection_diffusion_vortex", 2, 5),
    ("advection_diffusion_vortex_mf_3d", 3, 3),
])
def test_vortex_golden(name, dim, refinements):
    got = cases.vortex_case(dim, refinements)
    ref = GOLDEN[name]["values"]
    assert len(got) == len(ref) == 5
    for g, r in zip(got, ref):
        assert abs(g - r) / r < VORTEX_RTOL, (g, r)


@pytest.mark.parametrize("name,dim,refinements", [
    ("advection_diffusion_vortex_mf_inflow_outflow", 2, 5),
    ("advection_diffusion_vortex_mf_inflow_outflow_3d", 3, 3),
])
def test_vortex_inflow_outflow_golden(name, dim, refinements):
    """Inflow/outflow constraints: every boundary DoF with u . n <= 0 is fixed
    to -1 after each solve (advection_diffusion_operation.cpp:371-499)."""
    got = cases.vortex_case(dim, refinements, inflow_outflow=True)
    ref = GOLDEN[name]["values"]
    assert len(got) == len(ref) == 5
    for g, r in zip(got, ref):
        assert abs(g - r) / r < VORTEX_RTOL, (g, r)


def test_vortex_supg_golden():
    """SUPG stabilisation with the automatic parameter h_K / max_q |u|
    (advection_diffusion_operator.cpp:450-533)."""
    got = cases.vortex_case(2, 5, supg=True)
    ref = GOLDEN["advection_diffusion_vortex_mf_supg"]["values"]
    assert len(got) == len(ref) == 5
    for g, r in zip(got, ref):
        assert abs(g - r) / r < VORTEX_RTOL, (g, r)


def _fmt(v):
    return "%.5e" % v


def test_unidirectional_heat_golden():
    got = cases.unidirectional_heat_case()
    assert [_fmt(v) for v in got] == GOLDEN["unidirectional_heat_transfer"]["printed"]


@pytest.mark.parametrize("name", sorted(cases.HEAT_CASES))
def test_unidirectional_heat_phase_laws_and_radiation_golden(name):
    """Radiative faces, velocity, gas/liquid and liquid/solid material laws
    (material.templates.hpp:213-760; heat_diffuse_operator.cpp:719-778, 955-1129)."""
    got = cases.unidirectional_heat_case(**cases.HEAT_CASES[name])
    printed = GOLDEN[name]["printed"]
    assert len(got) == len(printed) == 5
    for g, p in zip(got, printed):
        assert cases.printed_match(g, p), (name, g, p)


def test_unidirectional_heat_convection_golden():
    got = cases.unidirectional_heat_case(dt=0.01, k=55.563, rho=7850.0, cp=460.0, convection=25.0)
    assert [_fmt(v) for v in got] == GOLDEN["unidirectional_heat_transfer_with_convection"]["printed"]


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_sum_factorisation_equals_element_matrices(dim, p):
    rng = np.random.Generator(np.random.PCG64(10 * dim + p))
    m = O.Mesh.box(dim, p, [3, 2, 2][:dim], perturb=0.1, seed=1)
    T = rng.uniform(300, 3000, m.n_dofs)
    vel = rng.uniform(-1, 1, (dim, m.n_dofs))
    mask = m.boundary_face_mask([(0, 0)])
    ops = [
        O.Operator(O.HEAT, 1e-3, rho_cp=2.0, k0=1.5, k_alpha=1e-3, temperature=T, dirichlet=mask),
        O.Operator(O.HEAT, 1e-3, rho_cp=2.0, k0=1.5, k_alpha=1e-3, temperature=T, full_tangent=True,
                   vel_kind=O.VEL_NODAL, vel_nodal=vel, robin_alpha=3.0, robin_faces=0b10),
        O.Operator(O.ADVDIFF, 1e-3, theta=0.5, diffusivity=1e-3, vel_kind=O.VEL_VORTEX, dirichlet=mask),
    ]
    for op in ops:
        u = rng.uniform(-1, 1, m.n_dofs)
        a = O.vmult(m, op, u)
        b = O.vmult(m, op, u, brute=True)
        assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()


def test_diagonal_equals_unit_vector_sweeps():
    m = O.Mesh.box(3, 2, [2, 2, 1], perturb=0.1, seed=3)
    rng = np.random.Generator(np.random.PCG64(5))
    T = rng.uniform(300, 3000, m.n_dofs)
    mask = m.boundary_face_mask([(2, 1)])
    op = O.Operator(O.HEAT, 1e-3, k0=2.0, k_alpha=1e-3, temperature=T, dirichlet=mask,
                    vel_kind=O.VEL_CONST, vel_param=(1.0, -2.0, 0.5))
    d = O.diagonal(m, op)
    e = np.array([O.vmult(m, op, np.eye(1, m.n_dofs, i)[0])[i] for i in range(m.n_dofs)])
    e[mask == 1] = 1.0
    assert np.abs(d - e).max() <= 1e-13 * np.abs(e).max()


def test_mass_row_sums_give_volume():
    """1^T M 1 / dt = |Omega| rho_cp / dt for the mass-only heat operator."""
    m = O.Mesh.box(3, 3, [3, 2, 2], perturb=0.1, seed=7)
    op = O.Operator(O.HEAT, 0.5, rho_cp=3.0, k0=0.0)
    one = np.ones(m.n_dofs)
    assert abs(O.vmult(m, op, one).sum() - 3.0 / 0.5) < 1e-12


def test_linear_field_has_no_interior_stiffness():
    """A linear field is in the kernel of the Laplacian rows away from the boundary."""
    m = O.Mesh.box(3, 2, [4, 4, 4], perturb=0.1, seed=8)
    x = m.dof_coordinates()
    op = O.Operator(O.HEAT, 1.0, rho_cp=0.0, k0=1.0)
    r = O.vmult(m, op, 1.0 + 2.0 * x[:, 0] - x[:, 1] + 0.5 * x[:, 2])
    gi = m.grid_index()
    interior = np.all((gi > 0) & (gi < np.array(m.shape) - 1), axis=1)
    assert np.abs(r[interior]).max() < 1e-12


def test_cg_and_gmres_reach_tolerance():
    m = O.Mesh.box(3, 2, [6, 6, 6])
    mask = m.boundary_face_mask()
    op = O.Operator(O.HEAT, 1e-3, k0=1.0, dirichlet=mask)
    rng = np.random.Generator(np.random.PCG64(1))
    xs = rng.uniform(-1, 1, m.n_dofs)
    xs[mask == 1] = 0
    b = O.vmult(m, op, xs)
    inv = O.inverse_diagonal(m, op)
    x, it, hist, ok = O.cg(m, op, b, inv_diag=inv, rel_tol=1e-10)
    assert ok and hist[-1] <= 1e-10 * hist[0]
    assert np.abs(x - xs).max() < 1e-8
    x2, it2, hist2, ok2 = O.gmres(m, op, b, inv_diag=inv, rel_tol=1e-10)
    assert ok2 and np.abs(x2 - xs).max() < 1e-8
    lam = O.lambda_max(m, op, inv, rng.uniform(-1, 1, m.n_dofs) * (1 - mask))
    x3, it3, hist3, ok3 = O.cg(m, op, b, inv_diag=inv, rel_tol=1e-10,
                               chebyshev={"degree": 5, "lambda_min": lam / 30, "lambda_max": 1.2 * lam})
    assert ok3 and it3 < it and np.abs(x3 - xs).max() < 1e-8


def test_oracle_nodal_velocity_of_a_constant_field_equals_the_constant_velocity():
    """The oracle's velocity-as-a-DoF-vector path (ORC_VEL_NODAL, the field
    interpolated to the quadrature points) against its prescribed constant
    velocity on perturbed cells: the two operators agree to rounding."""
    import numpy as np
    from oracle import oracle as O
    nc, p = (3, 4, 2), 3
    V = O.box_vertices(3, nc, (0, 0, 0), (1, 1, 1), 0.1, 5)
    om = O.Mesh(3, p, nc, V)
    vel = (0.3, -0.2, 0.7)
    U = np.concatenate([np.full(om.n_dofs, v) for v in vel])
    src = np.random.Generator(np.random.PCG64(1)).uniform(-1, 1, om.n_dofs)
    for kind in (O.HEAT, O.ADVDIFF):
        a = O.vmult(om, O.Operator(kind, 1e-2, theta=0.5, diffusivity=1e-2, vel_kind=O.VEL_CONST, vel_param=vel), src)
        b = O.vmult(om, O.Operator(kind, 1e-2, theta=0.5, diffusivity=1e-2, vel_kind=O.VEL_NODAL, vel_nodal=U), src)
        assert np.abs(a - b).max() <= 1e-13 * np.abs(a).max()
