"""CPU checks of the oracle's heat material laws and radiative faces
(material.templates.hpp:213-760, heat_diffuse_operator.cpp:719-778, 955-1129):

* the Newton tangent is the Jacobian of the residual: for every law (the k(T)
  law with its full tangent, gas/liquid, liquid/solid in the mushy zone,
  gas/liquid/solid with smooth and sharp interfaces, volume-specific capacity)
  with velocity, convective and radiative faces, central differences of
  create_rhs match the apply;
* the mass row sum is the law's rho c_p / dt times the volume, with rho c_p
  from an independent restatement of the law here;
* the apply equals the brute-force element matrices and the diagonal equals
  probing.
"""
import numpy as np
import pytest

from oracle import oracle as O

GLS = dict(rho=(3925.0, 7850.0, 7000.0), cp=(230.0, 460.0, 700.0), k=(27.7815, 55.563, 17.0),
           solidus=1966.0, liquidus=1974.0)
LAWS = {
    "linear_full": None,
    "gas_liquid": dict(GLS, kind=O.MAT_GAS_LIQUID),
    "gas_liquid_vol": dict(GLS, kind=O.MAT_GAS_LIQUID, volume_specific=True),
    "liquid_solid": dict(GLS, kind=O.MAT_LIQUID_SOLID),
    "liquid_solid_vol": dict(GLS, kind=O.MAT_LIQUID_SOLID, volume_specific=True),
    "gas_liquid_solid": dict(GLS, kind=O.MAT_GAS_LIQUID_SOLID),
    "gas_liquid_solid_sharp": dict(GLS, kind=O.MAT_GAS_LIQUID_SOLID, two_phase_sharp=True),
}


def _fields(m, seed):
    R = np.random.default_rng(seed)
    x = m.dof_coordinates()
    T = 1970.0 + 2.5 * np.sin(3.0 * x[:, 0] + 1.0) * np.cos(2.0 * x[:, 1]) + R.uniform(-0.2, 0.2, m.n_dofs)
    T_old = T + R.uniform(-0.5, 0.5, m.n_dofs)
    H = 0.5 + 0.45 * np.sin(4.0 * x[:, 0] - 2.0 * x[:, 1])
    return T, T_old, H


def _op(law, dim, T, T_old, H):
    kw = dict(rho_cp=3.0e6, k0=20.0, k_alpha=1e-3, full_tangent=law is None, material=law,
              robin_alpha=25.0, robin_t_inf=300.0, robin_faces=(1 << 1) | (1 << 2),
              rad_emissivity=0.9, rad_t_inf=350.0, rad_faces=(1 << 1) | (1 << 3),
              vel_kind=O.VEL_CONST, vel_param=(0.3, -0.2, 0.1)[:dim] + (0.0,) * (3 - dim))
    return O.Operator(O.HEAT, 0.01, temperature=T, temperature_old=T_old, heaviside=H, **kw)


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("law", list(LAWS))
def test_tangent_is_jacobian_of_residual(dim, law):
    m = O.Mesh.box(dim, 2, [3] * dim, perturb=0.1, seed=2)
    T, T_old, H = _fields(m, 3)
    op = _op(LAWS[law], dim, T, T_old, H)
    v = np.random.default_rng(4).uniform(-1, 1, m.n_dofs)
    Av = O.vmult(m, op, v)
    eps = 1e-3
    rp = O.rhs_heat(m, op.with_temperature(T + eps * v), T_old)
    rm = O.rhs_heat(m, op.with_temperature(T - eps * v), T_old)
    fd = (rm - rp) / (2.0 * eps)
    assert np.linalg.norm(fd - Av) <= 1e-6 * np.linalg.norm(Av), law


def _law_rho_cp(law, T, H):
    """rho c_p of a phase law at one (T, H), restated from material.templates.hpp."""
    fs = min(max((law["liquidus"] - T) / (law["liquidus"] - law["solidus"]), 0.0), 1.0)
    cub = lambda a, b: a + (b - a) * (3.0 * fs ** 2 - 2.0 * fs ** 3)  # noqa: E731
    sol = law["kind"] in (O.MAT_LIQUID_SOLID, O.MAT_GAS_LIQUID_SOLID)
    gas = law["kind"] in (O.MAT_GAS_LIQUID, O.MAT_GAS_LIQUID_SOLID)
    w = (1.0 if H > 0.5 else 0.0) if law.get("two_phase_sharp") else H
    rho, cp = law["rho"], law["cp"]
    if law.get("volume_specific"):
        rc = [rho[i] * cp[i] for i in range(3)]
        v = cub(rc[1], rc[2]) if sol else rc[1]
        return (1 - w) * rc[0] + w * v if gas else v
    r = cub(rho[1], rho[2]) if sol else rho[1]
    c = cub(cp[1], cp[2]) if sol else cp[1]
    if gas:
        r, c = (1 - w) * rho[0] + w * r, (1 - w) * cp[0] + w * c
    return r * c


@pytest.mark.parametrize("law", [k for k in LAWS if k != "linear_full"])
@pytest.mark.parametrize("T0,H0", [(1969.3, 0.3), (1972.1, 0.8), (1960.0, 0.6), (1990.0, 0.45)])
def test_mass_row_sum_is_law_capacity(law, T0, H0):
    m = O.Mesh.box(3, 2, [3, 3, 3], perturb=0.1, seed=5)
    N = m.n_dofs
    op = O.Operator(O.HEAT, 0.01, material=LAWS[law], temperature=np.full(N, T0),
                    temperature_old=np.full(N, T0), heaviside=np.full(N, H0))
    got = O.vmult(m, op, np.ones(N)).sum()
    want = _law_rho_cp(LAWS[law], T0, H0) / 0.01
    assert abs(got - want) <= 1e-12 * want


@pytest.mark.parametrize("law", list(LAWS))
def test_material_apply_matches_element_matrices_and_diagonal(law):
    m = O.Mesh.box(3, 2, [2, 3, 2], perturb=0.1, seed=6)
    T, T_old, H = _fields(m, 7)
    op = _op(LAWS[law], 3, T, T_old, H)
    u = np.random.default_rng(8).uniform(-1, 1, m.n_dofs)
    a, b = O.vmult(m, op, u), O.vmult(m, op, u, brute=True)
    assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max()
    d = O.diagonal(m, op)
    for i in range(0, m.n_dofs, max(1, m.n_dofs // 12)):
        e = np.zeros(m.n_dofs)
        e[i] = 1.0
        assert abs(O.vmult(m, op, e)[i] - d[i]) <= 1e-12 * abs(d[i])
