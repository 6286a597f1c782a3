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
  probing;
* the latent heat of fusion (apparent capacity, each profile) satisfies the
  reference's own unit-test properties (unit_tests/heat/apparent_capacity.cpp):
  the poly4_bell profile and its derivative vanish at solidus and liquidus,
  every profile integrates to the latent heat over the mushy zone (midpoint
  rule, 1000 steps, 1e-8), and the T derivative matches central differences.
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
    # latent heat of fusion through the apparent capacity, each profile
    "liquid_solid_latent_qlq": dict(GLS, kind=O.MAT_LIQUID_SOLID, latent_heat=2.7e5, apparent_capacity=O.AC_QLQ),
    "liquid_solid_latent_bell": dict(GLS, kind=O.MAT_LIQUID_SOLID, latent_heat=2.7e5,
                                     apparent_capacity=O.AC_POLY4_BELL),
    "gas_liquid_solid_latent_const": dict(GLS, kind=O.MAT_GAS_LIQUID_SOLID, latent_heat=2.7e5,
                                          apparent_capacity=O.AC_CONSTANT),
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


def _qlq_reference_form(x, x1, x2, y1, y2, delta):
    """The quadratic-linear-quadratic ramp in the polynomial-coefficient form of
    apparent_capacity.cpp (qlq_zero_slope)."""
    den = delta + x1 - x2
    a1 = (y1 - y2) / (2.0 * delta * den)
    b1 = -x1 * (y1 - y2) / (delta * den)
    c1 = (2 * delta * delta * y1 + 2 * delta * x1 * y1 - 2 * delta * x2 * y1 + x1 * x1 * y1 - x1 * x1 * y2) / (
        2 * delta * den)
    b2 = x2 * (y1 - y2) / (delta * den)
    c2 = (2 * delta * delta * y2 + 2 * delta * x1 * y2 - 2 * delta * x2 * y2 - x2 * x2 * y1 + x2 * x2 * y2) / (
        2 * delta * den)
    a3 = (y1 - y2) / den
    b3 = (delta * y1 + delta * y2 + 2 * x1 * y2 - 2 * x2 * y1) / (2 * den)
    if x < x1 + delta:
        return a1 * x * x + b1 * x + c1
    if x > x2 - delta:
        return -a1 * x * x + b2 * x + c2
    return a3 * x + b3


def _apparent_capacity(law, fs):
    """ApparentCapacity::evaluate (apparent_capacity.cpp), restated here."""
    L = law.get("latent_heat", 0.0)
    if L <= 0.0 or fs <= 0.0 or fs >= 1.0:
        return 0.0
    Ts, Tl = law["solidus"], law["liquidus"]
    dT = Tl - Ts
    kind = law.get("apparent_capacity", O.AC_QLQ)
    if kind == O.AC_CONSTANT:
        return L / dT
    if kind == O.AC_POLY4_BELL:
        xi = 1.0 - 2.0 * fs
        return L * (2.0 / dT) * (15.0 / 16.0 * xi ** 4 - 15.0 / 8.0 * xi ** 2 + 15.0 / 16.0)
    T, Tp, Cp = Tl - fs * dT, 0.5 * (Ts + Tl), 2.0 * L / dT
    return (_qlq_reference_form(T, Ts, Tp, 0.0, Cp, dT / 6.0) if T <= Tp
            else _qlq_reference_form(T, Tp, Tl, Cp, 0.0, dT / 6.0))


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
    c = cub(cp[1], cp[2]) + _apparent_capacity(law, fs) if sol else cp[1]
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
    # the reference's polynomial-coefficient form of the qlq ramp cancels about
    # six digits at T ~ 2000 K; the oracle evaluates it about the ramp's ends
    tol = 1e-9 if "latent_qlq" in law else 1e-12
    assert abs(got - want) <= tol * want


@pytest.mark.parametrize("law", list(LAWS))
def test_material_apply_matches_element_matrices_and_diagonal(law):
    m = O.Mesh.box(3, 2, [2, 3, 2], perturb=0.1, seed=6)
    T, T_old, H = _fields(m, 7)
    op = _op(LAWS[law], 3, T, T_old, H)
    u = np.random.default_rng(8).uniform(-1, 1, m.n_dofs)
    a, b = O.vmult(m, op, u), O.vmult(m, op, u, brute=True)
    # the apparent capacity makes c_p 100x larger in the mushy zone and the
    # mass term dominate the entries: the sums round a few ulps further
    tol = 1e-11 if "latent" in law else 1e-12
    assert np.abs(a - b).max() <= tol * np.abs(a).max()
    d = O.diagonal(m, op)
    for i in range(0, m.n_dofs, max(1, m.n_dofs // 12)):
        e = np.zeros(m.n_dofs)
        e[i] = 1.0
        assert abs(O.vmult(m, op, e)[i] - d[i]) <= tol * abs(d[i])


AC_MATERIAL = dict(kind=O.MAT_LIQUID_SOLID, rho=(1.0, 1.0, 1.0), cp=(1.0, 1.0, 1.0), k=(1.0, 1.0, 1.0),
                   solidus=271.0, liquidus=275.0, latent_heat=338e3)


def _ac_op(kind):
    return O.Operator(O.HEAT, 0.01, material=dict(AC_MATERIAL, apparent_capacity=kind))


@pytest.mark.parametrize("kind", [O.AC_POLY4_BELL, O.AC_CONSTANT, O.AC_QLQ])
def test_apparent_capacity_reference_properties(kind):
    op = _ac_op(kind)
    Ts, Tl, L = AC_MATERIAL["solidus"], AC_MATERIAL["liquidus"], AC_MATERIAL["latent_heat"]
    if kind == O.AC_POLY4_BELL:
        for T in (Ts, Tl):
            c, dc = O.apparent_capacity(op, T)
            assert abs(c) <= 1e-6 and abs(dc) <= 1e-6
    steps = 1000
    h = (Tl - Ts) / steps
    integral = sum(O.apparent_capacity(op, Ts + (i + 0.5) * h)[0] for i in range(steps)) * h
    assert abs(integral - L) / L <= 1e-8
    eps, T = 1e-5, Ts + 0.1
    for _ in range(3):
        want = (O.apparent_capacity(op, T + eps)[0] - O.apparent_capacity(op, T - eps)[0]) / (2 * eps)
        got = O.apparent_capacity(op, T)[1]
        assert abs(got - want) <= 1e-5 * max(1.0, abs(want)), T
        T += (Tl - Ts) / 5.0
    # outside the mushy zone nothing is added
    assert O.apparent_capacity(op, Ts - 1.0) == (0.0, 0.0)
    assert O.apparent_capacity(op, Tl + 1.0) == (0.0, 0.0)


def test_apparent_capacity_matches_reference_coefficient_form():
    """The oracle evaluates each qlq ramp about its ends; the reference's
    coefficient form a x^2 + b x + c at x ~ 273 K cancels about six digits, so
    the two agree to 1e-10 of the peak capacity (absolute), not to the ulp."""
    op = _ac_op(O.AC_QLQ)
    law = dict(AC_MATERIAL, apparent_capacity=O.AC_QLQ)
    peak = 2.0 * AC_MATERIAL["latent_heat"] / 4.0
    for T in np.linspace(271.01, 274.99, 57):
        fs = (275.0 - T) / 4.0
        want = _apparent_capacity(law, fs)
        assert abs(O.apparent_capacity(op, T)[0] - want) <= 1e-10 * peak, T
