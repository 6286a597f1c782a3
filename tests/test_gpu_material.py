"""Heat material laws and radiative faces on the device against the oracle:
the gas/liquid, liquid/solid and gas/liquid/solid laws with their Newton terms
(T_old and heaviside fields), convective plus radiative faces and velocity
(vmult and create_rhs FP64 to 1e-12, FP32 to 2e-5; the diagonal to 1e-12), and
the reference's unidirectional heat-transfer goldens with radiation, velocity,
two phases and solidification through the CUDA path.  The laws with a solid
phase also run with the latent heat of fusion (apparent capacity: qlq,
constant and poly4_bell profiles)."""
import json
import os

import numpy as np
import pytest

from gpu_helpers import dev, meshes, relerr
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-5

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_outputs.json")))

PHASES = dict(rho=(3925.0, 7850.0, 7000.0), cp=(230.0, 460.0, 700.0), k=(27.7815, 55.563, 17.0),
              solidus=1966.0, liquidus=1974.0)
LAWS = {
    "gas_liquid": (dict(PHASES, kind="gas_liquid"), O.MAT_GAS_LIQUID),
    "gas_liquid_vol_sharp": (dict(PHASES, kind="gas_liquid", volume_specific=True, two_phase_sharp=True),
                             O.MAT_GAS_LIQUID),
    "liquid_solid": (dict(PHASES, kind="liquid_solid"), O.MAT_LIQUID_SOLID),
    "liquid_solid_sharp": (dict(PHASES, kind="liquid_solid", solid_liquid_sharp=True), O.MAT_LIQUID_SOLID),
    "gas_liquid_solid": (dict(PHASES, kind="gas_liquid_solid"), O.MAT_GAS_LIQUID_SOLID),
    # latent heat of fusion through the apparent capacity, each profile
    "liquid_solid_latent_qlq": (dict(PHASES, kind="liquid_solid", latent_heat=2.7e5, apparent_capacity=O.AC_QLQ),
                                O.MAT_LIQUID_SOLID),
    "liquid_solid_latent_const": (dict(PHASES, kind="liquid_solid", latent_heat=2.7e5,
                                       apparent_capacity=O.AC_CONSTANT), O.MAT_LIQUID_SOLID),
    "gas_liquid_solid_latent_bell": (dict(PHASES, kind="gas_liquid_solid", latent_heat=2.7e5,
                                          apparent_capacity=O.AC_POLY4_BELL), O.MAT_GAS_LIQUID_SOLID),
}


def _fields(om, seed):
    R = np.random.default_rng(seed)
    x = om.dof_coordinates()
    T = 1970.0 + 5.0 * np.sin(3.0 * x[:, 0] + 1.0) * np.cos(2.0 * x[:, 1]) + R.uniform(-0.5, 0.5, om.n_dofs)
    T_old = T + R.uniform(-0.5, 0.5, om.n_dofs)
    H = 0.5 + 0.45 * np.sin(4.0 * x[:, 0] - 2.0 * x[:, 2])
    return T, T_old, H


def _oracle_material(mat, kind):
    m = {k: v for k, v in mat.items() if k != "kind"}
    m["kind"] = kind
    return m


@pytest.mark.parametrize("p", [1, 2, 4])
@pytest.mark.parametrize("perturb", [0.0, 0.1])
@pytest.mark.parametrize("law", sorted(LAWS))
def test_material_law_parity(cuda, p, perturb, law):
    import torch
    import meltpooldg_b200 as M
    nc = (3, 4, 3)
    mask = M.boundary_mask(nc, p, faces=[(2, 0)])
    gm, om = meshes(nc, p, perturb, seed=5 + p, mask=mask)
    T, T_old, H = _fields(om, 11 + p)
    mat, okind = LAWS[law]
    faces = dict(robin_alpha=25.0, robin_t_inf=300.0, rad_emissivity=0.9, rad_t_inf=350.0)
    op = M.HeatDiffuseOperator(gm, 0.01, velocity=(0.3, -0.2, 0.1), precisions=("fp64", "fp32"),
                               robin_faces=[(0, 1), (1, 0)], rad_faces=[(0, 1), (1, 1)], material=mat, **faces)
    Td, Od, Hd = dev(T), dev(T_old), dev(H)
    op.set_temperature(Td)
    op.set_temperature_old(Od)
    op.set_heaviside(Hd)
    oop = O.Operator(O.HEAT, 0.01, temperature=T, temperature_old=T_old, heaviside=H, dirichlet=mask,
                     robin_faces=(1 << 1) | (1 << 2), rad_faces=(1 << 1) | (1 << 3),
                     vel_kind=O.VEL_CONST, vel_param=(0.3, -0.2, 0.1),
                     material=_oracle_material(mat, okind), **faces)
    src = np.random.default_rng(20 + p).uniform(-1, 1, gm.n_dofs)
    ref = O.vmult(om, oop, src)
    dst = torch.empty(gm.n_dofs, dtype=torch.float64, device="cuda")
    op.vmult(dst, dev(src))
    assert relerr(dst.cpu().numpy(), ref) < TOL64
    d32 = torch.empty(gm.n_dofs, dtype=torch.float32, device="cuda")
    op.vmult(d32, dev(src, torch.float32))
    assert relerr(d32.double().cpu().numpy(), ref) < TOL32
    diag = torch.empty_like(dst)
    op.compute_diagonal(diag)
    assert relerr(diag.cpu().numpy(), O.diagonal(om, oop)) < TOL64
    rhs = torch.zeros_like(dst)
    op.create_rhs(rhs, Od)
    # the residual subtracts T_old from T at the points (|T| / |T - T_old| ~ 4e3 here):
    # its rounding is measured against the size of its terms, the residual at T_old = 0
    ref = O.rhs_heat(om, oop, T_old, scatter_mask=mask)
    scale = np.abs(O.rhs_heat(om, oop, np.zeros_like(T_old), scatter_mask=mask)).max()
    assert np.abs(rhs.cpu().numpy() - ref).max() < TOL64 * scale


def test_material_law_needs_its_fields(cuda):
    import torch
    import meltpooldg_b200 as M
    gm, om = meshes((2, 2, 2), 2)
    op = M.HeatDiffuseOperator(gm, 0.01, material=LAWS["gas_liquid_solid"][0])
    T = dev(np.full(gm.n_dofs, 1970.0))
    op.set_temperature(T)
    dst = torch.empty_like(T)
    with pytest.raises(Exception, match="T_old"):
        op.vmult(dst, T)
    op.set_temperature_old(T)
    with pytest.raises(Exception, match="heaviside"):
        op.vmult(dst, T)
    op.set_heaviside(dev(np.full(gm.n_dofs, 0.5)))
    op.vmult(dst, T)


def test_radiation_needs_temperature(cuda):
    import torch
    import meltpooldg_b200 as M
    gm, _ = meshes((2, 2, 2), 1)
    op = M.HeatDiffuseOperator(gm, 0.01, rad_emissivity=0.5, rad_t_inf=300.0, rad_faces=[(0, 0)])
    x = dev(np.ones(gm.n_dofs))
    with pytest.raises(Exception, match="temperature"):
        op.vmult(torch.empty_like(x), x)


@pytest.mark.parametrize("name", [
    "unidirectional_heat_transfer_with_radiation",
    "unidirectional_heat_transfer_with_radiation_and_convection",
    "unidirectional_heat_transfer_with_velocity",
    "unidirectional_heat_transfer_with_two_phase",
    "unidirectional_heat_transfer_with_two_phase_rho_times_cp",
    "unidirectional_heat_transfer_with_velocity_and_solidification",
    "unidirectional_heat_transfer_with_two_phase_and_solidification",
])
def test_unidirectional_heat_golden_on_gpu(cuda, name):
    """The 2D case (Q1, 32^2 on [0,0.1]^2) extruded to one layer of hexahedra
    of unit depth: convective/radiative faces at x = 0.1, velocity (-v, 0, 0),
    the heaviside of the case's level set re-interpolated each step; the
    solution is z-independent, so the 3D L2 norm equals the 2D one."""
    import meltpooldg_b200 as M
    from meltpooldg_b200.operations import HeatDiffuseOperation
    from oracle import cases
    c = dict(cases.HEAT_CASES[name])
    nc = (32, 32, 1)
    V = M.box_vertices(nc, (0.0, 0.0, 0.0), (0.1, 0.1, 1.0))
    mesh = M.Mesh(V, nc, 1)
    X = np.tile(np.linspace(0.0, 0.1, 33), 33 * 2)
    Y = np.tile(np.repeat(np.linspace(0.0, 0.1, 33), 33), 2)
    v = c.get("velocity", 0.0)
    kw = {}
    if c.get("material"):
        om = dict(c["material"])
        om["kind"] = {O.MAT_GAS_LIQUID: "gas_liquid", O.MAT_LIQUID_SOLID: "liquid_solid",
                      O.MAT_GAS_LIQUID_SOLID: "gas_liquid_solid"}[om["kind"]]
        kw["material"] = om
    else:
        kw.update(rho_cp=c["rho"] * c["cp"], k0=c["k"])
    if c.get("convection", 0.0) > 0.0:
        kw.update(robin_alpha=c["convection"], robin_t_inf=300.0, robin_faces=[(0, 1)])
    if c.get("emissivity", 0.0) > 0.0:
        kw.update(rad_emissivity=c["emissivity"], rad_t_inf=300.0, rad_faces=[(0, 1)])
    if v != 0.0:
        kw["velocity"] = (-v, 0.0, 0.0)
    if c.get("two_phase"):
        if c.get("solidification"):
            kw["heaviside"] = lambda t: cases.smoothed_heaviside(0.1 * 2.0 / 3.0 - X - v * t, 0.01)
        else:
            kw["heaviside"] = lambda t: cases.smoothed_heaviside(0.05 - Y, 0.01)
    opn = HeatDiffuseOperation(mesh, c["dt"], residual_tolerance=c.get("residual_tolerance", 5e-9),
                               linear_solver=M.LinearSolverData(rel_tolerance=1e-12), **kw)
    if c.get("solidification"):
        T0 = 1960.0 + 20.0 * X / 0.1
    elif c.get("convection", 0.0) > 0.0 or c.get("emissivity", 0.0) > 0.0:
        T0 = np.full(mesh.n_dofs, 1000.0)
    else:
        T0 = X.copy()
    opn.set_initial_condition(T0)
    for printed in GOLDEN[name]["printed"]:
        opn.solve()
        assert cases.printed_match(opn.l2_norm(), printed), (opn.l2_norm(), printed)


def test_latent_heat_refusals(cuda):
    import meltpooldg_b200 as M
    nc = (2, 2, 2)
    gm, _ = meshes(nc, 2, 0.0)
    with pytest.raises(Exception, match="volume-specific"):
        M.HeatDiffuseOperator(gm, 1e-3, material=dict(PHASES, kind="liquid_solid", volume_specific=True,
                                                       latent_heat=1e5))
    with pytest.raises(Exception, match="latent heat"):
        M.HeatDiffuseOperator(gm, 1e-3, material=dict(PHASES, kind="liquid_solid", latent_heat=-1.0))
    with pytest.raises(Exception, match="apparent capacity profile"):
        M.HeatDiffuseOperator(gm, 1e-3, material=dict(PHASES, kind="liquid_solid", latent_heat=1e5,
                                                       apparent_capacity=7))
