"""Mapped meshes (mpdg_mesh_create_mapped, the ingestion form of an
unstructured mesh) on the device against the oracle's mapped operator:
vmult (FP64 1e-12, FP32 2e-5) and the diagonal (1e-12) on structured meshes
handed over with a random DoF numbering and cell order, and on the two-level
mesh handed over with its hanging-node constraints; equal to the structured
and two-level device paths on the same meshes; CG iteration counts as the
oracle's; create_rhs as the structured path's."""
import numpy as np
import pytest

from gpu_helpers import dev, meshes, relerr, rng
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-5


def device_mesh(mm, mask):
    import meltpooldg_b200 as M
    return M.MappedMesh(mm.cell_vertices, mm.cell_dofs, mm.n_dofs, mm.degree, dirichlet_mask=mask,
                        constraints=mm.constraints)


def _ops(gm, kind, mask, prec=("fp64", "fp32")):
    import meltpooldg_b200 as M
    if kind == "heat":
        return (M.HeatDiffuseOperator(gm, 1e-2, rho_cp=2.0, k0=1.5, precisions=prec),
                O.Operator(O.HEAT, 1e-2, rho_cp=2.0, k0=1.5, dirichlet=mask))
    return (M.AdvectionDiffusionOperator(gm, 1e-2, theta=0.5, diffusivity=0.05, velocity="vortex", precisions=prec),
            O.Operator(O.ADVDIFF, 1e-2, theta=0.5, diffusivity=0.05, vel_kind=O.VEL_VORTEX, dirichlet=mask))


@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("kind", ["heat", "advdiff"])
def test_mapped_structured_renumbered(cuda, p, kind):
    import torch
    import meltpooldg_b200 as M
    nc = (3, 4, 2)
    mask_s = M.boundary_mask(nc, p, faces=[(0, 0), (1, 1)])
    gs, om = meshes(nc, p, 0.1, seed=p, mask=mask_s, lo=(-1, -1, -1), hi=(1, 1, 1))
    R = rng(50 + p)
    perm = R.permutation(om.n_dofs)
    mm = O.mapped_from_mesh(om, perm=perm, cell_order=R.permutation(om.n_cells))
    mask = np.empty_like(mask_s)
    mask[perm] = mask_s
    gm = device_mesh(mm, mask)
    op, oop = _ops(gm, kind, mask)
    x = R.uniform(-1, 1, om.n_dofs)
    ref = O.mapped_vmult(mm, oop, x)
    y = torch.empty(om.n_dofs, dtype=torch.float64, device="cuda")
    op.vmult(y, dev(x))
    assert relerr(y.cpu().numpy(), ref) < TOL64
    y32 = torch.empty(om.n_dofs, dtype=torch.float32, device="cuda")
    op.vmult(y32, dev(x, torch.float32))
    assert relerr(y32.double().cpu().numpy(), ref) < TOL32
    d = torch.empty_like(y)
    op.compute_diagonal(d)
    assert relerr(d.cpu().numpy(), O.mapped_diagonal(mm, oop)) < TOL64
    # the structured path on the same mesh, renumbered
    ops, _ = _ops(gs, kind, mask_s, prec=("fp64",))
    xs = x[perm]
    ys = torch.empty_like(y)
    ops.vmult(ys, dev(xs))
    assert relerr(y.cpu().numpy()[perm], ys.cpu().numpy()) < TOL64


@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("kind", ["heat", "advdiff"])
def test_mapped_hanging_constraints(cuda, p, kind):
    import torch
    import meltpooldg_b200 as M
    m2 = O.Mesh2(p, (2, 2, 2), 2, perturb=0.1, seed=20 + p)
    mask = m2.boundary_face_mask()
    mm = O.mapped_from_mesh2(m2)
    gm = device_mesh(mm, mask)
    op, oop = _ops(gm, kind, mask)
    x = rng(60 + p).uniform(-1, 1, m2.n_dofs)
    ref = O.mapped_vmult(mm, oop, x)
    y = torch.empty(m2.n_dofs, dtype=torch.float64, device="cuda")
    op.vmult(y, dev(x))
    assert relerr(y.cpu().numpy(), ref) < TOL64
    assert relerr(ref, O.vmult2(m2, oop, x)) < 1e-14
    y32 = torch.empty(m2.n_dofs, dtype=torch.float32, device="cuda")
    op.vmult(y32, dev(x, torch.float32))
    assert relerr(y32.double().cpu().numpy(), ref) < TOL32
    d = torch.empty_like(y)
    op.compute_diagonal(d)
    assert relerr(d.cpu().numpy(), O.mapped_diagonal(mm, oop)) < TOL64
    # the two-level device path on the same mesh
    nc_f = (2, 4, 4)
    gt = M.TwoLevelMesh(m2.coarse.vert, (2, 2, 2), m2.fine.vert, nc_f, p, mask[:m2.n_coarse], mask[m2.n_coarse:])
    ot, _ = _ops(gt, kind, mask, prec=("fp64",))
    yt = torch.empty_like(y)
    ot.vmult(yt, dev(x))
    assert relerr(y.cpu().numpy(), yt.cpu().numpy()) < TOL64


@pytest.mark.parametrize("p", [2, 3])
def test_mapped_cg_iterations_match_oracle(cuda, p):
    import torch
    import meltpooldg_b200 as M
    m2 = O.Mesh2(p, (2, 3, 2), 2, perturb=0.1, seed=30 + p)
    mask = m2.boundary_face_mask()
    mm = O.mapped_from_mesh2(m2)
    gm = device_mesh(mm, mask)
    op, oop = _ops(gm, "heat", mask, prec=("fp64",))
    fixed = mm.constrained_mask().astype(bool) | mask.astype(bool)
    R = rng(70 + p)
    xs = R.uniform(-1, 1, m2.n_dofs)
    xs[fixed] = 0.0
    b = O.mapped_vmult(mm, oop, xs)
    inv = 1.0 / O.mapped_diagonal(mm, oop)
    x, r = np.zeros_like(b), b.copy()
    z = inv * r
    pdir, rz, res0, its_ref = z.copy(), r @ z, np.linalg.norm(b), 0
    for it in range(1, 2000):
        Ap = O.mapped_vmult(mm, oop, pdir)
        alpha = rz / (pdir @ Ap)
        x += alpha * pdir
        r -= alpha * Ap
        if np.linalg.norm(r) <= 1e-10 * res0:
            its_ref = it
            break
        z = inv * r
        rz_new = r @ z
        pdir = z + (rz_new / rz) * pdir
        rz = rz_new
    xd = torch.zeros(m2.n_dofs, dtype=torch.float64, device="cuda")
    its = M.LinearSolver.solve(op, xd, dev(b), M.LinearSolverData(solver_type="CG", preconditioner_type="Diagonal",
                                                                  rel_tolerance=1e-10, abs_tolerance=0.0))
    assert abs(its - its_ref) <= 1, (its, its_ref)
    assert np.linalg.norm(xd.cpu().numpy() - x) <= 1e-8 * np.linalg.norm(x)


def test_mapped_rhs_equals_structured(cuda):
    import torch
    import meltpooldg_b200 as M
    p, nc = 2, (3, 3, 3)
    gs, om = meshes(nc, p, 0.1, seed=4, lo=(-1, -1, -1), hi=(1, 1, 1))
    perm = rng(80).permutation(om.n_dofs)
    gm = device_mesh(O.mapped_from_mesh(om, perm=perm), None)
    ops, _ = _ops(gs, "advdiff", None, prec=("fp64",))
    opm, _ = _ops(gm, "advdiff", None, prec=("fp64",))
    phi = rng(81).uniform(-1, 1, om.n_dofs)
    rs = torch.zeros(om.n_dofs, dtype=torch.float64, device="cuda")
    ops.create_rhs(rs, dev(phi))
    phim = np.empty_like(phi)
    phim[perm] = phi
    rm = torch.zeros_like(rs)
    opm.create_rhs(rm, dev(phim))
    assert relerr(rm.cpu().numpy()[perm], rs.cpu().numpy()) < TOL64


def test_mapped_rejects_chained_constraints(cuda):
    import meltpooldg_b200 as M
    om = O.Mesh.box(3, 1, [2, 1, 1])
    mm = O.mapped_from_mesh(om)
    with pytest.raises(Exception, match="masters"):
        M.MappedMesh(mm.cell_vertices, mm.cell_dofs, mm.n_dofs, 1, constraints={0: [(1, 1.0)], 1: [(2, 1.0)]})


def test_vortex_3d_golden_through_a_mapped_mesh(cuda):
    """advection_diffusion_vortex_mf_3d (Q1, 8^3 cells on [-1,1]^3, CN, GMRES +
    Diagonal) with the mesh handed over in the ingestion form, DoFs renumbered
    at random and cells shuffled: operator, lifting, rhs, solver and integrated
    norm all run through the cell->DoF map."""
    import json
    import os
    import meltpooldg_b200 as M
    from meltpooldg_b200.operations import AdvectionDiffusionOperation
    from oracle import cases
    golden = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_outputs.json")))
    om, phi0, mask0 = cases.vortex_setup(3, 3)
    R = rng(90)
    perm = R.permutation(om.n_dofs)
    mm = O.mapped_from_mesh(om, perm=perm, cell_order=R.permutation(om.n_cells))
    mask = np.empty_like(mask0)
    mask[perm] = mask0
    phi = np.empty_like(phi0)
    phi[perm] = phi0
    gm = device_mesh(mm, mask)
    opn = AdvectionDiffusionOperation(gm, 0.01, theta=0.5, diffusivity=0.0, velocity=("rotation", 4.0),
                                      dirichlet_values=np.full(gm.n_dofs, -1.0))
    opn.set_initial_condition(phi)
    for r in golden["advection_diffusion_vortex_mf_3d"]["values"]:
        opn.solve()
        assert abs(opn.l2_norm() - r) / r < 5e-8


@pytest.mark.parametrize("law", ["kT_full", "liquid_solid"])
def test_mapped_field_dependent_heat_equals_structured(cuda, law):
    """k(T) with its full tangent, and the liquid/solid law, on a mapped mesh
    (no constraints): vmult, the diagonal and the Newton residual equal the
    structured path's on the same mesh with the DoFs renumbered."""
    import torch
    import meltpooldg_b200 as M
    p, nc = 2, (3, 4, 3)
    gs, om = meshes(nc, p, 0.1, seed=6)
    R = rng(91)
    perm = R.permutation(om.n_dofs)
    gm = device_mesh(O.mapped_from_mesh(om, perm=perm, cell_order=R.permutation(om.n_cells)), None)
    x = om.dof_coordinates()
    T = 1970.0 + 4.0 * np.sin(3.0 * x[:, 0]) * np.cos(2.0 * x[:, 1]) + R.uniform(-0.3, 0.3, om.n_dofs)
    T_old = T + R.uniform(-0.5, 0.5, om.n_dofs)
    if law == "kT_full":
        kw = dict(rho_cp=2.0, k0=1.5, k_alpha=1e-3, full_tangent=True, velocity=(0.3, -0.2, 0.1))
    else:
        kw = dict(velocity=(0.3, -0.2, 0.1), material=dict(kind="liquid_solid", rho=(0, 7850, 7000),
                                                           cp=(0, 460, 700), k=(0, 55.563, 17.0),
                                                           solidus=1966.0, liquidus=1974.0))
    ops = M.HeatDiffuseOperator(gs, 0.01, **kw)
    opm = M.HeatDiffuseOperator(gm, 0.01, **kw)

    def renum(v):
        out = np.empty_like(v)
        out[perm] = v
        return out

    Ts, Os = dev(T), dev(T_old)
    Tm, Om = dev(renum(T)), dev(renum(T_old))
    ops.set_temperature(Ts)
    ops.set_temperature_old(Os)
    opm.set_temperature(Tm)
    opm.set_temperature_old(Om)
    u = R.uniform(-1, 1, om.n_dofs)
    ys, ym = torch.empty_like(Ts), torch.empty_like(Ts)
    ops.vmult(ys, dev(u))
    opm.vmult(ym, dev(renum(u)))
    assert relerr(ym.cpu().numpy()[perm], ys.cpu().numpy()) < TOL64
    ops.compute_diagonal(ys)
    opm.compute_diagonal(ym)
    assert relerr(ym.cpu().numpy()[perm], ys.cpu().numpy()) < TOL64
    rs, rm = torch.zeros_like(Ts), torch.zeros_like(Ts)
    ops.create_rhs(rs, Os)
    opm.create_rhs(rm, Om)
    scale = np.abs(rs.cpu().numpy()).max() + 1.0
    assert np.abs(rm.cpu().numpy()[perm] - rs.cpu().numpy()).max() < 1e-10 * scale


def test_solidification_golden_through_a_mapped_mesh(cuda):
    """unidirectional_heat_transfer_with_velocity_and_solidification (liquid/solid
    mushy zone, velocity 0.005) on the 2D case extruded to one layer, handed over
    as a mapped mesh with renumbered DoFs: Newton with the law's tangent, the
    residual and the integrated norm through the cell->DoF map."""
    import json
    import os
    import meltpooldg_b200 as M
    from meltpooldg_b200.operations import HeatDiffuseOperation
    from oracle import cases
    golden = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_outputs.json")))
    name = "unidirectional_heat_transfer_with_velocity_and_solidification"
    c = cases.HEAT_CASES[name]
    nc = (32, 32, 1)
    om = O.Mesh(3, 1, nc, M.box_vertices(nc, (0.0, 0.0, 0.0), (0.1, 0.1, 1.0)))
    perm = rng(92).permutation(om.n_dofs)
    gm = device_mesh(O.mapped_from_mesh(om, perm=perm), None)
    mat = dict(c["material"])
    mat["kind"] = "liquid_solid"
    opn = HeatDiffuseOperation(gm, c["dt"], residual_tolerance=c["residual_tolerance"],
                               linear_solver=M.LinearSolverData(rel_tolerance=1e-12), material=mat,
                               velocity=(-c["velocity"], 0.0, 0.0))
    X = om.dof_coordinates()[:, 0]
    T0 = np.empty(om.n_dofs)
    T0[perm] = 1960.0 + 20.0 * X / 0.1
    opn.set_initial_condition(T0)
    for printed in golden[name]["printed"]:
        opn.solve()
        assert cases.printed_match(opn.l2_norm(), printed), (opn.l2_norm(), printed)


@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("kind", ["heat", "advdiff"])
def test_locally_refined_mesh(cuda, p, kind):
    """A 3^3 mesh with a column of refined cells (face and edge hanging nodes,
    perturbed coarse vertices) through refine_box: vmult, FP32 and the
    diagonal against the oracle's mapped operator."""
    import torch
    from meltpooldg_b200.refine import refine_box
    V = O.box_vertices(3, (3, 3, 3), [-1.0] * 3, [1.0] * 3, 0.1, 11)
    r = refine_box((3, 3, 3), p, [13, 4, 22], vertices=V)
    mm = O.MappedMesh(p, r["cell_vertices"], r["cell_dofs"], r["n_dofs"], r["constraints"])
    mask = r["boundary"]
    gm = device_mesh(mm, mask)
    op, oop = _ops(gm, kind, mask)
    x = rng(100 + p).uniform(-1, 1, mm.n_dofs)
    ref = O.mapped_vmult(mm, oop, x)
    y = torch.empty(mm.n_dofs, dtype=torch.float64, device="cuda")
    op.vmult(y, dev(x))
    assert relerr(y.cpu().numpy(), ref) < TOL64
    y32 = torch.empty(mm.n_dofs, dtype=torch.float32, device="cuda")
    op.vmult(y32, dev(x, torch.float32))
    assert relerr(y32.double().cpu().numpy(), ref) < TOL32
    d = torch.empty_like(y)
    op.compute_diagonal(d)
    assert relerr(d.cpu().numpy(), O.mapped_diagonal(mm, oop)) < TOL64


def test_mapped_inflow_outflow_identity_rows(cuda):
    """Identity rows (do_pre_vmult / do_post_vmult,
    advection_diffusion_operator.cpp:537-578) on a mapped mesh with a random
    DoF numbering and hanging-node constraints: src read as 0 at the flagged
    DoFs, the result there equal to src, the inverse diagonal 1 there."""
    import torch
    import meltpooldg_b200 as M
    from meltpooldg_b200.refine import refine_box
    p = 2
    V = O.box_vertices(3, (3, 3, 3), [-1.0] * 3, [1.0] * 3, 0.1, 12)
    r = refine_box((3, 3, 3), p, [13, 4], vertices=V)
    mm = O.MappedMesh(p, r["cell_vertices"], r["cell_dofs"], r["n_dofs"], r["constraints"])
    gm = device_mesh(mm, None)
    R = rng(88)
    io = (R.uniform(size=mm.n_dofs) < 0.2).astype(np.uint8)
    io[mm.constrained_mask().astype(bool)] = 0
    op, oop = _ops(gm, "advdiff", None)
    src = R.uniform(-1, 1, mm.n_dofs)
    ref = O.mapped_vmult(mm, oop, np.where(io == 1, 0.0, src))
    ref[io == 1] = src[io == 1]
    op.set_inflow_outflow(io)
    d_src = dev(src)
    dst = torch.empty_like(d_src)
    op.vmult(dst, d_src)
    assert relerr(dst.cpu().numpy(), ref) < TOL64
    assert torch.equal(d_src, dev(src))
    d32 = torch.empty(mm.n_dofs, dtype=torch.float32, device="cuda")
    op.vmult(d32, dev(src, torch.float32))
    assert relerr(d32.double().cpu().numpy(), ref) < TOL32
    inv = torch.empty_like(d_src)
    op.compute_inverse_diagonal_from_matrixfree(inv)
    d = O.mapped_diagonal(mm, oop)
    thr = 1e-14 * max(1.0, np.abs(d).max())
    want = np.where(np.abs(d) > thr, 1.0 / np.where(d == 0, 1.0, d), 1.0)
    want[io == 1] = 1.0
    got = inv.cpu().numpy()
    free = mm.constrained_mask() == 0
    assert relerr(got[free], want[free]) < TOL64


def _supg_ops(gm, mask, coef):
    import meltpooldg_b200 as M
    return (M.AdvectionDiffusionOperator(gm, 1e-2, theta=0.5, diffusivity=0.05, velocity="vortex",
                                         precisions=("fp64", "fp32"), supg=True, supg_coefficient=coef),
            O.Operator(O.ADVDIFF, 1e-2, theta=0.5, diffusivity=0.05, vel_kind=O.VEL_VORTEX, dirichlet=mask,
                       supg=True, supg_coefficient=coef))


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("coef", [-1.0, 0.7])
def test_mapped_supg_renumbered(cuda, p, coef):
    """SUPG with diffusion (tau_K from the cell's corners, the Laplacian with
    the map's curvature) through a mapped mesh with a random numbering: vmult
    (FP64, FP32) and the element-matrix diagonal against the oracle's mapped
    operator; create_rhs as the structured device path's."""
    import torch
    import meltpooldg_b200 as M
    nc = (3, 2, 3)
    mask_s = M.boundary_mask(nc, p, faces=[(1, 0)])
    gs, om = meshes(nc, p, 0.15, seed=30 + p, mask=mask_s, lo=(-1, -1, -1), hi=(1, 1, 1))
    R = rng(60 + p)
    perm = R.permutation(om.n_dofs)
    mm = O.mapped_from_mesh(om, perm=perm, cell_order=R.permutation(om.n_cells))
    mask = np.empty_like(mask_s)
    mask[perm] = mask_s
    gm = device_mesh(mm, mask)
    op, oop = _supg_ops(gm, mask, coef)
    x = R.uniform(-1, 1, om.n_dofs)
    ref = O.mapped_vmult(mm, oop, x)
    y = torch.empty(om.n_dofs, dtype=torch.float64, device="cuda")
    op.vmult(y, dev(x))
    assert relerr(y.cpu().numpy(), ref) < TOL64
    y32 = torch.empty(om.n_dofs, dtype=torch.float32, device="cuda")
    op.vmult(y32, dev(x, torch.float32))
    assert relerr(y32.double().cpu().numpy(), ref) < TOL32
    d = torch.empty_like(y)
    op.compute_diagonal(d)
    assert relerr(d.cpu().numpy(), O.mapped_diagonal(mm, oop)) < TOL64
    # create_rhs: as the structured path on the same mesh
    ops, _ = _supg_ops(gs, mask_s, coef)
    phi = R.uniform(-1, 1, om.n_dofs)
    rs = torch.zeros(om.n_dofs, dtype=torch.float64, device="cuda")
    ops.create_rhs(rs, dev(phi))
    phim = np.empty_like(phi)
    phim[perm] = phi
    rm = torch.zeros_like(rs)
    op.create_rhs(rm, dev(phim))
    assert relerr(rm.cpu().numpy()[perm], rs.cpu().numpy()) < TOL64
    assert op.device_error() == 0


@pytest.mark.parametrize("p", [1, 2])
def test_mapped_supg_with_hanging_constraints(cuda, p):
    """SUPG on a locally refined mesh (face and edge hanging nodes, perturbed
    vertices): vmult and the diagonal of the condensed operator against the
    oracle's mapped operator."""
    import torch
    from meltpooldg_b200.refine import refine_box
    V = O.box_vertices(3, (3, 3, 3), [-1.0] * 3, [1.0] * 3, 0.1, 17)
    r = refine_box((3, 3, 3), p, [13, 4], vertices=V)
    mm = O.MappedMesh(p, r["cell_vertices"], r["cell_dofs"], r["n_dofs"], r["constraints"])
    mask = r["boundary"]
    gm = device_mesh(mm, mask)
    op, oop = _supg_ops(gm, mask, -1.0)
    x = rng(70 + p).uniform(-1, 1, mm.n_dofs)
    ref = O.mapped_vmult(mm, oop, x)
    y = torch.empty(mm.n_dofs, dtype=torch.float64, device="cuda")
    op.vmult(y, dev(x))
    assert relerr(y.cpu().numpy(), ref) < TOL64
    d = torch.empty_like(y)
    op.compute_diagonal(d)
    assert relerr(d.cpu().numpy(), O.mapped_diagonal(mm, oop)) < TOL64


# local corners (x fastest) of face 2 d + s of a hexahedron
_FACE_CORNERS = {2 * d + s: [v for v in range(8) if ((v >> d) & 1) == s] for d in range(3) for s in range(2)}


def box_face_ids(cell_vertices, lo=(-1.0, -1.0, -1.0), hi=(1.0, 1.0, 1.0)):
    """Boundary id 2 d + s of every cell face that lies on the box face (d, s)."""
    cv = np.asarray(cell_vertices).reshape(-1, 8, 3)
    ids = -np.ones((cv.shape[0], 6), np.int8)
    for f, corners in _FACE_CORNERS.items():
        d, s = f // 2, f % 2
        plane = hi[d] if s else lo[d]
        on = np.all(np.abs(cv[:, corners, d] - plane) < 1e-12, axis=1)
        ids[on, f] = f
    return ids


def _face_ops(gm, T, mask):
    import meltpooldg_b200 as M
    kw = dict(robin_alpha=25.0, robin_t_inf=300.0, rad_emissivity=0.8, rad_t_inf=350.0)
    op = M.HeatDiffuseOperator(gm, 1e-2, rho_cp=2.0, k0=1.5, precisions=("fp64", "fp32"),
                               robin_faces=[(0, 1), (1, 0)], rad_faces=[(0, 1), (2, 1)], **kw)
    oop = O.Operator(O.HEAT, 1e-2, rho_cp=2.0, k0=1.5, temperature=T, dirichlet=mask,
                     robin_faces=(1 << 1) | (1 << 2), rad_faces=(1 << 1) | (1 << 5), **kw)
    return op, oop


@pytest.mark.parametrize("p", [1, 2, 3])
def test_mapped_boundary_faces(cuda, p):
    """Convective and radiative faces selected by the cells' boundary ids on a
    renumbered perturbed mesh: vmult (FP64, FP32) and the diagonal against the
    oracle's mapped operator, create_rhs as the structured device path's."""
    import torch
    import meltpooldg_b200 as M
    nc = (3, 2, 3)
    mask_s = M.boundary_mask(nc, p, faces=[(2, 0)])
    gs, om = meshes(nc, p, 0.1, seed=40 + p, mask=mask_s, lo=(-1, -1, -1), hi=(1, 1, 1))
    R = rng(90 + p)
    perm = R.permutation(om.n_dofs)
    mm = O.mapped_from_mesh(om, perm=perm, cell_order=R.permutation(om.n_cells))
    mask = np.empty_like(mask_s)
    mask[perm] = mask_s
    gm = M.MappedMesh(mm.cell_vertices, mm.cell_dofs, mm.n_dofs, p, dirichlet_mask=mask, face_ids=mm.face_ids)
    T = 300.0 + 50.0 * R.uniform(size=om.n_dofs)
    Tp = np.empty_like(T)
    Tp[perm] = T
    op, oop = _face_ops(gm, Tp, mask)
    Td = dev(Tp)
    op.set_temperature(Td)
    x = R.uniform(-1, 1, om.n_dofs)
    ref = O.mapped_vmult(mm, oop, x)
    y = torch.empty(om.n_dofs, dtype=torch.float64, device="cuda")
    op.vmult(y, dev(x))
    assert relerr(y.cpu().numpy(), ref) < TOL64
    y32 = torch.empty(om.n_dofs, dtype=torch.float32, device="cuda")
    op.vmult(y32, dev(x, torch.float32))
    assert relerr(y32.double().cpu().numpy(), ref) < TOL32
    d = torch.empty_like(y)
    op.compute_diagonal(d)
    assert relerr(d.cpu().numpy(), O.mapped_diagonal(mm, oop)) < TOL64
    # the Newton residual with its face terms: as the structured path's
    ops, _ = _face_ops(gs, T, mask_s)
    Ts = dev(T)
    ops.set_temperature(Ts)
    t_old = R.uniform(290.0, 310.0, om.n_dofs)
    rs = torch.zeros(om.n_dofs, dtype=torch.float64, device="cuda")
    ops.create_rhs(rs, dev(t_old))
    t_oldp = np.empty_like(t_old)
    t_oldp[perm] = t_old
    rm = torch.zeros_like(rs)
    op.create_rhs(rm, dev(t_oldp))
    assert relerr(rm.cpu().numpy()[perm], rs.cpu().numpy()) < TOL64


def test_mapped_boundary_faces_through_hanging_nodes(cuda):
    """Convective and radiative faces on a locally refined mesh whose refined
    cell touches the boundary (hanging DoFs on the selected faces): vmult and
    the diagonal (face matrices inside the constrained cells' element
    matrices) against the oracle's mapped operator."""
    import torch
    import meltpooldg_b200 as M
    from meltpooldg_b200.refine import refine_box
    p = 2
    V = O.box_vertices(3, (3, 3, 3), [-1.0] * 3, [1.0] * 3, 0.1, 1)
    r = refine_box((3, 3, 3), p, [4], vertices=V)  # cell 4 touches the face z = -1
    ids = box_face_ids(r["cell_vertices"])
    mm = O.MappedMesh(p, r["cell_vertices"], r["cell_dofs"], r["n_dofs"], r["constraints"], face_ids=ids)
    gm = M.MappedMesh(r["cell_vertices"], r["cell_dofs"], r["n_dofs"], p, constraints=r["constraints"],
                      face_ids=ids)
    N = mm.n_dofs
    T = 300.0 + 50.0 * rng(5).uniform(size=N)
    kw = dict(robin_alpha=25.0, robin_t_inf=300.0, rad_emissivity=0.8, rad_t_inf=350.0)
    op = M.HeatDiffuseOperator(gm, 1e-2, rho_cp=2.0, k0=1.5, precisions=("fp64", "fp32"),
                               robin_faces=[(2, 0), (0, 1)], rad_faces=[(2, 0), (1, 1)], **kw)
    oop = O.Operator(O.HEAT, 1e-2, rho_cp=2.0, k0=1.5, temperature=T, robin_faces=(1 << 4) | (1 << 1),
                     rad_faces=(1 << 4) | (1 << 3), **kw)
    Td = dev(T)
    op.set_temperature(Td)
    x = rng(6).uniform(-1, 1, N)
    ref = O.mapped_vmult(mm, oop, x)
    y = torch.empty(N, dtype=torch.float64, device="cuda")
    op.vmult(y, dev(x))
    assert relerr(y.cpu().numpy(), ref) < TOL64
    y32 = torch.empty(N, dtype=torch.float32, device="cuda")
    op.vmult(y32, dev(x, torch.float32))
    assert relerr(y32.double().cpu().numpy(), ref) < TOL32
    d = torch.empty_like(y)
    op.compute_diagonal(d)
    assert relerr(d.cpu().numpy(), O.mapped_diagonal(mm, oop)) < TOL64


@pytest.mark.parametrize("p", [1, 2])
@pytest.mark.parametrize("law", ["kT_full", "liquid_solid_latent"])
def test_mapped_hanging_constraints_with_field_coefficients(cuda, p, law):
    """k(T) with its full tangent, and the liquid/solid law with latent heat,
    on a locally refined mesh (hanging constraints, perturbed vertices): vmult
    (FP64, FP32) and the diagonal (element matrices with the fields at the
    Gauss points for the constrained cells) against the oracle's mapped operator."""
    import torch
    import meltpooldg_b200 as M
    from meltpooldg_b200.refine import refine_box
    V = O.box_vertices(3, (3, 3, 3), [-1.0] * 3, [1.0] * 3, 0.1, 23)
    r = refine_box((3, 3, 3), p, [13, 22], vertices=V)
    mm = O.MappedMesh(p, r["cell_vertices"], r["cell_dofs"], r["n_dofs"], r["constraints"])
    mask = r["boundary"]
    gm = device_mesh(mm, mask)
    N = mm.n_dofs
    R = rng(110 + p)
    T = 1970.0 + 4.0 * R.uniform(-1, 1, N)
    T_old = T + R.uniform(-0.5, 0.5, N)
    if law == "kT_full":
        op = M.HeatDiffuseOperator(gm, 1e-2, rho_cp=2.0, k0=1.5, k_alpha=1e-3, full_tangent=True,
                                   velocity=(0.3, -0.2, 0.1), precisions=("fp64", "fp32"))
        oop = O.Operator(O.HEAT, 1e-2, rho_cp=2.0, k0=1.5, k_alpha=1e-3, full_tangent=True, temperature=T,
                         dirichlet=mask, vel_kind=O.VEL_CONST, vel_param=(0.3, -0.2, 0.1))
    else:
        mat = dict(rho=(1.0, 7850.0, 7000.0), cp=(1.0, 460.0, 700.0), k=(1.0, 55.0, 17.0), solidus=1966.0,
                   liquidus=1974.0, latent_heat=2.7e5)
        op = M.HeatDiffuseOperator(gm, 1e-2, material=dict(mat, kind="liquid_solid"), precisions=("fp64", "fp32"))
        oop = O.Operator(O.HEAT, 1e-2, material=dict(mat, kind=O.MAT_LIQUID_SOLID), temperature=T,
                         temperature_old=T_old, dirichlet=mask)
    Td, Od = dev(T), dev(T_old)
    op.set_temperature(Td)
    if law != "kT_full":
        op.set_temperature_old(Od)
    x = R.uniform(-1, 1, N)
    ref = O.mapped_vmult(mm, oop, x)
    y = torch.empty(N, dtype=torch.float64, device="cuda")
    op.vmult(y, dev(x))
    assert relerr(y.cpu().numpy(), ref) < TOL64
    y32 = torch.empty(N, dtype=torch.float32, device="cuda")
    op.vmult(y32, dev(x, torch.float32))
    assert relerr(y32.double().cpu().numpy(), ref) < TOL32
    d = torch.empty_like(y)
    op.compute_diagonal(d)
    assert relerr(d.cpu().numpy(), O.mapped_diagonal(mm, oop)) < TOL64
