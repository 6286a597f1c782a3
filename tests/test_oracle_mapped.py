"""CPU checks of the oracle's mapped-mesh operator (the ingestion form of an
unstructured mesh: per-cell corners, cell->DoF map, affine constraints):
it reproduces the structured oracle on the same mesh, is invariant under
renumbering the DoFs and reordering the cells, and with the hanging-node
constraints of a two-level mesh reproduces the two-level oracle."""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.mark.parametrize("p", [1, 2, 3])
def test_mapped_equals_structured_and_is_permutation_invariant(p):
    m = O.Mesh.box(3, p, [3, 2, 4], perturb=0.1, seed=1)
    mask = m.boundary_face_mask([(0, 0), (2, 1)])
    op = O.Operator(O.ADVDIFF, 1e-2, theta=0.5, diffusivity=0.1, vel_kind=O.VEL_VORTEX, dirichlet=mask)
    x = np.random.default_rng(p).uniform(-1, 1, m.n_dofs)
    a = O.vmult(m, op, x)
    assert np.abs(O.mapped_vmult(O.mapped_from_mesh(m), op, x) - a).max() <= 1e-14 * np.abs(a).max()
    assert np.abs(O.mapped_diagonal(O.mapped_from_mesh(m), op) - O.diagonal(m, op)).max() <= 1e-14 * np.abs(
        O.diagonal(m, op)).max()
    R = np.random.default_rng(10 + p)
    perm = R.permutation(m.n_dofs)
    mp = O.mapped_from_mesh(m, perm=perm, cell_order=R.permutation(m.n_cells))
    opp = op.with_dirichlet(mask[np.argsort(perm)])
    xp = np.empty_like(x)
    xp[perm] = x
    assert np.abs(O.mapped_vmult(mp, opp, xp)[perm] - a).max() <= 1e-14 * np.abs(a).max()


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("kind", [O.HEAT, O.ADVDIFF])
def test_mapped_hanging_constraints_equal_two_level(p, kind):
    m2 = O.Mesh2(p, (2, 2, 2), 2, perturb=0.1, seed=3)
    mask = m2.boundary_face_mask()
    if kind == O.HEAT:
        op = O.Operator(O.HEAT, 1e-2, rho_cp=2.0, k0=1.5, dirichlet=mask)
    else:
        op = O.Operator(O.ADVDIFF, 1e-2, theta=0.5, diffusivity=0.05, vel_kind=O.VEL_VORTEX, dirichlet=mask)
    mm = O.mapped_from_mesh2(m2)
    assert set(mm.constraints) == set(np.flatnonzero(m2.hanging_mask()))
    x = np.random.default_rng(p).uniform(-1, 1, m2.n_dofs)
    a = O.vmult2(m2, op, x)
    assert np.abs(O.mapped_vmult(mm, op, x) - a).max() <= 1e-14 * np.abs(a).max()
    d = O.diagonal2(m2, op)
    assert np.abs(O.mapped_diagonal(mm, op) - d).max() <= 1e-13 * np.abs(d).max()


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("coef", [-1.0, 0.7])
def test_mapped_supg_equals_structured(p, coef):
    """SUPG with diffusion (the Laplacian with the map's curvature) through the
    mapped path, with tau_K from the mapped cell's corners and Gauss points,
    equals the structured oracle on the same perturbed mesh, renumbered."""
    m = O.Mesh.box(3, p, [3, 2, 3], perturb=0.15, seed=4)
    mask = m.boundary_face_mask([(1, 0)])
    op = O.Operator(O.ADVDIFF, 1e-2, theta=0.5, diffusivity=0.05, vel_kind=O.VEL_VORTEX, dirichlet=mask,
                    supg=True, supg_coefficient=coef)
    x = np.random.default_rng(p).uniform(-1, 1, m.n_dofs)
    a = O.vmult(m, op, x)
    R = np.random.default_rng(20 + p)
    perm = R.permutation(m.n_dofs)
    mp = O.mapped_from_mesh(m, perm=perm, cell_order=R.permutation(m.n_cells))
    opp = op.with_dirichlet(mask[np.argsort(perm)])
    xp = np.empty_like(x)
    xp[perm] = x
    assert np.abs(O.mapped_vmult(mp, opp, xp)[perm] - a).max() <= 1e-13 * np.abs(a).max()
    d = O.diagonal(m, op)
    assert np.abs(O.mapped_diagonal(mp, opp)[perm] - d).max() <= 1e-13 * np.abs(d).max()


def test_mapped_nodal_velocity_equals_structured():
    """A velocity DoF vector read through the cell->DoF map of a renumbered mesh
    (component stride = the mapped mesh's DoF count)."""
    m = O.Mesh.box(3, 2, [3, 2, 2], perturb=0.1, seed=6)
    R = np.random.default_rng(7)
    U = R.uniform(-1, 1, (3, m.n_dofs))
    op = O.Operator(O.HEAT, 1e-2, rho_cp=2.0, k0=1.5, vel_kind=O.VEL_NODAL, vel_nodal=U.reshape(-1))
    x = R.uniform(-1, 1, m.n_dofs)
    a = O.vmult(m, op, x)
    perm = R.permutation(m.n_dofs)
    mp = O.mapped_from_mesh(m, perm=perm)
    Up = np.empty_like(U)
    Up[:, perm] = U
    opp = O.Operator(O.HEAT, 1e-2, rho_cp=2.0, k0=1.5, vel_kind=O.VEL_NODAL, vel_nodal=Up.reshape(-1))
    xp = np.empty_like(x)
    xp[perm] = x
    assert np.abs(O.mapped_vmult(mp, opp, xp)[perm] - a).max() <= 1e-13 * np.abs(a).max()


@pytest.mark.parametrize("p", [1, 2, 3])
def test_mapped_boundary_faces_equal_structured(p):
    """Convective and radiative faces selected by the cells' boundary ids equal
    the structured oracle's box faces on the same mesh, renumbered (apply and
    the diagonal)."""
    m = O.Mesh.box(3, p, [2, 3, 2], perturb=0.1, seed=8)
    T = 300.0 + 50.0 * np.random.default_rng(1).uniform(size=m.n_dofs)
    op = O.Operator(O.HEAT, 1e-2, rho_cp=2.0, k0=1.5, temperature=T, robin_alpha=25.0, robin_t_inf=300.0,
                    robin_faces=(1 << 1) | (1 << 2), rad_emissivity=0.8, rad_t_inf=350.0,
                    rad_faces=(1 << 1) | (1 << 5))
    x = np.random.default_rng(p).uniform(-1, 1, m.n_dofs)
    a = O.vmult(m, op, x)
    R = np.random.default_rng(30 + p)
    perm = R.permutation(m.n_dofs)
    mp = O.mapped_from_mesh(m, perm=perm, cell_order=R.permutation(m.n_cells))
    Tp = np.empty_like(T)
    Tp[perm] = T
    opp = op.with_temperature(Tp)
    xp = np.empty_like(x)
    xp[perm] = x
    assert np.abs(O.mapped_vmult(mp, opp, xp)[perm] - a).max() <= 1e-13 * np.abs(a).max()
    d = O.diagonal(m, op)
    assert np.abs(O.mapped_diagonal(mp, opp)[perm] - d).max() <= 1e-13 * np.abs(d).max()


@pytest.mark.parametrize("p", [1, 2])
@pytest.mark.parametrize("law", ["kT_full", "liquid_solid"])
def test_mapped_hanging_constraints_with_field_coefficients(p, law):
    """k(T) with its full tangent, and the liquid/solid law with latent heat,
    through the hanging-node constraints of a mapped mesh: the operator is
    C^T A C with A the same cells without constraints (the fields read plain),
    and its diagonal is (C e_g)^T A (C e_g)."""
    m2 = O.Mesh2(p, (2, 2, 2), 2, perturb=0.1, seed=5)
    x2 = m2.dof_coordinates()
    R = np.random.default_rng(9 + p)
    N = m2.n_dofs
    T = 1970.0 + 4.0 * np.sin(3.0 * x2[:, 0]) * np.cos(2.0 * x2[:, 1]) + R.uniform(-0.3, 0.3, N)
    T_old = T + R.uniform(-0.5, 0.5, N)
    if law == "kT_full":
        op = O.Operator(O.HEAT, 1e-2, rho_cp=2.0, k0=1.5, k_alpha=1e-3, full_tangent=True, temperature=T,
                        vel_kind=O.VEL_CONST, vel_param=(0.3, -0.2, 0.1))
    else:
        mat = dict(kind=O.MAT_LIQUID_SOLID, rho=(1.0, 7850.0, 7000.0), cp=(1.0, 460.0, 700.0),
                   k=(1.0, 55.0, 17.0), solidus=1966.0, liquidus=1974.0, latent_heat=2.7e5)
        op = O.Operator(O.HEAT, 1e-2, material=mat, temperature=T, temperature_old=T_old)
    mm = O.mapped_from_mesh2(m2)
    free = O.MappedMesh(p, mm.cell_vertices, mm.cell_dofs, N)
    cons = mm.constraints

    def C(x):  # constrained entries from their masters
        y = x.copy()
        for c, ent in cons.items():
            y[c] = sum(w * x[mst] for mst, w in ent)
        return y

    def Ct(y):  # transpose: constrained rows to their masters, then 0
        z = y.copy()
        for c, ent in cons.items():
            for mst, w in ent:
                z[mst] += w * y[c]
            z[c] = 0.0
        return z

    x = R.uniform(-1, 1, N)
    want = Ct(O.mapped_vmult(free, op, C(x)))
    got = O.mapped_vmult(mm, op, x)
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    d = O.mapped_diagonal(mm, op)
    masters = sorted({mst for ent in cons.values() for mst, _ in ent})
    for g in masters[:: max(1, len(masters) // 8)] + [0, N // 2]:
        if g in cons:
            continue
        e = np.zeros(N)
        e[g] = 1.0
        ce = C(e)
        assert abs(ce @ O.mapped_vmult(free, op, ce) - d[g]) <= 1e-12 * abs(d[g])


def test_mapped_faces_through_hanging_nodes_are_CtAC():
    """Convective and radiative faces through hanging DoFs of a locally refined
    mesh: the operator is C^T A C with A the same cells and faces without
    constraints, and its diagonal (C e_g)^T A (C e_g)."""
    from meltpooldg_b200.refine import refine_box
    p = 2
    V = O.box_vertices(3, (3, 3, 3), [-1.0] * 3, [1.0] * 3, 0.1, 1)
    r = refine_box((3, 3, 3), p, [4], vertices=V)
    cv = np.asarray(r["cell_vertices"]).reshape(-1, 8, 3)
    ids = -np.ones((cv.shape[0], 6), np.int8)
    for d in range(3):
        for s in range(2):
            corners = [v for v in range(8) if ((v >> d) & 1) == s]
            on = np.all(np.abs(cv[:, corners, d] - (1.0 if s else -1.0)) < 1e-12, axis=1)
            ids[on, 2 * d + s] = 2 * d + s
    N = r["n_dofs"]
    mm = O.MappedMesh(p, r["cell_vertices"], r["cell_dofs"], N, r["constraints"], face_ids=ids)
    free = O.MappedMesh(p, r["cell_vertices"], r["cell_dofs"], N, face_ids=ids)
    cons = mm.constraints
    assert (ids[:, 4] >= 0).any()
    T = 300.0 + 50.0 * np.random.default_rng(2).uniform(size=N)
    op = O.Operator(O.HEAT, 1e-2, rho_cp=2.0, k0=1.5, temperature=T, robin_alpha=25.0, robin_t_inf=300.0,
                    robin_faces=1 << 4, rad_emissivity=0.8, rad_t_inf=350.0, rad_faces=1 << 4)

    def C(x):
        y = x.copy()
        for c, ent in cons.items():
            y[c] = sum(w * x[mst] for mst, w in ent)
        return y

    def Ct(y):
        z = y.copy()
        for c, ent in cons.items():
            for mst, w in ent:
                z[mst] += w * y[c]
            z[c] = 0.0
        return z

    x = np.random.default_rng(3).uniform(-1, 1, N)
    want = Ct(O.mapped_vmult(free, op, C(x)))
    assert np.abs(O.mapped_vmult(mm, op, x) - want).max() <= 1e-12 * np.abs(want).max()
    d = O.mapped_diagonal(mm, op)
    masters = sorted({mst for ent in cons.values() for mst, _ in ent})
    for g in masters[:: max(1, len(masters) // 10)]:
        e = np.zeros(N)
        e[g] = 1.0
        ce = C(e)
        assert abs(ce @ O.mapped_vmult(free, op, ce) - d[g]) <= 1e-12 * abs(d[g])
