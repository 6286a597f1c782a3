"""The allocation-free CG entry point (mpdg_solve_cg_noalloc) against the
regular solve entry point (mpdg_solve, CG + Jacobi), both called through the
C ABI, on two calls in a row.

Callers that cannot allocate device memory while they solve (a host whose
device memory belongs to its own pool, a time loop that must not synchronise
the device, an application that forbids allocations after start-up) use the
allocation-free entry point; it must give the regular solver's answer and
make no allocation at all, which the library's own allocation counter
(mpdg_allocations) shows.  Operators whose diagonal needs probe vectors
(two-level meshes) and mapped meshes with constraints are refused with
MPDG_ERR_ARG, again without allocating.  This file is collected last so that
a run stopping at the first failure has run every other test already.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-10  # agreement of the two solutions (relative, max norm)


def _rhs(op, mesh_n, mask, seed, count=2):
    import torch
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(count):
        xs = torch.tensor(rng.uniform(-1.0, 1.0, mesh_n), device="cuda")
        if mask is not None:
            xs[torch.tensor(np.asarray(mask).astype(bool), device="cuda")] = 0.0
        b = torch.empty_like(xs)
        op.vmult(b, xs)  # also builds the operator's lazily made data
        out.append(b)
    return out


def _heat_lattice(perturb):
    import torch
    import meltpooldg_b200 as M
    nc, p = (16, 16, 16), 2
    mask = M.boundary_mask(nc, p)
    V = M.box_vertices(nc, perturb=perturb, seed=2)
    mesh = M.Mesh(V, nc, p, mask)
    op = M.HeatDiffuseOperator(mesh, 1e-3, rho_cp=1.0, k0=1.0, k_alpha=1e-3 if perturb else 0.0)
    if perturb:
        rng = np.random.Generator(np.random.PCG64(11))
        T = torch.tensor(rng.uniform(300.0, 3000.0, mesh.n_dofs), device="cuda")
        op.set_temperature(T)
        op._keep_T = T
    return mesh, op, _rhs(op, mesh.n_dofs, mask, 12)


def _advdiff_inflow_outflow():
    """Advection-diffusion (vortex velocity, mass-dominated at dt = 1e-3) with
    identity rows at the inflow/outflow DoFs of the vortex case."""
    import meltpooldg_b200 as M
    from oracle import cases
    from oracle import oracle as O
    nc, p = (12, 12, 12), 2
    V = M.box_vertices(nc, (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0))
    mesh = M.Mesh(V, nc, p)
    io = cases.vortex_io_mask(O.Mesh(3, p, nc, V), 4.0)
    op = M.AdvectionDiffusionOperator(mesh, 1e-3, theta=0.5, diffusivity=1e-3, velocity=("rotation", 4.0))
    op.set_inflow_outflow(io)
    return mesh, op, _rhs(op, mesh.n_dofs, io, 13)


def _mapped_unconstrained():
    """A perturbed lattice handed over as a mapped mesh (renumbered DoFs, no
    constraints), constant coefficients: the warp kernel through the map."""
    import meltpooldg_b200 as M
    from oracle import oracle as O
    nc, p = (10, 10, 10), 2
    V = M.box_vertices(nc, perturb=0.1, seed=5)
    om = O.Mesh(3, p, nc, V)
    perm = np.random.Generator(np.random.PCG64(3)).permutation(om.n_dofs)
    mm = O.mapped_from_mesh(om, perm=perm)
    mask = np.zeros(om.n_dofs, np.uint8)
    mask[perm] = M.boundary_mask(nc, p)
    mesh = M.MappedMesh(mm.cell_vertices, mm.cell_dofs, mm.n_dofs, mm.degree, dirichlet_mask=mask)
    op = M.HeatDiffuseOperator(mesh, 1e-3, rho_cp=1.0, k0=1.0)
    return mesh, op, _rhs(op, mesh.n_dofs, mask, 14)


def _regular(op, b):
    import torch
    from meltpooldg_b200 import _capi as A
    d = A.SolverDesc()
    A.lib().mpdg_solver_desc_default(C.byref(d))
    d.solver, d.preconditioner = A.SOLVER_CG, A.PREC_JACOBI
    d.rel_tolerance, d.abs_tolerance, d.max_iterations = 1e-10, 1e-20, 10000
    x = torch.zeros_like(b)
    rep = A.SolveReport()
    st = A.lib().mpdg_solve(op._h, C.byref(d), C.c_void_p(x.data_ptr()), C.c_void_p(b.data_ptr()),
                            C.byref(rep))
    assert st == A.OK, A.lib().mpdg_last_error()
    return x, rep


def _noalloc(op, b):
    import torch
    from meltpooldg_b200 import _capi as A
    x = torch.zeros_like(b)
    rep = A.SolveReport()
    st = A.lib().mpdg_solve_cg_noalloc(op._h, C.c_void_p(x.data_ptr()), C.c_void_p(b.data_ptr()),
                                       1e-10, 1e-20, 10000, C.byref(rep))
    return st, x, rep


@pytest.mark.parametrize("case", ["uniform", "perturbed", "inflow_outflow", "mapped"])
def test_noalloc_cg_matches_regular_solve_twice(cuda, case):
    import torch
    from meltpooldg_b200 import _capi as A
    mesh, op, rhs = {"uniform": lambda: _heat_lattice(0.0), "perturbed": lambda: _heat_lattice(0.1),
                     "inflow_outflow": _advdiff_inflow_outflow, "mapped": _mapped_unconstrained}[case]()
    ref = [_regular(op, b) for b in rhs]
    torch.cuda.synchronize()
    allocs_before = A.allocations()
    free_before = None
    for call, b in enumerate(rhs):
        if call == 1:
            # the first call may load the library's device code (lazy module
            # loading brings the static scratch array into device memory); the
            # second call must leave the free memory exactly as it was
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info()[0]
        st, x, rep = _noalloc(op, b)
        assert st == A.OK, A.lib().mpdg_last_error()
        xr, rr = ref[call]
        err = float((x - xr).abs().max() / xr.abs().max())
        assert err < REL_TOL, (call, err)
        assert rep.iterations == rr.iterations
        assert rep.final_residual <= 1e-10 * rep.initial_residual
    torch.cuda.synchronize()
    # neither call allocated (the library's own count), nor did the second
    # change the device's free memory
    assert A.allocations() == allocs_before
    assert torch.cuda.mem_get_info()[0] == free_before


def test_noalloc_refuses_two_level_meshes_without_allocating(cuda):
    import torch
    import meltpooldg_b200 as M
    from meltpooldg_b200 import _capi as A
    from oracle import oracle as O
    p, nc = 2, (2, 2, 2)
    om = O.Mesh2(p, nc, 3)
    mask = om.boundary_face_mask()
    gm = M.TwoLevelMesh(om.coarse.vert, nc, om.fine.vert, (3, 4, 4), p, mask[:om.n_coarse], mask[om.n_coarse:])
    op = M.HeatDiffuseOperator(gm, 1e-2, rho_cp=2.0, k0=1.5)
    b = _rhs(op, gm.n_dofs, mask, 15, count=1)[0]
    torch.cuda.synchronize()
    allocs_before = A.allocations()
    st, _, _ = _noalloc(op, b)
    assert st == A.ERR_ARG
    assert b"two-level" in A.lib().mpdg_last_error()
    assert A.allocations() == allocs_before


def test_noalloc_refuses_constrained_mapped_meshes_without_allocating(cuda):
    import torch
    import meltpooldg_b200 as M
    from meltpooldg_b200 import _capi as A
    from meltpooldg_b200.refine import refine_box
    p = 2
    r = refine_box((3, 3, 3), p, [13])
    gm = M.MappedMesh(r["cell_vertices"], r["cell_dofs"], r["n_dofs"], p, dirichlet_mask=r["boundary"],
                      constraints=r["constraints"])
    op = M.HeatDiffuseOperator(gm, 1e-2, rho_cp=2.0, k0=1.5)
    b = _rhs(op, gm.n_dofs, r["boundary"], 16, count=1)[0]
    torch.cuda.synchronize()
    allocs_before = A.allocations()
    st, _, _ = _noalloc(op, b)
    assert st == A.ERR_ARG
    assert b"constraints" in A.lib().mpdg_last_error()
    assert A.allocations() == allocs_before


def test_noalloc_rejects_oversized_problems(cuda):
    import torch
    import meltpooldg_b200 as M
    from meltpooldg_b200 import _capi as A
    nc = (66, 66, 66)  # 67^3 = 300,763 DoFs > 262,144
    mesh = M.Mesh(M.box_vertices(nc), nc, 1)
    op = M.HeatDiffuseOperator(mesh, 1e-3)
    b = torch.ones(mesh.n_dofs, dtype=torch.float64, device="cuda")
    x = torch.zeros_like(b)
    rep = A.SolveReport()
    st = A.lib().mpdg_solve_cg_noalloc(op._h, C.c_void_p(x.data_ptr()), C.c_void_p(b.data_ptr()),
                                       1e-10, 1e-20, 100, C.byref(rep))
    assert st == A.ERR_SIZE
    assert b"262144" in A.lib().mpdg_last_error()
