"""The allocation-free CG entry point (mpdg_solve_cg_noalloc) against the
regular solve entry point (mpdg_solve, CG + Jacobi), both called through the
C ABI, on two calls in a row.

Callers that cannot allocate device memory while they solve (a host whose
device memory belongs to its own pool, a time loop that must not synchronise
the device, an application that forbids allocations after start-up) use the
allocation-free entry point; it must give the regular solver's answer.  This
file is collected last so that a run stopping at the first failure has run
every other test already.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-10  # agreement of the two solutions (relative, max norm)


def _problem(perturb):
    import torch
    import meltpooldg_b200 as M
    nc, p = (16, 16, 16), 2
    mask = M.boundary_mask(nc, p)
    V = M.box_vertices(nc, perturb=perturb, seed=2)
    mesh = M.Mesh(V, nc, p, mask)
    rng = np.random.Generator(np.random.PCG64(11))
    op = M.HeatDiffuseOperator(mesh, 1e-3, rho_cp=1.0, k0=1.0, k_alpha=1e-3 if perturb else 0.0)
    if perturb:
        T = torch.tensor(rng.uniform(300.0, 3000.0, mesh.n_dofs), device="cuda")
        op.set_temperature(T)
        op._keep_T = T
    rhs = []
    for _ in range(2):
        xs = torch.tensor(rng.uniform(-1.0, 1.0, mesh.n_dofs), device="cuda")
        xs[torch.tensor(mask.astype(bool), device="cuda")] = 0.0
        b = torch.empty_like(xs)
        op.vmult(b, xs)  # also builds the operator's coefficient stream
        rhs.append(b)
    return mesh, op, rhs


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
    assert st == A.OK, A.lib().mpdg_last_error()
    return x, rep


@pytest.mark.parametrize("perturb", [0.0, 0.1])
def test_noalloc_cg_matches_regular_solve_twice(cuda, perturb):
    import torch
    mesh, op, rhs = _problem(perturb)
    ref = [_regular(op, b) for b in rhs]
    torch.cuda.synchronize()
    free_before = None
    for call, b in enumerate(rhs):
        if call == 1:
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info()[0]
        x, rep = _noalloc(op, b)
        if call == 1:
            torch.cuda.synchronize()
            # the second call allocated no device memory
            assert torch.cuda.mem_get_info()[0] == free_before
        xr, rr = ref[call]
        err = float((x - xr).abs().max() / xr.abs().max())
        assert err < REL_TOL, (call, err)
        assert rep.iterations == rr.iterations
        assert rep.final_residual <= 1e-10 * rep.initial_residual


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
