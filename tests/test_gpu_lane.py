"""The lane apply (one thread per cell, x-segments of 32 cells that add their
shared faces by warp shuffles, colours by segment parity): degrees 1 and 2 on
uniform lattices, the heat and advection-diffusion operators with every
in-kernel velocity, Dirichlet rows, FP64 against the oracle at 1e-12 and FP32
at 2e-5, on rows of one, two and three segments (the last one partial, or
one cell long), with and without overlapping colour launches, in z-slabs and
through the host-buffer pipeline.  Its results agree with the warp apply to
rounding."""
import numpy as np
import pytest

from gpu_helpers import dev, meshes, relerr, rng
from oracle import oracle as O

pytestmark = pytest.mark.gpu

VELOCITIES = {
    "none": (None, dict()),
    "const": ((0.7, -0.4, 0.25), dict(vel_kind=O.VEL_CONST, vel_param=(0.7, -0.4, 0.25))),
    "vortex": ("vortex", dict(vel_kind=O.VEL_VORTEX)),
    "rotation": (("rotation", 0.8), dict(vel_kind=O.VEL_ROTATION, vel_param=(0.8, 0.0, 0.0))),
}


def _ops(kind, vel, gm, mask):
    import meltpooldg_b200 as M
    v, ov = VELOCITIES[vel]
    if kind == "heat":
        op = M.HeatDiffuseOperator(gm, 1e-3, rho_cp=2.0, k0=1.5, velocity=v, precisions=("fp64", "fp32"))
        oop = O.Operator(O.HEAT, 1e-3, rho_cp=2.0, k0=1.5, dirichlet=mask, **ov)
    else:
        op = M.AdvectionDiffusionOperator(gm, 1e-3, theta=0.5, diffusivity=1e-2, velocity=v,
                                          precisions=("fp64", "fp32"))
        oop = O.Operator(O.ADVDIFF, 1e-3, theta=0.5, diffusivity=1e-2, dirichlet=mask, **ov)
    return op, oop


@pytest.mark.parametrize("p", [1, 2])
@pytest.mark.parametrize("nc", [(7, 6, 9), (70, 3, 4), (33, 4, 5)])
@pytest.mark.parametrize("kind,vel", [("heat", "none"), ("heat", "const"), ("advdiff", "vortex"),
                                      ("advdiff", "rotation"), ("advdiff", "const")])
@pytest.mark.parametrize("dirichlet", [True, False])
def test_lane_apply_parity(cuda, p, nc, kind, vel, dirichlet):
    import torch
    import meltpooldg_b200 as M
    mask = M.boundary_mask(nc, p) if dirichlet else None
    gm, om = meshes(nc, p, 0.0, seed=3, mask=mask, hi=(1.0, 0.8, 1.3))
    op, oop = _ops(kind, vel, gm, mask)
    src = rng(70 + p).uniform(-1, 1, gm.n_dofs)
    ref = O.vmult(om, oop, src)
    for prec, dtype, tol in (("fp64", torch.float64, 1e-12), ("fp32", torch.float32, 2e-5)):
        s = dev(src, dtype)
        op.set_schedule(1, False, prec, overlap_colours=True, lane_cells=0)
        warp = torch.empty_like(s)
        op.vmult(warp, s)
        for lane in (1, 2):
            for overlap in (False, True):
                op.set_schedule(1, False, prec, overlap_colours=overlap, lane_cells=lane)
                assert op.schedule(prec)["lane_cells"] == lane
                out = torch.full_like(s, float("nan"))
                op.vmult(out, s)
                got = out.cpu().numpy().astype(np.float64)
                assert relerr(got, ref) < tol, (prec, lane, overlap)
                if prec == "fp64":
                    assert relerr(got, warp.cpu().numpy()) < 1e-13
    assert op.device_error() == 0


@pytest.mark.parametrize("p", [1, 2])
def test_lane_apply_slabs_and_host_pipeline(cuda, p):
    import torch
    import meltpooldg_b200 as M
    nc = (40, 5, 12)
    mask = M.boundary_mask(nc, p)
    gm, om = meshes(nc, p, 0.0, seed=5, mask=mask)
    op, oop = _ops("advdiff", "vortex", gm, mask)
    src = rng(90 + p).uniform(-1, 1, gm.n_dofs)
    ref = O.vmult(om, oop, src)
    s = dev(src)
    for slabs in (1, 2, 3):
        op.set_schedule(slabs, False, "fp64", overlap_colours=True, lane_cells=1)
        out = torch.full_like(s, float("nan"))
        op.vmult(out, s)
        assert relerr(out.cpu().numpy(), ref) < 1e-12, slabs
    # the host-buffer pipeline runs the apply over ranges of cell layers
    op.set_schedule(1, False, "fp64", overlap_colours=True, lane_cells=2)
    h = np.empty(gm.n_dofs)
    op.vmult_host(h, np.ascontiguousarray(src))
    assert relerr(h, ref) < 1e-12
    assert op.device_error() == 0


def test_lane_apply_declines_what_it_does_not_serve(cuda):
    """Perturbed cells, degree 3, the nodal velocity: lane_cells is accepted and
    the warp apply runs (results unchanged to the bit)."""
    import torch
    import meltpooldg_b200 as M
    for p, perturb in ((3, 0.0), (2, 0.1)):
        nc = (6, 5, 4)
        gm, om = meshes(nc, p, perturb, seed=7)
        op = M.HeatDiffuseOperator(gm, 1e-3, rho_cp=1.0, k0=1.0)
        src = dev(rng(3).uniform(-1, 1, gm.n_dofs))
        a, b = torch.empty_like(src), torch.empty_like(src)
        op.set_schedule(1, False, "fp64", overlap_colours=True, lane_cells=0)
        op.vmult(a, src)
        op.set_schedule(1, False, "fp64", overlap_colours=True, lane_cells=1)
        op.vmult(b, src)
        assert torch.equal(a, b)


def test_lane_autotune_candidates(cuda):
    """The autotuner times the lane apply on a Q2 uniform lattice and keeps a
    schedule whose result matches the oracle."""
    import torch
    import meltpooldg_b200 as M
    nc = (20, 12, 10)
    mask = M.boundary_mask(nc, 2)
    gm, om = meshes(nc, 2, 0.0, seed=1, mask=mask)
    op, oop = _ops("advdiff", "vortex", gm, mask)
    best, ms, cand = op.autotune("fp64", reps=2)
    assert ms > 0 and len(cand) >= 6
    src = rng(11).uniform(-1, 1, gm.n_dofs)
    out = torch.empty(gm.n_dofs, dtype=torch.float64, device="cuda")
    op.vmult(out, dev(src))
    assert relerr(out.cpu().numpy(), O.vmult(om, oop, src)) < 1e-12
