"""Every schedule of the resident apply (z-slabs, L2 evict-first hint on the
coefficient stream, colour launches overlapping as programmatic dependents,
cell groups shared by a whole CTA) returns the same bits as the plain
one-launch-per-colour, warp-per-group apply, for every degree, uniform and
perturbed cells, the heat and the advection-diffusion operator, Dirichlet
rows, FP64 and FP32, on a mesh whose colours end in partial cell groups; and
FP64 matches the oracle to 1e-12."""
import pytest

from gpu_helpers import dev, meshes, relerr, rng
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SCHEDULES = [dict(slabs=1, l2_evict_first=False, overlap_colours=True, cta_cell_groups=False, lane_cells=0),
             dict(slabs=1, l2_evict_first=False, overlap_colours=True, cta_cell_groups=True, lane_cells=0),
             dict(slabs=1, l2_evict_first=True, overlap_colours=False, cta_cell_groups=True, lane_cells=0),
             dict(slabs=2, l2_evict_first=True, overlap_colours=True, cta_cell_groups=True, lane_cells=0)]


@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("perturb", [0.0, 0.1])
@pytest.mark.parametrize("kind", ["heat", "advdiff"])
def test_schedules_bit_identical(cuda, p, perturb, kind):
    import torch
    import meltpooldg_b200 as M
    nc = (7, 6, 9)
    mask = M.boundary_mask(nc, p)
    gm, om = meshes(nc, p, perturb, seed=3, mask=mask)
    if kind == "heat":
        op = M.HeatDiffuseOperator(gm, 1e-3, rho_cp=2.0, k0=1.5, precisions=("fp64", "fp32"))
        oop = O.Operator(O.HEAT, 1e-3, rho_cp=2.0, k0=1.5, dirichlet=mask)
    else:
        op = M.AdvectionDiffusionOperator(gm, 1e-3, theta=0.5, diffusivity=1e-2, velocity="vortex",
                                          precisions=("fp64", "fp32"))
        oop = O.Operator(O.ADVDIFF, 1e-3, theta=0.5, diffusivity=1e-2, vel_kind=O.VEL_VORTEX, dirichlet=mask)
    src = rng(40 + p).uniform(-1, 1, gm.n_dofs)
    ref64 = O.vmult(om, oop, src)
    for prec, dtype in (("fp64", torch.float64), ("fp32", torch.float32)):
        s = dev(src, dtype)
        op.set_schedule(1, False, prec, overlap_colours=False, cta_cell_groups=False)
        base = torch.empty_like(s)
        op.vmult(base, s)
        if prec == "fp64":
            assert relerr(base.cpu().numpy(), ref64) < 1e-12
        for sc in SCHEDULES:
            op.set_schedule(sc["slabs"], sc["l2_evict_first"], prec, overlap_colours=sc["overlap_colours"],
                            cta_cell_groups=sc["cta_cell_groups"])
            assert op.schedule(prec) == sc
            out = torch.empty_like(s)
            op.vmult(out, s)
            assert torch.equal(out, base), (prec, sc)
    assert op.device_error() == 0
