"""SUPG stabilisation of the advection-diffusion operator on the device
(MODE_SUPG of the block cell kernel, per-cell tau_K, probing diagonal) against
the oracle: vmult, create_rhs and the diagonal (FP64 to 1e-12, FP32 to 2e-5),
on uniform, graded (axis-aligned) and perturbed cells, all with diffusion (the
perturbed ones through the map-curvature term of the Laplacian), and the
reference's golden case advection_diffusion_vortex_mf_supg."""
import json
import os

import numpy as np
import pytest

from gpu_helpers import dev, meshes, relerr, rng
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-5

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_outputs.json")))

VELOCITIES = [("vortex", O.VEL_VORTEX, (0.0, 0.0, 0.0)),
              (("rotation", 4.0), O.VEL_ROTATION, (4.0, 0.0, 0.0)),
              ((0.7, -0.3, 1.1), O.VEL_CONST, (0.7, -0.3, 1.1))]


def graded_vertices(nc, seed):
    """Axis-aligned lattice with random spacings: every cell an axis-aligned box
    of its own size (the general-geometry path with the Laplacian term)."""
    R = rng(seed)
    ax = [np.concatenate([[0.0], np.cumsum(R.uniform(0.5, 1.5, nc[d]))]) for d in range(3)]
    ax = [a / a[-1] * 2.0 - 1.0 for a in ax]
    Z, Y, X = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)


def _case(kind, nc, p, seed, mask):
    import meltpooldg_b200 as M
    if kind == "uniform":
        return meshes(nc, p, 0.0, seed=seed, mask=mask, lo=(-1, -1, -1), hi=(1, 1, 1)) + (0.05,)
    if kind == "perturbed":
        return meshes(nc, p, 0.15, seed=seed, mask=mask, lo=(-1, -1, -1), hi=(1, 1, 1)) + (0.05,)
    V = graded_vertices(nc, seed)
    return M.Mesh(V, nc, p, mask, geometry="general"), O.Mesh(3, p, nc, V), 0.05


@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("kind", ["uniform", "perturbed", "graded"])
@pytest.mark.parametrize("coef", [-1.0, 0.7])
def test_supg_vmult_parity(cuda, p, kind, coef):
    import torch
    import meltpooldg_b200 as M
    nc = (4, 3, 5)
    mask = M.boundary_mask(nc, p, faces=[(0, 0), (2, 1)])
    gm, om, D = _case(kind, nc, p, 7 + p, mask)
    src = rng(30 + p).uniform(-1, 1, gm.n_dofs)
    for vel, okind, oparam in VELOCITIES:
        op = M.AdvectionDiffusionOperator(gm, 1e-2, theta=0.5, diffusivity=D, velocity=vel,
                                          precisions=("fp64", "fp32"), supg=True, supg_coefficient=coef)
        oop = O.Operator(O.ADVDIFF, 1e-2, theta=0.5, diffusivity=D, vel_kind=okind, vel_param=oparam,
                         dirichlet=mask, supg=True, supg_coefficient=coef)
        ref = O.vmult(om, oop, src)
        dst = torch.empty(gm.n_dofs, dtype=torch.float64, device="cuda")
        op.vmult(dst, dev(src))
        assert relerr(dst.cpu().numpy(), ref) < TOL64, vel
        d32 = torch.empty(gm.n_dofs, dtype=torch.float32, device="cuda")
        op.vmult(d32, dev(src, torch.float32))
        assert relerr(d32.double().cpu().numpy(), ref) < TOL32, vel


@pytest.mark.parametrize("p", [1, 2, 4])
@pytest.mark.parametrize("kind", ["uniform", "perturbed", "graded"])
def test_supg_rhs_and_diagonal(cuda, p, kind):
    import torch
    import meltpooldg_b200 as M
    nc = (3, 4, 3)
    mask = M.boundary_mask(nc, p, faces=[(1, 0)])
    gm, om, D = _case(kind, nc, p, 40 + p, mask)
    phi = rng(50 + p).uniform(-1, 1, gm.n_dofs)
    op = M.AdvectionDiffusionOperator(gm, 1e-2, theta=0.5, diffusivity=D, velocity="vortex", supg=True)
    oop = O.Operator(O.ADVDIFF, 1e-2, theta=0.5, diffusivity=D, vel_kind=O.VEL_VORTEX, dirichlet=mask,
                     supg=True)
    base = rng(60 + p).uniform(-1, 1, gm.n_dofs)
    rhs = dev(base.copy())
    op.create_rhs(rhs, dev(phi))
    # the right-hand side is scattered without the constrained rows (integrate_scatter
    # through the Dirichlet constraints, advection_diffusion_operator.cpp:350)
    ref = O.rhs_advdiff(om, oop, phi, scatter_mask=mask, dst=base.copy())
    assert relerr(rhs.cpu().numpy(), ref) < TOL64
    d = torch.empty(gm.n_dofs, dtype=torch.float64, device="cuda")
    op.compute_diagonal(d)
    assert relerr(d.cpu().numpy(), O.diagonal(om, oop)) < TOL64


def test_supg_coefficient_zero_equals_plain_operator(cuda):
    import torch
    import meltpooldg_b200 as M
    nc = (4, 4, 3)
    gm, _ = meshes(nc, 2, 0.1, seed=3, lo=(-1, -1, -1), hi=(1, 1, 1))
    src = dev(rng(3).uniform(-1, 1, gm.n_dofs))
    a = torch.empty_like(src)
    b = torch.empty_like(src)
    M.AdvectionDiffusionOperator(gm, 1e-2, velocity="vortex", supg=True, supg_coefficient=0.0).vmult(a, src)
    M.AdvectionDiffusionOperator(gm, 1e-2, velocity="vortex").vmult(b, src)
    assert relerr(a.cpu().numpy(), b.cpu().numpy()) < 1e-14


def test_supg_rejections(cuda):
    import meltpooldg_b200 as M
    nc = (3, 3, 3)
    gm, _ = meshes(nc, 2, 0.1, seed=5)
    d = M._capi.OpDesc(M._capi.OP_HEAT, 1e-2, 1.0, 1.0, 0.0, 0, 0.5, 0.0, 0,
                       (M._capi.C.c_double * 3)(0, 0, 0), 0)
    d.supg = 1
    with pytest.raises(Exception, match="advection-diffusion"):
        M.operators._MatrixFreeOperator(gm, d, ("fp64",))


def test_vortex_supg_golden_on_gpu(cuda):
    """advection_diffusion_vortex_mf_supg (2D, Q1, 32^2 on [-1,1]^2, SUPG with
    tau_K = h_K / max |u|, CN, GMRES + Diagonal) extruded to one layer of
    hexahedra of thickness h = 1/16 in y: the 2D plane is (x, z), where the
    device's rotation velocity s (z, 0, -x) is the 2D s (y, -x); the cell size
    diameter / sqrt(3) of an h-cube equals the 2D diameter / sqrt(2) of an
    h-square, the field stays y-independent, and the 3D L2 norm is sqrt(h)
    times the 2D one."""
    import meltpooldg_b200 as M
    from meltpooldg_b200.operations import AdvectionDiffusionOperation
    from oracle import cases
    om2, phi2, mask2 = cases.vortex_setup(2, 5)
    h = 2.0 / 32
    nc = (32, 1, 32)
    V = M.box_vertices(nc, (-1.0, 0.0, -1.0), (1.0, h, 1.0))

    def extrude(a):  # 2D lattice (Y2, X) -> 3D (Z = Y2, Y in {0, 1}, X)
        a = np.asarray(a).reshape(33, 33)
        return np.stack([a, a], axis=1).ravel()

    mask = extrude(mask2).astype(np.uint8)
    mesh = M.Mesh(V, nc, 1, mask)
    opn = AdvectionDiffusionOperation(mesh, 0.01, theta=0.5, diffusivity=0.0, velocity=("rotation", 4.0),
                                      dirichlet_values=np.full(mesh.n_dofs, -1.0), supg=True)
    opn.set_initial_condition(extrude(phi2))
    for r in GOLDEN["advection_diffusion_vortex_mf_supg"]["values"]:
        opn.solve()
        got = opn.l2_norm() / np.sqrt(h)
        assert abs(got - r) / r < 5e-8, (got, r)
