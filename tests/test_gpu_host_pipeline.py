"""The host-buffer apply (mpdg_vmult_host) runs its copy-in, apply and
copy-out over z-slabs of cell layers on three streams.  Against the oracle
(1e-12) and the device-resident apply (the slab order only changes the order
of the additions on the slab boundary planes): general and uniform geometry,
degrees 1-4, layer counts from 2 to 17 (odd and even), k(T), velocity and
Dirichlet rows; operators with boundary faces take the one-stream path."""
import numpy as np
import pytest

from gpu_helpers import dev, meshes, relerr, rng
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("nz", [2, 3, 5, 8, 17])
@pytest.mark.parametrize("perturb", [0.0, 0.1])
def test_host_apply_slabs(cuda, p, nz, perturb):
    import torch
    import meltpooldg_b200 as M
    nc = (3, 4, nz)
    mask = M.boundary_mask(nc, p, faces=[(0, 0), (2, 1)])
    gm, om = meshes(nc, p, perturb, seed=nz + p, mask=mask)
    T = rng(7).uniform(300, 3000, gm.n_dofs)
    src = rng(8 + p).uniform(-1, 1, gm.n_dofs)
    if perturb > 0.0:
        op = M.HeatDiffuseOperator(gm, 1e-3, k0=1.0, k_alpha=1e-3, velocity=(0.3, -0.2, 0.5))
        op.set_temperature(dev(T))
        oop = O.Operator(O.HEAT, 1e-3, k0=1.0, k_alpha=1e-3, temperature=T, dirichlet=mask,
                         vel_kind=O.VEL_CONST, vel_param=(0.3, -0.2, 0.5))
    else:
        op = M.HeatDiffuseOperator(gm, 1e-3, rho_cp=2.0, k0=1.5, velocity=(0.3, -0.2, 0.5))
        oop = O.Operator(O.HEAT, 1e-3, rho_cp=2.0, k0=1.5, dirichlet=mask,
                         vel_kind=O.VEL_CONST, vel_param=(0.3, -0.2, 0.5))
    ref = O.vmult(om, oop, src)
    host = np.full(gm.n_dofs, np.nan)
    op.vmult_host(host, src)
    assert relerr(host, ref) < 1e-12
    d = torch.empty(gm.n_dofs, dtype=torch.float64, device="cuda")
    op.vmult(d, dev(src))
    assert relerr(host, d.cpu().numpy()) < 1e-14
    # repeated calls reuse the staging, streams and events
    host2 = np.full(gm.n_dofs, np.nan)
    op.vmult_host(host2, src)
    assert np.array_equal(host, host2)


def test_host_apply_with_faces_takes_one_stream(cuda):
    import meltpooldg_b200 as M
    nc, p = (3, 3, 6), 2
    gm, om = meshes(nc, p, 0.1, seed=3)
    src = rng(9).uniform(-1, 1, gm.n_dofs)
    op = M.HeatDiffuseOperator(gm, 1e-3, robin_alpha=25.0, robin_t_inf=300.0, robin_faces=[(2, 1)])
    oop = O.Operator(O.HEAT, 1e-3, robin_alpha=25.0, robin_t_inf=300.0, robin_faces=1 << 5)
    host = np.empty(gm.n_dofs)
    op.vmult_host(host, src)
    assert relerr(host, O.vmult(om, oop, src)) < 1e-12
