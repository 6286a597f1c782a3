"""The bounded wait of the warp apply (the mbarrier wait for the coefficient
block's bulk copy) reports expiry through the operator's device error word
(mpdg_op_device_error) and still returns the right result: the test hook
mpdg_debug_set_wait_polls(0) makes every first-phase wait expire at once, and
the retry with the full limit then waits for the copy.  No GPU fault or hang
is involved: every copy completes."""
import pytest

from gpu_helpers import dev, meshes, rng

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_expired_wait_sets_the_error_word_and_keeps_the_result(cuda, precision):
    import torch
    import meltpooldg_b200 as M
    from meltpooldg_b200 import _capi as A
    nc, p = (6, 5, 4), 4
    gm, _ = meshes(nc, p, 0.1, seed=2, mask=M.boundary_mask(nc, p))
    op = M.HeatDiffuseOperator(gm, 1e-3, rho_cp=1.0, k0=1.0, precisions=("fp64", "fp32"))
    dt = torch.float32 if precision == "fp32" else torch.float64
    src = dev(rng(1).uniform(-1, 1, gm.n_dofs), dt)
    ref = torch.empty_like(src)
    op.vmult(ref, src)
    assert op.device_error() == 0
    try:
        A.check(A.lib().mpdg_debug_set_wait_polls(0), "mpdg_debug_set_wait_polls")
        out = torch.empty_like(src)
        op.vmult(out, src)
        assert op.device_error() != 0
        assert torch.equal(out, ref)
    finally:
        A.check(A.lib().mpdg_debug_set_wait_polls(-1), "mpdg_debug_set_wait_polls")
    out = torch.empty_like(src)
    op.vmult(out, src)
    assert op.device_error() == 0
    assert torch.equal(out, ref)
